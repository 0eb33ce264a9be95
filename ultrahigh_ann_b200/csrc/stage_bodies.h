// The persistent multi-index batch kernels (certify.cu, launch_persistent_batch)
// and the shapes of the stage kernels they stand in for.
//
// Three kernels answer many (hierarchical index, query batch) pairs, one
// cooperative launch each. A kernel's work is a device queue of units drawn
// from all pairs (a unit is one block of the stage kernel that the standalone
// path would launch for that pair, run by the same device code from
// tile_body.cuh, hier_body.cuh and certify.cu, so both paths compute the same
// values), ordered stage by stage. Every CTA takes the next unit from the
// queue head (one atomic), waits until the unit's pair has completed all its
// units of earlier stages (a per-pair completion count), runs it and counts it
// complete. There is no grid-wide barrier: a pair's later stages run while
// other pairs are still in earlier ones, and a heavy unit delays only the
// units that depend on it. The stages:
//   0 clear per-pair counters and accumulators   4 median counts (L1)
//   1 gather of the sampled coordinates          5 median survivors (L1), argmin (L2)
//   2 binary32 projection with its error bound   6 argmin (L1), reported distances (L2)
//   3 L2 tile scan + error root, median samples  7 reported distances (L1)
// Stages 0-2 run in a first kernel (8 CTAs per SM), stage 3 in a second (the
// tile scan's register budget, 2 CTAs per SM), stages 4-7 in a third (4 CTAs
// per SM).
//
// Progress: units leave the queue in order, and a unit waits only on units of
// its own pair earlier in the queue, all of them already taken by CTAs that
// are resident (cooperative launch); the earliest unfinished unit never
// waits. A wait still gives up after about two seconds: it sets the batch
// status and ends its CTA (the others stop taking units, and the later
// kernels return at once), so a fault can never hold the GPU.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "kernels.h"

namespace uha {

// ---- shapes of the stage kernels (the persistent kernel's units)
uint64_t project_queries_smem_bytes();
void project_queries_grid(uint64_t batch, uint64_t padded_p, uint32_t* gx, uint32_t* gy);
// median scan of the L1 hierarchy (launch_median_scan's stages)
struct MedianArgs {
    const float* rows;
    const float* rows_t;
    uint32_t r_pitch;
    uint32_t row_count;
    uint32_t padded_p;
    uint32_t p;
    const float* queries;
    uint32_t batch;
    const float* query_err;
    const float* coord_err;
    float row_err_max;
    float rel;
    float abs_err;
    unsigned int* min_bits;  // 0xffffffff before the sample stage
    float* partials;
    float* pair_err;
    uint32_t samples;        // MedianPlan::samples
    uint32_t count_queries;  // MedianPlan::count_queries
};
uint32_t median_sample_blocks(uint32_t samples, uint32_t batch);
// the default queries per count CTA for a batch
int median_count_queries(uint32_t batch);
void median_count_grid(uint32_t row_count, uint32_t batch, uint32_t count_queries,
                       uint32_t* gx, uint32_t* gy);
uint32_t median_survivor_blocks(uint32_t row_count, uint32_t batch);
// the binary32 L2 tile scan
uint64_t tile_scan_smem_bytes();
void tile_scan_grid(uint64_t row_count, uint64_t batch, uint32_t splits, uint32_t* gx,
                    uint32_t* gy, uint32_t* gz);
// the certified argmin and the reported distances
void argmin_grid(uint32_t rows, uint32_t batch, uint32_t* gx, uint32_t* span);
void argmin_scratch(void* scratch, uint64_t capacity, uint32_t rows, void** summaries,
                    uint32_t** done);
uint64_t replay_smem_bytes(const ReplayInputs& in);
uint64_t refine_group_smem_bytes(const ReplayInputs& in);
uint32_t refine_group_blocks(uint32_t batch);

// ---- the persistent batch
constexpr int kPersistentStages = 8;
// The kernels of a run: stages [0, kPersistentSplit0) (clear, gather,
// projection: latency-bound, run at 8 CTAs per SM), [kPersistentSplit0,
// kPersistentSplit) (tile scans and median samples, at the tile scan's
// register budget, 2 CTAs per SM) and [kPersistentSplit, kPersistentStages)
// (4 CTAs per SM).
constexpr int kPersistentKernels = 3;
constexpr int kPersistentSplit0 = 3;
constexpr int kPersistentSplit = 4;
constexpr int persistent_part_of(int stage)
{
    return stage < kPersistentSplit0 ? 0 : stage < kPersistentSplit ? 1 : 2;
}

// Everything one pair's stages read and write (device pointers into the
// pair's workspace and index).
struct PersistentPair {
    int l2;                    // 1: L2 hierarchy (JL, tile scan); 0: L1 (median)
    uint32_t batch;
    // stage 0
    uint32_t* counters;        // [0] replayed queries, [1] error flags
    uint32_t counter_words;
    // stage 1: gather
    const float* raw_queries;  // batch x dim
    uint64_t dim;
    const uint32_t* columns;
    uint64_t sample_size;
    float* prepared;           // batch x padded_sample
    uint64_t padded_sample;
    // stage 2: projection
    const float* projection32;
    uint64_t proj_dim;
    float* projected;          // batch x padded_p
    uint64_t padded_p;
    float* query_err;
    float* coord_err;          // L1
    double err_per_abs;
    uint32_t proj_gx, proj_gy;
    // stage 3: L2 tile scan
    const float* scan_rows;
    uint32_t rows;
    float* partials;
    uint32_t k_per_split;
    uint32_t tile_gx, tile_gy, tile_gz;
    // stages 3-5: L1 median scan
    MedianArgs median;
    uint32_t sample_blocks;
    uint32_t count_gx, count_gy;
    uint32_t survivor_blocks;
    // stages 5-6: certified argmin
    PartialView view;
    Bound bound;
    ReplayInputs replay;
    Result* results;
    double* exact_distances;
    void* summaries;
    uint32_t* done;
    uint32_t argmin_gx;
    uint32_t argmin_span;
    // stages 6-7: reported distances
    uint32_t refine_blocks;
};

// One stage's work from one pair: `units` units of one kind, numbered from
// `first` within the stage.
struct PersistentSegment {
    uint32_t pair;
    uint32_t kind;
    uint32_t units;
    uint32_t first;
};

constexpr uint32_t kPersistentMaxPairs = 32;
constexpr uint32_t kPersistentMaxSegments = 2 * kPersistentMaxPairs * kPersistentStages + 1;

// Words of the work queue's device state (zero at creation; the last CTA of
// the last kernel zeroes them again at the end of a run):
constexpr uint32_t kQueueHead = 0;  // [0, kPersistentKernels): units taken, per kernel
constexpr uint32_t kQueueFinished = kPersistentKernels;  // CTAs of the last kernel done
constexpr uint32_t kQueueStageDone = kQueueFinished + 1;  // units completed, per stage
constexpr uint32_t kQueuePairDone = kQueueStageDone + kPersistentStages;  // per pair
constexpr uint32_t kPersistentQueueWords = kQueuePairDone + kPersistentMaxPairs;

struct PersistentPlan {
    uint32_t stage_begin[kPersistentStages + 1];  // segment ranges per stage
    uint32_t stage_units[kPersistentStages];
    // queue position of each stage's first unit (the units of all earlier
    // stages, both kernels counted)
    uint32_t stage_first[kPersistentStages + 1];
    // a pair's units in stages before each stage: a unit of stage s starts
    // once its pair has completed pair_wait[pair][s] units
    uint32_t pair_wait[kPersistentMaxPairs][kPersistentStages];
    unsigned int* queue;  // device, kPersistentQueueWords words
    int* status;          // device: nonzero when a wait ran out
    // device, kPersistentStages + 1 entries (%globaltimer, ns): [s] for the
    // first stage of a kernel its start as CTA 0 sees it, [s + 1] when the
    // last unit of stage s completed (untouched for a stage without units)
    unsigned long long* clock;
    uint32_t smem_bytes[kPersistentKernels];  // dynamic shared memory per kernel
};

// The kernels' one parameter (about 26 KB, read from the constant bank like
// any kernel argument: the units address the pairs' fields in place instead
// of copying them into registers): the plan, the pairs and the segments,
// grouped by stage.
struct PersistentParams {
    PersistentPlan plan;
    PersistentPair pairs[kPersistentMaxPairs];
    PersistentSegment segments[kPersistentMaxSegments];
};

// Builds the segment list of `pairs` (host copies) into `segments` (room for
// persistent_segment_capacity(count)), the stage ranges and units of `plan`
// and the dynamic shared memory the kernel needs.
void plan_persistent_batch(const PersistentPair* pairs, uint32_t count,
                           PersistentSegment* segments, uint32_t* segment_count,
                           PersistentPlan* plan);
uint32_t persistent_segment_capacity(uint32_t count);
// CTAs of one cooperative launch of kernel `part` (< kPersistentKernels) on
// the current device for `smem_bytes` of dynamic shared memory (all resident
// at once); 0 if it cannot be launched.
uint32_t persistent_grid(int part, uint32_t smem_bytes);
// The run's cooperative launches, one per kernel (capturable in a graph).
void launch_persistent_batch(const PersistentParams& params,
                             const uint32_t grid[kPersistentKernels], cudaStream_t stream);

}  // namespace uha
