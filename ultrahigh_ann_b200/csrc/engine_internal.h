// Query pipeline pieces shared by the engine's host translation units
// (engine.cu: single calls; batch.cu: captured multi-index batches, the
// autotuner and the request loop).
#pragma once

#include "common.h"
#include "index_types.h"
#include "kernels.h"
#include "stage_bodies.h"

namespace uha_engine {

bool precision_strategy(uha_strategy s);
bool fp32_rescore_strategy(uha_strategy s);
bool small_path_applies(const uha_index* index, uha_strategy strategy);
uha::LowpType lowp_type(uha_strategy s);

// The index's low-precision rows of `type` (built on first use) and the
// workspace buffers of the precision strategies.
const uha::LowpRows& lowp_rows(const uha_index* index, uha::LowpType type,
                               cudaStream_t stream);
void ensure_lowp_workspace(uha_workspace* ws, const uha_index* index,
                           cudaStream_t stream);

struct BatchContext {
    const uha_index* index;
    uha_workspace* ws;
    uha_strategy strategy;
    bool want_distances;
    // Pipelined calls (exact and flat indexes): this batch's prepared queries
    // and partial sums (direct / gemm) or candidate buffers (precision),
    // sized by the caller, and the stream its argmin / re-score runs on after
    // `handoff` is recorded behind the scan. Null: the workspace's own buffers
    // and stream.
    float* prepared = nullptr;
    float* partials = nullptr;
    uint32_t* candidates = nullptr;   // precision: this batch's candidate slot
    double* cand_dist = nullptr;
    uint32_t* rescore_done = nullptr;
    cudaStream_t finish_stream = nullptr;
    cudaEvent_t handoff = nullptr;
    // The precision strategies may take the fused candidate selection: the
    // caller answers the call again without it when a candidate list
    // overflows (error bit uha::kCandidateOverflow).
    bool filter_candidates = false;
    // The fused flat query of this batch runs on stream lane `flat_lane`
    // (0: ws->stream; others: ws->flat_streams, forked and joined by the
    // caller) with that lane's scratch slots.
    int flat_lane = 0;
};

// Allocates and clears (on ws->stream) the fused flat query's scratch of
// every stream lane, if it does not exist yet.
void ensure_flat_scratch(const uha_index* index, uha_workspace* ws);

// Enqueues one batch of n queries (`source`: device, n x dimension floats) on
// ws->stream; returns the number of kernel launches. Buffers grow (with a
// stream synchronisation) only when n needs more than an earlier call did.
uint64_t enqueue_batch(const BatchContext& c, const float* source, uint64_t n,
                       uha::Result* results, double* exact, bool time_scan,
                       cudaEvent_t scan_start, cudaEvent_t scan_stop);

// The persistent batch's description of one pair (a hierarchical index and n
// queries in ws->raw_queries, certified direct strategy), read from the
// index and from workspace buffers that a standalone run of n queries has
// sized; false when the pair has no persistent form (projection dimension
// above 256, the streaming scan of batches up to 8, oversized shared memory).
// Median bound of the L1 hierarchy: the binary32 |diff| and midpoint
// roundings (the binary64 ones are within them): 6 * 2^-24 relative, 2^-126
// absolute.
constexpr float kMedianRel = 0x1.8p-22f;
constexpr float kMedianAbs = 0x1p-126f;

// The median passes' shape for batches of n on this workspace: the tuned
// one, else the default.
uha::MedianPlan median_plan(const uha_index* index, const uha_workspace* ws, uint64_t n);
bool persistent_pair(const uha_index* index, uha_workspace* ws, uint64_t n,
                     uha::PersistentPair* d);

// Answers of a call whose queries need no device work (row 0, distance 0).
void fill_trivial(uint64_t n, uint64_t* out_indices, double* out_distances);

// Reads the status words copied to ws->host_counters and converts the host
// copies of results / exact distances into the caller's arrays.
void finish_call(const uha_index* index, uha_workspace* ws, uint64_t n,
                 const uha::Result* results, const double* exact,
                 uint64_t* out_indices, double* out_distances);

void validate_query_call(const uha_index* index, uha_workspace* ws,
                         const float* queries, uint64_t count, uint64_t batch,
                         uha_strategy strategy, const uint64_t* out_indices);

}  // namespace uha_engine
