// Internal definitions of the opaque C-ABI handles (uha_index,
// uha_workspace) shared by the engine's translation units.
#pragma once

#include "common.h"
#include "kernels.h"

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

namespace uha {

enum class IndexKind { exact, weighted, sampled, hierarchical };

constexpr uint64_t kColumnAlign = 4;  // padded row length: 16-byte multiple
constexpr uint64_t kMaxExtent = 0x7fffffffull;

// Low-precision copy of an index's scanned rows for the precision
// strategies: lowp_padded_count(rows) vectors of `pitch` elements (zero past
// the scanned columns and past the last row), per-row scales (FP8) and the
// squared norms of the rounded rows.
struct LowpRows {
    DeviceBuffer<unsigned char> data;
    DeviceBuffer<float> scales;
    DeviceBuffer<float> norms;
    uint64_t pitch = 0;
    bool ready = false;
};

// Relative and absolute certification bound for a binary32 distance (defined
// in engine.cu).
Bound make_bound(uint32_t depth, uint64_t terms, int term_roundings);
// The same for a parallel binary64 sum of the CPU's terms.
Bound64 make_bound64(uint32_t depth, uint64_t terms);

}  // namespace uha

struct uha_index {
    int device = 0;
    std::string device_name;
    int sm_count = 148;
    uha::IndexKind kind = uha::IndexKind::exact;
    uha_metric metric = UHA_L2;
    uint64_t rows = 0;
    uint64_t dimension = 0;   // original query dimension d
    uint64_t scan_dim = 0;    // columns scanned (d or k)
    uint64_t padded_dim = 0;  // scan_dim rounded up to kColumnAlign
    uint64_t sample_size = 0;
    uint64_t sampled_multiplicity = 0;
    uha::DeviceBuffer<float> scan_rows;   // rows x padded_dim
    uha::DeviceBuffer<float> row_norms;   // rows (L2, norm-identity strategy)
    uha::DeviceBuffer<float> weights32;   // padded_dim (weighted L1 scan)
    uha::DeviceBuffer<double> weights64;  // scan_dim (weighted L1 replay)
    uha::DeviceBuffer<float> weights_ff;  // 2 x scan_dim: weights64 as hi, lo
    uha::DeviceBuffer<uint32_t> columns;  // sample_size (sampled)
    uha::DeviceBuffer<float> scales;      // sample_size (sampled L2)
    // hierarchical: scan_dim = p; scan_rows = binary32 projected rows
    uint64_t projection_dimension = 0;
    uint64_t padded_sample = 0;             // sample_size rounded up
    uha::DeviceBuffer<double> rows64;       // rows x p (binary64 projected)
    uha::DeviceBuffer<double> projection64; // p x sample_size
    uha::DeviceBuffer<float> projection32;  // p x padded_sample
    uha::DeviceBuffer<float> row_err;       // rows
    float row_err_max = 0.f;                // largest row_err
    // L1 hierarchy: scan_rows transposed, padded_dim x rows_pitch
    uha::DeviceBuffer<float> scan_rows_t;
    uint64_t rows_pitch = 0;
    // L2 hierarchy: projection64 transposed, sample_size x p
    uha::DeviceBuffer<double> projection64_t;
    uha_space_usage usage{};
    // precision strategies: built on first use (index_bf16 / index_fp8)
    mutable std::mutex lowp_mutex;
    mutable uha::LowpRows lowp[2];
    mutable uha::LowpRows lowp_projection[2];  // L2 hierarchy: the p x k projection
};

// A scan shape chosen by the autotuner for one (batch size, strategy) of a
// workspace, with the device time it measured.
struct TunedPlan {
    uint64_t batch = 0;
    int strategy = 0;
    bool lowp = false;
    bool median = false;  // median_plan holds the L1 hierarchy's median passes
    uha::ScanPlan scan{};
    uha::LowpPlan lowp_plan{};
    uha::MedianPlan median_plan{};
    double ms = 0.0;
    int candidates = 0;
};

struct uha_workspace {
    const uha_index* owner = nullptr;
    int device = 0;  // the owner's device, kept so destruction never reads the owner
    uint64_t max_batch = 0;
    uint64_t payload_bytes = 0;
    cudaStream_t stream = nullptr;
    uha::DeviceBuffer<float> raw_queries;
    uha::DeviceBuffer<float> prepared;
    uha::DeviceBuffer<float> projected;   // hierarchical: batch x padded p
    uha::DeviceBuffer<float> query_err;   // hierarchical: batch
    uha::DeviceBuffer<float> query_norms;
    uha::DeviceBuffer<float> partials;
    uha::DeviceBuffer<uha::Result> call_results;  // one call's answers
    uha::DeviceBuffer<double> call_exact;         // replayed distances (NaN: none)
    uha::DeviceBuffer<uint32_t> counters;  // [0] replayed queries, [1] error flag
    uha::DeviceBuffer<unsigned char> finalize_scratch;
    // fused flat query (allocated and zeroed on first use): two scratch slots
    // per stream lane (uha::kFlatLanes lanes; lane 0 is `stream`), the slot
    // parity each lane's next launch uses, the lanes' other streams and the
    // fork / join events of a call that spreads its batches over them
    uha::DeviceBuffer<unsigned char> flat_scratch;
    uint32_t flat_parity[uha::kFlatLanes] = {};
    cudaStream_t flat_streams[uha::kFlatLanes] = {};
    cudaEvent_t flat_events[uha::kFlatLanes] = {};
    // precision strategies (allocated on first use)
    uha::DeviceBuffer<unsigned char> queries_lp;  // lowp_padded_count(max_batch) vectors
    uha::DeviceBuffer<float> query_scales;        // FP8 scale per query
    uha::DeviceBuffer<unsigned int> query_amax;   // FP8 max |x| bits per query
    // fused candidate selection (allocated on first use): per-query key
    // lists, their counts and thresholds, the sample's candidates
    uha::DeviceBuffer<unsigned long long> filter_keys;
    uha::DeviceBuffer<uint32_t> filter_count;
    uha::DeviceBuffer<float> filter_tau;
    uha::DeviceBuffer<uint32_t> filter_sample;
    uha::DeviceBuffer<float> filter_norms;  // the sample rows' norms
    bool filter_disabled = false;  // answering again after an overflow
    uha::DeviceBuffer<uint32_t> candidates;       // [batch][candidates_per_query]
    uha::DeviceBuffer<double> cand_dist;          // [batch][candidates_per_query]
    uha::DeviceBuffer<uint32_t> rescore_done;     // per query, zero between calls
    uha::DeviceBuffer<unsigned int> median_min;   // L1 hierarchy: sampled minimum per query
    uha::DeviceBuffer<float> coord_err;   // L1 hierarchy: batch x padded p query errors
    uha::DeviceBuffer<float> pair_err;    // L1 hierarchy: batch x rows median errors
    // precision form of the L2 hierarchy: rounded gathered queries, their
    // scales, and the reference's binary64 projection of each query
    uha::DeviceBuffer<unsigned char> gathered_lp;
    uha::DeviceBuffer<float> gathered_scales;
    uha::DeviceBuffer<unsigned int> gathered_amax;
    uha::DeviceBuffer<double> projected64;
    uint32_t candidates_per_query = 32;
    bool emulated_replay = false;  // uha_workspace_set_replay
    std::vector<TunedPlan> tuned;  // autotuned shapes (uha_workspace_autotune)

    const TunedPlan* find_tuned(uint64_t batch, int strategy) const
    {
        for (const TunedPlan& t : tuned) {
            if (t.batch == batch && t.strategy == strategy) {
                return &t;
            }
        }
        return nullptr;
    }
    uha::PinnedBuffer<uha::Result> host_results;
    uha::PinnedBuffer<double> host_exact;
    uha::PinnedBuffer<uint32_t> host_counters;
    uha_query_stats last{};
    bool timing = false;
    uint32_t timing_stride = 1;  // scan events on every timing_stride-th batch
    cudaEvent_t events[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> scan_events;  // start/stop of each batch's scan
    // pipelined small batches: a second stream for the argmins, two slots of
    // prepared queries and partial sums, hand-off / slot-free / join events
    cudaStream_t finish_stream = nullptr;
    cudaEvent_t pipe_events[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    uha::DeviceBuffer<float> pipe_prepared;
    uha::DeviceBuffer<float> pipe_partials;
    uha::DeviceBuffer<uint32_t> pipe_candidates;   // precision pipeline slots
    uha::DeviceBuffer<double> pipe_cand_dist;
    uha::DeviceBuffer<uint32_t> pipe_rescore_done;

    ~uha_workspace()
    {
        for (cudaEvent_t e : events) {
            if (e != nullptr) {
                cudaEventDestroy(e);
            }
        }
        for (cudaEvent_t e : scan_events) {
            cudaEventDestroy(e);
        }
        for (cudaEvent_t e : pipe_events) {
            if (e != nullptr) {
                cudaEventDestroy(e);
            }
        }
        for (int i = 0; i < uha::kFlatLanes; ++i) {
            if (flat_events[i] != nullptr) {
                cudaEventDestroy(flat_events[i]);
            }
            if (i > 0 && flat_streams[i] != nullptr) {
                cudaStreamDestroy(flat_streams[i]);
            }
        }
        if (finish_stream != nullptr) {
            cudaStreamDestroy(finish_stream);
        }
        if (stream != nullptr) {
            cudaStreamDestroy(stream);
        }
    }
};

