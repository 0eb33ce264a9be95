// uha_query_noalloc: the certified query path for small batches of
// device-resident queries that allocates no memory at all.
//
// Who needs it: callers that cannot call cudaMalloc while they answer queries
// — a serving process whose device memory is fully reserved up front by its
// own pool allocator (a cudaMalloc would fail or fragment the reservation),
// code running where allocation is not allowed or would be unsafe to
// interleave (for example while other threads of the process capture CUDA
// graphs), and embedded callers that must keep their device footprint fixed
// after start-up. uha_query needs a workspace, which owns device buffers that
// uha_workspace_create allocates; this entry point needs none.
//
// The scratch every step of the pipeline writes (the prepared queries, the
// per-chunk partial distances, the certified-argmin merge state, the results
// and replayed distances before conversion, and the status counters) lives in one file-scope
// __device__ array of kNoAllocScratchBytes. Every GPU that loads the library
// holds that array until the process exits. Host code never uses the array's
// name as an address: on each device, the first call looks the address up
// with cudaGetSymbolAddress (with that device current) and keeps it.
#include "common.h"
#include "index_types.h"
#include "kernels.h"

#include <cmath>
#include <mutex>

namespace {

// 32 MiB: enough for an exact scan of r = 7,028 rows in d = 60,660
// coordinates at up to 8 queries per call, or much larger sampled indexes.
constexpr uint64_t kNoAllocScratchBytes = 32ull << 20;
constexpr uint64_t kNoAllocMaxBatch = 8;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_address[uha::kMaxDevices] = {};

// Device address of the static scratch on the current device; looked up once
// per device.
void* scratch_address(int device)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_address[device] == nullptr) {
        void* ptr = nullptr;
        uha::check_cuda(cudaGetSymbolAddress(&ptr, g_noalloc_scratch),
                        "cannot resolve the static query scratch");
        g_scratch_address[device] = ptr;
    }
    return g_scratch_address[device];
}

// Bump carving of the scratch array (256-byte aligned pieces).
struct Carver {
    unsigned char* base;
    uint64_t used = 0;
    template <typename T>
    T* take(uint64_t count)
    {
        T* p = reinterpret_cast<T*>(base + used);
        used += (count * sizeof(T) + 255) / 256 * 256;
        return p;
    }
};

// Writes the caller's outputs: the row of every query and its distance (the
// binary64 replayed distance where the replay ran, else the certified
// binary32 distance).
__global__ void write_outputs_kernel(const uha::Result* results,
                                     const double* replayed, uint32_t n,
                                     uint64_t* out_indices,
                                     double* out_distances)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) {
        return;
    }
    out_indices[q] = results[q].row;
    if (out_distances != nullptr) {
        const double r = replayed[q];
        out_distances[q] = isnan(r) ? static_cast<double>(results[q].distance) : r;
    }
}

}  // namespace

extern "C" uha_status uha_query_noalloc(const uha_index* index,
                                        const float* queries,
                                        uint64_t query_count,
                                        uint64_t* out_indices,
                                        double* out_distances, void* stream)
{
    return uha::guarded([&] {
        using uha::fail;
        if (index == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "index must not be null");
        }
        if (index->kind == uha::IndexKind::hierarchical) {
            fail(UHA_INVALID_ARGUMENT,
                 "uha_query_noalloc serves exact and flat indexes only");
        }
        if (query_count == 0) {
            return;
        }
        if (query_count > kNoAllocMaxBatch) {
            fail(UHA_LENGTH_ERROR,
                 "uha_query_noalloc answers at most 8 queries per call");
        }
        if (out_indices == nullptr ||
            (queries == nullptr && index->dimension != 0)) {
            fail(UHA_INVALID_ARGUMENT,
                 "query and output device pointers must not be null");
        }
        uha::DeviceGuard guard(index->device);
        uha::clear_stale_cuda_error();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const uint64_t n = query_count;

        if (index->padded_dim == 0) {
            // No sampled coordinates: every query selects row 0 at distance 0.
            uha::check_cuda(cudaMemsetAsync(out_indices, 0, n * sizeof(uint64_t), s),
                            "cannot write query results");
            if (out_distances != nullptr) {
                uha::check_cuda(
                    cudaMemsetAsync(out_distances, 0, n * sizeof(double), s),
                    "cannot write query distances");
            }
            uha::check_cuda(cudaStreamSynchronize(s), "query failed");
            return;
        }

        const uha::ScanPlan plan = uha::plan_scan(index->rows, index->padded_dim,
                                                  n, index->sm_count);
        Carver c{static_cast<unsigned char*>(scratch_address(index->device))};
        uint32_t* counters = c.take<uint32_t>(4);  // [0] replay count, [1] error flag
        uha::Result* results = c.take<uha::Result>(n);
        double* replayed = c.take<double>(n);
        float* prepared = c.take<float>(n * index->padded_dim);
        float* partials = c.take<float>(uint64_t(plan.chunks) * n * index->rows);
        unsigned char* finalize =
            c.take<unsigned char>(uha::finalize_scratch_bytes(n, index->rows));
        if (c.used > kNoAllocScratchBytes) {
            fail(UHA_LENGTH_ERROR,
                 "index and batch need more than the 32 MiB static query "
                 "scratch of uha_query_noalloc; use uha_query with a workspace");
        }

        // The scratch keeps the previous call's contents: clear the counters
        // and the merge state that must start at zero.
        uha::check_cuda(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s),
                        "cannot clear query counters");
        uha::check_cuda(cudaMemsetAsync(finalize, 0,
                                        uha::finalize_scratch_bytes(n, index->rows), s),
                        "cannot clear merge state");

        int* error_flag = reinterpret_cast<int*>(counters + 1);
        if (index->kind == uha::IndexKind::sampled) {
            uha::launch_prepare_sampled(
                queries, n, index->dimension, index->columns.get(),
                index->metric == UHA_L2 ? index->scales.get() : nullptr,
                index->sample_size, prepared, index->padded_dim, error_flag, s);
        } else {
            uha::launch_prepare_dense(queries, n, index->dimension, prepared,
                                      index->padded_dim, error_flag, s);
        }
        uha::ScanOp op = uha::ScanOp::l2;
        if (index->metric == UHA_L1) {
            op = index->weights32.size() != 0 ? uha::ScanOp::l1_weighted
                                              : uha::ScanOp::l1;
        }
        uha::launch_scan(plan, op, index->scan_rows.get(), index->rows,
                         index->padded_dim, index->weights32.get(), prepared, n,
                         partials, s);
        const uha::PartialView view{partials, plan.chunks, static_cast<uint32_t>(n),
                                    static_cast<uint32_t>(index->rows)};
        const uha::Bound bound = uha::make_bound(
            plan.depth, index->scan_dim, op == uha::ScanOp::l1 ? 1 : 2);
        uha::ReplayInputs in{};
        in.rows = index->scan_rows.get();
        in.queries = prepared;
        in.dim = index->scan_dim;
        in.padded_dim = index->padded_dim;
        in.weights64 = index->weights64.get();
        in.op = index->metric == UHA_L2 ? uha::ReplayOp::l2_sequential
                : index->weights64.size() != 0
                    ? uha::ReplayOp::l1_weighted_sequential
                    : uha::ReplayOp::l1_grouped4;
        uha::launch_argmin(view, bound, in, results, replayed, finalize, n, counters,
                           s);
        write_outputs_kernel<<<1, 32, 0, s>>>(results, replayed,
                                              static_cast<uint32_t>(n), out_indices,
                                              out_distances);
        uha::check_cuda(cudaGetLastError(), "cannot launch output kernel");
        uint32_t host_counters[2] = {0, 0};
        uha::check_cuda(cudaMemcpyAsync(host_counters, counters, sizeof(host_counters),
                                        cudaMemcpyDeviceToHost, s),
                        "cannot read query counters");
        uha::check_cuda(cudaStreamSynchronize(s), "query failed");
        if (host_counters[1] != 0) {
            fail(UHA_INVALID_ARGUMENT,
                 index->kind == uha::IndexKind::sampled
                     ? "sampled query coordinate must be finite"
                     : "queries must be finite");
        }
    });
}
