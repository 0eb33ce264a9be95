// Batches over many indexes and the scan-shape autotuner (no reference
// counterpart: the reference answers one index per call, and its benchmark
// loops over query_batch per chunk, src/benchmarks/
// nearest_neighbor_benchmark.cpp:386-413).
//
// uha_workspace_autotune times every candidate scan shape of one (index,
// batch size, strategy) on the device with CUDA events and keeps the fastest
// on the workspace; every later query of that batch size uses it. The
// certification bound follows the chosen shape (its accumulation depth), so
// the answers stay the reference CPU's.
//
// uha_batch captures the whole pipeline of many (index, query count) pairs
// into one CUDA graph: each pair's preparation, projection, scan, argmin /
// re-score and result copies run on their own branch, forked from and joined
// into one stream, so small indexes overlap on the device and the host issues
// one launch per run. uha_batch_create_persistent captures instead the
// cooperative launches of the persistent batch kernels (stage_bodies.h:
// gather and projection, tile scans and median samples, the late stages),
// each draining a device work queue of every pair's units, plus the result
// copies.
#include "common.h"
#include "engine_internal.h"
#include "index_types.h"
#include "kernels.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

using namespace uha_engine;
using uha::check_cuda;
using uha::checked_mul;
using uha::DeviceGuard;
using uha::fail;
using uha::guarded;
using uha::IndexKind;

namespace {

void require(bool condition, uha_status status, const char* message)
{
    if (!condition) {
        fail(status, message);
    }
}

uha::ScanOp scan_op(const uha_index* index, uha_strategy strategy)
{
    if (strategy == UHA_GEMM && index->metric == UHA_L2) {
        return uha::ScanOp::dot;
    }
    if (index->metric == UHA_L1) {
        return index->weights32.size() != 0 ? uha::ScanOp::l1_weighted : uha::ScanOp::l1;
    }
    return uha::ScanOp::l2;
}

// Median of `reps` event-timed launches of `launch` (after one untimed).
template <typename F>
double time_launches(cudaStream_t stream, int reps, F launch)
{
    cudaEvent_t a = nullptr;
    cudaEvent_t b = nullptr;
    check_cuda(cudaEventCreate(&a), "cannot create CUDA event");
    check_cuda(cudaEventCreate(&b), "cannot create CUDA event");
    std::vector<float> ms;
    try {
        launch();
        for (int i = 0; i < reps; ++i) {
            check_cuda(cudaEventRecord(a, stream), "event");
            launch();
            check_cuda(cudaEventRecord(b, stream), "event");
            check_cuda(cudaEventSynchronize(b), "autotune launch failed");
            float t = 0.f;
            check_cuda(cudaEventElapsedTime(&t, a, b), "event");
            ms.push_back(t);
        }
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::sort(ms.begin(), ms.end());
    return ms[ms.size() / 2];
}

void autotune(const uha_index* index, uha_workspace* ws, uint64_t batch,
              uha_strategy strategy, uha_tune_report* report)
{
    uha_tune_report rep{};
    const bool trivial = (index->kind == IndexKind::hierarchical && index->rows == 1) ||
                         index->padded_dim == 0;
    const bool median = index->kind == IndexKind::hierarchical && index->metric == UHA_L1;
    if (trivial || batch == 0) {
        // one shape only: nothing to choose
        if (report != nullptr) {
            *report = rep;
        }
        return;
    }
    DeviceGuard guard(index->device);
    cudaStream_t stream = ws->stream;
    TunedPlan best{};
    best.batch = batch;
    best.strategy = static_cast<int>(strategy);
    best.ms = -1.0;
    const int reps = 3;
    if (median) {
        // The median passes' cost depends on the data (the pruning threshold,
        // the survivors), so they are timed on stand-in queries like the
        // index's own data: midpoints of row pairs, with zero projection
        // errors. The passes' answers do not depend on the shape.
        const uint64_t pp = index->padded_dim;
        const uint64_t rows = index->rows;
        require(ws->projected.size() >= batch * pp && ws->query_err.size() >= batch &&
                    ws->coord_err.size() >= batch * pp &&
                    ws->pair_err.size() >= batch * rows,
                UHA_RUNTIME_ERROR, "the workspace has no room for tuning the median passes");
        if (ws->median_min.size() < batch || ws->partials.size() < batch * rows) {
            check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
            if (ws->median_min.size() < batch) {
                ws->median_min.allocate(std::max<uint64_t>(batch, ws->max_batch));
            }
            if (ws->partials.size() < batch * rows) {
                ws->partials.allocate(batch * rows);
            }
        }
        uha::launch_median_tuning_queries(index->scan_rows.get(), rows, pp,
                                          index->projection_dimension, batch,
                                          ws->projected.get(), stream);
        check_cuda(cudaMemsetAsync(ws->query_err.get(), 0, batch * sizeof(float), stream),
                   "cannot clear query errors");
        check_cuda(cudaMemsetAsync(ws->coord_err.get(), 0, batch * pp * sizeof(float), stream),
                   "cannot clear query errors");
        const std::vector<uha::MedianPlan> cands = uha::median_candidates(rows, batch);
        for (size_t i = 0; i < cands.size(); ++i) {
            const double ms = time_launches(stream, reps, [&] {
                uha::launch_median_scan(cands[i], index->scan_rows.get(),
                                        index->scan_rows_t.get(), index->rows_pitch, rows, pp,
                                        index->projection_dimension, ws->projected.get(),
                                        batch, ws->query_err.get(), ws->coord_err.get(),
                                        index->row_err_max, kMedianRel, kMedianAbs,
                                        ws->median_min.get(), ws->partials.get(),
                                        ws->pair_err.get(), stream);
            });
            if (i == 0) {
                rep.default_ms = ms;
            }
            if (best.ms < 0 || ms < best.ms) {
                best.ms = ms;
                best.median = true;
                best.median_plan = cands[i];
            }
        }
        best.candidates = static_cast<int>(cands.size());
        rep.kernel = 3;
        rep.queries_per_pass = best.median_plan.count_queries;
        rep.splits = best.median_plan.samples;
    } else if (precision_strategy(strategy)) {
        const uha::LowpType type = lowp_type(strategy);
        const uha::LowpRows& lp = lowp_rows(index, type, stream);
        ensure_lowp_workspace(ws, index, stream);
        check_cuda(cudaMemsetAsync(ws->queries_lp.get(), 0, ws->queries_lp.bytes(), stream),
                   "cannot clear the query buffer");
        check_cuda(cudaMemsetAsync(ws->query_scales.get(), 0, ws->query_scales.bytes(), stream),
                   "cannot clear query scales");
        const std::vector<uha::LowpPlan> cands =
            uha::lowp_candidates(type, index->rows, lp.pitch, batch, index->sm_count);
        uint64_t most = 0;
        for (const uha::LowpPlan& p : cands) {
            most = std::max<uint64_t>(most, p.splits);
        }
        const uint64_t need = checked_mul(checked_mul(most, batch, "partials"), index->rows,
                                          "partials");
        if (ws->partials.size() < need) {
            check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
            ws->partials.allocate(need);
        }
        int* flag = reinterpret_cast<int*>(ws->counters.get() + 1);
        for (size_t i = 0; i < cands.size(); ++i) {
            const uha::LowpPlan& p = cands[i];
            const double ms = time_launches(stream, reps, [&] {
                uha::launch_lowp_scores(p, type, lp.data.get(), lp.scales.get(), index->rows,
                                        ws->queries_lp.get(), ws->query_scales.get(), batch,
                                        lp.pitch, ws->partials.get(), flag, stream);
            });
            if (i == 0) {
                rep.default_ms = ms;
            }
            if (best.ms < 0 || ms < best.ms) {
                best.ms = ms;
                best.lowp = true;
                best.lowp_plan = p;
            }
        }
        best.candidates = static_cast<int>(cands.size());
        rep.kernel = 2;
        rep.tile_queries = static_cast<uint32_t>(best.lowp_plan.bn);
        rep.splits = best.lowp_plan.splits;
    } else {
        const bool hierarchical = index->kind == IndexKind::hierarchical;
        const float* queries = hierarchical ? ws->projected.get() : ws->prepared.get();
        const uint64_t qcount = hierarchical ? ws->projected.size() : ws->prepared.size();
        check_cuda(cudaMemsetAsync(const_cast<float*>(queries), 0, qcount * sizeof(float),
                                   stream),
                   "cannot clear prepared queries");
        const std::vector<uha::ScanPlan> cands =
            uha::scan_candidates(index->rows, index->padded_dim, batch, index->sm_count);
        uint64_t most = 0;
        for (const uha::ScanPlan& p : cands) {
            most = std::max<uint64_t>(most, p.chunks);
        }
        const uint64_t need = checked_mul(checked_mul(most, batch, "partials"), index->rows,
                                          "partials");
        if (ws->partials.size() < need) {
            check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
            ws->partials.allocate(need);
        }
        const uha::ScanOp op = scan_op(index, strategy);
        for (size_t i = 0; i < cands.size(); ++i) {
            const uha::ScanPlan& p = cands[i];
            const double ms = time_launches(stream, reps, [&] {
                uha::launch_scan(p, op, index->scan_rows.get(), index->rows, index->padded_dim,
                                 index->weights32.get(), queries, batch, ws->partials.get(),
                                 stream);
            });
            if (i == 0) {
                rep.default_ms = ms;
            }
            if (best.ms < 0 || ms < best.ms) {
                best.ms = ms;
                best.lowp = false;
                best.scan = p;
            }
        }
        best.candidates = static_cast<int>(cands.size());
        rep.kernel = static_cast<uint32_t>(best.scan.kernel);
        rep.queries_per_pass = static_cast<uint32_t>(best.scan.queries_per_pass);
        rep.splits = best.scan.chunks;
        rep.tile_queries = best.scan.kernel == 1 ? 64u : 0u;
    }
    check_cuda(cudaStreamSynchronize(stream), "autotune failed");
    ws->tuned.erase(std::remove_if(ws->tuned.begin(), ws->tuned.end(),
                                   [&](const TunedPlan& t) {
                                       return t.batch == batch &&
                                              t.strategy == static_cast<int>(strategy);
                                   }),
                    ws->tuned.end());
    ws->tuned.push_back(best);
    rep.candidates = static_cast<uint32_t>(best.candidates);
    rep.best_ms = best.ms;
    if (report != nullptr) {
        *report = rep;
    }
}

}  // namespace

extern "C" uha_status uha_workspace_autotune(uha_workspace* workspace, uint64_t batch,
                                             uha_strategy strategy, uha_tune_report* report)
{
    return guarded([&] {
        require(workspace != nullptr, UHA_INVALID_ARGUMENT, "workspace must not be null");
        const uha_index* index = workspace->owner;
        require(batch >= 1 && batch <= workspace->max_batch, UHA_INVALID_ARGUMENT,
                "query count exceeds CUDA workspace capacity");
        validate_query_call(index, workspace, nullptr, 0, batch, strategy, nullptr);
        DeviceGuard guard(index->device);
        uha::clear_stale_cuda_error();
        autotune(index, workspace, batch, strategy, report);
    });
}

// ------------------------------------------------------------------ batch

struct uha_batch {
    struct Pair {
        const uha_index* index = nullptr;
        uha_workspace* ws = nullptr;
        uint64_t count = 0;
        uha_strategy strategy = UHA_DIRECT;
        uint64_t offset = 0;
        bool trivial = false;
        cudaEvent_t join = nullptr;
        uha_tune_report tuning{};
    };
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Pair> pairs;
    uint64_t total = 0;
    uint64_t launches = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t graph_nodes = 0;
    cudaEvent_t fork = nullptr;
    cudaEvent_t start = nullptr;
    cudaEvent_t stop = nullptr;
    uha_batch_stats last{};
    // persistent form
    bool persistent = false;
    // the work queue words (kPersistentQueueWords), then the status word
    uha::DeviceBuffer<unsigned int> queue;
    uha::PinnedBuffer<int> host_status;
    uha::DeviceBuffer<unsigned long long> clock;  // stage boundaries (ns)
    uha::PinnedBuffer<unsigned long long> host_clock;
    std::unique_ptr<uha::PersistentParams> params;  // the kernels' parameter
    uint32_t grid[uha::kPersistentKernels] = {};  // CTAs of the persistent kernels

    ~uha_batch()
    {
        int previous = 0;
        const bool ok = cudaGetDevice(&previous) == cudaSuccess;
        cudaSetDevice(device);
        if (exec != nullptr) {
            cudaGraphExecDestroy(exec);
        }
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        for (Pair& p : pairs) {
            if (p.join != nullptr) {
                cudaEventDestroy(p.join);
            }
            if (p.ws != nullptr) {
                uha_workspace_destroy(p.ws);
            }
        }
        for (cudaEvent_t e : {fork, start, stop}) {
            if (e != nullptr) {
                cudaEventDestroy(e);
            }
        }
        if (stream != nullptr) {
            cudaStreamDestroy(stream);
        }
        if (ok) {
            cudaSetDevice(previous);
        }
        uha::clear_stale_cuda_error();
    }
};

namespace {

// One pair's device work on its workspace stream: status words, the
// pipeline over the queries already in ws->raw_queries, result copies into
// the workspace's pinned host mirrors.
uint64_t enqueue_pair(uha_batch::Pair& p)
{
    uha_workspace* ws = p.ws;
    check_cuda(cudaMemsetAsync(ws->counters.get(), 0, ws->counters.bytes(), ws->stream),
               "cannot clear query counters");
    BatchContext ctx{p.index, ws, p.strategy, true};
    ctx.filter_candidates = true;
    const uint64_t launches =
        enqueue_batch(ctx, ws->raw_queries.get(), p.count, ws->call_results.get(),
                      ws->call_exact.get(), false, nullptr, nullptr);
    check_cuda(cudaMemcpyAsync(ws->host_results.get(), ws->call_results.get(),
                               p.count * sizeof(uha::Result), cudaMemcpyDeviceToHost,
                               ws->stream),
               "cannot copy query results from the CUDA device");
    check_cuda(cudaMemcpyAsync(ws->host_exact.get(), ws->call_exact.get(),
                               p.count * sizeof(double), cudaMemcpyDeviceToHost, ws->stream),
               "cannot copy query distances from the CUDA device");
    check_cuda(cudaMemcpyAsync(ws->host_counters.get(), ws->counters.get(),
                               ws->counters.bytes(), cudaMemcpyDeviceToHost, ws->stream),
               "cannot copy query counters from the CUDA device");
    return launches;
}

// Builds the persistent plan of a batch whose pairs are sized (after their
// warm-up runs) and uploads it; fails when a pair has no persistent form.
void build_persistent(uha_batch* batch)
{
    std::vector<uha::PersistentPair> pairs;
    for (uha_batch::Pair& p : batch->pairs) {
        if (p.trivial) {
            continue;
        }
        uha::PersistentPair d{};
        require(p.strategy == UHA_DIRECT && persistent_pair(p.index, p.ws, p.count, &d),
                UHA_INVALID_ARGUMENT,
                "the persistent batch serves hierarchical indexes with the certified "
                "direct strategy, projection dimensions up to 256 and more than 8 "
                "queries per L2 hierarchy");
        pairs.push_back(d);
    }
    require(!pairs.empty(), UHA_INVALID_ARGUMENT, "the persistent batch has no work");
    require(pairs.size() <= uha::kPersistentMaxPairs, UHA_INVALID_ARGUMENT,
            "the persistent batch serves up to 32 pairs");
    const uint32_t count = static_cast<uint32_t>(pairs.size());
    batch->params = std::make_unique<uha::PersistentParams>();
    uha::PersistentParams& params = *batch->params;
    uint32_t used = 0;
    uha::plan_persistent_batch(pairs.data(), count, params.segments, &used, &params.plan);
    std::copy(pairs.begin(), pairs.end(), params.pairs);
    batch->queue.allocate(uha::kPersistentQueueWords + 1);
    batch->host_status.allocate(1);
    batch->host_status.get()[0] = 0;
    batch->clock.allocate(uha::kPersistentStages + 1);
    batch->host_clock.allocate(uha::kPersistentStages + 1);
    std::fill(batch->host_clock.get(), batch->host_clock.get() + uha::kPersistentStages + 1,
              0ull);
    check_cuda(cudaMemsetAsync(batch->queue.get(), 0, batch->queue.bytes(), batch->stream),
               "cannot clear the persistent batch queue");
    check_cuda(cudaMemsetAsync(batch->clock.get(), 0, batch->clock.bytes(), batch->stream),
               "cannot clear the persistent batch stage clock");
    check_cuda(cudaStreamSynchronize(batch->stream), "cannot clear the persistent batch");
    params.plan.queue = batch->queue.get();
    params.plan.status =
        reinterpret_cast<int*>(batch->queue.get() + uha::kPersistentQueueWords);
    params.plan.clock = batch->clock.get();
    for (int part = 0; part < uha::kPersistentKernels; ++part) {
        batch->grid[part] = uha::persistent_grid(part, params.plan.smem_bytes[part]);
        require(batch->grid[part] != 0, UHA_RUNTIME_ERROR,
                "the persistent batch kernel cannot be resident with its shared memory");
    }
    batch->persistent = true;
}

uha_status create_batch(const uha_index* const* indexes, const uint64_t* query_counts,
                        const uha_strategy* strategies, uint64_t count, int autotune_shapes,
                        bool persistent, uha_batch** out)
{
    return guarded([&] {
        require(out != nullptr, UHA_INVALID_ARGUMENT, "output must not be null");
        *out = nullptr;
        require(count >= 1 && indexes != nullptr && query_counts != nullptr,
                UHA_INVALID_ARGUMENT, "a batch needs at least one index");
        auto batch = std::make_unique<uha_batch>();
        batch->device = indexes[0] != nullptr ? indexes[0]->device : 0;
        for (uint64_t i = 0; i < count; ++i) {
            require(indexes[i] != nullptr, UHA_INVALID_ARGUMENT, "index must not be null");
            require(indexes[i]->device == batch->device, UHA_INVALID_ARGUMENT,
                    "all indexes of a batch must be on one device");
            require(query_counts[i] >= 1, UHA_INVALID_ARGUMENT,
                    "every index of a batch needs at least one query");
        }
        DeviceGuard guard(batch->device);
        uha::clear_stale_cuda_error();
        check_cuda(cudaStreamCreateWithFlags(&batch->stream, cudaStreamNonBlocking),
                   "cannot create CUDA stream");
        for (cudaEvent_t* e : {&batch->fork, &batch->start, &batch->stop}) {
            check_cuda(cudaEventCreate(e), "cannot create CUDA event");
        }
        batch->pairs.resize(count);
        for (uint64_t i = 0; i < count; ++i) {
            uha_batch::Pair& p = batch->pairs[i];
            p.index = indexes[i];
            p.count = query_counts[i];
            p.strategy = strategies != nullptr ? strategies[i] : UHA_DIRECT;
            p.offset = batch->total;
            batch->total = uha::checked_add(batch->total, p.count, "batch queries");
            const uha_status st = uha_workspace_create(p.index, p.count, &p.ws);
            if (st != UHA_OK) {
                fail(st, uha_last_error());
            }
            validate_query_call(p.index, p.ws, nullptr, 0, p.count, p.strategy, nullptr);
            p.trivial = (p.index->kind == IndexKind::hierarchical && p.index->rows == 1) ||
                        p.index->padded_dim == 0;
            check_cuda(cudaEventCreateWithFlags(&p.join, cudaEventDisableTiming),
                       "cannot create CUDA event");
            uha_workspace* ws = p.ws;
            ws->call_results.allocate(p.count);
            ws->call_exact.allocate(p.count);
            ws->host_results.allocate(p.count);
            ws->host_exact.allocate(p.count);
            if (!p.trivial) {
                check_cuda(cudaMemsetAsync(ws->raw_queries.get(), 0, ws->raw_queries.bytes(),
                                           ws->stream),
                           "cannot clear the query buffer");
                if (autotune_shapes) {
                    autotune(p.index, ws, p.count, p.strategy, &p.tuning);
                }
                // eager run at the batch's sizes: every buffer reaches its size
                // before capture
                enqueue_pair(p);
                check_cuda(cudaStreamSynchronize(ws->stream), "CUDA batch warm-up failed");
            }
        }
        if (persistent) {
            build_persistent(batch.get());
        }
        // capture: fork every pair from the batch stream, join back (or the
        // persistent kernel and the result copies)
        check_cuda(cudaStreamBeginCapture(batch->stream, cudaStreamCaptureModeThreadLocal),
                   "cannot capture the batch");
        uint64_t launches = 0;
        try {
            if (batch->persistent) {
                uha::launch_persistent_batch(*batch->params, batch->grid, batch->stream);
                launches = uha::kPersistentKernels;
                for (uha_batch::Pair& p : batch->pairs) {
                    if (p.trivial) {
                        continue;
                    }
                    uha_workspace* ws = p.ws;
                    check_cuda(cudaMemcpyAsync(ws->host_results.get(), ws->call_results.get(),
                                               p.count * sizeof(uha::Result),
                                               cudaMemcpyDeviceToHost, batch->stream),
                               "cannot copy query results from the CUDA device");
                    check_cuda(cudaMemcpyAsync(ws->host_exact.get(), ws->call_exact.get(),
                                               p.count * sizeof(double), cudaMemcpyDeviceToHost,
                                               batch->stream),
                               "cannot copy query distances from the CUDA device");
                    check_cuda(cudaMemcpyAsync(ws->host_counters.get(), ws->counters.get(),
                                               ws->counters.bytes(), cudaMemcpyDeviceToHost,
                                               batch->stream),
                               "cannot copy query counters from the CUDA device");
                }
                check_cuda(cudaMemcpyAsync(batch->host_status.get(), batch->params->plan.status,
                                           sizeof(int), cudaMemcpyDeviceToHost, batch->stream),
                           "cannot copy the persistent batch status");
                check_cuda(cudaMemcpyAsync(batch->host_clock.get(), batch->clock.get(),
                                           batch->clock.bytes(), cudaMemcpyDeviceToHost,
                                           batch->stream),
                           "cannot copy the persistent batch stage clock");
            }
            check_cuda(cudaEventRecord(batch->fork, batch->stream), "event");
            for (uha_batch::Pair& p : batch->pairs) {
                if (p.trivial || batch->persistent) {
                    continue;
                }
                check_cuda(cudaStreamWaitEvent(p.ws->stream, batch->fork, 0), "event");
                launches += enqueue_pair(p);
                check_cuda(cudaEventRecord(p.join, p.ws->stream), "event");
                check_cuda(cudaStreamWaitEvent(batch->stream, p.join, 0), "event");
            }
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(batch->stream, &g);
            if (g != nullptr) {
                cudaGraphDestroy(g);
            }
            throw;
        }
        check_cuda(cudaStreamEndCapture(batch->stream, &batch->graph),
                   "cannot capture the batch");
        check_cuda(cudaGraphInstantiate(&batch->exec, batch->graph, 0),
                   "cannot instantiate the batch graph");
        check_cuda(cudaGraphGetNodes(batch->graph, nullptr, &batch->graph_nodes),
                   "cannot inspect the batch graph");
        batch->launches = launches;
        *out = batch.release();
    });
}

}  // namespace

extern "C" uha_status uha_batch_create(const uha_index* const* indexes,
                                       const uint64_t* query_counts,
                                       const uha_strategy* strategies, uint64_t count,
                                       int autotune_shapes, uha_batch** out)
{
    return create_batch(indexes, query_counts, strategies, count, autotune_shapes, false,
                        out);
}

extern "C" uha_status uha_batch_create_persistent(const uha_index* const* indexes,
                                                  const uint64_t* query_counts,
                                                  uint64_t count, int autotune_shapes,
                                                  uha_batch** out)
{
    return create_batch(indexes, query_counts, nullptr, count, autotune_shapes, true, out);
}

extern "C" float* uha_batch_query_buffer(uha_batch* batch, uint64_t pair)
{
    if (batch == nullptr || pair >= batch->pairs.size()) {
        return nullptr;
    }
    return batch->pairs[pair].ws->raw_queries.get();
}

extern "C" uha_status uha_batch_run(uha_batch* batch, const float* const* queries,
                                    int queries_on_device, uint64_t* out_indices,
                                    double* out_distances)
{
    return guarded([&] {
        require(batch != nullptr, UHA_INVALID_ARGUMENT, "batch must not be null");
        require(out_indices != nullptr, UHA_INVALID_ARGUMENT, "output must not be null");
        DeviceGuard guard(batch->device);
        uha::clear_stale_cuda_error();
        if (queries != nullptr) {
            for (const uha_batch::Pair& p : batch->pairs) {
                const float* src = queries[&p - batch->pairs.data()];
                const uint64_t bytes = p.count * p.index->dimension * sizeof(float);
                if (p.trivial || bytes == 0) {
                    continue;
                }
                require(src != nullptr, UHA_INVALID_ARGUMENT, "query pointer must not be null");
                check_cuda(cudaMemcpyAsync(p.ws->raw_queries.get(), src, bytes,
                                           queries_on_device ? cudaMemcpyDeviceToDevice
                                                             : cudaMemcpyHostToDevice,
                                           batch->stream),
                           "cannot copy queries to the CUDA device");
            }
        }
        check_cuda(cudaEventRecord(batch->start, batch->stream), "event");
        check_cuda(cudaGraphLaunch(batch->exec, batch->stream), "cannot launch the batch graph");
        check_cuda(cudaEventRecord(batch->stop, batch->stream), "event");
        check_cuda(cudaStreamSynchronize(batch->stream), "CUDA batch failed");
        if (batch->persistent && batch->host_status.get()[0] != 0) {
            // a work queue wait ran out: reset the queue for the next run
            check_cuda(cudaMemsetAsync(batch->queue.get(), 0, batch->queue.bytes(),
                                       batch->stream),
                       "cannot reset the persistent batch queue");
            check_cuda(cudaStreamSynchronize(batch->stream), "CUDA batch failed");
            batch->host_status.get()[0] = 0;
            fail(UHA_RUNTIME_ERROR, "persistent batch work queue wait timed out");
        }
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, batch->start, batch->stop), "event");
        uha_batch_stats st{};
        st.pairs = batch->pairs.size();
        st.queries = batch->total;
        st.graph_nodes = batch->graph_nodes;
        st.kernel_launches = batch->launches;
        st.device_ms = ms;
        for (uha_batch::Pair& p : batch->pairs) {
            uint64_t* idx = out_indices + p.offset;
            double* dist = out_distances != nullptr ? out_distances + p.offset : nullptr;
            if (p.trivial) {
                fill_trivial(p.count, idx, dist);
                continue;
            }
            if ((p.ws->host_counters.get()[1] & uha::kCandidateOverflow) != 0u) {
                // a filtered candidate list overflowed: this pair again,
                // eagerly, with the slab selection (its queries are still in
                // the workspace)
                p.ws->filter_disabled = true;
                try {
                    enqueue_pair(p);
                    check_cuda(cudaStreamSynchronize(p.ws->stream), "CUDA batch failed");
                } catch (...) {
                    p.ws->filter_disabled = false;
                    throw;
                }
                p.ws->filter_disabled = false;
            }
            finish_call(p.index, p.ws, p.count, p.ws->host_results.get(),
                        p.ws->host_exact.get(), idx, dist);
            st.replayed_queries += p.ws->last.replayed_queries;
        }
        batch->last = st;
    });
}

extern "C" uha_status uha_batch_stats_get(const uha_batch* batch, uha_batch_stats* out)
{
    return guarded([&] {
        require(batch != nullptr && out != nullptr, UHA_INVALID_ARGUMENT,
                "batch and output must not be null");
        *out = batch->last;
        if (out->pairs == 0) {
            out->pairs = batch->pairs.size();
            out->queries = batch->total;
            out->graph_nodes = batch->graph_nodes;
            out->kernel_launches = batch->launches;
        }
    });
}

extern "C" uha_status uha_batch_stage_times(const uha_batch* batch, double* out_ms,
                                            uint64_t count, uint64_t* stages)
{
    return guarded([&] {
        require(batch != nullptr && stages != nullptr && (out_ms != nullptr || count == 0),
                UHA_INVALID_ARGUMENT, "batch and outputs must not be null");
        *stages = batch->persistent ? uha::kPersistentStages : 0;
        // stages overlap (a pair's later stages run while others are in
        // earlier ones): stage s is reported from the time every unit of the
        // stages before it had completed to the time every unit up to s had
        // (a stage without units, whose entry is stale, reports zero)
        const unsigned long long* c = batch->host_clock.get();
        unsigned long long frontier = c[0];
        for (uint64_t s = 0; s < count; ++s) {
            const bool have = batch->persistent && s < uha::kPersistentStages && c[0] != 0;
            if (!have) {
                out_ms[s] = 0.0;
                continue;
            }
            const unsigned long long e = std::max(frontier, c[s + 1]);
            out_ms[s] = static_cast<double>(e - frontier) * 1e-6;
            frontier = e;
        }
    });
}

extern "C" uha_status uha_batch_tuning(const uha_batch* batch, uint64_t pair,
                                       uha_tune_report* out)
{
    return guarded([&] {
        require(batch != nullptr && out != nullptr && pair < batch->pairs.size(),
                UHA_INVALID_ARGUMENT, "no such batch pair");
        *out = batch->pairs[pair].tuning;
    });
}

extern "C" void uha_batch_destroy(uha_batch* batch)
{
    delete batch;
}
