// Request loop over device-resident indexes (no reference counterpart; the
// reference answers synchronous query / query_batch calls only).
//
// Requests are queued per index. One dispatcher thread owns the device side:
// whenever fewer than `slots` batches are in flight it takes the index whose
// oldest request is oldest, moves up to max_batch of its queued requests into
// a batch, and enqueues that batch's whole pipeline (query gather or copies,
// the index's kernels, result copies, a completion event) on the stream of a
// pooled workspace of that index. Completed batches are detected by their
// events; their answers go to a result queue with the latency from submission
// to the completion seen here. Requests that arrive while batches run wait
// in their queue for the next free slot (continuous batching), and batches of
// different indexes overlap on the device.
//
// Admission by HBM budget: a batch needs an idle pooled workspace of its
// index. A new workspace is created only while the pool's device bytes plus
// its size stay within the budget; idle workspaces of other indexes are
// released first when that makes room; otherwise the batch waits for a
// running one to finish.
//
// A batch whose answers fail validation (a non-finite query) is split: its
// requests go back to the front of their queue and run alone, so only the
// offending request reports the error.
#include "common.h"
#include "engine_internal.h"
#include "index_types.h"
#include "kernels.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace uha_engine;
using uha::check_cuda;
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

uint64_t now_ns()
{
    return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(
                                     std::chrono::steady_clock::now().time_since_epoch())
                                     .count());
}

uint64_t workspace_device_bytes(const uha_workspace* ws)
{
    return ws->raw_queries.bytes() + ws->prepared.bytes() + ws->projected.bytes() +
           ws->query_err.bytes() + ws->query_norms.bytes() + ws->partials.bytes() +
           ws->call_results.bytes() + ws->call_exact.bytes() + ws->counters.bytes() +
           ws->finalize_scratch.bytes() + ws->queries_lp.bytes() + ws->query_scales.bytes() +
           ws->query_amax.bytes() + ws->candidates.bytes() + ws->cand_dist.bytes() +
           ws->rescore_done.bytes() + ws->median_min.bytes() + ws->coord_err.bytes() +
           ws->pair_err.bytes() + ws->gathered_lp.bytes() + ws->gathered_scales.bytes() +
           ws->gathered_amax.bytes() + ws->projected64.bytes();
}

bool trivial_index(const uha_index* index)
{
    return (index->kind == IndexKind::hierarchical && index->rows == 1) ||
           index->padded_dim == 0;
}

// Largest partial-sum slab any batch size up to max_batch needs.
uint64_t max_partials(const uha_index* index, uha_strategy strategy, uint64_t max_batch)
{
    uint64_t most = 0;
    for (uint64_t n = 1; n <= max_batch; ++n) {
        uint64_t chunks = 1;
        if (precision_strategy(strategy)) {
            const uha::LowpType type = lowp_type(strategy);
            chunks = uha::plan_lowp(type, index->rows, uha::lowp_pitch(type, index->scan_dim),
                                    n, index->sm_count)
                         .splits;
        } else if (!(index->kind == IndexKind::hierarchical && index->metric == UHA_L1)) {
            chunks = uha::plan_scan(index->rows, index->padded_dim, n, index->sm_count).chunks;
        }
        most = std::max(most, chunks * n);
    }
    return uha::checked_mul(most, index->rows, "partials");
}

}  // namespace

struct uha_server {
    struct Request {
        uint64_t tag;
        uint32_t index_id;
        const float* query;
        uint64_t submit_ns;
        bool alone;
    };
    struct Pooled {
        uha_workspace* ws = nullptr;
        uint32_t index_id = 0;
        uha::DeviceBuffer<const float*> ptrs;
        uha::PinnedBuffer<const float*> host_ptrs;
        cudaEvent_t done = nullptr;
        uint64_t bytes = 0;
    };
    struct Entry {
        const uha_index* index = nullptr;
        uha_strategy strategy = UHA_DIRECT;
        std::deque<Request> pending;
        std::vector<Pooled*> idle;
        uint64_t ws_bytes = 0;
        bool trivial = false;
    };
    struct Flight {
        Pooled* pooled;
        std::vector<Request> reqs;
    };

    int device = 0;
    uha_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work;
    std::condition_variable cv_done;
    std::vector<std::unique_ptr<Entry>> entries;
    std::vector<std::unique_ptr<Pooled>> pool;
    std::vector<Flight> flights;  // dispatcher thread only
    std::deque<uha_server_result> results;
    std::vector<double> latencies;
    uint64_t submitted = 0;
    uint64_t completed = 0;
    uint64_t failed = 0;
    uint64_t batches = 0;
    uint64_t batched_queries = 0;
    uint64_t admission_waits = 0;
    uint64_t evictions = 0;
    uint64_t pool_bytes = 0;
    uint64_t peak_pool_bytes = 0;
    uint32_t peak_in_flight = 0;
    uint64_t first_submit_ns = 0;
    uint64_t last_done_ns = 0;
    bool stopping = false;
    std::string loop_error;
    std::thread thread;

    ~uha_server()
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            stopping = true;
        }
        cv_work.notify_all();
        if (thread.joinable()) {
            thread.join();
        }
        int previous = 0;
        const bool ok = cudaGetDevice(&previous) == cudaSuccess;
        cudaSetDevice(device);
        for (auto& p : pool) {
            release(p.get());
        }
        if (ok) {
            cudaSetDevice(previous);
        }
        uha::clear_stale_cuda_error();
    }

    static void release(Pooled* p)
    {
        if (p->ws != nullptr) {
            cudaStreamSynchronize(p->ws->stream);
            uha_workspace_destroy(p->ws);
            p->ws = nullptr;
        }
        if (p->done != nullptr) {
            cudaEventDestroy(p->done);
            p->done = nullptr;
        }
        p->ptrs.release();
        p->host_ptrs.release();
    }

    // A workspace of `id` sized for max_batch and warmed once at that size.
    std::unique_ptr<Pooled> make_pooled(uint32_t id)
    {
        auto p = std::make_unique<Pooled>();
        try {
            build_pooled(id, *p);
        } catch (...) {
            release(p.get());
            throw;
        }
        return p;
    }

    void build_pooled(uint32_t id, Pooled& pooled)
    {
        Entry& e = *entries[id];
        Pooled* p = &pooled;
        p->index_id = id;
        const uha_status st = uha_workspace_create(e.index, cfg.max_batch, &p->ws);
        if (st != UHA_OK) {
            fail(st, uha_last_error());
        }
        check_cuda(cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming),
                   "cannot create CUDA event");
        uha_workspace* ws = p->ws;
        ws->call_results.allocate(cfg.max_batch);
        ws->call_exact.allocate(cfg.max_batch);
        ws->host_results.allocate(cfg.max_batch);
        ws->host_exact.allocate(cfg.max_batch);
        p->ptrs.allocate(cfg.max_batch);
        p->host_ptrs.allocate(cfg.max_batch);
        if (!e.trivial) {
            ws->partials.allocate(max_partials(e.index, e.strategy, cfg.max_batch));
            check_cuda(cudaMemsetAsync(ws->raw_queries.get(), 0, ws->raw_queries.bytes(),
                                       ws->stream),
                       "cannot clear the query buffer");
            check_cuda(cudaMemsetAsync(ws->counters.get(), 0, ws->counters.bytes(), ws->stream),
                       "cannot clear query counters");
            const BatchContext ctx{e.index, ws, e.strategy, true};
            enqueue_batch(ctx, ws->raw_queries.get(), cfg.max_batch, ws->call_results.get(),
                          ws->call_exact.get(), false, nullptr, nullptr);
            check_cuda(cudaStreamSynchronize(ws->stream), "CUDA warm-up failed");
        }
        p->bytes = workspace_device_bytes(ws) + p->ptrs.bytes();
    }

    // An idle workspace of `id`, or a new one within the budget; nullptr when
    // the budget admits none now. Called with `mu` held.
    Pooled* acquire(uint32_t id)
    {
        Entry& e = *entries[id];
        if (!e.idle.empty()) {
            Pooled* p = e.idle.back();
            e.idle.pop_back();
            return p;
        }
        // release idle workspaces of other indexes while that is needed
        while (pool_bytes + e.ws_bytes > cfg.hbm_budget_bytes) {
            Entry* donor = nullptr;
            for (auto& other : entries) {
                if (other.get() != &e && !other->idle.empty()) {
                    donor = other.get();
                    break;
                }
            }
            if (donor == nullptr) {
                return nullptr;
            }
            Pooled* victim = donor->idle.back();
            donor->idle.pop_back();
            pool_bytes -= victim->bytes;
            ++evictions;
            release(victim);
            pool.erase(std::remove_if(pool.begin(), pool.end(),
                                      [&](const std::unique_ptr<Pooled>& q) {
                                          return q.get() == victim;
                                      }),
                       pool.end());
        }
        std::unique_ptr<Pooled> fresh = make_pooled(id);
        Pooled* p = fresh.get();
        pool_bytes += p->bytes;
        peak_pool_bytes = std::max(peak_pool_bytes, pool_bytes);
        pool.push_back(std::move(fresh));
        return p;
    }

    // Enqueues one batch (no lock held).
    void launch(Flight& f)
    {
        Pooled* p = f.pooled;
        Entry& e = *entries[p->index_id];
        uha_workspace* ws = p->ws;
        const uint64_t n = f.reqs.size();
        const uint64_t d = e.index->dimension;
        if (!e.trivial) {
            if (cfg.queries_on_device) {
                for (uint64_t j = 0; j < n; ++j) {
                    p->host_ptrs.get()[j] = f.reqs[j].query;
                }
                check_cuda(cudaMemcpyAsync(p->ptrs.get(), p->host_ptrs.get(),
                                           n * sizeof(const float*), cudaMemcpyHostToDevice,
                                           ws->stream),
                           "cannot copy query addresses");
                uha::launch_gather_vectors(p->ptrs.get(), n, d, ws->raw_queries.get(),
                                           ws->stream);
            } else {
                for (uint64_t j = 0; j < n; ++j) {
                    check_cuda(cudaMemcpyAsync(ws->raw_queries.get() + j * d, f.reqs[j].query,
                                               d * sizeof(float), cudaMemcpyHostToDevice,
                                               ws->stream),
                               "cannot copy queries to the CUDA device");
                }
            }
            check_cuda(cudaMemsetAsync(ws->counters.get(), 0, ws->counters.bytes(), ws->stream),
                       "cannot clear query counters");
            const BatchContext ctx{e.index, ws, e.strategy, true};
            enqueue_batch(ctx, ws->raw_queries.get(), n, ws->call_results.get(),
                          ws->call_exact.get(), false, nullptr, nullptr);
            check_cuda(cudaMemcpyAsync(ws->host_results.get(), ws->call_results.get(),
                                       n * sizeof(uha::Result), cudaMemcpyDeviceToHost,
                                       ws->stream),
                       "cannot copy query results from the CUDA device");
            check_cuda(cudaMemcpyAsync(ws->host_exact.get(), ws->call_exact.get(),
                                       n * sizeof(double), cudaMemcpyDeviceToHost, ws->stream),
                       "cannot copy query distances from the CUDA device");
            check_cuda(cudaMemcpyAsync(ws->host_counters.get(), ws->counters.get(),
                                       ws->counters.bytes(), cudaMemcpyDeviceToHost,
                                       ws->stream),
                       "cannot copy query counters from the CUDA device");
        }
        check_cuda(cudaEventRecord(p->done, ws->stream), "event");
    }

    // Answers of a finished batch (no lock held); returns the requests to run
    // alone when a multi-request batch failed validation.
    std::vector<Request> finish(Flight& f, std::vector<uha_server_result>& out)
    {
        Pooled* p = f.pooled;
        Entry& e = *entries[p->index_id];
        const uint64_t n = f.reqs.size();
        std::vector<uint64_t> rows(n, 0);
        std::vector<double> dist(n, 0.0);
        uha_status status = UHA_OK;
        if (e.trivial) {
            fill_trivial(n, rows.data(), dist.data());
        } else {
            try {
                check_cuda(cudaEventSynchronize(p->done), "CUDA batch failed");
                finish_call(e.index, p->ws, n, p->ws->host_results.get(),
                            p->ws->host_exact.get(), rows.data(), dist.data());
            } catch (const uha::Error& err) {
                status = err.status;
            }
        }
        if (status != UHA_OK && n > 1 && status != UHA_RUNTIME_ERROR) {
            std::vector<Request> retry = f.reqs;
            for (Request& r : retry) {
                r.alone = true;
            }
            return retry;
        }
        const uint64_t t = now_ns();
        for (uint64_t j = 0; j < n; ++j) {
            const Request& r = f.reqs[j];
            uha_server_result res{};
            res.tag = r.tag;
            res.index_id = r.index_id;
            res.status = static_cast<uint32_t>(status);
            res.row = status == UHA_OK ? rows[j] : 0;
            res.distance = status == UHA_OK ? dist[j] : 0.0;
            res.latency_us = static_cast<double>(t - r.submit_ns) * 1e-3;
            out.push_back(res);
        }
        return {};
    }

    // The entry whose oldest queued request is oldest (mu held).
    Entry* next_entry(uint32_t* id)
    {
        Entry* best = nullptr;
        for (uint32_t i = 0; i < entries.size(); ++i) {
            Entry* e = entries[i].get();
            if (!e->pending.empty() &&
                (best == nullptr || e->pending.front().submit_ns < best->pending.front().submit_ns)) {
                best = e;
                *id = i;
            }
        }
        return best;
    }

    void loop()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lock(mu);
        while (true) {
            bool progressed = false;
            // completions
            for (size_t i = 0; i < flights.size();) {
                Flight& f = flights[i];
                const cudaError_t q = cudaEventQuery(f.pooled->done);
                if (q == cudaErrorNotReady) {
                    ++i;
                    continue;
                }
                if (q != cudaSuccess) {
                    cudaGetLastError();
                }
                Flight done = std::move(f);
                flights.erase(flights.begin() + static_cast<long>(i));
                lock.unlock();
                std::vector<uha_server_result> out;
                std::vector<Request> retry;
                try {
                    retry = finish(done, out);
                } catch (const std::exception& ex) {
                    lock.lock();
                    loop_error = ex.what();
                    lock.unlock();
                }
                lock.lock();
                Entry& e = *entries[done.pooled->index_id];
                e.idle.push_back(done.pooled);
                for (auto it = retry.rbegin(); it != retry.rend(); ++it) {
                    e.pending.push_front(*it);
                }
                for (const uha_server_result& r : out) {
                    results.push_back(r);
                    latencies.push_back(r.latency_us);
                    ++completed;
                    failed += r.status != UHA_OK ? 1 : 0;
                }
                if (!out.empty()) {
                    last_done_ns = now_ns();
                    cv_done.notify_all();
                }
                progressed = true;
            }
            // dispatch
            while (flights.size() < cfg.slots) {
                uint32_t id = 0;
                Entry* e = next_entry(&id);
                if (e == nullptr) {
                    break;
                }
                Pooled* p = nullptr;
                try {
                    p = acquire(id);
                } catch (const std::exception& ex) {
                    loop_error = ex.what();
                }
                if (p == nullptr) {
                    ++admission_waits;
                    break;
                }
                Flight f{p, {}};
                const uint64_t take =
                    e->pending.front().alone
                        ? 1
                        : std::min<uint64_t>(cfg.max_batch, e->pending.size());
                for (uint64_t j = 0; j < take; ++j) {
                    if (j > 0 && e->pending.front().alone) {
                        break;
                    }
                    f.reqs.push_back(e->pending.front());
                    e->pending.pop_front();
                }
                ++batches;
                batched_queries += f.reqs.size();
                lock.unlock();
                bool ok = true;
                try {
                    launch(f);
                } catch (const std::exception& ex) {
                    ok = false;
                    lock.lock();
                    loop_error = ex.what();
                    lock.unlock();
                }
                lock.lock();
                if (!ok) {
                    // report the batch as failed
                    const uint64_t t = now_ns();
                    for (const Request& r : f.reqs) {
                        uha_server_result res{};
                        res.tag = r.tag;
                        res.index_id = r.index_id;
                        res.status = UHA_RUNTIME_ERROR;
                        res.latency_us = static_cast<double>(t - r.submit_ns) * 1e-3;
                        results.push_back(res);
                        ++completed;
                        ++failed;
                    }
                    entries[id]->idle.push_back(p);
                    cv_done.notify_all();
                    continue;
                }
                flights.push_back(std::move(f));
                peak_in_flight = std::max<uint32_t>(peak_in_flight,
                                                    static_cast<uint32_t>(flights.size()));
                progressed = true;
            }
            if (progressed) {
                continue;
            }
            bool queued = false;
            for (auto& e : entries) {
                queued = queued || !e->pending.empty();
            }
            if (stopping && flights.empty()) {
                break;
            }
            if (flights.empty() && !queued) {
                cv_work.wait(lock);
            } else {
                // batches on the device: poll their events
                lock.unlock();
                std::this_thread::yield();
                lock.lock();
            }
        }
    }
};

extern "C" uha_status uha_server_create(int device, const uha_server_config* config,
                                        uha_server** out)
{
    return guarded([&] {
        require(out != nullptr && config != nullptr, UHA_INVALID_ARGUMENT,
                "config and output must not be null");
        *out = nullptr;
        require(config->max_batch >= 1 && config->slots >= 1, UHA_INVALID_ARGUMENT,
                "max_batch and slots must be positive");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            fail(UHA_RUNTIME_ERROR, "no usable CUDA device");
        }
        require(device >= 0 && device < count, UHA_INVALID_ARGUMENT, "invalid CUDA device");
        auto server = std::make_unique<uha_server>();
        server->device = device;
        server->cfg = *config;
        uha_server* s = server.get();
        server->thread = std::thread([s] { s->loop(); });
        *out = server.release();
    });
}

extern "C" uha_status uha_server_add_index(uha_server* server, const uha_index* index,
                                           uha_strategy strategy, uint32_t* out_id)
{
    return guarded([&] {
        require(server != nullptr && index != nullptr, UHA_INVALID_ARGUMENT,
                "server and index must not be null");
        require(index->device == server->device, UHA_INVALID_ARGUMENT,
                "index is on another device than the server");
        DeviceGuard guard(server->device);
        auto entry = std::make_unique<uha_server::Entry>();
        entry->index = index;
        entry->strategy = strategy;
        entry->trivial = trivial_index(index);
        std::lock_guard<std::mutex> lock(server->mu);
        {
            // validate the strategy against the index as a query would
            uha_workspace* probe = nullptr;
            const uha_status st = uha_workspace_create(index, 1, &probe);
            if (st != UHA_OK) {
                fail(st, uha_last_error());
            }
            std::unique_ptr<uha_workspace, void (*)(uha_workspace*)> hold(probe,
                                                                          uha_workspace_destroy);
            validate_query_call(index, probe, nullptr, 0, 1, strategy, nullptr);
        }
        const uint32_t id = static_cast<uint32_t>(server->entries.size());
        server->entries.push_back(std::move(entry));
        try {
            std::unique_ptr<uha_server::Pooled> first = server->make_pooled(id);
            require(first->bytes <= server->cfg.hbm_budget_bytes, UHA_LENGTH_ERROR,
                    "one query workspace of this index exceeds the HBM budget");
            server->entries[id]->ws_bytes = first->bytes;
            if (server->pool_bytes + first->bytes <= server->cfg.hbm_budget_bytes) {
                server->pool_bytes += first->bytes;
                server->peak_pool_bytes = std::max(server->peak_pool_bytes, server->pool_bytes);
                server->entries[id]->idle.push_back(first.get());
                server->pool.push_back(std::move(first));
            } else {
                uha_server::release(first.get());
            }
        } catch (...) {
            server->entries.pop_back();
            throw;
        }
        if (out_id != nullptr) {
            *out_id = id;
        }
    });
}

extern "C" uha_status uha_server_reserve(uha_server* server, uint32_t index_id,
                                         uint32_t count, uint32_t* held)
{
    return guarded([&] {
        require(server != nullptr, UHA_INVALID_ARGUMENT, "server must not be null");
        DeviceGuard guard(server->device);
        std::lock_guard<std::mutex> lock(server->mu);
        require(index_id < server->entries.size(), UHA_INVALID_ARGUMENT,
                "unknown server index");
        uha_server::Entry& e = *server->entries[index_id];
        uint32_t have = 0;
        for (const auto& p : server->pool) {
            have += p->index_id == index_id ? 1u : 0u;
        }
        while (have < count && server->pool_bytes + e.ws_bytes <= server->cfg.hbm_budget_bytes) {
            std::unique_ptr<uha_server::Pooled> fresh = server->make_pooled(index_id);
            server->pool_bytes += fresh->bytes;
            server->peak_pool_bytes = std::max(server->peak_pool_bytes, server->pool_bytes);
            e.idle.push_back(fresh.get());
            server->pool.push_back(std::move(fresh));
            ++have;
        }
        if (held != nullptr) {
            *held = have;
        }
    });
}

namespace {

void push_request(uha_server* server, uint32_t index_id, const float* query, uint64_t tag,
                  uint64_t t)
{
    require(index_id < server->entries.size(), UHA_INVALID_ARGUMENT, "unknown server index");
    require(query != nullptr || server->entries[index_id]->index->dimension == 0,
            UHA_INVALID_ARGUMENT, "query pointer must not be null");
    if (server->submitted == 0 || server->first_submit_ns == 0) {
        server->first_submit_ns = t;
    }
    server->entries[index_id]->pending.push_back({tag, index_id, query, t, false});
    ++server->submitted;
}

}  // namespace

extern "C" uha_status uha_server_submit(uha_server* server, uint32_t index_id,
                                        const float* query, uint64_t tag)
{
    return guarded([&] {
        require(server != nullptr, UHA_INVALID_ARGUMENT, "server must not be null");
        {
            std::lock_guard<std::mutex> lock(server->mu);
            push_request(server, index_id, query, tag, now_ns());
        }
        server->cv_work.notify_one();
    });
}

extern "C" uha_status uha_server_replay(uha_server* server, uint64_t count,
                                        const uint32_t* index_ids,
                                        const float* const* queries,
                                        const double* arrival_us, const uint64_t* tags)
{
    return guarded([&] {
        require(server != nullptr, UHA_INVALID_ARGUMENT, "server must not be null");
        require(count == 0 || (index_ids != nullptr && queries != nullptr &&
                               arrival_us != nullptr),
                UHA_INVALID_ARGUMENT, "replay arrays must not be null");
        const uint64_t start = now_ns();
        uint64_t i = 0;
        while (i < count) {
            const uint64_t due = start + static_cast<uint64_t>(arrival_us[i] * 1e3);
            uint64_t t = now_ns();
            while (t < due) {
                if (due - t > 200000) {
                    std::this_thread::sleep_for(std::chrono::microseconds(100));
                } else {
                    std::this_thread::yield();
                }
                t = now_ns();
            }
            {
                // every request whose arrival has passed, in one locked section
                std::lock_guard<std::mutex> lock(server->mu);
                while (i < count && start + static_cast<uint64_t>(arrival_us[i] * 1e3) <= t) {
                    push_request(server, index_ids[i], queries[i],
                                 tags != nullptr ? tags[i] : i,
                                 start + static_cast<uint64_t>(arrival_us[i] * 1e3));
                    ++i;
                }
            }
            server->cv_work.notify_one();
        }
    });
}

extern "C" uha_status uha_server_drain(uha_server* server)
{
    return guarded([&] {
        require(server != nullptr, UHA_INVALID_ARGUMENT, "server must not be null");
        std::unique_lock<std::mutex> lock(server->mu);
        server->cv_done.wait(lock, [&] { return server->completed >= server->submitted; });
        if (!server->loop_error.empty()) {
            const std::string message = server->loop_error;
            server->loop_error.clear();
            fail(UHA_RUNTIME_ERROR, message);
        }
    });
}

extern "C" uha_status uha_server_poll(uha_server* server, uha_server_result* out,
                                      uint64_t capacity, uint64_t* count)
{
    return guarded([&] {
        require(server != nullptr && count != nullptr, UHA_INVALID_ARGUMENT,
                "server and count must not be null");
        require(out != nullptr || capacity == 0, UHA_INVALID_ARGUMENT,
                "output must not be null");
        std::lock_guard<std::mutex> lock(server->mu);
        const uint64_t n = std::min<uint64_t>(capacity, server->results.size());
        for (uint64_t i = 0; i < n; ++i) {
            out[i] = server->results.front();
            server->results.pop_front();
        }
        *count = n;
    });
}

extern "C" uha_status uha_server_stats_get(uha_server* server, uha_server_stats* out)
{
    return guarded([&] {
        require(server != nullptr && out != nullptr, UHA_INVALID_ARGUMENT,
                "server and output must not be null");
        std::lock_guard<std::mutex> lock(server->mu);
        uha_server_stats st{};
        st.submitted = server->submitted;
        st.completed = server->completed;
        st.failed = server->failed;
        st.batches = server->batches;
        st.mean_batch = server->batches != 0 ? static_cast<double>(server->batched_queries) /
                                                   static_cast<double>(server->batches)
                                             : 0.0;
        if (!server->latencies.empty()) {
            std::vector<double> lat = server->latencies;
            auto pick = [&](double q) {
                const size_t k = std::min(lat.size() - 1,
                                          static_cast<size_t>(q * static_cast<double>(lat.size())));
                std::nth_element(lat.begin(), lat.begin() + static_cast<long>(k), lat.end());
                return lat[k];
            };
            st.p50_us = pick(0.50);
            st.p99_us = pick(0.99);
            st.max_us = *std::max_element(lat.begin(), lat.end());
        }
        if (server->last_done_ns > server->first_submit_ns && server->completed != 0) {
            st.throughput_qps = static_cast<double>(server->completed) /
                                (static_cast<double>(server->last_done_ns -
                                                     server->first_submit_ns) *
                                 1e-9);
        }
        st.workspace_bytes = server->pool_bytes;
        st.peak_workspace_bytes = server->peak_pool_bytes;
        st.admission_waits = server->admission_waits;
        st.evictions = server->evictions;
        st.peak_in_flight = server->peak_in_flight;
        *out = st;
    });
}

extern "C" uha_status uha_server_reset_stats(uha_server* server)
{
    return guarded([&] {
        require(server != nullptr, UHA_INVALID_ARGUMENT, "server must not be null");
        std::lock_guard<std::mutex> lock(server->mu);
        server->latencies.clear();
        server->submitted -= server->completed;
        server->completed = 0;
        server->failed = 0;
        server->batches = 0;
        server->batched_queries = 0;
        server->admission_waits = 0;
        server->evictions = 0;
        server->peak_in_flight = 0;
        server->peak_pool_bytes = server->pool_bytes;
        server->first_submit_ns = 0;
        server->last_done_ns = 0;
    });
}

extern "C" void uha_server_destroy(uha_server* server)
{
    delete server;
}
