// ORACLE (test infrastructure only): the reference's own hierarchical query,
// run on the sampled columns of an index whose full representative matrix is
// too large for host memory (65,536 x 262,144 values).
//
// A hierarchical index reads only its sampled columns: the projected rows are
// sum_i P[.][i] * row[col_i] (src/hnsvw25/l2/hierarchical/
// l2_hierarchical_projection.cpp:79-117, l1/.../l1_hierarchical_projection.cpp
// :84-124) and the query projection reads query[col_i] the same way
// (detail::project_l{2,1}_hierarchical_query). The same index is therefore
// the reference index over the r x k matrix of sampled columns with the
// sample's columns renumbered 0..k-1 (same multiplicities and inverse
// probabilities, same order), queried with the sampled query values.
//
// The reference builds that index through a private constructor from a
// CoordinateSample and the engine state after sampling
// (hierarchical_l2_ann_index.hpp / hierarchical_l1_ann_index.hpp); this file
// reaches it by compiling those headers with `private` read as `public`
// (access does not change the class layout). Its binary64 projected rows are
// computed in row blocks on several threads, each block by the reference's own
// build_l{2,1}_hierarchical_projection from a copy of the same engine state,
// so every block draws the identical projection matrix. The index then answers
// with its own query().
#include <algorithm>
#include <cmath>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <exception>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <ranges>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#define private public
#include "ultrahigh_ann/hnsvw25/l1/hierarchical/hierarchical_l1_ann_index.hpp"
#include "ultrahigh_ann/hnsvw25/l2/hierarchical/hierarchical_l2_ann_index.hpp"
#undef private
#include "hnsvw25/l1/hierarchical/l1_hierarchical_projection.hpp"
#include "hnsvw25/l2/hierarchical/l2_hierarchical_projection.hpp"

using namespace ultrahigh_ann;

namespace {

thread_local std::string g_hier_error;

template <typename F>
void on_threads(uint64_t n, int threads, F body)
{
    threads = std::max(1, threads);
    const uint64_t per = (n + threads - 1) / threads;
    std::vector<std::thread> pool;
    std::exception_ptr error;
    std::mutex m;
    for (int t = 0; t < threads; ++t) {
        const uint64_t b = std::min(n, t * per);
        const uint64_t e = std::min(n, b + per);
        if (b >= e) {
            break;
        }
        pool.emplace_back([&, b, e] {
            try {
                body(b, e);
            } catch (...) {
                std::lock_guard<std::mutex> lock(m);
                error = std::current_exception();
            }
        });
    }
    for (auto& th : pool) {
        th.join();
    }
    if (error) {
        std::rethrow_exception(error);
    }
}

CoordinateSample renumbered(const uint64_t* mult, const double* invp, uint64_t k)
{
    CoordinateSample s;
    for (uint64_t i = 0; i < k; ++i) {
        s.columns.push_back(SampledColumn{i, mult[i], invp[i]});
    }
    return s;
}

template <typename Index, typename Build>
void answer(Build build, const float* rows, uint64_t r, uint64_t k,
            const CoordinateSample& sample, uint64_t p, const std::mt19937_64& engine,
            const float* queries, uint64_t n, int threads, uint64_t* out)
{
    // projected rows, row block by row block, each from the same engine state
    std::vector<double> projected(r * p);
    const uint64_t blocks = std::min<uint64_t>(r, std::max(1, threads) * 4);
    on_threads(blocks, threads, [&](uint64_t b0, uint64_t b1) {
        for (uint64_t b = b0; b < b1; ++b) {
            const uint64_t lo = r * b / blocks;
            const uint64_t hi = r * (b + 1) / blocks;
            if (lo == hi) {
                continue;
            }
            const DenseMatrix block(std::vector<float>(rows + lo * k, rows + hi * k),
                                    hi - lo, k);
            std::mt19937_64 copy = engine;
            auto proj = build(block, sample, p, copy);
            const auto v = proj.projected_representatives.values();
            std::copy(v.begin(), v.end(), projected.begin() + lo * p);
        }
    });
    // the index itself, built by its own constructor on the first row, then
    // given every row's projection
    std::mt19937_64 copy = engine;
    const DenseMatrix first(std::vector<float>(rows, rows + k), 1, k);
    Index index(first, sample, p, copy);
    index.reduced_representatives_ = DoubleDenseMatrix(std::move(projected), r, p);
    on_threads(n, threads, [&](uint64_t b, uint64_t e) {
        auto ws = index.make_query_workspace();
        for (uint64_t q = b; q < e; ++q) {
            out[q] = index.query(std::span<const float>(queries + q * k, k), ws);
        }
    });
}

}  // namespace

extern "C" {

const char* ref_hier_last_error() { return g_hier_error.c_str(); }

// metric 0 = L2 (Rademacher JL), 1 = L1 (Cauchy, median). rows: r x k sampled
// columns; mult / invp: the sample in column order; state: the engine state
// after sampling (operator<< text); queries: n x k sampled values.
int ref_hierarchical_sampled(int metric, const float* rows, uint64_t r, uint64_t k,
                             const uint64_t* mult, const double* invp, uint64_t p,
                             const char* state, const float* queries, uint64_t n,
                             int threads, uint64_t* out)
{
    try {
        if (r == 0 || k == 0 || p == 0 || state == nullptr) {
            throw std::invalid_argument("empty hierarchy");
        }
        std::mt19937_64 engine;
        std::istringstream is{std::string(state)};
        is >> engine;
        const CoordinateSample sample = renumbered(mult, invp, k);
        if (metric == 0) {
            answer<HierarchicalL2AnnIndex>(
                [](const DenseMatrix& m, const CoordinateSample& s, uint64_t pd,
                   std::mt19937_64& e) {
                    return detail::build_l2_hierarchical_projection(m, s, pd, e);
                },
                rows, r, k, sample, p, engine, queries, n, threads, out);
        } else {
            answer<HierarchicalL1AnnIndex>(
                [](const DenseMatrix& m, const CoordinateSample& s, uint64_t pd,
                   std::mt19937_64& e) {
                    return detail::build_l1_hierarchical_projection(m, s, pd, e);
                },
                rows, r, k, sample, p, engine, queries, n, threads, out);
        }
        return 0;
    } catch (const std::exception& e) {
        g_hier_error = e.what();
        return 1;
    }
}

}  // extern "C"
