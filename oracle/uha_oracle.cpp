// ORACLE — test infrastructure only. A CPU restatement of the reference's
// query-path arithmetic, used by tests/, smoke() and bench.py's cpu_baseline
// leg as the checker. The engine never links or calls it.
//
// Every function cites the reference code it restates (paths relative to the
// reference project root). All arithmetic is binary64 with the reference's
// operation order; the build flags (-O2 -fno-fast-math -ffp-contract=off)
// keep the compiler from fusing or reordering it. Pinned against the
// reference itself (oracle/_ref, built from its sources by oracle/Makefile)
// and against the fixtures in tests/golden/.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include <omp.h>

namespace {

// src/core/l2_distance.cpp:9-25
double squared_l2(const float* a, const float* b, uint64_t n)
{
    double s = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        const double d = static_cast<double>(a[i]) - static_cast<double>(b[i]);
        s += d * d;
    }
    return s;
}

// src/core/l1_distance.cpp:12-28 — std::transform_reduce over random-access
// ranges in libstdc++ 13 (<numeric>): groups of four as
// init + ((t0 + t1) + (t2 + t3)), then the tail one by one.
double l1_transform_reduce(const float* a, const float* b, uint64_t n)
{
    auto t = [&](uint64_t i) {
        return std::abs(static_cast<double>(a[i]) - static_cast<double>(b[i]));
    };
    double init = 0.0;
    uint64_t i = 0;
    for (; n - i >= 4; i += 4) {
        const double v1 = t(i) + t(i + 1);
        const double v2 = t(i + 2) + t(i + 3);
        const double v3 = v1 + v2;
        init = init + v3;
    }
    for (; i < n; ++i) {
        init = init + t(i);
    }
    return init;
}

// strict < scan keeps the first minimum (src/core/dense_l2_scan_index.cpp:25-41)
template <typename Dist>
uint64_t argmin_rows(uint64_t r, Dist dist, double* best_out)
{
    uint64_t best = 0;
    double best_d = dist(0);
    for (uint64_t row = 1; row < r; ++row) {
        const double d = dist(row);
        if (d < best_d) {
            best_d = d;
            best = row;
        }
    }
    if (best_out != nullptr) {
        *best_out = best_d;
    }
    return best;
}

}  // namespace

extern "C" {

int oracle_threads(void)
{
    return omp_get_max_threads();
}

// ------------------------------------------------------------- sampling
// src/coordinate_sampling/coordinate_sampling.cpp:14-45. Returns k, or -1 on
// an invalid probability (the reference throws std::domain_error).
int64_t oracle_sample(const double* probs, uint64_t d, uint64_t repetitions,
                      uint64_t seed, uint64_t* cols, uint64_t* mult,
                      double* invp, char* state_out, uint64_t state_capacity)
{
    std::mt19937_64 engine(seed);
    int64_t k = 0;
    for (uint64_t j = 0; j < d; ++j) {
        const double p = probs[j];
        if (!std::isfinite(p) || p < 0.0 || p > 1.0) {
            return -1;
        }
        if (p == 0.0 || repetitions == 0) {
            continue;
        }
        std::binomial_distribution<std::size_t> dist(repetitions, p);
        const std::size_t m = dist(engine);
        if (m != 0) {
            cols[k] = j;
            mult[k] = m;
            invp[k] = 1.0 / p;
            ++k;
        }
    }
    if (state_out != nullptr) {
        std::ostringstream os;
        os << engine;
        const std::string s = os.str();
        if (s.size() + 1 <= state_capacity) {
            std::memcpy(state_out, s.c_str(), s.size() + 1);
        }
    }
    return k;
}

// ------------------------------------------------------ projection matrices
// src/hnsvw25/l2/hierarchical/l2_hierarchical_projection.cpp:53-77; the engine
// state continues from `state` (operator<< text), or from `seed` when null.
void oracle_jl_matrix(const uint64_t* mult, const double* invp, uint64_t k,
                      uint64_t p, const char* state, uint64_t seed, double* out)
{
    std::mt19937_64 engine(seed);
    if (state != nullptr) {
        std::istringstream is{std::string(state)};
        is >> engine;
    }
    const double row_scaling = 1.0 / std::sqrt(static_cast<double>(p));
    uint64_t idx = 0;
    for (uint64_t row = 0; row < p; ++row) {
        for (uint64_t i = 0; i < k; ++i) {
            std::binomial_distribution<std::size_t> signs(mult[i], 0.5);
            const std::size_t pos = signs(engine);
            const double signed_sum =
                2.0 * static_cast<double>(pos) - static_cast<double>(mult[i]);
            out[idx++] = signed_sum * std::sqrt(invp[i]) * row_scaling;
        }
    }
}

// src/hnsvw25/l1/hierarchical/l1_hierarchical_projection.cpp:54-77
void oracle_cauchy_matrix(const uint64_t* mult, const double* invp, uint64_t k,
                          uint64_t p, const char* state, uint64_t seed,
                          double* out)
{
    std::mt19937_64 engine(seed);
    if (state != nullptr) {
        std::istringstream is{std::string(state)};
        is >> engine;
    }
    std::cauchy_distribution<double> cauchy(0.0, 1.0);
    uint64_t idx = 0;
    for (uint64_t row = 0; row < p; ++row) {
        for (uint64_t i = 0; i < k; ++i) {
            out[idx++] =
                cauchy(engine) * invp[i] * static_cast<double>(mult[i]);
        }
    }
}

// ----------------------------------------------------------- exact scans
// ExactL2Index -> DenseL2ScanIndex::query_batch (src/core/dense_l2_scan_index.cpp:124-172)
void oracle_exact_l2(const float* rows, uint64_t r, uint64_t d,
                     const float* queries, uint64_t n, uint64_t* out,
                     double* dist)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        const float* qv = queries + q * d;
        out[q] = argmin_rows(
            r, [&](uint64_t row) { return squared_l2(qv, rows + row * d, d); },
            dist != nullptr ? dist + q : nullptr);
    }
}

// ExactL1Index::query (src/exact/l1/exact_l1_index.cpp:26-57)
void oracle_exact_l1(const float* rows, uint64_t r, uint64_t d,
                     const float* queries, uint64_t n, uint64_t* out,
                     double* dist)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        const float* qv = queries + q * d;
        out[q] = argmin_rows(
            r,
            [&](uint64_t row) { return l1_transform_reduce(qv, rows + row * d, d); },
            dist != nullptr ? dist + q : nullptr);
    }
}

// Weighted L1 over binary32 weights: sum_j double(w_j) |q_j - r_j| in column
// order. (The reference has no CPU class for this; it is the binary64 value
// the CUDA weighted scan approximates, cuda_dense_l1_scan_index.hpp:13-16.)
void oracle_weighted_l1(const float* rows, uint64_t r, uint64_t d,
                        const float* weights, const float* queries, uint64_t n,
                        uint64_t* out, double* dist)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        const float* qv = queries + q * d;
        out[q] = argmin_rows(
            r,
            [&](uint64_t row) {
                const float* rv = rows + row * d;
                double s = 0.0;
                for (uint64_t j = 0; j < d; ++j) {
                    s += static_cast<double>(weights[j]) *
                         std::abs(static_cast<double>(qv[j]) -
                                  static_cast<double>(rv[j]));
                }
                return s;
            },
            dist != nullptr ? dist + q : nullptr);
    }
}

// ------------------------------------------------------------ flat scans
// SampledCoordinateL2AnnIndex: embedding rows' = float(row[col] * scale),
// scale = float(sqrt(double(mult) * invp))
// (src/coordinate_sampling/l2_coordinate_embedding.cpp:29-88), packed query
// float(q[col] * scale) (:90-127), DenseL2ScanIndex scan (:124-172).
// Returns 0, or -1 when a sampled query value or its product is not finite.
int oracle_flat_l2(const float* rows, uint64_t r, uint64_t d,
                   const uint64_t* cols, const uint64_t* mult,
                   const double* invp, uint64_t k, const float* queries,
                   uint64_t n, uint64_t* out, double* dist)
{
    std::vector<float> scale(k);
    for (uint64_t i = 0; i < k; ++i) {
        scale[i] = static_cast<float>(
            std::sqrt(static_cast<double>(mult[i]) * invp[i]));
    }
    std::vector<float> emb(r * k);
    for (uint64_t row = 0; row < r; ++row) {
        for (uint64_t i = 0; i < k; ++i) {
            emb[row * k + i] = rows[row * d + cols[i]] * scale[i];
        }
    }
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        std::vector<float> packed(k);
        for (uint64_t i = 0; i < k; ++i) {
            const float v = queries[q * d + cols[i]];
            const float t = v * scale[i];
            if (!std::isfinite(v) || !std::isfinite(t)) {
                bad = 1;
            }
            packed[i] = t;
        }
        out[q] = argmin_rows(
            r,
            [&](uint64_t row) { return squared_l2(packed.data(), emb.data() + row * k, k); },
            dist != nullptr ? dist + q : nullptr);
    }
    return bad ? -1 : 0;
}

// SampledCoordinateL1AnnIndex::query with weighted_l1_distance
// (src/coordinate_sampling/sampled_coordinate_l1_ann_index.cpp:63-83, 119-154)
int oracle_flat_l1(const float* rows, uint64_t r, uint64_t d,
                   const uint64_t* cols, const uint64_t* mult,
                   const double* invp, uint64_t k, const float* queries,
                   uint64_t n, uint64_t* out, double* dist)
{
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        const float* qv = queries + q * d;
        for (uint64_t i = 0; i < k; ++i) {
            if (!std::isfinite(qv[cols[i]])) {
                bad = 1;
            }
        }
        if (r == 1) {
            out[q] = 0;
            if (dist != nullptr) {
                dist[q] = 0.0;
            }
            continue;
        }
        out[q] = argmin_rows(
            r,
            [&](uint64_t row) {
                double s = 0.0;
                for (uint64_t i = 0; i < k; ++i) {
                    const double diff =
                        std::abs(static_cast<double>(qv[cols[i]]) -
                                 static_cast<double>(rows[row * d + cols[i]]));
                    s += static_cast<double>(mult[i]) * invp[i] * diff;
                }
                return s;
            },
            dist != nullptr ? dist + q : nullptr);
    }
    return bad ? -1 : 0;
}

// ---------------------------------------------------- hierarchical scans
// Projected rows: BasicDenseMatrix::multiply_right_transposed with a binary64
// accumulator (include/ultrahigh_ann/core/dense_matrix.hpp:59-113), i.e.
// reps[row][j] = sum_i double(sampled[row][i]) * P[j][i] in i order.
void oracle_project_rows(const float* rows, uint64_t r, uint64_t d,
                         const uint64_t* cols, uint64_t k, const double* proj,
                         uint64_t p, double* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t row = 0; row < static_cast<int64_t>(r); ++row) {
        for (uint64_t j = 0; j < p; ++j) {
            double s = 0.0;
            for (uint64_t i = 0; i < k; ++i) {
                s += static_cast<double>(rows[row * d + cols[i]]) *
                     proj[j * k + i];
            }
            out[row * p + j] = s;
        }
    }
}

// project_l{1,2}_hierarchical_query (l2_hierarchical_projection.cpp:164-200)
static int project_query(const float* q, const uint64_t* cols, uint64_t k,
                         const double* proj, uint64_t p, double* y)
{
    for (uint64_t i = 0; i < k; ++i) {
        if (!std::isfinite(q[cols[i]])) {
            return -1;
        }
    }
    for (uint64_t j = 0; j < p; ++j) {
        double s = 0.0;
        for (uint64_t i = 0; i < k; ++i) {
            s += static_cast<double>(q[cols[i]]) * proj[j * k + i];
        }
        if (!std::isfinite(s)) {
            return -2;
        }
        y[j] = s;
    }
    return 0;
}

// HierarchicalL2AnnIndex::query (src/hnsvw25/l2/hierarchical/
// hierarchical_l2_ann_index.cpp:152-188). Returns 0, -1 (non-finite sampled
// query value) or -2 (non-finite projected query).
int oracle_hier_l2(const double* reps, uint64_t r, const float* queries,
                   uint64_t n, uint64_t d, const uint64_t* cols, uint64_t k,
                   const double* proj, uint64_t p, uint64_t* out, double* dist)
{
    int status = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        if (r == 1) {
            out[q] = 0;
            if (dist != nullptr) {
                dist[q] = 0.0;
            }
            continue;
        }
        std::vector<double> y(p);
        const int s = project_query(queries + q * d, cols, k, proj, p, y.data());
        if (s != 0) {
#pragma omp critical
            status = status == 0 ? s : status;
            continue;
        }
        out[q] = argmin_rows(
            r,
            [&](uint64_t row) {
                double acc = 0.0;
                for (uint64_t j = 0; j < p; ++j) {
                    const double diff = reps[row * p + j] - y[j];
                    acc += diff * diff;
                }
                return acc;
            },
            dist != nullptr ? dist + q : nullptr);
    }
    return status;
}

// HierarchicalL1AnnIndex::query with median_absolute_difference
// (src/hnsvw25/l1/hierarchical/hierarchical_l1_ann_index.cpp:65-99, 189-236)
int oracle_hier_l1(const double* reps, uint64_t r, const float* queries,
                   uint64_t n, uint64_t d, const uint64_t* cols, uint64_t k,
                   const double* proj, uint64_t p, uint64_t* out, double* dist)
{
    int status = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < static_cast<int64_t>(n); ++q) {
        if (r == 1) {
            out[q] = 0;
            if (dist != nullptr) {
                dist[q] = 0.0;
            }
            continue;
        }
        std::vector<double> y(p);
        const int s = project_query(queries + q * d, cols, k, proj, p, y.data());
        if (s != 0) {
#pragma omp critical
            status = status == 0 ? s : status;
            continue;
        }
        std::vector<double> diff(p);
        out[q] = argmin_rows(
            r,
            [&](uint64_t row) {
                for (uint64_t j = 0; j < p; ++j) {
                    diff[j] = std::abs(reps[row * p + j] - y[j]);
                }
                auto upper = diff.begin() + static_cast<std::ptrdiff_t>(p / 2);
                std::nth_element(diff.begin(), upper, diff.end());
                if (p % 2 != 0) {
                    return *upper;
                }
                const double lower = *std::max_element(diff.begin(), upper);
                return lower + (*upper - lower) * 0.5;
            },
            dist != nullptr ? dist + q : nullptr);
    }
    return status;
}

// ---------------------------------------------------------- probabilities
// src/hnsvw25/l2/importance_sampling.cpp:19-45 (metric 0) and
// src/hnsvw25/l1/importance_sampling.cpp:19-47 (metric 1). Pairs are split
// over threads; the maximum is exact, so the result equals the sequential one.
void oracle_probabilities(int metric, const float* rows, uint64_t r,
                          uint64_t d, double* out)
{
    std::fill(out, out + d, 0.0);
    if (r < 2) {
        return;
    }
    const int threads = omp_get_max_threads();
    std::vector<std::vector<double>> local(threads, std::vector<double>(d, 0.0));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < static_cast<int64_t>(r) - 1; ++a) {
        std::vector<double>& m = local[omp_get_thread_num()];
        const float* ra = rows + a * d;
        for (uint64_t b = a + 1; b < r; ++b) {
            const float* rb = rows + b * d;
            const double dist = metric == 0 ? squared_l2(ra, rb, d)
                                            : l1_transform_reduce(ra, rb, d);
            if (dist == 0.0) {
                continue;
            }
            const double inv = 1.0 / dist;
            for (uint64_t j = 0; j < d; ++j) {
                const double diff =
                    static_cast<double>(ra[j]) - static_cast<double>(rb[j]);
                const double v = metric == 0 ? std::min(1.0, diff * diff * inv)
                                             : std::abs(diff) * inv;
                m[j] = std::max(m[j], v);
            }
        }
    }
    for (const auto& m : local) {
        for (uint64_t j = 0; j < d; ++j) {
            out[j] = std::max(out[j], m[j]);
        }
    }
}

}  // extern "C"
