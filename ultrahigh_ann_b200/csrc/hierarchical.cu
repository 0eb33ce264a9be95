// Hierarchical-index kernels: the projection of rows (build) and queries
// (query time) and the median-|diff| scan of the L1 hierarchy.
//
// Reference semantics: projected rows are the binary64 product of the sampled
// rows with the p x k projection (include/ultrahigh_ann/core/
// dense_matrix.hpp:59-113, used by src/hnsvw25/l{1,2}/hierarchical/
// *_projection.cpp), the query is projected in binary64
// (l2_hierarchical_projection.cpp:164-200), and rows are compared by squared
// L2 (hierarchical_l2_ann_index.cpp:63-77) or by the median of |diff|
// (hierarchical_l1_ann_index.cpp:65-99).
//
// On the device the rows are projected once in binary64 with the reference's
// summation order (so the replay works on the reference's exact values) and
// narrowed to binary32 for the scans; queries are projected in binary32 with a
// certified bound on their distance to the reference's binary64 projection.
#include "common.h"
#include "kernels.h"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace uha {
namespace {

constexpr int kThreads = 256;

__global__ void project_rows64_kernel(const float* __restrict__ sampled,
                                      uint64_t row_count, uint64_t padded_k,
                                      uint64_t k,
                                      const double* __restrict__ projection,
                                      uint64_t p, double* __restrict__ reps,
                                      int* bad)
{
    const uint64_t total = row_count * p;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) +
                        threadIdx.x;
         idx < total; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t row = idx / p;
        const uint64_t j = idx - row * p;
        const float* x = sampled + row * padded_k;
        const double* c = projection + j * k;
        double s = 0.0;
        for (uint64_t i = 0; i < k; ++i) {
            s = __dadd_rn(s, __dmul_rn(static_cast<double>(x[i]), c[i]));
        }
        if (!isfinite(s)) {
            atomicOr(bad, 1);
        }
        reps[idx] = s;
    }
}

// One warp per row.
__global__ void narrow_rows_kernel(const double* __restrict__ reps,
                                   uint64_t row_count, uint64_t p,
                                   float* __restrict__ out, uint64_t padded_p,
                                   float* __restrict__ row_err, bool euclidean,
                                   int* bad)
{
    const uint64_t warp_id =
        (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (warp_id >= row_count) {
        return;
    }
    const double* r = reps + warp_id * p;
    float* o = out + warp_id * padded_p;
    double acc = 0.0;
    for (uint64_t j = lane; j < padded_p; j += 32) {
        float v = 0.f;
        if (j < p) {
            v = static_cast<float>(r[j]);
            if (!isfinite(v)) {
                atomicOr(bad, 2);
            }
            const double e = fabs(static_cast<double>(v) - r[j]);
            acc = euclidean ? fma(e, e, acc) : fmax(acc, e);
        }
        o[j] = v;
    }
    for (int offset = 16; offset > 0; offset /= 2) {
        const double other = __shfl_xor_sync(0xffffffffu, acc, offset);
        acc = euclidean ? acc + other : fmax(acc, other);
    }
    if (lane == 0) {
        double e = euclidean ? sqrt(acc) : acc;
        // the binary64 sum/sqrt above carry relative error far below 1e-12
        e = e * (1.0 + 1e-12) + 1e-300;
        row_err[warp_id] = __double2float_ru(e);
    }
}

constexpr int kProjQueries = 4;    // queries per CTA
constexpr int kProjCols = 64;      // projected coordinates per CTA
constexpr int kProjK = 32;         // k per shared-memory stage

// y[b][j] = sum_i x[b][i] P[j][i] with a two-level binary32 sum (32-term
// stages), plus a = sum_i |x[b][i] P[j][i]| for the error bound. Thread
// (jj, qq) owns one (query, coordinate); stages of x and P go through shared
// memory. The per-coordinate error e = err_per_abs * a (+ an underflow term)
// is folded into err_acc[b]: a maximum (max-norm, atomicMax on the bit
// pattern) or a sum of squares rounded up (2-norm, finished by
// finish_query_err_kernel).
__global__ void __launch_bounds__(kProjQueries * kProjCols)
    project_queries_kernel(const float* __restrict__ x, uint64_t batch,
                           uint64_t padded_k, uint64_t k,
                           const float* __restrict__ proj, uint64_t p,
                           float* __restrict__ y, uint64_t padded_p,
                           float* __restrict__ err_acc, double err_per_abs,
                           bool euclidean, int* error_flag)
{
    __shared__ float sx[kProjQueries][kProjK];
    __shared__ float sp[kProjCols][kProjK + 1];
    const int jj = threadIdx.x % kProjCols;
    const int qq = threadIdx.x / kProjCols;
    const uint64_t j = blockIdx.x * static_cast<uint64_t>(kProjCols) + jj;
    const uint64_t b = blockIdx.y * static_cast<uint64_t>(kProjQueries) + qq;
    float total = 0.f;
    float total_abs = 0.f;
    for (uint64_t k0 = 0; k0 < k; k0 += kProjK) {
        __syncthreads();
        for (int i = threadIdx.x; i < kProjQueries * kProjK; i += blockDim.x) {
            const int r = i / kProjK;
            const int c = i % kProjK;
            const uint64_t bb = blockIdx.y * static_cast<uint64_t>(kProjQueries) + r;
            sx[r][c] = (bb < batch && k0 + c < k) ? x[bb * padded_k + k0 + c] : 0.f;
        }
        for (int i = threadIdx.x; i < kProjCols * kProjK; i += blockDim.x) {
            const int r = i / kProjK;
            const int c = i % kProjK;
            const uint64_t jr = blockIdx.x * static_cast<uint64_t>(kProjCols) + r;
            sp[r][c] = (jr < p && k0 + c < k) ? proj[jr * padded_k + k0 + c] : 0.f;
        }
        __syncthreads();
        float part = 0.f;
        float part_abs = 0.f;
#pragma unroll 8
        for (int c = 0; c < kProjK; ++c) {
            const float t = sx[qq][c] * sp[jj][c];
            part = fmaf(sx[qq][c], sp[jj][c], part);
            part_abs += fabsf(t);
        }
        total += part;
        total_abs += part_abs;
    }
    if (b >= batch || j >= padded_p) {
        return;
    }
    if (j >= p) {
        y[b * padded_p + j] = 0.f;
        return;
    }
    if (!isfinite(total)) {
        atomicOr(error_flag, 4);
    }
    y[b * padded_p + j] = total;
    // a bound on the exact sum of |x P| from its binary32 evaluation, then the
    // per-coordinate error
    const double e = err_per_abs * static_cast<double>(total_abs) +
                     static_cast<double>(k + 2) * 1.0e-44;
    if (euclidean) {
        atomicAdd(err_acc + b, __double2float_ru(e * e));
    } else {
        atomicMax(reinterpret_cast<unsigned int*>(err_acc + b),
                  __float_as_uint(__double2float_ru(e)));
    }
}

__global__ void finish_query_err_kernel(float* err, uint64_t batch,
                                        bool euclidean)
{
    const uint64_t b = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (b < batch && euclidean) {
        // err holds a binary32 sum of squares, each term rounded up; the
        // rounding of up to 16384 additions stays below 1e-3 relative,
        // covered by the factor.
        err[b] = __fmul_ru(__fsqrt_ru(err[b]), 1.001f);
    }
}

// k-th smallest (0-based) of the lane's values across the warp; values are
// nonnegative binary32 (their bit patterns order like the values).
template <int PER_LANE>
__device__ float warp_select(const float (&v)[PER_LANE], int count_valid,
                             uint32_t k)
{
    uint32_t prefix = 0;
    for (int bit = 30; bit >= 0; --bit) {
        const uint32_t trial = prefix | (1u << bit);
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < PER_LANE; ++i) {
            c += (i < count_valid && __float_as_uint(v[i]) < trial) ? 1u : 0u;
        }
        c = __reduce_add_sync(0xffffffffu, c);
        if (c <= k) {
            prefix = trial;
        }
    }
    return __uint_as_float(prefix);
}

// |r_j - y_j| for j < p into the lane's registers (lane + 32 i); +inf for a
// binary32 overflow, 0 past p.
template <int PER_LANE>
__device__ __forceinline__ int load_abs_diffs(const float* r, const float* y, uint32_t p,
                                              int lane, float (&v)[PER_LANE])
{
    int valid = 0;
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) {
        const uint32_t j = lane + 32u * i;
        v[i] = 0.f;
        if (j < p) {
            float d = fabsf(r[j] - y[j]);
            if (!(d <= FLT_MAX)) {
                d = __int_as_float(0x7f800000);
            }
            v[i] = d;
            valid = i + 1;
        }
    }
    return valid;
}

// Binary32 median of the warp's p values: the (p/2)-th smallest, and for
// even p the midpoint with the (p/2 - 1)-th, which is the upper middle itself
// when it occurs twice there, else the largest value below it.
template <int PER_LANE>
__device__ __forceinline__ float warp_median(const float (&v)[PER_LANE], int valid,
                                             uint32_t p)
{
    const uint32_t mid = p / 2;
    const float upper = warp_select<PER_LANE>(v, valid, mid);
    if (p % 2 != 0) {
        return upper;
    }
    const uint32_t ub = __float_as_uint(upper);
    uint32_t below = 0;
    uint32_t largest_below = 0;
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) {
        const uint32_t b = __float_as_uint(v[i]);
        if (i < valid && b < ub) {
            ++below;
            largest_below = b > largest_below ? b : largest_below;
        }
    }
    below = __reduce_add_sync(0xffffffffu, below);
    largest_below = __reduce_max_sync(0xffffffffu, largest_below);
    const float lower = below < mid ? upper : __uint_as_float(largest_below);
    return lower + (upper - lower) * 0.5f;
}

// Stage 1 of the median scan: exact binary32 medians of `samples` rows spread
// over the index (row s * rows / samples) for every query; their minimum per
// query goes to min_bits[q] (binary32 bits; nonnegative values order like
// them; the slots hold 0xffffffff before the launch).
template <int PER_LANE>
__global__ void __launch_bounds__(kThreads)
    median_sample_kernel(const float* __restrict__ rows, uint32_t row_count,
                         uint32_t padded_p, uint32_t p, const float* __restrict__ queries,
                         uint32_t batch, uint32_t samples, float* __restrict__ partials,
                         unsigned int* __restrict__ min_bits)
{
    const int lane = threadIdx.x % 32;
    const uint64_t total = static_cast<uint64_t>(samples) * batch;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
    for (uint64_t w = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 32;
         w < total; w += stride) {
        const uint32_t q = static_cast<uint32_t>(w / samples);
        const uint32_t s = static_cast<uint32_t>(w - uint64_t(q) * samples);
        const uint32_t row = static_cast<uint32_t>(uint64_t(s) * row_count / samples);
        float v[PER_LANE];
        const int valid = load_abs_diffs<PER_LANE>(rows + uint64_t(row) * padded_p,
                                                   queries + uint64_t(q) * padded_p, p, lane,
                                                   v);
        const float median = warp_median<PER_LANE>(v, valid, p);
        if (lane == 0) {
            partials[static_cast<uint64_t>(q) * row_count + row] = median;
            atomicMin(min_bits + q, __float_as_uint(median));
        }
    }
}

// Stage 2. With U the sampled minimum, E the largest row error plus the
// query's error and (rel, abs) the median bound,
//   T = (U (1 + rel) + 2 E + 2 abs) / (1 - rel)   (rounded up)
// exceeds every upper bound the sampled rows give, so a row whose binary32
// median is above T has a lower bound above the query's smallest upper bound
// and cannot be the argmin. One count decides it: fewer than p/2 + 1 values
// <= T (odd p), fewer than p/2 (even p: the lower middle is above T). Such a
// row stores -T (a negative distance: "at least T, no upper bound"); every
// other row stores its binary32 median.
// Each warp takes a contiguous run of (query, row) pairs in query-major
// order, so the query's values and threshold stay in registers across rows
// and the next row's values are loaded while the current one is decided.
template <int PER_LANE>
__device__ __forceinline__ void load_lane_values(const float* v, uint32_t p, int lane,
                                                 float (&out)[PER_LANE])
{
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) {
        const uint32_t j = lane + 32u * i;
        out[i] = j < p ? v[j] : 0.f;
    }
}

__device__ __forceinline__ float median_threshold(const unsigned int* min_bits,
                                                  const float* query_err, uint32_t q,
                                                  float row_err_max, float rel, float abs_err)
{
    const float u = __uint_as_float(min_bits[q]);
    if (!(u <= FLT_MAX)) {
        return __int_as_float(0x7f800000);
    }
    const float e = __fadd_ru(row_err_max, query_err[q]);
    const float num = __fadd_ru(__fadd_ru(__fmul_ru(u, __fadd_ru(1.f, rel)), __fmul_ru(2.f, e)),
                                __fmul_ru(2.f, abs_err));
    return __fmul_ru(__fdiv_ru(num, __fsub_rd(1.f, rel)), 1.0000005f);
}

template <int PER_LANE>
__global__ void __launch_bounds__(kThreads)
    median_scan_kernel(const float* __restrict__ rows, uint32_t row_count,
                       uint32_t padded_p, uint32_t p,
                       const float* __restrict__ queries, uint32_t batch,
                       const unsigned int* __restrict__ min_bits,
                       const float* __restrict__ query_err, float row_err_max,
                       float rel, float abs_err, float* __restrict__ partials)
{
    const int lane = threadIdx.x % 32;
    const uint64_t total = static_cast<uint64_t>(row_count) * batch;
    const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
    const uint64_t warp_id = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 32;
    const uint64_t per_warp = (total + warps - 1) / warps;
    const uint64_t begin = warp_id * per_warp;
    const uint64_t end = begin + per_warp < total ? begin + per_warp : total;
    if (begin >= end) {
        return;
    }
    const uint32_t needed = p % 2 != 0 ? p / 2 + 1 : p / 2;
    uint32_t q = static_cast<uint32_t>(begin / row_count);
    uint32_t row = static_cast<uint32_t>(begin - uint64_t(q) * row_count);
    float y[PER_LANE];
    load_lane_values<PER_LANE>(queries + uint64_t(q) * padded_p, p, lane, y);
    float t = median_threshold(min_bits, query_err, q, row_err_max, rel, abs_err);
    float next[PER_LANE];
    load_lane_values<PER_LANE>(rows + uint64_t(row) * padded_p, p, lane, next);
    for (uint64_t w = begin; w < end; ++w) {
        float v[PER_LANE];
        int valid = 0;
#pragma unroll
        for (int i = 0; i < PER_LANE; ++i) {
            const uint32_t j = lane + 32u * i;
            v[i] = 0.f;
            if (j < p) {
                float d = fabsf(next[i] - y[i]);
                if (!(d <= FLT_MAX)) {
                    d = __int_as_float(0x7f800000);
                }
                v[i] = d;
                valid = i + 1;
            }
        }
        const uint32_t cur_q = q;
        const uint32_t cur_row = row;
        const float cur_t = t;
        // advance to the next pair and start its loads
        if (++row == row_count) {
            row = 0;
            ++q;
        }
        if (w + 1 < end) {
            if (q != cur_q) {
                load_lane_values<PER_LANE>(queries + uint64_t(q) * padded_p, p, lane, y);
                t = median_threshold(min_bits, query_err, q, row_err_max, rel, abs_err);
            }
            load_lane_values<PER_LANE>(rows + uint64_t(row) * padded_p, p, lane, next);
        }
        float* out = partials + static_cast<uint64_t>(cur_q) * row_count + cur_row;
        if (cur_t <= FLT_MAX) {
            const uint32_t tb = __float_as_uint(cur_t);
            uint32_t at_most = 0;
#pragma unroll
            for (int i = 0; i < PER_LANE; ++i) {
                at_most += (i < valid && __float_as_uint(v[i]) <= tb) ? 1u : 0u;
            }
            at_most = __reduce_add_sync(0xffffffffu, at_most);
            if (at_most < needed) {
                if (lane == 0) {
                    *out = -cur_t;
                }
                continue;
            }
        }
        const float median = warp_median<PER_LANE>(v, valid, p);
        if (lane == 0) {
            *out = median;
        }
    }
}

uint32_t grid_for(uint64_t total)
{
    const uint64_t blocks = (total + kThreads - 1) / kThreads;
    return static_cast<uint32_t>(blocks == 0 ? 1 : (blocks < 148ull * 64 ? blocks : 148ull * 64));
}

}  // namespace

void launch_project_rows64(const float* sampled, uint64_t row_count,
                           uint64_t padded_k, uint64_t k,
                           const double* projection, uint64_t p, double* reps,
                           int* bad, cudaStream_t stream)
{
    project_rows64_kernel<<<grid_for(row_count * p), kThreads, 0, stream>>>(
        sampled, row_count, padded_k, k, projection, p, reps, bad);
    check_cuda(cudaGetLastError(), "cannot launch row projection kernel");
}

void launch_narrow_rows(const double* reps, uint64_t row_count, uint64_t p,
                        float* out, uint64_t padded_p, float* row_err,
                        bool euclidean, int* bad, cudaStream_t stream)
{
    const uint64_t threads = row_count * 32;
    narrow_rows_kernel<<<static_cast<uint32_t>((threads + kThreads - 1) / kThreads),
                         kThreads, 0, stream>>>(reps, row_count, p, out, padded_p,
                                                row_err, euclidean, bad);
    check_cuda(cudaGetLastError(), "cannot launch row narrowing kernel");
}

void launch_project_queries(const float* gathered, uint64_t batch,
                            uint64_t padded_k, uint64_t k,
                            const float* proj32, uint64_t p, float* out,
                            uint64_t padded_p, float* query_err,
                            double err_per_abs, bool euclidean,
                            int* error_flag, cudaStream_t stream)
{
    check_cuda(cudaMemsetAsync(query_err, 0, batch * sizeof(float), stream),
               "cannot clear projection error");
    const dim3 grid(static_cast<uint32_t>((padded_p + kProjCols - 1) / kProjCols),
                    static_cast<uint32_t>((batch + kProjQueries - 1) / kProjQueries));
    project_queries_kernel<<<grid, kProjQueries * kProjCols, 0, stream>>>(
        gathered, batch, padded_k, k, proj32, p, out, padded_p, query_err,
        err_per_abs, euclidean, error_flag);
    check_cuda(cudaGetLastError(), "cannot launch query projection kernel");
    finish_query_err_kernel<<<static_cast<uint32_t>((batch + kThreads - 1) / kThreads),
                              kThreads, 0, stream>>>(query_err, batch, euclidean);
    check_cuda(cudaGetLastError(), "cannot launch projection error kernel");
}

namespace {

uint32_t median_samples(uint64_t row_count)
{
    return static_cast<uint32_t>(row_count < 32 ? row_count : 32);
}

template <int PER_LANE>
void launch_median_pair(const float* rows, uint32_t rc, uint32_t pp, uint32_t pv,
                        const float* queries, uint32_t b, const float* query_err,
                        float row_err_max, float rel, float abs_err,
                        unsigned int* min_bits, float* partials, cudaStream_t stream)
{
    // grid-stride warps over the pairs: at most 16 resident CTAs' worth per SM
    const uint64_t cap = 148ull * 16;
    const uint32_t samples = median_samples(rc);
    const uint64_t sample_blocks =
        (static_cast<uint64_t>(samples) * b * 32 + kThreads - 1) / kThreads;
    median_sample_kernel<PER_LANE>
        <<<static_cast<uint32_t>(std::min(sample_blocks, cap)), kThreads, 0, stream>>>(
            rows, rc, pp, pv, queries, b, samples, partials, min_bits);
    const uint64_t blocks = (static_cast<uint64_t>(rc) * b * 32 + kThreads - 1) / kThreads;
    median_scan_kernel<PER_LANE>
        <<<static_cast<uint32_t>(std::min(blocks, cap)), kThreads, 0, stream>>>(
            rows, rc, pp, pv, queries, b, min_bits, query_err, row_err_max, rel, abs_err,
            partials);
}

}  // namespace

void launch_median_scan(const float* rows, uint64_t row_count, uint64_t padded_p,
                        uint64_t p, const float* queries, uint64_t batch,
                        const float* query_err, float row_err_max, float rel,
                        float abs_err, unsigned int* min_bits, float* partials,
                        cudaStream_t stream)
{
    const uint32_t rc = static_cast<uint32_t>(row_count);
    const uint32_t pp = static_cast<uint32_t>(padded_p);
    const uint32_t pv = static_cast<uint32_t>(p);
    const uint32_t b = static_cast<uint32_t>(batch);
    check_cuda(cudaMemsetAsync(min_bits, 0xff, batch * sizeof(unsigned int), stream),
               "cannot clear median thresholds");
    if (p <= 32) {
        launch_median_pair<1>(rows, rc, pp, pv, queries, b, query_err, row_err_max, rel,
                              abs_err, min_bits, partials, stream);
    } else if (p <= 64) {
        launch_median_pair<2>(rows, rc, pp, pv, queries, b, query_err, row_err_max, rel,
                              abs_err, min_bits, partials, stream);
    } else if (p <= 128) {
        launch_median_pair<4>(rows, rc, pp, pv, queries, b, query_err, row_err_max, rel,
                              abs_err, min_bits, partials, stream);
    } else if (p <= 256) {
        launch_median_pair<8>(rows, rc, pp, pv, queries, b, query_err, row_err_max, rel,
                              abs_err, min_bits, partials, stream);
    } else if (p <= 512) {
        launch_median_pair<16>(rows, rc, pp, pv, queries, b, query_err, row_err_max, rel,
                               abs_err, min_bits, partials, stream);
    } else if (p <= 1024) {
        launch_median_pair<32>(rows, rc, pp, pv, queries, b, query_err, row_err_max, rel,
                               abs_err, min_bits, partials, stream);
    } else {
        fail(UHA_LENGTH_ERROR,
             "the L1 hierarchy supports projection dimensions up to 1024");
    }
    check_cuda(cudaGetLastError(), "cannot launch median scan kernel");
}

}  // namespace uha
