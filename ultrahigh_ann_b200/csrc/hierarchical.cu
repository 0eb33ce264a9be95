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
                           float* __restrict__ err_acc, float* __restrict__ coord_err,
                           double err_per_abs, bool euclidean, int* error_flag)
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
        if (coord_err != nullptr) {
            coord_err[b * padded_p + j] = 0.f;
        }
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
    if (coord_err != nullptr) {
        coord_err[b * padded_p + j] = __double2float_ru(e);
    }
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
__device__ __forceinline__ void warp_middles(const float (&v)[PER_LANE], int valid,
                                             uint32_t p, float& lower_out, float& upper_out)
{
    const uint32_t mid = p / 2;
    const float upper = warp_select<PER_LANE>(v, valid, mid);
    upper_out = upper;
    lower_out = upper;
    if (p % 2 != 0) {
        return;
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
    lower_out = below < mid ? upper : __uint_as_float(largest_below);
}

template <int PER_LANE>
__device__ __forceinline__ float warp_median(const float (&v)[PER_LANE], int valid,
                                             uint32_t p)
{
    float lower, upper;
    warp_middles<PER_LANE>(v, valid, p, lower, upper);
    return p % 2 != 0 ? upper : lower + (upper - lower) * 0.5f;
}

// Bound on |m - m64| for an order statistic m of the lane values v (binary32
// |r - y|) against the same order statistic of the reference values, which
// lie within eps_j of v_j: the k-th smallest of the perturbed values is at
// least min(m, min over v_j >= m of v_j - eps_j) and at most
// max(m, max over v_j <= m of v_j + eps_j), so only coordinates within eps_j
// of m contribute. Returns the larger side, over the lower and upper middle.
template <int PER_LANE>
__device__ __forceinline__ float warp_middle_error(const float (&v)[PER_LANE],
                                                   const float (&eps)[PER_LANE], int valid,
                                                   float m_lower, float m_upper)
{
    if (!(m_upper <= 1.0e37f)) {
        return __int_as_float(0x7f800000);
    }
    float e = 0.f;
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) {
        // an overflowed |diff| lies far above either middle
        if (i < valid && v[i] <= FLT_MAX) {
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const float m = side == 0 ? m_lower : m_upper;
                const float gap = v[i] >= m ? __fsub_rd(v[i], m) : __fsub_rd(m, v[i]);
                e = fmaxf(e, __fsub_ru(eps[i], gap));
            }
        }
    }
    return __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(e)));
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
// other row gets its binary32 median in stage 3.
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

// The stage-2 count over the transposed rows (rows_t[j][row], row pitch
// r_pitch): R rows per thread and Q queries per CTA, so each row value read
// from L2 serves Q queries and each query value broadcast from shared memory
// serves R rows. A pruned pair stores -T, any other pair the survivor mark (bits
// 0xffffffff, a NaN no distance takes) for median_survivor_kernel. Values
// above T are counted from the sign bit of T - |r_j - y_j|: a rounded
// difference of binary32 values has the sign of the exact one (and is +0
// when they are equal), so the count is that of |r_j - y_j| > T exactly.
constexpr int kCountRows = 128;
constexpr uint32_t kSurvivorMark = 0xffffffffu;

// Rows per thread: 2 with 4 or 8 queries per CTA (4 rows measured no faster:
// 128 registers), 1 for the smallest batches so that the grid still spreads
// over the SMs.
template <int Q>
__host__ __device__ constexpr int count_rows_per_thread()
{
    return Q >= 4 ? 2 : 1;
}

template <int Q>
__global__ void __launch_bounds__(kCountRows)
    median_count_kernel(const float* __restrict__ rows_t, uint32_t r_pitch,
                        uint32_t row_count, uint32_t padded_p, uint32_t p,
                        const float* __restrict__ queries, uint32_t batch,
                        uint32_t q_begin, const unsigned int* __restrict__ min_bits,
                        const float* __restrict__ query_err, float row_err_max, float rel,
                        float abs_err, float* __restrict__ partials)
{
    constexpr int R = count_rows_per_thread<Q>();
    extern __shared__ float4 ys4[];  // [Q][padded_p / 4]
    float* ys = reinterpret_cast<float*>(ys4);
    const uint32_t q0 = q_begin + blockIdx.y * Q;
    for (uint32_t i = threadIdx.x; i < Q * padded_p; i += blockDim.x) {
        const uint32_t qq = i / padded_p;
        const uint32_t j = i - qq * padded_p;
        ys[i] = (q0 + qq < batch && j < p) ? queries[uint64_t(q0 + qq) * padded_p + j] : 0.f;
    }
    float t[Q];
    uint32_t over[Q][R];
#pragma unroll
    for (int qq = 0; qq < Q; ++qq) {
        t[qq] = q0 + qq < batch
                    ? median_threshold(min_bits, query_err, q0 + qq, row_err_max, rel, abs_err)
                    : 0.f;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            over[qq][k] = 0;
        }
    }
    __syncthreads();
    // rows row0 + k * kCountRows (k < R): each broadcast
    // query value serves them all
    const uint32_t row0 = blockIdx.x * (kCountRows * R) + threadIdx.x;
    const float* col[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t row = row0 + k * kCountRows;
        col[k] = rows_t + (row < row_count ? row : 0);
    }
    const uint32_t p4 = p & ~3u;
    const uint32_t pitch4 = padded_p / 4;
    for (uint32_t j = 0; j < p4; j += 4) {
        float r[R][4];
#pragma unroll
        for (int k = 0; k < R; ++k) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                r[k][m] = col[k][uint64_t(j + m) * r_pitch];
            }
        }
#pragma unroll
        for (int qq = 0; qq < Q; ++qq) {
            const float4 y4 = ys4[qq * pitch4 + j / 4];
            const float y[4] = {y4.x, y4.y, y4.z, y4.w};
#pragma unroll
            for (int k = 0; k < R; ++k) {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    over[qq][k] +=
                        __float_as_uint(__fsub_rn(t[qq], fabsf(__fsub_rn(r[k][m], y[m])))) >> 31;
                }
            }
        }
    }
    for (uint32_t j = p4; j < p; ++j) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const float rv = col[k][uint64_t(j) * r_pitch];
#pragma unroll
            for (int qq = 0; qq < Q; ++qq) {
                over[qq][k] += __float_as_uint(__fsub_rn(
                                   t[qq], fabsf(__fsub_rn(rv, ys[qq * padded_p + j])))) >>
                               31;
            }
        }
    }
    const uint32_t needed = p % 2 != 0 ? p / 2 + 1 : p / 2;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t row = row0 + k * kCountRows;
        if (row >= row_count) {
            continue;
        }
#pragma unroll
        for (int qq = 0; qq < Q; ++qq) {
            if (q0 + qq < batch) {
                const bool pruned = t[qq] <= FLT_MAX && p - over[qq][k] < needed;
                partials[uint64_t(q0 + qq) * row_count + row] =
                    pruned ? -t[qq] : __uint_as_float(kSurvivorMark);
            }
        }
    }
}

// Stage 3: the binary32 median of every pair marked by the count, one warp
// per marked pair; warps take runs of 32 pairs and vote on their marks.
template <int PER_LANE>
__global__ void __launch_bounds__(kThreads)
    median_survivor_kernel(const float* __restrict__ rows, uint32_t row_count,
                           uint32_t padded_p, uint32_t p,
                           const float* __restrict__ queries, uint32_t batch,
                           const float* __restrict__ coord_err,
                           float* __restrict__ partials, float* __restrict__ pair_err)
{
    const int lane = threadIdx.x % 32;
    const uint64_t total = static_cast<uint64_t>(row_count) * batch;
    const uint64_t runs = (total + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
    for (uint64_t run = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 32;
         run < runs; run += stride) {
        const uint64_t mine = run * 32 + lane;
        const bool marked =
            mine < total && __float_as_uint(partials[mine]) == kSurvivorMark;
        uint32_t mask = __ballot_sync(0xffffffffu, marked);
        while (mask != 0) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1;
            const uint64_t pair = run * 32 + bit;
            const uint32_t q = static_cast<uint32_t>(pair / row_count);
            const uint32_t row = static_cast<uint32_t>(pair - uint64_t(q) * row_count);
            const float* r = rows + uint64_t(row) * padded_p;
            const float* y = queries + uint64_t(q) * padded_p;
            const float* ye = coord_err + uint64_t(q) * padded_p;
            float v[PER_LANE];
            float eps[PER_LANE];
            const int valid = load_abs_diffs<PER_LANE>(r, y, p, lane, v);
            // per coordinate: the row's binary32 rounding (at most 2^-24 |r|),
            // the query's projection error and the rounding of r - y
#pragma unroll
            for (int i = 0; i < PER_LANE; ++i) {
                const uint32_t j = lane + 32u * i;
                eps[i] = j < p ? __fadd_ru(__fadd_ru(__fmul_ru(fabsf(r[j]), 0x1p-24f), ye[j]),
                                           __fmul_ru(v[i], 0x1p-24f))
                               : 0.f;
            }
            float lower, upper;
            warp_middles<PER_LANE>(v, valid, p, lower, upper);
            const float median = p % 2 != 0 ? upper : lower + (upper - lower) * 0.5f;
            const float err = warp_middle_error<PER_LANE>(v, eps, valid, lower, upper);
            if (lane == 0) {
                partials[pair] = median;
                pair_err[pair] = err;
            }
        }
    }
}

__global__ void sum_slabs_kernel(const float* __restrict__ partials, uint32_t splits,
                                 uint64_t batch, uint64_t rows, float* __restrict__ out,
                                 uint64_t out_pitch)
{
    const uint64_t total = batch * out_pitch;
    const uint64_t slab = batch * rows;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         idx < total; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t q = idx / out_pitch;
        const uint64_t j = idx - q * out_pitch;
        float v = 0.f;
        if (j < rows) {
            for (uint32_t sp = 0; sp < splits; ++sp) {
                v += partials[sp * slab + q * rows + j];
            }
        }
        out[idx] = v;
    }
}

// One thread per (query, j), j fastest: the warp reads 32 consecutive
// coefficients of one transposed row and broadcasts the query value.
__global__ void project_queries64_kernel(const float* __restrict__ x, uint64_t batch,
                                         uint64_t padded_k, uint64_t k,
                                         const double* __restrict__ proj_t, uint64_t p,
                                         double* __restrict__ y, int* error_flag)
{
    const uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (idx >= batch * p) {
        return;
    }
    const uint64_t q = idx / p;
    const uint64_t j = idx - q * p;
    const float* xq = x + q * padded_k;
    double acc = 0.0;
    for (uint64_t i = 0; i < k; ++i) {
        acc = __dadd_rn(acc, __dmul_rn(static_cast<double>(xq[i]), proj_t[i * p + j]));
    }
    if (!isfinite(acc)) {
        atomicOr(error_flag, 4);
    }
    y[idx] = acc;
}

__global__ void transpose_rows_kernel(const float* __restrict__ rows, uint64_t row_count,
                                      uint64_t padded_p, float* __restrict__ out,
                                      uint64_t r_pitch)
{
    const uint64_t total = padded_p * r_pitch;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         idx < total; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t j = idx / r_pitch;
        const uint64_t row = idx - j * r_pitch;
        out[idx] = row < row_count ? rows[row * padded_p + j] : 0.f;
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

void launch_sum_slabs(const float* partials, uint32_t splits, uint64_t batch,
                      uint64_t rows, float* out, uint64_t out_pitch, cudaStream_t stream)
{
    sum_slabs_kernel<<<grid_for(batch * out_pitch), kThreads, 0, stream>>>(
        partials, splits, batch, rows, out, out_pitch);
    check_cuda(cudaGetLastError(), "cannot launch slab sum kernel");
}

void launch_project_queries64(const float* x, uint64_t batch, uint64_t padded_k,
                              uint64_t k, const double* proj_t, uint64_t p, double* y,
                              int* error_flag, cudaStream_t stream)
{
    const uint64_t threads = batch * p;
    project_queries64_kernel<<<static_cast<uint32_t>((threads + kThreads - 1) / kThreads),
                               kThreads, 0, stream>>>(x, batch, padded_k, k, proj_t, p, y,
                                                      error_flag);
    check_cuda(cudaGetLastError(), "cannot launch binary64 query projection kernel");
}

void launch_transpose_rows(const float* rows, uint64_t row_count, uint64_t padded_p,
                           float* out, uint64_t r_pitch, cudaStream_t stream)
{
    transpose_rows_kernel<<<grid_for(padded_p * r_pitch), kThreads, 0, stream>>>(
        rows, row_count, padded_p, out, r_pitch);
    check_cuda(cudaGetLastError(), "cannot launch row transpose kernel");
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
                            uint64_t padded_p, float* query_err, float* coord_err,
                            double err_per_abs, bool euclidean,
                            int* error_flag, cudaStream_t stream)
{
    check_cuda(cudaMemsetAsync(query_err, 0, batch * sizeof(float), stream),
               "cannot clear projection error");
    const dim3 grid(static_cast<uint32_t>((padded_p + kProjCols - 1) / kProjCols),
                    static_cast<uint32_t>((batch + kProjQueries - 1) / kProjQueries));
    project_queries_kernel<<<grid, kProjQueries * kProjCols, 0, stream>>>(
        gathered, batch, padded_k, k, proj32, p, out, padded_p, query_err, coord_err,
        err_per_abs, euclidean, error_flag);
    check_cuda(cudaGetLastError(), "cannot launch query projection kernel");
    finish_query_err_kernel<<<static_cast<uint32_t>((batch + kThreads - 1) / kThreads),
                              kThreads, 0, stream>>>(query_err, batch, euclidean);
    check_cuda(cudaGetLastError(), "cannot launch projection error kernel");
}

namespace {

// Rows whose exact medians set the pruning threshold: about sqrt(rows)
// (balancing these medians against the ~rows / samples survivors per
// query), in [32, 256] and at most the row count.
uint32_t median_samples(uint64_t row_count)
{
    uint64_t s = 32;
    while (s < 256 && s * s < row_count) {
        s += 32;
    }
    return static_cast<uint32_t>(row_count < s ? row_count : s);
}

template <int Q>
void launch_median_count(const float* rows_t, uint32_t r_pitch, uint32_t rc, uint32_t pp,
                         uint32_t pv, const float* queries, uint32_t b,
                         const unsigned int* min_bits, const float* query_err,
                         float row_err_max, float rel, float abs_err, float* partials,
                         cudaStream_t stream)
{
    // at most 8 x 1024 binary32 values: within the default 48 KB
    const size_t smem = static_cast<size_t>(Q) * pp * sizeof(float);
    // grid.y is limited to 65,535 query groups per launch
    const uint64_t groups = (static_cast<uint64_t>(b) + Q - 1) / Q;
    for (uint64_t g = 0; g < groups; g += 65535) {
        constexpr uint32_t per_cta = kCountRows * count_rows_per_thread<Q>();
        const dim3 grid((rc + per_cta - 1) / per_cta,
                        static_cast<uint32_t>(std::min<uint64_t>(65535, groups - g)));
        median_count_kernel<Q><<<grid, kCountRows, smem, stream>>>(
            rows_t, r_pitch, rc, pp, pv, queries, b, static_cast<uint32_t>(g * Q), min_bits,
            query_err, row_err_max, rel, abs_err, partials);
    }
}

template <int PER_LANE>
void launch_median_pair(const float* rows, const float* rows_t, uint32_t r_pitch,
                        uint32_t rc, uint32_t pp, uint32_t pv, const float* queries,
                        uint32_t b, const float* query_err, const float* coord_err,
                        float row_err_max, float rel, float abs_err,
                        unsigned int* min_bits, float* partials, float* pair_err,
                        cudaStream_t stream)
{
    // grid-stride warps over the pairs: at most 16 resident CTAs' worth per SM
    const uint64_t cap = 148ull * 16;
    const uint32_t samples = median_samples(rc);
    const uint64_t sample_blocks =
        (static_cast<uint64_t>(samples) * b * 32 + kThreads - 1) / kThreads;
    median_sample_kernel<PER_LANE>
        <<<static_cast<uint32_t>(std::min(sample_blocks, cap)), kThreads, 0, stream>>>(
            rows, rc, pp, pv, queries, b, samples, partials, min_bits);
    if (b >= 8) {
        launch_median_count<8>(rows_t, r_pitch, rc, pp, pv, queries, b, min_bits, query_err,
                               row_err_max, rel, abs_err, partials, stream);
    } else if (b >= 4) {
        launch_median_count<4>(rows_t, r_pitch, rc, pp, pv, queries, b, min_bits, query_err,
                               row_err_max, rel, abs_err, partials, stream);
    } else if (b >= 2) {
        launch_median_count<2>(rows_t, r_pitch, rc, pp, pv, queries, b, min_bits, query_err,
                               row_err_max, rel, abs_err, partials, stream);
    } else {
        launch_median_count<1>(rows_t, r_pitch, rc, pp, pv, queries, b, min_bits, query_err,
                               row_err_max, rel, abs_err, partials, stream);
    }
    const uint64_t runs = (static_cast<uint64_t>(rc) * b + 31) / 32;
    const uint64_t blocks = (runs * 32 + kThreads - 1) / kThreads;
    median_survivor_kernel<PER_LANE>
        <<<static_cast<uint32_t>(std::min(blocks, cap)), kThreads, 0, stream>>>(
            rows, rc, pp, pv, queries, b, coord_err, partials, pair_err);
}

}  // namespace

void launch_median_scan(const float* rows, const float* rows_t, uint64_t r_pitch,
                        uint64_t row_count, uint64_t padded_p,
                        uint64_t p, const float* queries, uint64_t batch,
                        const float* query_err, const float* coord_err,
                        float row_err_max, float rel,
                        float abs_err, unsigned int* min_bits, float* partials,
                        float* pair_err, cudaStream_t stream)
{
    const uint32_t rp = static_cast<uint32_t>(r_pitch);
    const uint32_t rc = static_cast<uint32_t>(row_count);
    const uint32_t pp = static_cast<uint32_t>(padded_p);
    const uint32_t pv = static_cast<uint32_t>(p);
    const uint32_t b = static_cast<uint32_t>(batch);
    check_cuda(cudaMemsetAsync(min_bits, 0xff, batch * sizeof(unsigned int), stream),
               "cannot clear median thresholds");
    if (p <= 32) {
        launch_median_pair<1>(rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 64) {
        launch_median_pair<2>(rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 128) {
        launch_median_pair<4>(rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 256) {
        launch_median_pair<8>(rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 512) {
        launch_median_pair<16>(rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 1024) {
        launch_median_pair<32>(rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else {
        fail(UHA_LENGTH_ERROR,
             "the L1 hierarchy supports projection dimensions up to 1024");
    }
    check_cuda(cudaGetLastError(), "cannot launch median scan kernel");
}

}  // namespace uha
