// Device code of the hierarchical query stages shared by the stage kernels
// (hierarchical.cu, prep.cu) and the persistent multi-index batch kernel
// (certify.cu): the gather of sampled coordinates, the binary32 query
// projection with its error bound, the warp selections of the median scan and
// its three stages, as block or grid-stride bodies with the block coordinates
// passed in.
#pragma once

#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>

#include "kernels.h"

namespace uha {
namespace hierbody {

// The gather of each query's sampled coordinates (scaled for L2) into the
// padded prepared layout, with the finiteness flags (prepare_sampled_kernel).
__device__ __forceinline__ void prepare_sampled_loop(
    const float* __restrict__ queries, uint64_t batch, uint64_t dim,
    const uint32_t* __restrict__ columns, const float* __restrict__ scales,
    uint64_t sample_size, float* __restrict__ out, uint64_t padded_dim, int* error_flag,
    uint32_t vx, uint32_t gx, uint32_t threads)
{
    const uint64_t total = batch * padded_dim;
    for (uint64_t idx = vx * static_cast<uint64_t>(threads) + threadIdx.x; idx < total;
         idx += static_cast<uint64_t>(gx) * threads) {
        const uint64_t b = idx / padded_dim;
        const uint64_t i = idx - b * padded_dim;
        float v = 0.f;
        if (i < sample_size) {
            v = queries[b * dim + columns[i]];
            if (!isfinite(v)) {
                atomicOr(error_flag, 1);
            }
            if (scales != nullptr) {
                v = __fmul_rn(v, scales[i]);
                if (!isfinite(v)) {
                    atomicOr(error_flag, 2);
                }
            }
        }
        out[idx] = v;
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
struct ProjShared {
    float sx[kProjQueries][kProjK];
    float sp[kProjCols][kProjK + 1];
};

__device__ __forceinline__ void project_queries_block(
    const float* __restrict__ x, uint64_t batch, uint64_t padded_k, uint64_t k,
    const float* __restrict__ proj, uint64_t p, float* __restrict__ y, uint64_t padded_p,
    float* __restrict__ err_acc, float* __restrict__ coord_err, double err_per_abs,
    bool euclidean, int* error_flag, uint32_t bx, uint32_t by, ProjShared& sh)
{
    auto& sx = sh.sx;
    auto& sp = sh.sp;
    const int jj = threadIdx.x % kProjCols;
    const int qq = threadIdx.x / kProjCols;
    const uint64_t j = bx * static_cast<uint64_t>(kProjCols) + jj;
    const uint64_t b = by * static_cast<uint64_t>(kProjQueries) + qq;
    float total = 0.f;
    float total_abs = 0.f;
    for (uint64_t k0 = 0; k0 < k; k0 += kProjK) {
        __syncthreads();
        for (int i = threadIdx.x; i < kProjQueries * kProjK; i += blockDim.x) {
            const int r = i / kProjK;
            const int c = i % kProjK;
            const uint64_t bb = by * static_cast<uint64_t>(kProjQueries) + r;
            sx[r][c] = (bb < batch && k0 + c < k) ? x[bb * padded_k + k0 + c] : 0.f;
        }
        for (int i = threadIdx.x; i < kProjCols * kProjK; i += blockDim.x) {
            const int r = i / kProjK;
            const int c = i % kProjK;
            const uint64_t jr = bx * static_cast<uint64_t>(kProjCols) + r;
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


__device__ __forceinline__ void finish_query_err_loop(float* err, uint64_t batch,
                                                      bool euclidean, uint32_t vx,
                                                      uint32_t gx, uint32_t threads)
{
    for (uint64_t b = vx * static_cast<uint64_t>(threads) + threadIdx.x; b < batch;
         b += static_cast<uint64_t>(gx) * threads) {
        if (euclidean) {
            // err holds a binary32 sum of squares, each term rounded up; the
            // rounding of up to 16384 additions stays below 1e-3 relative,
            // covered by the factor.
            err[b] = __fmul_ru(__fsqrt_ru(err[b]), 1.001f);
        }
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
__device__ __forceinline__ void median_sample_loop(
    const float* __restrict__ rows, uint32_t row_count, uint32_t padded_p, uint32_t p,
    const float* __restrict__ queries, uint32_t batch, uint32_t samples,
    float* __restrict__ partials, unsigned int* __restrict__ min_bits, uint32_t vx,
    uint32_t gx, uint32_t threads)
{
    const int lane = threadIdx.x % 32;
    const uint64_t total = static_cast<uint64_t>(samples) * batch;
    const uint64_t stride = static_cast<uint64_t>(gx) * (threads / 32);
    for (uint64_t w = (vx * static_cast<uint64_t>(threads) + threadIdx.x) / 32; w < total;
         w += stride) {
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

// Block (bx, by) of the count grid on threads tid < kCountRows that
// synchronise on barrier `bar` (bar 0 with a kCountRows-thread CTA is
// __syncthreads); ys4: Q x padded_p floats.
template <int Q>
__device__ __forceinline__ void median_count_block(
    const float* __restrict__ rows_t, uint32_t r_pitch, uint32_t row_count,
    uint32_t padded_p, uint32_t p, const float* __restrict__ queries, uint32_t batch,
    uint32_t q_begin, const unsigned int* __restrict__ min_bits,
    const float* __restrict__ query_err, float row_err_max, float rel, float abs_err,
    float* __restrict__ partials, uint32_t bx, uint32_t by, float4* ys4, uint32_t tid,
    uint32_t bar)
{
    constexpr int R = count_rows_per_thread<Q>();
    float* ys = reinterpret_cast<float*>(ys4);
    const uint32_t q0 = q_begin + by * Q;
    for (uint32_t i = tid; i < Q * padded_p; i += kCountRows) {
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
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(kCountRows) : "memory");
    // rows row0 + k * kCountRows (k < R): each broadcast
    // query value serves them all
    const uint32_t row0 = bx * (kCountRows * R) + tid;
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
__device__ __forceinline__ void median_survivor_loop(
    const float* __restrict__ rows, uint32_t row_count, uint32_t padded_p, uint32_t p,
    const float* __restrict__ queries, uint32_t batch, const float* __restrict__ coord_err,
    float* __restrict__ partials, float* __restrict__ pair_err, uint32_t vx, uint32_t gx,
    uint32_t threads)
{
    const int lane = threadIdx.x % 32;
    const uint64_t total = static_cast<uint64_t>(row_count) * batch;
    const uint64_t runs = (total + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gx) * (threads / 32);
    for (uint64_t run = (vx * static_cast<uint64_t>(threads) + threadIdx.x) / 32; run < runs;
         run += stride) {
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

}  // namespace hierbody
}  // namespace uha
