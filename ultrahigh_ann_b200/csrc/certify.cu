// Argmin with lowest-index tie-break, certified against the reference CPU.
//
// The reference CPU scans (src/core/dense_l2_scan_index.cpp:25-41,
// src/exact/l1/exact_l1_index.cpp:26-57,
// src/coordinate_sampling/sampled_coordinate_l1_ann_index.cpp:119-154) keep the
// first row with the smallest binary64 distance. The device computes binary32
// distances D with a known bound |D_cpu - D| <= rel * D + abs. Per query:
//   U* = min over rows of (D + err)            (an upper bound on the CPU min)
//   candidates = rows with D - err <= U*        (every row that can be the min)
// One candidate means the CPU's answer is known. Otherwise the candidates are
// re-scored by replaying the CPU's binary64 operation sequence (the same
// operations in the same order, no contraction) and the lexicographic minimum
// of (distance, row) is the CPU's argmin. The replay runs inside the argmin
// kernel, in the block that merges the query's summaries, so a query batch
// needs no host decision between its kernels.
#include "async_copy.cuh"
#include "common.h"
#include "exact64.h"
#include "hier_body.cuh"
#include "kernels.h"
#include "stage_bodies.h"
#include "tile_body.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

namespace uha {
namespace {

constexpr int kFinalizeThreads = 256;
constexpr int kArgminUnroll = 8;

struct Bounds2 {
    float lower;
    float upper;
};

// Bounds of a finite binary32 distance d given the row's error term e (row
// plus query error; median: the pair's own error for a computed median;
// unused in plain mode). Monotone: nondecreasing in d, nonincreasing in e.
__device__ __forceinline__ Bounds2 bound_with(float d, const Bound& b, float e)
{
    const float inf = __int_as_float(0x7f800000);
    if (b.mode == BoundMode::plain) {
        const float err = __fadd_ru(__fmul_ru(b.rel, d), b.abs);
        return {fmaxf(0.f, __fsub_rd(d, err)), __fadd_ru(d, err)};
    }
    if (b.mode == BoundMode::median) {
        if (d < 0.f) {
            // a row the median scan set aside: binary32 median at least -d
            const float t = -d;
            const float err = __fadd_ru(__fadd_ru(__fmul_ru(b.rel, t), e), b.abs);
            return {fmaxf(0.f, __fsub_rd(t, err)), inf};
        }
        const float err = __fadd_ru(__fadd_ru(__fmul_ru(b.rel, d), e), b.abs);
        return {fmaxf(0.f, __fsub_rd(d, err)), __fadd_ru(d, err)};
    }
    // projected_l2: ||a|| within e of ||b|| (triangle inequality on the
    // projected difference vectors)
    const float lo_root =
        fmaxf(0.f, __fsub_rd(__fsqrt_rd(__fmul_rd(d, __fsub_rd(1.f, b.rel))), e));
    const float hi_root =
        __fadd_ru(__fsqrt_ru(__fmul_ru(d, __fadd_ru(1.f, b.rel))), e);
    const float lo = __fmul_rd(__fmul_rd(lo_root, lo_root), __fsub_rd(1.f, b.cpu_rel));
    const float hi = __fmul_ru(__fmul_ru(hi_root, hi_root), __fadd_ru(1.f, b.cpu_rel));
    return {fmaxf(0.f, __fsub_rd(lo, b.abs)), __fadd_ru(hi, b.abs)};
}

__device__ __forceinline__ Bounds2 bound_of(float d, const Bound& b,
                                            uint32_t row, uint32_t q)
{
    if (!(d <= FLT_MAX)) {
        // binary32 overflow: no finite upper bound; every row below stays a
        // candidate and the replay decides
        return {0.f, __int_as_float(0x7f800000)};
    }
    if (b.mode == BoundMode::plain) {
        return bound_with(d, b, 0.f);
    }
    float e = __fadd_ru(b.row_err[row], b.query_err[q]);
    if (b.mode == BoundMode::median && d >= 0.f && b.pair_err != nullptr) {
        // a computed median: its own error bound
        e = b.pair_err[static_cast<uint64_t>(q) * b.pair_rows + row];
    }
    return bound_with(d, b, e);
}

// A lower bound valid for every row of query q whose binary32 distance is at
// least d (finite): the largest row error in place of the row's own.
__device__ __forceinline__ float lower_any(float d, const Bound& b, uint32_t q)
{
    const float e =
        b.mode == BoundMode::plain ? 0.f : __fadd_ru(b.row_err_max, b.query_err[q]);
    return bound_with(d, b, e).lower;
}

// Sum of the chunk partials of one (query, row) in chunk order. The loads are
// issued four at a time; the additions keep the sequential order, so finalize
// and resolve compute bit-identical distances.
__device__ __forceinline__ float row_distance(const PartialView& v, uint32_t q,
                                              uint32_t row)
{
    const uint64_t stride = static_cast<uint64_t>(v.batch) * v.rows;
    const float* p = v.partials + static_cast<uint64_t>(q) * v.rows + row;
    float d = 0.f;
    uint32_t c = 0;
    for (; c + 4 <= v.chunks; c += 4) {
        const float a0 = p[(c + 0) * stride];
        const float a1 = p[(c + 1) * stride];
        const float a2 = p[(c + 2) * stride];
        const float a3 = p[(c + 3) * stride];
        d += a0;
        d += a1;
        d += a2;
        d += a3;
    }
    for (; c < v.chunks; ++c) {
        d += p[c * stride];
    }
    return d;
}

// Two smallest lower bounds (with the row of the smallest) and the smallest
// upper bound seen by a thread / warp / block.
struct Summary {
    float min_upper;
    float first;
    float second;
    uint32_t first_row;
    float first_distance;
};

__device__ __forceinline__ void summary_insert(Summary& s, float lower,
                                               float upper, uint32_t row,
                                               float distance)
{
    s.min_upper = fminf(s.min_upper, upper);
    if (lower < s.first || (lower == s.first && row < s.first_row)) {
        s.second = s.first;
        s.first = lower;
        s.first_row = row;
        s.first_distance = distance;
    } else if (lower < s.second) {
        s.second = lower;
    }
}

__device__ __forceinline__ Summary summary_merge(const Summary& a,
                                                 const Summary& b)
{
    Summary r;
    r.min_upper = fminf(a.min_upper, b.min_upper);
    const bool a_first =
        a.first < b.first || (a.first == b.first && a.first_row < b.first_row);
    const Summary& lo = a_first ? a : b;
    const Summary& hi = a_first ? b : a;
    r.first = lo.first;
    r.first_row = lo.first_row;
    r.first_distance = lo.first_distance;
    r.second = fminf(lo.second, hi.first);
    return r;
}

__device__ __forceinline__ Summary shfl_summary(const Summary& s, int offset)
{
    Summary o;
    o.min_upper = __shfl_xor_sync(0xffffffffu, s.min_upper, offset);
    o.first = __shfl_xor_sync(0xffffffffu, s.first, offset);
    o.second = __shfl_xor_sync(0xffffffffu, s.second, offset);
    o.first_row = __shfl_xor_sync(0xffffffffu, s.first_row, offset);
    o.first_distance = __shfl_xor_sync(0xffffffffu, s.first_distance, offset);
    return o;
}

__device__ Summary block_reduce_summary(Summary s)
{
    const float inf = __int_as_float(0x7f800000);
    for (int offset = 16; offset > 0; offset /= 2) {
        s = summary_merge(s, shfl_summary(s, offset));
    }
    __shared__ Summary warp_summaries[kFinalizeThreads / 32];
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    __syncthreads();
    if (lane == 0) {
        warp_summaries[warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
        s = lane < kFinalizeThreads / 32
                ? warp_summaries[lane]
                : Summary{inf, inf, inf, 0xffffffffu, inf};
        for (int offset = 16; offset > 0; offset /= 2) {
            s = summary_merge(s, shfl_summary(s, offset));
        }
    }
    return s;  // valid in thread 0
}

__device__ __forceinline__ unsigned int ordered_bits(float f)
{
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(kFinalizeThreads)
    finalize_gemm_kernel(PartialView view, const float* row_norms,
                         const float* query_norms, Result* results)
{
    const uint32_t q = blockIdx.x;
    const float qn = query_norms[q];
    unsigned long long best = ~0ull;
    for (uint32_t row = threadIdx.x; row < view.rows; row += blockDim.x) {
        const float dot = row_distance(view, q, row);
        const float d =
            __fsub_rn(__fadd_rn(row_norms[row], qn), __fmul_rn(2.0f, dot));
        const unsigned long long key =
            (static_cast<unsigned long long>(ordered_bits(d)) << 32) | row;
        best = key < best ? key : best;
    }
    for (int offset = 16; offset > 0; offset /= 2) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, offset);
        best = o < best ? o : best;
    }
    __shared__ unsigned long long warp_best[kFinalizeThreads / 32];
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (lane == 0) {
        warp_best[warp] = best;
    }
    __syncthreads();
    if (warp == 0) {
        best = lane < kFinalizeThreads / 32 ? warp_best[lane] : ~0ull;
        for (int offset = 16; offset > 0; offset /= 2) {
            const unsigned long long o =
                __shfl_xor_sync(0xffffffffu, best, offset);
            best = o < best ? o : best;
        }
        if (lane == 0) {
            const unsigned int bits = static_cast<unsigned int>(best >> 32);
            const unsigned int raw =
                (bits & 0x80000000u) ? (bits & 0x7fffffffu) : ~bits;
            results[q] = Result{static_cast<uint32_t>(best & 0xffffffffu),
                                __uint_as_float(raw)};
        }
    }
}

// Reference CPU distance of one row, replayed by one warp. Every lane ends
// with the same value. Terms are formed in parallel; the additions are applied
// in the CPU's order through warp broadcasts.
__device__ double replay_row(const ReplayInputs& in, const float* qrow,
                             const float* rrow, int lane)
{
    double s = 0.0;
    if (in.op == ReplayOp::l1_grouped4) {
        // std::transform_reduce over random-access ranges (libstdc++ <numeric>):
        // init += ((t0 + t1) + (t2 + t3)) per full group of four, then the
        // remaining terms one by one.
        const uint64_t groups = in.dim / 4;
        for (uint64_t base = 0; base < groups; base += 32) {
            const uint64_t g = base + lane;
            double v3 = 0.0;
            if (g < groups) {
                const uint64_t i = 4 * g;
                const double t0 = fabs(__dsub_rn(qrow[i], rrow[i]));
                const double t1 = fabs(__dsub_rn(qrow[i + 1], rrow[i + 1]));
                const double t2 = fabs(__dsub_rn(qrow[i + 2], rrow[i + 2]));
                const double t3 = fabs(__dsub_rn(qrow[i + 3], rrow[i + 3]));
                v3 = __dadd_rn(__dadd_rn(t0, t1), __dadd_rn(t2, t3));
            }
            const uint64_t n = groups - base < 32 ? groups - base : 32;
            for (uint64_t j = 0; j < n; ++j) {
                s = __dadd_rn(s, __shfl_sync(0xffffffffu, v3, static_cast<int>(j)));
            }
        }
        for (uint64_t i = 4 * groups; i < in.dim; ++i) {
            s = __dadd_rn(s, fabs(__dsub_rn(qrow[i], rrow[i])));
        }
        return s;
    }
    for (uint64_t base = 0; base < in.dim; base += 32) {
        const uint64_t i = base + lane;
        double t = 0.0;
        if (i < in.dim) {
            const double diff =
                __dsub_rn(static_cast<double>(qrow[i]), static_cast<double>(rrow[i]));
            if (in.op == ReplayOp::l2_sequential) {
                t = __dmul_rn(diff, diff);
            } else {
                t = __dmul_rn(in.weights64[i], fabs(diff));
            }
        }
        const uint64_t n = in.dim - base < 32 ? in.dim - base : 32;
        for (uint64_t j = 0; j < n; ++j) {
            s = __dadd_rn(s, __shfl_sync(0xffffffffu, t, static_cast<int>(j)));
        }
    }
    return s;
}

// Reference binary64 squared distance between a projected row and the
// projected query (hierarchical_l2_ann_index.cpp:63-77): s += (r_j - y_j)^2
// in j order.
__device__ double replay_projected_l2(const double* row, const double* y,
                                      uint64_t p, int lane)
{
    double s = 0.0;
    for (uint64_t base = 0; base < p; base += 32) {
        const uint64_t j = base + lane;
        double t = 0.0;
        if (j < p) {
            const double diff = __dsub_rn(row[j], y[j]);
            t = __dmul_rn(diff, diff);
        }
        const uint64_t n = p - base < 32 ? p - base : 32;
        for (uint64_t i = 0; i < n; ++i) {
            s = __dadd_rn(s, __shfl_sync(0xffffffffu, t, static_cast<int>(i)));
        }
    }
    return s;
}

// Number of j < p with |row_j - y_j| (as binary64 bits) below `bound`.
__device__ uint32_t count_below(const double* row, const double* y, uint64_t p,
                                unsigned long long bound, int lane)
{
    uint32_t c = 0;
    for (uint64_t j = lane; j < p; j += 32) {
        const unsigned long long bits = static_cast<unsigned long long>(
            __double_as_longlong(fabs(__dsub_rn(row[j], y[j]))));
        c += bits < bound ? 1u : 0u;
    }
    return __reduce_add_sync(0xffffffffu, c);
}

// The k-th smallest (0-based) |row_j - y_j|: binary search on the bit pattern
// (nonnegative binary64 values order like their bits).
__device__ double select_abs_diff(const double* row, const double* y,
                                  uint64_t p, uint32_t k, int lane)
{
    unsigned long long prefix = 0;
    for (int bit = 62; bit >= 0; --bit) {
        const unsigned long long trial = prefix | (1ull << bit);
        if (count_below(row, y, p, trial, lane) <= k) {
            prefix = trial;
        }
    }
    return __longlong_as_double(static_cast<long long>(prefix));
}

// Reference median of |r_j - y_j| with the even-p midpoint
// (hierarchical_l1_ann_index.cpp:65-99): nth_element puts the (p/2)-th
// smallest at the upper middle; the lower middle is the largest of the
// smaller half; median = lower + (upper - lower) * 0.5.
__device__ double replay_median(const double* row, const double* y, uint64_t p,
                                int lane)
{
    const uint32_t mid = static_cast<uint32_t>(p / 2);
    const double upper = select_abs_diff(row, y, p, mid, lane);
    if (p % 2 != 0) {
        return upper;
    }
    const double lower = select_abs_diff(row, y, p, mid - 1, lane);
    return __dadd_rn(lower, __dmul_rn(__dsub_rn(upper, lower), 0.5));
}

__device__ __forceinline__ bool lex_less(double a, uint32_t ar, double b,
                                         uint32_t br)
{
    return a < b || (a == b && ar < br);
}

// Reference binary64 query projection (l2_hierarchical_projection.cpp:186-198)
// into `y`: y_j = sum_i double(x_i) * P[j][i] in i order, one thread per j.
__device__ void project_query64(const ReplayInputs& in, const float* x, double* y)
{
    for (uint64_t j = threadIdx.x; j < in.proj_dim; j += blockDim.x) {
        const double* coeff = in.projection64 + j * in.dim;
        double acc = 0.0;
        for (uint64_t i = 0; i < in.dim; ++i) {
            acc = __dadd_rn(acc, __dmul_rn(static_cast<double>(x[i]), coeff[i]));
        }
        y[j] = acc;
    }
}

__host__ __device__ __forceinline__ bool projected_op(ReplayOp op)
{
    return op == ReplayOp::l2_projected || op == ReplayOp::median_projected;
}

// Reference distance of one candidate row, replayed by one warp.
__device__ double replay_candidate(const ReplayInputs& in, const float* qrow,
                                   const double* y, uint32_t row, int lane)
{
    if (in.op == ReplayOp::l2_projected) {
        return replay_projected_l2(in.rows64 + uint64_t(row) * in.proj_dim, y,
                                   in.proj_dim, lane);
    }
    if (in.op == ReplayOp::median_projected) {
        return replay_median(in.rows64 + uint64_t(row) * in.proj_dim, y,
                             in.proj_dim, lane);
    }
    return replay_row(in, qrow, in.rows + uint64_t(row) * in.padded_dim, lane);
}

// ------------------------------------------ replay without the FP64 units

// Float-float distance of one candidate row, evaluated by one warp: each
// lane forms the terms i = lane, lane + 32, ... (the L2 and weighted-L1 terms
// within 2^-45 relative, the L1 terms exactly) and adds them in float-float,
// then a butterfly adds the lanes (ff_add is commutative, so every lane ends
// with the same value).
__device__ x64::FF ff_row(const ReplayInputs& in, const float* qrow, const float* rrow,
                          int lane)
{
    x64::FF s{0.f, 0.f};
    for (uint64_t i = lane; i < in.dim; i += 32) {
        x64::FF d = x64::two_sum(qrow[i], -rrow[i]);  // q - r exactly
        x64::FF t;
        if (in.op == ReplayOp::l2_sequential) {
            const x64::FF p = x64::two_prod(d.hi, d.hi);
            const float cross = __fmul_rn(__fmul_rn(2.f, d.hi), d.lo);
            t = x64::two_sum(p.hi, __fadd_rn(p.lo, cross));
        } else {
            if (d.hi < 0.f) {
                d = x64::FF{-d.hi, -d.lo};
            }
            t = d;
            if (in.op == ReplayOp::l1_weighted_sequential) {
                const float wh = in.weights_ff[2 * i];
                const float wl = in.weights_ff[2 * i + 1];
                const x64::FF p = x64::two_prod(wh, d.hi);
                const float c = __fmaf_rn(wh, d.lo, __fmul_rn(wl, d.hi));
                t = x64::two_sum(p.hi, __fadd_rn(p.lo, c));
            }
        }
        s = x64::ff_add(s, t);
    }
    for (int o = 16; o > 0; o /= 2) {
        const x64::FF other{__shfl_xor_sync(0xffffffffu, s.hi, o),
                            __shfl_xor_sync(0xffffffffu, s.lo, o)};
        s = x64::ff_add(s, other);
    }
    return s;
}

// The reference CPU's binary64 distance of one row, bit for bit, in emulated
// binary64 (the operations and order of replay_row). Every lane returns it.
__device__ uint64_t x64_row(const ReplayInputs& in, const float* qrow, const float* rrow,
                            int lane)
{
    uint64_t s = 0;
    if (in.op == ReplayOp::l1_grouped4) {
        const uint64_t groups = in.dim / 4;
        for (uint64_t base = 0; base < groups; base += 32) {
            const uint64_t g = base + lane;
            uint64_t v3 = 0;
            if (g < groups) {
                const uint64_t i = 4 * g;
                uint64_t t[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    t[e] = x64::sub(x64::from_float(qrow[i + e]), x64::from_float(rrow[i + e])) &
                           ~x64::kSignBit;
                }
                v3 = x64::add(x64::add(t[0], t[1]), x64::add(t[2], t[3]));
            }
            const uint64_t n = groups - base < 32 ? groups - base : 32;
            for (uint64_t j = 0; j < n; ++j) {
                s = x64::add(s, __shfl_sync(0xffffffffu, v3, static_cast<int>(j)));
            }
        }
        for (uint64_t i = 4 * groups; i < in.dim; ++i) {
            s = x64::add(s, x64::sub(x64::from_float(qrow[i]), x64::from_float(rrow[i])) &
                                ~x64::kSignBit);
        }
        return s;
    }
    const uint64_t* w64 = reinterpret_cast<const uint64_t*>(in.weights64);
    for (uint64_t base = 0; base < in.dim; base += 32) {
        const uint64_t i = base + lane;
        uint64_t t = 0;
        if (i < in.dim) {
            const uint64_t d = x64::sub(x64::from_float(qrow[i]), x64::from_float(rrow[i]));
            t = in.op == ReplayOp::l2_sequential ? x64::mul(d, d)
                                                 : x64::mul(w64[i], d & ~x64::kSignBit);
        }
        const uint64_t n = in.dim - base < 32 ? in.dim - base : 32;
        for (uint64_t j = 0; j < n; ++j) {
            s = x64::add(s, __shfl_sync(0xffffffffu, t, static_cast<int>(j)));
        }
    }
    return s;
}

constexpr uint32_t kResolveCap = 512;

struct ResolveSmem {
    uint32_t row[kResolveCap];
    float hi[kResolveCap];
    float lo[kResolveCap];
    float delta[kResolveCap];
    unsigned char replay[kResolveCap];
    uint32_t count;
    uint32_t winner;
    uint32_t unseparated;
};

__device__ __forceinline__ void resolve_begin(ResolveSmem& sm)
{
    if (threadIdx.x == 0) {
        sm.count = 0;
    }
    __syncthreads();
}

// Appends a candidate row (any thread); false when the list is full.
__device__ __forceinline__ bool resolve_push(ResolveSmem& sm, uint32_t row)
{
    const uint32_t slot = atomicAdd(&sm.count, 1u);
    if (slot < kResolveCap) {
        sm.row[slot] = row;
        return true;
    }
    return false;
}

__device__ __forceinline__ void lex_update_bits(unsigned long long& best, uint32_t& best_row,
                                                unsigned long long bits, uint32_t row)
{
    if (bits < best || (bits == best && row < best_row)) {
        best = bits;
        best_row = row;
    }
}

// The block's lexicographic minimum of the warps' (binary64 bits, row), all
// distances nonnegative (their bits order like the values), into the result.
__device__ void resolve_finish(unsigned long long best, uint32_t best_row, Result* result,
                               double* exact_distance)
{
    constexpr int warps = kFinalizeThreads / 32;
    __shared__ unsigned long long warp_bits[warps];
    __shared__ uint32_t warp_rows[warps];
    if (threadIdx.x % 32 == 0) {
        warp_bits[threadIdx.x / 32] = best;
        warp_rows[threadIdx.x / 32] = best_row;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int v = 0; v < warps; ++v) {
            lex_update_bits(best, best_row, warp_bits[v], warp_rows[v]);
        }
        *result = Result{best_row, x64::to_float(best)};
        *exact_distance = __longlong_as_double(static_cast<long long>(best));
    }
}

// Block-wide: the reference CPU's argmin among the listed candidate rows of
// one query (every one of which may hold the minimum), without FP64
// instructions. (1) Float-float distance S_i of every candidate; the
// reference's value lies within delta_i = ff_rel S_i + ff_abs of it. (2) The
// candidate i* with the smallest S_i + delta_i wins outright when every other
// candidate j is separated: a lower bound of S_j - S_i* exceeds
// delta_j + delta_i*, so the reference's distance of j is larger. (3)
// Otherwise i* and the candidates not separated from it are replayed in
// emulated binary64 and the lexicographic minimum of (distance, row) wins.
// When the list overflowed (more than kResolveCap candidates), every row for
// which `is_candidate` holds is replayed in emulated binary64 instead.
// Writes results[q] / exact_distances[q] (binary64 bits of the distance).
template <typename IsCandidate>
__device__ void resolve_without_fp64(const ReplayInputs& in, const float* qrow,
                                     ResolveSmem& sm, uint32_t row_count,
                                     IsCandidate is_candidate, Result* result,
                                     double* exact_distance)
{
    constexpr int warps = kFinalizeThreads / 32;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    __syncthreads();
    const uint32_t n = sm.count;
    unsigned long long best = ~0ull;
    uint32_t best_row = 0xffffffffu;
    if (n > kResolveCap) {
        for (uint32_t base = warp * 32; base < row_count; base += warps * 32) {
            const uint32_t r = base + lane;
            unsigned int mask = __ballot_sync(0xffffffffu, r < row_count && is_candidate(r));
            while (mask != 0u) {
                const int bit = __ffs(mask) - 1;
                mask &= mask - 1u;
                const uint32_t crow = base + bit;
                lex_update_bits(best, best_row,
                                x64_row(in, qrow, in.rows + uint64_t(crow) * in.padded_dim,
                                        lane),
                                crow);
            }
        }
        resolve_finish(best, best_row, result, exact_distance);
        return;
    }
    for (uint32_t i = warp; i < n; i += warps) {
        const x64::FF s = ff_row(in, qrow, in.rows + uint64_t(sm.row[i]) * in.padded_dim, lane);
        if (lane == 0) {
            sm.hi[i] = s.hi;
            sm.lo[i] = s.lo;
            sm.delta[i] = __fadd_ru(__fmul_ru(in.ff_rel, __fmul_ru(fabsf(s.hi), 1.0000002f)),
                                    in.ff_abs);
            sm.replay[i] = 0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // any choice of i* is valid; the smallest approximate upper end makes
        // separation likely
        uint32_t w = 0;
        for (uint32_t i = 1; i < n; ++i) {
            const float ui = __fadd_ru(sm.hi[i], sm.delta[i]);
            const float uw = __fadd_ru(sm.hi[w], sm.delta[w]);
            if (ui < uw || (ui == uw && sm.row[i] < sm.row[w])) {
                w = i;
            }
        }
        sm.winner = w;
        sm.unseparated = 0;
        sm.replay[w] = 1;
    }
    __syncthreads();
    const uint32_t w = sm.winner;
    for (uint32_t j = threadIdx.x; j < n; j += kFinalizeThreads) {
        if (j == w) {
            continue;
        }
        // lower bound of S_j - S_w: exact difference of the high parts, the
        // rest rounded down (a NaN from overflowed sums fails the test)
        const x64::FF a = x64::two_sum(sm.hi[j], -sm.hi[w]);
        const float lower =
            __fadd_rd(a.hi, __fadd_rd(a.lo, __fsub_rd(sm.lo[j], sm.lo[w])));
        if (!(lower > __fadd_ru(sm.delta[j], sm.delta[w]))) {
            sm.replay[j] = 1;
            atomicAdd(&sm.unseparated, 1u);
        }
    }
    __syncthreads();
    if (sm.unseparated == 0) {
        if (threadIdx.x == 0) {
            const uint64_t bits = x64::add(x64::from_float(sm.hi[w]), x64::from_float(sm.lo[w]));
            *result = Result{sm.row[w], x64::to_float(bits)};
            *exact_distance = __longlong_as_double(static_cast<long long>(bits));
        }
        return;
    }
    for (uint32_t i = warp; i < n; i += warps) {
        if (sm.replay[i]) {
            const uint32_t r = sm.row[i];
            lex_update_bits(best, best_row,
                            x64_row(in, qrow, in.rows + uint64_t(r) * in.padded_dim, lane), r);
        }
    }
    resolve_finish(best, best_row, result, exact_distance);
}

// One block per query: each warp re-scores candidates by the reference's
// binary64 squared distance in the projected space (j order); the block keeps
// the lexicographic minimum of (distance, row).
__global__ void __launch_bounds__(kFinalizeThreads)
    rescore_projected_kernel(const uint32_t* __restrict__ candidates, uint32_t k,
                             const double* __restrict__ rows64,
                             const double* __restrict__ y64, uint32_t p, Result* results,
                             double* exact_distances)
{
    constexpr int warps = kFinalizeThreads / 32;
    const uint32_t q = blockIdx.x;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const double* y = y64 + static_cast<uint64_t>(q) * p;
    double best = __longlong_as_double(0x7ff0000000000000ll);
    uint32_t best_row = 0xffffffffu;
    for (uint32_t i = warp; i < k; i += warps) {
        const uint32_t row = candidates[static_cast<uint64_t>(q) * k + i];
        if (row == 0xffffffffu) {
            continue;
        }
        const double d = replay_projected_l2(rows64 + static_cast<uint64_t>(row) * p, y, p,
                                             lane);
        if (lex_less(d, row, best, best_row)) {
            best = d;
            best_row = row;
        }
    }
    __shared__ double warp_best[warps];
    __shared__ uint32_t warp_row[warps];
    if (lane == 0) {
        warp_best[warp] = best;
        warp_row[warp] = best_row;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < warps; ++w) {
            if (lex_less(warp_best[w], warp_row[w], best, best_row)) {
                best = warp_best[w];
                best_row = warp_row[w];
            }
        }
        results[q] = Result{best_row, static_cast<float>(best)};
        exact_distances[q] = best;
    }
}

// One thread's pass over its rows of a query in the argmin kernel.
struct RowScan {
    float k1 = __builtin_huge_valf();  // smallest distance
    float k2 = __builtin_huge_valf();  // second smallest
    uint32_t r1 = 0xffffffffu;              // row of k1 (lowest on ties)
    float set_aside = __builtin_huge_valf();  // median: smallest -d < 0
    bool overflow = false;
};

template <bool kSingleChunk>
__device__ __forceinline__ float load_distance(const PartialView& v, uint32_t q, uint32_t row)
{
    if constexpr (kSingleChunk) {
        return v.partials[static_cast<uint64_t>(q) * v.rows + row];
    } else {
        return row_distance(v, q, row);
    }
}

// One row of a thread's keyed scan (plain and projected bounds): binary32
// overflow (inf or NaN) sets the flag, any other distance updates the two
// smallest (the first row keeps a tie: rows arrive in increasing order).
__device__ __forceinline__ void scan_keyed_row(RowScan& scan, float x, uint32_t row)
{
    if (!(x <= FLT_MAX)) {
        scan.overflow = true;
    } else if (x < scan.k1) {
        scan.k2 = scan.k1;
        scan.k1 = x;
        scan.r1 = row;
    } else if (x < scan.k2) {
        scan.k2 = x;
    }
}

// One full step of kArgminUnroll keyed distances (rows base, base +
// kFinalizeThreads, ...) into a thread's two smallest: when the distances are
// finite (their sum is), the step's smallest m and second smallest s2 (with
// multiplicity) by min / max and one merge, the row of m (its first
// occurrence) looked up only when m is a new smallest; otherwise row by row.
// Equal to scan_keyed_row applied to the rows in order.
__device__ __forceinline__ void merge_step(RowScan& scan, const float* d, uint32_t base)
{
    float sum = d[0];
#pragma unroll
    for (int u = 1; u < kArgminUnroll; ++u) {
        sum += d[u];
    }
    if (fabsf(sum) <= FLT_MAX) {
        float m = d[0];
        float s2 = __int_as_float(0x7f800000);
#pragma unroll
        for (int u = 1; u < kArgminUnroll; ++u) {
            s2 = fminf(s2, fmaxf(m, d[u]));
            m = fminf(m, d[u]);
        }
        if (m < scan.k1) {
            // the first row holding m, and its own value (m's sign of zero
            // may differ)
            uint32_t first = kArgminUnroll - 1;
            float value = d[kArgminUnroll - 1];
#pragma unroll
            for (int u = kArgminUnroll - 2; u >= 0; --u) {
                const bool hit = d[u] == m;
                first = hit ? u : first;
                value = hit ? d[u] : value;
            }
            scan.k2 = fminf(scan.k1, s2);
            scan.k1 = value;
            scan.r1 = base + first * kFinalizeThreads;
        } else {
            scan.k2 = fminf(scan.k2, m);
        }
    } else {
#pragma unroll
        for (int u = 0; u < kArgminUnroll; ++u) {
            scan_keyed_row(scan, d[u], base + u * kFinalizeThreads);
        }
    }
}

// One median-mode distance of a thread's scan: overflow sets the flag, a row
// the median scan set aside (-T) joins the shared lower bound, a computed
// median is inserted with its own bounds.
__device__ __forceinline__ void scan_median_row(RowScan& scan, Summary& s, float x,
                                                const Bound& bound, uint32_t row, uint32_t q)
{
    if (!(x <= FLT_MAX)) {
        scan.overflow = true;
    } else if (x < 0.f) {
        scan.set_aside = fminf(scan.set_aside, -x);
    } else {
        const Bounds2 b = bound_of(x, bound, row, q);
        summary_insert(s, b.lower, b.upper, row, x);
    }
}

// One full step of kArgminUnroll median-mode distances: when all are rows set
// aside (finite and negative: their sum finite, their maximum negative), one
// minimum into the shared lower bound; otherwise row by row. Equal to
// scan_median_row applied to the rows in order.
__device__ __forceinline__ void merge_step_median(RowScan& scan, Summary& s, const float* d,
                                                  const Bound& bound, uint32_t base, uint32_t q)
{
    float sum = d[0];
    float mx = d[0];
#pragma unroll
    for (int u = 1; u < kArgminUnroll; ++u) {
        sum += d[u];
        mx = fmaxf(mx, d[u]);
    }
    if (fabsf(sum) <= FLT_MAX && mx < 0.f) {
        scan.set_aside = fminf(scan.set_aside, -mx);
    } else {
#pragma unroll
        for (int u = 0; u < kArgminUnroll; ++u) {
            scan_median_row(scan, s, d[u], bound, base + u * kFinalizeThreads, q);
        }
    }
}

// kArgminUnroll rows per thread per step, their loads issued together (with
// one partial slab the load is a single instruction the compiler can batch).
// Full steps go by merge_step (keyed bounds; two steps' loads, 16 rows, in
// flight while two whole steps remain) or merge_step_median; the last,
// partial step, and every step when !kStepMerge (the persistent kernel's
// register budget), go row by row.
template <bool kSingleChunk, bool kStepMerge>
__device__ __forceinline__ void scan_rows(const PartialView& view, const Bound& bound,
                                          uint32_t q, uint32_t first_row, uint32_t end_row,
                                          RowScan& scan, Summary& s)
{
    const bool keyed = bound.mode != BoundMode::median;
    auto merge = [&](const float* d, uint32_t at) {
        if (keyed) {
            merge_step(scan, d, at);
        } else {
            merge_step_median(scan, s, d, bound, at, q);
        }
    };
    uint32_t base = first_row + threadIdx.x;
    if (kStepMerge && keyed) {
        for (; base + (2 * kArgminUnroll - 1) * kFinalizeThreads < end_row;
             base += 2 * kFinalizeThreads * kArgminUnroll) {
            float d[2 * kArgminUnroll];
#pragma unroll
            for (int u = 0; u < 2 * kArgminUnroll; ++u) {
                d[u] = load_distance<kSingleChunk>(view, q, base + u * kFinalizeThreads);
            }
            merge_step(scan, d, base);
            merge_step(scan, d + kArgminUnroll, base + kArgminUnroll * kFinalizeThreads);
        }
    }
    for (; base < end_row; base += kFinalizeThreads * kArgminUnroll) {
        if (kStepMerge && base + (kArgminUnroll - 1) * kFinalizeThreads < end_row) {
            float d[kArgminUnroll];
#pragma unroll
            for (int u = 0; u < kArgminUnroll; ++u) {
                d[u] = load_distance<kSingleChunk>(view, q, base + u * kFinalizeThreads);
            }
            merge(d, base);
            continue;
        }
        float d[kArgminUnroll];
#pragma unroll
        for (int u = 0; u < kArgminUnroll; ++u) {
            const uint32_t row = base + u * kFinalizeThreads;
            d[u] = row < end_row ? load_distance<kSingleChunk>(view, q, row) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kArgminUnroll; ++u) {
            const uint32_t row = base + u * kFinalizeThreads;
            if (row >= end_row) {
                continue;
            }
            const float x = d[u];
            if (!(x <= FLT_MAX)) {
                scan.overflow = true;
            } else if (keyed) {
                if (x < scan.k1) {
                    scan.k2 = scan.k1;
                    scan.k1 = x;
                    scan.r1 = row;
                } else if (x < scan.k2) {
                    scan.k2 = x;
                }
            } else if (x < 0.f) {
                scan.set_aside = fminf(scan.set_aside, -x);
            } else {
                const Bounds2 b = bound_of(x, bound, row, q);
                summary_insert(s, b.lower, b.upper, row, x);
            }
        }
    }
}

// grid = (row blocks, batch). Every CTA summarises kFinalizeThreads rows of
// one query; the last CTA of the query to finish merges the summaries. A
// certified query is answered there; otherwise the same CTA replays every
// candidate row (D - err <= U*) in binary64, one warp per candidate, and keeps
// the lexicographic minimum of (distance, row). exact_distances[q] is the
// replayed distance, or NaN when the query was certified.
template <bool kEmulated, bool kStepMerge = true>
__device__ __forceinline__ void argmin_block(const PartialView& view, const Bound& bound,
                                             const ReplayInputs& in, Result* results,
                                             double* exact_distances,
                                             Summary* block_summaries, uint32_t* done,
                                             uint32_t* replay_count, uint32_t span,
                                             uint32_t bx, uint32_t by, uint32_t gx,
                                             double* projected_query)
{
    const uint32_t q = by;
    const uint32_t blocks = gx;
    const float inf = __int_as_float(0x7f800000);
    Summary s{inf, inf, inf, 0xffffffffu, inf};
    const uint32_t first_row = bx * span;
    const uint32_t end_row = min(view.rows, first_row + span);
    // Plain and projected_l2 bounds are monotone in d, so a thread keeps only
    // its smallest distance (lowest row on ties) and its second smallest; the
    // bounds are formed once, from the best row's own error and, for all its
    // other rows, the largest row error. Median rows set aside by the scan
    // share one lower bound; computed medians (few) are inserted with their
    // own bounds. Binary32 overflows enter as a lower bound of 0.
    RowScan scan;
    if (view.chunks == 1) {
        scan_rows<true, kStepMerge>(view, bound, q, first_row, end_row, scan, s);
    } else {
        scan_rows<false, kStepMerge>(view, bound, q, first_row, end_row, scan, s);
    }
    if (bound.mode != BoundMode::median && scan.r1 != 0xffffffffu) {
        const Bounds2 b1 = bound_of(scan.k1, bound, scan.r1, q);
        s = Summary{b1.upper, b1.lower,
                    scan.k2 <= FLT_MAX ? lower_any(scan.k2, bound, q) : inf, scan.r1,
                    scan.k1};
    }
    if (scan.set_aside <= FLT_MAX) {
        summary_insert(s, lower_any(-scan.set_aside, bound, q), inf, 0xffffffffu,
                       -scan.set_aside);
    }
    if (scan.overflow) {
        summary_insert(s, 0.f, inf, 0xffffffffu, inf);
    }
    s = block_reduce_summary(s);
    __shared__ bool is_last;
    if (blocks > 1) {
        if (threadIdx.x == 0) {
            block_summaries[static_cast<uint64_t>(q) * blocks + bx] = s;
            __threadfence();
            is_last = atomicAdd(done + q, 1u) == blocks - 1;
        }
        __syncthreads();
        if (!is_last) {
            return;
        }
        __threadfence();
        Summary m{inf, inf, inf, 0xffffffffu, inf};
        for (uint32_t i = threadIdx.x; i < blocks; i += kFinalizeThreads) {
            const volatile Summary* src =
                block_summaries + static_cast<uint64_t>(q) * blocks + i;
            Summary b;
            b.min_upper = src->min_upper;
            b.first = src->first;
            b.second = src->second;
            b.first_row = src->first_row;
            b.first_distance = src->first_distance;
            m = summary_merge(m, b);
        }
        s = block_reduce_summary(m);
        if (threadIdx.x == 0) {
            done[q] = 0;
        }
    }
    __shared__ bool certified;
    __shared__ float min_upper;
    if (threadIdx.x == 0) {
        certified = s.second > s.min_upper && s.first_row != 0xffffffffu;
        min_upper = s.min_upper;
        if (certified) {
            results[q] = Result{s.first_row, s.first_distance};
            exact_distances[q] = __longlong_as_double(0x7ff8000000000000ll);
        } else {
            atomicAdd(replay_count, 1u);
        }
    }
    __syncthreads();
    if (certified) {
        return;
    }

    const float* qrow = in.queries + static_cast<uint64_t>(q) * in.padded_dim;
    if constexpr (kEmulated) {
        // exact and flat ops only: settled without FP64 instructions
        __shared__ ResolveSmem rs;
        auto is_candidate = [&](uint32_t r) {
            return bound_of(row_distance(view, q, r), bound, r, q).lower <= min_upper;
        };
        resolve_begin(rs);
        for (uint32_t r = threadIdx.x; r < view.rows; r += kFinalizeThreads) {
            if (is_candidate(r)) {
                resolve_push(rs, r);
            }
        }
        resolve_without_fp64(in, qrow, rs, view.rows, is_candidate, results + q,
                             exact_distances + q);
        return;
    }
    if (projected_op(in.op)) {
        project_query64(in, qrow, projected_query);
        __syncthreads();
    }
    constexpr int warps = kFinalizeThreads / 32;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    double best = __longlong_as_double(0x7ff0000000000000ll);
    uint32_t best_row = 0xffffffffu;
    // candidate flags for kArgminUnroll runs of 32 rows per warp step (loads
    // in flight together), then the replays of the step's candidates in one
    // rolled loop (a single copy of the replay code)
    for (uint32_t base = warp * 32; base < view.rows; base += warps * 32 * kArgminUnroll) {
        unsigned int masks[kArgminUnroll];
#pragma unroll
        for (int u = 0; u < kArgminUnroll; ++u) {
            const uint32_t r = base + u * warps * 32 + lane;
            masks[u] = __ballot_sync(
                0xffffffffu,
                r < view.rows &&
                    bound_of(row_distance(view, q, r), bound, r, q).lower <= min_upper);
        }
#pragma unroll 1
        for (int u = 0; u < kArgminUnroll; ++u) {
            unsigned int mask = masks[u];
            while (mask != 0u) {
                const int bit = __ffs(mask) - 1;
                mask &= mask - 1u;
                const uint32_t crow = base + u * warps * 32 + bit;
                const double d = replay_candidate(in, qrow, projected_query, crow, lane);
                if (lex_less(d, crow, best, best_row)) {
                    best = d;
                    best_row = crow;
                }
            }
        }
    }
    __shared__ double warp_best[warps];
    __shared__ uint32_t warp_best_row[warps];
    if (lane == 0) {
        warp_best[warp] = best;
        warp_best_row[warp] = best_row;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < warps; ++w) {
            if (lex_less(warp_best[w], warp_best_row[w], best, best_row)) {
                best = warp_best[w];
                best_row = warp_best_row[w];
            }
        }
        results[q] = Result{best_row, static_cast<float>(best)};
        exact_distances[q] = best;
    }
}

template <bool kEmulated>
__global__ void __launch_bounds__(kFinalizeThreads)
    argmin_kernel(PartialView view, Bound bound, ReplayInputs in, Result* results,
                  double* exact_distances, Summary* block_summaries,
                  uint32_t* done, uint32_t* replay_count, uint32_t span)
{
    extern __shared__ double argmin_projected_query[];
    argmin_block<kEmulated>(view, bound, in, results, exact_distances, block_summaries, done,
                            replay_count, span, blockIdx.x, blockIdx.y, gridDim.x,
                            argmin_projected_query);
}

// The reference binary64 distance of each query's selected row (hierarchical
// indexes: their binary32 projected distances can differ from the reference's
// by more than 1e-5 relative when rows are close, so the reported distance is
// replayed). One CTA per query: the binary64 projected query, then one warp
// replays the selected row.
__global__ void __launch_bounds__(kFinalizeThreads)
    refine_kernel(ReplayInputs in, Bound bound, const Result* results,
                  double* exact_distances)
{
    const uint32_t q = blockIdx.x;
    // replayed by the argmin already, or the certified interval is within the
    // 1e-5 relative tolerance: the binary32 distance stands
    const double known = exact_distances[q];
    if (known == known) {
        return;
    }
    const Result res = results[q];
    const Bounds2 b = bound_of(res.distance, bound, res.row, q);
    if (__fsub_ru(b.upper, b.lower) <= __fmul_rd(0.999e-5f, b.lower)) {
        return;
    }
    extern __shared__ double projected_query[];
    const float* qrow = in.queries + static_cast<uint64_t>(q) * in.padded_dim;
    project_query64(in, qrow, projected_query);
    __syncthreads();
    if (threadIdx.x >= 32) {
        return;
    }
    const double d = replay_candidate(in, qrow, projected_query, results[q].row,
                                      threadIdx.x);
    if (threadIdx.x == 0) {
        exact_distances[q] = d;
    }
}

// The same for groups of kRefineGroup consecutive queries per CTA: thread j
// projects every query of the group that needs it (each coefficient of row j
// of the binary64 projection is read once for the group; each query's sum
// keeps the reference order), then one warp per such query replays its row.
constexpr int kRefineGroup = 8;

__device__ __forceinline__ void refine_group_block(const ReplayInputs& in, const Bound& bound,
                                                   const Result* results,
                                                   double* exact_distances, uint32_t batch,
                                                   uint32_t bx, unsigned char* refine_smem)
{
    double* y = reinterpret_cast<double*>(refine_smem);           // group x proj_dim
    float* x = reinterpret_cast<float*>(y + kRefineGroup * in.proj_dim);  // group x dim
    __shared__ uint32_t members[kRefineGroup];
    __shared__ int count;
    const uint32_t q0 = bx * kRefineGroup;
    if (threadIdx.x == 0) {
        int c = 0;
        for (int g = 0; g < kRefineGroup; ++g) {
            const uint32_t q = q0 + g;
            if (q >= batch) {
                break;
            }
            const double known = exact_distances[q];
            if (known == known) {
                continue;
            }
            const Result res = results[q];
            const Bounds2 b = bound_of(res.distance, bound, res.row, q);
            if (__fsub_ru(b.upper, b.lower) <= __fmul_rd(0.999e-5f, b.lower)) {
                continue;
            }
            members[c++] = q;
        }
        count = c;
    }
    __syncthreads();
    const int n = count;
    if (n == 0) {
        return;
    }
    const uint64_t dim = in.dim;
    for (uint64_t idx = threadIdx.x; idx < static_cast<uint64_t>(n) * dim;
         idx += kFinalizeThreads) {
        const uint64_t m = idx / dim;
        const uint64_t i = idx - m * dim;
        x[idx] = in.queries[static_cast<uint64_t>(members[m]) * in.padded_dim + i];
    }
    __syncthreads();
    for (uint64_t j = threadIdx.x; j < in.proj_dim; j += kFinalizeThreads) {
        const double* coeff = in.projection64 + j * dim;
        double acc[kRefineGroup];
#pragma unroll
        for (int m = 0; m < kRefineGroup; ++m) {
            acc[m] = 0.0;
        }
        for (uint64_t i = 0; i < dim; ++i) {
            const double c = coeff[i];
#pragma unroll
            for (int m = 0; m < kRefineGroup; ++m) {
                if (m < n) {
                    acc[m] = __dadd_rn(acc[m], __dmul_rn(static_cast<double>(x[m * dim + i]), c));
                }
            }
        }
#pragma unroll
        for (int m = 0; m < kRefineGroup; ++m) {
            if (m < n) {
                y[m * in.proj_dim + j] = acc[m];
            }
        }
    }
    __syncthreads();
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (warp < n) {
        const uint32_t q = members[warp];
        const float* qrow = in.queries + static_cast<uint64_t>(q) * in.padded_dim;
        const double d = replay_candidate(in, qrow, y + warp * in.proj_dim, results[q].row, lane);
        if (lane == 0) {
            exact_distances[q] = d;
        }
    }
}

__global__ void __launch_bounds__(kFinalizeThreads)
    refine_group_kernel(ReplayInputs in, Bound bound, const Result* results,
                        double* exact_distances, uint32_t batch)
{
    extern __shared__ unsigned char refine_group_smem[];
    refine_group_block(in, bound, results, exact_distances, batch, blockIdx.x,
                       refine_group_smem);
}

// ------------------------------------------------ small indexes, one launch

// One CTA per query for indexes small enough that a single CTA scans all of
// them (rows x padded columns <= kSmallCells): the query's sampled (or all)
// coordinates are gathered into shared memory with the preparation kernels'
// finiteness flags, one warp per row computes the binary32 distance (lane
// partial sums in column order, then a warp butterfly), and the block
// certifies the argmin, replaying the candidates in binary64 when needed.
// Answers are those of the three-kernel path; only the accumulation depth
// (and with it the bound) differs.
template <bool kEmulated>
__global__ void __launch_bounds__(kFinalizeThreads)
    small_query_kernel(SmallQuery sq, Bound bound, ReplayInputs in, Result* results,
                       double* exact_distances, uint32_t* replay_count, int* error_flag)
{
    extern __shared__ float small_smem[];
    float* qv = small_smem;                      // padded_dim
    float* dist = small_smem + sq.padded_dim;    // row_count
    __shared__ int bad;
    const uint32_t q = blockIdx.x;
    if (threadIdx.x == 0) {
        bad = 0;
    }
    __syncthreads();
    const float* src = sq.queries + static_cast<uint64_t>(q) * sq.dim;
    for (uint64_t i = threadIdx.x; i < sq.padded_dim; i += kFinalizeThreads) {
        float v = 0.f;
        if (sq.columns == nullptr) {
            if (i < sq.dim) {
                v = src[i];
                if (!isfinite(v)) {
                    atomicOr(error_flag, 1);
                    bad = 1;
                }
            }
        } else if (i < sq.sample_size) {
            v = src[sq.columns[i]];
            if (!isfinite(v)) {
                atomicOr(error_flag, 1);
                bad = 1;
            }
            if (sq.scales != nullptr) {
                v = __fmul_rn(v, sq.scales[i]);
                if (!isfinite(v)) {
                    atomicOr(error_flag, 2);
                    bad = 1;
                }
            }
        }
        qv[i] = v;
    }
    __syncthreads();
    if (bad) {
        // the call fails on the flag; nothing to certify
        if (threadIdx.x == 0) {
            results[q] = Result{0, 0.f};
            exact_distances[q] = __longlong_as_double(0x7ff8000000000000ll);
        }
        return;
    }
    constexpr int warps = kFinalizeThreads / 32;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const uint64_t groups = sq.padded_dim / 4;
    const float4* q4 = reinterpret_cast<const float4*>(qv);
    for (uint32_t row = warp; row < sq.row_count; row += warps) {
        const float4* r4 =
            reinterpret_cast<const float4*>(sq.rows + static_cast<uint64_t>(row) * sq.padded_dim);
        const float4* w4 = reinterpret_cast<const float4*>(sq.weights32);
        float acc = 0.f;
        for (uint64_t g = lane; g < groups; g += 32) {
            const float4 a = q4[g];
            const float4 b = __ldg(r4 + g);
            if (sq.op == static_cast<int>(ScanOp::l2)) {
                float d = a.x - b.x; acc = fmaf(d, d, acc);
                d = a.y - b.y; acc = fmaf(d, d, acc);
                d = a.z - b.z; acc = fmaf(d, d, acc);
                d = a.w - b.w; acc = fmaf(d, d, acc);
            } else if (sq.op == static_cast<int>(ScanOp::l1)) {
                acc += fabsf(a.x - b.x);
                acc += fabsf(a.y - b.y);
                acc += fabsf(a.z - b.z);
                acc += fabsf(a.w - b.w);
            } else {
                const float4 w = __ldg(w4 + g);
                acc = fmaf(fabsf(a.x - b.x), w.x, acc);
                acc = fmaf(fabsf(a.y - b.y), w.y, acc);
                acc = fmaf(fabsf(a.z - b.z), w.z, acc);
                acc = fmaf(fabsf(a.w - b.w), w.w, acc);
            }
        }
        for (int o = 16; o > 0; o /= 2) {
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
        }
        if (lane == 0) {
            dist[row] = acc;
        }
    }
    __syncthreads();
    const float inf = __int_as_float(0x7f800000);
    Summary s{inf, inf, inf, 0xffffffffu, inf};
    for (uint32_t row = threadIdx.x; row < sq.row_count; row += kFinalizeThreads) {
        const Bounds2 b = bound_of(dist[row], bound, row, q);
        summary_insert(s, b.lower, b.upper, row, dist[row]);
    }
    s = block_reduce_summary(s);
    __shared__ bool certified;
    __shared__ float min_upper;
    if (threadIdx.x == 0) {
        certified = s.second > s.min_upper;
        min_upper = s.min_upper;
        if (certified) {
            results[q] = Result{s.first_row, s.first_distance};
            exact_distances[q] = __longlong_as_double(0x7ff8000000000000ll);
        } else {
            atomicAdd(replay_count, 1u);
        }
    }
    __syncthreads();
    if (certified) {
        return;
    }
    if constexpr (kEmulated) {
        __shared__ ResolveSmem rs;
        auto is_candidate = [&](uint32_t r) {
            return bound_of(dist[r], bound, r, q).lower <= min_upper;
        };
        resolve_begin(rs);
        for (uint32_t r = threadIdx.x; r < sq.row_count; r += kFinalizeThreads) {
            if (is_candidate(r)) {
                resolve_push(rs, r);
            }
        }
        resolve_without_fp64(in, qv, rs, sq.row_count, is_candidate, results + q,
                             exact_distances + q);
        return;
    }
    double best = __longlong_as_double(0x7ff0000000000000ll);
    uint32_t best_row = 0xffffffffu;
    for (uint32_t row = warp; row < sq.row_count; row += warps) {
        if (bound_of(dist[row], bound, row, q).lower > min_upper) {
            continue;
        }
        const double d = replay_row(in, qv, in.rows + static_cast<uint64_t>(row) * in.padded_dim,
                                    lane);
        if (lex_less(d, row, best, best_row)) {
            best = d;
            best_row = row;
        }
    }
    __shared__ double warp_best[warps];
    __shared__ uint32_t warp_best_row[warps];
    if (lane == 0) {
        warp_best[warp] = best;
        warp_best_row[warp] = best_row;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < warps; ++w) {
            if (lex_less(warp_best[w], warp_best_row[w], best, best_row)) {
                best = warp_best[w];
                best_row = warp_best_row[w];
            }
        }
        results[q] = Result{best_row, static_cast<float>(best)};
        exact_distances[q] = best;
    }
}

// ------------------------------------- flat indexes at small batches, one launch

// Programmatic dependent launch: a grid launched with programmatic stream
// serialization may start while the previous kernel of the stream runs;
// griddepcontrol.wait returns once that kernel has completed and its memory
// is visible (immediately when the launch had no programmatic edge), and
// griddepcontrol.launch_dependents lets the next such grid start.
__device__ __forceinline__ void wait_for_previous_grid()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void allow_next_grid()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Polls of a flat query copy wait before it gives up (well above any copy's
// time), and the error bit it then sets.
constexpr uint32_t kFlatCopySpins = 1u << 22;
constexpr int kFlatCopyTimeout = 16;
// bytes of rows per bulk copy of the flat query kernel (two buffers per CTA)
constexpr uint64_t kFlatChunkBytes = 32 * 1024;
// query entries a flat query thread gathers at a time
constexpr int kFlatGather = 8;
// float4 loads in flight per lane when rows are read from global memory
constexpr int kFlatDirectLoads = 8;

// Per-row accumulation of one lane: binary32, column order, four terms per
// float4 group (the same arithmetic as small_query_kernel); the query and the
// weights are in shared memory.
__device__ __forceinline__ float flat_terms(int op, float acc, const float4 a,
                                            const float4 b, const float4* w4, uint64_t g)
{
    if (op == static_cast<int>(ScanOp::l2)) {
        float d = a.x - b.x; acc = fmaf(d, d, acc);
        d = a.y - b.y; acc = fmaf(d, d, acc);
        d = a.z - b.z; acc = fmaf(d, d, acc);
        d = a.w - b.w; acc = fmaf(d, d, acc);
    } else if (op == static_cast<int>(ScanOp::l1)) {
        acc += fabsf(a.x - b.x);
        acc += fabsf(a.y - b.y);
        acc += fabsf(a.z - b.z);
        acc += fabsf(a.w - b.w);
    } else {
        const float4 w = w4[g];
        acc = fmaf(fabsf(a.x - b.x), w.x, acc);
        acc = fmaf(fabsf(a.y - b.y), w.y, acc);
        acc = fmaf(fabsf(a.z - b.z), w.z, acc);
        acc = fmaf(fabsf(a.w - b.w), w.w, acc);
    }
    return acc;
}

// grid = (row blocks, batch), kFinalizeThreads threads. At entry one thread
// of every CTA starts bulk copies (the TMA engine, cp.async.bulk) of its row
// block into shared memory: `chunk_rows` rows per copy, two buffers, the next
// chunk copied while one is scanned (rows too long for a pass of the CTA in
// one copy, chunk_rows 0, are instead loaded from global memory into
// registers, kFlatDirectLoads per lane in flight). Meanwhile the CTA gathers its query's
// sampled (or all) coordinates into shared memory with the preparation
// kernels' finiteness flags (and the column weights of a weighted L1 index).
// Then it computes the binary32 distance of each row with kLanes lanes per row
// (each lane sums its float4 groups g = lane, lane + kLanes, ... in column
// order; a butterfly within the lane group adds the kLanes partial sums),
// stores it in the query's distance slab and keeps its two smallest. The last
// CTA of the query to finish merges the CTA summaries and certifies the
// argmin, replaying the candidates in binary64 when the bounds overlap,
// exactly as argmin_kernel does.
//
// Consecutive launches alternate between two scratch slots (distance slabs,
// summaries, completion counters), so a launch's copies, gather and scan
// depend on nothing the previous launch writes and run while it finishes
// (programmatic serialization). Every CTA passes wait_for_previous_grid() --
// the previous grid has completed -- before it publishes its summary or
// writes a result, and only then lets the next grid start; so at most two
// grids are in flight, and the grid after next, which reuses this grid's
// slot, starts only once this grid has completed.
//
// A copy wait gives up after kFlatCopySpins polls: the CTA sets error bit 16
// (the call fails), waits (bounded) for the copies it issued, and still
// takes part in the query's merge with an empty summary, so the completion
// counters stay consistent.
template <int kLanes, bool kEmulated>
__global__ void __launch_bounds__(kFinalizeThreads, 3)
    flat_query_kernel(SmallQuery sq, Bound bound, ReplayInputs in, float* distances,
                      Summary* block_summaries, uint32_t* done, uint32_t summary_stride,
                      uint32_t span, uint32_t chunk_rows, Result* results,
                      double* exact_distances, uint32_t* replay_count, int* error_flag)
{
    extern __shared__ __align__(16) float flat_smem[];
    const bool weighted = sq.op == static_cast<int>(ScanOp::l1_weighted);
    float* qv = flat_smem;                  // padded_dim
    float* wv = flat_smem + sq.padded_dim;  // padded_dim, weighted L1 only
    float* chunks = flat_smem + sq.padded_dim * (weighted ? 2 : 1);  // 2 x chunk rows
    __shared__ uint64_t full[2];
    __shared__ int bad;
    __shared__ int copy_failed;
    const uint32_t q = blockIdx.y;
    const uint32_t blocks = gridDim.x;
    const uint32_t first_row = blockIdx.x * span;
    const uint32_t end_row = min(sq.row_count, first_row + span);
    const uint32_t row_words = static_cast<uint32_t>(sq.padded_dim);
    // chunk_rows 0: rows too long for a pass of the CTA in one copy are read
    // straight from global memory instead
    const uint32_t nchunks =
        chunk_rows != 0 ? (end_row - first_row + chunk_rows - 1) / chunk_rows : 0u;
    auto issue = [&](uint32_t c) {
        const uint32_t r0 = first_row + c * chunk_rows;
        const uint32_t bytes = min(chunk_rows, end_row - r0) * row_words * 4u;
        uint64_t* bar = full + (c & 1u);
        async::mbar_expect_tx(bar, bytes);
        async::bulk_copy_g2s(chunks + (c & 1u) * chunk_rows * row_words,
                             sq.rows + static_cast<uint64_t>(r0) * row_words, bytes, bar);
    };
    if (threadIdx.x == 0) {
        bad = 0;
        copy_failed = 0;
        async::mbar_init(full, 1);
        async::mbar_init(full + 1, 1);
        async::mbar_init_fence();
        for (uint32_t c = 0; c < nchunks && c < 2; ++c) {
            issue(c);
        }
    }
    __syncthreads();
    const float* src = sq.queries + static_cast<uint64_t>(q) * sq.dim;
    int local_bad = 0;
    // kFlatGather entries per thread at a time: their column indices (and
    // scales, weights) in flight together, then their query values together,
    // so the gather costs two memory round trips, not two per entry
    for (uint64_t base = threadIdx.x; base < sq.padded_dim;
         base += static_cast<uint64_t>(kFinalizeThreads) * kFlatGather) {
        uint32_t col[kFlatGather];
        float scale[kFlatGather];
        float weight[kFlatGather];
#pragma unroll
        for (int u = 0; u < kFlatGather; ++u) {
            const uint64_t i = base + static_cast<uint64_t>(u) * kFinalizeThreads;
            const bool sampled = sq.columns != nullptr && i < sq.sample_size;
            col[u] = sampled ? sq.columns[i] : 0u;
            scale[u] = sampled && sq.scales != nullptr ? sq.scales[i] : 1.f;
            weight[u] = weighted && i < sq.padded_dim ? sq.weights32[i] : 0.f;
        }
        float value[kFlatGather];
#pragma unroll
        for (int u = 0; u < kFlatGather; ++u) {
            const uint64_t i = base + static_cast<uint64_t>(u) * kFinalizeThreads;
            value[u] = 0.f;
            if (sq.columns == nullptr) {
                if (i < sq.dim) {
                    value[u] = src[i];
                }
            } else if (i < sq.sample_size) {
                value[u] = src[col[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kFlatGather; ++u) {
            const uint64_t i = base + static_cast<uint64_t>(u) * kFinalizeThreads;
            if (i >= sq.padded_dim) {
                continue;
            }
            float v = value[u];
            if (sq.columns == nullptr ? i < sq.dim : i < sq.sample_size) {
                local_bad |= isfinite(v) ? 0 : 1;
                if (sq.columns != nullptr && sq.scales != nullptr) {
                    v = __fmul_rn(v, scale[u]);
                    local_bad |= isfinite(v) ? 0 : 2;
                }
            }
            qv[i] = v;
            if (weighted) {
                wv[i] = weight[u];
            }
        }
    }
    if (local_bad != 0) {
        bad = 1;
    }
    __syncthreads();

    const float inf = __int_as_float(0x7f800000);
    Summary s{inf, inf, inf, 0xffffffffu, inf};
    const int lane = threadIdx.x % 32;
    float* dist = distances + static_cast<uint64_t>(q) * sq.row_count;
    {
        constexpr int kRowsPerStep = kFinalizeThreads / kLanes;
        const int sub = threadIdx.x % kLanes;
        const int group = threadIdx.x / kLanes;
        const uint64_t groups = sq.padded_dim / 4;
        const float4* q4 = reinterpret_cast<const float4*>(qv);
        const float4* w4 = reinterpret_cast<const float4*>(wv);
        RowScan scan;
        // the butterfly over the row's lanes, the distance and the CTA's two
        // smallest
        auto record = [&](float acc, uint32_t row, bool valid) {
#pragma unroll
            for (int o = kLanes / 2; o > 0; o /= 2) {
                acc += __shfl_xor_sync(0xffffffffu, acc, o);
            }
            if (valid && sub == 0) {
                dist[row] = acc;
                if (!(acc <= FLT_MAX)) {
                    scan.overflow = true;
                } else if (acc < scan.k1) {
                    scan.k2 = scan.k1;
                    scan.k1 = acc;
                    scan.r1 = row;
                } else if (acc < scan.k2) {
                    scan.k2 = acc;
                }
            }
        };
        if (chunk_rows == 0 && !bad) {
            // long rows: kFlatDirectLoads float4 loads in flight per lane, the
            // same column order per lane
            for (uint32_t base = first_row; base < end_row; base += kRowsPerStep) {
                const uint32_t row = base + group;
                const bool valid = row < end_row;
                const float4* r4 = reinterpret_cast<const float4*>(
                    sq.rows + static_cast<uint64_t>(valid ? row : first_row) * row_words);
                float acc = 0.f;
                for (uint64_t g0 = sub; g0 < groups; g0 += kFlatDirectLoads * kLanes) {
                    float4 b[kFlatDirectLoads];
#pragma unroll
                    for (int j = 0; j < kFlatDirectLoads; ++j) {
                        const uint64_t g = g0 + static_cast<uint64_t>(j) * kLanes;
                        b[j] = g < groups ? __ldg(r4 + g) : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
#pragma unroll
                    for (int j = 0; j < kFlatDirectLoads; ++j) {
                        const uint64_t g = g0 + static_cast<uint64_t>(j) * kLanes;
                        if (g < groups) {
                            acc = flat_terms(sq.op, acc, q4[g], b[j], w4, g);
                        }
                    }
                }
                record(acc, row, valid);
            }
        }
        uint32_t failed_chunk = nchunks;
        for (uint32_t c = 0; c < nchunks; ++c) {
            // every thread sees the chunk complete (or the copy given up)
            if (!async::mbar_wait(full + (c & 1u), (c >> 1) & 1u, kFlatCopySpins)) {
                copy_failed = 1;
            }
            __syncthreads();
            if (copy_failed) {
                failed_chunk = c;  // chunks c and c + 1 may still be in flight
                break;
            }
            const uint32_t r0 = first_row + c * chunk_rows;
            const uint32_t rows_here = min(chunk_rows, end_row - r0);
            const float4* buf =
                reinterpret_cast<const float4*>(chunks + (c & 1u) * chunk_rows * row_words);
            if (!bad) {
                // the same trip count on every lane (warp-wide shuffles below)
                for (uint32_t base = 0; base < rows_here; base += kRowsPerStep) {
                    const uint32_t lr = base + group;
                    const bool valid = lr < rows_here;
                    const float4* r4 =
                        buf + static_cast<uint64_t>(valid ? lr : 0) * (row_words / 4);
                    float acc = 0.f;
#pragma unroll 4
                    for (uint64_t g = sub; g < groups; g += kLanes) {
                        acc = flat_terms(sq.op, acc, q4[g], r4[g], w4, g);
                    }
                    record(acc, r0 + lr, valid);
                }
            }
            // the buffer is free again: copy chunk c + 2 into it
            __syncthreads();
            if (threadIdx.x == 0 && c + 2 < nchunks) {
                async::fence_proxy_async_smem();
                issue(c + 2);
            }
        }
        if (failed_chunk < nchunks) {
            // wait (bounded) for the copies that may still be in flight
            if (threadIdx.x == 0) {
                for (uint32_t c = failed_chunk; c < nchunks && c < failed_chunk + 2; ++c) {
                    async::mbar_wait(full + (c & 1u), (c >> 1) & 1u, kFlatCopySpins);
                }
                atomicOr(error_flag, kFlatCopyTimeout);
            }
        } else if (!bad) {
            if (scan.r1 != 0xffffffffu) {
                const Bounds2 b1 = bound_of(scan.k1, bound, scan.r1, q);
                s = Summary{b1.upper, b1.lower,
                            scan.k2 <= FLT_MAX ? lower_any(scan.k2, bound, q) : inf, scan.r1,
                            scan.k1};
            }
            if (scan.overflow) {
                summary_insert(s, 0.f, inf, 0xffffffffu, inf);
            }
        }
        s = block_reduce_summary(s);
    }

    wait_for_previous_grid();
    allow_next_grid();
    if (bad) {
        // the call fails on the flag; nothing to certify
        if (local_bad != 0) {
            atomicOr(error_flag, local_bad);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            results[q] = Result{0, 0.f};
            exact_distances[q] = __longlong_as_double(0x7ff8000000000000ll);
        }
        return;
    }
    __shared__ bool is_last;
    if (blocks > 1) {
        if (threadIdx.x == 0) {
            block_summaries[static_cast<uint64_t>(q) * summary_stride + blockIdx.x] = s;
            __threadfence();
            is_last = atomicAdd(done + q, 1u) == blocks - 1;
        }
        __syncthreads();
        if (!is_last) {
            return;
        }
        __threadfence();
        Summary m{inf, inf, inf, 0xffffffffu, inf};
        // two summaries per thread in flight together
        for (uint32_t i0 = threadIdx.x; i0 < blocks; i0 += 2 * kFinalizeThreads) {
            Summary b[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const uint32_t i = i0 + u * kFinalizeThreads;
                b[u] = Summary{inf, inf, inf, 0xffffffffu, inf};
                if (i < blocks) {
                    const volatile Summary* src_s =
                        block_summaries + static_cast<uint64_t>(q) * summary_stride + i;
                    b[u].min_upper = src_s->min_upper;
                    b[u].first = src_s->first;
                    b[u].second = src_s->second;
                    b[u].first_row = src_s->first_row;
                    b[u].first_distance = src_s->first_distance;
                }
            }
            m = summary_merge(m, b[0]);
            m = summary_merge(m, b[1]);
        }
        s = block_reduce_summary(m);
        if (threadIdx.x == 0) {
            done[q] = 0;
        }
    }
    __shared__ bool certified;
    __shared__ float min_upper;
    if (threadIdx.x == 0) {
        certified = s.second > s.min_upper && s.first_row != 0xffffffffu;
        min_upper = s.min_upper;
        if (certified) {
            results[q] = Result{s.first_row, s.first_distance};
            exact_distances[q] = __longlong_as_double(0x7ff8000000000000ll);
        } else {
            atomicAdd(replay_count, 1u);
        }
    }
    __syncthreads();
    if (certified) {
        return;
    }
    if constexpr (kEmulated) {
        __shared__ ResolveSmem rs;
        auto is_candidate = [&](uint32_t r) {
            return bound_of(__ldcg(dist + r), bound, r, q).lower <= min_upper;
        };
        resolve_begin(rs);
        for (uint32_t r = threadIdx.x; r < sq.row_count; r += kFinalizeThreads) {
            if (is_candidate(r)) {
                resolve_push(rs, r);
            }
        }
        resolve_without_fp64(in, qv, rs, sq.row_count, is_candidate, results + q,
                             exact_distances + q);
        return;
    }
    constexpr int warps = kFinalizeThreads / 32;
    const int warp = threadIdx.x / 32;
    double best = __longlong_as_double(0x7ff0000000000000ll);
    uint32_t best_row = 0xffffffffu;
    for (uint32_t base = warp * 32; base < sq.row_count; base += warps * 32) {
        const uint32_t r = base + lane;
        unsigned int mask = __ballot_sync(
            0xffffffffu,
            r < sq.row_count && bound_of(__ldcg(dist + r), bound, r, q).lower <= min_upper);
        while (mask != 0u) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1u;
            const uint32_t crow = base + bit;
            const double d = replay_row(
                in, qv, in.rows + static_cast<uint64_t>(crow) * in.padded_dim, lane);
            if (lex_less(d, crow, best, best_row)) {
                best = d;
                best_row = crow;
            }
        }
    }
    __shared__ double warp_best[warps];
    __shared__ uint32_t warp_best_row[warps];
    if (lane == 0) {
        warp_best[warp] = best;
        warp_best_row[warp] = best_row;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < warps; ++w) {
            if (lex_less(warp_best[w], warp_best_row[w], best, best_row)) {
                best = warp_best[w];
                best_row = warp_best_row[w];
            }
        }
        results[q] = Result{best_row, static_cast<float>(best)};
        exact_distances[q] = best;
    }
}

constexpr uint32_t kMaxCandidates = 64;
constexpr int kRescoreUnroll = 4;

// Reference binary64 squared distance of one row, summed in parallel by the
// whole block: the terms are the reference CPU's own
// (t_j = (double(q_j) - double(r_j))^2, l2_distance.cpp:9-25), only the order
// of the additions differs. Thread t folds the float4 groups t, t + 256, ...
// into four accumulators (one per component); then (a0 + a1) + (a2 + a3), a
// warp butterfly (every lane ends with the same value) and a fixed tree over
// the eight warps. Longest chain of additions: rescore_depth().
__device__ double block_l2_64(const float* q, const float* r, uint64_t padded_dim,
                              double* scratch)
{
    const uint64_t groups = padded_dim / 4;
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* r4 = reinterpret_cast<const float4*>(r);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    uint64_t g = threadIdx.x;
    for (; g + (kRescoreUnroll - 1) * kFinalizeThreads < groups;
         g += kRescoreUnroll * kFinalizeThreads) {
        float4 x[kRescoreUnroll];
        float4 y[kRescoreUnroll];
#pragma unroll
        for (int u = 0; u < kRescoreUnroll; ++u) {
            x[u] = q4[g + u * kFinalizeThreads];
            y[u] = __ldg(r4 + g + u * kFinalizeThreads);
        }
#pragma unroll
        for (int u = 0; u < kRescoreUnroll; ++u) {
            const double d0 = __dsub_rn(x[u].x, y[u].x);
            const double d1 = __dsub_rn(x[u].y, y[u].y);
            const double d2 = __dsub_rn(x[u].z, y[u].z);
            const double d3 = __dsub_rn(x[u].w, y[u].w);
            a0 = __dadd_rn(a0, __dmul_rn(d0, d0));
            a1 = __dadd_rn(a1, __dmul_rn(d1, d1));
            a2 = __dadd_rn(a2, __dmul_rn(d2, d2));
            a3 = __dadd_rn(a3, __dmul_rn(d3, d3));
        }
    }
    for (; g < groups; g += kFinalizeThreads) {
        const float4 x = q4[g];
        const float4 y = __ldg(r4 + g);
        const double d0 = __dsub_rn(x.x, y.x);
        const double d1 = __dsub_rn(x.y, y.y);
        const double d2 = __dsub_rn(x.z, y.z);
        const double d3 = __dsub_rn(x.w, y.w);
        a0 = __dadd_rn(a0, __dmul_rn(d0, d0));
        a1 = __dadd_rn(a1, __dmul_rn(d1, d1));
        a2 = __dadd_rn(a2, __dmul_rn(d2, d2));
        a3 = __dadd_rn(a3, __dmul_rn(d3, d3));
    }
    double t = __dadd_rn(__dadd_rn(a0, a1), __dadd_rn(a2, a3));
    for (int o = 16; o > 0; o /= 2) {
        t = __dadd_rn(t, __shfl_xor_sync(0xffffffffu, t, o));
    }
    if (threadIdx.x % 32 == 0) {
        scratch[threadIdx.x / 32] = t;
    }
    __syncthreads();
    static_assert(kFinalizeThreads / 32 == 8, "tree over eight warps");
    return __dadd_rn(__dadd_rn(__dadd_rn(scratch[0], scratch[1]),
                               __dadd_rn(scratch[2], scratch[3])),
                     __dadd_rn(__dadd_rn(scratch[4], scratch[5]),
                               __dadd_rn(scratch[6], scratch[7])));
}

struct Interval64 {
    double lower;
    double upper;
};

// [S (1 - rel) - abs, S (1 + rel) + abs], directed roundings; an overflowed
// sum keeps every candidate below it.
__device__ __forceinline__ Interval64 interval64(double s, const Bound64& b)
{
    if (!(s <= DBL_MAX)) {
        return {0.0, __longlong_as_double(0x7ff0000000000000ll)};
    }
    const double lo = __dsub_rd(__dmul_rd(s, __dsub_rd(1.0, b.rel)), b.abs);
    const double hi = __dadd_ru(__dmul_ru(s, __dadd_ru(1.0, b.rel)), b.abs);
    return {lo > 0.0 ? lo : 0.0, hi};
}

// Certified argmin of each query over its candidate rows (the precision
// form). grid = (k, batch): CTA (c, q) computes the binary64 distance of
// candidate c; the last CTA of the query to finish decides. One candidate
// whose interval can hold the reference minimum is the answer; otherwise the
// candidates that can are replayed in the reference CPU's order (one warp
// each) and the lexicographic minimum of (distance, row) wins. exact[q] is
// the binary64 distance of the answer (the replayed one when replayed).
__global__ void __launch_bounds__(kFinalizeThreads)
    rescore_kernel(Bound64 bound, ReplayInputs in, const uint32_t* candidates,
                   uint32_t k, uint32_t row_count, double* cand_dist,
                   uint32_t* done, Result* results, double* exact_distances,
                   uint32_t* replay_count)
{
    const uint32_t c = blockIdx.x;
    const uint32_t q = blockIdx.y;
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    __shared__ double scratch[kFinalizeThreads / 32];
    __shared__ bool is_last;
    const float* qrow = in.queries + static_cast<uint64_t>(q) * in.padded_dim;
    const uint32_t row = candidates[static_cast<uint64_t>(q) * k + c];
    double d = inf;
    if (row < row_count) {
        d = block_l2_64(qrow, in.rows + static_cast<uint64_t>(row) * in.padded_dim,
                        in.padded_dim, scratch);
    }
    if (threadIdx.x == 0) {
        cand_dist[static_cast<uint64_t>(q) * k + c] = d;
        __threadfence();
        is_last = atomicAdd(done + q, 1u) == k - 1;
    }
    __syncthreads();
    if (!is_last) {
        return;
    }
    __threadfence();
    __shared__ double dist[kMaxCandidates];
    __shared__ uint32_t cand[kMaxCandidates];
    for (uint32_t i = threadIdx.x; i < k; i += kFinalizeThreads) {
        dist[i] = static_cast<volatile double*>(cand_dist)[static_cast<uint64_t>(q) * k + i];
        cand[i] = candidates[static_cast<uint64_t>(q) * k + i];
    }
    __syncthreads();
    __shared__ bool certified;
    __shared__ double min_upper;
    if (threadIdx.x == 0) {
        done[q] = 0;
        double first = inf, second = inf, upper = inf;
        uint32_t first_i = 0xffffffffu;
        for (uint32_t i = 0; i < k; ++i) {
            if (cand[i] >= row_count) {
                continue;
            }
            const Interval64 b = interval64(dist[i], bound);
            upper = fmin(upper, b.upper);
            if (first_i == 0xffffffffu || b.lower < first ||
                (b.lower == first && cand[i] < cand[first_i])) {
                second = first;
                first = b.lower;
                first_i = i;
            } else if (b.lower < second) {
                second = b.lower;
            }
        }
        certified = first_i != 0xffffffffu && second > upper;
        min_upper = upper;
        if (certified) {
            results[q] = Result{cand[first_i], static_cast<float>(dist[first_i])};
            exact_distances[q] = dist[first_i];
        } else {
            atomicAdd(replay_count, 1u);
        }
    }
    __syncthreads();
    if (certified) {
        return;
    }
    constexpr int warps = kFinalizeThreads / 32;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    double best = inf;
    uint32_t best_row = 0xffffffffu;
    for (uint32_t i = warp; i < k; i += warps) {
        const uint32_t r = cand[i];
        if (r >= row_count || interval64(dist[i], bound).lower > min_upper) {
            continue;
        }
        const double v = replay_row(in, qrow, in.rows + static_cast<uint64_t>(r) * in.padded_dim,
                                    lane);
        if (lex_less(v, r, best, best_row)) {
            best = v;
            best_row = r;
        }
    }
    __shared__ double warp_best[warps];
    __shared__ uint32_t warp_best_row[warps];
    if (lane == 0) {
        warp_best[warp] = best;
        warp_best_row[warp] = best_row;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < warps; ++w) {
            if (lex_less(warp_best[w], warp_best_row[w], best, best_row)) {
                best = warp_best[w];
                best_row = warp_best_row[w];
            }
        }
        results[q] = Result{best_row, static_cast<float>(best)};
        exact_distances[q] = best;
    }
}

// Binary32 squared distance of one row summed by the whole block with the
// structure of block_l2_64 (four accumulators per thread over its float4
// groups, pairwise, warp butterfly, fixed tree over the eight warps), so its
// longest addition chain is rescore_depth() as well.
__device__ float block_l2_32(const float* q, const float* r, uint64_t padded_dim,
                             float* scratch)
{
    const uint64_t groups = padded_dim / 4;
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* r4 = reinterpret_cast<const float4*>(r);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    uint64_t g = threadIdx.x;
    for (; g + (kRescoreUnroll - 1) * kFinalizeThreads < groups;
         g += kRescoreUnroll * kFinalizeThreads) {
        float4 x[kRescoreUnroll];
        float4 y[kRescoreUnroll];
#pragma unroll
        for (int u = 0; u < kRescoreUnroll; ++u) {
            x[u] = q4[g + u * kFinalizeThreads];
            y[u] = __ldg(r4 + g + u * kFinalizeThreads);
        }
#pragma unroll
        for (int u = 0; u < kRescoreUnroll; ++u) {
            const float d0 = __fsub_rn(x[u].x, y[u].x);
            const float d1 = __fsub_rn(x[u].y, y[u].y);
            const float d2 = __fsub_rn(x[u].z, y[u].z);
            const float d3 = __fsub_rn(x[u].w, y[u].w);
            a0 = __fmaf_rn(d0, d0, a0);
            a1 = __fmaf_rn(d1, d1, a1);
            a2 = __fmaf_rn(d2, d2, a2);
            a3 = __fmaf_rn(d3, d3, a3);
        }
    }
    for (; g < groups; g += kFinalizeThreads) {
        const float4 x = q4[g];
        const float4 y = __ldg(r4 + g);
        const float d0 = __fsub_rn(x.x, y.x);
        const float d1 = __fsub_rn(x.y, y.y);
        const float d2 = __fsub_rn(x.z, y.z);
        const float d3 = __fsub_rn(x.w, y.w);
        a0 = __fmaf_rn(d0, d0, a0);
        a1 = __fmaf_rn(d1, d1, a1);
        a2 = __fmaf_rn(d2, d2, a2);
        a3 = __fmaf_rn(d3, d3, a3);
    }
    float t = __fadd_rn(__fadd_rn(a0, a1), __fadd_rn(a2, a3));
    for (int o = 16; o > 0; o /= 2) {
        t = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, o));
    }
    if (threadIdx.x % 32 == 0) {
        scratch[threadIdx.x / 32] = t;
    }
    __syncthreads();
    return __fadd_rn(__fadd_rn(__fadd_rn(scratch[0], scratch[1]),
                               __fadd_rn(scratch[2], scratch[3])),
                     __fadd_rn(__fadd_rn(scratch[4], scratch[5]),
                               __fadd_rn(scratch[6], scratch[7])));
}

// The FP32 re-score of the precision strategies, without FP64 instructions.
// grid = (k, batch): CTA (c, q) computes candidate c's binary32 distance from
// the original rows; the last CTA of the query certifies: one candidate whose
// bound can hold the reference minimum is the answer (its binary32 distance
// reported); otherwise the candidates that can are settled by
// resolve_without_fp64 (float-float, then emulated binary64 for unseparated
// ones).
__global__ void __launch_bounds__(kFinalizeThreads)
    rescore32_kernel(Bound bound, ReplayInputs in, const uint32_t* candidates,
                     uint32_t k, uint32_t row_count, float* cand_dist, uint32_t* done,
                     Result* results, double* exact_distances, uint32_t* replay_count)
{
    const uint32_t c = blockIdx.x;
    const uint32_t q = blockIdx.y;
    const float inf = __int_as_float(0x7f800000);
    __shared__ float scratch[kFinalizeThreads / 32];
    __shared__ bool is_last;
    const float* qrow = in.queries + static_cast<uint64_t>(q) * in.padded_dim;
    const uint32_t row = candidates[static_cast<uint64_t>(q) * k + c];
    float d = inf;
    if (row < row_count) {
        d = block_l2_32(qrow, in.rows + static_cast<uint64_t>(row) * in.padded_dim,
                        in.padded_dim, scratch);
    }
    if (threadIdx.x == 0) {
        cand_dist[static_cast<uint64_t>(q) * k + c] = d;
        __threadfence();
        is_last = atomicAdd(done + q, 1u) == k - 1;
    }
    __syncthreads();
    if (!is_last) {
        return;
    }
    __threadfence();
    __shared__ float dist[kMaxCandidates];
    __shared__ uint32_t cand[kMaxCandidates];
    for (uint32_t i = threadIdx.x; i < k; i += kFinalizeThreads) {
        dist[i] = static_cast<volatile float*>(cand_dist)[static_cast<uint64_t>(q) * k + i];
        cand[i] = candidates[static_cast<uint64_t>(q) * k + i];
    }
    __syncthreads();
    __shared__ bool certified;
    __shared__ float min_upper;
    if (threadIdx.x == 0) {
        done[q] = 0;
        float first = inf, second = inf, upper = inf;
        uint32_t first_i = 0xffffffffu;
        for (uint32_t i = 0; i < k; ++i) {
            if (cand[i] >= row_count) {
                continue;
            }
            const Bounds2 b = bound_of(dist[i], bound, cand[i], q);
            upper = fminf(upper, b.upper);
            if (first_i == 0xffffffffu || b.lower < first ||
                (b.lower == first && cand[i] < cand[first_i])) {
                second = first;
                first = b.lower;
                first_i = i;
            } else if (b.lower < second) {
                second = b.lower;
            }
        }
        certified = first_i != 0xffffffffu && second > upper;
        min_upper = upper;
        if (certified) {
            results[q] = Result{cand[first_i], dist[first_i]};
            exact_distances[q] = __longlong_as_double(
                static_cast<long long>(x64::from_float(dist[first_i])));
        } else {
            atomicAdd(replay_count, 1u);
        }
    }
    __syncthreads();
    if (certified) {
        return;
    }
    __shared__ ResolveSmem rs;
    resolve_begin(rs);
    for (uint32_t i = threadIdx.x; i < k; i += kFinalizeThreads) {
        if (cand[i] < row_count && bound_of(dist[i], bound, cand[i], q).lower <= min_upper) {
            resolve_push(rs, cand[i]);
        }
    }
    // k <= kMaxCandidates < kResolveCap: the list never overflows
    resolve_without_fp64(in, qrow, rs, row_count, [](uint32_t) { return false; },
                         results + q, exact_distances + q);
}

// ------------------------------------------ the persistent multi-index batch

enum PersistentKind : uint32_t {
    kUnitClear = 0,
    kUnitGather,
    kUnitProject,
    kUnitFinishErr,
    kUnitTile,
    kUnitSample,
    kUnitCount,
    kUnitSurvivor,
    kUnitArgmin,
    kUnitRefine,
};

// about 2^23 polls of ~256 ns: seconds, far above any stage of a batch
constexpr uint32_t kQueueSpins = 1u << 23;

// Thread 0 of a CTA: waits until `*count` reaches `target` (bounded). False,
// with the status set, when the wait ran out or another CTA already failed.
__device__ bool persistent_wait(const unsigned int* count, unsigned int target, int* status)
{
    const volatile unsigned int* c = count;
    const volatile int* st = status;
    for (uint32_t i = 0; i < kQueueSpins; ++i) {
        if (*c >= target) {
            __threadfence();  // the counted units' writes before this CTA's reads
            return true;
        }
        if (*st != 0) {
            return false;
        }
        __nanosleep(i < 64 ? 32 : 256);
    }
    atomicOr(status, 1);
    return false;
}

template <int PER_LANE>
__device__ __forceinline__ void persistent_sample(const MedianArgs& a, uint32_t u,
                                                  uint32_t units)
{
    hierbody::median_sample_loop<PER_LANE>(a.rows, a.row_count, a.padded_p, a.p, a.queries,
                                           a.batch, a.samples, a.partials, a.min_bits, u,
                                           units, kFinalizeThreads);
}

template <int PER_LANE>
__device__ __forceinline__ void persistent_survivor(const MedianArgs& a, uint32_t u,
                                                    uint32_t units)
{
    hierbody::median_survivor_loop<PER_LANE>(a.rows, a.row_count, a.padded_p, a.p, a.queries,
                                             a.batch, a.coord_err, a.partials, a.pair_err, u,
                                             units, kFinalizeThreads);
}

template <int Q>
__device__ __forceinline__ void persistent_count(const MedianArgs& a, uint32_t b,
                                                 uint32_t gx, float* smem, uint32_t half)
{
    hierbody::median_count_block<Q>(a.rows_t, a.r_pitch, a.row_count, a.padded_p, a.p,
                                    a.queries, a.batch, 0, a.min_bits, a.query_err,
                                    a.row_err_max, a.rel, a.abs_err, a.partials, b % gx,
                                    b / gx, reinterpret_cast<float4*>(smem),
                                    threadIdx.x % hierbody::kCountRows, 1 + half);
}

// Unit u (of `units`) of one kind for one pair: one block of the stage kernel
// the standalone path launches for it.
// Units of kernel kPart's stages only (0: clear, gather, projection; 1: L2
// error roots, tile scans, median samples; 2: median counts and survivors,
// argmin, reported distances), so no kernel carries another's register
// budget.
template <int kPart>
__device__ void persistent_unit(const PersistentPair& d, uint32_t kind, uint32_t u,
                                uint32_t units, unsigned char* smem)
{
    if constexpr (kPart == 0) {
    int* error_flag = reinterpret_cast<int*>(d.counters + 1);
    switch (kind) {
    case kUnitClear: {
        const uint64_t stride = static_cast<uint64_t>(units) * kFinalizeThreads;
        for (uint64_t i = u * static_cast<uint64_t>(kFinalizeThreads) + threadIdx.x;
             i < d.batch; i += stride) {
            d.query_err[i] = 0.f;
            if (!d.l2) {
                d.median.min_bits[i] = 0xffffffffu;
            }
        }
        if (u == 0) {
            for (uint32_t i = threadIdx.x; i < d.counter_words; i += kFinalizeThreads) {
                d.counters[i] = 0;
            }
        }
        break;
    }
    case kUnitGather:
        hierbody::prepare_sampled_loop(d.raw_queries, d.batch, d.dim, d.columns, nullptr,
                                       d.sample_size, d.prepared, d.padded_sample, error_flag,
                                       u, units, kFinalizeThreads);
        break;
    case kUnitProject:
        hierbody::project_queries_block(
            d.prepared, d.batch, d.padded_sample, d.sample_size, d.projection32, d.proj_dim,
            d.projected, d.padded_p, d.query_err, d.l2 ? nullptr : d.coord_err, d.err_per_abs,
            d.l2 != 0, error_flag, u % d.proj_gx, u / d.proj_gx,
            *reinterpret_cast<hierbody::ProjShared*>(smem));
        break;
    default:
        break;
    }
    } else if constexpr (kPart == 1) {
    switch (kind) {
    case kUnitFinishErr:
        hierbody::finish_query_err_loop(d.query_err, d.batch, true, u, units, kFinalizeThreads);
        break;
    case kUnitTile: {
        const uint32_t plane = d.tile_gx * d.tile_gy;
        tilebody::tile_scan_wide_tile<static_cast<int>(ScanOp::l2)>(
            d.scan_rows, d.rows, static_cast<uint32_t>(d.padded_p), nullptr, d.projected,
            d.batch, d.k_per_split, d.partials, u % d.tile_gx, (u % plane) / d.tile_gx,
            u / plane, smem);
        break;
    }
    case kUnitSample: {
        const MedianArgs& a = d.median;
        if (a.p <= 32) {
            persistent_sample<1>(a, u, units);
        } else if (a.p <= 64) {
            persistent_sample<2>(a, u, units);
        } else if (a.p <= 128) {
            persistent_sample<4>(a, u, units);
        } else {
            persistent_sample<8>(a, u, units);
        }
        break;
    }
    default:
        break;
    }
    } else {
    switch (kind) {
    case kUnitCount: {
        // two count blocks per unit, one per half of the CTA (own barrier and
        // shared memory)
        const MedianArgs& a = d.median;
        const uint32_t half = threadIdx.x / hierbody::kCountRows;
        const uint32_t b = 2 * u + half;
        if (b < d.count_gx * d.count_gy) {
            const uint32_t q = a.count_queries;
            float* half_smem = reinterpret_cast<float*>(smem) + half * q * a.padded_p;
            if (q == 8) {
                persistent_count<8>(a, b, d.count_gx, half_smem, half);
            } else if (q == 4) {
                persistent_count<4>(a, b, d.count_gx, half_smem, half);
            } else if (q == 2) {
                persistent_count<2>(a, b, d.count_gx, half_smem, half);
            } else {
                persistent_count<1>(a, b, d.count_gx, half_smem, half);
            }
        }
        break;
    }
    case kUnitSurvivor: {
        const MedianArgs& a = d.median;
        if (a.p <= 32) {
            persistent_survivor<1>(a, u, units);
        } else if (a.p <= 64) {
            persistent_survivor<2>(a, u, units);
        } else if (a.p <= 128) {
            persistent_survivor<4>(a, u, units);
        } else {
            persistent_survivor<8>(a, u, units);
        }
        break;
    }
    case kUnitArgmin: {
        argmin_block<false, false>(d.view, d.bound, d.replay, d.results, d.exact_distances,
                            static_cast<Summary*>(d.summaries), d.done, d.counters,
                            d.argmin_span, u % d.argmin_gx, u / d.argmin_gx, d.argmin_gx,
                            reinterpret_cast<double*>(smem));
        break;
    }
    case kUnitRefine: {
        refine_group_block(d.replay, d.bound, d.results, d.exact_distances, d.batch, u, smem);
        break;
    }
    default:
        break;
    }
    }
}

// The batch in three cooperative launches: stages [0, kPersistentSplit0)
// (clear, gather, projection) at 8 CTAs per SM, stage kPersistentSplit0 (tile
// scans, median samples) with the tile scan's register budget (2 CTAs per
// SM), then the late stages [kPersistentSplit, kPersistentStages) at 4 CTAs
// per SM. Each CTA takes units
// from its kernel's queue head until the queue is drained; before a unit it
// waits for the unit's pair to have completed its units of earlier stages,
// after it counts the unit complete for its pair and its stage (the stage
// count also dates the stage's end). A wait that ran out, or a status set by
// another CTA, ends the CTA; the last CTA of the last kernel to finish zeroes
// the queue for the next run.
__device__ __forceinline__ unsigned long long global_timer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int kPart, int kFirst, int kEnd, int kMinBlocks>
__global__ void __launch_bounds__(kFinalizeThreads, kMinBlocks)
    persistent_stages_kernel(const __grid_constant__ PersistentParams params)
{
    extern __shared__ __align__(16) unsigned char persistent_smem[];
    constexpr bool kLast = kPart == kPersistentKernels - 1;
    __shared__ uint32_t next_unit;
    __shared__ int unit_ready;
    const PersistentPlan& plan = params.plan;
    unsigned int* queue = plan.queue;
    if (*static_cast<volatile int*>(plan.status) != 0) {
        return;  // the earlier kernel of this run gave up
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && plan.clock != nullptr) {
        plan.clock[kFirst] = global_timer_ns();
    }
    const uint32_t end = plan.stage_first[kEnd];
    uint32_t stage = kFirst;
    uint32_t seg = plan.stage_begin[kFirst];
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t item = end;
            if (*static_cast<volatile int*>(plan.status) == 0) {
                item = plan.stage_first[kFirst] +
                       atomicAdd(queue + kQueueHead + kPart, 1u);
            }
            next_unit = item;
        }
        __syncthreads();
        const uint32_t item = next_unit;
        if (item >= end) {
            break;
        }
        while (item >= plan.stage_first[stage + 1]) {
            ++stage;
        }
        const uint32_t u = item - plan.stage_first[stage];
        seg = max(seg, plan.stage_begin[stage]);
        while (seg + 1 < plan.stage_begin[stage + 1] && params.segments[seg + 1].first <= u) {
            ++seg;
        }
        const PersistentSegment& sg = params.segments[seg];
        if (threadIdx.x == 0) {
            unit_ready = persistent_wait(queue + kQueuePairDone + sg.pair,
                                         plan.pair_wait[sg.pair][stage], plan.status)
                             ? 1
                             : 0;
        }
        __syncthreads();
        if (unit_ready == 0) {
            return;  // the wait ran out, or another CTA's did (status set)
        }
        persistent_unit<kPart>(params.pairs[sg.pair], sg.kind, u - sg.first, sg.units,
                               persistent_smem);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();  // the unit's writes before its completion count
            atomicAdd(queue + kQueuePairDone + sg.pair, 1u);
            const unsigned int done = atomicAdd(queue + kQueueStageDone + stage, 1u) + 1u;
            if (done == plan.stage_units[stage] && plan.clock != nullptr) {
                plan.clock[stage + 1] = global_timer_ns();
            }
        }
    }
    if constexpr (kLast) {
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(queue + kQueueFinished, 1u) == gridDim.x - 1) {
                // every CTA of every kernel is past its last queue access
                __threadfence();
                for (uint32_t w = 0; w < kPersistentQueueWords; ++w) {
                    queue[w] = 0u;
                }
            }
        }
    }
}

// kernel parameters are limited to 32,764 bytes
static_assert(sizeof(PersistentParams) <= 32764, "persistent batch parameters too large");

constexpr auto persistent_gather_kernel = persistent_stages_kernel<0, 0, kPersistentSplit0, 8>;
constexpr auto persistent_scan_kernel =
    persistent_stages_kernel<1, kPersistentSplit0, kPersistentSplit, 2>;
constexpr auto persistent_late_kernel =
    persistent_stages_kernel<2, kPersistentSplit, kPersistentStages, 4>;

// Raises a kernel's dynamic shared-memory limit when a launch needs more than
// the default allows: 48 KB less the kernel's static shared memory (read once
// per kernel and device). A call that needs no more makes no runtime call
// beyond reading the current device, so captured launches after a warm-up
// make none.
void set_dynamic_smem(const void* kernel, size_t smem)
{
    // the last kernel this thread configured
    thread_local const void* last_kernel = nullptr;
    thread_local int last_device = -1;
    thread_local size_t last_ok = 0;
    const int device = current_device();
    if (kernel == last_kernel && device == last_device && smem <= last_ok) {
        return;
    }
    static std::mutex mutex;
    // dynamic bytes a launch may use without raising the limit again
    static std::map<std::pair<int, const void*>, size_t> launchable;
    std::lock_guard<std::mutex> lock(mutex);
    auto it = launchable.find({device, kernel});
    if (it == launchable.end()) {
        cudaFuncAttributes attr{};
        check_cuda(cudaFuncGetAttributes(&attr, kernel), "cannot read kernel attributes");
        const size_t base =
            attr.sharedSizeBytes < 48 * 1024 ? 48 * 1024 - attr.sharedSizeBytes : 0;
        it = launchable.emplace(std::make_pair(device, kernel), base).first;
    }
    if (smem > it->second) {
        check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)),
                   "cannot configure kernel shared memory");
        it->second = smem;
    }
    last_kernel = kernel;
    last_device = device;
    last_ok = it->second;
}

size_t replay_smem(const ReplayInputs& in)
{
    return projected_op(in.op) ? in.proj_dim * sizeof(double) : 0;
}
// Carves the argmin scratch region: per-(query, row block) summaries and the
// per-query completion counters (zero between calls). The layout depends only
// on the workspace capacity, never on the batch of one call, so the counters
// stay at fixed addresses across calls.
struct FinalizeScratch {
    Summary* summaries;
    uint32_t* done;
};

FinalizeScratch finalize_scratch(void* base, uint32_t capacity, uint32_t rows)
{
    const uint64_t blocks = (rows + kFinalizeThreads - 1) / kFinalizeThreads;
    char* p = static_cast<char*>(base);
    FinalizeScratch fs;
    fs.summaries = reinterpret_cast<Summary*>(p);
    p += capacity * blocks * sizeof(Summary);
    p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
    fs.done = reinterpret_cast<uint32_t*>(p);
    return fs;
}

}  // namespace

void launch_refine_winners(ReplayInputs in, Bound bound, const Result* results,
                           uint32_t batch, double* exact_distances,
                           cudaStream_t stream)
{
    static_assert(kRefineGroup <= kFinalizeThreads / 32, "one warp per group member");
    const size_t group_smem =
        kRefineGroup * (in.proj_dim * sizeof(double) + in.dim * sizeof(float));
    if (group_smem <= 200 * 1024) {
        set_dynamic_smem(reinterpret_cast<const void*>(refine_group_kernel), group_smem);
        refine_group_kernel<<<(batch + kRefineGroup - 1) / kRefineGroup, kFinalizeThreads,
                              group_smem, stream>>>(in, bound, results, exact_distances,
                                                    batch);
    } else {
        const size_t smem = replay_smem(in);
        set_dynamic_smem(reinterpret_cast<const void*>(refine_kernel), smem);
        refine_kernel<<<batch, kFinalizeThreads, smem, stream>>>(in, bound, results,
                                                                 exact_distances);
    }
    check_cuda(cudaGetLastError(), "cannot launch refine kernel");
}

uint64_t finalize_scratch_bytes(uint64_t batch, uint64_t rows)
{
    const uint64_t blocks = (rows + kFinalizeThreads - 1) / kFinalizeThreads;
    return batch * blocks * sizeof(Summary) + batch * sizeof(uint32_t) + 64;
}

void launch_argmin(PartialView view, Bound bound, ReplayInputs in,
                   Result* results, double* exact_distances, void* scratch,
                   uint64_t capacity, uint32_t* replay_count, cudaStream_t stream)
{
    // Rows per CTA: one block of kFinalizeThreads rows, or several when the
    // grid would exceed about 32 CTAs per SM (the scratch layout stays that of
    // one block per kFinalizeThreads rows, so the counters keep their place).
    const uint32_t min_span_blocks = (view.rows + kFinalizeThreads - 1) / kFinalizeThreads;
    const uint64_t cap = 148ull * 32;
    const uint64_t want = static_cast<uint64_t>(min_span_blocks) * view.batch;
    const uint32_t factor = want > cap ? static_cast<uint32_t>((want + cap - 1) / cap) : 1u;
    const uint32_t span = kFinalizeThreads * factor;
    const uint32_t blocks = (view.rows + span - 1) / span;
    FinalizeScratch fs = finalize_scratch(scratch, static_cast<uint32_t>(capacity),
                                          view.rows);
    const size_t smem = replay_smem(in);
    const auto kernel = in.emulated ? argmin_kernel<true> : argmin_kernel<false>;
    set_dynamic_smem(reinterpret_cast<const void*>(kernel), smem);
    kernel<<<dim3(blocks, view.batch), kFinalizeThreads, smem, stream>>>(
        view, bound, in, results, exact_distances, fs.summaries, fs.done,
        replay_count, span);
    check_cuda(cudaGetLastError(), "cannot launch argmin kernel");
}

void launch_rescore_projected(const uint32_t* candidates, uint32_t k, uint32_t batch,
                              const double* rows64, const double* y64, uint32_t p,
                              Result* results, double* exact_distances,
                              cudaStream_t stream)
{
    rescore_projected_kernel<<<batch, kFinalizeThreads, 0, stream>>>(
        candidates, k, rows64, y64, p, results, exact_distances);
    check_cuda(cudaGetLastError(), "cannot launch projected re-score kernel");
}

uint32_t rescore_depth(uint64_t padded_dim)
{
    const uint64_t groups = padded_dim / 4;
    return static_cast<uint32_t>((groups + kFinalizeThreads - 1) / kFinalizeThreads) + 10;
}

uint32_t max_rerank_candidates()
{
    return kMaxCandidates;
}

void launch_rescore(Bound64 bound, ReplayInputs in, const uint32_t* candidates,
                    uint32_t k, uint32_t batch, uint32_t rows, double* cand_dist,
                    uint32_t* done, Result* results, double* exact_distances,
                    uint32_t* replay_count, cudaStream_t stream)
{
    if (batch == 0 || k == 0) {
        return;
    }
    rescore_kernel<<<dim3(k, batch), kFinalizeThreads, 0, stream>>>(
        bound, in, candidates, k, rows, cand_dist, done, results, exact_distances,
        replay_count);
    check_cuda(cudaGetLastError(), "cannot launch re-score kernel");
}

void launch_rescore32(Bound bound, ReplayInputs in, const uint32_t* candidates,
                      uint32_t k, uint32_t batch, uint32_t rows, float* cand_dist,
                      uint32_t* done, Result* results, double* exact_distances,
                      uint32_t* replay_count, cudaStream_t stream)
{
    if (batch == 0 || k == 0) {
        return;
    }
    rescore32_kernel<<<dim3(k, batch), kFinalizeThreads, 0, stream>>>(
        bound, in, candidates, k, rows, cand_dist, done, results, exact_distances,
        replay_count);
    check_cuda(cudaGetLastError(), "cannot launch FP32 re-score kernel");
}

void emulated_replay_bound(uint64_t dim, float* rel, float* abs)
{
    // float-float: terms within 2^-45, each lane's chain of ceil(dim / 32)
    // additions and five butterfly levels at 2^-45 each; the reference CPU's
    // own binary64 rounding, gamma(dim + 3); binary32 underflow of tiny terms
    // as an absolute term
    const double u = std::ldexp(1.0, -53);
    const double n64 = static_cast<double>(dim) + 3;
    const double chain = static_cast<double>((dim + 31) / 32) + 7;
    const double r = 1.01 * (chain * std::ldexp(1.0, -45) + n64 * u / (1.0 - n64 * u)) +
                     std::ldexp(1.0, -40);
    *rel = std::nextafter(static_cast<float>(r), 1.0f);
    *abs = static_cast<float>((2.0 * static_cast<double>(dim) + 16.0) * std::ldexp(1.0, -148));
}

bool small_query_fits(uint64_t rows, uint64_t padded_dim)
{
    return rows >= 1 && rows <= kSmallRows && padded_dim <= kSmallColumns &&
           rows * padded_dim <= kSmallCells;
}

uint32_t small_query_depth(uint64_t padded_dim)
{
    const uint64_t groups = padded_dim / 4;
    return static_cast<uint32_t>(4 * ((groups + 31) / 32) + 5);
}

void launch_small_query(const SmallQuery& sq, uint32_t batch, Bound bound, ReplayInputs in,
                        Result* results, double* exact_distances, uint32_t* replay_count,
                        int* error_flag, cudaStream_t stream)
{
    if (batch == 0) {
        return;
    }
    const size_t smem = (sq.padded_dim + sq.row_count) * sizeof(float);
    const auto kernel = in.emulated ? small_query_kernel<true> : small_query_kernel<false>;
    kernel<<<batch, kFinalizeThreads, smem, stream>>>(
        sq, bound, in, results, exact_distances, replay_count, error_flag);
    check_cuda(cudaGetLastError(), "cannot launch small-index query kernel");
}

bool flat_query_fits(uint64_t rows, uint64_t padded_dim, uint64_t batch)
{
    return rows >= 1 && rows <= 0x7fffffffull && padded_dim >= 4 &&
           padded_dim <= kFlatColumns && batch >= 1 && batch <= kFlatBatch;
}

FlatPlan plan_flat_query(uint64_t rows, uint64_t padded_dim, uint64_t batch,
                         int sm_count)
{
    const uint64_t groups = padded_dim / 4;
    // lanes per row: enough float4 groups per lane (about four or more) to
    // keep several loads in flight, at least 8 lanes
    uint32_t lanes = 32;
    if (groups < 32 * 4) {
        lanes = groups < 16 * 4 ? 8 : 16;
    }
    const uint32_t step = kFinalizeThreads / lanes;  // rows per CTA pass
    // about three CTAs per SM over the whole launch (one wave)
    const uint64_t target = static_cast<uint64_t>(sm_count) * 3;
    const uint64_t per_query = std::max<uint64_t>(1, target / batch);
    uint64_t span = (rows + per_query - 1) / per_query;
    span = std::max<uint64_t>(step, (span + step - 1) / step * step);
    FlatPlan plan;
    plan.lanes = lanes;
    plan.span = static_cast<uint32_t>(span);
    plan.blocks = static_cast<uint32_t>((rows + span - 1) / span);
    // rows per bulk copy: whole passes of the CTA up to kFlatChunkBytes; rows
    // too long for one pass in a copy (a pass would leave most threads idle
    // and serialise many small copies) are read from global memory directly
    // (chunk_rows 0)
    const uint64_t row_bytes = padded_dim * sizeof(float);
    const uint64_t chunk = kFlatChunkBytes / row_bytes / step * step;
    plan.chunk_rows = static_cast<uint32_t>(std::min<uint64_t>(chunk, span));
    plan.buffers = plan.chunk_rows == 0 ? 0u : plan.chunk_rows >= span ? 1u : 2u;
    uint32_t log_lanes = 0;
    while ((1u << log_lanes) < lanes) {
        ++log_lanes;
    }
    plan.depth = static_cast<uint32_t>(4 * ((groups + lanes - 1) / lanes) + log_lanes);
    return plan;
}

namespace {

// Scratch of the fused flat query for a workspace of `capacity` queries:
// slots (two per stream lane; consecutive launches on a stream alternate),
// each with the distance slabs, the
// CTA summaries (room for the most CTAs any plan uses) and the per-query
// completion counters at a fixed place (zero between launches).
struct FlatScratch {
    float* distances;
    Summary* summaries;
    uint32_t* done;
    uint32_t summary_stride;
};

uint64_t round_up(uint64_t v, uint64_t to)
{
    return (v + to - 1) / to * to;
}

uint64_t flat_max_blocks(uint64_t rows)
{
    return (rows + 7) / 8;  // span >= 8 rows
}

// offsets within a slot (the scratch starts 256-byte aligned)
uint64_t flat_summaries_offset(uint64_t capacity, uint64_t rows)
{
    return round_up(capacity * rows * sizeof(float), 16);
}

uint64_t flat_done_offset(uint64_t capacity, uint64_t rows)
{
    return round_up(flat_summaries_offset(capacity, rows) +
                        capacity * flat_max_blocks(rows) * sizeof(Summary),
                    16);
}

uint64_t flat_slot_bytes(uint64_t capacity, uint64_t rows)
{
    return round_up(flat_done_offset(capacity, rows) + capacity * sizeof(uint32_t), 256);
}

FlatScratch flat_scratch(void* base, uint64_t capacity, uint64_t rows, uint32_t slot)
{
    char* p = static_cast<char*>(base) + slot * flat_slot_bytes(capacity, rows);
    FlatScratch fs;
    fs.distances = reinterpret_cast<float*>(p);
    fs.summaries = reinterpret_cast<Summary*>(p + flat_summaries_offset(capacity, rows));
    fs.done = reinterpret_cast<uint32_t*>(p + flat_done_offset(capacity, rows));
    fs.summary_stride = static_cast<uint32_t>(flat_max_blocks(rows));
    return fs;
}

template <int kLanes>
void launch_flat_lanes(const SmallQuery& sq, const FlatPlan& plan, uint32_t batch,
                       Bound bound, ReplayInputs in, const FlatScratch& fs,
                       Result* results, double* exact_distances, uint32_t* replay_count,
                       int* error_flag, cudaStream_t stream)
{
    // the gathered query (and the column weights of a weighted L1 index),
    // then the copy buffers of the rows
    const size_t smem =
        sq.padded_dim * sizeof(float) *
        ((sq.op == static_cast<int>(ScanOp::l1_weighted) ? 2 : 1) +
         static_cast<size_t>(plan.buffers) * plan.chunk_rows);
    const auto kernel =
        in.emulated ? flat_query_kernel<kLanes, true> : flat_query_kernel<kLanes, false>;
    set_dynamic_smem(reinterpret_cast<const void*>(kernel), smem);
    cudaLaunchConfig_t config{};
    config.gridDim = dim3(plan.blocks, batch);
    config.blockDim = dim3(kFinalizeThreads);
    config.dynamicSmemBytes = smem;
    config.stream = stream;
    cudaLaunchAttribute attr[1];
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(stream, &capture), "cannot query stream capture");
    if (capture == cudaStreamCaptureStatusNone) {
        // this grid's gather and scan overlap the end of the previous one
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        config.attrs = attr;
        config.numAttrs = 1;
    }
    check_cuda(cudaLaunchKernelEx(&config, kernel, sq, bound, in, fs.distances,
                                  fs.summaries, fs.done, fs.summary_stride, plan.span,
                                  plan.chunk_rows, results, exact_distances, replay_count,
                                  error_flag),
               "cannot launch flat query kernel");
}

}  // namespace

uint64_t flat_query_scratch_bytes(uint64_t capacity, uint64_t rows, uint32_t slots)
{
    return slots * flat_slot_bytes(capacity, rows);
}

void launch_flat_query(const SmallQuery& sq, const FlatPlan& plan, uint32_t batch,
                       Bound bound, ReplayInputs in, void* scratch, uint64_t capacity,
                       uint32_t slot, Result* results, double* exact_distances,
                       uint32_t* replay_count, int* error_flag, cudaStream_t stream)
{
    if (batch == 0) {
        return;
    }
    const FlatScratch fs = flat_scratch(scratch, capacity, sq.row_count, slot);
    if (plan.lanes == 8) {
        launch_flat_lanes<8>(sq, plan, batch, bound, in, fs, results, exact_distances,
                             replay_count, error_flag, stream);
    } else if (plan.lanes == 16) {
        launch_flat_lanes<16>(sq, plan, batch, bound, in, fs, results, exact_distances,
                              replay_count, error_flag, stream);
    } else {
        launch_flat_lanes<32>(sq, plan, batch, bound, in, fs, results, exact_distances,
                              replay_count, error_flag, stream);
    }
}

void launch_finalize_gemm(PartialView view, const float* row_norms,
                          const float* query_norms, Result* results,
                          cudaStream_t stream)
{
    finalize_gemm_kernel<<<view.batch, kFinalizeThreads, 0, stream>>>(
        view, row_norms, query_norms, results);
    check_cuda(cudaGetLastError(), "cannot launch gemm finalize kernel");
}

// ------------------------------------ shapes for the persistent batch kernel

void argmin_grid(uint32_t rows, uint32_t batch, uint32_t* gx, uint32_t* span)
{
    // launch_argmin's shape
    const uint32_t min_span_blocks = (rows + kFinalizeThreads - 1) / kFinalizeThreads;
    const uint64_t cap = 148ull * 32;
    const uint64_t want = static_cast<uint64_t>(min_span_blocks) * batch;
    const uint32_t factor = want > cap ? static_cast<uint32_t>((want + cap - 1) / cap) : 1u;
    *span = kFinalizeThreads * factor;
    *gx = (rows + *span - 1) / *span;
}

void argmin_scratch(void* scratch, uint64_t capacity, uint32_t rows, void** summaries,
                    uint32_t** done)
{
    const FinalizeScratch fs = finalize_scratch(scratch, static_cast<uint32_t>(capacity), rows);
    *summaries = fs.summaries;
    *done = fs.done;
}

uint64_t replay_smem_bytes(const ReplayInputs& in)
{
    return replay_smem(in);
}

uint64_t refine_group_smem_bytes(const ReplayInputs& in)
{
    return kRefineGroup * (in.proj_dim * sizeof(double) + in.dim * sizeof(float));
}

uint32_t refine_group_blocks(uint32_t batch)
{
    return (batch + kRefineGroup - 1) / kRefineGroup;
}

// ------------------------------------------ the persistent batch (host side)

uint32_t persistent_segment_capacity(uint32_t count)
{
    // at most two unit kinds per pair in any stage
    return 2 * count * kPersistentStages + 1;
}

void plan_persistent_batch(const PersistentPair* pairs, uint32_t count,
                           PersistentSegment* segments, uint32_t* segment_count,
                           PersistentPlan* plan)
{
    uint32_t n = 0;
    uint64_t smem_group[kPersistentKernels] = {};
    uint64_t smem = 0;
    auto add = [&](int stage, uint32_t pair, uint32_t kind, uint64_t units) {
        if (units == 0) {
            return;
        }
        const uint64_t total = static_cast<uint64_t>(plan->stage_units[stage]) + units;
        if (total > 0xffffffffull) {
            fail(UHA_LENGTH_ERROR, "persistent batch stage exceeds 2^32 units");
        }
        PersistentSegment sg{};
        sg.pair = pair;
        sg.kind = kind;
        sg.units = static_cast<uint32_t>(units);
        sg.first = plan->stage_units[stage];
        plan->stage_units[stage] = static_cast<uint32_t>(total);
        segments[n++] = sg;
    };
    for (int stage = 0; stage < kPersistentStages; ++stage) {
        plan->stage_units[stage] = 0;
    }
    for (int stage = 0; stage < kPersistentStages; ++stage) {
        plan->stage_begin[stage] = n;
        smem = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const PersistentPair& d = pairs[i];
            const uint64_t per_query = (d.batch + kFinalizeThreads - 1) / kFinalizeThreads;
            switch (stage) {
            case 0:
                add(0, i, kUnitClear, std::max<uint64_t>(1, per_query));
                break;
            case 1: {
                const uint64_t total = d.batch * d.padded_sample;
                const uint64_t blocks = (total + kFinalizeThreads - 1) / kFinalizeThreads;
                add(1, i, kUnitGather,
                    std::max<uint64_t>(1, std::min<uint64_t>(blocks, 148ull * 64)));
                break;
            }
            case 2:
                add(2, i, kUnitProject, static_cast<uint64_t>(d.proj_gx) * d.proj_gy);
                smem = std::max<uint64_t>(smem, project_queries_smem_bytes());
                break;
            case 3:
                if (d.l2) {
                    add(3, i, kUnitFinishErr, std::max<uint64_t>(1, per_query));
                    add(3, i, kUnitTile,
                        static_cast<uint64_t>(d.tile_gx) * d.tile_gy * d.tile_gz);
                    smem = std::max<uint64_t>(smem, tile_scan_smem_bytes());
                } else {
                    add(3, i, kUnitSample, d.sample_blocks);
                }
                break;
            case 4:
                if (!d.l2) {
                    add(4, i, kUnitCount,
                        (static_cast<uint64_t>(d.count_gx) * d.count_gy + 1) / 2);
                    smem = std::max<uint64_t>(
                        smem, 2ull * d.median.count_queries * d.padded_p * sizeof(float));
                }
                break;
            case 5:
                if (d.l2) {
                    add(5, i, kUnitArgmin, static_cast<uint64_t>(d.argmin_gx) * d.batch);
                    smem = std::max<uint64_t>(smem, replay_smem(d.replay));
                } else {
                    add(5, i, kUnitSurvivor, d.survivor_blocks);
                }
                break;
            case 6:
                if (d.l2) {
                    add(6, i, kUnitRefine, d.refine_blocks);
                    smem = std::max<uint64_t>(smem, refine_group_smem_bytes(d.replay));
                } else {
                    add(6, i, kUnitArgmin, static_cast<uint64_t>(d.argmin_gx) * d.batch);
                    smem = std::max<uint64_t>(smem, replay_smem(d.replay));
                }
                break;
            default:
                if (!d.l2) {
                    add(7, i, kUnitRefine, d.refine_blocks);
                    smem = std::max<uint64_t>(smem, refine_group_smem_bytes(d.replay));
                }
                break;
            }
        }
        uint64_t& group = smem_group[persistent_part_of(stage)];
        group = std::max(group, smem);
    }
    plan->stage_begin[kPersistentStages] = n;
    // queue positions of the stages and the per-pair completion targets
    uint64_t first = 0;
    for (int stage = 0; stage < kPersistentStages; ++stage) {
        plan->stage_first[stage] = static_cast<uint32_t>(first);
        first += plan->stage_units[stage];
        if (first > 0xffffffffull) {
            fail(UHA_LENGTH_ERROR, "persistent batch exceeds 2^32 units");
        }
    }
    plan->stage_first[kPersistentStages] = static_cast<uint32_t>(first);
    for (uint32_t i = 0; i < kPersistentMaxPairs; ++i) {
        uint64_t before = 0;
        for (int stage = 0; stage < kPersistentStages; ++stage) {
            plan->pair_wait[i][stage] = static_cast<uint32_t>(before);
            for (uint32_t g = plan->stage_begin[stage]; g < plan->stage_begin[stage + 1]; ++g) {
                if (segments[g].pair == i) {
                    before += segments[g].units;
                }
            }
        }
    }
    for (int k = 0; k < kPersistentKernels; ++k) {
        plan->smem_bytes[k] = static_cast<uint32_t>((smem_group[k] + 15) / 16 * 16);
    }
    *segment_count = n;
}

namespace {

const void* persistent_kernel(int part)
{
    return part == 0   ? reinterpret_cast<const void*>(persistent_gather_kernel)
           : part == 1 ? reinterpret_cast<const void*>(persistent_scan_kernel)
                       : reinterpret_cast<const void*>(persistent_late_kernel);
}

}  // namespace

uint32_t persistent_grid(int part, uint32_t smem_bytes)
{
    const void* kernel = persistent_kernel(part);
    set_dynamic_smem(kernel, smem_bytes);
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kFinalizeThreads,
                                                             smem_bytes),
               "cannot size the persistent batch kernel");
    int sms = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, current_device()),
               "cannot query the SM count");
    return static_cast<uint32_t>(std::max(0, per_sm) * sms);
}

void launch_persistent_batch(const PersistentParams& params,
                             const uint32_t grid[kPersistentKernels], cudaStream_t stream)
{
    const PersistentPlan& plan = params.plan;
    for (int part = 0; part < kPersistentKernels; ++part) {
        const void* kernel = persistent_kernel(part);
        set_dynamic_smem(kernel, plan.smem_bytes[part]);
        cudaLaunchConfig_t config{};
        config.gridDim = dim3(grid[part]);
        config.blockDim = dim3(kFinalizeThreads);
        config.dynamicSmemBytes = plan.smem_bytes[part];
        config.stream = stream;
        cudaLaunchAttribute attr[1];
        // every CTA resident at once: a unit never waits for one taken by a
        // CTA that has not started
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        config.attrs = attr;
        config.numAttrs = 1;
        void* args[] = {const_cast<PersistentParams*>(&params)};
        check_cuda(cudaLaunchKernelExC(&config, kernel, args),
                   "cannot launch the persistent batch kernel");
    }
}

}  // namespace uha
