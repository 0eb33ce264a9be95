// Importance probabilities on the device.
//
// Reference semantics (src/hnsvw25/l2/importance_sampling.cpp:19-45,
// src/hnsvw25/l1/importance_sampling.cpp:19-47): for every pair of rows a < b
// with nonzero distance, L2 contributes min(1, (a_j - b_j)^2 / ||a - b||^2) and
// L1 contributes |a_j - b_j| / ||a - b||_1 to column j; p_j is the maximum
// contribution. Pair distances and the per-column maxima use binary64 (the
// normalisation of the probabilities). The direct backend performs the CPU's
// own operations in the CPU's order (sequential squared differences for L2,
// libstdc++'s transform_reduce grouping for L1, one IEEE division per pair,
// the same two roundings per contribution) and the maximum is exact, so its
// probabilities equal the reference CPU's bit for bit. The Gram backend
// agrees to a few ulps.
//
// Stage 1 (pair kernel): a 32 x 32 block of pairs per CTA, columns staged
// through shared memory in 64-column slabs; each thread accumulates four
// pairs. The inverse distance of every pair a < b (0 for zero distance and for
// a >= b) is written to an r x r matrix.
// Stage 2 (column kernel): a CTA owns 256 columns and one 32-row block A and
// walks every row block B >= A; per pair the contribution is formed with the
// inverse distance and folded into a per-column maximum. Zero inverse
// distances contribute 0, so no branch is needed. Column maxima are combined
// across CTAs with a 64-bit atomicMax on the bit pattern (nonnegative binary64
// values order like their bit patterns).
#include "common.h"
#include "kernels.h"

#include <algorithm>

namespace uha {
namespace {

constexpr int kPairBlock = 32;
constexpr int kPairSlab = 64;
constexpr int kColumns = 256;

__global__ void __launch_bounds__(256)
    pair_distance_kernel(int metric, const float* __restrict__ rows,
                         uint32_t row_count, uint64_t dim,
                         double* __restrict__ inverse)
{
    const uint32_t ta = blockIdx.y;
    const uint32_t tb = blockIdx.x;
    if (tb < ta) {
        return;
    }
    // the slabs converted to binary64 once as they are staged (the values are
    // exact), not once per pair in the loops below
    __shared__ double sa[kPairBlock][kPairSlab + 1];
    __shared__ double sb[kPairBlock][kPairSlab + 1];
    const int ty = threadIdx.x / 8;  // 0..31: row a within block
    const int tx = threadIdx.x % 8;  // b = tx + 8 j
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const uint32_t a0 = ta * kPairBlock;
    const uint32_t b0 = tb * kPairBlock;
    for (uint64_t c0 = 0; c0 < dim; c0 += kPairSlab) {
        for (int i = threadIdx.x; i < kPairBlock * kPairSlab; i += blockDim.x) {
            const int r = i / kPairSlab;
            const int c = i % kPairSlab;
            const uint64_t col = c0 + c;
            float va = 0.f;
            float vb = 0.f;
            if (col < dim) {
                if (a0 + r < row_count) {
                    va = rows[static_cast<uint64_t>(a0 + r) * dim + col];
                }
                if (b0 + r < row_count) {
                    vb = rows[static_cast<uint64_t>(b0 + r) * dim + col];
                }
            }
            sa[r][c] = static_cast<double>(va);
            sb[r][c] = static_cast<double>(vb);
        }
        __syncthreads();
        if (metric == 0) {
            // squared_l2_dist: sequential binary64 sum of separately rounded
            // squares, column order (src/core/l2_distance.cpp:17-23)
#pragma unroll 4
            for (int c = 0; c < kPairSlab; ++c) {
                const double va = sa[ty][c];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double d = __dsub_rn(va, sb[tx + 8 * j][c]);
                    acc[j] = __dadd_rn(acc[j], __dmul_rn(d, d));
                }
            }
        } else {
            // l1_dist: std::transform_reduce as libstdc++ 13 evaluates it
            // (src/core/l1_distance.cpp:17-26): init + ((t0 + t1) + (t2 + t3))
            // per group of four from column 0, then the last dim % 4 columns
            // one by one. Slabs are 64 columns, so groups never straddle one.
            const uint64_t grouped_end = dim & ~uint64_t(3);
            for (int c = 0; c < kPairSlab; c += 4) {
                if (c0 + c + 4 <= grouped_end) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const double* vb = &sb[tx + 8 * j][c];
                        const double t0 = fabs(__dsub_rn(sa[ty][c], vb[0]));
                        const double t1 = fabs(__dsub_rn(sa[ty][c + 1], vb[1]));
                        const double t2 = fabs(__dsub_rn(sa[ty][c + 2], vb[2]));
                        const double t3 = fabs(__dsub_rn(sa[ty][c + 3], vb[3]));
                        acc[j] = __dadd_rn(acc[j], __dadd_rn(__dadd_rn(t0, t1),
                                                             __dadd_rn(t2, t3)));
                    }
                } else {
                    for (int e = 0; e < 4 && c0 + c + e < dim; ++e) {
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            acc[j] = __dadd_rn(
                                acc[j], fabs(__dsub_rn(sa[ty][c + e],
                                                       sb[tx + 8 * j][c + e])));
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    const uint32_t a = a0 + ty;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t b = b0 + tx + 8 * j;
        if (a < row_count && b < row_count && a < b && acc[j] != 0.0) {
            inverse[static_cast<uint64_t>(a) * row_count + b] = 1.0 / acc[j];
        }
    }
}

// Gram backend, stage 1: G[a][b] = sum_j a_j b_j in binary64 for a <= b,
// same tiling as the pair kernel.
__global__ void __launch_bounds__(256)
    gram_kernel(const float* __restrict__ rows, uint32_t row_count, uint64_t dim,
                double* __restrict__ gram)
{
    const uint32_t ta = blockIdx.y;
    const uint32_t tb = blockIdx.x;
    if (tb < ta) {
        return;
    }
    __shared__ float sa[kPairBlock][kPairSlab + 1];
    __shared__ float sb[kPairBlock][kPairSlab + 1];
    const int ty = threadIdx.x / 8;
    const int tx = threadIdx.x % 8;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const uint32_t a0 = ta * kPairBlock;
    const uint32_t b0 = tb * kPairBlock;
    for (uint64_t c0 = 0; c0 < dim; c0 += kPairSlab) {
        for (int i = threadIdx.x; i < kPairBlock * kPairSlab; i += blockDim.x) {
            const int r = i / kPairSlab;
            const int c = i % kPairSlab;
            const uint64_t col = c0 + c;
            float va = 0.f;
            float vb = 0.f;
            if (col < dim) {
                if (a0 + r < row_count) {
                    va = rows[static_cast<uint64_t>(a0 + r) * dim + col];
                }
                if (b0 + r < row_count) {
                    vb = rows[static_cast<uint64_t>(b0 + r) * dim + col];
                }
            }
            sa[r][c] = va;
            sb[r][c] = vb;
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < kPairSlab; ++c) {
            const double va = sa[ty][c];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc[j] = fma(va, static_cast<double>(sb[tx + 8 * j][c]), acc[j]);
            }
        }
        __syncthreads();
    }
    const uint32_t a = a0 + ty;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t b = b0 + tx + 8 * j;
        if (a < row_count && b < row_count && a <= b) {
            gram[static_cast<uint64_t>(a) * row_count + b] = acc[j];
        }
    }
}

// Gram backend, stage 2: ||a - b||^2 = G_aa + G_bb - 2 G_ab. The identity's
// absolute error is at most about (dim + 2) * 2^-53 * (G_aa + G_bb); pairs
// where that could exceed 2^-24 of the result (binary32-level accuracy) are
// recomputed directly as a binary64 sum of squared differences.
__global__ void gram_to_inverse_kernel(const double* __restrict__ gram,
                                       const float* __restrict__ rows,
                                       uint32_t row_count, uint64_t dim,
                                       double* __restrict__ inverse)
{
    const uint64_t pairs = static_cast<uint64_t>(row_count) * row_count;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         idx < pairs; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t a = static_cast<uint32_t>(idx / row_count);
        const uint32_t b = static_cast<uint32_t>(idx - uint64_t(a) * row_count);
        if (a >= b) {
            continue;
        }
        const double na = gram[uint64_t(a) * row_count + a];
        const double nb = gram[uint64_t(b) * row_count + b];
        double sd = na + nb - 2.0 * gram[idx];
        const double cancellation =
            static_cast<double>(dim + 2) * 1.1102230246251565e-16 * 16777216.0;
        if (!(sd > cancellation * (na + nb))) {
            const float* ra = rows + uint64_t(a) * dim;
            const float* rb = rows + uint64_t(b) * dim;
            sd = 0.0;
            for (uint64_t j = 0; j < dim; ++j) {
                const double d = static_cast<double>(ra[j]) - static_cast<double>(rb[j]);
                sd = fma(d, d, sd);
            }
        }
        inverse[idx] = sd != 0.0 ? 1.0 / sd : 0.0;
    }
}

__global__ void __launch_bounds__(kColumns)
    coordinate_max_kernel(int metric, const float* __restrict__ rows,
                          uint32_t row_count, uint64_t dim,
                          const double* __restrict__ inverse,
                          unsigned long long* __restrict__ maxima_bits,
                          uint32_t first_block, uint64_t pair_begin,
                          uint64_t pair_end)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double* sinv = reinterpret_cast<double*>(smem);                 // [32][32]
    float* sa = reinterpret_cast<float*>(sinv + kPairBlock * kPairBlock);  // [32][256]
    float* sb = sa + kPairBlock * kColumns;                          // [32][256]

    const uint64_t col = blockIdx.x * static_cast<uint64_t>(kColumns) +
                         threadIdx.x;
    const uint32_t ta = first_block + blockIdx.y;
    const uint32_t a0 = ta * kPairBlock;
    const uint32_t blocks = (row_count + kPairBlock - 1) / kPairBlock;
    const uint64_t r64 = row_count;

    for (int r = 0; r < kPairBlock; ++r) {
        float v = 0.f;
        if (a0 + r < row_count && col < dim) {
            v = rows[static_cast<uint64_t>(a0 + r) * dim + col];
        }
        sa[r * kColumns + threadIdx.x] = v;
    }
    double m = 0.0;
    for (uint32_t tb = ta; tb < blocks; ++tb) {
        const uint32_t b0 = tb * kPairBlock;
        __syncthreads();
        for (int r = 0; r < kPairBlock; ++r) {
            float v = 0.f;
            if (b0 + r < row_count && col < dim) {
                v = rows[static_cast<uint64_t>(b0 + r) * dim + col];
            }
            sb[r * kColumns + threadIdx.x] = v;
        }
        for (int i = threadIdx.x; i < kPairBlock * kPairBlock; i += blockDim.x) {
            const int ra = i / kPairBlock;
            const int rb = i % kPairBlock;
            double v = 0.0;
            const uint64_t a = a0 + ra;
            const uint64_t b = b0 + rb;
            if (a < b && b < row_count) {
                // position of (a, b) in the row-major order of pairs a < b;
                // pairs outside this launch's chunk contribute nothing
                const uint64_t pair = a * (2 * r64 - a - 1) / 2 + (b - a - 1);
                if (pair >= pair_begin && pair < pair_end) {
                    v = inverse[a * row_count + b];
                }
            }
            sinv[i] = v;
        }
        __syncthreads();
        {
            for (int ra = 0; ra < kPairBlock; ++ra) {
                const double va = sa[ra * kColumns + threadIdx.x];
#pragma unroll 8
                for (int rb = 0; rb < kPairBlock; ++rb) {
                    const double d =
                        __dsub_rn(va, static_cast<double>(sb[rb * kColumns + threadIdx.x]));
                    const double w = sinv[ra * kPairBlock + rb];
                    // (d * d) * inverse or |d| * inverse, each product rounded
                    // as the CPU rounds it (importance_sampling.cpp:36-41 of
                    // l2, :26-30 of l1)
                    const double c = metric == 0 ? __dmul_rn(__dmul_rn(d, d), w)
                                                 : __dmul_rn(fabs(d), w);
                    m = fmax(m, c);
                }
            }
        }
    }
    if (col < dim && m > 0.0) {
        atomicMax(maxima_bits + col,
                  static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// The binary32 form of coordinate_max_kernel's fold (the same pairs, the
// same contributions rounded in binary32: within 3e-7 relative), arranged for
// the binary32 pipe: each thread's 32 values of its column of row blocks A and
// B stay in registers (every thread reads only its own column), a pair
// block's inverse distances are rounded to binary32 once in shared memory, and
// the 32 x 32 pairs are unrolled: about four binary32 instructions per
// pair-column. A pair block holding a distance below 2^-100 is folded in
// binary64, exactly as coordinate_max_kernel folds it.
__global__ void __launch_bounds__(kColumns)
    coordinate_max32_kernel(int metric, const float* __restrict__ rows,
                            uint32_t row_count, uint64_t dim,
                            const double* __restrict__ inverse,
                            unsigned long long* __restrict__ maxima_bits,
                            uint32_t first_block, uint64_t pair_begin, uint64_t pair_end)
{
    __shared__ __align__(16) float sw[kPairBlock * kPairBlock];
    __shared__ double sw64[kPairBlock * kPairBlock];
    const uint64_t col = blockIdx.x * static_cast<uint64_t>(kColumns) + threadIdx.x;
    const uint32_t ta = first_block + blockIdx.y;
    const uint32_t a0 = ta * kPairBlock;
    const uint32_t blocks = (row_count + kPairBlock - 1) / kPairBlock;
    const uint64_t r64 = row_count;
    float va[kPairBlock];
#pragma unroll
    for (int r = 0; r < kPairBlock; ++r) {
        va[r] = a0 + r < row_count && col < dim
                    ? rows[static_cast<uint64_t>(a0 + r) * dim + col]
                    : 0.f;
    }
    float m32[4] = {0.f, 0.f, 0.f, 0.f};  // four chains of the maximum
    double m = 0.0;
    for (uint32_t tb = ta; tb < blocks; ++tb) {
        const uint32_t b0 = tb * kPairBlock;
        float vb[kPairBlock];
#pragma unroll
        for (int r = 0; r < kPairBlock; ++r) {
            vb[r] = b0 + r < row_count && col < dim
                        ? rows[static_cast<uint64_t>(b0 + r) * dim + col]
                        : 0.f;
        }
        __syncthreads();  // the previous block's weights are no longer read
        bool large = false;
        for (int i = threadIdx.x; i < kPairBlock * kPairBlock; i += blockDim.x) {
            const int ra = i / kPairBlock;
            const int rb = i % kPairBlock;
            double v = 0.0;
            const uint64_t a = a0 + ra;
            const uint64_t b = b0 + rb;
            if (a < b && b < row_count) {
                const uint64_t pair = a * (2 * r64 - a - 1) / 2 + (b - a - 1);
                if (pair >= pair_begin && pair < pair_end) {
                    v = inverse[a * row_count + b];
                }
            }
            sw64[i] = v;
            sw[i] = v > 0x1p100 ? 0.f : __double2float_rn(v);
            large = large || v > 0x1p100;
        }
        if (__syncthreads_or(large ? 1 : 0) == 0) {
#pragma unroll
            for (int ra = 0; ra < kPairBlock; ++ra) {
#pragma unroll
                for (int rb = 0; rb < kPairBlock; ++rb) {
                    const float d = __fsub_rn(va[ra], vb[rb]);
                    const float w = sw[ra * kPairBlock + rb];
                    const float c = metric == 0 ? __fmul_rn(__fmul_rn(d, d), w)
                                                : __fmul_rn(fabsf(d), w);
                    m32[ra % 4] = fmaxf(m32[ra % 4], c);
                }
            }
        } else {
#pragma unroll 1
            for (int ra = 0; ra < kPairBlock; ++ra) {
#pragma unroll 1
                for (int rb = 0; rb < kPairBlock; ++rb) {
                    // the values again from memory: runtime indices would
                    // move va and vb out of registers
                    const double xa = a0 + ra < row_count && col < dim
                                          ? rows[static_cast<uint64_t>(a0 + ra) * dim + col]
                                          : 0.f;
                    const double xb = b0 + rb < row_count && col < dim
                                          ? rows[static_cast<uint64_t>(b0 + rb) * dim + col]
                                          : 0.f;
                    const double d = __dsub_rn(xa, xb);
                    const double w = sw64[ra * kPairBlock + rb];
                    const double c = metric == 0 ? __dmul_rn(__dmul_rn(d, d), w)
                                                 : __dmul_rn(fabs(d), w);
                    m = fmax(m, c);
                }
            }
        }
    }
    m = fmax(m, static_cast<double>(fmaxf(fmaxf(m32[0], m32[1]), fmaxf(m32[2], m32[3]))));
    if (col < dim && m > 0.0) {
        atomicMax(maxima_bits + col,
                  static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

}  // namespace

void launch_pair_distances(int metric, const float* rows, uint64_t row_count,
                           uint64_t dim, double* inverse_distances,
                           cudaStream_t stream)
{
    const uint32_t blocks =
        static_cast<uint32_t>((row_count + kPairBlock - 1) / kPairBlock);
    if (blocks > 65535u) {
        fail(UHA_LENGTH_ERROR, "probability pair grid exceeds device limit");
    }
    const dim3 grid(blocks, blocks);
    pair_distance_kernel<<<grid, 256, 0, stream>>>(
        metric, rows, static_cast<uint32_t>(row_count), dim, inverse_distances);
    check_cuda(cudaGetLastError(), "cannot launch pair distance kernel");
}

void launch_gram_inverse_distances(const float* rows, uint64_t row_count,
                                   uint64_t dim, double* gram,
                                   double* inverse_distances,
                                   cudaStream_t stream)
{
    const uint32_t blocks =
        static_cast<uint32_t>((row_count + kPairBlock - 1) / kPairBlock);
    if (blocks > 65535u) {
        fail(UHA_LENGTH_ERROR, "probability pair grid exceeds device limit");
    }
    gram_kernel<<<dim3(blocks, blocks), 256, 0, stream>>>(
        rows, static_cast<uint32_t>(row_count), dim, gram);
    check_cuda(cudaGetLastError(), "cannot launch Gram kernel");
    gram_to_inverse_kernel<<<148 * 16, 256, 0, stream>>>(
        gram, rows, static_cast<uint32_t>(row_count), dim, inverse_distances);
    check_cuda(cudaGetLastError(), "cannot launch Gram refinement kernel");
}

namespace {

__global__ void finite_check_kernel(const float* __restrict__ values, uint64_t count,
                                    int* flag)
{
    bool bad = false;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         i < count; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        bad = bad || !isfinite(values[i]);
    }
    if (__any_sync(0xffffffffu, bad) && threadIdx.x % 32 == 0) {
        atomicOr(flag, 1);
    }
}

}  // namespace

void launch_finite_check(const float* values, uint64_t count, int* flag,
                         cudaStream_t stream)
{
    if (count == 0) {
        return;
    }
    const uint64_t blocks = std::min<uint64_t>((count + 255) / 256, 148ull * 32);
    finite_check_kernel<<<static_cast<uint32_t>(blocks), 256, 0, stream>>>(values, count,
                                                                           flag);
    check_cuda(cudaGetLastError(), "cannot launch the finiteness check");
}

void launch_coordinate_maxima(int metric, const float* rows,
                              uint64_t row_count, uint64_t dim,
                              const double* inverse_distances,
                              unsigned long long* maxima_bits,
                              uint64_t pair_begin, uint64_t pair_end,
                              cudaStream_t stream, bool single)
{
    if (pair_begin >= pair_end) {
        return;
    }
    // row of the first and last pair of the chunk
    auto row_of = [&](uint64_t pair) {
        uint64_t a = 0;
        uint64_t before = 0;
        while (before + (row_count - a - 1) <= pair) {
            before += row_count - a - 1;
            ++a;
        }
        return a;
    };
    const uint32_t first_block = static_cast<uint32_t>(row_of(pair_begin) / kPairBlock);
    const uint32_t last_block = static_cast<uint32_t>(row_of(pair_end - 1) / kPairBlock);
    const uint32_t blocks =
        static_cast<uint32_t>((row_count + kPairBlock - 1) / kPairBlock);
    const uint64_t column_blocks = (dim + kColumns - 1) / kColumns;
    if (column_blocks > 0x7fffffffull || blocks > 65535u) {
        fail(UHA_LENGTH_ERROR, "probability column grid exceeds device limit");
    }
    const size_t smem = kPairBlock * kPairBlock * sizeof(double) +
                        2 * kPairBlock * kColumns * sizeof(float);
    const dim3 grid(static_cast<uint32_t>(column_blocks), last_block - first_block + 1);
    if (single) {
        coordinate_max32_kernel<<<grid, kColumns, 0, stream>>>(
            metric, rows, static_cast<uint32_t>(row_count), dim, inverse_distances,
            maxima_bits, first_block, pair_begin, pair_end);
        check_cuda(cudaGetLastError(), "cannot launch probability column kernel");
        return;
    }
    static bool configured[kMaxDevices] = {};
    const int dev = current_device();
    if (!configured[dev]) {
        check_cuda(cudaFuncSetAttribute(coordinate_max_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)),
                   "cannot configure probability column kernel");
        configured[dev] = true;
    }
    coordinate_max_kernel<<<grid, kColumns, smem, stream>>>(
        metric, rows, static_cast<uint32_t>(row_count), dim, inverse_distances,
        maxima_bits, first_block, pair_begin, pair_end);
    check_cuda(cudaGetLastError(), "cannot launch probability column kernel");
}

}  // namespace uha
