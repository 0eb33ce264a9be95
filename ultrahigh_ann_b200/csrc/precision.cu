// Precision form of the exact and flat L2 scans (no reference counterpart;
// the reference's `gemm` strategy is the binary32 cublasSgemm of
// src/core/cuda_dense_l2_scan_index.cu:718-729).
//
// Rows and queries are rounded to BF16, or to FP8-E4M3 with one binary32
// scale per row and per query. The score matrix S[q][row] = q~ . v~ runs on
// the fifth-generation tensor cores (tcgen05.mma, FP32 accumulation in TMEM)
// with both operands staged in shared memory by TMA. The estimate
// e = ||v~||^2 - 2 S ranks the rows of a query (||q~||^2 is common to all of
// them); the k smallest estimates (lowest row on ties) are the candidates that
// the re-score of certify.cu settles against the original rows.
//
// Kernel layout of the score GEMM (one CTA per 128-row x BN-query tile and
// K split, 192 threads):
//   warp 0      TMA producer: one 128-byte K slice of the row tile and of the
//               query tile per pipeline stage, 128-byte swizzle
//   warp 1      TMEM allocation and the MMA issuer (one elected thread):
//               4 x tcgen05.mma (M=128, N=BN, K=16 BF16 / K=32 FP8) per stage,
//               tcgen05.commit frees the stage
//   warps 2-5   epilogue: tcgen05.ld of the 128 x BN FP32 accumulator, one
//               TMEM lane quarter per warp, coalesced stores of the partial
//               scores [split][query][row]
// Every mbarrier wait is bounded; a wait that runs out sets bit 8 of the
// error flag and the CTA drains its pipeline (bounded) and returns.
#include "async_copy.cuh"
#include "common.h"
#include "kernels.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <mutex>

namespace uha {
namespace {

constexpr int kTileRows = 128;        // UMMA M: rows per tile (TMEM lanes)
constexpr uint32_t kSliceBytes = 128; // K bytes per stage: one swizzle atom row
constexpr int kGemmThreads = 192;
constexpr uint32_t kSpinLimit = 1u << 24;
constexpr int kConvertThreads = 256;
constexpr int kTopkThreads = 256;
constexpr int kPipelineTimeout = 8;   // error-flag bit

// ------------------------------------------------------------ PTX helpers

using async::mbar_expect_tx;
using async::mbar_init;
using async::smem_u32;

// Waits for the phase of `parity` to complete; false after kSpinLimit tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    return async::mbar_wait(bar, parity, kSpinLimit);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map,
                                            uint64_t* bar, int32_t x, int32_t y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile written by TMA
// with 128-byte swizzling: rows of 128 bytes, 8-row core groups 1024 bytes
// apart (stride byte offset), descriptor version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t smem_addr)
{
    uint64_t d = static_cast<uint64_t>((smem_addr >> 4) & 0x3fffu);
    d |= static_cast<uint64_t>(1) << 16;           // leading byte offset (16 B)
    d |= static_cast<uint64_t>(1024 >> 4) << 32;   // stride byte offset
    d |= static_cast<uint64_t>(1) << 46;           // version
    d |= static_cast<uint64_t>(2) << 61;           // 128-byte swizzle
    return d;
}

// Instruction descriptor: FP32 accumulator, A and B of the same type (BF16,
// or E4M3 for kind::f8f6f4), both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t mma_idesc(bool fp8, int n)
{
    return (1u << 4) | (fp8 ? 0u : ((1u << 7) | (1u << 10))) |
           (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(kTileRows >> 4) << 24);
}

template <bool FP8>
__device__ __forceinline__ void mma_issue(uint32_t tmem, uint64_t a, uint64_t b,
                                          uint32_t idesc, uint32_t accumulate)
{
    if constexpr (FP8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
            : "memory");
    }
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load16(uint32_t addr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
          "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    // the registers are read only after the load has completed
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]),
                   "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]),
                   "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

// Unsigned key bits that order like the binary32 value (negative values
// below positive ones).
__device__ __forceinline__ unsigned int ordered_key_bits(float f)
{
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

template <int BN, int STAGES>
struct GemmSmem {
    static constexpr uint32_t a_bytes = kTileRows * kSliceBytes;
    static constexpr uint32_t b_bytes = BN * kSliceBytes;
    static constexpr uint32_t tiles = STAGES * (a_bytes + b_bytes);
    // 1024-byte alignment slack + barriers + TMEM slot + abort word
    static constexpr uint32_t total = 1024 + tiles + (2 * STAGES + 1) * 8 + 16;
    static constexpr uint32_t tmem_cols = BN < 32 ? 32 : BN;
};

// Partial scores of one (row tile, query tile, K split):
// partials[split][q][row] = sum over the split's K range of q~ . v~ (times
// the row and query scales for FP8).
//
// With FILTER (one K split only) nothing is stored per score: the epilogue
// forms the estimate e = ||v~||^2 - 2 S exactly as the candidate selection
// does and appends the key (e, row) of every row with e <= f.tau[q] to the
// query's list f.keys[q][0 .. f.cap) (f.count[q] counts them all, also past
// the capacity).
//
// Row tile y reads the index's tile y * tile_stride (rows below source_rows);
// its scores are row y * 128 + i of the output (rows below row_count). A
// stride above 1 scores a sample of whole tiles spread over the index.
template <int BN, int STAGES, bool FP8, bool FILTER>
__global__ void __launch_bounds__(kGemmThreads, 1)
    lowp_score_kernel(const __grid_constant__ CUtensorMap rows_map,
                      const __grid_constant__ CUtensorMap queries_map,
                      uint32_t kblocks, uint32_t kblocks_per_split,
                      uint32_t row_count, uint32_t batch, const float* row_scale,
                      const float* query_scale, float* partials, FilterArgs f,
                      uint32_t tile_stride, uint32_t source_rows, int* error_flag)
{
    using L = GemmSmem<BN, STAGES>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* a_tiles = smem;
    unsigned char* b_tiles = smem + STAGES * L::a_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::tiles);
    uint64_t* empty = full + STAGES;
    uint64_t* accum = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
    volatile int* aborted = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const uint32_t split = blockIdx.z;
    const uint32_t kb_begin = split * kblocks_per_split;
    const uint32_t kb_end = min(kblocks, kb_begin + kblocks_per_split);
    const uint32_t steps = kb_end > kb_begin ? kb_end - kb_begin : 0;
    const int32_t row0 = static_cast<int32_t>(blockIdx.y) * kTileRows;  // output rows
    const int32_t src0 = static_cast<int32_t>(blockIdx.y * tile_stride) * kTileRows;
    const int32_t q0 = static_cast<int32_t>(blockIdx.x) * BN;

    if (warp == 0 && lane == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(accum, 1);
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&rows_map))
                     : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(
                         reinterpret_cast<uint64_t>(&queries_map))
                     : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(L::tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::
                         : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t issued = 0;
            for (uint32_t i = 0; i < steps && !*aborted; ++i) {
                const uint32_t s = i % STAGES;
                const uint32_t phase = (i / STAGES) & 1u;
                if (!mbar_wait(empty + s, phase ^ 1u)) {
                    *aborted = 1;
                    atomicOr(error_flag, kPipelineTimeout);
                    break;
                }
                mbar_expect_tx(full + s, L::a_bytes + L::b_bytes);
                const int32_t x = static_cast<int32_t>((kb_begin + i) * (FP8 ? 128u : 64u));
                tma_load_2d(a_tiles + s * L::a_bytes, &rows_map, full + s, x, src0);
                tma_load_2d(b_tiles + s * L::b_bytes, &queries_map, full + s, x, q0);
                ++issued;
            }
            if (*aborted) {
                // drain: every issued copy lands before the CTA exits
                const uint32_t first = issued > STAGES ? issued - STAGES : 0;
                for (uint32_t i = first; i < issued; ++i) {
                    mbar_wait(full + i % STAGES, (i / STAGES) & 1u);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = mma_idesc(FP8, BN);
            for (uint32_t i = 0; i < steps && !*aborted; ++i) {
                const uint32_t s = i % STAGES;
                const uint32_t phase = (i / STAGES) & 1u;
                if (!mbar_wait(full + s, phase)) {
                    *aborted = 1;
                    atomicOr(error_flag, kPipelineTimeout);
                    break;
                }
                tc_fence_after();
                const uint64_t da = sw128_desc(smem_u32(a_tiles + s * L::a_bytes));
                const uint64_t db = sw128_desc(smem_u32(b_tiles + s * L::b_bytes));
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk) {
                    // +32 bytes of K per instruction inside the swizzle atom
                    mma_issue<FP8>(tmem, da + 2 * kk, db + 2 * kk, idesc,
                                   (i | kk) != 0 ? 1u : 0u);
                }
                mma_commit(empty + s);
            }
            // tracks every MMA issued above (also on the abort path)
            mma_commit(accum);
        }
        __syncwarp();
    } else {
        const uint32_t quarter = static_cast<uint32_t>(warp % 4) * 32;
        // warp-uniform decisions: tcgen05.ld is executed by all 32 lanes or none
        const bool ready = __all_sync(0xffffffffu, mbar_wait(accum, 0));
        tc_fence_after();
        const bool store = __shfl_sync(0xffffffffu, ready && !*aborted && steps != 0, 0);
        if (!ready) {
            if (lane == 0) {
                atomicOr(error_flag, kPipelineTimeout);
            }
        } else if (store && FILTER) {
            // Three passes, so that a tile waits for one round of atomics:
            // (1) the pass mask of every query column (warp ballot over the
            // warp's 32 rows) into shared memory; (2) one atomic per column
            // with passes, all of the warp's in flight together (lane l takes
            // columns l, l + 32, ...); (3) the keys into their slots. The
            // operand tiles are free once every MMA has completed.
            // per warp: thresholds, query scales, masks, slot bases (BN words
            // each; a warp that gave up never leaves another one waiting)
            const uint32_t qi = static_cast<uint32_t>(warp % 4);
            uint32_t* area = reinterpret_cast<uint32_t*>(a_tiles) + qi * 4 * BN;
            float* tau_s = reinterpret_cast<float*>(area);
            float* qscale_s = tau_s + BN;
            uint32_t* masks = area + 2 * BN;
            uint32_t* bases = area + 3 * BN;
            for (int c = lane; c < BN; c += 32) {
                const uint32_t q = static_cast<uint32_t>(q0 + c);
                tau_s[c] = q < batch ? f.tau[q] : -__int_as_float(0x7f800000);
                qscale_s[c] = FP8 && q < batch ? query_scale[q] : 1.f;
            }
            __syncwarp();
            const uint32_t row = static_cast<uint32_t>(src0) + quarter + lane;
            const bool row_ok = row < source_rows;
            const float rs = FP8 && row_ok ? row_scale[row] : 1.f;
            const float norm = row_ok ? f.norms[row] : 0.f;
            auto estimate = [&](float v, int c) {
                const float value = FP8 ? __fmul_rn(__fmul_rn(v, rs), qscale_s[c]) : v;
                // the selection sums one slab from zero: 0 + value
                return __fmaf_rn(-2.f, 0.f + value, norm);
            };
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_load16(tmem + (quarter << 16) + static_cast<uint32_t>(c), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const bool pass = row_ok && estimate(v[j], c + j) <= tau_s[c + j];
                    const unsigned int mask = __ballot_sync(0xffffffffu, pass);
                    if (lane == 0) {
                        masks[c + j] = mask;
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int c0 = 0; c0 < BN; c0 += 32) {
                const int c = c0 + lane;
                const uint32_t mask = c < BN ? masks[c] : 0u;
                uint32_t base = 0;
                if (mask != 0u) {
                    base = atomicAdd(f.count + q0 + c, static_cast<uint32_t>(__popc(mask)));
                }
                if (c < BN) {
                    bases[c] = base;
                }
            }
            __syncwarp();
            const unsigned int below = (1u << lane) - 1u;
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                bool any = false;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    any = any || masks[c + j] != 0u;
                }
                if (!any) {
                    continue;  // warp-uniform: the masks are shared
                }
                float v[16];
                tmem_load16(tmem + (quarter << 16) + static_cast<uint32_t>(c), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const unsigned int mask = masks[c + j];
                    if ((mask >> lane) & 1u) {
                        const uint32_t slot =
                            bases[c + j] + static_cast<uint32_t>(__popc(mask & below));
                        if (slot < f.cap) {
                            const float est = estimate(v[j], c + j);
                            f.keys[static_cast<uint64_t>(q0 + c + j) * f.cap + slot] =
                                (static_cast<unsigned long long>(ordered_key_bits(est)) << 32) |
                                row;
                        }
                    }
                }
            }
        } else if (store) {
            const uint32_t row = static_cast<uint32_t>(row0) + quarter + lane;
            const uint32_t src_row = static_cast<uint32_t>(src0) + quarter + lane;
            const bool row_ok = row < row_count && src_row < source_rows;
            const float rs = FP8 && row_ok ? row_scale[src_row] : 1.f;
            float* out = partials + static_cast<uint64_t>(split) * batch * row_count + row;
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_load16(tmem + (quarter << 16) + static_cast<uint32_t>(c), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const uint32_t q = static_cast<uint32_t>(q0 + c + j);
                    if (row_ok && q < batch) {
                        const float value = FP8 ? __fmul_rn(__fmul_rn(v[j], rs), query_scale[q])
                                                : v[j];
                        out[static_cast<uint64_t>(q) * row_count] = value;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(L::tmem_cols)
                     : "memory");
    }
}

// ------------------------------------------------------ rounding kernels

__device__ __forceinline__ float block_sum(float v, float* scratch)
{
    for (int o = 16; o > 0; o /= 2) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    const int warp = threadIdx.x / 32;
    __syncthreads();
    if (threadIdx.x % 32 == 0) {
        scratch[warp] = v;
    }
    __syncthreads();
    float t = 0.f;
    for (int w = 0; w < kConvertThreads / 32; ++w) {
        t += scratch[w];
    }
    return t;
}

__device__ __forceinline__ float block_max(float v, float* scratch)
{
    for (int o = 16; o > 0; o /= 2) {
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    const int warp = threadIdx.x / 32;
    __syncthreads();
    if (threadIdx.x % 32 == 0) {
        scratch[warp] = v;
    }
    __syncthreads();
    float t = 0.f;
    for (int w = 0; w < kConvertThreads / 32; ++w) {
        t = fmaxf(t, scratch[w]);
    }
    return t;
}

// One block per vector: BF16 (round to nearest even) of the first `dim`
// values, zeros up to `pitch`; norms[i] = sum of squares of the rounded values.
__global__ void __launch_bounds__(kConvertThreads)
    to_bf16_kernel(const float* src, uint64_t src_pitch, uint64_t dim,
                   __nv_bfloat16* out, uint64_t pitch, float* norms)
{
    __shared__ float scratch[kConvertThreads / 32];
    const uint64_t v = blockIdx.x;
    const float* in = src + v * src_pitch;
    __nv_bfloat16* o = out + v * pitch;
    float acc = 0.f;
    for (uint64_t j = threadIdx.x; j < pitch; j += kConvertThreads) {
        const float x = j < dim ? in[j] : 0.f;
        const __nv_bfloat16 b = __float2bfloat16_rn(x);
        o[j] = b;
        const float r = __bfloat162float(b);
        acc = __fmaf_rn(r, r, acc);
    }
    const float total = block_sum(acc, scratch);
    if (threadIdx.x == 0 && norms != nullptr) {
        norms[v] = total;
    }
}

// One block per vector: scale = max|x| / 448 (1 for a zero vector),
// E4M3 = satfinite(round(x / scale)); norms[i] = sum of squares of the
// dequantized values e4m3 * scale.
__global__ void __launch_bounds__(kConvertThreads)
    to_fp8_kernel(const float* src, uint64_t src_pitch, uint64_t dim,
                  __nv_fp8_storage_t* out, uint64_t pitch, float* scales,
                  float* norms)
{
    __shared__ float scratch[kConvertThreads / 32];
    const uint64_t v = blockIdx.x;
    const float* in = src + v * src_pitch;
    __nv_fp8_storage_t* o = out + v * pitch;
    float amax = 0.f;
    for (uint64_t j = threadIdx.x; j < dim; j += kConvertThreads) {
        amax = fmaxf(amax, fabsf(in[j]));
    }
    amax = block_max(amax, scratch);
    const float scale = amax > 0.f ? __fdiv_rn(amax, 448.f) : 1.f;
    float acc = 0.f;
    for (uint64_t j = threadIdx.x; j < pitch; j += kConvertThreads) {
        const float x = j < dim ? __fdiv_rn(in[j], scale) : 0.f;
        const __nv_fp8_storage_t e = __nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
        o[j] = e;
        const __half_raw h = __nv_cvt_fp8_to_halfraw(e, __NV_E4M3);
        const float r = __fmul_rn(__half2float(__half(h)), scale);
        acc = __fmaf_rn(r, r, acc);
    }
    const float total = block_sum(acc, scratch);
    if (threadIdx.x == 0) {
        scales[v] = scale;
        if (norms != nullptr) {
            norms[v] = total;
        }
    }
}

// Query batches: grid (column chunks, queries); each thread rounds 8 (BF16)
// or 16 (FP8) consecutive columns of a zero-padded binary32 vector (`src`,
// src_pitch apart, a multiple of 4) with vector loads and one 16-byte store.
constexpr int kQueryThreads = 256;

__device__ __forceinline__ float4 load4_or_zero(const float* v, uint64_t j,
                                                uint64_t src_pitch)
{
    return j + 4 <= src_pitch ? *reinterpret_cast<const float4*>(v + j)
                              : make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void __launch_bounds__(kQueryThreads)
    queries_to_bf16_kernel(const float* src, uint64_t src_pitch,
                           __nv_bfloat16* out, uint64_t pitch)
{
    const uint64_t q = blockIdx.y;
    const uint64_t j = (static_cast<uint64_t>(blockIdx.x) * kQueryThreads + threadIdx.x) * 8;
    if (j >= pitch) {
        return;
    }
    const float* v = src + q * src_pitch;
    const float4 a = load4_or_zero(v, j, src_pitch);
    const float4 b = load4_or_zero(v, j + 4, src_pitch);
    __nv_bfloat162 h[4];
    h[0] = __floats2bfloat162_rn(a.x, a.y);
    h[1] = __floats2bfloat162_rn(a.z, a.w);
    h[2] = __floats2bfloat162_rn(b.x, b.y);
    h[3] = __floats2bfloat162_rn(b.z, b.w);
    *reinterpret_cast<uint4*>(out + q * pitch + j) = *reinterpret_cast<uint4*>(h);
}

// amax_bits[q] = bits of max |src[q][j]| (non-negative binary32 values order
// like their bit patterns; the slots are zero before the launch).
__global__ void __launch_bounds__(kQueryThreads)
    queries_amax_kernel(const float* src, uint64_t src_pitch, unsigned int* amax_bits)
{
    const uint64_t q = blockIdx.y;
    const uint64_t j = (static_cast<uint64_t>(blockIdx.x) * kQueryThreads + threadIdx.x) * 16;
    const float* v = src + q * src_pitch;
    float m = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float4 a = load4_or_zero(v, j + 4 * c, src_pitch);
        m = fmaxf(m, fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(a.w))));
    }
    for (int o = 16; o > 0; o /= 2) {
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if (threadIdx.x % 32 == 0) {
        atomicMax(amax_bits + q, __float_as_uint(m));
    }
}

__global__ void __launch_bounds__(kQueryThreads)
    queries_to_fp8_kernel(const float* src, uint64_t src_pitch,
                          const unsigned int* amax_bits, __nv_fp8_storage_t* out,
                          uint64_t pitch, float* scales)
{
    const uint64_t q = blockIdx.y;
    const float amax = __uint_as_float(amax_bits[q]);
    const float scale = amax > 0.f ? __fdiv_rn(amax, 448.f) : 1.f;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scales[q] = scale;
    }
    const uint64_t j = (static_cast<uint64_t>(blockIdx.x) * kQueryThreads + threadIdx.x) * 16;
    if (j >= pitch) {
        return;
    }
    const float* v = src + q * src_pitch;
    uint32_t packed[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float4 a = load4_or_zero(v, j + 4 * c, src_pitch);
        const __nv_fp8x2_storage_t lo = __nv_cvt_float2_to_fp8x2(
            make_float2(__fdiv_rn(a.x, scale), __fdiv_rn(a.y, scale)), __NV_SATFINITE, __NV_E4M3);
        const __nv_fp8x2_storage_t hi = __nv_cvt_float2_to_fp8x2(
            make_float2(__fdiv_rn(a.z, scale), __fdiv_rn(a.w, scale)), __NV_SATFINITE, __NV_E4M3);
        packed[c] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(hi) << 16);
    }
    *reinterpret_cast<uint4*>(out + q * pitch + j) =
        make_uint4(packed[0], packed[1], packed[2], packed[3]);
}

// ---------------------------------------------------------------- top-k

template <int KCAP>
__device__ __forceinline__ void keep_smallest(unsigned long long (&best)[KCAP],
                                              unsigned long long key)
{
    if (key < best[KCAP - 1]) {
        best[KCAP - 1] = key;
#pragma unroll
        for (int i = KCAP - 1; i > 0; --i) {
            const unsigned long long a = best[i - 1];
            const unsigned long long b = best[i];
            best[i - 1] = a < b ? a : b;
            best[i] = a < b ? b : a;
        }
    }
}

// The KCAP smallest keys of a warp's sorted per-lane lists, ascending, into
// out[0..KCAP) (lane 0 writes).
template <int KCAP>
__device__ __forceinline__ void warp_merge(unsigned long long (&best)[KCAP],
                                           unsigned long long* out, int lane)
{
#pragma unroll 1
    for (int i = 0; i < KCAP; ++i) {
        const unsigned long long head = best[0];
        unsigned long long m = head;
        for (int o = 16; o > 0; o /= 2) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, m, o);
            m = other < m ? other : m;
        }
        if (lane == 0) {
            out[i] = m;
        }
        if (head == m) {
#pragma unroll
            for (int j = 0; j + 1 < KCAP; ++j) {
                best[j] = best[j + 1];
            }
            best[KCAP - 1] = ~0ull;
        }
    }
}

// One block per query: the k rows with the smallest (||v~||^2 - 2 S, row).
// candidates[q * k + i], ascending; 0xffffffff where the index has fewer rows.
template <int KCAP>
__global__ void __launch_bounds__(kTopkThreads)
    topk_kernel(const float* partials, uint32_t splits, uint32_t batch,
                uint32_t row_count, const float* norms, uint32_t k,
                uint32_t* candidates)
{
    __shared__ unsigned long long lists[kTopkThreads / 32][KCAP];
    __shared__ unsigned long long final_list[KCAP];
    const uint32_t q = blockIdx.x;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    unsigned long long best[KCAP];
#pragma unroll
    for (int i = 0; i < KCAP; ++i) {
        best[i] = ~0ull;
    }
    const uint64_t split_stride = static_cast<uint64_t>(batch) * row_count;
    const float* base = partials + static_cast<uint64_t>(q) * row_count;
    // ROWS rows x 8 split slabs of loads in flight per thread; every row's
    // slabs are added in split order
    constexpr int ROWS = KCAP >= 64 ? 1 : (KCAP >= 32 ? 2 : 4);
    constexpr int SPLITS = 8;
    for (uint32_t first = threadIdx.x; first < row_count; first += ROWS * kTopkThreads) {
        float dot[ROWS];
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            dot[r] = 0.f;
        }
        for (uint32_t s0 = 0; s0 < splits; s0 += SPLITS) {
            float v[ROWS][SPLITS];
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                const uint32_t row = first + r * kTopkThreads;
#pragma unroll
                for (int u = 0; u < SPLITS; ++u) {
                    v[r][u] = row < row_count && s0 + u < splits
                                  ? base[(s0 + u) * split_stride + row]
                                  : 0.f;
                }
            }
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
#pragma unroll
                for (int u = 0; u < SPLITS; ++u) {
                    if (s0 + u < splits) {
                        dot[r] += v[r][u];
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const uint32_t row = first + r * kTopkThreads;
            if (row < row_count) {
                const float e = __fmaf_rn(-2.f, dot[r], norms[row]);
                keep_smallest(best,
                              (static_cast<unsigned long long>(ordered_key_bits(e)) << 32) | row);
            }
        }
    }
    warp_merge(best, lists[warp], lane);
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < KCAP; ++i) {
            best[i] = ~0ull;
        }
        for (int i = lane; i < (kTopkThreads / 32) * KCAP; i += 32) {
            keep_smallest(best, lists[i / KCAP][i % KCAP]);
        }
        warp_merge(best, final_list, lane);
        __syncwarp();
        for (uint32_t i = lane; i < k; i += 32) {
            const unsigned long long key = final_list[i];
            candidates[static_cast<uint64_t>(q) * k + i] =
                key == ~0ull ? 0xffffffffu : static_cast<uint32_t>(key & 0xffffffffu);
        }
    }
}

// Top-k for k <= 32 as a warp-wide sorted list (one key per lane, ascending
// by lane) with a two-slot queue per lane (the warp-select scheme of Johnson,
// Douze and Jegou, "Billion-scale similarity search with GPUs", 2017): a key
// below the list's largest enters the lane's queue; when a queue fills, the
// warp sorts each queue slot across its lanes (bitonic network over the 32
// lanes) and merges it into the list. Most keys cost a load, an FMA and one
// comparison.
__device__ __forceinline__ unsigned long long warp_sort32(unsigned long long v, int lane)
{
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size / 2; stride > 0; stride /= 2) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool ascending = (lane & size) == 0;
            const bool low = (lane & stride) == 0;
            v = (low == ascending) ? (o < v ? o : v) : (o < v ? v : o);
        }
    }
    return v;
}

// The 32 smallest of two ascending warp lists, ascending: min(w_i, e_{31-i})
// is bitonic and holds them; one bitonic merge sorts it.
__device__ __forceinline__ unsigned long long warp_merge32(unsigned long long w,
                                                           unsigned long long e, int lane)
{
    const unsigned long long er = __shfl_sync(0xffffffffu, e, 31 - lane);
    unsigned long long m = er < w ? er : w;
#pragma unroll
    for (int stride = 16; stride > 0; stride /= 2) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, m, stride);
        const bool low = (lane & stride) == 0;
        m = low ? (o < m ? o : m) : (o < m ? m : o);
    }
    return m;
}

template <bool kSingleSlab>
__global__ void __launch_bounds__(kTopkThreads)
    warp_topk_kernel(const float* __restrict__ partials, uint32_t splits, uint32_t batch,
                     uint32_t row_count, const float* __restrict__ norms, uint32_t k,
                     uint32_t* __restrict__ candidates)
{
    constexpr int kWarps = kTopkThreads / 32;
    constexpr int U = 8;  // rows per lane whose loads are in flight together
    __shared__ unsigned long long lists[kWarps][32];
    const uint32_t q = blockIdx.x;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const uint64_t split_stride = static_cast<uint64_t>(batch) * row_count;
    const float* base = partials + static_cast<uint64_t>(q) * row_count;
    unsigned long long list = ~0ull;
    unsigned long long largest = ~0ull;
    unsigned long long slot0 = ~0ull;
    unsigned long long slot1 = ~0ull;
    int queued = 0;
    auto flush = [&]() {
        list = warp_merge32(list, warp_sort32(slot0, lane), lane);
        list = warp_merge32(list, warp_sort32(slot1, lane), lane);
        slot0 = ~0ull;
        slot1 = ~0ull;
        queued = 0;
        largest = __shfl_sync(0xffffffffu, list, 31);
    };
    for (uint32_t first = warp * 32; first < row_count; first += kTopkThreads * U) {
        float e[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t row = first + lane + u * kTopkThreads;
            float dot = 0.f;
            if (row < row_count) {
                if constexpr (kSingleSlab) {
                    dot = base[row];
                } else {
                    for (uint32_t sp = 0; sp < splits; ++sp) {
                        dot += base[sp * split_stride + row];
                    }
                }
            }
            e[u] = dot;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t row = first + lane + u * kTopkThreads;
            if (row < row_count) {
                const float est = __fmaf_rn(-2.f, e[u], norms[row]);
                const unsigned long long key =
                    (static_cast<unsigned long long>(ordered_key_bits(est)) << 32) | row;
                if (key < largest) {
                    if (queued == 0) {
                        slot0 = key;
                    } else {
                        slot1 = key;
                    }
                    ++queued;
                }
            }
            if (__any_sync(0xffffffffu, queued == 2)) {
                flush();
            }
        }
    }
    if (__any_sync(0xffffffffu, queued != 0)) {
        flush();
    }
    lists[warp][lane] = list;
    __syncthreads();
    if (warp == 0) {
        list = lists[0][lane];
#pragma unroll 1
        for (int w = 1; w < kWarps; ++w) {
            list = warp_merge32(list, lists[w][lane], lane);
        }
        if (static_cast<uint32_t>(lane) < k) {
            candidates[static_cast<uint64_t>(q) * k + lane] =
                list == ~0ull ? 0xffffffffu : static_cast<uint32_t>(list & 0xffffffffu);
        }
    }
}

// tau[q]: the estimate of the query's k-th candidate over the sample's one
// slab (the selection's own arithmetic: 0 + S, then the FMA with the norm;
// norms in sample order).
__global__ void threshold_kernel(const float* __restrict__ partials, uint32_t batch,
                                 uint32_t rows, const float* __restrict__ norms, uint32_t k,
                                 const uint32_t* __restrict__ candidates,
                                 float* __restrict__ tau)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= batch) {
        return;
    }
    const uint32_t row = candidates[static_cast<uint64_t>(q) * k + k - 1];
    float t = __int_as_float(0x7f800000);
    if (row != 0xffffffffu) {
        const float dot = 0.f + partials[static_cast<uint64_t>(q) * rows + row];
        t = __fmaf_rn(-2.f, dot, norms[row]);
    }
    tau[q] = t;
}

// out[i] = norms of the index row that sample row i stands for (tile i / 128
// is the index's tile (i / 128) * tile_stride).
__global__ void sample_norms_kernel(const float* __restrict__ norms, uint32_t sample_rows,
                                    uint32_t tile_stride, float* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < sample_rows) {
        out[i] = norms[(i / kTileRows) * tile_stride * kTileRows + i % kTileRows];
    }
}

// One block per query: the k smallest keys of the query's filtered list,
// ascending (the keys order by estimate, then row, as the slab selection's).
template <int KCAP>
__global__ void __launch_bounds__(kTopkThreads)
    select_kernel(const unsigned long long* __restrict__ keys,
                  const uint32_t* __restrict__ count, uint32_t cap, uint32_t k,
                  uint32_t* __restrict__ candidates, int* error_flag)
{
    __shared__ unsigned long long lists[kTopkThreads / 32][KCAP];
    __shared__ unsigned long long final_list[KCAP];
    const uint32_t q = blockIdx.x;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const uint32_t total = count[q];
    if (total > cap && threadIdx.x == 0) {
        atomicOr(error_flag, kCandidateOverflow);
    }
    const uint32_t n = min(total, cap);
    unsigned long long best[KCAP];
#pragma unroll
    for (int i = 0; i < KCAP; ++i) {
        best[i] = ~0ull;
    }
    const unsigned long long* list = keys + static_cast<uint64_t>(q) * cap;
    for (uint32_t i = threadIdx.x; i < n; i += kTopkThreads) {
        keep_smallest(best, list[i]);
    }
    warp_merge(best, lists[warp], lane);
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < KCAP; ++i) {
            best[i] = ~0ull;
        }
        for (int i = lane; i < (kTopkThreads / 32) * KCAP; i += 32) {
            keep_smallest(best, lists[i / KCAP][i % KCAP]);
        }
        warp_merge(best, final_list, lane);
        __syncwarp();
        for (uint32_t i = lane; i < k; i += 32) {
            const unsigned long long key = final_list[i];
            candidates[static_cast<uint64_t>(q) * k + i] =
                key == ~0ull ? 0xffffffffu : static_cast<uint32_t>(key & 0xffffffffu);
        }
    }
}

// One warp per query (k <= 32): the k smallest keys of the query's filtered
// list with the warp list and two-slot lane queues of warp_topk_kernel.
__global__ void __launch_bounds__(kTopkThreads)
    warp_select_kernel(const unsigned long long* __restrict__ keys,
                       const uint32_t* __restrict__ count, uint32_t cap, uint32_t batch,
                       uint32_t k, uint32_t* __restrict__ candidates, int* error_flag)
{
    const uint32_t q = blockIdx.x * (kTopkThreads / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (q >= batch) {
        return;
    }
    const uint32_t total = count[q];
    if (total > cap && lane == 0) {
        atomicOr(error_flag, kCandidateOverflow);
    }
    const uint32_t n = min(total, cap);
    const unsigned long long* list_in = keys + static_cast<uint64_t>(q) * cap;
    unsigned long long list = ~0ull;
    unsigned long long largest = ~0ull;
    unsigned long long slot0 = ~0ull;
    unsigned long long slot1 = ~0ull;
    int queued = 0;
    for (uint32_t first = 0; first < n; first += 32) {
        const uint32_t i = first + lane;
        const unsigned long long key = i < n ? list_in[i] : ~0ull;
        if (key < largest) {
            if (queued == 0) {
                slot0 = key;
            } else {
                slot1 = key;
            }
            ++queued;
        }
        if (__any_sync(0xffffffffu, queued == 2)) {
            list = warp_merge32(list, warp_sort32(slot0, lane), lane);
            list = warp_merge32(list, warp_sort32(slot1, lane), lane);
            slot0 = ~0ull;
            slot1 = ~0ull;
            queued = 0;
            largest = __shfl_sync(0xffffffffu, list, 31);
        }
    }
    if (__any_sync(0xffffffffu, queued != 0)) {
        list = warp_merge32(list, warp_sort32(slot0, lane), lane);
        list = warp_merge32(list, warp_sort32(slot1, lane), lane);
    }
    if (static_cast<uint32_t>(lane) < k) {
        candidates[static_cast<uint64_t>(q) * k + lane] =
            list == ~0ull ? 0xffffffffu : static_cast<uint32_t>(list & 0xffffffffu);
    }
}

// ------------------------------------------------------------ host side

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult status{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                    &status) == cudaSuccess &&
            status == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        } else {
            cudaGetLastError();
        }
    });
    if (fn == nullptr) {
        fail(UHA_RUNTIME_ERROR, "cuTensorMapEncodeTiled is unavailable");
    }
    return fn;
}

// 2-D tensor map over [outer][pitch] one-byte or two-byte elements, box of
// 128 bytes x box_outer with 128-byte swizzling. Callers keep every box inside
// the tensor.
CUtensorMap make_map(const void* base, bool fp8, uint64_t pitch, uint64_t outer,
                     uint32_t box_outer)
{
    CUtensorMap map{};
    const uint64_t elem = fp8 ? 1 : 2;
    const cuuint64_t dims[2] = {pitch, outer};
    const cuuint64_t strides[1] = {pitch * elem};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kSliceBytes / elem), box_outer};
    const cuuint32_t element_strides[2] = {1, 1};
    const CUresult r = encode_fn()(
        &map, fp8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
        const_cast<void*>(base), dims, strides, box, element_strides,
        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fail(UHA_RUNTIME_ERROR, "cannot describe a tensor-core operand (tensor map)");
    }
    return map;
}

// Row tiles a score launch reads: tile y of the output is the index's tile
// y * stride (rows below source_rows).
struct RowTiles {
    uint32_t stride;
    uint32_t source_rows;
};

template <int BN, int STAGES, bool FP8, bool FILTER>
void launch_gemm_filtered(const LowpPlan& plan, const CUtensorMap& rows_map,
                          const CUtensorMap& queries_map, uint32_t row_count,
                          uint32_t batch, const float* row_scale,
                          const float* query_scale, float* partials, const FilterArgs& f,
                          const RowTiles& tiles, int* error_flag, cudaStream_t stream)
{
    using L = GemmSmem<BN, STAGES>;
    auto kernel = lowp_score_kernel<BN, STAGES, FP8, FILTER>;
    static std::once_flag once[kMaxDevices];
    std::call_once(once[current_device()], [&] {
        check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(L::total)),
                   "cannot configure the tensor-core score kernel");
    });
    const dim3 grid((batch + BN - 1) / BN, (row_count + kTileRows - 1) / kTileRows,
                    plan.splits);
    kernel<<<grid, kGemmThreads, L::total, stream>>>(rows_map, queries_map, plan.kblocks,
                                                      plan.kblocks_per_split, row_count,
                                                      batch, row_scale, query_scale,
                                                      partials, f, tiles.stride,
                                                      tiles.source_rows, error_flag);
    check_cuda(cudaGetLastError(), "cannot launch the tensor-core score kernel");
}

template <int BN, int STAGES, bool FP8>
void launch_gemm_instance(const LowpPlan& plan, const CUtensorMap& rows_map,
                          const CUtensorMap& queries_map, uint32_t row_count,
                          uint32_t batch, const float* row_scale,
                          const float* query_scale, float* partials,
                          const FilterArgs* filter, const RowTiles& tiles, int* error_flag,
                          cudaStream_t stream)
{
    if (filter != nullptr && plan.kblocks <= 8) {
        // few K slices (the hierarchies' projected rows): two stages, so two
        // CTAs share an SM and one's filter epilogue overlaps the other's
        // loads and MMAs
        launch_gemm_filtered<BN, 2, FP8, true>(plan, rows_map, queries_map, row_count,
                                               batch, row_scale, query_scale, partials,
                                               *filter, tiles, error_flag, stream);
    } else if (filter != nullptr) {
        launch_gemm_filtered<BN, STAGES, FP8, true>(plan, rows_map, queries_map, row_count,
                                                    batch, row_scale, query_scale, partials,
                                                    *filter, tiles, error_flag, stream);
    } else {
        launch_gemm_filtered<BN, STAGES, FP8, false>(plan, rows_map, queries_map, row_count,
                                                     batch, row_scale, query_scale, partials,
                                                     FilterArgs{}, tiles, error_flag, stream);
    }
}

template <bool FP8>
void launch_gemm_typed(const LowpPlan& plan, const CUtensorMap& rows_map,
                       const void* queries, uint64_t pitch, uint32_t row_count,
                       uint32_t batch, const float* row_scale, const float* query_scale,
                       float* partials, const FilterArgs* filter, const RowTiles& tiles,
                       int* error_flag, cudaStream_t stream)
{
    // the query buffer holds lowp_padded_count(batch) vectors: every box is
    // inside it (the vectors past `batch` are computed and not stored)
    const CUtensorMap queries_map = make_map(queries, FP8, pitch,
                                             round_up(batch, static_cast<uint64_t>(plan.bn)),
                                             static_cast<uint32_t>(plan.bn));
    switch (plan.bn) {
    case 16:
        launch_gemm_instance<16, 8, FP8>(plan, rows_map, queries_map, row_count, batch,
                                         row_scale, query_scale, partials, filter,
                                         tiles, error_flag, stream);
        break;
    case 32:
        launch_gemm_instance<32, 8, FP8>(plan, rows_map, queries_map, row_count, batch,
                                         row_scale, query_scale, partials, filter,
                                         tiles, error_flag, stream);
        break;
    case 64:
        launch_gemm_instance<64, 8, FP8>(plan, rows_map, queries_map, row_count, batch,
                                         row_scale, query_scale, partials, filter,
                                         tiles, error_flag, stream);
        break;
    case 128:
        launch_gemm_instance<128, 6, FP8>(plan, rows_map, queries_map, row_count, batch,
                                          row_scale, query_scale, partials, filter,
                                          tiles, error_flag, stream);
        break;
    default:
        launch_gemm_instance<256, 4, FP8>(plan, rows_map, queries_map, row_count, batch,
                                          row_scale, query_scale, partials, filter,
                                          tiles, error_flag, stream);
        break;
    }
}

}  // namespace

uint64_t lowp_pitch(LowpType type, uint64_t dim)
{
    // one K slice of 128 bytes per pipeline stage
    const uint64_t slice = type == LowpType::fp8_e4m3 ? 128 : 64;
    return round_up(dim == 0 ? 1 : dim, slice);
}

uint64_t lowp_padded_count(uint64_t count)
{
    // a multiple of the row tile and of every query tile width
    return round_up(count == 0 ? 1 : count, 256);
}

uint64_t lowp_element_bytes(LowpType type)
{
    return type == LowpType::fp8_e4m3 ? 1 : 2;
}

void launch_lowp_convert(LowpType type, const float* src, uint64_t count,
                         uint64_t src_pitch, uint64_t dim, void* out, uint64_t pitch,
                         float* scales, float* norms, cudaStream_t stream)
{
    if (count == 0) {
        return;
    }
    if (type == LowpType::bf16) {
        to_bf16_kernel<<<static_cast<unsigned>(count), kConvertThreads, 0, stream>>>(
            src, src_pitch, dim, static_cast<__nv_bfloat16*>(out), pitch, norms);
    } else {
        to_fp8_kernel<<<static_cast<unsigned>(count), kConvertThreads, 0, stream>>>(
            src, src_pitch, dim, static_cast<__nv_fp8_storage_t*>(out), pitch, scales,
            norms);
    }
    check_cuda(cudaGetLastError(), "cannot launch the low-precision rounding kernel");
}

void launch_lowp_queries(LowpType type, const float* src, uint64_t count,
                         uint64_t src_pitch, void* out, uint64_t pitch, float* scales,
                         unsigned int* amax_scratch, cudaStream_t stream)
{
    if (count == 0) {
        return;
    }
    if (type == LowpType::bf16) {
        const dim3 grid(static_cast<unsigned>((pitch / 8 + kQueryThreads - 1) / kQueryThreads),
                        static_cast<unsigned>(count));
        queries_to_bf16_kernel<<<grid, kQueryThreads, 0, stream>>>(
            src, src_pitch, static_cast<__nv_bfloat16*>(out), pitch);
    } else {
        const dim3 grid(static_cast<unsigned>((pitch / 16 + kQueryThreads - 1) / kQueryThreads),
                        static_cast<unsigned>(count));
        check_cuda(cudaMemsetAsync(amax_scratch, 0, count * sizeof(unsigned int), stream),
                   "cannot clear query maxima");
        queries_amax_kernel<<<grid, kQueryThreads, 0, stream>>>(src, src_pitch, amax_scratch);
        queries_to_fp8_kernel<<<grid, kQueryThreads, 0, stream>>>(
            src, src_pitch, amax_scratch, static_cast<__nv_fp8_storage_t*>(out), pitch,
            scales);
    }
    check_cuda(cudaGetLastError(), "cannot launch the query rounding kernel");
}

LowpPlan plan_lowp(LowpType type, uint64_t rows, uint64_t pitch, uint64_t batch,
                   int sm_count)
{
    LowpPlan plan{};
    plan.bn = batch <= 16 ? 16 : batch <= 32 ? 32 : batch <= 64 ? 64 : batch <= 128 ? 128 : 256;
    plan.kblocks = static_cast<uint32_t>(pitch / (type == LowpType::fp8_e4m3 ? 128 : 64));
    const uint64_t tiles = ((batch + plan.bn - 1) / plan.bn) * ((rows + kTileRows - 1) / kTileRows);
    // One CTA per SM at a time: pick the K split count whose CTA count fills
    // its last wave best (at least 4 K slices per split, at most 4 waves
    // unless one split already exceeds that); ties go to fewer splits.
    const uint64_t sms = static_cast<uint64_t>(sm_count > 0 ? sm_count : 148);
    const uint64_t most = std::max<uint64_t>(1, plan.kblocks / 4);
    uint64_t splits = 1;
    double best = -1.0;
    for (uint64_t s = 1; s <= most; ++s) {
        const uint64_t ctas = tiles * s;
        if (s > 1 && ctas > 4 * sms) {
            break;
        }
        const uint64_t waves = (ctas + sms - 1) / sms;
        const double fill = static_cast<double>(ctas) / static_cast<double>(waves * sms);
        if (fill > best + 1e-9) {
            best = fill;
            splits = s;
        }
    }
    plan.kblocks_per_split =
        static_cast<uint32_t>((plan.kblocks + splits - 1) / splits);
    plan.splits = (plan.kblocks + plan.kblocks_per_split - 1) / plan.kblocks_per_split;
    return plan;
}

LowpPlan lowp_plan(LowpType type, uint64_t pitch, int bn, uint64_t splits)
{
    LowpPlan plan{};
    plan.bn = bn;
    plan.kblocks = static_cast<uint32_t>(pitch / (type == LowpType::fp8_e4m3 ? 128 : 64));
    splits = std::max<uint64_t>(1, std::min<uint64_t>(splits, plan.kblocks));
    plan.kblocks_per_split = static_cast<uint32_t>((plan.kblocks + splits - 1) / splits);
    plan.splits = (plan.kblocks + plan.kblocks_per_split - 1) / plan.kblocks_per_split;
    return plan;
}

std::vector<LowpPlan> lowp_candidates(LowpType type, uint64_t rows, uint64_t pitch,
                                      uint64_t batch, int sm_count)
{
    std::vector<LowpPlan> out;
    out.push_back(plan_lowp(type, rows, pitch, batch, sm_count));
    const uint64_t kblocks = pitch / (type == LowpType::fp8_e4m3 ? 128 : 64);
    for (int bn : {16, 32, 64, 128, 256}) {
        if (bn > 16 && static_cast<uint64_t>(bn) / 2 >= batch) {
            continue;  // wider than twice the batch: only padding
        }
        for (uint64_t splits : {1, 2, 3, 4, 6, 8, 12, 16}) {
            if (splits <= std::max<uint64_t>(1, kblocks / 4)) {
                out.push_back(lowp_plan(type, pitch, bn, splits));
            }
        }
    }
    std::vector<LowpPlan> unique;
    for (const LowpPlan& p : out) {
        bool seen = false;
        for (const LowpPlan& u : unique) {
            seen = seen || (u.bn == p.bn && u.splits == p.splits &&
                            u.kblocks_per_split == p.kblocks_per_split);
        }
        if (!seen) {
            unique.push_back(p);
        }
    }
    return unique;
}

void launch_lowp_scores(const LowpPlan& plan, LowpType type, const void* rows_lp,
                        const float* row_scale, uint64_t row_count,
                        const void* queries_lp, const float* query_scale,
                        uint64_t batch, uint64_t pitch, float* partials,
                        int* error_flag, cudaStream_t stream, const FilterArgs* filter,
                        uint64_t sample_rows)
{
    if (filter != nullptr && plan.splits != 1) {
        fail(UHA_LOGIC_ERROR, "the fused candidate filter needs one K split");
    }
    // every row, or a sample of whole tiles spread over the index
    RowTiles tiles{1, static_cast<uint32_t>(row_count)};
    uint64_t out_rows = row_count;
    if (sample_rows != 0 && sample_rows < row_count) {
        tiles.stride = sample_tile_stride(row_count, sample_rows);
        out_rows = sample_rows;
    }
    const bool fp8 = type == LowpType::fp8_e4m3;
    // the row buffer holds lowp_padded_count(row_count) vectors (zero past
    // row_count), so no box leaves it
    const CUtensorMap rows_map =
        make_map(rows_lp, fp8, pitch, round_up(row_count, kTileRows), kTileRows);
    if (fp8) {
        launch_gemm_typed<true>(plan, rows_map, queries_lp, pitch,
                                static_cast<uint32_t>(out_rows),
                                static_cast<uint32_t>(batch), row_scale, query_scale,
                                partials, filter, tiles, error_flag, stream);
    } else {
        launch_gemm_typed<false>(plan, rows_map, queries_lp, pitch,
                                 static_cast<uint32_t>(out_rows),
                                 static_cast<uint32_t>(batch), row_scale, query_scale,
                                 partials, filter, tiles, error_flag, stream);
    }
}

void launch_lowp_topk(const float* partials, uint32_t splits, uint32_t batch,
                      uint32_t rows, const float* norms, uint32_t k,
                      uint32_t* candidates, cudaStream_t stream)
{
    if (batch == 0) {
        return;
    }
    // up to 16 candidates: short per-thread lists; up to 32: the warp list
    if (k <= 8) {
        topk_kernel<8><<<batch, kTopkThreads, 0, stream>>>(partials, splits, batch, rows,
                                                           norms, k, candidates);
    } else if (k <= 16) {
        topk_kernel<16><<<batch, kTopkThreads, 0, stream>>>(partials, splits, batch, rows,
                                                            norms, k, candidates);
    } else if (k <= 32 && splits == 1) {
        warp_topk_kernel<true><<<batch, kTopkThreads, 0, stream>>>(partials, splits, batch,
                                                                   rows, norms, k, candidates);
    } else if (k <= 32) {
        warp_topk_kernel<false><<<batch, kTopkThreads, 0, stream>>>(partials, splits, batch,
                                                                    rows, norms, k, candidates);
    } else {
        topk_kernel<64><<<batch, kTopkThreads, 0, stream>>>(partials, splits, batch, rows,
                                                            norms, k, candidates);
    }
    check_cuda(cudaGetLastError(), "cannot launch the candidate selection kernel");
}

uint32_t sample_tile_stride(uint64_t rows, uint64_t sample_rows)
{
    const uint64_t tiles = (rows + kTileRows - 1) / kTileRows;
    const uint64_t sampled = std::max<uint64_t>(1, sample_rows / kTileRows);
    return static_cast<uint32_t>(std::max<uint64_t>(1, tiles / sampled));
}

uint64_t filter_sample_rows(uint64_t rows)
{
    // about a sixteenth of the rows in whole tiles: about 16 k keys per query
    // pass the threshold
    const uint64_t s = rows / 16 / kTileRows * kTileRows;
    return std::min<uint64_t>(rows, std::max<uint64_t>(s, 1024));
}

uint32_t filter_capacity(uint64_t rows, uint32_t k)
{
    // four times the expected list length, at least 2,048
    const uint64_t expected = static_cast<uint64_t>(k) *
                              ((rows + filter_sample_rows(rows) - 1) / filter_sample_rows(rows));
    return static_cast<uint32_t>(std::max<uint64_t>(2048, 4 * expected));
}

void launch_lowp_threshold(const float* partials, uint32_t batch, uint32_t sample_rows,
                           const float* sample_norms, uint32_t k,
                           const uint32_t* sample_candidates, float* tau,
                           cudaStream_t stream)
{
    if (batch == 0) {
        return;
    }
    threshold_kernel<<<(batch + 255) / 256, 256, 0, stream>>>(partials, batch, sample_rows,
                                                              sample_norms, k,
                                                              sample_candidates, tau);
    check_cuda(cudaGetLastError(), "cannot launch the candidate threshold kernel");
}

void launch_gather_sample_norms(const float* norms, uint64_t rows, uint32_t sample_rows,
                                float* out, cudaStream_t stream)
{
    if (sample_rows == 0) {
        return;
    }
    const uint32_t stride = sample_rows < rows ? sample_tile_stride(rows, sample_rows) : 1u;
    sample_norms_kernel<<<(sample_rows + 255) / 256, 256, 0, stream>>>(norms, sample_rows,
                                                                       stride, out);
    check_cuda(cudaGetLastError(), "cannot launch the sample norm kernel");
}

void launch_lowp_select(const unsigned long long* keys, const uint32_t* count, uint32_t cap,
                        uint32_t batch, uint32_t k, uint32_t* candidates, int* error_flag,
                        cudaStream_t stream)
{
    if (batch == 0) {
        return;
    }
    if (k <= 32) {
        constexpr uint32_t per_cta = kTopkThreads / 32;
        warp_select_kernel<<<(batch + per_cta - 1) / per_cta, kTopkThreads, 0, stream>>>(
            keys, count, cap, batch, k, candidates, error_flag);
    } else {
        select_kernel<64><<<batch, kTopkThreads, 0, stream>>>(keys, count, cap, k,
                                                             candidates, error_flag);
    }
    check_cuda(cudaGetLastError(), "cannot launch the filtered selection kernel");
}

}  // namespace uha
