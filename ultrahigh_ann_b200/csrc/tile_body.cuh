// Device code of the binary32 tile scan shared by the scan kernels (scan.cu)
// and the persistent multi-index batch kernel (certify.cu): the per-component
// accumulation step of every scan, the cp.async staging helpers, the tile's
// shared-memory layout, and a 256-thread tile body.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "kernels.h"

namespace uha {
namespace tilebody {

constexpr uint32_t kTileRows = 128;
constexpr uint32_t kTileQueries = 64;
constexpr uint32_t kTileK = 32;
constexpr uint32_t kTileStride = kTileK + 4;  // padded smem row (floats)
constexpr uint32_t kTileThreads = 128;

// One accumulation step acc <- acc (+) f(q, r[, w]) per component, in the
// fixed order x, y, z, w.
template <int OP>
__device__ __forceinline__ float accumulate4(float acc, const float4& q,
                                             const float4& r, const float4& w)
{
    if constexpr (OP == static_cast<int>(ScanOp::l2)) {
        float d;
        d = q.x - r.x; acc = fmaf(d, d, acc);
        d = q.y - r.y; acc = fmaf(d, d, acc);
        d = q.z - r.z; acc = fmaf(d, d, acc);
        d = q.w - r.w; acc = fmaf(d, d, acc);
    } else if constexpr (OP == static_cast<int>(ScanOp::l1)) {
        acc += fabsf(q.x - r.x);
        acc += fabsf(q.y - r.y);
        acc += fabsf(q.z - r.z);
        acc += fabsf(q.w - r.w);
    } else if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
        acc = fmaf(fabsf(q.x - r.x), w.x, acc);
        acc = fmaf(fabsf(q.y - r.y), w.y, acc);
        acc = fmaf(fabsf(q.z - r.z), w.z, acc);
        acc = fmaf(fabsf(q.w - r.w), w.w, acc);
    } else {
        acc = fmaf(q.x, r.x, acc);
        acc = fmaf(q.y, r.y, acc);
        acc = fmaf(q.z, r.z, acc);
        acc = fmaf(q.w, r.w, acc);
    }
    return acc;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem,
                                           bool in_range)
{
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    const int src_bytes = in_range ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s),
                 "l"(gmem), "r"(src_bytes));
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;");
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N));
}

struct TileShared {
    float rows[2][kTileRows][kTileStride];
    float queries[2][kTileQueries][kTileStride];
    float weights[2][kTileK];
};

// The tile of tile_scan_kernel (128 rows x 64 queries, 32-column stages, the
// same per-output accumulation: a stage sum over the stage's columns in
// order, then one addition into the total) computed by 256 threads with an
// 8 x 4 micro-tile, about half the registers. Every output goes through the
// identical sequence of operations, so the partial sums are bit-identical to
// tile_scan_kernel's. Block (bx, by, bz) of the tile grid; smem: TileShared.
constexpr uint32_t kWideThreads = 256;

template <int OP>
__device__ __forceinline__ void tile_scan_wide_tile(
    const float* __restrict__ rows, uint32_t row_count, uint32_t padded_dim,
    const float* __restrict__ weights, const float* __restrict__ queries, uint32_t batch,
    uint32_t k_per_split, float* __restrict__ partials, uint32_t bx, uint32_t by,
    uint32_t bz, unsigned char* smem_raw)
{
    TileShared& sm = *reinterpret_cast<TileShared*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    const uint32_t tr = tid % 16;  // rows tr + 16 i, i < 8
    const uint32_t tq = tid / 16;  // queries tq + 16 j, j < 4
    const uint32_t row_base = bx * kTileRows;
    const uint32_t query_base = by * kTileQueries;
    const uint32_t split = bz;
    const uint32_t k_begin = split * k_per_split;
    const uint32_t k_end = min(padded_dim, k_begin + k_per_split);
    const uint32_t stages = (k_end - k_begin + kTileK - 1) / kTileK;

    auto load_stage = [&](uint32_t stage, uint32_t buffer) {
        const uint32_t k0 = k_begin + stage * kTileK;
#pragma unroll
        for (uint32_t it = 0; it < 4; ++it) {
            const uint32_t idx = tid + it * kWideThreads;
            const uint32_t r = idx / 8;
            const uint32_t c4 = idx % 8;
            const uint32_t col = k0 + c4 * 4;
            const bool ok = (row_base + r < row_count) && (col < k_end);
            const float* src =
                ok ? rows + static_cast<uint64_t>(row_base + r) * padded_dim + col : rows;
            cp_async16(&sm.rows[buffer][r][c4 * 4], src, ok);
        }
#pragma unroll
        for (uint32_t it = 0; it < 2; ++it) {
            const uint32_t idx = tid + it * kWideThreads;
            const uint32_t q = idx / 8;
            const uint32_t c4 = idx % 8;
            const uint32_t col = k0 + c4 * 4;
            const bool ok = (query_base + q < batch) && (col < k_end);
            const float* src =
                ok ? queries + static_cast<uint64_t>(query_base + q) * padded_dim + col
                   : queries;
            cp_async16(&sm.queries[buffer][q][c4 * 4], src, ok);
        }
        if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
            if (tid < 8) {
                const uint32_t col = k0 + tid * 4;
                const bool ok = col < k_end;
                cp_async16(&sm.weights[buffer][tid * 4], ok ? weights + col : weights, ok);
            }
        }
        cp_async_commit();
    };

    float total[8][4];
    float part[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            total[i][j] = 0.f;
            part[i][j] = 0.f;
        }
    }
    if (stages > 0) {
        load_stage(0, 0);
    }
    for (uint32_t s = 0; s < stages; ++s) {
        const uint32_t buffer = s & 1u;
        if (s + 1 < stages) {
            load_stage(s + 1, buffer ^ 1u);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (uint32_t kk = 0; kk < kTileK; kk += 4) {
            float4 qv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                qv[j] = *reinterpret_cast<const float4*>(&sm.queries[buffer][tq + 16 * j][kk]);
            }
            float4 w = make_float4(1.f, 1.f, 1.f, 1.f);
            if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
                w = *reinterpret_cast<const float4*>(&sm.weights[buffer][kk]);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float4 rv =
                    *reinterpret_cast<const float4*>(&sm.rows[buffer][tr + 16 * i][kk]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    part[i][j] = accumulate4<OP>(part[i][j], qv[j], rv, w);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                total[i][j] += part[i][j];
                part[i][j] = 0.f;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t q = query_base + tq + 16 * j;
        if (q >= batch) {
            continue;
        }
        float* out = partials + (static_cast<uint64_t>(split) * batch + q) * row_count;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t r = row_base + tr + 16 * i;
            if (r < row_count) {
                out[r] = total[i][j];
            }
        }
    }
}

}  // namespace tilebody
}  // namespace uha
