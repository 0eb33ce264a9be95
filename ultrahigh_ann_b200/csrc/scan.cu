// Distance scans of prepared queries against the device rows.
//
// Both kernels write binary32 partial sums partials[chunk][query][row]; the
// certifying finalize kernel adds the chunks in order and bounds the result.
// The accumulation structure of each kernel is fixed, so the longest chain of
// binary32 additions per distance (plan.depth) is known on the host and turns
// into the certification bound.
//
// * stream kernel (batch <= 8): HBM-bound regime. A CTA owns 16 rows x one
//   2048-column chunk; the query chunk is staged in shared memory once and each
//   warp streams two rows with 128-bit non-allocating loads.
// * tile kernel (batch > 8): CUDA-core-bound regime. A CTA computes a 128-row x
//   64-query tile with an 8x8 register micro-tile per thread; 32-column stages
//   are double-buffered through shared memory with cp.async, and the K range
//   may be split across CTAs (split-K) to fill the 148 SMs.
#include "common.h"
#include "kernels.h"
#include "stage_bodies.h"
#include "tile_body.cuh"

#include <vector>

#include <algorithm>

namespace uha {
namespace {

using namespace tilebody;

constexpr uint32_t kStreamChunk = 2048;  // columns per stream chunk
constexpr uint32_t kStreamWarps = 8;
constexpr uint32_t kRowsPerWarp = 2;
constexpr uint32_t kStreamRows = kStreamWarps * kRowsPerWarp;


__device__ __forceinline__ float4 load_streaming(const float4* p)
{
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}

template <int NQ, int OP>
__global__ void __launch_bounds__(kStreamWarps * 32)
    stream_scan_kernel(const float* __restrict__ rows, uint32_t row_count,
                       uint32_t padded_dim, const float* __restrict__ weights,
                       const float* __restrict__ queries, uint32_t batch,
                       float* __restrict__ partials)
{
    extern __shared__ float4 smem4[];
    float4* sq = smem4;                              // [NQ][kStreamChunk / 4]
    float4* sw = smem4 + NQ * (kStreamChunk / 4);    // [kStreamChunk / 4]

    const uint32_t chunk = blockIdx.y;
    const uint32_t c0 = chunk * kStreamChunk;
    const uint32_t clen = min(kStreamChunk, padded_dim - c0);
    const uint32_t n4 = clen / 4;
    const uint32_t q0 = blockIdx.z * NQ;

    for (uint32_t i = threadIdx.x; i < NQ * n4; i += blockDim.x) {
        const uint32_t qq = i / n4;
        const uint32_t j = i - qq * n4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q0 + qq < batch) {
            v = __ldg(reinterpret_cast<const float4*>(
                          queries + static_cast<uint64_t>(q0 + qq) * padded_dim +
                          c0) + j);
        }
        sq[qq * (kStreamChunk / 4) + j] = v;
    }
    if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
        for (uint32_t j = threadIdx.x; j < n4; j += blockDim.x) {
            sw[j] = __ldg(reinterpret_cast<const float4*>(weights + c0) + j);
        }
    }
    __syncthreads();

    const uint32_t warp = threadIdx.x / 32;
    const uint32_t lane = threadIdx.x % 32;
    const uint32_t row0 = blockIdx.x * kStreamRows + warp * kRowsPerWarp;

    float acc[kRowsPerWarp][NQ];
    const float4* rp[kRowsPerWarp];
    bool valid[kRowsPerWarp];
#pragma unroll
    for (uint32_t rr = 0; rr < kRowsPerWarp; ++rr) {
        valid[rr] = row0 + rr < row_count;
        rp[rr] = reinterpret_cast<const float4*>(
            rows + static_cast<uint64_t>(valid[rr] ? row0 + rr : 0) *
                       padded_dim + c0);
#pragma unroll
        for (int qq = 0; qq < NQ; ++qq) {
            acc[rr][qq] = 0.f;
        }
    }

    const float4 one4 = make_float4(1.f, 1.f, 1.f, 1.f);
#pragma unroll 4
    for (uint32_t j = lane; j < n4; j += 32) {
        float4 rv[kRowsPerWarp];
#pragma unroll
        for (uint32_t rr = 0; rr < kRowsPerWarp; ++rr) {
            rv[rr] = valid[rr] ? load_streaming(rp[rr] + j)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float4 w = one4;
        if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
            w = sw[j];
        }
#pragma unroll
        for (int qq = 0; qq < NQ; ++qq) {
            const float4 q = sq[qq * (kStreamChunk / 4) + j];
#pragma unroll
            for (uint32_t rr = 0; rr < kRowsPerWarp; ++rr) {
                acc[rr][qq] = accumulate4<OP>(acc[rr][qq], q, rv[rr], w);
            }
        }
    }

#pragma unroll
    for (uint32_t rr = 0; rr < kRowsPerWarp; ++rr) {
#pragma unroll
        for (int qq = 0; qq < NQ; ++qq) {
            float v = acc[rr][qq];
#pragma unroll
            for (int offset = 16; offset > 0; offset /= 2) {
                v += __shfl_xor_sync(0xffffffffu, v, offset);
            }
            if (lane == rr * NQ + qq && valid[rr] && q0 + qq < batch) {
                partials[(static_cast<uint64_t>(chunk) * batch + q0 + qq) *
                             row_count + row0 + rr] = v;
            }
        }
    }
}

template <int OP>
__global__ void __launch_bounds__(kTileThreads)
    tile_scan_kernel(const float* __restrict__ rows, uint32_t row_count,
                     uint32_t padded_dim, const float* __restrict__ weights,
                     const float* __restrict__ queries, uint32_t batch,
                     uint32_t k_per_split, float* __restrict__ partials)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileShared& sm = *reinterpret_cast<TileShared*>(smem_raw);

    const uint32_t tid = threadIdx.x;
    const uint32_t tr = tid % 16;
    const uint32_t tq = tid / 16;
    const uint32_t row_base = blockIdx.x * kTileRows;
    const uint32_t query_base = blockIdx.y * kTileQueries;
    const uint32_t split = blockIdx.z;
    const uint32_t k_begin = split * k_per_split;
    const uint32_t k_end = min(padded_dim, k_begin + k_per_split);
    const uint32_t stages = (k_end - k_begin + kTileK - 1) / kTileK;

    auto load_stage = [&](uint32_t stage, uint32_t buffer) {
        const uint32_t k0 = k_begin + stage * kTileK;
        // rows: 128 x 8 float4 = 1024 copies, 8 per thread
#pragma unroll
        for (uint32_t it = 0; it < 8; ++it) {
            const uint32_t idx = tid + it * kTileThreads;
            const uint32_t r = idx / 8;
            const uint32_t c4 = idx % 8;
            const uint32_t col = k0 + c4 * 4;
            const bool ok = (row_base + r < row_count) && (col < k_end);
            const float* src =
                ok ? rows + static_cast<uint64_t>(row_base + r) * padded_dim +
                         col
                   : rows;
            cp_async16(&sm.rows[buffer][r][c4 * 4], src, ok);
        }
        // queries: 64 x 8 float4 = 512 copies, 4 per thread
#pragma unroll
        for (uint32_t it = 0; it < 4; ++it) {
            const uint32_t idx = tid + it * kTileThreads;
            const uint32_t q = idx / 8;
            const uint32_t c4 = idx % 8;
            const uint32_t col = k0 + c4 * 4;
            const bool ok = (query_base + q < batch) && (col < k_end);
            const float* src =
                ok ? queries +
                         static_cast<uint64_t>(query_base + q) * padded_dim +
                         col
                   : queries;
            cp_async16(&sm.queries[buffer][q][c4 * 4], src, ok);
        }
        if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
            if (tid < 8) {
                const uint32_t col = k0 + tid * 4;
                const bool ok = col < k_end;
                cp_async16(&sm.weights[buffer][tid * 4], ok ? weights + col
                                                            : weights,
                           ok);
            }
        }
        cp_async_commit();
    };

    float total[8][8];
    float part[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
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
            float4 qv[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                qv[j] = *reinterpret_cast<const float4*>(
                    &sm.queries[buffer][tq + 8 * j][kk]);
            }
            float4 w = make_float4(1.f, 1.f, 1.f, 1.f);
            if constexpr (OP == static_cast<int>(ScanOp::l1_weighted)) {
                w = *reinterpret_cast<const float4*>(&sm.weights[buffer][kk]);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float4 rv = *reinterpret_cast<const float4*>(
                    &sm.rows[buffer][tr + 16 * i][kk]);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    part[i][j] = accumulate4<OP>(part[i][j], qv[j], rv, w);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                total[i][j] += part[i][j];
                part[i][j] = 0.f;
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t q = query_base + tq + 8 * j;
        if (q >= batch) {
            continue;
        }
        float* out = partials + (static_cast<uint64_t>(split) * batch + q) *
                                    row_count;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t r = row_base + tr + 16 * i;
            if (r < row_count) {
                out[r] = total[i][j];
            }
        }
    }
}

template <int NQ>
void launch_stream_nq(ScanOp op, dim3 grid, size_t smem, cudaStream_t stream,
                      const float* rows, uint32_t row_count, uint32_t pd,
                      const float* weights, const float* queries,
                      uint32_t batch, float* partials)
{
    switch (op) {
    case ScanOp::l2:
        stream_scan_kernel<NQ, 0><<<grid, kStreamWarps * 32, smem, stream>>>(
            rows, row_count, pd, weights, queries, batch, partials);
        break;
    case ScanOp::l1:
        stream_scan_kernel<NQ, 1><<<grid, kStreamWarps * 32, smem, stream>>>(
            rows, row_count, pd, weights, queries, batch, partials);
        break;
    case ScanOp::l1_weighted:
        stream_scan_kernel<NQ, 2><<<grid, kStreamWarps * 32, smem, stream>>>(
            rows, row_count, pd, weights, queries, batch, partials);
        break;
    case ScanOp::dot:
        stream_scan_kernel<NQ, 3><<<grid, kStreamWarps * 32, smem, stream>>>(
            rows, row_count, pd, weights, queries, batch, partials);
        break;
    }
}

template <int OP>
void launch_tile_op(dim3 grid, cudaStream_t stream, const float* rows,
                    uint32_t row_count, uint32_t pd, const float* weights,
                    const float* queries, uint32_t batch, uint32_t k_per_split,
                    float* partials)
{
    const size_t smem = sizeof(TileShared);
    static bool configured[kMaxDevices] = {};
    const int dev = current_device();
    if (!configured[dev]) {
        check_cuda(cudaFuncSetAttribute(
                       tile_scan_kernel<OP>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem)),
                   "cannot configure tile scan kernel");
        configured[dev] = true;
    }
    tile_scan_kernel<OP><<<grid, kTileThreads, smem, stream>>>(
        rows, row_count, pd, weights, queries, batch, k_per_split, partials);
}

}  // namespace

uint64_t tile_scan_smem_bytes()
{
    return sizeof(TileShared);
}

void tile_scan_grid(uint64_t row_count, uint64_t batch, uint32_t splits, uint32_t* gx,
                    uint32_t* gy, uint32_t* gz)
{
    *gx = static_cast<uint32_t>((row_count + kTileRows - 1) / kTileRows);
    *gy = static_cast<uint32_t>((batch + kTileQueries - 1) / kTileQueries);
    *gz = splits;
}

ScanPlan stream_plan(uint64_t padded_dim, int queries_per_pass)
{
    ScanPlan plan{};
    plan.kernel = 0;
    plan.queries_per_pass = queries_per_pass;
    plan.chunks = static_cast<uint32_t>((padded_dim + kStreamChunk - 1) / kStreamChunk);
    // per lane: 4 additions per float4, kStreamChunk / 128 float4s per lane;
    // then 5 shuffle levels; then the chunk sum in the argmin.
    plan.depth = 4 * (kStreamChunk / 128) + 5 + plan.chunks;
    return plan;
}

ScanPlan tile_plan(uint64_t padded_dim, uint64_t splits)
{
    ScanPlan plan{};
    plan.kernel = 1;
    splits = std::max<uint64_t>(1, std::min(splits, std::max<uint64_t>(1, padded_dim / 512)));
    uint64_t k_per_split = round_up((padded_dim + splits - 1) / splits, kTileK);
    if (k_per_split == 0) {
        k_per_split = kTileK;
    }
    splits = (padded_dim + k_per_split - 1) / k_per_split;
    plan.k_per_split = static_cast<uint32_t>(k_per_split);
    plan.chunks = static_cast<uint32_t>(std::max<uint64_t>(1, splits));
    // 32 sequential additions inside a stage, one per stage into the total,
    // then the split sum in the argmin.
    plan.depth = static_cast<uint32_t>(kTileK + (k_per_split / kTileK) + plan.chunks);
    return plan;
}

ScanPlan plan_scan(uint64_t rows, uint64_t padded_dim, uint64_t batch,
                   int sm_count)
{
    if (batch <= 8) {
        int nq = 1;
        while (nq < static_cast<int>(batch)) {
            nq *= 2;
        }
        return stream_plan(padded_dim, nq);
    }
    const uint64_t row_tiles = (rows + kTileRows - 1) / kTileRows;
    const uint64_t query_tiles = (batch + kTileQueries - 1) / kTileQueries;
    const uint64_t tiles = row_tiles * query_tiles;
    // Two CTAs of the tile kernel fit an SM (registers). Pick the column split
    // count whose CTA count fills its last wave best, within four waves unless
    // one split already exceeds that; ties go to fewer splits.
    const uint64_t slots = 2ull * static_cast<uint64_t>(sm_count > 0 ? sm_count : 148);
    const uint64_t most = std::max<uint64_t>(1, padded_dim / 512);
    // at most 8192 columns per split: the accumulation depth (and with it the
    // certification bound, and the share of queries that need the binary64
    // replay) stays small
    const uint64_t least = std::min<uint64_t>(most, (padded_dim + 8191) / 8192);
    uint64_t splits = least;
    double best = -1.0;
    for (uint64_t s = least; s <= most; ++s) {
        const uint64_t ctas = tiles * s;
        if (s > least && ctas > 4 * slots) {
            break;
        }
        const uint64_t waves = (ctas + slots - 1) / slots;
        const double fill = static_cast<double>(ctas) / static_cast<double>(waves * slots);
        if (fill > best + 1e-9) {
            best = fill;
            splits = s;
        }
    }
    return tile_plan(padded_dim, splits);
}

std::vector<ScanPlan> scan_candidates(uint64_t rows, uint64_t padded_dim,
                                      uint64_t batch, int sm_count)
{
    std::vector<ScanPlan> out;
    out.push_back(plan_scan(rows, padded_dim, batch, sm_count));
    if (batch <= 64 || padded_dim <= 2048) {
        // the stream kernel re-reads the rows once per pass of up to 8
        // queries: a candidate for small batches, and for narrow rows (the
        // projected rows of hierarchies) whose re-reads stay in L2
        for (int nq : {1, 2, 4, 8}) {
            if (nq <= static_cast<int>(2 * batch)) {
                out.push_back(stream_plan(padded_dim, nq));
            }
        }
    }
    if (batch > 1) {
        for (uint64_t splits : {1, 2, 3, 4, 6, 8, 12, 16}) {
            out.push_back(tile_plan(padded_dim, splits));
        }
    }
    // drop duplicates (same kernel, pass width and split)
    std::vector<ScanPlan> unique;
    for (const ScanPlan& p : out) {
        bool seen = false;
        for (const ScanPlan& u : unique) {
            seen = seen || (u.kernel == p.kernel && u.queries_per_pass == p.queries_per_pass &&
                            u.chunks == p.chunks && u.k_per_split == p.k_per_split);
        }
        if (!seen) {
            unique.push_back(p);
        }
    }
    return unique;
}

void launch_scan(const ScanPlan& plan, ScanOp op, const float* rows,
                 uint64_t row_count, uint64_t padded_dim, const float* weights,
                 const float* queries, uint64_t batch, float* partials,
                 cudaStream_t stream)
{
    const uint32_t rc = static_cast<uint32_t>(row_count);
    const uint32_t pd = static_cast<uint32_t>(padded_dim);
    const uint32_t b = static_cast<uint32_t>(batch);
    if (plan.kernel == 0) {
        const int nq = plan.queries_per_pass;
        const dim3 grid(static_cast<uint32_t>((row_count + kStreamRows - 1) /
                                              kStreamRows),
                        plan.chunks, static_cast<uint32_t>(
                                         (batch + nq - 1) / nq));
        const size_t smem = (static_cast<size_t>(nq) + 1) * kStreamChunk *
                            sizeof(float);
        switch (nq) {
        case 1:
            launch_stream_nq<1>(op, grid, smem, stream, rows, rc, pd, weights,
                                queries, b, partials);
            break;
        case 2:
            launch_stream_nq<2>(op, grid, smem, stream, rows, rc, pd, weights,
                                queries, b, partials);
            break;
        case 4:
            launch_stream_nq<4>(op, grid, smem, stream, rows, rc, pd, weights,
                                queries, b, partials);
            break;
        default: {
            static bool configured[kMaxDevices] = {};
            const int dev = current_device();
            if (!configured[dev]) {
                for (auto fn : {stream_scan_kernel<8, 0>, stream_scan_kernel<8, 1>,
                                stream_scan_kernel<8, 2>, stream_scan_kernel<8, 3>}) {
                    check_cuda(cudaFuncSetAttribute(
                                   fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)),
                               "cannot configure stream scan kernel");
                }
                configured[dev] = true;
            }
            launch_stream_nq<8>(op, grid, smem, stream, rows, rc, pd, weights,
                                queries, b, partials);
            break;
        }
        }
    } else {
        const uint32_t k_per_split = plan.k_per_split;
        const dim3 grid(
            static_cast<uint32_t>((row_count + kTileRows - 1) / kTileRows),
            static_cast<uint32_t>((batch + kTileQueries - 1) / kTileQueries),
            plan.chunks);
        switch (op) {
        case ScanOp::l2:
            launch_tile_op<0>(grid, stream, rows, rc, pd, weights, queries, b,
                              k_per_split, partials);
            break;
        case ScanOp::l1:
            launch_tile_op<1>(grid, stream, rows, rc, pd, weights, queries, b,
                              k_per_split, partials);
            break;
        case ScanOp::l1_weighted:
            launch_tile_op<2>(grid, stream, rows, rc, pd, weights, queries, b,
                              k_per_split, partials);
            break;
        case ScanOp::dot:
            launch_tile_op<3>(grid, stream, rows, rc, pd, weights, queries, b,
                              k_per_split, partials);
            break;
        }
    }
    check_cuda(cudaGetLastError(), "cannot launch scan kernel");
}

}  // namespace uha
