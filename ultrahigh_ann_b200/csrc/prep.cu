// Query preparation and index-build kernels.
//
// Query side (one launch per batch):
// * dense: copy the B x d queries into the padded B x kp layout (kp a multiple
//   of 4 so every row starts on a 16-byte boundary) and flag non-finite
//   values (reference: detail::validate_finite_values(queries, "queries"),
//   src/core/cuda_dense_l2_scan_index.cu:611).
// * sampled: gather the sampled columns of each query, scale them for L2 with
//   one binary32 multiply (the host pack of the reference,
//   src/coordinate_sampling/l2_coordinate_embedding.cpp:114-124, and the
//   unscaled L1 pack, l1_coordinate_embedding.cpp:103-109) and flag
//   non-finite sampled values or products. Unsampled columns are never read.
//
// Build side: the same gather applied to the representative rows
// (l2_coordinate_embedding.cpp:71-79, filter_columns.cpp:10-36) and the row
// norms of the binary32 norm-identity strategy.
#include "common.h"
#include "hier_body.cuh"
#include "kernels.h"

#include <algorithm>

namespace uha {
namespace {

using hierbody::prepare_sampled_loop;

constexpr int kThreads = 256;

// error_flag bits: 1 = non-finite (sampled) query value,
//                  2 = non-finite weighted/scaled value
__global__ void prepare_dense_kernel(const float* __restrict__ queries,
                                     uint64_t batch, uint64_t dim,
                                     float* __restrict__ out,
                                     uint64_t padded_dim, int* error_flag)
{
    const uint64_t total = batch * padded_dim;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) +
                        threadIdx.x;
         idx < total; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t b = idx / padded_dim;
        const uint64_t i = idx - b * padded_dim;
        float v = 0.f;
        if (i < dim) {
            v = queries[b * dim + i];
            if (!isfinite(v)) {
                atomicOr(error_flag, 1);
            }
        }
        out[idx] = v;
    }
}

// The same for rows of a multiple of 4 floats starting on 16-byte
// boundaries: grid (column groups of 4 x kThreads, queries).
__global__ void prepare_dense_vec_kernel(const float* __restrict__ queries, uint64_t dim,
                                         float* __restrict__ out, uint64_t padded_dim,
                                         int* error_flag)
{
    const uint64_t b = blockIdx.y;
    const uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t i = 4 * g;
    if (i >= padded_dim) {
        return;
    }
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (i < dim) {
        v = __ldg(reinterpret_cast<const float4*>(queries + b * dim + i));
        if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w))) {
            atomicOr(error_flag, 1);
        }
    }
    *reinterpret_cast<float4*>(out + b * padded_dim + i) = v;
}

__global__ void prepare_sampled_kernel(const float* __restrict__ queries,
                                       uint64_t batch, uint64_t dim,
                                       const uint32_t* __restrict__ columns,
                                       const float* __restrict__ scales,
                                       uint64_t sample_size,
                                       float* __restrict__ out,
                                       uint64_t padded_dim, int* error_flag)
{
    prepare_sampled_loop(queries, batch, dim, columns, scales, sample_size, out, padded_dim,
                         error_flag, blockIdx.x, gridDim.x, blockDim.x);
}

__global__ void query_norms_kernel(const float* __restrict__ prepared,
                                   uint64_t batch, uint64_t padded_dim,
                                   float* __restrict__ norms)
{
    const uint64_t warp_id =
        (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (warp_id >= batch) {
        return;
    }
    const float* row = prepared + warp_id * padded_dim;
    float acc = 0.f;
    for (uint64_t i = lane; i < padded_dim; i += 32) {
        acc = fmaf(row[i], row[i], acc);
    }
    for (int offset = 16; offset > 0; offset /= 2) {
        acc += __shfl_xor_sync(0xffffffffu, acc, offset);
    }
    if (lane == 0) {
        norms[warp_id] = acc;
    }
}

__global__ void gather_rows_kernel(const float* __restrict__ source,
                                   uint64_t row_count, uint64_t dim,
                                   const uint32_t* __restrict__ columns,
                                   const float* __restrict__ scales,
                                   uint64_t sample_size,
                                   float* __restrict__ out,
                                   uint64_t padded_dim)
{
    const uint64_t total = row_count * padded_dim;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) +
                        threadIdx.x;
         idx < total; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t r = idx / padded_dim;
        const uint64_t i = idx - r * padded_dim;
        float v = 0.f;
        if (i < sample_size) {
            v = source[r * dim + columns[i]];
            if (scales != nullptr) {
                v = __fmul_rn(v, scales[i]);
            }
        }
        out[idx] = v;
    }
}

// Build-time gather from a device-resident matrix (binary32, or BF16 decoded
// exactly to binary32) with a row stride: out[r][i] = source[r][column i]
// (times scales[i] when given; columns == nullptr reads column i). When
// first_bad is given, first_bad[0] / [1] receive the smallest r * k + i whose
// source value / scaled value is not finite (the host validation's order).
template <bool BF16>
__global__ void gather_device_rows_kernel(const void* __restrict__ source,
                                          uint64_t stride, uint64_t row_count,
                                          const uint32_t* __restrict__ columns,
                                          const float* __restrict__ scales,
                                          uint64_t sample_size,
                                          float* __restrict__ out,
                                          uint64_t padded_dim,
                                          unsigned long long* first_bad)
{
    const uint64_t total = row_count * padded_dim;
    for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) +
                        threadIdx.x;
         idx < total; idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t r = idx / padded_dim;
        const uint64_t i = idx - r * padded_dim;
        float v = 0.f;
        if (i < sample_size) {
            const uint64_t at = r * stride + (columns != nullptr ? columns[i] : i);
            if constexpr (BF16) {
                const uint32_t bits = static_cast<const uint16_t*>(source)[at];
                v = __uint_as_float(bits << 16);
            } else {
                v = static_cast<const float*>(source)[at];
            }
            const unsigned long long linear = r * sample_size + i;
            if (first_bad != nullptr && !isfinite(v)) {
                atomicMin(first_bad, linear);
            }
            if (scales != nullptr) {
                v = __fmul_rn(v, scales[i]);
                if (first_bad != nullptr && !isfinite(v)) {
                    atomicMin(first_bad + 1, linear);
                }
            }
        }
        out[idx] = v;
    }
}

uint32_t grid_for(uint64_t total)
{
    const uint64_t blocks = (total + kThreads - 1) / kThreads;
    return static_cast<uint32_t>(blocks < 148ull * 64 ? (blocks == 0 ? 1 : blocks)
                                                      : 148ull * 64);
}

// out[q][j] = sources[q][j] for j < dim: the queries of one batch gathered
// from individually addressed device vectors (grid: column chunks x queries).
__global__ void gather_vectors_kernel(const float* const* __restrict__ sources,
                                      uint64_t dim, float* __restrict__ out)
{
    const uint64_t q = blockIdx.y;
    const float* src = sources[q];
    float* dst = out + q * dim;
    for (uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; j < dim;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        dst[j] = src[j];
    }
}

}  // namespace

void launch_gather_vectors(const float* const* sources, uint64_t count, uint64_t dim,
                           float* out, cudaStream_t stream)
{
    if (count == 0 || dim == 0) {
        return;
    }
    const uint64_t chunks = std::min<uint64_t>((dim + kThreads - 1) / kThreads, 64);
    gather_vectors_kernel<<<dim3(static_cast<uint32_t>(chunks), static_cast<uint32_t>(count)),
                            kThreads, 0, stream>>>(sources, dim, out);
    check_cuda(cudaGetLastError(), "cannot launch query gather kernel");
}

void launch_prepare_dense(const float* queries, uint64_t batch, uint64_t dim,
                          float* out, uint64_t padded_dim, int* error_flag,
                          cudaStream_t stream)
{
    if (batch == 0 || padded_dim == 0) {
        return;
    }
    const bool aligned = dim % 4 == 0 && (reinterpret_cast<uintptr_t>(queries) % 16) == 0;
    if (aligned && batch <= 65535) {
        // one thread per 4 columns, 16-byte loads and stores
        const uint64_t groups = padded_dim / 4;
        const dim3 grid(static_cast<uint32_t>((groups + kThreads - 1) / kThreads),
                        static_cast<uint32_t>(batch));
        prepare_dense_vec_kernel<<<grid, kThreads, 0, stream>>>(queries, dim, out, padded_dim,
                                                                 error_flag);
    } else {
        prepare_dense_kernel<<<grid_for(batch * padded_dim), kThreads, 0, stream>>>(
            queries, batch, dim, out, padded_dim, error_flag);
    }
    check_cuda(cudaGetLastError(), "cannot launch query preparation kernel");
}

void launch_prepare_sampled(const float* queries, uint64_t batch, uint64_t dim,
                            const uint32_t* columns, const float* scales,
                            uint64_t sample_size, float* out,
                            uint64_t padded_dim, int* error_flag,
                            cudaStream_t stream)
{
    prepare_sampled_kernel<<<grid_for(batch * padded_dim), kThreads, 0,
                             stream>>>(queries, batch, dim, columns, scales,
                                       sample_size, out, padded_dim,
                                       error_flag);
    check_cuda(cudaGetLastError(), "cannot launch query gather kernel");
}

void launch_query_norms(const float* prepared, uint64_t batch,
                        uint64_t padded_dim, float* norms, cudaStream_t stream)
{
    const uint64_t threads = batch * 32;
    query_norms_kernel<<<static_cast<uint32_t>((threads + kThreads - 1) /
                                               kThreads),
                         kThreads, 0, stream>>>(prepared, batch, padded_dim,
                                                norms);
    check_cuda(cudaGetLastError(), "cannot launch query norm kernel");
}

void launch_gather_rows(const float* source, uint64_t row_count, uint64_t dim,
                        const uint32_t* columns, const float* scales,
                        uint64_t sample_size, float* out, uint64_t padded_dim,
                        cudaStream_t stream)
{
    gather_rows_kernel<<<grid_for(row_count * padded_dim), kThreads, 0,
                         stream>>>(source, row_count, dim, columns, scales,
                                   sample_size, out, padded_dim);
    check_cuda(cudaGetLastError(), "cannot launch row gather kernel");
}

void launch_gather_device_rows(const void* source, bool bf16, uint64_t stride,
                               uint64_t row_count, const uint32_t* columns,
                               const float* scales, uint64_t sample_size,
                               float* out, uint64_t padded_dim,
                               unsigned long long* first_bad, cudaStream_t stream)
{
    const uint32_t grid = grid_for(row_count * padded_dim);
    if (bf16) {
        gather_device_rows_kernel<true><<<grid, kThreads, 0, stream>>>(
            source, stride, row_count, columns, scales, sample_size, out, padded_dim,
            first_bad);
    } else {
        gather_device_rows_kernel<false><<<grid, kThreads, 0, stream>>>(
            source, stride, row_count, columns, scales, sample_size, out, padded_dim,
            first_bad);
    }
    check_cuda(cudaGetLastError(), "cannot launch device row gather kernel");
}

void launch_row_norms(const float* rows, uint64_t row_count,
                      uint64_t padded_dim, float* norms, cudaStream_t stream)
{
    launch_query_norms(rows, row_count, padded_dim, norms, stream);
}

}  // namespace uha
