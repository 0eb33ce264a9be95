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
#include "hier_body.cuh"
#include "kernels.h"
#include "stage_bodies.h"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace uha {
namespace {

using namespace hierbody;

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

__global__ void __launch_bounds__(kProjQueries * kProjCols)
    project_queries_kernel(const float* __restrict__ x, uint64_t batch,
                           uint64_t padded_k, uint64_t k,
                           const float* __restrict__ proj, uint64_t p,
                           float* __restrict__ y, uint64_t padded_p,
                           float* __restrict__ err_acc, float* __restrict__ coord_err,
                           double err_per_abs, bool euclidean, int* error_flag)
{
    __shared__ ProjShared sh;
    project_queries_block(x, batch, padded_k, k, proj, p, y, padded_p, err_acc, coord_err,
                          err_per_abs, euclidean, error_flag, blockIdx.x, blockIdx.y, sh);
}

__global__ void finish_query_err_kernel(float* err, uint64_t batch,
                                        bool euclidean)
{
    // one thread per query: the grid covers the batch
    finish_query_err_loop(err, batch, euclidean, blockIdx.x, gridDim.x, blockDim.x);
}

template <int PER_LANE>
__global__ void __launch_bounds__(kThreads)
    median_sample_kernel(const float* __restrict__ rows, uint32_t row_count,
                         uint32_t padded_p, uint32_t p, const float* __restrict__ queries,
                         uint32_t batch, uint32_t samples, float* __restrict__ partials,
                         unsigned int* __restrict__ min_bits)
{
    median_sample_loop<PER_LANE>(rows, row_count, padded_p, p, queries, batch, samples,
                                 partials, min_bits, blockIdx.x, gridDim.x, blockDim.x);
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
    extern __shared__ float4 ys4[];  // [Q][padded_p / 4]
    median_count_block<Q>(rows_t, r_pitch, row_count, padded_p, p, queries, batch, q_begin,
                          min_bits, query_err, row_err_max, rel, abs_err, partials,
                          blockIdx.x, blockIdx.y, ys4, threadIdx.x, 0);
}

template <int PER_LANE>
__global__ void __launch_bounds__(kThreads)
    median_survivor_kernel(const float* __restrict__ rows, uint32_t row_count,
                           uint32_t padded_p, uint32_t p,
                           const float* __restrict__ queries, uint32_t batch,
                           const float* __restrict__ coord_err,
                           float* __restrict__ partials, float* __restrict__ pair_err)
{
    median_survivor_loop<PER_LANE>(rows, row_count, padded_p, p, queries, batch, coord_err,
                                   partials, pair_err, blockIdx.x, gridDim.x, blockDim.x);
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
void launch_median_pair(const MedianPlan& plan, const float* rows, const float* rows_t,
                        uint32_t r_pitch, uint32_t rc, uint32_t pp, uint32_t pv,
                        const float* queries, uint32_t b, const float* query_err,
                        const float* coord_err, float row_err_max, float rel, float abs_err,
                        unsigned int* min_bits, float* partials, float* pair_err,
                        cudaStream_t stream)
{
    // grid-stride warps over the pairs: at most 16 resident CTAs' worth per SM
    const uint64_t cap = 148ull * 16;
    const uint32_t samples = plan.samples;
    const uint64_t sample_blocks =
        (static_cast<uint64_t>(samples) * b * 32 + kThreads - 1) / kThreads;
    median_sample_kernel<PER_LANE>
        <<<static_cast<uint32_t>(std::min(sample_blocks, cap)), kThreads, 0, stream>>>(
            rows, rc, pp, pv, queries, b, samples, partials, min_bits);
    const uint32_t q = plan.count_queries;
    if (q >= 8) {
        launch_median_count<8>(rows_t, r_pitch, rc, pp, pv, queries, b, min_bits, query_err,
                               row_err_max, rel, abs_err, partials, stream);
    } else if (q >= 4) {
        launch_median_count<4>(rows_t, r_pitch, rc, pp, pv, queries, b, min_bits, query_err,
                               row_err_max, rel, abs_err, partials, stream);
    } else if (q >= 2) {
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

__global__ void median_tuning_queries_kernel(const float* __restrict__ rows, uint32_t rc,
                                             uint32_t pp, uint32_t pv, uint32_t batch,
                                             float* __restrict__ queries)
{
    const uint64_t total = static_cast<uint64_t>(batch) * pp;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t q = i / pp;
        const uint32_t j = static_cast<uint32_t>(i % pp);
        const uint64_t a = (7919ull * q + 1) % rc;
        const uint64_t b = (104729ull * q + 3) % rc;
        queries[i] = j < pv ? 0.5f * (rows[a * pp + j] + rows[b * pp + j]) : 0.f;
    }
}

}  // namespace

MedianPlan default_median_plan(uint64_t row_count, uint64_t batch)
{
    return MedianPlan{median_samples(row_count),
                      static_cast<uint32_t>(median_count_queries(
                          static_cast<uint32_t>(std::min<uint64_t>(batch, 8))))};
}

std::vector<MedianPlan> median_candidates(uint64_t row_count, uint64_t batch)
{
    const MedianPlan base = default_median_plan(row_count, batch);
    std::vector<MedianPlan> out{base};
    // half and twice the sampled rows (32 to 1024, at most the row count)
    std::vector<uint32_t> samples{base.samples};
    for (uint64_t s : {static_cast<uint64_t>(base.samples) / 2,
                       static_cast<uint64_t>(base.samples) * 2}) {
        s = std::min<uint64_t>(std::max<uint64_t>(s, 32), std::min<uint64_t>(row_count, 1024));
        if (std::find(samples.begin(), samples.end(), s) == samples.end()) {
            samples.push_back(static_cast<uint32_t>(s));
        }
    }
    // the count with the default's queries per CTA and with half as many
    std::vector<uint32_t> widths{base.count_queries};
    if (base.count_queries > 1) {
        widths.push_back(base.count_queries / 2);
    }
    for (uint32_t s : samples) {
        for (uint32_t q : widths) {
            if (s != base.samples || q != base.count_queries) {
                out.push_back(MedianPlan{s, q});
            }
        }
    }
    return out;
}

void launch_median_tuning_queries(const float* rows, uint64_t row_count, uint64_t padded_p,
                                  uint64_t p, uint64_t batch, float* queries,
                                  cudaStream_t stream)
{
    if (row_count == 0 || batch == 0 || padded_p == 0) {
        return;
    }
    const uint64_t total = batch * padded_p;
    const uint32_t blocks =
        static_cast<uint32_t>(std::min<uint64_t>((total + kThreads - 1) / kThreads, 148 * 8));
    median_tuning_queries_kernel<<<blocks, kThreads, 0, stream>>>(
        rows, static_cast<uint32_t>(row_count), static_cast<uint32_t>(padded_p),
        static_cast<uint32_t>(p), static_cast<uint32_t>(batch), queries);
    check_cuda(cudaGetLastError(), "cannot launch tuning query kernel");
}

void launch_median_scan(const MedianPlan& plan, const float* rows, const float* rows_t,
                        uint64_t r_pitch, uint64_t row_count, uint64_t padded_p,
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
        launch_median_pair<1>(plan, rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 64) {
        launch_median_pair<2>(plan, rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 128) {
        launch_median_pair<4>(plan, rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 256) {
        launch_median_pair<8>(plan, rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 512) {
        launch_median_pair<16>(plan, rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else if (p <= 1024) {
        launch_median_pair<32>(plan, rows, rows_t, rp, rc, pp, pv, queries, b, query_err,
                               coord_err, row_err_max, rel, abs_err, min_bits, partials,
                               pair_err, stream);
    } else {
        fail(UHA_LENGTH_ERROR,
             "the L1 hierarchy supports projection dimensions up to 1024");
    }
    check_cuda(cudaGetLastError(), "cannot launch median scan kernel");
}

// ------------------------------------ shapes for the persistent batch kernel

uint64_t project_queries_smem_bytes()
{
    return sizeof(ProjShared);
}

void project_queries_grid(uint64_t batch, uint64_t padded_p, uint32_t* gx, uint32_t* gy)
{
    *gx = static_cast<uint32_t>((padded_p + kProjCols - 1) / kProjCols);
    *gy = static_cast<uint32_t>((batch + kProjQueries - 1) / kProjQueries);
}

uint32_t median_sample_blocks(uint32_t samples, uint32_t batch)
{
    const uint64_t cap = 148ull * 16;
    const uint64_t blocks =
        (static_cast<uint64_t>(samples) * batch * 32 + kThreads - 1) / kThreads;
    return static_cast<uint32_t>(std::min(blocks, cap));
}

int median_count_queries(uint32_t batch)
{
    return batch >= 8 ? 8 : batch >= 4 ? 4 : batch >= 2 ? 2 : 1;
}

void median_count_grid(uint32_t row_count, uint32_t batch, uint32_t q, uint32_t* gx,
                       uint32_t* gy)
{
    const uint32_t per_cta = kCountRows * (q >= 4 ? 2 : 1);
    *gx = (row_count + per_cta - 1) / per_cta;
    *gy = (batch + q - 1) / q;
}

uint32_t median_survivor_blocks(uint32_t row_count, uint32_t batch)
{
    const uint64_t cap = 148ull * 16;
    const uint64_t runs = (static_cast<uint64_t>(row_count) * batch + 31) / 32;
    const uint64_t blocks = (runs * 32 + kThreads - 1) / kThreads;
    return static_cast<uint32_t>(std::min(blocks, cap));
}

}  // namespace uha
