// C-ABI implementation: device-resident indexes, per-caller workspaces and
// the query pipeline
//
//   H2D (host queries only) -> prepare (gather/scale/validate) -> scan
//   -> finalize (certified argmin | binary32 norm identity)
//   -> D2H -> [resolve: binary64 replay of uncertified queries -> D2H]
//
// on the workspace's own stream. The resolve step runs only when the
// finalize kernel reported uncertified queries.
#include "common.h"
#include "index_types.h"
#include "engine_internal.h"
#include "kernels.h"
#include "stage_bodies.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

using uha::checked_add;
using uha::checked_mul;
using uha::check_cuda;
using uha::DeviceBuffer;
using uha::DeviceGuard;
using uha::fail;
using uha::guarded;
using uha::PinnedBuffer;

using uha::IndexKind;
using uha::kColumnAlign;
using uha::kMaxExtent;

namespace {

void require(bool condition, uha_status status, const char* message)
{
    if (!condition) {
        fail(status, message);
    }
}

void select_device(uha_index& index, int device)
{
    uha::clear_stale_cuda_error();
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        fail(UHA_RUNTIME_ERROR, "no usable CUDA device");
    }
    require(device >= 0 && device < count, UHA_INVALID_ARGUMENT,
            "CUDA device index is out of range");
    cudaDeviceProp prop{};
    check_cuda(cudaGetDeviceProperties(&prop, device),
               "cannot query CUDA device properties");
    index.device = device;
    index.device_name = prop.name;
    index.sm_count = prop.multiProcessorCount;
}

void validate_rows(const float* rows, uint64_t r, uint64_t d)
{
    require(r != 0, UHA_INVALID_ARGUMENT,
            "CUDA index expects at least one representative");
    require(r <= kMaxExtent && d <= kMaxExtent, UHA_LENGTH_ERROR,
            "CUDA index dimensions exceed the device grid limits");
    checked_mul(r, d, "representative matrix");
    require(rows != nullptr || d == 0, UHA_INVALID_ARGUMENT,
            "representative matrix must not be null");
}

// Where an index's representative matrix comes from: a host binary32 r x d
// matrix, or a matrix already on the index's device.
struct RowSource {
    const float* host = nullptr;
    const uha_device_matrix* device = nullptr;
};

void validate_device_matrix(const uha_device_matrix* m)
{
    require(m != nullptr, UHA_INVALID_ARGUMENT, "device matrix must not be null");
    require(m->type == UHA_VALUES_F32 || m->type == UHA_VALUES_BF16,
            UHA_INVALID_ARGUMENT, "unknown device matrix value type");
    require(m->rows != 0, UHA_INVALID_ARGUMENT,
            "CUDA index expects at least one representative");
    require(m->rows <= kMaxExtent && m->columns <= kMaxExtent, UHA_LENGTH_ERROR,
            "CUDA index dimensions exceed the device grid limits");
    require(m->row_stride >= m->columns, UHA_INVALID_ARGUMENT,
            "device matrix row stride is shorter than a row");
    checked_mul(m->rows, m->row_stride, "representative matrix");
    require(m->data != nullptr || m->columns == 0, UHA_INVALID_ARGUMENT,
            "representative matrix must not be null");
    const uint64_t element = m->type == UHA_VALUES_BF16 ? 2 : 4;
    require(reinterpret_cast<uintptr_t>(m->data) % element == 0, UHA_INVALID_ARGUMENT,
            "device matrix is not aligned to its element size");
}

// After select_device: the matrix must be memory of that device.
void require_on_device(const uha_device_matrix* m, int device)
{
    if (m->data == nullptr) {
        return;
    }
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, m->data);
    if (e != cudaSuccess) {
        cudaGetLastError();
    }
    require(e == cudaSuccess &&
                (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) &&
                a.device == device,
            UHA_INVALID_ARGUMENT, "device matrix is not memory of the index's device");
}

// Gathers columns (nullptr: 0..k-1) of a device-resident source into the
// r x padded layout `out`, times `scales` when given; returns the first
// non-finite source / scaled value's r * k + i (~0 when none).
std::pair<uint64_t, uint64_t> gather_device_source(const uha_device_matrix* m,
                                                   const uint32_t* columns,
                                                   const float* scales, uint64_t k,
                                                   float* out, uint64_t padded)
{
    DeviceBuffer<unsigned long long> bad(2);
    check_cuda(cudaMemset(bad.get(), 0xFF, bad.bytes()), "cannot clear flag");
    if (m->rows * padded != 0) {
        uha::launch_gather_device_rows(m->data, m->type == UHA_VALUES_BF16, m->row_stride,
                                       m->rows, columns, scales, k, out, padded, bad.get(),
                                       nullptr);
    }
    unsigned long long host[2] = {0, 0};
    check_cuda(cudaMemcpy(host, bad.get(), sizeof(host), cudaMemcpyDeviceToHost),
               "device row gather kernel failed");
    return {host[0], host[1]};
}

// Uploads a host r x d matrix into the padded r x pd device layout.
void upload_padded(DeviceBuffer<float>& dst, const float* src, uint64_t r,
                   uint64_t d, uint64_t pd)
{
    dst.allocate(checked_mul(r, pd, "padded representative matrix"));
    if (dst.size() == 0) {
        return;
    }
    check_cuda(cudaMemset(dst.get(), 0, dst.bytes()),
               "cannot clear representative matrix");
    if (d != 0) {
        check_cuda(cudaMemcpy2D(dst.get(), pd * sizeof(float), src,
                                d * sizeof(float), d * sizeof(float), r,
                                cudaMemcpyHostToDevice),
                   "cannot copy representatives to the CUDA device");
    }
}

template <typename T>
void upload(DeviceBuffer<T>& dst, const T* src, uint64_t count)
{
    dst.allocate(count);
    if (count != 0) {
        check_cuda(cudaMemcpy(dst.get(), src, count * sizeof(T),
                              cudaMemcpyHostToDevice),
                   "cannot copy index data to the CUDA device");
    }
}

// The binary64 weights as float pairs (hi = nearest binary32, lo = the
// nearest binary32 to the rest) for the emulated replay's float-float terms.
void upload_weights_ff(uha_index& index, const std::vector<double>& w64)
{
    std::vector<float> ff(2 * w64.size());
    for (size_t i = 0; i < w64.size(); ++i) {
        const float hi = static_cast<float>(w64[i]);
        ff[2 * i] = hi;
        ff[2 * i + 1] = static_cast<float>(w64[i] - static_cast<double>(hi));
    }
    upload(index.weights_ff, ff.data(), ff.size());
}

void compute_row_norms(uha_index& index)
{
    index.row_norms.allocate(index.rows);
    if (index.padded_dim == 0) {
        check_cuda(cudaMemset(index.row_norms.get(), 0, index.row_norms.bytes()),
                   "cannot clear row norms");
        return;
    }
    uha::launch_row_norms(index.scan_rows.get(), index.rows, index.padded_dim,
                          index.row_norms.get(), nullptr);
    check_cuda(cudaDeviceSynchronize(), "row norm kernel failed");
}

uint64_t workspace_payload(const uha_index& index, uint64_t b)
{
    const uint64_t r = index.rows;
    const uint64_t f = sizeof(float);
    const uint64_t z = sizeof(std::size_t);
    switch (index.kind) {
    case IndexKind::exact:
    case IndexKind::weighted:
        if (index.metric == UHA_L2) {
            return b * index.dimension * f + b * r * f + b * f + b * z;
        }
        return b * index.dimension * f + b * r * f + b * z;
    case IndexKind::sampled:
        if (index.metric == UHA_L2) {
            return 2 * (b * index.sample_size * f) + b * r * f + b * f + b * z;
        }
        return 2 * (b * index.sample_size * f) + b * r * f + b * z;
    case IndexKind::hierarchical: {
        // host sampled values, device sampled + projected values, the
        // projection's flag, then the scan buffers
        const uint64_t k = index.sample_size;
        const uint64_t p = index.projection_dimension;
        if (index.metric == UHA_L2) {
            return 2 * (b * k * f) + 2 * (b * p * f) + sizeof(int) + b * r * f +
                   b * f + b * z;
        }
        return 2 * (b * k * f) + b * p * f + sizeof(int) + b * r * f + b * z +
               sizeof(int);
    }
    }
    return 0;
}

}  // namespace

namespace uha {

// Relative and absolute certification bound for a binary32 distance built
// from per-term relative error (1 + u)^term_roundings and `depth` sequential
// binary32 additions, against the CPU's binary64 sum over `terms` terms.
Bound make_bound(uint32_t depth, uint64_t terms, int term_roundings)
{
    const double u32 = std::ldexp(1.0, -24);
    const double u64 = std::ldexp(1.0, -53);
    const double n32 = static_cast<double>(depth) + term_roundings + 1;
    const double n64 = static_cast<double>(terms) + 3;
    const double g32 = n32 * u32 / (1.0 - n32 * u32);
    const double g64 = n64 * u64 / (1.0 - n64 * u64);
    const double rel = 1.01 * (g32 + g64) / (1.0 - g32) + 4 * u32;
    const double abs = std::ldexp(n32 + 4, -149) * 4;
    return Bound{
        std::nextafter(static_cast<float>(rel), 1.0f),
        std::max(static_cast<float>(abs), std::ldexp(1.0f, -140)),
    };
}

// Bound of a parallel binary64 sum (longest addition chain `depth`) of the
// same `terms` rounded terms that the CPU adds sequentially:
// |S_gpu - S_cpu| <= (g(depth) + g(terms)) / (1 - g(depth)) * S_gpu, plus an
// absolute term for subnormal roundings.
Bound64 make_bound64(uint32_t depth, uint64_t terms)
{
    const double u = std::ldexp(1.0, -53);
    const double nd = static_cast<double>(depth) + 1;
    const double nt = static_cast<double>(terms) + 1;
    const double gd = nd * u / (1.0 - nd * u);
    const double gt = nt * u / (1.0 - nt * u);
    return Bound64{1.01 * (gd + gt) / (1.0 - gd) + 4 * u,
                   std::ldexp(nd + nt + 4, -1074) * 4};
}

}  // namespace uha

using uha::make_bound;

// ------------------------------------------------------------------ device

extern "C" int uha_cuda_available(void)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count > 0 ? 1 : 0;
}

extern "C" uha_status uha_device_info_get(int device, uha_device_info* out)
{
    return guarded([&] {
        require(out != nullptr, UHA_INVALID_ARGUMENT,
                "output pointer must not be null");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 ||
            device >= count) {
            cudaGetLastError();
            fail(UHA_RUNTIME_ERROR, "no usable CUDA device");
        }
        cudaDeviceProp prop{};
        check_cuda(cudaGetDeviceProperties(&prop, device),
                   "cannot query CUDA device properties");
        std::memset(out, 0, sizeof(*out));
        out->device = device;
        std::strncpy(out->device_name, prop.name, sizeof(out->device_name) - 1);
        out->compute_capability_major = prop.major;
        out->compute_capability_minor = prop.minor;
        out->total_global_memory_bytes = prop.totalGlobalMem;
        out->compiled_runtime_version = CUDART_VERSION;
        check_cuda(cudaRuntimeGetVersion(&out->runtime_version),
                   "cannot query CUDA runtime version");
        check_cuda(cudaDriverGetVersion(&out->driver_version),
                   "cannot query CUDA driver version");
    });
}

// ----------------------------------------------------------------- indexes

namespace {

void create_exact_index(int device, uha_metric metric, const RowSource& src,
                        uint64_t row_count, uint64_t dimension, uha_index** out)
{
    require(out != nullptr, UHA_INVALID_ARGUMENT,
            "output pointer must not be null");
    require(metric == UHA_L2 || metric == UHA_L1, UHA_INVALID_ARGUMENT,
            "unknown metric");
    if (src.host != nullptr || src.device == nullptr) {
        const float* rows = src.host;
        validate_rows(rows, row_count, dimension);
        const uint64_t total = row_count * dimension;
        for (uint64_t i = 0; i < total; ++i) {
            if (!std::isfinite(rows[i])) {
                fail(UHA_INVALID_ARGUMENT, "representatives must be finite");
            }
        }
    } else {
        validate_device_matrix(src.device);
    }
    auto index = std::make_unique<uha_index>();
    select_device(*index, device);
    DeviceGuard guard(device);
    index->kind = IndexKind::exact;
    index->metric = metric;
    index->rows = row_count;
    index->dimension = dimension;
    index->scan_dim = dimension;
    index->padded_dim = uha::round_up(dimension, kColumnAlign);
    require(index->padded_dim <= kMaxExtent, UHA_LENGTH_ERROR,
            "CUDA index dimensions exceed the device grid limits");
    if (src.device == nullptr) {
        upload_padded(index->scan_rows, src.host, row_count, dimension,
                      index->padded_dim);
    } else {
        require_on_device(src.device, device);
        index->scan_rows.allocate(
            checked_mul(row_count, index->padded_dim, "padded representative matrix"));
        if (gather_device_source(src.device, nullptr, nullptr, dimension,
                                 index->scan_rows.get(), index->padded_dim)
                .first != ~0ull) {
            fail(UHA_INVALID_ARGUMENT, "representatives must be finite");
        }
    }
    const uint64_t f = sizeof(float);
    if (metric == UHA_L2) {
        compute_row_norms(*index);
        index->usage.index_payload_bytes =
            row_count * dimension * f + row_count * f;
    } else {
        index->usage.index_payload_bytes = row_count * dimension * f;
    }
    index->usage.query_workspace_payload_bytes = 0;
    index->usage.unique_query_coordinates = dimension;
    index->usage.sampled_multiplicity = dimension;
    *out = index.release();
}

}  // namespace

extern "C" uha_status uha_exact_index_create(int device, uha_metric metric,
                                             const float* rows,
                                             uint64_t row_count,
                                             uint64_t dimension,
                                             uha_index** out)
{
    return guarded([&] {
        create_exact_index(device, metric, RowSource{rows, nullptr}, row_count, dimension,
                           out);
    });
}

extern "C" uha_status uha_exact_index_create_device(int device, uha_metric metric,
                                                    const uha_device_matrix* rows,
                                                    uha_index** out)
{
    return guarded([&] {
        require(rows != nullptr, UHA_INVALID_ARGUMENT, "device matrix must not be null");
        create_exact_index(device, metric, RowSource{nullptr, rows}, rows->rows,
                           rows->columns, out);
    });
}

extern "C" uha_status uha_weighted_l1_index_create(int device,
                                                   const float* rows,
                                                   uint64_t row_count,
                                                   uint64_t dimension,
                                                   const float* weights,
                                                   uha_index** out)
{
    return guarded([&] {
        require(out != nullptr, UHA_INVALID_ARGUMENT,
                "output pointer must not be null");
        validate_rows(rows, row_count, dimension);
        require(weights != nullptr || dimension == 0, UHA_INVALID_ARGUMENT,
                "coordinate weights must not be null");
        for (uint64_t i = 0; i < row_count * dimension; ++i) {
            if (!std::isfinite(rows[i])) {
                fail(UHA_INVALID_ARGUMENT, "representatives must be finite");
            }
        }
        for (uint64_t i = 0; i < dimension; ++i) {
            if (!std::isfinite(weights[i]) || weights[i] < 0.0f) {
                fail(UHA_INVALID_ARGUMENT,
                     "coordinate weights must be finite and nonnegative");
            }
        }
        auto index = std::make_unique<uha_index>();
        select_device(*index, device);
        DeviceGuard guard(device);
        index->kind = IndexKind::weighted;
        index->metric = UHA_L1;
        index->rows = row_count;
        index->dimension = dimension;
        index->scan_dim = dimension;
        index->padded_dim = uha::round_up(dimension, kColumnAlign);
        upload_padded(index->scan_rows, rows, row_count, dimension,
                      index->padded_dim);
        std::vector<float> w32(index->padded_dim, 0.0f);
        std::vector<double> w64(dimension);
        for (uint64_t i = 0; i < dimension; ++i) {
            w32[i] = weights[i];
            w64[i] = static_cast<double>(weights[i]);
        }
        upload(index->weights32, w32.data(), w32.size());
        upload(index->weights64, w64.data(), w64.size());
        upload_weights_ff(*index, w64);
        const uint64_t f = sizeof(float);
        index->usage.index_payload_bytes =
            row_count * dimension * f + dimension * f;
        index->usage.unique_query_coordinates = dimension;
        index->usage.sampled_multiplicity = dimension;
        *out = index.release();
    });
}

namespace {

void create_sampled_index(int device, uha_metric metric, const RowSource& src,
                          uint64_t row_count, uint64_t dimension,
                          const uint64_t* columns, const uint64_t* multiplicities,
                          const double* inverse_probabilities, uint64_t sample_size,
                          uha_index** out)
{
    const float* rows = src.host;
    require(out != nullptr, UHA_INVALID_ARGUMENT,
            "output pointer must not be null");
    require(metric == UHA_L2 || metric == UHA_L1, UHA_INVALID_ARGUMENT,
            "unknown metric");
    if (src.device == nullptr) {
        validate_rows(rows, row_count, dimension);
    } else {
        validate_device_matrix(src.device);
    }
    require(sample_size == 0 ||
                (columns != nullptr && multiplicities != nullptr &&
                 inverse_probabilities != nullptr),
            UHA_INVALID_ARGUMENT, "coordinate sample must not be null");
    require(sample_size <= kMaxExtent, UHA_LENGTH_ERROR,
            "coordinate sample exceeds the device grid limits");
    uint64_t multiplicity_sum = 0;
    std::vector<uint32_t> cols(sample_size);
    std::vector<float> scales(sample_size);
    std::vector<float> w32(uha::round_up(sample_size, kColumnAlign), 0.0f);
    std::vector<double> w64(sample_size);
    for (uint64_t i = 0; i < sample_size; ++i) {
        if (columns[i] >= dimension) {
            fail(UHA_OUT_OF_RANGE, "sampled column index out of range");
        }
        if (multiplicities[i] == 0 ||
            !std::isfinite(inverse_probabilities[i]) ||
            inverse_probabilities[i] <= 0.0) {
            fail(UHA_INVALID_ARGUMENT,
                 "sampled columns require positive finite weights");
        }
        if (multiplicity_sum > UINT64_MAX - multiplicities[i]) {
            fail(UHA_LENGTH_ERROR, "sampled multiplicity overflows");
        }
        multiplicity_sum += multiplicities[i];
        // weight = double(multiplicity) * (1/p), as in
        // l2_coordinate_embedding.cpp:56-57 and l1_coordinate_embedding.cpp:53-54
        const double weight = static_cast<double>(multiplicities[i]) *
                              inverse_probabilities[i];
        if (metric == UHA_L2) {
            const float scale = static_cast<float>(std::sqrt(weight));
            if (!std::isfinite(weight) || weight <= 0.0 ||
                !std::isfinite(scale) || scale <= 0.0f) {
                fail(UHA_INVALID_ARGUMENT,
                     "sampled coordinate weight is not representable in "
                     "float32");
            }
            scales[i] = scale;
        } else {
            const float fw = static_cast<float>(weight);
            if (!std::isfinite(weight) || weight <= 0.0 ||
                !std::isfinite(fw) || fw <= 0.0f) {
                fail(UHA_INVALID_ARGUMENT,
                     "sampled coordinate weight is not representable in "
                     "float32");
            }
            w32[i] = fw;
            w64[i] = weight;
        }
        cols[i] = static_cast<uint32_t>(columns[i]);
    }
    // Validate the sampled representative values (only sampled columns
    // are part of the index) and, for L2, their scaled binary32 values;
    // a device-resident matrix is validated by its gather below.
    for (uint64_t r = 0; src.device == nullptr && r < row_count; ++r) {
        const float* row = rows + r * dimension;
        for (uint64_t i = 0; i < sample_size; ++i) {
            const float v = row[cols[i]];
            if (!std::isfinite(v)) {
                fail(UHA_INVALID_ARGUMENT,
                     "sampled representatives must be finite");
            }
            if (metric == UHA_L2 && !std::isfinite(v * scales[i])) {
                fail(UHA_INVALID_ARGUMENT,
                     "transformed representatives must be finite");
            }
        }
    }

    auto index = std::make_unique<uha_index>();
    select_device(*index, device);
    DeviceGuard guard(device);
    index->kind = IndexKind::sampled;
    index->metric = metric;
    index->rows = row_count;
    index->dimension = dimension;
    index->scan_dim = sample_size;
    index->sample_size = sample_size;
    index->sampled_multiplicity = multiplicity_sum;
    index->padded_dim = uha::round_up(sample_size, kColumnAlign);
    upload(index->columns, cols.data(), cols.size());
    if (metric == UHA_L2) {
        upload(index->scales, scales.data(), scales.size());
    } else {
        upload(index->weights32, w32.data(), w32.size());
        upload(index->weights64, w64.data(), w64.size());
        upload_weights_ff(*index, w64);
    }
    // Gather (and scale) the sampled columns of the rows on the device.
    if (src.device != nullptr) {
        require_on_device(src.device, device);
        index->scan_rows.allocate(row_count * index->padded_dim);
        const auto bad = gather_device_source(
            src.device, index->columns.get(),
            metric == UHA_L2 ? index->scales.get() : nullptr, sample_size,
            index->scan_rows.get(), index->padded_dim);
        if (bad.first != ~0ull || bad.second != ~0ull) {
            fail(UHA_INVALID_ARGUMENT, bad.first <= bad.second
                                           ? "sampled representatives must be finite"
                                           : "transformed representatives must be finite");
        }
    } else if (index->padded_dim != 0) {
        DeviceBuffer<float> source(checked_mul(row_count, dimension,
                                               "representative matrix"));
        check_cuda(cudaMemcpy(source.get(), rows, source.bytes(),
                              cudaMemcpyHostToDevice),
                   "cannot copy representatives to the CUDA device");
        index->scan_rows.allocate(row_count * index->padded_dim);
        uha::launch_gather_rows(source.get(), row_count, dimension,
                                index->columns.get(),
                                metric == UHA_L2 ? index->scales.get()
                                                 : nullptr,
                                sample_size, index->scan_rows.get(),
                                index->padded_dim, nullptr);
        check_cuda(cudaDeviceSynchronize(), "row gather kernel failed");
    }
    const uint64_t f = sizeof(float);
    const uint64_t k = sample_size;
    if (metric == UHA_L2) {
        compute_row_norms(*index);
        index->usage.index_payload_bytes = row_count * k * f +
                                           row_count * f +
                                           k * sizeof(std::size_t) + k * f;
    } else {
        index->usage.index_payload_bytes =
            row_count * k * f + k * f + k * sizeof(std::size_t);
    }
    index->usage.query_workspace_payload_bytes = 0;
    index->usage.unique_query_coordinates = k;
    index->usage.sampled_multiplicity = multiplicity_sum;
    *out = index.release();
}

}  // namespace

extern "C" uha_status uha_sampled_index_create(
    int device, uha_metric metric, const float* rows, uint64_t row_count,
    uint64_t dimension, const uint64_t* columns, const uint64_t* multiplicities,
    const double* inverse_probabilities, uint64_t sample_size, uha_index** out)
{
    return guarded([&] {
        create_sampled_index(device, metric, RowSource{rows, nullptr}, row_count, dimension,
                             columns, multiplicities, inverse_probabilities, sample_size,
                             out);
    });
}

extern "C" uha_status uha_sampled_index_create_device(
    int device, uha_metric metric, const uha_device_matrix* rows, const uint64_t* columns,
    const uint64_t* multiplicities, const double* inverse_probabilities,
    uint64_t sample_size, uha_index** out)
{
    return guarded([&] {
        require(rows != nullptr, UHA_INVALID_ARGUMENT, "device matrix must not be null");
        create_sampled_index(device, metric, RowSource{nullptr, rows}, rows->rows,
                             rows->columns, columns, multiplicities, inverse_probabilities,
                             sample_size, out);
    });
}


namespace {

// Per-unit coefficient of the binary32 query projection's certified error:
// |y32_j - y64_j| <= coefficient * sum_i |x_i P32_ji| (binary32 two-level sum
// over k terms, binary32 rounding of the coefficients, the CPU's own binary64
// rounding).
double projection_error_per_abs(uint64_t k)
{
    const double u32 = std::ldexp(1.0, -24);
    const double u64 = std::ldexp(1.0, -53);
    const double n = 32.0 + static_cast<double>((k + 31) / 32) + 3.0;
    const double g32 = n * u32 / (1.0 - n * u32);
    const double g32b = (n + 1) * u32 / (1.0 - (n + 1) * u32);
    const double n64 = static_cast<double>(k) + 3.0;
    const double g64 = n64 * u64 / (1.0 - n64 * u64);
    return 1.01 * (g32 + u32 * (1 + 2 * u32) + g64 * (1 + u32)) * (1 + g32b) /
           (1 - g32b);
}

void create_hierarchical_index(int device, uha_metric metric, const RowSource& src,
                               uint64_t row_count, uint64_t dimension,
                               const uint64_t* columns, const uint64_t* multiplicities,
                               const double* inverse_probabilities, uint64_t sample_size,
                               const double* projection, uint64_t projection_dimension,
                               uha_index** out)
{
    const float* rows = src.host;
    require(out != nullptr, UHA_INVALID_ARGUMENT,
            "output pointer must not be null");
    require(metric == UHA_L2 || metric == UHA_L1, UHA_INVALID_ARGUMENT,
            "unknown metric");
    if (src.device == nullptr) {
        validate_rows(rows, row_count, dimension);
    } else {
        validate_device_matrix(src.device);
    }
    const uint64_t k = sample_size;
    const uint64_t p = projection_dimension;
    require(p != 0, UHA_INVALID_ARGUMENT,
            "projection_dimension has to be a positive integer");
    if (k == 0 && row_count > 1) {
        fail(UHA_RUNTIME_ERROR, "importance sampling selected no coordinates");
    }
    require(k == 0 || (columns != nullptr && multiplicities != nullptr &&
                       inverse_probabilities != nullptr &&
                       projection != nullptr),
            UHA_INVALID_ARGUMENT, "coordinate sample must not be null");
    require(k <= kMaxExtent, UHA_LENGTH_ERROR,
            "coordinate sample exceeds the device grid limits");
    require(p <= (metric == UHA_L2 ? 16384u : 1024u), UHA_LENGTH_ERROR,
            "projection dimension exceeds the supported maximum "
            "(16384 for L2, 1024 for L1)");
    checked_mul(p, k, "projection matrix");
    uint64_t multiplicity_sum = 0;
    std::vector<uint32_t> cols(k);
    for (uint64_t i = 0; i < k; ++i) {
        if (columns[i] >= dimension) {
            fail(UHA_OUT_OF_RANGE, "sampled column index out of range");
        }
        if (multiplicities[i] == 0 ||
            !std::isfinite(inverse_probabilities[i]) ||
            inverse_probabilities[i] <= 0.0) {
            fail(UHA_INVALID_ARGUMENT,
                 "sampled columns require positive finite weights");
        }
        if (multiplicity_sum > UINT64_MAX - multiplicities[i]) {
            fail(UHA_LENGTH_ERROR, "sampled multiplicity overflows");
        }
        multiplicity_sum += multiplicities[i];
        cols[i] = static_cast<uint32_t>(columns[i]);
    }
    const uint64_t kp = uha::round_up(k, kColumnAlign);
    const uint64_t pp = uha::round_up(p, kColumnAlign);
    std::vector<float> proj32(p * kp, 0.0f);
    for (uint64_t j = 0; j < p; ++j) {
        for (uint64_t i = 0; i < k; ++i) {
            const double c = projection[j * k + i];
            const float f = static_cast<float>(c);
            if (!std::isfinite(c)) {
                fail(UHA_OVERFLOW_ERROR, "projection coefficient is not finite");
            }
            if (!std::isfinite(f)) {
                fail(UHA_OVERFLOW_ERROR,
                     "binary32 projection coefficient is not finite");
            }
            proj32[j * kp + i] = f;
        }
    }

    auto index = std::make_unique<uha_index>();
    select_device(*index, device);
    DeviceGuard guard(device);
    index->kind = IndexKind::hierarchical;
    index->metric = metric;
    index->rows = row_count;
    index->dimension = dimension;
    index->sample_size = k;
    index->padded_sample = kp;
    index->sampled_multiplicity = multiplicity_sum;
    index->projection_dimension = p;
    index->scan_dim = p;
    index->padded_dim = pp;
    upload(index->columns, cols.data(), cols.size());
    upload(index->projection64, projection, p * k);
    upload(index->projection32, proj32.data(), proj32.size());

    DeviceBuffer<int> bad(1);
    check_cuda(cudaMemset(bad.get(), 0, sizeof(int)), "cannot clear flag");
    DeviceBuffer<float> sampled(std::max<uint64_t>(1, row_count * kp));
    check_cuda(cudaMemset(sampled.get(), 0, sampled.bytes()),
               "cannot clear sampled rows");
    if (k != 0 && src.device != nullptr) {
        // the reference does not validate the sampled values of a
        // hierarchy; a non-finite one fails as a non-finite projection
        require_on_device(src.device, device);
        gather_device_source(src.device, index->columns.get(), nullptr, k,
                             sampled.get(), kp);
    } else if (k != 0) {
        DeviceBuffer<float> source(checked_mul(row_count, dimension,
                                               "representative matrix"));
        check_cuda(cudaMemcpy(source.get(), rows, source.bytes(),
                              cudaMemcpyHostToDevice),
                   "cannot copy representatives to the CUDA device");
        uha::launch_gather_rows(source.get(), row_count, dimension,
                                index->columns.get(), nullptr, k,
                                sampled.get(), kp, nullptr);
    }
    index->rows64.allocate(row_count * p);
    uha::launch_project_rows64(sampled.get(), row_count, kp, k,
                               index->projection64.get(), p,
                               index->rows64.get(), bad.get(), nullptr);
    index->scan_rows.allocate(row_count * pp);
    index->row_err.allocate(row_count);
    uha::launch_narrow_rows(index->rows64.get(), row_count, p,
                            index->scan_rows.get(), pp, index->row_err.get(),
                            metric == UHA_L2, bad.get(), nullptr);
    int host_bad = 0;
    check_cuda(cudaMemcpy(&host_bad, bad.get(), sizeof(int),
                          cudaMemcpyDeviceToHost),
               "row projection failed");
    {
        std::vector<float> err(row_count);
        check_cuda(cudaMemcpy(err.data(), index->row_err.get(), row_count * sizeof(float),
                              cudaMemcpyDeviceToHost),
                   "row projection failed");
        index->row_err_max = 0.f;
        for (float e : err) {
            index->row_err_max = std::isnan(e) ? std::numeric_limits<float>::infinity()
                                               : std::max(index->row_err_max, e);
        }
    }
    if (host_bad & 1) {
        fail(UHA_OVERFLOW_ERROR, "projected representatives is not finite");
    }
    if (host_bad & 2) {
        fail(UHA_OVERFLOW_ERROR,
             "binary32 projected representative is not finite");
    }
    const uint64_t f = sizeof(float);
    const uint64_t column_bytes = 2 * sizeof(uint64_t) + sizeof(double);
    if (metric == UHA_L2) {
        // the precision strategies' binary64 query projection reads it
        std::vector<double> proj_t(p * k);
        for (uint64_t j = 0; j < p; ++j) {
            for (uint64_t i = 0; i < k; ++i) {
                proj_t[i * p + j] = projection[j * k + i];
            }
        }
        upload(index->projection64_t, proj_t.data(), proj_t.size());
        compute_row_norms(*index);
        index->usage.index_payload_bytes = row_count * p * f + row_count * f +
                                           k * column_bytes + p * k * f;
    } else {
        index->usage.index_payload_bytes =
            k * column_bytes + p * k * f + row_count * p * f;
        // the median scan's pruning count reads the rows transposed
        index->rows_pitch = uha::round_up(row_count, 32);
        index->scan_rows_t.allocate(checked_mul(pp, index->rows_pitch, "transposed rows"));
        uha::launch_transpose_rows(index->scan_rows.get(), row_count, pp,
                                   index->scan_rows_t.get(), index->rows_pitch, nullptr);
        check_cuda(cudaDeviceSynchronize(), "row transpose kernel failed");
    }
    index->usage.query_workspace_payload_bytes = 0;
    index->usage.unique_query_coordinates = k;
    index->usage.sampled_multiplicity = multiplicity_sum;
    *out = index.release();
}

}  // namespace

extern "C" uha_status uha_hierarchical_index_create(
    int device, uha_metric metric, const float* rows, uint64_t row_count,
    uint64_t dimension, const uint64_t* columns, const uint64_t* multiplicities,
    const double* inverse_probabilities, uint64_t sample_size,
    const double* projection, uint64_t projection_dimension, uha_index** out)
{
    return guarded([&] {
        create_hierarchical_index(device, metric, RowSource{rows, nullptr}, row_count,
                                  dimension, columns, multiplicities,
                                  inverse_probabilities, sample_size, projection,
                                  projection_dimension, out);
    });
}

extern "C" uha_status uha_hierarchical_index_create_device(
    int device, uha_metric metric, const uha_device_matrix* rows, const uint64_t* columns,
    const uint64_t* multiplicities, const double* inverse_probabilities,
    uint64_t sample_size, const double* projection, uint64_t projection_dimension,
    uha_index** out)
{
    return guarded([&] {
        require(rows != nullptr, UHA_INVALID_ARGUMENT, "device matrix must not be null");
        create_hierarchical_index(device, metric, RowSource{nullptr, rows}, rows->rows,
                                  rows->columns, columns, multiplicities,
                                  inverse_probabilities, sample_size, projection,
                                  projection_dimension, out);
    });
}

extern "C" void uha_index_destroy(uha_index* index)
{
    if (index != nullptr) {
        int previous = 0;
        const bool ok = cudaGetDevice(&previous) == cudaSuccess;
        cudaSetDevice(index->device);
        delete index;
        if (ok) {
            cudaSetDevice(previous);
        }
        uha::clear_stale_cuda_error();
    }
}

extern "C" uha_status uha_index_space_usage(const uha_index* index,
                                            uha_space_usage* out)
{
    return guarded([&] {
        require(index != nullptr && out != nullptr, UHA_INVALID_ARGUMENT,
                "index and output must not be null");
        *out = index->usage;
    });
}

extern "C" uha_status uha_index_device(const uha_index* index, int* device,
                                       char* name, uint64_t name_capacity)
{
    return guarded([&] {
        require(index != nullptr, UHA_INVALID_ARGUMENT,
                "index must not be null");
        if (device != nullptr) {
            *device = index->device;
        }
        if (name != nullptr && name_capacity > 0) {
            const uint64_t n =
                std::min<uint64_t>(index->device_name.size(), name_capacity - 1);
            std::memcpy(name, index->device_name.data(), n);
            name[n] = '\0';
        }
    });
}

// -------------------------------------------------------------- workspaces

extern "C" uha_status uha_workspace_create(const uha_index* index,
                                           uint64_t maximum_batch_size,
                                           uha_workspace** out)
{
    return guarded([&] {
        require(index != nullptr && out != nullptr, UHA_INVALID_ARGUMENT,
                "index and output must not be null");
        require(maximum_batch_size != 0, UHA_INVALID_ARGUMENT,
                "workspace batch size must be positive");
        require(maximum_batch_size <= kMaxExtent, UHA_LENGTH_ERROR,
                "workspace batch size exceeds the device grid limits");
        checked_mul(maximum_batch_size, index->dimension, "query workspace");
        checked_mul(maximum_batch_size, index->rows, "distance workspace");
        DeviceGuard guard(index->device);
        auto ws = std::make_unique<uha_workspace>();
        ws->owner = index;
        ws->device = index->device;
        ws->max_batch = maximum_batch_size;
        ws->payload_bytes = workspace_payload(*index, maximum_batch_size);
        check_cuda(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking),
                   "cannot create CUDA stream");
        const uint64_t b = maximum_batch_size;
        ws->raw_queries.allocate(b * index->dimension);
        if (index->kind == IndexKind::hierarchical) {
            ws->prepared.allocate(b * index->padded_sample);
            ws->projected.allocate(b * index->padded_dim);
            ws->query_err.allocate(b);
            if (index->metric == UHA_L1) {
                ws->coord_err.allocate(b * index->padded_dim);
                ws->pair_err.allocate(checked_mul(b, index->rows, "median errors"));
            }
        } else {
            ws->prepared.allocate(b * index->padded_dim);
        }
        ws->query_norms.allocate(b);
        ws->call_results.allocate(b);
        ws->call_exact.allocate(b);
        ws->counters.allocate(2);
        ws->finalize_scratch.allocate(
            uha::finalize_scratch_bytes(b, index->rows));
        check_cuda(cudaMemset(ws->finalize_scratch.get(), 0,
                              ws->finalize_scratch.bytes()),
                   "cannot clear finalize scratch");
        ws->host_results.allocate(b);
        ws->host_exact.allocate(b);
        ws->host_counters.allocate(2);
        for (cudaEvent_t& e : ws->events) {
            check_cuda(cudaEventCreate(&e), "cannot create CUDA event");
        }
        *out = ws.release();
    });
}

extern "C" void uha_workspace_destroy(uha_workspace* workspace)
{
    if (workspace != nullptr) {
        int previous = 0;
        const bool ok = cudaGetDevice(&previous) == cudaSuccess;
        cudaSetDevice(workspace->device);
        delete workspace;
        if (ok) {
            cudaSetDevice(previous);
        }
        uha::clear_stale_cuda_error();
    }
}

extern "C" uha_status uha_workspace_info(const uha_workspace* workspace,
                                         uint64_t* maximum_batch_size,
                                         uint64_t* payload_bytes)
{
    return guarded([&] {
        require(workspace != nullptr, UHA_INVALID_ARGUMENT,
                "workspace must not be null");
        if (maximum_batch_size != nullptr) {
            *maximum_batch_size = workspace->max_batch;
        }
        if (payload_bytes != nullptr) {
            *payload_bytes = workspace->payload_bytes;
        }
    });
}

extern "C" void* uha_workspace_stream(const uha_workspace* workspace)
{
    return workspace == nullptr ? nullptr
                                : static_cast<void*>(workspace->stream);
}

extern "C" uha_status uha_workspace_set_timing(uha_workspace* workspace,
                                               int enabled)
{
    return guarded([&] {
        require(workspace != nullptr, UHA_INVALID_ARGUMENT,
                "workspace must not be null");
        require(enabled >= 0, UHA_INVALID_ARGUMENT, "timing must be 0 or a positive stride");
        workspace->timing = enabled != 0;
        workspace->timing_stride = enabled > 0 ? static_cast<uint32_t>(enabled) : 1u;
    });
}

extern "C" uha_status uha_workspace_last_stats(const uha_workspace* workspace,
                                               uha_query_stats* out)
{
    return guarded([&] {
        require(workspace != nullptr && out != nullptr, UHA_INVALID_ARGUMENT,
                "workspace and output must not be null");
        *out = workspace->last;
    });
}

// ------------------------------------------------------------------ query

namespace uha_engine {

// Certified queries on exact and flat indexes small enough for one CTA per
// query run as one fused launch.
bool small_path_applies(const uha_index* index, uha_strategy strategy)
{
    return strategy == UHA_DIRECT && index->kind != IndexKind::hierarchical &&
           uha::small_query_fits(index->rows, index->padded_dim);
}

// Certified queries of at most uha::kFlatBatch on flat and small exact
// indexes run as one fused launch with many CTAs per query (also the indexes
// one CTA could scan: a CTA per query walks its rows one after another, which
// at small batches leaves the GPU waiting on memory).
bool flat_path_applies(const uha_index* index, uha_strategy strategy, uint64_t batch)
{
    return strategy == UHA_DIRECT && index->kind != IndexKind::hierarchical &&
           uha::flat_query_fits(index->rows, index->padded_dim, batch);
}

bool precision_strategy(uha_strategy s)
{
    return s == UHA_GEMM_BF16_RERANK || s == UHA_GEMM_FP8_RERANK ||
           s == UHA_GEMM_BF16_RERANK_FP32 || s == UHA_GEMM_FP8_RERANK_FP32;
}

// The precision strategies that re-score in binary32 (no FP64 instructions).
bool fp32_rescore_strategy(uha_strategy s)
{
    return s == UHA_GEMM_BF16_RERANK_FP32 || s == UHA_GEMM_FP8_RERANK_FP32;
}

// Replay inputs of the emulated (FP64-free) replay of exact and flat ops.
void set_emulated(uha::ReplayInputs& in, const uha_index* index)
{
    in.emulated = true;
    in.weights_ff = index->weights_ff.get();
    uha::emulated_replay_bound(index->scan_dim, &in.ff_rel, &in.ff_abs);
}

uha::LowpType lowp_type(uha_strategy s)
{
    return s == UHA_GEMM_FP8_RERANK || s == UHA_GEMM_FP8_RERANK_FP32
               ? uha::LowpType::fp8_e4m3
               : uha::LowpType::bf16;
}

// The index's low-precision rows of `type`, rounded from the scanned binary32
// rows on first use (on `stream`, synchronised before it is published).
const uha::LowpRows& lowp_rows(const uha_index* index, uha::LowpType type,
                               cudaStream_t stream)
{
    std::lock_guard<std::mutex> lock(index->lowp_mutex);
    uha::LowpRows& lp = index->lowp[static_cast<int>(type)];
    if (lp.ready) {
        return lp;
    }
    lp.pitch = uha::lowp_pitch(type, index->scan_dim);
    const uint64_t vectors = uha::lowp_padded_count(index->rows);
    lp.data.allocate(checked_mul(checked_mul(vectors, lp.pitch, "low-precision rows"),
                                 uha::lowp_element_bytes(type), "low-precision rows"));
    lp.scales.allocate(vectors);
    lp.norms.allocate(index->rows);
    check_cuda(cudaMemsetAsync(lp.data.get(), 0, lp.data.bytes(), stream),
               "cannot clear low-precision rows");
    uha::launch_lowp_convert(type, index->scan_rows.get(), index->rows, index->padded_dim,
                             index->scan_dim, lp.data.get(), lp.pitch, lp.scales.get(),
                             lp.norms.get(), stream);
    check_cuda(cudaStreamSynchronize(stream), "cannot build low-precision rows");
    lp.ready = true;
    return lp;
}

// Workspace buffers of the precision strategies for batches up to max_batch.
void ensure_lowp_workspace(uha_workspace* ws, const uha_index* index,
                           cudaStream_t stream)
{
    const uint64_t bytes = checked_mul(
        checked_mul(uha::lowp_padded_count(ws->max_batch),
                    uha::lowp_pitch(uha::LowpType::bf16, index->scan_dim), "query buffer"),
        2, "query buffer");
    if (ws->queries_lp.size() < bytes) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->queries_lp.allocate(bytes);
        // vectors past a batch are read by the score kernel (and not stored)
        check_cuda(cudaMemsetAsync(ws->queries_lp.get(), 0, bytes, stream),
                   "cannot clear the query buffer");
        ws->query_scales.allocate(uha::lowp_padded_count(ws->max_batch));
        ws->query_amax.allocate(uha::lowp_padded_count(ws->max_batch));
    }
    const uint64_t cand = checked_mul(ws->max_batch, uha::max_rerank_candidates(),
                                      "candidates");
    if (ws->candidates.size() < cand) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->candidates.allocate(cand);
        ws->cand_dist.allocate(cand);
        ws->rescore_done.allocate(ws->max_batch);
        check_cuda(cudaMemsetAsync(ws->rescore_done.get(), 0, ws->rescore_done.bytes(),
                                   stream),
                   "cannot clear re-score counters");
    }
}

// The p x k projection of an L2 hierarchy rounded like index rows (built on
// first use).
const uha::LowpRows& lowp_projection(const uha_index* index, uha::LowpType type,
                                     cudaStream_t stream)
{
    std::lock_guard<std::mutex> lock(index->lowp_mutex);
    uha::LowpRows& lp = index->lowp_projection[static_cast<int>(type)];
    if (lp.ready) {
        return lp;
    }
    const uint64_t p = index->projection_dimension;
    lp.pitch = uha::lowp_pitch(type, index->sample_size);
    const uint64_t vectors = uha::lowp_padded_count(p);
    lp.data.allocate(checked_mul(checked_mul(vectors, lp.pitch, "low-precision projection"),
                                 uha::lowp_element_bytes(type), "low-precision projection"));
    lp.scales.allocate(vectors);
    lp.norms.allocate(p);
    check_cuda(cudaMemsetAsync(lp.data.get(), 0, lp.data.bytes(), stream),
               "cannot clear low-precision projection");
    uha::launch_lowp_convert(type, index->projection32.get(), p, index->padded_sample,
                             index->sample_size, lp.data.get(), lp.pitch, lp.scales.get(),
                             lp.norms.get(), stream);
    check_cuda(cudaStreamSynchronize(stream), "cannot build low-precision projection");
    lp.ready = true;
    return lp;
}

// Precision form of the L2 hierarchy, before the scores: the gathered
// queries are rounded and projected on the tensor cores (the projection as
// a GEMM of the rounded p x k matrix with the batch) into ws->projected, the
// approximate queries of the score GEMM; the reference's binary64 projection
// goes to ws->projected64 for the re-score.
void enqueue_hierarchical_projection(const uha_index* index, uha_workspace* ws,
                                     uha_strategy strategy, uint64_t n, int* error_flag,
                                     cudaStream_t stream)
{
    const uha::LowpType type = lowp_type(strategy);
    const uha::LowpRows& lp = lowp_projection(index, type, stream);
    const uint64_t p = index->projection_dimension;
    const uint64_t bytes = checked_mul(
        checked_mul(uha::lowp_padded_count(ws->max_batch),
                    uha::lowp_pitch(uha::LowpType::bf16, index->sample_size),
                    "query buffer"),
        2, "query buffer");
    if (ws->gathered_lp.size() < bytes) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->gathered_lp.allocate(bytes);
        // vectors past a batch are read by the score kernel (and not stored)
        check_cuda(cudaMemsetAsync(ws->gathered_lp.get(), 0, bytes, stream),
                   "cannot clear the query buffer");
        ws->gathered_scales.allocate(uha::lowp_padded_count(ws->max_batch));
        ws->gathered_amax.allocate(uha::lowp_padded_count(ws->max_batch));
        ws->projected64.allocate(checked_mul(ws->max_batch, p, "projected queries"));
    }
    uha::launch_lowp_queries(type, ws->prepared.get(), n, index->padded_sample,
                             ws->gathered_lp.get(), lp.pitch, ws->gathered_scales.get(),
                             ws->gathered_amax.get(), stream);
    const uha::LowpPlan plan = uha::plan_lowp(type, p, lp.pitch, n, index->sm_count);
    const uint64_t partial_count =
        checked_mul(checked_mul(plan.splits, n, "partials"), p, "partials");
    if (ws->partials.size() < partial_count) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->partials.allocate(partial_count);
    }
    uha::launch_lowp_scores(plan, type, lp.data.get(), lp.scales.get(), p,
                            ws->gathered_lp.get(), ws->gathered_scales.get(), n, lp.pitch,
                            ws->partials.get(), error_flag, stream);
    uha::launch_sum_slabs(ws->partials.get(), plan.splits, n, p, ws->projected.get(),
                          index->padded_dim, stream);
    uha::launch_project_queries64(ws->prepared.get(), n, index->padded_sample,
                                  index->sample_size, index->projection64_t.get(), p,
                                  ws->projected64.get(), error_flag, stream);
}

// Rounds the prepared queries and runs the tensor-core scores; returns the
// plan (the partial-score slabs are in ws->partials).
uha::LowpPlan enqueue_lowp_scores(const uha_index* index, uha_workspace* ws,
                                  uha_strategy strategy, uint64_t n, bool time_scan,
                                  cudaEvent_t scan_start, cudaEvent_t scan_stop,
                                  const float* prepared = nullptr, bool scores = true)
{
    cudaStream_t stream = ws->stream;
    const uha::LowpType type = lowp_type(strategy);
    const uha::LowpRows& lp = lowp_rows(index, type, stream);
    ensure_lowp_workspace(ws, index, stream);
    uha::launch_lowp_queries(type, prepared != nullptr ? prepared : ws->prepared.get(), n,
                             index->padded_dim,
                             ws->queries_lp.get(), lp.pitch, ws->query_scales.get(),
                             ws->query_amax.get(), stream);
    const TunedPlan* tuned = ws->find_tuned(n, static_cast<int>(strategy));
    const uha::LowpPlan plan = tuned != nullptr && tuned->lowp
                                   ? tuned->lowp_plan
                                   : uha::plan_lowp(type, index->rows, lp.pitch, n,
                                                    index->sm_count);
    if (!scores) {
        return plan;  // the caller sizes the partials for its selection
    }
    const uint64_t partial_count =
        checked_mul(checked_mul(plan.splits, n, "partials"), index->rows, "partials");
    if (ws->partials.size() < partial_count) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->partials.allocate(partial_count);
    }
    if (time_scan) {
        check_cuda(cudaEventRecord(scan_start, stream), "event");
    }
    uha::launch_lowp_scores(plan, type, lp.data.get(), lp.scales.get(), index->rows,
                            ws->queries_lp.get(), ws->query_scales.get(), n, lp.pitch,
                            ws->partials.get(),
                            reinterpret_cast<int*>(ws->counters.get() + 1), stream);
    if (time_scan) {
        check_cuda(cudaEventRecord(scan_stop, stream), "event");
    }
    return plan;
}

// Whether a batch of n takes the fused selection: plans of one K split on
// indexes of at least kFilterMinRows rows, up to 64 candidates, and not
// turned off for this call. Every kernel of the selection runs on the
// workspace stream and writes the batch's own candidate slot before a
// pipelined call hands the batch to its re-score stream, so the next batch
// reuses the selection's buffers in stream order.
bool filter_applies(const BatchContext& c, const uha::LowpPlan& plan, uint32_t k)
{
    return c.filter_candidates && !c.ws->filter_disabled && plan.splits == 1 &&
           c.index->rows >= uha::kFilterMinRows && k >= 1 && k <= 64;
}

// The k candidates per query of a precision strategy into `candidates`; the
// rounded queries are in ws->queries_lp. The slab path stores every partial
// score and selects from the slab. The fused path scores the first sample
// rows the same way (bit-identical estimates: the same plan and tiles), takes
// each query's k-th smallest estimate as its threshold, and scores all rows
// with the filter epilogue, which keeps only the keys at or below the
// threshold; the selection over those keys gives the slab path's candidates.
// Returns the kernel launches.
uint64_t enqueue_lowp_candidates(const BatchContext& c, uint64_t n, const uha::LowpPlan& plan,
                                 uint32_t k, uint32_t* candidates, bool time_scan,
                                 cudaEvent_t scan_start, cudaEvent_t scan_stop)
{
    const uha_index* index = c.index;
    uha_workspace* ws = c.ws;
    cudaStream_t stream = ws->stream;
    const uha::LowpType type = lowp_type(c.strategy);
    const uha::LowpRows& lp = lowp_rows(index, type, stream);
    const float* norms = index->lowp[static_cast<int>(type)].norms.get();
    int* error_flag = reinterpret_cast<int*>(ws->counters.get() + 1);
    const uint32_t b = static_cast<uint32_t>(n);
    const uint32_t rows = static_cast<uint32_t>(index->rows);
    const bool fused = filter_applies(c, plan, k);
    // the slab path's partial scores, or the fused path's sample slab
    const uint64_t partial_count =
        fused ? checked_mul(n, uha::filter_sample_rows(index->rows), "partials")
              : checked_mul(checked_mul(plan.splits, n, "partials"), index->rows, "partials");
    if (ws->partials.size() < partial_count) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->partials.allocate(partial_count);
    }
    if (!fused) {
        if (time_scan) {
            check_cuda(cudaEventRecord(scan_start, stream), "event");
        }
        uha::launch_lowp_scores(plan, type, lp.data.get(), lp.scales.get(), index->rows,
                                ws->queries_lp.get(), ws->query_scales.get(), n, lp.pitch,
                                ws->partials.get(), error_flag, stream);
        if (time_scan) {
            check_cuda(cudaEventRecord(scan_stop, stream), "event");
        }
        uha::launch_lowp_topk(ws->partials.get(), plan.splits, b, rows, norms, k, candidates,
                              stream);
        return 2;
    }
    const uint64_t sample = uha::filter_sample_rows(index->rows);
    const uint32_t cap = uha::filter_capacity(index->rows, k);
    if (ws->filter_keys.size() < ws->max_batch * cap) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->filter_keys.allocate(checked_mul(ws->max_batch, cap, "candidate lists"));
        ws->filter_count.allocate(ws->max_batch);
        ws->filter_tau.allocate(ws->max_batch);
        ws->filter_sample.allocate(ws->max_batch * 64);
    }
    if (ws->filter_norms.size() < sample) {
        ws->filter_norms.allocate(sample);
    }
    if (time_scan) {
        check_cuda(cudaEventRecord(scan_start, stream), "event");
    }
    // the sample's one slab: whole tiles spread over the index
    uha::launch_lowp_scores(plan, type, lp.data.get(), lp.scales.get(), index->rows,
                            ws->queries_lp.get(), ws->query_scales.get(), n, lp.pitch,
                            ws->partials.get(), error_flag, stream, nullptr, sample);
    // the sample rows' norms in sample order, for its selection and threshold
    uha::launch_gather_sample_norms(norms, index->rows, static_cast<uint32_t>(sample),
                                    ws->filter_norms.get(), stream);
    uha::launch_lowp_topk(ws->partials.get(), 1, b, static_cast<uint32_t>(sample),
                          ws->filter_norms.get(), k, ws->filter_sample.get(), stream);
    uha::launch_lowp_threshold(ws->partials.get(), b, static_cast<uint32_t>(sample),
                               ws->filter_norms.get(), k, ws->filter_sample.get(),
                               ws->filter_tau.get(), stream);
    check_cuda(cudaMemsetAsync(ws->filter_count.get(), 0, n * sizeof(uint32_t), stream),
               "cannot clear candidate counts");
    const uha::FilterArgs filter{norms, ws->filter_tau.get(), ws->filter_keys.get(),
                                 ws->filter_count.get(), cap};
    uha::launch_lowp_scores(plan, type, lp.data.get(), lp.scales.get(), index->rows,
                            ws->queries_lp.get(), ws->query_scales.get(), n, lp.pitch,
                            nullptr, error_flag, stream, &filter);
    uha::launch_lowp_select(ws->filter_keys.get(), ws->filter_count.get(), cap, b, k,
                            candidates, error_flag, stream);
    if (time_scan) {
        check_cuda(cudaEventRecord(scan_stop, stream), "event");
    }
    return 6;
}

// One query batch's kernels on the workspace stream: gather / copy with
// validation, (projection), scan, certified argmin with in-kernel replay (or
// the norm identity), (the replayed distance of each selected row of a
// hierarchy). `results` / `exact` receive this batch's answers; flags and the
// replay count accumulate in ws.counters.

// The certification bound and replay inputs of a scan of `plan` (operation
// `op`) over `index`, the workspace holding the query-side buffers; shared by
// the standalone pipeline and the persistent batch.
void certification_inputs(const uha_index* index, const uha_workspace* ws,
                          const uha::ScanPlan& plan, uha::ScanOp op, const float* prepared,
                          uha::Bound* bound_out, uha::ReplayInputs* in_out)
{
    const bool hierarchical = index->kind == IndexKind::hierarchical;
    const bool median = hierarchical && index->metric == UHA_L1;
    const int term_roundings = op == uha::ScanOp::l1 ? 1 : 2;
    uha::Bound bound = make_bound(plan.depth, index->scan_dim, term_roundings);
    uha::ReplayInputs in{};
    in.rows = index->scan_rows.get();
    in.queries = prepared;
    in.dim = index->scan_dim;
    in.padded_dim = index->padded_dim;
    in.weights64 = index->weights64.get();
    if (hierarchical) {
        bound.row_err = index->row_err.get();
        bound.query_err = ws->query_err.get();
        bound.row_err_max = index->row_err_max;
        if (median) {
            bound.mode = uha::BoundMode::median;
            bound.rel = kMedianRel;
            bound.abs = kMedianAbs;
            bound.pair_err = ws->pair_err.get();
            bound.pair_rows = static_cast<uint32_t>(index->rows);
        } else {
            bound.mode = uha::BoundMode::projected_l2;
            const double n64 = static_cast<double>(index->scan_dim) + 3;
            const double g64 = n64 * std::ldexp(1.0, -53);
            bound.cpu_rel = std::nextafter(static_cast<float>(1.01 * g64), 1.0f);
        }
        in.op = median ? uha::ReplayOp::median_projected : uha::ReplayOp::l2_projected;
        in.dim = index->sample_size;
        in.padded_dim = index->padded_sample;
        in.rows64 = index->rows64.get();
        in.projection64 = index->projection64.get();
        in.proj_dim = index->projection_dimension;
    } else if (index->metric == UHA_L2) {
        in.op = uha::ReplayOp::l2_sequential;
    } else if (index->weights64.size() != 0) {
        in.op = uha::ReplayOp::l1_weighted_sequential;
    } else {
        in.op = uha::ReplayOp::l1_grouped4;
    }
    if (!hierarchical && ws->emulated_replay) {
        set_emulated(in, index);
    }
    *bound_out = bound;
    *in_out = in;
}

uha::MedianPlan median_plan(const uha_index* index, const uha_workspace* ws, uint64_t n)
{
    for (const TunedPlan& t : ws->tuned) {
        if (t.median && t.batch == n) {
            return t.median_plan;
        }
    }
    return uha::default_median_plan(index->rows, n);
}

bool persistent_pair(const uha_index* index, uha_workspace* ws, uint64_t n,
                     uha::PersistentPair* d)
{
    if (index->kind != IndexKind::hierarchical || index->rows < 2 || index->padded_dim == 0 ||
        index->projection_dimension > 256 || n == 0 || n > 0xffffffffull ||
        index->rows > 0xffffffffull) {
        return false;
    }
    const bool median = index->metric == UHA_L1;
    // the tuned plan when it is a tile scan (the tuner may pick the streaming
    // scan, which has no unit kind), else the default plan
    const TunedPlan* tuned = ws->find_tuned(n, static_cast<int>(UHA_DIRECT));
    uha::ScanPlan plan = uha::plan_scan(index->rows, index->padded_dim, n, index->sm_count);
    if (!median && tuned != nullptr && !tuned->lowp && !tuned->median &&
        tuned->scan.kernel == 1) {
        plan = tuned->scan;
    }
    if (median) {
        plan.chunks = 1;
        plan.depth = 0;
    } else if (plan.kernel != 1) {
        return false;  // the streaming scan of batches up to 8 is not a unit kind
    }
    *d = uha::PersistentPair{};
    const uint32_t rows = static_cast<uint32_t>(index->rows);
    const uint32_t b = static_cast<uint32_t>(n);
    d->l2 = median ? 0 : 1;
    d->batch = b;
    d->counters = ws->counters.get();
    d->counter_words = static_cast<uint32_t>(ws->counters.size());
    d->raw_queries = ws->raw_queries.get();
    d->dim = index->dimension;
    d->columns = index->columns.get();
    d->sample_size = index->sample_size;
    d->prepared = ws->prepared.get();
    d->padded_sample = index->padded_sample;
    d->projection32 = index->projection32.get();
    d->proj_dim = index->projection_dimension;
    d->projected = ws->projected.get();
    d->padded_p = index->padded_dim;
    d->query_err = ws->query_err.get();
    d->coord_err = ws->coord_err.get();
    d->err_per_abs = projection_error_per_abs(index->sample_size);
    uha::project_queries_grid(n, index->padded_dim, &d->proj_gx, &d->proj_gy);
    d->scan_rows = index->scan_rows.get();
    d->rows = rows;
    d->partials = ws->partials.get();
    if (!median) {
        d->k_per_split = plan.k_per_split;
        uha::tile_scan_grid(index->rows, n, plan.chunks, &d->tile_gx, &d->tile_gy,
                            &d->tile_gz);
    } else {
        if (ws->median_min.size() < n || ws->pair_err.size() < n * index->rows) {
            return false;
        }
        uha::MedianArgs& m = d->median;
        m.rows = index->scan_rows.get();
        m.rows_t = index->scan_rows_t.get();
        m.r_pitch = static_cast<uint32_t>(index->rows_pitch);
        m.row_count = rows;
        m.padded_p = static_cast<uint32_t>(index->padded_dim);
        m.p = static_cast<uint32_t>(index->projection_dimension);
        m.queries = ws->projected.get();
        m.batch = b;
        m.query_err = ws->query_err.get();
        m.coord_err = ws->coord_err.get();
        m.row_err_max = index->row_err_max;
        m.rel = kMedianRel;
        m.abs_err = kMedianAbs;
        m.min_bits = ws->median_min.get();
        m.partials = ws->partials.get();
        m.pair_err = ws->pair_err.get();
        const uha::MedianPlan mp = median_plan(index, ws, n);
        m.samples = mp.samples;
        m.count_queries = mp.count_queries;
        d->sample_blocks = uha::median_sample_blocks(mp.samples, b);
        uha::median_count_grid(rows, b, mp.count_queries, &d->count_gx, &d->count_gy);
        d->survivor_blocks = uha::median_survivor_blocks(rows, b);
    }
    d->view = uha::PartialView{ws->partials.get(), plan.chunks, b, rows};
    certification_inputs(index, ws, plan, median ? uha::ScanOp::l1 : uha::ScanOp::l2,
                         ws->prepared.get(), &d->bound, &d->replay);
    d->results = ws->call_results.get();
    d->exact_distances = ws->call_exact.get();
    uha::argmin_scratch(ws->finalize_scratch.get(), ws->max_batch, rows, &d->summaries,
                        &d->done);
    uha::argmin_grid(rows, b, &d->argmin_gx, &d->argmin_span);
    d->refine_blocks = uha::refine_group_blocks(b);
    // the grouped reported-distance pass must fit the kernel's shared memory
    return uha::refine_group_smem_bytes(d->replay) <= 96 * 1024 &&
           ws->partials.size() >= uint64_t(plan.chunks) * n * index->rows;
}

void ensure_flat_scratch(const uha_index* index, uha_workspace* ws)
{
    if (ws->flat_scratch.size() != 0) {
        return;
    }
    // zero once: the kernel leaves its completion counters at zero
    ws->flat_scratch.allocate(
        uha::flat_query_scratch_bytes(ws->max_batch, index->rows, 2 * uha::kFlatLanes));
    check_cuda(cudaMemsetAsync(ws->flat_scratch.get(), 0, ws->flat_scratch.bytes(),
                               ws->stream),
               "cannot clear flat query scratch");
}

uint64_t enqueue_batch(const BatchContext& c, const float* source, uint64_t n,
                       uha::Result* results, double* exact, bool time_scan,
                       cudaEvent_t scan_start, cudaEvent_t scan_stop)
{
    const uha_index* index = c.index;
    uha_workspace* ws = c.ws;
    cudaStream_t stream = ws->stream;
    int* error_flag = reinterpret_cast<int*>(ws->counters.get() + 1);
    uint32_t* replay_count = ws->counters.get();
    uint64_t launches = 0;

    const bool hierarchical = index->kind == IndexKind::hierarchical;
    const bool flat = flat_path_applies(index, c.strategy, n);
    if (small_path_applies(index, c.strategy) || flat) {
        uha::SmallQuery sq{};
        sq.queries = source;
        sq.dim = index->dimension;
        sq.columns = index->kind == IndexKind::sampled ? index->columns.get() : nullptr;
        sq.scales = index->kind == IndexKind::sampled && index->metric == UHA_L2
                        ? index->scales.get()
                        : nullptr;
        sq.sample_size = index->sample_size;
        sq.rows = index->scan_rows.get();
        sq.row_count = static_cast<uint32_t>(index->rows);
        sq.padded_dim = index->padded_dim;
        sq.weights32 = index->weights32.get();
        uha::ScanOp op = uha::ScanOp::l2;
        if (index->metric == UHA_L1) {
            op = index->weights32.size() != 0 ? uha::ScanOp::l1_weighted : uha::ScanOp::l1;
        }
        sq.op = static_cast<int>(op);
        const uha::FlatPlan flat_plan =
            flat ? uha::plan_flat_query(index->rows, index->padded_dim, n, index->sm_count)
                 : uha::FlatPlan{};
        const uha::Bound bound =
            make_bound(flat ? flat_plan.depth : uha::small_query_depth(index->padded_dim),
                       index->scan_dim, op == uha::ScanOp::l1 ? 1 : 2);
        uha::ReplayInputs in{};
        in.op = index->metric == UHA_L2 ? uha::ReplayOp::l2_sequential
                : index->weights64.size() != 0 ? uha::ReplayOp::l1_weighted_sequential
                                               : uha::ReplayOp::l1_grouped4;
        in.rows = index->scan_rows.get();
        in.dim = index->scan_dim;
        in.padded_dim = index->padded_dim;
        in.weights64 = index->weights64.get();
        if (ws->emulated_replay) {
            set_emulated(in, index);
        }
        if (flat) {
            ensure_flat_scratch(index, ws);
        }
        if (time_scan) {
            check_cuda(cudaEventRecord(scan_start, stream), "event");
        }
        if (flat) {
            const int lane = c.flat_lane;
            const cudaStream_t lane_stream = lane == 0 ? stream : ws->flat_streams[lane];
            uha::launch_flat_query(sq, flat_plan, static_cast<uint32_t>(n), bound, in,
                                   ws->flat_scratch.get(), ws->max_batch,
                                   2u * static_cast<uint32_t>(lane) + ws->flat_parity[lane],
                                   results, exact, replay_count, error_flag, lane_stream);
            ws->flat_parity[lane] ^= 1u;
        } else {
            uha::launch_small_query(sq, static_cast<uint32_t>(n), bound, in, results,
                                    exact, replay_count, error_flag, stream);
        }
        if (time_scan) {
            check_cuda(cudaEventRecord(scan_stop, stream), "event");
        }
        return 1;
    }
    float* prepared = c.prepared != nullptr ? c.prepared : ws->prepared.get();
    const float* scan_queries = prepared;
    if (hierarchical && precision_strategy(c.strategy)) {
        uha::launch_prepare_sampled(source, n, index->dimension, index->columns.get(),
                                    nullptr, index->sample_size, ws->prepared.get(),
                                    index->padded_sample, error_flag, stream);
        enqueue_hierarchical_projection(index, ws, c.strategy, n, error_flag, stream);
        scan_queries = ws->projected.get();
        launches += 6;
    } else if (hierarchical) {
        uha::launch_prepare_sampled(source, n, index->dimension, index->columns.get(),
                                    nullptr, index->sample_size, ws->prepared.get(),
                                    index->padded_sample, error_flag, stream);
        uha::launch_project_queries(
            ws->prepared.get(), n, index->padded_sample, index->sample_size,
            index->projection32.get(), index->projection_dimension,
            ws->projected.get(), index->padded_dim, ws->query_err.get(),
            index->metric == UHA_L1 ? ws->coord_err.get() : nullptr,
            projection_error_per_abs(index->sample_size), index->metric == UHA_L2,
            error_flag, stream);
        scan_queries = ws->projected.get();
        launches += 3;
    } else if (index->kind == IndexKind::sampled) {
        uha::launch_prepare_sampled(
            source, n, index->dimension, index->columns.get(),
            index->metric == UHA_L2 ? index->scales.get() : nullptr,
            index->sample_size, prepared, index->padded_dim, error_flag, stream);
        ++launches;
    } else {
        uha::launch_prepare_dense(source, n, index->dimension, prepared,
                                  index->padded_dim, error_flag, stream);
        ++launches;
    }

    if (precision_strategy(c.strategy)) {
        const uha::LowpPlan plan =
            enqueue_lowp_scores(index, ws, c.strategy, n, false, nullptr, nullptr,
                                hierarchical ? scan_queries : prepared, false);
        const uint32_t k = static_cast<uint32_t>(
            std::min<uint64_t>(ws->candidates_per_query, index->rows));
        uint32_t* candidates = c.candidates != nullptr ? c.candidates : ws->candidates.get();
        launches += enqueue_lowp_candidates(c, n, plan, k, candidates, time_scan, scan_start,
                                            scan_stop) - 2;
        if (hierarchical) {
            // the reference's binary64 distance of every candidate, in the
            // projected space; the smallest (lowest row on ties) is the answer
            uha::launch_rescore_projected(candidates, k, static_cast<uint32_t>(n),
                                          index->rows64.get(), ws->projected64.get(),
                                          static_cast<uint32_t>(index->projection_dimension),
                                          results, exact, stream);
            return launches + 3;
        }
        if (c.finish_stream != nullptr) {
            // the re-score of this batch runs on the finish stream, behind the
            // candidate selection (it overlaps the next batch's scores)
            check_cuda(cudaEventRecord(c.handoff, stream), "event");
            check_cuda(cudaStreamWaitEvent(c.finish_stream, c.handoff, 0), "event");
            stream = c.finish_stream;
        }
        uha::ReplayInputs in{};
        in.op = uha::ReplayOp::l2_sequential;
        in.rows = index->scan_rows.get();
        in.queries = prepared;
        in.dim = index->scan_dim;
        in.padded_dim = index->padded_dim;
        if (fp32_rescore_strategy(c.strategy)) {
            set_emulated(in, index);
            const uha::Bound bound32 =
                make_bound(uha::rescore_depth(index->padded_dim), index->scan_dim, 2);
            double* slot = c.cand_dist != nullptr ? c.cand_dist : ws->cand_dist.get();
            uha::launch_rescore32(bound32, in, candidates, k, static_cast<uint32_t>(n),
                                  static_cast<uint32_t>(index->rows),
                                  reinterpret_cast<float*>(slot),
                                  c.rescore_done != nullptr ? c.rescore_done
                                                            : ws->rescore_done.get(),
                                  results, exact, replay_count, stream);
            return launches + 4;
        }
        const uha::Bound64 bound =
            uha::make_bound64(uha::rescore_depth(index->padded_dim), index->scan_dim);
        uha::launch_rescore(bound, in, candidates, k, static_cast<uint32_t>(n),
                            static_cast<uint32_t>(index->rows),
                            c.cand_dist != nullptr ? c.cand_dist : ws->cand_dist.get(),
                            c.rescore_done != nullptr ? c.rescore_done
                                                      : ws->rescore_done.get(),
                            results, exact, replay_count, stream);
        return launches + 4;
    }

    const bool gemm = c.strategy == UHA_GEMM && index->metric == UHA_L2;
    uha::ScanOp op = uha::ScanOp::l2;
    if (gemm) {
        op = uha::ScanOp::dot;
    } else if (index->metric == UHA_L1) {
        op = index->weights32.size() != 0 ? uha::ScanOp::l1_weighted : uha::ScanOp::l1;
    }
    const bool median = hierarchical && index->metric == UHA_L1;
    const TunedPlan* tuned = ws->find_tuned(n, static_cast<int>(c.strategy));
    uha::ScanPlan plan = tuned != nullptr && !tuned->lowp && !tuned->median
                             ? tuned->scan
                             : uha::plan_scan(index->rows, index->padded_dim, n,
                                              index->sm_count);
    if (median) {
        plan.chunks = 1;
        plan.depth = 0;
    }
    const uint64_t partial_count =
        checked_mul(checked_mul(plan.chunks, n, "partials"), index->rows, "partials");
    if (c.partials == nullptr && ws->partials.size() < partial_count) {
        // Grows to the largest plan used so far; the previous contents are not
        // needed (stream order: earlier kernels have consumed them).
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        ws->partials.allocate(partial_count);
    }
    if (time_scan) {
        check_cuda(cudaEventRecord(scan_start, stream), "event");
    }
    if (median) {
        if (ws->median_min.size() < n) {
            check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
            ws->median_min.allocate(std::max<uint64_t>(n, ws->max_batch));
        }
        uha::launch_median_scan(median_plan(index, ws, n), index->scan_rows.get(),
                                index->scan_rows_t.get(),
                                index->rows_pitch, index->rows, index->padded_dim,
                                index->projection_dimension, scan_queries, n,
                                ws->query_err.get(), ws->coord_err.get(),
                                index->row_err_max, kMedianRel, kMedianAbs,
                                ws->median_min.get(), ws->partials.get(),
                                ws->pair_err.get(), stream);
    } else {
        uha::launch_scan(plan, op, index->scan_rows.get(), index->rows,
                         index->padded_dim, index->weights32.get(), scan_queries, n,
                         c.partials != nullptr ? c.partials : ws->partials.get(), stream);
    }
    if (time_scan) {
        check_cuda(cudaEventRecord(scan_stop, stream), "event");
    }
    ++launches;
    if (c.finish_stream != nullptr) {
        // the argmin of this batch runs on the finish stream, behind the scan
        check_cuda(cudaEventRecord(c.handoff, stream), "event");
        check_cuda(cudaStreamWaitEvent(c.finish_stream, c.handoff, 0), "event");
        stream = c.finish_stream;
    }

    const uha::PartialView view{c.partials != nullptr ? c.partials : ws->partials.get(),
                                plan.chunks,
                                static_cast<uint32_t>(n),
                                static_cast<uint32_t>(index->rows)};
    if (gemm) {
        uha::launch_query_norms(scan_queries, n, index->padded_dim,
                                ws->query_norms.get(), stream);
        uha::launch_finalize_gemm(view, index->row_norms.get(), ws->query_norms.get(),
                                  results, stream);
        check_cuda(cudaMemsetAsync(exact, 0xff, n * sizeof(double), stream),
                   "cannot clear distances");
        return launches + 2;
    }

    uha::Bound bound{};
    uha::ReplayInputs in{};
    certification_inputs(index, ws, plan, op, prepared, &bound, &in);
    uha::launch_argmin(view, bound, in, results, exact, ws->finalize_scratch.get(),
                       ws->max_batch, replay_count, stream);
    ++launches;
    if (hierarchical && c.want_distances) {
        // reported distances of a hierarchy: the reference's binary64 value of
        // each selected row
        uha::launch_refine_winners(in, bound, results, static_cast<uint32_t>(n), exact,
                                   stream);
        ++launches;
    }
    return launches;
}

void fill_trivial(uint64_t n, uint64_t* out_indices, double* out_distances)
{
    for (uint64_t q = 0; q < n; ++q) {
        out_indices[q] = 0;
        if (out_distances != nullptr) {
            out_distances[q] = 0.0;
        }
    }
}

// The host side of one call: check the status words (synchronised), then
// convert Result / replayed distances into the caller's arrays.
void finish_call(const uha_index* index, uha_workspace* ws, uint64_t n,
                 const uha::Result* results, const double* exact,
                 uint64_t* out_indices, double* out_distances)
{
    const uint32_t flag = ws->host_counters.get()[1];
    if (flag & 8u) {
        fail(UHA_RUNTIME_ERROR, "tensor-core pipeline wait timed out");
    }
    if (flag & 16u) {
        fail(UHA_RUNTIME_ERROR, "flat query row copy wait timed out");
    }
    if (flag & static_cast<uint32_t>(uha::kCandidateOverflow)) {
        fail(UHA_RUNTIME_ERROR, "filtered candidate list overflowed");
    }
    if (flag != 0) {
        if ((flag & 1u) && index->kind == IndexKind::hierarchical) {
            fail(UHA_INVALID_ARGUMENT, "sampled query coordinate must be finite");
        }
        if (flag & 4u) {
            fail(UHA_OVERFLOW_ERROR, "projected query is not finite");
        }
        if (index->kind == IndexKind::sampled) {
            fail(UHA_INVALID_ARGUMENT,
                 (flag & 1u) ? "sampled query coordinate must be finite"
                             : "weighted sampled query coordinate must be finite");
        }
        fail(UHA_INVALID_ARGUMENT, "queries must be finite");
    }
    for (uint64_t q = 0; q < n; ++q) {
        out_indices[q] = results[q].row;
        if (out_distances != nullptr) {
            out_distances[q] = std::isnan(exact[q]) ? static_cast<double>(results[q].distance)
                                                    : exact[q];
        }
    }
    const uint32_t replayed = ws->host_counters.get()[0];
    ws->last.replayed_queries = replayed;
    ws->last.certified_queries = n - std::min<uint64_t>(n, replayed);
}

void validate_query_call(const uha_index* index, uha_workspace* ws,
                         const float* queries, uint64_t count, uint64_t batch,
                         uha_strategy strategy, const uint64_t* out_indices)
{
    require(index != nullptr, UHA_INVALID_ARGUMENT, "index must not be null");
    require(ws != nullptr && ws->owner == index, UHA_INVALID_ARGUMENT,
            "CUDA workspace belongs to a different index");
    require(batch <= ws->max_batch, UHA_INVALID_ARGUMENT,
            "query count exceeds CUDA workspace capacity");
    require(strategy == UHA_DIRECT || strategy == UHA_GEMM || precision_strategy(strategy),
            UHA_INVALID_ARGUMENT, "unknown CUDA query strategy");
    require(!precision_strategy(strategy) || index->metric == UHA_L2, UHA_INVALID_ARGUMENT,
            "precision strategies serve L2 indexes");
    require(!fp32_rescore_strategy(strategy) || index->kind != IndexKind::hierarchical,
            UHA_INVALID_ARGUMENT, "FP32 re-score strategies serve exact and flat L2 indexes");
    if (count != 0) {
        require(out_indices != nullptr, UHA_INVALID_ARGUMENT, "output must not be null");
        require(queries != nullptr || index->dimension == 0, UHA_INVALID_ARGUMENT,
                "query pointer must not be null");
    }
}

// Calls of many small batches on exact and flat indexes with the certified or
// norm-identity strategy run as a two-stage pipeline: batch b's preparation
// and scan (workspace stream) overlap the argmin of batch b - 1 (a second
// stream), with two slots of prepared queries and partial sums.
bool pipeline_applies(const uha_index* index, uha_strategy strategy, uint64_t batch,
                      uint64_t batches)
{
    if (batches < 2 || index->kind == IndexKind::hierarchical) {
        return false;
    }
    if (precision_strategy(strategy)) {
        return true;  // scores of batch b overlap the re-score of batch b - 1
    }
    return batch <= 8 && (strategy == UHA_DIRECT || strategy == UHA_GEMM) &&
           !small_path_applies(index, strategy) && !flat_path_applies(index, strategy, batch);
}

void prepare_pipeline(const uha_index* index, uha_workspace* ws, uha_strategy strategy,
                      uint64_t batch)
{
    cudaStream_t stream = ws->stream;
    if (ws->finish_stream == nullptr) {
        check_cuda(cudaStreamCreateWithFlags(&ws->finish_stream, cudaStreamNonBlocking),
                   "cannot create CUDA stream");
        for (cudaEvent_t& e : ws->pipe_events) {
            check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming),
                       "cannot create CUDA event");
        }
    }
    const uint64_t prepared_slot = checked_mul(batch, index->padded_dim, "prepared queries");
    if (precision_strategy(strategy)) {
        const uint64_t cand = checked_mul(batch, uha::max_rerank_candidates(), "candidates");
        if (ws->pipe_prepared.size() < 2 * prepared_slot || ws->pipe_candidates.size() < 2 * cand) {
            check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
            check_cuda(cudaStreamSynchronize(ws->finish_stream), "CUDA query failed");
            ws->pipe_prepared.allocate(2 * prepared_slot);
            ws->pipe_candidates.allocate(2 * cand);
            ws->pipe_cand_dist.allocate(2 * cand);
            ws->pipe_rescore_done.allocate(2 * batch);
            check_cuda(cudaMemsetAsync(ws->pipe_rescore_done.get(), 0,
                                       ws->pipe_rescore_done.bytes(), stream),
                       "cannot clear re-score counters");
        }
        check_cuda(cudaEventRecord(ws->pipe_events[4], stream), "event");
        check_cuda(cudaStreamWaitEvent(ws->finish_stream, ws->pipe_events[4], 0), "event");
        return;
    }
    // the largest plan any batch size up to `batch` uses
    uint64_t per_slot = 0;
    for (uint64_t n = 1; n <= batch; ++n) {
        const TunedPlan* tuned = ws->find_tuned(n, static_cast<int>(strategy));
        const uha::ScanPlan plan = tuned != nullptr && !tuned->lowp && !tuned->median
                                       ? tuned->scan
                                       : uha::plan_scan(index->rows, index->padded_dim, n,
                                                        index->sm_count);
        per_slot = std::max(per_slot, checked_mul(checked_mul(plan.chunks, n, "partials"),
                                                  index->rows, "partials"));
    }
    const uint64_t prepared = prepared_slot;
    if (ws->pipe_partials.size() < 2 * per_slot ||
        ws->pipe_prepared.size() < 2 * prepared) {
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        check_cuda(cudaStreamSynchronize(ws->finish_stream), "CUDA query failed");
        ws->pipe_partials.allocate(2 * per_slot);
        ws->pipe_prepared.allocate(2 * prepared);
    }
    // the argmin stream starts behind everything already on the workspace stream
    check_cuda(cudaEventRecord(ws->pipe_events[4], stream), "event");
    check_cuda(cudaStreamWaitEvent(ws->finish_stream, ws->pipe_events[4], 0), "event");
}

// Event pairs for timing the scan of every batch of a call.
void ensure_scan_events(uha_workspace* ws, uint64_t batches)
{
    while (ws->scan_events.size() < 2 * batches) {
        cudaEvent_t e = nullptr;
        check_cuda(cudaEventCreate(&e), "cannot create CUDA event");
        ws->scan_events.push_back(e);
    }
}

}  // namespace uha_engine

using namespace uha_engine;

extern "C" uha_status uha_query(const uha_index* index, uha_workspace* ws,
                                const float* queries, uint64_t query_count,
                                int queries_on_device, uha_strategy strategy,
                                uint64_t* out_indices, double* out_distances)
{
    return uha_query_many(index, ws, queries, query_count, query_count == 0 ? 1 : query_count,
                          queries_on_device, strategy, out_indices, out_distances);
}

extern "C" uha_status uha_query_many(const uha_index* index, uha_workspace* ws,
                                     const float* queries, uint64_t query_count,
                                     uint64_t batch, int queries_on_device,
                                     uha_strategy strategy, uint64_t* out_indices,
                                     double* out_distances)
{
    return guarded([&] {
        require(batch != 0, UHA_INVALID_ARGUMENT, "batch size must be positive");
        validate_query_call(index, ws, queries, query_count,
                            std::min(batch, query_count == 0 ? batch : query_count),
                            strategy, out_indices);
        ws->last = uha_query_stats{};
        ws->last.query_count = query_count;
        if (query_count == 0) {
            return;
        }
        if ((index->kind == IndexKind::hierarchical && index->rows == 1) ||
            index->padded_dim == 0) {
            // A one-row hierarchy answers row 0 without projecting (or
            // validating) the query (hierarchical_l2_ann_index.cpp:164-166);
            // with no sampled coordinate every distance is zero and row 0 wins.
            fill_trivial(query_count, out_indices, out_distances);
            ws->last.certified_queries = query_count;
            return;
        }

        DeviceGuard guard(index->device);
        uha::clear_stale_cuda_error();
        cudaStream_t stream = ws->stream;
        const uint64_t n = query_count;
        const uint64_t batches = (n + batch - 1) / batch;
        // device-side answers of the whole call
        if (ws->call_results.size() < n) {
            ws->call_results.allocate(n);
            ws->call_exact.allocate(n);
            ws->host_results.allocate(n);
            ws->host_exact.allocate(n);
        }
        if (ws->timing) {
            ensure_scan_events(ws, batches);
            check_cuda(cudaEventRecord(ws->events[0], stream), "event");
        }
        check_cuda(cudaMemsetAsync(ws->counters.get(), 0, ws->counters.bytes(), stream),
                   "cannot clear query counters");
        BatchContext ctx{index, ws, strategy, out_distances != nullptr};
        ctx.filter_candidates = true;
        const bool pipelined = pipeline_applies(index, strategy, batch, batches);
        if (pipelined) {
            prepare_pipeline(index, ws, strategy, batch);
        }
        // Fused flat batches of device-resident queries go round-robin over
        // kFlatLanes streams: every launch still answers its own batch, and
        // the lanes' launch chains run side by side.
        const int lanes = !pipelined && queries_on_device && !ws->timing && batches > 1 &&
                                  flat_path_applies(index, strategy, batch)
                              ? uha::kFlatLanes
                              : 1;
        if (lanes > 1) {
            ensure_flat_scratch(index, ws);
            ws->flat_streams[0] = stream;
            for (int i = 0; i < lanes; ++i) {
                if (i > 0 && ws->flat_streams[i] == nullptr) {
                    check_cuda(cudaStreamCreateWithFlags(&ws->flat_streams[i],
                                                         cudaStreamNonBlocking),
                               "cannot create CUDA stream");
                }
                if (ws->flat_events[i] == nullptr) {
                    check_cuda(cudaEventCreateWithFlags(&ws->flat_events[i],
                                                        cudaEventDisableTiming),
                               "cannot create CUDA event");
                }
            }
            check_cuda(cudaEventRecord(ws->flat_events[0], stream), "event");
            for (int i = 1; i < lanes; ++i) {
                check_cuda(cudaStreamWaitEvent(ws->flat_streams[i], ws->flat_events[0], 0),
                           "event");
            }
        }
        uint64_t launches = 0;
        for (uint64_t b = 0; b < batches; ++b) {
            const uint64_t start = b * batch;
            const uint64_t count = std::min(batch, n - start);
            const float* source = queries + start * index->dimension;
            BatchContext bc = ctx;
            if (pipelined) {
                // slot b % 2 is free once the argmin of batch b - 2 is done
                const uint64_t slot = b % 2;
                if (b >= 2) {
                    check_cuda(cudaStreamWaitEvent(stream, ws->pipe_events[2 + slot], 0),
                               "event");
                }
                bc.prepared = ws->pipe_prepared.get() + slot * batch * index->padded_dim;
                if (precision_strategy(strategy)) {
                    const uint64_t cand = batch * uha::max_rerank_candidates();
                    bc.candidates = ws->pipe_candidates.get() + slot * cand;
                    bc.cand_dist = ws->pipe_cand_dist.get() + slot * cand;
                    bc.rescore_done = ws->pipe_rescore_done.get() + slot * batch;
                } else {
                    bc.partials =
                        ws->pipe_partials.get() + slot * (ws->pipe_partials.size() / 2);
                }
                bc.finish_stream = ws->finish_stream;
                bc.handoff = ws->pipe_events[slot];
            }
            if (!queries_on_device) {
                check_cuda(cudaMemcpyAsync(ws->raw_queries.get(), source,
                                           count * index->dimension * sizeof(float),
                                           cudaMemcpyHostToDevice, stream),
                           "cannot copy queries to the CUDA device");
                source = ws->raw_queries.get();
            }
            const bool timed = ws->timing && b % ws->timing_stride == 0;
            bc.flat_lane = static_cast<int>(b % static_cast<uint64_t>(lanes));
            launches += enqueue_batch(bc, source, count, ws->call_results.get() + start,
                                      ws->call_exact.get() + start, timed,
                                      timed ? ws->scan_events[2 * b] : nullptr,
                                      timed ? ws->scan_events[2 * b + 1] : nullptr);
            if (pipelined) {
                check_cuda(cudaEventRecord(ws->pipe_events[2 + b % 2], ws->finish_stream),
                           "event");
            }
        }
        if (pipelined) {
            check_cuda(cudaEventRecord(ws->pipe_events[4], ws->finish_stream), "event");
            check_cuda(cudaStreamWaitEvent(stream, ws->pipe_events[4], 0), "event");
        }
        for (int i = 1; i < lanes; ++i) {
            check_cuda(cudaEventRecord(ws->flat_events[i], ws->flat_streams[i]), "event");
            check_cuda(cudaStreamWaitEvent(stream, ws->flat_events[i], 0), "event");
        }
        check_cuda(cudaMemcpyAsync(ws->host_results.get(), ws->call_results.get(),
                                   n * sizeof(uha::Result), cudaMemcpyDeviceToHost,
                                   stream),
                   "cannot copy query results from the CUDA device");
        check_cuda(cudaMemcpyAsync(ws->host_exact.get(), ws->call_exact.get(),
                                   n * sizeof(double), cudaMemcpyDeviceToHost, stream),
                   "cannot copy query distances from the CUDA device");
        check_cuda(cudaMemcpyAsync(ws->host_counters.get(), ws->counters.get(),
                                   ws->counters.bytes(), cudaMemcpyDeviceToHost, stream),
                   "cannot copy query counters from the CUDA device");
        if (ws->timing) {
            check_cuda(cudaEventRecord(ws->events[3], stream), "event");
        }
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        if (ws->timing) {
            float ms = 0.f;
            double scan = 0.0;
            uint64_t timed = 0;
            for (uint64_t b = 0; b < batches; b += ws->timing_stride) {
                check_cuda(cudaEventElapsedTime(&ms, ws->scan_events[2 * b],
                                                ws->scan_events[2 * b + 1]),
                           "event");
                scan += ms;
                ++timed;
            }
            ws->last.scan_ms = scan;
            ws->last.timed_scans = timed;
            check_cuda(cudaEventElapsedTime(&ms, ws->events[0], ws->events[3]), "event");
            ws->last.device_ms = ms;
        }
        ws->last.kernel_launches = launches;
        if ((ws->host_counters.get()[1] & uha::kCandidateOverflow) != 0u &&
            !ws->filter_disabled) {
            // a query's filtered candidate list overflowed: answer the whole
            // call again with the slab selection
            ws->filter_disabled = true;
            const uha_status again =
                uha_query_many(index, ws, queries, query_count, batch, queries_on_device,
                               strategy, out_indices, out_distances);
            ws->filter_disabled = false;
            if (again != UHA_OK) {
                fail(again, uha_last_error());
            }
            return;
        }
        finish_call(index, ws, n, ws->host_results.get(), ws->host_exact.get(),
                    out_indices, out_distances);
    });
}

extern "C" uha_status uha_workspace_set_replay(uha_workspace* workspace,
                                               uha_replay_arithmetic arithmetic)
{
    return guarded([&] {
        require(workspace != nullptr, UHA_INVALID_ARGUMENT,
                "workspace must not be null");
        require(arithmetic == UHA_REPLAY_BINARY64 || arithmetic == UHA_REPLAY_EMULATED,
                UHA_INVALID_ARGUMENT, "unknown replay arithmetic");
        workspace->emulated_replay = arithmetic == UHA_REPLAY_EMULATED;
    });
}

extern "C" uha_status uha_workspace_set_candidates(uha_workspace* workspace,
                                                   uint32_t candidates)
{
    return guarded([&] {
        require(workspace != nullptr, UHA_INVALID_ARGUMENT,
                "workspace must not be null");
        require(candidates >= 1 && candidates <= uha::max_rerank_candidates(),
                UHA_INVALID_ARGUMENT, "candidate count must be between 1 and 64");
        workspace->candidates_per_query = candidates;
    });
}

extern "C" uha_status uha_precision_scores(const uha_index* index, uha_workspace* ws,
                                           const float* queries, uint64_t query_count,
                                           uha_strategy strategy, float* out_scores,
                                           float* out_norms)
{
    return guarded([&] {
        require(precision_strategy(strategy), UHA_INVALID_ARGUMENT,
                "not a precision strategy");
        require(index == nullptr || index->kind != IndexKind::hierarchical,
                UHA_INVALID_ARGUMENT, "precision scores serve exact and flat L2 indexes");
        validate_query_call(index, ws, queries, query_count, query_count, strategy,
                            reinterpret_cast<const uint64_t*>(out_scores));
        if (query_count == 0 || index->padded_dim == 0) {
            return;
        }
        DeviceGuard guard(index->device);
        uha::clear_stale_cuda_error();
        cudaStream_t stream = ws->stream;
        const uint64_t n = query_count;
        check_cuda(cudaMemsetAsync(ws->counters.get(), 0, ws->counters.bytes(), stream),
                   "cannot clear query counters");
        check_cuda(cudaMemcpyAsync(ws->raw_queries.get(), queries,
                                   n * index->dimension * sizeof(float),
                                   cudaMemcpyHostToDevice, stream),
                   "cannot copy queries to the CUDA device");
        int* error_flag = reinterpret_cast<int*>(ws->counters.get() + 1);
        if (index->kind == IndexKind::sampled) {
            uha::launch_prepare_sampled(ws->raw_queries.get(), n, index->dimension,
                                        index->columns.get(), index->scales.get(),
                                        index->sample_size, ws->prepared.get(),
                                        index->padded_dim, error_flag, stream);
        } else {
            uha::launch_prepare_dense(ws->raw_queries.get(), n, index->dimension,
                                      ws->prepared.get(), index->padded_dim, error_flag,
                                      stream);
        }
        const uha::LowpPlan plan =
            enqueue_lowp_scores(index, ws, strategy, n, false, nullptr, nullptr);
        const uint64_t per_split = n * index->rows;
        std::vector<float> slabs(plan.splits * per_split);
        check_cuda(cudaMemcpyAsync(slabs.data(), ws->partials.get(),
                                   slabs.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                   stream),
                   "cannot copy scores from the CUDA device");
        if (out_norms != nullptr) {
            check_cuda(cudaMemcpyAsync(out_norms,
                                       index->lowp[static_cast<int>(lowp_type(strategy))]
                                           .norms.get(),
                                       index->rows * sizeof(float), cudaMemcpyDeviceToHost,
                                       stream),
                       "cannot copy norms from the CUDA device");
        }
        check_cuda(cudaMemcpyAsync(ws->host_counters.get(), ws->counters.get(),
                                   ws->counters.bytes(), cudaMemcpyDeviceToHost, stream),
                   "cannot copy query counters from the CUDA device");
        check_cuda(cudaStreamSynchronize(stream), "CUDA query failed");
        const uint32_t flag = ws->host_counters.get()[1];
        if (flag & 8u) {
            fail(UHA_RUNTIME_ERROR, "tensor-core pipeline wait timed out");
        }
        require(flag == 0, UHA_INVALID_ARGUMENT, "queries must be finite");
        // split slabs summed in split order, as the candidate selection does
        for (uint64_t i = 0; i < per_split; ++i) {
            float acc = 0.f;
            for (uint32_t sp = 0; sp < plan.splits; ++sp) {
                acc += slabs[sp * per_split + i];
            }
            out_scores[i] = acc;
        }
    });
}

// ---------------------------------------------------------- probabilities

namespace {

// The probability build of uha_importance_probabilities(_device): the rows
// either copied from the host (host_rows) or already on the device
// (device_rows, checked for finiteness there).
void importance_probabilities(int device, uha_metric metric, const float* host_rows,
                              const float* device_rows, uint64_t row_count,
                              uint64_t dimension, uha_pair_backend backend,
                              uint64_t pair_chunks, double* out,
                              uha_probability_report* report)
{
    require(pair_chunks != 0, UHA_INVALID_ARGUMENT, "GPU pair chunk count must be positive");
    require(metric == UHA_L2 || metric == UHA_L1, UHA_INVALID_ARGUMENT, "unknown metric");
    require(backend == UHA_PAIRS_DIRECT || backend == UHA_PAIRS_GRAM ||
                backend == UHA_PAIRS_DIRECT_MAX32 || backend == UHA_PAIRS_GRAM_MAX32,
            UHA_INVALID_ARGUMENT, "unknown pair-distance backend");
    const bool gram = backend == UHA_PAIRS_GRAM || backend == UHA_PAIRS_GRAM_MAX32;
    const bool single = backend == UHA_PAIRS_DIRECT_MAX32 || backend == UHA_PAIRS_GRAM_MAX32;
    require(!(metric == UHA_L1 && gram), UHA_INVALID_ARGUMENT,
            "L1 distance has no matrix-multiplication identity");
    require(out != nullptr || dimension == 0, UHA_INVALID_ARGUMENT, "output must not be null");
    const float* given = host_rows != nullptr ? host_rows : device_rows;
    require(given != nullptr || row_count * dimension == 0, UHA_INVALID_ARGUMENT,
            "representative matrix must not be null");
    checked_mul(row_count, dimension, "representative matrix");
    if (host_rows != nullptr) {
        for (uint64_t i = 0; i < row_count * dimension; ++i) {
            if (!std::isfinite(host_rows[i])) {
                fail(UHA_INVALID_ARGUMENT, "representatives must be finite");
            }
        }
    }
    uha_probability_report rep{};
    rep.pair_count = row_count < 2 ? 0 : row_count * (row_count - 1) / 2;
    rep.pair_chunks = rep.pair_count == 0
                          ? 0
                          : (dimension == 0 ? 1 : std::min(pair_chunks, rep.pair_count));
    for (uint64_t j = 0; j < dimension; ++j) {
        out[j] = 0.0;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        fail(UHA_RUNTIME_ERROR, "no usable CUDA device");
    }
    require(device >= 0 && device < count, UHA_INVALID_ARGUMENT,
            "CUDA device index is out of range");
    if (row_count < 2 || dimension == 0) {
        if (report != nullptr) {
            *report = rep;
        }
        return;
    }
    require(row_count <= 65535ull * 32, UHA_LENGTH_ERROR,
            "probability construction supports at most 2097120 rows");
    DeviceGuard guard(device);
    const uint64_t pair_bytes =
        checked_mul(row_count, row_count * sizeof(double), "pair matrix");
    const uint64_t row_bytes =
        host_rows != nullptr ? checked_mul(row_count, dimension * sizeof(float), "rows") : 0;
    const uint64_t need = checked_add(
        checked_add(row_bytes, gram ? checked_add(pair_bytes, pair_bytes, "pair matrix")
                                    : pair_bytes,
                    "probability working set"),
        dimension * sizeof(double), "probability working set");
    size_t free_bytes = 0;
    size_t total_bytes = 0;
    check_cuda(cudaMemGetInfo(&free_bytes, &total_bytes), "cannot query CUDA memory");
    if (need > free_bytes) {
        fail(UHA_RUNTIME_ERROR, "probability working set exceeds free device memory");
    }
    rep.device_working_set_bytes = need;
    cudaStream_t stream = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking),
               "cannot create CUDA stream");
    struct StreamOwner {
        cudaStream_t s;
        ~StreamOwner() { cudaStreamDestroy(s); }
    } owner{stream};
    cudaEvent_t ev[5];
    for (auto& e : ev) {
        check_cuda(cudaEventCreate(&e), "cannot create CUDA event");
    }
    struct EventOwner {
        cudaEvent_t* e;
        ~EventOwner()
        {
            for (int i = 0; i < 5; ++i) {
                cudaEventDestroy(e[i]);
            }
        }
    } event_owner{ev};
    DeviceBuffer<float> copied(host_rows != nullptr ? row_count * dimension : 0);
    DeviceBuffer<double> inverse(row_count * row_count);
    DeviceBuffer<double> gram_matrix(gram ? row_count * row_count : 0);
    DeviceBuffer<unsigned long long> maxima(dimension);
    DeviceBuffer<int> flag(1);
    const float* rows = host_rows != nullptr ? copied.get() : device_rows;
    check_cuda(cudaEventRecord(ev[0], stream), "event");
    if (host_rows != nullptr) {
        check_cuda(cudaMemcpyAsync(copied.get(), host_rows, copied.bytes(),
                                   cudaMemcpyHostToDevice, stream),
                   "cannot copy representatives to the CUDA device");
    } else {
        int host_flag = 0;
        check_cuda(cudaMemsetAsync(flag.get(), 0, sizeof(int), stream), "cannot clear flag");
        uha::launch_finite_check(device_rows, row_count * dimension, flag.get(), stream);
        check_cuda(cudaMemcpyAsync(&host_flag, flag.get(), sizeof(int),
                                   cudaMemcpyDeviceToHost, stream),
                   "cannot copy the finiteness flag");
        check_cuda(cudaStreamSynchronize(stream), "finiteness check failed");
        require(host_flag == 0, UHA_INVALID_ARGUMENT, "representatives must be finite");
    }
    check_cuda(cudaMemsetAsync(inverse.get(), 0, inverse.bytes(), stream),
               "cannot clear pair matrix");
    check_cuda(cudaMemsetAsync(maxima.get(), 0, maxima.bytes(), stream),
               "cannot clear column maxima");
    check_cuda(cudaEventRecord(ev[1], stream), "event");
    const int m = metric == UHA_L2 ? 0 : 1;
    if (gram) {
        uha::launch_gram_inverse_distances(rows, row_count, dimension, gram_matrix.get(),
                                           inverse.get(), stream);
    } else {
        uha::launch_pair_distances(m, rows, row_count, dimension, inverse.get(), stream);
    }
    check_cuda(cudaEventRecord(ev[2], stream), "event");
    for (uint64_t c = 0; c < rep.pair_chunks; ++c) {
        const uint64_t begin = rep.pair_count * c / rep.pair_chunks;
        const uint64_t end = rep.pair_count * (c + 1) / rep.pair_chunks;
        uha::launch_coordinate_maxima(m, rows, row_count, dimension, inverse.get(),
                                      maxima.get(), begin, end, stream, single);
    }
    check_cuda(cudaEventRecord(ev[3], stream), "event");
    std::vector<unsigned long long> bits(dimension);
    check_cuda(cudaMemcpyAsync(bits.data(), maxima.get(), maxima.bytes(),
                               cudaMemcpyDeviceToHost, stream),
               "cannot copy probabilities from the CUDA device");
    check_cuda(cudaEventRecord(ev[4], stream), "event");
    check_cuda(cudaStreamSynchronize(stream), "probability kernels failed");
    for (uint64_t j = 0; j < dimension; ++j) {
        double v = 0.0;
        std::memcpy(&v, &bits[j], sizeof(v));
        out[j] = metric == UHA_L2 ? std::min(1.0, v) : v;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    rep.host_to_device_ms = ms;
    cudaEventElapsedTime(&ms, ev[1], ev[2]);
    rep.inverse_distance_ms = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    rep.coordinate_maximum_ms = ms;
    cudaEventElapsedTime(&ms, ev[3], ev[4]);
    rep.device_to_host_ms = ms;
    cudaEventElapsedTime(&ms, ev[0], ev[4]);
    rep.total_ms = ms;
    if (report != nullptr) {
        *report = rep;
    }
}

}  // namespace

extern "C" uha_status uha_importance_probabilities(
    int device, uha_metric metric, const float* rows, uint64_t row_count,
    uint64_t dimension, uha_pair_backend backend, uint64_t pair_chunks,
    double* out, uha_probability_report* report)
{
    return guarded([&] {
        require(rows != nullptr || row_count * dimension == 0, UHA_INVALID_ARGUMENT,
                "representative matrix must not be null");
        importance_probabilities(device, metric, rows != nullptr ? rows : nullptr, nullptr,
                                 row_count, dimension, backend, pair_chunks, out, report);
    });
}

extern "C" uha_status uha_importance_probabilities_device(
    int device, uha_metric metric, const float* device_rows, uint64_t row_count,
    uint64_t dimension, uha_pair_backend backend, uint64_t pair_chunks, double* out,
    uha_probability_report* report)
{
    return guarded([&] {
        require(device_rows != nullptr || row_count * dimension == 0, UHA_INVALID_ARGUMENT,
                "representative matrix must not be null");
        importance_probabilities(device, metric, nullptr, device_rows, row_count, dimension,
                                 backend, pair_chunks, out, report);
    });
}
