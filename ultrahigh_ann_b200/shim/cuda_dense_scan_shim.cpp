// CudaDenseL2ScanIndex, CudaDenseL1ScanIndex and cuda_runtime_info over the
// engine's C ABI. Replaces the reference translation units
// src/core/cuda_dense_l2_scan_index.cu, src/core/cuda_dense_l1_scan_index.cu
// and src/core/cuda_runtime_info.cu (their declarations:
// include/ultrahigh_ann/core/cuda_dense_l{2,1}_scan_index.hpp,
// include/ultrahigh_ann/core/cuda_runtime_info.hpp).
#include "ultrahigh_ann/core/cuda_dense_l1_scan_index.hpp"
#include "ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp"
#include "ultrahigh_ann/core/cuda_runtime_info.hpp"

#include "shim_support.hpp"

#include <cstdint>
#include <limits>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>

static_assert(sizeof(std::size_t) == sizeof(std::uint64_t),
              "row indices are passed through the C ABI as uint64_t");

namespace ultrahigh_ann {
namespace {

std::size_t checked_product(std::size_t a, std::size_t b, const char* what)
{
    if (b != 0 && a > std::numeric_limits<std::size_t>::max() / b) {
        throw std::length_error(std::string(what) + " size overflows");
    }
    return a * b;
}

// State shared by both dense engines.
struct DenseState {
    engine::IndexHandle handle;
    std::size_t dimension = 0;
    int device = 0;
    std::string device_name;

    void attach(uha_index* index, std::size_t d)
    {
        handle.index = index;
        dimension = d;
        device = engine::device_of(index);
        device_name = engine::device_name_of(index);
    }
    IndexSpaceUsage usage() const
    {
        uha_space_usage u{};
        engine::check(uha_index_space_usage(handle.index, &u));
        return IndexSpaceUsage{u.index_payload_bytes, u.query_workspace_payload_bytes,
                               u.unique_query_coordinates, u.sampled_multiplicity};
    }
};

struct DenseWorkspaceState {
    engine::WorkspaceHandle handle;
    const void* owner = nullptr;
    std::size_t maximum_batch_size = 0;
    std::size_t payload_bytes = 0;

    void attach(const DenseState& index, const void* owner_key, std::size_t batch)
    {
        engine::check(uha_workspace_create(index.handle.index, batch, &handle.workspace));
        owner = owner_key;
        uint64_t b = 0;
        uint64_t p = 0;
        engine::check(uha_workspace_info(handle.workspace, &b, &p));
        maximum_batch_size = b;
        payload_bytes = p;
    }
};

void run_query(const DenseState& index, DenseWorkspaceState* ws, const void* owner,
               const float* queries, std::size_t query_count, bool on_device,
               std::size_t output_size, std::size_t* output, int strategy,
               const char* name)
{
    if (ws == nullptr || ws->owner != owner) {
        throw std::invalid_argument(std::string("CUDA dense ") + name +
                                    " workspace belongs to a different index");
    }
    if (query_count > ws->maximum_batch_size) {
        throw std::invalid_argument(std::string("query count exceeds CUDA dense ") +
                                    name + " workspace capacity");
    }
    if (output_size != query_count) {
        throw std::invalid_argument(std::string("CUDA dense ") + name +
                                    " output size does not match query count");
    }
    if (query_count == 0) {
        return;
    }
    if (on_device && index.dimension != 0 && queries == nullptr) {
        throw std::invalid_argument(std::string("CUDA dense ") + name +
                                    " device query pointer must not be null");
    }
    engine::check(uha_query(index.handle.index, ws->handle.workspace, queries,
                            query_count, on_device ? 1 : 0,
                            static_cast<uha_strategy>(strategy),
                            reinterpret_cast<std::uint64_t*>(output), nullptr));
}

}  // namespace

bool cuda_dense_l2_scan_available() noexcept
{
    return uha_cuda_available() != 0;
}

bool cuda_dense_l1_scan_available() noexcept
{
    return uha_cuda_available() != 0;
}

std::optional<CudaRuntimeInfo> cuda_runtime_info(int device) noexcept
{
    uha_device_info info{};
    if (uha_device_info_get(device, &info) != UHA_OK) {
        return std::nullopt;
    }
    try {
        return CudaRuntimeInfo{
            .device = info.device,
            .device_name = info.device_name,
            .compute_capability_major = info.compute_capability_major,
            .compute_capability_minor = info.compute_capability_minor,
            .total_global_memory_bytes = info.total_global_memory_bytes,
            .compiled_runtime_version = info.compiled_runtime_version,
            .runtime_version = info.runtime_version,
            .driver_version = info.driver_version,
        };
    } catch (...) {
        return std::nullopt;
    }
}

// ------------------------------------------------------------------ L2

struct CudaDenseL2ScanIndex::Impl : DenseState {};
struct CudaDenseL2ScanIndex::QueryWorkspace::Impl : DenseWorkspaceState {};

CudaDenseL2ScanIndex::QueryWorkspace::QueryWorkspace(std::unique_ptr<Impl> implementation)
    : implementation_(std::move(implementation))
{
}
CudaDenseL2ScanIndex::QueryWorkspace::QueryWorkspace(QueryWorkspace&&) noexcept = default;
CudaDenseL2ScanIndex::QueryWorkspace&
CudaDenseL2ScanIndex::QueryWorkspace::operator=(QueryWorkspace&&) noexcept = default;
CudaDenseL2ScanIndex::QueryWorkspace::~QueryWorkspace() = default;

std::size_t CudaDenseL2ScanIndex::QueryWorkspace::maximum_batch_size() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->maximum_batch_size;
}

std::size_t CudaDenseL2ScanIndex::QueryWorkspace::payload_bytes() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->payload_bytes;
}

CudaDenseL2ScanIndex::CudaDenseL2ScanIndex(const DenseMatrix& representatives,
                                           int device)
    : implementation_(std::make_unique<Impl>())
{
    uha_index* index = nullptr;
    engine::check(uha_exact_index_create(device, UHA_L2,
                                         representatives.values().data(),
                                         representatives.rows(),
                                         representatives.cols(), &index));
    implementation_->attach(index, representatives.cols());
}

CudaDenseL2ScanIndex::CudaDenseL2ScanIndex(CudaDenseL2ScanIndex&&) noexcept = default;
CudaDenseL2ScanIndex&
CudaDenseL2ScanIndex::operator=(CudaDenseL2ScanIndex&&) noexcept = default;
CudaDenseL2ScanIndex::~CudaDenseL2ScanIndex() = default;

CudaDenseL2ScanIndex::QueryWorkspace
CudaDenseL2ScanIndex::make_query_workspace(std::size_t maximum_batch_size) const
{
    auto ws = std::make_unique<QueryWorkspace::Impl>();
    ws->attach(*implementation_, implementation_.get(), maximum_batch_size);
    return QueryWorkspace(std::move(ws));
}

std::size_t CudaDenseL2ScanIndex::query(std::span<const float> query,
                                        QueryWorkspace& workspace) const
{
    std::size_t output = 0;
    query_batch(query, 1, std::span<std::size_t>(&output, 1), workspace);
    return output;
}

void CudaDenseL2ScanIndex::query_batch(std::span<const float> queries,
                                       std::size_t query_count,
                                       std::span<std::size_t> output,
                                       QueryWorkspace& workspace,
                                       CudaDenseL2QueryStrategy strategy) const
{
    if (strategy != CudaDenseL2QueryStrategy::direct &&
        strategy != CudaDenseL2QueryStrategy::gemm) {
        throw std::invalid_argument("unknown CUDA dense L2 query strategy");
    }
    auto* ws = workspace.implementation_.get();
    if (ws != nullptr && ws->owner == implementation_.get() &&
        query_count <= ws->maximum_batch_size &&
        queries.size() != checked_product(query_count, implementation_->dimension,
                                          "CUDA dense L2 query batch")) {
        throw std::invalid_argument(
            "query batch dimensions do not match index dimension");
    }
    run_query(*implementation_, ws, implementation_.get(), queries.data(), query_count,
              false, output.size(), output.data(), static_cast<int>(strategy), "L2");
}

void CudaDenseL2ScanIndex::query_device_batch(const float* device_queries,
                                              std::size_t query_count,
                                              std::span<std::size_t> output,
                                              QueryWorkspace& workspace,
                                              CudaDenseL2QueryStrategy strategy) const
{
    if (strategy != CudaDenseL2QueryStrategy::direct &&
        strategy != CudaDenseL2QueryStrategy::gemm) {
        throw std::invalid_argument("unknown CUDA dense L2 query strategy");
    }
    run_query(*implementation_, workspace.implementation_.get(), implementation_.get(),
              device_queries, query_count, true, output.size(), output.data(),
              static_cast<int>(strategy), "L2");
}

IndexSpaceUsage CudaDenseL2ScanIndex::space_usage() const noexcept
{
    try {
        return implementation_->usage();
    } catch (...) {
        return IndexSpaceUsage{};
    }
}

int CudaDenseL2ScanIndex::device() const noexcept
{
    return implementation_->device;
}

const std::string& CudaDenseL2ScanIndex::device_name() const noexcept
{
    return implementation_->device_name;
}

// ------------------------------------------------------------------ L1

struct CudaDenseL1ScanIndex::Impl : DenseState {};
struct CudaDenseL1ScanIndex::QueryWorkspace::Impl : DenseWorkspaceState {};

CudaDenseL1ScanIndex::QueryWorkspace::QueryWorkspace(std::unique_ptr<Impl> implementation)
    : implementation_(std::move(implementation))
{
}
CudaDenseL1ScanIndex::QueryWorkspace::QueryWorkspace(QueryWorkspace&&) noexcept = default;
CudaDenseL1ScanIndex::QueryWorkspace&
CudaDenseL1ScanIndex::QueryWorkspace::operator=(QueryWorkspace&&) noexcept = default;
CudaDenseL1ScanIndex::QueryWorkspace::~QueryWorkspace() = default;

std::size_t CudaDenseL1ScanIndex::QueryWorkspace::maximum_batch_size() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->maximum_batch_size;
}

std::size_t CudaDenseL1ScanIndex::QueryWorkspace::payload_bytes() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->payload_bytes;
}

CudaDenseL1ScanIndex::CudaDenseL1ScanIndex(const DenseMatrix& representatives,
                                           int device)
    : implementation_(std::make_unique<Impl>())
{
    uha_index* index = nullptr;
    engine::check(uha_exact_index_create(device, UHA_L1,
                                         representatives.values().data(),
                                         representatives.rows(),
                                         representatives.cols(), &index));
    implementation_->attach(index, representatives.cols());
}

CudaDenseL1ScanIndex::CudaDenseL1ScanIndex(const DenseMatrix& representatives,
                                           std::span<const float> coordinate_weights,
                                           int device)
    : implementation_(std::make_unique<Impl>())
{
    if (coordinate_weights.size() != representatives.cols()) {
        throw std::invalid_argument(
            "CUDA dense L1 coordinate weights do not match the dimension");
    }
    uha_index* index = nullptr;
    engine::check(uha_weighted_l1_index_create(
        device, representatives.values().data(), representatives.rows(),
        representatives.cols(), coordinate_weights.data(), &index));
    implementation_->attach(index, representatives.cols());
}

CudaDenseL1ScanIndex::CudaDenseL1ScanIndex(CudaDenseL1ScanIndex&&) noexcept = default;
CudaDenseL1ScanIndex&
CudaDenseL1ScanIndex::operator=(CudaDenseL1ScanIndex&&) noexcept = default;
CudaDenseL1ScanIndex::~CudaDenseL1ScanIndex() = default;

CudaDenseL1ScanIndex::QueryWorkspace
CudaDenseL1ScanIndex::make_query_workspace(std::size_t maximum_batch_size) const
{
    auto ws = std::make_unique<QueryWorkspace::Impl>();
    ws->attach(*implementation_, implementation_.get(), maximum_batch_size);
    return QueryWorkspace(std::move(ws));
}

std::size_t CudaDenseL1ScanIndex::query(std::span<const float> query,
                                        QueryWorkspace& workspace) const
{
    std::size_t output = 0;
    query_batch(query, 1, std::span<std::size_t>(&output, 1), workspace);
    return output;
}

void CudaDenseL1ScanIndex::query_batch(std::span<const float> queries,
                                       std::size_t query_count,
                                       std::span<std::size_t> output,
                                       QueryWorkspace& workspace) const
{
    auto* ws = workspace.implementation_.get();
    if (ws != nullptr && ws->owner == implementation_.get() &&
        query_count <= ws->maximum_batch_size &&
        queries.size() != checked_product(query_count, implementation_->dimension,
                                          "CUDA dense L1 query batch")) {
        throw std::invalid_argument(
            "query batch dimensions do not match index dimension");
    }
    run_query(*implementation_, ws, implementation_.get(), queries.data(), query_count,
              false, output.size(), output.data(), UHA_DIRECT, "L1");
}

IndexSpaceUsage CudaDenseL1ScanIndex::space_usage() const noexcept
{
    try {
        return implementation_->usage();
    } catch (...) {
        return IndexSpaceUsage{};
    }
}

int CudaDenseL1ScanIndex::device() const noexcept
{
    return implementation_->device;
}

const std::string& CudaDenseL1ScanIndex::device_name() const noexcept
{
    return implementation_->device_name;
}

}  // namespace ultrahigh_ann
