// CudaSampledCoordinateL{2,1}AnnIndex over the engine's C ABI. Replaces the
// reference translation units src/coordinate_sampling/
// cuda_sampled_coordinate_l{2,1}_ann_index.cpp, which pack the sampled query
// coordinates on the host; the engine gathers them on the device. The
// coordinate sample is drawn by the reference's own build_coordinate_sample.
#include "ultrahigh_ann/coordinate_sampling/coordinate_sampling.hpp"
#include "ultrahigh_ann/coordinate_sampling/cuda_sampled_coordinate_l1_ann_index.hpp"
#include "ultrahigh_ann/coordinate_sampling/cuda_sampled_coordinate_l2_ann_index.hpp"

#include "cuda_index_shim.hpp"

#include <memory>
#include <utility>
#include <vector>

namespace ultrahigh_ann {
namespace {

CoordinateSample sample_checked(const DenseMatrix& input,
                                std::span<const double> probabilities,
                                std::size_t repetitions,
                                std::mt19937_64& random_engine)
{
    if (probabilities.size() != input.cols()) {
        throw std::invalid_argument(
            "sampling probability dimension does not match input");
    }
    return build_coordinate_sample(probabilities, repetitions, random_engine);
}

uha_index* create_sampled(uha_metric metric, const DenseMatrix& input,
                          const CoordinateSample& sample, int device)
{
    std::vector<std::uint64_t> cols;
    std::vector<std::uint64_t> mult;
    std::vector<double> inv;
    for (const SampledColumn& c : sample.columns) {
        cols.push_back(c.source_column);
        mult.push_back(c.multiplicity);
        inv.push_back(c.inverse_probability);
    }
    uha_index* index = nullptr;
    engine::check(uha_sampled_index_create(device, metric, input.values().data(),
                                           input.rows(), input.cols(), cols.data(),
                                           mult.data(), inv.data(), cols.size(),
                                           &index));
    return index;
}

}  // namespace

bool cuda_sampled_coordinate_l2_available() noexcept
{
    return uha_cuda_available() != 0;
}

bool cuda_sampled_coordinate_l1_available() noexcept
{
    return uha_cuda_available() != 0;
}

// ------------------------------------------------------------------ L2

struct CudaSampledCoordinateL2AnnIndex::Impl : engine::IndexState {};
struct CudaSampledCoordinateL2AnnIndex::QueryWorkspace::Impl : engine::WorkspaceState {};

CudaSampledCoordinateL2AnnIndex::QueryWorkspace::QueryWorkspace(
    std::unique_ptr<Impl> implementation)
    : implementation_(std::move(implementation))
{
}
CudaSampledCoordinateL2AnnIndex::QueryWorkspace::QueryWorkspace(
    QueryWorkspace&&) noexcept = default;
CudaSampledCoordinateL2AnnIndex::QueryWorkspace&
CudaSampledCoordinateL2AnnIndex::QueryWorkspace::operator=(QueryWorkspace&&) noexcept =
    default;
CudaSampledCoordinateL2AnnIndex::QueryWorkspace::~QueryWorkspace() = default;

std::size_t
CudaSampledCoordinateL2AnnIndex::QueryWorkspace::maximum_batch_size() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->maximum_batch_size;
}

std::size_t CudaSampledCoordinateL2AnnIndex::QueryWorkspace::payload_bytes() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->payload_bytes;
}

CudaSampledCoordinateL2AnnIndex::CudaSampledCoordinateL2AnnIndex(
    const DenseMatrix& input, std::span<const double> probabilities,
    std::size_t repetitions, std::mt19937_64& random_engine, int device)
    : CudaSampledCoordinateL2AnnIndex(
          input, sample_checked(input, probabilities, repetitions, random_engine),
          device)
{
}

CudaSampledCoordinateL2AnnIndex::CudaSampledCoordinateL2AnnIndex(
    const DenseMatrix& input, CoordinateSample coordinate_sample, int device)
    : implementation_(std::make_unique<Impl>())
{
    implementation_->attach(create_sampled(UHA_L2, input, coordinate_sample, device),
                            input.cols());
}

CudaSampledCoordinateL2AnnIndex::CudaSampledCoordinateL2AnnIndex(
    CudaSampledCoordinateL2AnnIndex&&) noexcept = default;
CudaSampledCoordinateL2AnnIndex& CudaSampledCoordinateL2AnnIndex::operator=(
    CudaSampledCoordinateL2AnnIndex&&) noexcept = default;
CudaSampledCoordinateL2AnnIndex::~CudaSampledCoordinateL2AnnIndex() = default;

CudaSampledCoordinateL2AnnIndex::QueryWorkspace
CudaSampledCoordinateL2AnnIndex::make_query_workspace(
    std::size_t maximum_batch_size) const
{
    auto ws = std::make_unique<QueryWorkspace::Impl>();
    ws->attach(*implementation_, implementation_.get(), maximum_batch_size);
    return QueryWorkspace(std::move(ws));
}

std::size_t CudaSampledCoordinateL2AnnIndex::query(
    std::span<const float> query, QueryWorkspace& workspace,
    CudaSampledCoordinateL2QueryStrategy strategy) const
{
    std::size_t output = 0;
    query_batch(query, 1, std::span<std::size_t>(&output, 1), workspace, strategy);
    return output;
}

void CudaSampledCoordinateL2AnnIndex::query_batch(
    std::span<const float> queries, std::size_t query_count,
    std::span<std::size_t> output, QueryWorkspace& workspace,
    CudaSampledCoordinateL2QueryStrategy strategy) const
{
    if (strategy != CudaSampledCoordinateL2QueryStrategy::direct &&
        strategy != CudaSampledCoordinateL2QueryStrategy::gemm) {
        throw std::invalid_argument("unknown CUDA sampled L2 query strategy");
    }
    engine::facade_query(*implementation_, workspace.implementation_.get(),
                         implementation_.get(), queries, query_count, output,
                         static_cast<uha_strategy>(strategy), "sampled", false);
}

IndexSpaceUsage CudaSampledCoordinateL2AnnIndex::space_usage() const noexcept
{
    return implementation_->usage();
}

int CudaSampledCoordinateL2AnnIndex::device() const noexcept
{
    return implementation_->device;
}

const std::string& CudaSampledCoordinateL2AnnIndex::device_name() const noexcept
{
    return implementation_->device_name;
}

// ------------------------------------------------------------------ L1

struct CudaSampledCoordinateL1AnnIndex::Impl : engine::IndexState {};
struct CudaSampledCoordinateL1AnnIndex::QueryWorkspace::Impl : engine::WorkspaceState {};

CudaSampledCoordinateL1AnnIndex::QueryWorkspace::QueryWorkspace(
    std::unique_ptr<Impl> implementation)
    : implementation_(std::move(implementation))
{
}
CudaSampledCoordinateL1AnnIndex::QueryWorkspace::QueryWorkspace(
    QueryWorkspace&&) noexcept = default;
CudaSampledCoordinateL1AnnIndex::QueryWorkspace&
CudaSampledCoordinateL1AnnIndex::QueryWorkspace::operator=(QueryWorkspace&&) noexcept =
    default;
CudaSampledCoordinateL1AnnIndex::QueryWorkspace::~QueryWorkspace() = default;

std::size_t
CudaSampledCoordinateL1AnnIndex::QueryWorkspace::maximum_batch_size() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->maximum_batch_size;
}

std::size_t CudaSampledCoordinateL1AnnIndex::QueryWorkspace::payload_bytes() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->payload_bytes;
}

CudaSampledCoordinateL1AnnIndex::CudaSampledCoordinateL1AnnIndex(
    const DenseMatrix& input, std::span<const double> probabilities,
    std::size_t repetitions, std::mt19937_64& random_engine, int device)
    : CudaSampledCoordinateL1AnnIndex(
          input, sample_checked(input, probabilities, repetitions, random_engine),
          device)
{
}

CudaSampledCoordinateL1AnnIndex::CudaSampledCoordinateL1AnnIndex(
    const DenseMatrix& input, CoordinateSample coordinate_sample, int device)
    : implementation_(std::make_unique<Impl>())
{
    implementation_->attach(create_sampled(UHA_L1, input, coordinate_sample, device),
                            input.cols());
}

CudaSampledCoordinateL1AnnIndex::CudaSampledCoordinateL1AnnIndex(
    CudaSampledCoordinateL1AnnIndex&&) noexcept = default;
CudaSampledCoordinateL1AnnIndex& CudaSampledCoordinateL1AnnIndex::operator=(
    CudaSampledCoordinateL1AnnIndex&&) noexcept = default;
CudaSampledCoordinateL1AnnIndex::~CudaSampledCoordinateL1AnnIndex() = default;

CudaSampledCoordinateL1AnnIndex::QueryWorkspace
CudaSampledCoordinateL1AnnIndex::make_query_workspace(
    std::size_t maximum_batch_size) const
{
    auto ws = std::make_unique<QueryWorkspace::Impl>();
    ws->attach(*implementation_, implementation_.get(), maximum_batch_size);
    return QueryWorkspace(std::move(ws));
}

std::size_t CudaSampledCoordinateL1AnnIndex::query(std::span<const float> query,
                                                   QueryWorkspace& workspace) const
{
    std::size_t output = 0;
    query_batch(query, 1, std::span<std::size_t>(&output, 1), workspace);
    return output;
}

void CudaSampledCoordinateL1AnnIndex::query_batch(std::span<const float> queries,
                                                  std::size_t query_count,
                                                  std::span<std::size_t> output,
                                                  QueryWorkspace& workspace) const
{
    engine::facade_query(*implementation_, workspace.implementation_.get(),
                         implementation_.get(), queries, query_count, output,
                         UHA_DIRECT, "sampled L1", false);
}

IndexSpaceUsage CudaSampledCoordinateL1AnnIndex::space_usage() const noexcept
{
    return implementation_->usage();
}

int CudaSampledCoordinateL1AnnIndex::device() const noexcept
{
    return implementation_->device;
}

const std::string& CudaSampledCoordinateL1AnnIndex::device_name() const noexcept
{
    return implementation_->device_name;
}

}  // namespace ultrahigh_ann
