// CudaHierarchicalL{2,1}AnnIndex over the engine's C ABI. Replaces the
// reference translation units src/hnsvw25/l{2,1}/hierarchical/
// cuda_hierarchical_l{2,1}_ann_index.cpp together with the internal
// CudaFloatProjection (src/core/cuda_float_projection.cu) and
// CudaMedianL1ScanIndex (src/hnsvw25/l1/hierarchical/
// cuda_median_l1_scan_index.cu) they use. The sample is drawn by the
// reference's own functions; the projection matrix is drawn by the engine from
// the caller's std::mt19937_64 (same distributions, same order), and the
// projected rows are formed on the device.
#include "ultrahigh_ann/hnsvw25/l1/hierarchical/cuda_hierarchical_l1_ann_index.hpp"
#include "ultrahigh_ann/hnsvw25/l2/hierarchical/cuda_hierarchical_l2_ann_index.hpp"

#include "cuda_index_shim.hpp"

#include <cmath>
#include <memory>
#include <utility>
#include <vector>

namespace ultrahigh_ann {
namespace {

void validate_parameters(const DenseMatrix& input, std::size_t projection_dimension,
                         const char* name)
{
    if (input.rows() == 0) {
        throw std::invalid_argument(std::string(name) +
                                    " expects at least one representative");
    }
    if (projection_dimension == 0) {
        throw std::invalid_argument("projection_dimension has to be a positive integer");
    }
}

// The reference's projection-basis checks (before the matrix draw), then the
// draw on the caller's engine, then the device index.
uha_index* create_hierarchy(uha_metric metric, const DenseMatrix& input,
                            const CoordinateSample& sample,
                            std::size_t projection_dimension,
                            std::mt19937_64& random_engine, int device,
                            const char* name)
{
    validate_parameters(input, projection_dimension, name);
    if (sample.columns.empty() && input.rows() > 1) {
        throw std::runtime_error("importance sampling selected no coordinates");
    }
    std::vector<std::uint64_t> cols;
    std::vector<std::uint64_t> mult;
    std::vector<double> inv;
    std::size_t multiplicity = 0;
    for (const SampledColumn& c : sample.columns) {
        if (c.source_column >= input.cols()) {
            throw std::out_of_range("sampled column index out of range");
        }
        if (c.multiplicity == 0 || !std::isfinite(c.inverse_probability) ||
            c.inverse_probability <= 0.0) {
            throw std::invalid_argument(
                "sampled columns require positive finite weights");
        }
        if (multiplicity > std::numeric_limits<std::size_t>::max() - c.multiplicity) {
            throw std::length_error("sampled multiplicity overflows");
        }
        multiplicity += c.multiplicity;
        cols.push_back(c.source_column);
        mult.push_back(c.multiplicity);
        inv.push_back(c.inverse_probability);
    }
    std::vector<double> matrix(projection_dimension * cols.size());
    {
        engine::EngineBridge bridge(random_engine);
        engine::check(metric == UHA_L2
                          ? uha_jl_matrix(mult.data(), inv.data(), cols.size(),
                                          projection_dimension, bridge.get(),
                                          matrix.data())
                          : uha_cauchy_matrix(mult.data(), inv.data(), cols.size(),
                                              projection_dimension, bridge.get(),
                                              matrix.data()));
        bridge.commit();
    }
    uha_index* index = nullptr;
    engine::check(uha_hierarchical_index_create(
        device, metric, input.values().data(), input.rows(), input.cols(),
        cols.data(), mult.data(), inv.data(), cols.size(), matrix.data(),
        projection_dimension, &index));
    return index;
}

CoordinateSample l2_sample(const DenseMatrix& input, std::size_t repetitions,
                           std::size_t projection_dimension,
                           std::mt19937_64& random_engine, int device,
                           ExecutionPolicy policy)
{
    validate_parameters(input, projection_dimension, "CudaHierarchicalL2AnnIndex");
    switch (policy) {
    case ExecutionPolicy::sequential:
    case ExecutionPolicy::cpu_parallel:
        return build_l2_importance_sample(input, repetitions, random_engine, policy);
    case ExecutionPolicy::gpu_fp32:
    case ExecutionPolicy::gpu_cublas_fp32: {
        const L2GpuProbabilityResult result = compute_l2_importance_probabilities_gpu(
            input, device, 128,
            policy == ExecutionPolicy::gpu_cublas_fp32 ? L2GpuDistanceBackend::cublas
                                                       : L2GpuDistanceBackend::direct);
        return build_l2_importance_sample(result.probabilities, repetitions,
                                          random_engine);
    }
    }
    throw std::invalid_argument("unknown L2 probability execution policy");
}

CoordinateSample l1_sample(const DenseMatrix& input, std::size_t repetitions,
                           std::size_t projection_dimension,
                           std::mt19937_64& random_engine, int device,
                           ExecutionPolicy policy)
{
    validate_parameters(input, projection_dimension, "CudaHierarchicalL1AnnIndex");
    switch (policy) {
    case ExecutionPolicy::sequential:
    case ExecutionPolicy::cpu_parallel:
        return build_l1_importance_sample(input, repetitions, random_engine, policy);
    case ExecutionPolicy::gpu_fp32: {
        const L1GpuProbabilityResult result =
            compute_l1_importance_probabilities_gpu(input, device);
        return build_l1_importance_sample(result.probabilities, repetitions,
                                          random_engine);
    }
    case ExecutionPolicy::gpu_cublas_fp32:
        throw std::invalid_argument(
            "gpu_cublas_fp32 is unavailable for L1 probability computation; "
            "L1 distance has no matrix-multiplication identity");
    }
    throw std::invalid_argument("unknown L1 probability execution policy");
}

template <typename Build>
CoordinateSample probabilities_sample(const DenseMatrix& input,
                                      std::span<const double> probabilities,
                                      std::size_t repetitions,
                                      std::size_t projection_dimension,
                                      std::mt19937_64& random_engine,
                                      const char* name, Build build)
{
    validate_parameters(input, projection_dimension, name);
    if (probabilities.size() != input.cols()) {
        throw std::invalid_argument(
            "importance probability dimension does not match input");
    }
    return build(probabilities, repetitions, random_engine);
}

}  // namespace

bool cuda_hierarchical_l2_available() noexcept
{
    return uha_cuda_available() != 0;
}

bool cuda_hierarchical_l1_available() noexcept
{
    return uha_cuda_available() != 0;
}

// ------------------------------------------------------------------ L2

struct CudaHierarchicalL2AnnIndex::Impl : engine::IndexState {};
struct CudaHierarchicalL2AnnIndex::QueryWorkspace::Impl : engine::WorkspaceState {};

CudaHierarchicalL2AnnIndex::QueryWorkspace::QueryWorkspace(
    std::unique_ptr<Impl> implementation)
    : implementation_(std::move(implementation))
{
}
CudaHierarchicalL2AnnIndex::QueryWorkspace::QueryWorkspace(QueryWorkspace&&) noexcept =
    default;
CudaHierarchicalL2AnnIndex::QueryWorkspace&
CudaHierarchicalL2AnnIndex::QueryWorkspace::operator=(QueryWorkspace&&) noexcept = default;
CudaHierarchicalL2AnnIndex::QueryWorkspace::~QueryWorkspace() = default;

std::size_t CudaHierarchicalL2AnnIndex::QueryWorkspace::maximum_batch_size() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->maximum_batch_size;
}

std::size_t CudaHierarchicalL2AnnIndex::QueryWorkspace::payload_bytes() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->payload_bytes;
}

CudaHierarchicalL2AnnIndex::CudaHierarchicalL2AnnIndex(
    const DenseMatrix& input, std::size_t repetitions,
    std::size_t projection_dimension, std::mt19937_64& random_engine, int device,
    ExecutionPolicy probability_execution_policy)
    : CudaHierarchicalL2AnnIndex(input,
                                 l2_sample(input, repetitions, projection_dimension,
                                           random_engine, device,
                                           probability_execution_policy),
                                 projection_dimension, random_engine, device)
{
}

CudaHierarchicalL2AnnIndex::CudaHierarchicalL2AnnIndex(
    const DenseMatrix& input, std::span<const double> importance_probabilities,
    std::size_t repetitions, std::size_t projection_dimension,
    std::mt19937_64& random_engine, int device)
    : CudaHierarchicalL2AnnIndex(
          input,
          probabilities_sample(input, importance_probabilities, repetitions,
                               projection_dimension, random_engine,
                               "CudaHierarchicalL2AnnIndex",
                               [](std::span<const double> p, std::size_t t,
                                  std::mt19937_64& e) {
                                   return build_l2_importance_sample(p, t, e);
                               }),
          projection_dimension, random_engine, device)
{
}

CudaHierarchicalL2AnnIndex::CudaHierarchicalL2AnnIndex(
    const DenseMatrix& input, CoordinateSample importance_sample,
    std::size_t projection_dimension, std::mt19937_64& random_engine, int device)
    : implementation_(std::make_unique<Impl>())
{
    implementation_->attach(create_hierarchy(UHA_L2, input, importance_sample,
                                             projection_dimension, random_engine,
                                             device, "CudaHierarchicalL2AnnIndex"),
                            input.cols());
}

CudaHierarchicalL2AnnIndex::CudaHierarchicalL2AnnIndex(
    CudaHierarchicalL2AnnIndex&&) noexcept = default;
CudaHierarchicalL2AnnIndex&
CudaHierarchicalL2AnnIndex::operator=(CudaHierarchicalL2AnnIndex&&) noexcept = default;
CudaHierarchicalL2AnnIndex::~CudaHierarchicalL2AnnIndex() = default;

CudaHierarchicalL2AnnIndex::QueryWorkspace
CudaHierarchicalL2AnnIndex::make_query_workspace(std::size_t maximum_batch_size) const
{
    auto ws = std::make_unique<QueryWorkspace::Impl>();
    ws->attach(*implementation_, implementation_.get(), maximum_batch_size);
    return QueryWorkspace(std::move(ws));
}

std::size_t CudaHierarchicalL2AnnIndex::query(std::span<const float> query,
                                              QueryWorkspace& workspace,
                                              CudaHierarchicalL2QueryStrategy strategy) const
{
    std::size_t output = 0;
    query_batch(query, 1, std::span<std::size_t>(&output, 1), workspace, strategy);
    return output;
}

void CudaHierarchicalL2AnnIndex::query_batch(std::span<const float> queries,
                                             std::size_t query_count,
                                             std::span<std::size_t> output,
                                             QueryWorkspace& workspace,
                                             CudaHierarchicalL2QueryStrategy strategy) const
{
    if (strategy != CudaHierarchicalL2QueryStrategy::direct &&
        strategy != CudaHierarchicalL2QueryStrategy::gemm) {
        throw std::invalid_argument("unknown CUDA hierarchical L2 query strategy");
    }
    engine::facade_query(*implementation_, workspace.implementation_.get(),
                         implementation_.get(), queries, query_count, output,
                         static_cast<uha_strategy>(strategy), "hierarchical", true);
}

IndexSpaceUsage CudaHierarchicalL2AnnIndex::space_usage() const noexcept
{
    return implementation_->usage();
}

int CudaHierarchicalL2AnnIndex::device() const noexcept
{
    return implementation_->device;
}

const std::string& CudaHierarchicalL2AnnIndex::device_name() const noexcept
{
    return implementation_->device_name;
}

// ------------------------------------------------------------------ L1

struct CudaHierarchicalL1AnnIndex::Impl : engine::IndexState {};
struct CudaHierarchicalL1AnnIndex::QueryWorkspace::Impl : engine::WorkspaceState {};

CudaHierarchicalL1AnnIndex::QueryWorkspace::QueryWorkspace(
    std::unique_ptr<Impl> implementation)
    : implementation_(std::move(implementation))
{
}
CudaHierarchicalL1AnnIndex::QueryWorkspace::QueryWorkspace(QueryWorkspace&&) noexcept =
    default;
CudaHierarchicalL1AnnIndex::QueryWorkspace&
CudaHierarchicalL1AnnIndex::QueryWorkspace::operator=(QueryWorkspace&&) noexcept = default;
CudaHierarchicalL1AnnIndex::QueryWorkspace::~QueryWorkspace() = default;

std::size_t CudaHierarchicalL1AnnIndex::QueryWorkspace::maximum_batch_size() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->maximum_batch_size;
}

std::size_t CudaHierarchicalL1AnnIndex::QueryWorkspace::payload_bytes() const noexcept
{
    return implementation_ == nullptr ? 0 : implementation_->payload_bytes;
}

CudaHierarchicalL1AnnIndex::CudaHierarchicalL1AnnIndex(const DenseMatrix& input,
                                                       std::size_t repetitions,
                                                       std::size_t projection_dimension,
                                                       std::mt19937_64& random_engine,
                                                       int device)
    : CudaHierarchicalL1AnnIndex(input, repetitions, projection_dimension, random_engine,
                                 device, ExecutionPolicy::sequential)
{
}

CudaHierarchicalL1AnnIndex::CudaHierarchicalL1AnnIndex(
    const DenseMatrix& input, std::size_t repetitions,
    std::size_t projection_dimension, std::mt19937_64& random_engine, int device,
    ExecutionPolicy probability_execution_policy)
    : CudaHierarchicalL1AnnIndex(input,
                                 l1_sample(input, repetitions, projection_dimension,
                                           random_engine, device,
                                           probability_execution_policy),
                                 projection_dimension, random_engine, device)
{
}

CudaHierarchicalL1AnnIndex::CudaHierarchicalL1AnnIndex(
    const DenseMatrix& input, std::span<const double> importance_probabilities,
    std::size_t repetitions, std::size_t projection_dimension,
    std::mt19937_64& random_engine, int device)
    : CudaHierarchicalL1AnnIndex(
          input,
          probabilities_sample(input, importance_probabilities, repetitions,
                               projection_dimension, random_engine,
                               "CudaHierarchicalL1AnnIndex",
                               [](std::span<const double> p, std::size_t t,
                                  std::mt19937_64& e) {
                                   return build_l1_importance_sample(p, t, e);
                               }),
          projection_dimension, random_engine, device)
{
}

CudaHierarchicalL1AnnIndex::CudaHierarchicalL1AnnIndex(
    const DenseMatrix& input, CoordinateSample importance_sample,
    std::size_t projection_dimension, std::mt19937_64& random_engine, int device)
    : implementation_(std::make_unique<Impl>())
{
    implementation_->attach(create_hierarchy(UHA_L1, input, importance_sample,
                                             projection_dimension, random_engine,
                                             device, "CudaHierarchicalL1AnnIndex"),
                            input.cols());
}

CudaHierarchicalL1AnnIndex::CudaHierarchicalL1AnnIndex(
    CudaHierarchicalL1AnnIndex&&) noexcept = default;
CudaHierarchicalL1AnnIndex&
CudaHierarchicalL1AnnIndex::operator=(CudaHierarchicalL1AnnIndex&&) noexcept = default;
CudaHierarchicalL1AnnIndex::~CudaHierarchicalL1AnnIndex() = default;

CudaHierarchicalL1AnnIndex::QueryWorkspace
CudaHierarchicalL1AnnIndex::make_query_workspace(std::size_t maximum_batch_size) const
{
    auto ws = std::make_unique<QueryWorkspace::Impl>();
    ws->attach(*implementation_, implementation_.get(), maximum_batch_size);
    return QueryWorkspace(std::move(ws));
}

std::size_t CudaHierarchicalL1AnnIndex::query(std::span<const float> query,
                                              QueryWorkspace& workspace,
                                              CudaHierarchicalL1QueryStrategy strategy) const
{
    std::size_t output = 0;
    query_batch(query, 1, std::span<std::size_t>(&output, 1), workspace, strategy);
    return output;
}

void CudaHierarchicalL1AnnIndex::query_batch(std::span<const float> queries,
                                             std::size_t query_count,
                                             std::span<std::size_t> output,
                                             QueryWorkspace& workspace,
                                             CudaHierarchicalL1QueryStrategy strategy) const
{
    if (strategy != CudaHierarchicalL1QueryStrategy::direct &&
        strategy != CudaHierarchicalL1QueryStrategy::gemm) {
        throw std::invalid_argument("unknown CUDA hierarchical L1 query strategy");
    }
    // both strategies only choose how the projection is computed; the engine
    // answers both with its certified path
    engine::facade_query(*implementation_, workspace.implementation_.get(),
                         implementation_.get(), queries, query_count, output,
                         UHA_DIRECT, "hierarchical L1", true);
}

IndexSpaceUsage CudaHierarchicalL1AnnIndex::space_usage() const noexcept
{
    return implementation_->usage();
}

int CudaHierarchicalL1AnnIndex::device() const noexcept
{
    return implementation_->device;
}

const std::string& CudaHierarchicalL1AnnIndex::device_name() const noexcept
{
    return implementation_->device_name;
}

}  // namespace ultrahigh_ann
