// compute_l{2,1}_importance_probabilities_gpu and l{2,1}_gpu_backend_available
// over the engine's C ABI. Replaces the reference translation units
// src/hnsvw25/l2/cuda_importance_sampling.cu and
// src/hnsvw25/l1/cuda_importance_sampling.cu (declarations:
// include/ultrahigh_ann/hnsvw25/l{2,1}/importance_sampling.hpp). Pair
// distances and the normalisation are binary64 on the device.
#include "ultrahigh_ann/hnsvw25/l1/importance_sampling.hpp"
#include "ultrahigh_ann/hnsvw25/l2/importance_sampling.hpp"

#include "shim_support.hpp"

#include <stdexcept>
#include <string>
#include <vector>

namespace ultrahigh_ann {
namespace {

template <typename Result, typename Backend>
Result run(uha_metric metric, const DenseMatrix& representatives, int device,
           std::size_t pair_chunks, Backend backend, bool gram)
{
    if (pair_chunks == 0) {
        throw std::invalid_argument("GPU pair chunk count must be positive");
    }
    Result result;
    result.probabilities.assign(representatives.cols(), 0.0);
    uha_probability_report report{};
    engine::check(uha_importance_probabilities(
        device, metric, representatives.values().data(), representatives.rows(),
        representatives.cols(), gram ? UHA_PAIRS_GRAM : UHA_PAIRS_DIRECT,
        pair_chunks, result.probabilities.data(), &report));
    uha_device_info info{};
    engine::check(uha_device_info_get(device, &info));
    result.device_name = info.device_name;
    result.device = device;
    result.distance_backend = backend;
    result.pair_count = report.pair_count;
    result.pair_chunks = report.pair_chunks;
    result.device_working_set_bytes = report.device_working_set_bytes;
    result.timings.host_to_device_ms = report.host_to_device_ms;
    result.timings.inverse_distance_ms = report.inverse_distance_ms;
    result.timings.coordinate_maximum_ms = report.coordinate_maximum_ms;
    result.timings.device_to_host_ms = report.device_to_host_ms;
    result.timings.total_ms = report.total_ms;
    return result;
}

}  // namespace

bool l2_gpu_backend_available() noexcept
{
    return uha_cuda_available() != 0;
}

bool l1_gpu_backend_available() noexcept
{
    return uha_cuda_available() != 0;
}

L2GpuProbabilityResult compute_l2_importance_probabilities_gpu(
    const DenseMatrix& representatives, int device, std::size_t pair_chunks,
    L2GpuDistanceBackend distance_backend)
{
    if (distance_backend != L2GpuDistanceBackend::direct &&
        distance_backend != L2GpuDistanceBackend::cublas) {
        throw std::invalid_argument("unknown L2 GPU distance backend");
    }
    // The reference's cuBLAS backend is the Gram-matrix identity with
    // cancellation refinement; the engine's own binary64 Gram kernel does it.
    return run<L2GpuProbabilityResult>(UHA_L2, representatives, device, pair_chunks,
                                       distance_backend,
                                       distance_backend == L2GpuDistanceBackend::cublas);
}

L1GpuProbabilityResult compute_l1_importance_probabilities_gpu(
    const DenseMatrix& representatives, int device, std::size_t pair_chunks,
    L1GpuDistanceBackend distance_backend)
{
    if (distance_backend != L1GpuDistanceBackend::direct) {
        throw std::invalid_argument("unknown L1 GPU distance backend");
    }
    return run<L1GpuProbabilityResult>(UHA_L1, representatives, device, pair_chunks,
                                       distance_backend, false);
}

}  // namespace ultrahigh_ann
