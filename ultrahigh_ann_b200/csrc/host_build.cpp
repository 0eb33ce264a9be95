// Host-side index build: the coordinate sample, the hierarchical projection
// matrices and the CPU-policy importance probabilities.
//
// These stay on the host on purpose. The index set I and the projection
// coefficients are defined by std::mt19937_64 together with libstdc++'s
// std::binomial_distribution / std::cauchy_distribution, whose algorithms are
// implementation-defined; drawing the same distributions from the same engine
// in the same order is what makes I identical to the reference's for a given
// seed (src/coordinate_sampling/coordinate_sampling.cpp:14-45,
// src/hnsvw25/l2/hierarchical/l2_hierarchical_projection.cpp:53-77,
// src/hnsvw25/l1/hierarchical/l1_hierarchical_projection.cpp:54-77).
#include "common.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

struct uha_rng {
    std::mt19937_64 engine;
};

namespace uha {

thread_local std::string g_last_error;

void set_last_error(const char* message)
{
    g_last_error = message == nullptr ? "" : message;
}

}  // namespace uha

using uha::fail;
using uha::guarded;

extern "C" const char* uha_last_error(void)
{
    return uha::g_last_error.c_str();
}

extern "C" uha_status uha_rng_create(uint64_t seed, uha_rng** out)
{
    return guarded([&] {
        if (out == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "output pointer must not be null");
        }
        *out = new uha_rng{std::mt19937_64(seed)};
    });
}

extern "C" void uha_rng_destroy(uha_rng* rng)
{
    delete rng;
}

extern "C" uha_status uha_rng_state(const uha_rng* rng, char* buffer,
                                    uint64_t capacity, uint64_t* length)
{
    return guarded([&] {
        if (rng == nullptr || length == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "engine and length must not be null");
        }
        std::ostringstream stream;
        stream << rng->engine;
        const std::string text = stream.str();
        *length = text.size() + 1;
        if (buffer != nullptr) {
            if (capacity < text.size() + 1) {
                fail(UHA_LENGTH_ERROR, "engine state buffer is too small");
            }
            std::memcpy(buffer, text.c_str(), text.size() + 1);
        }
    });
}

extern "C" uha_status uha_rng_set_state(uha_rng* rng, const char* state)
{
    return guarded([&] {
        if (rng == nullptr || state == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "engine and state must not be null");
        }
        std::istringstream stream{std::string(state)};
        std::mt19937_64 engine;
        stream >> engine;
        if (stream.fail()) {
            fail(UHA_INVALID_ARGUMENT, "malformed engine state");
        }
        rng->engine = engine;
    });
}

extern "C" uha_status uha_sample_coordinates(const double* probabilities,
                                             uint64_t dimension,
                                             uint64_t repetitions,
                                             uha_rng* rng, uint64_t* columns,
                                             uint64_t* multiplicities,
                                             double* inverse_probabilities,
                                             uint64_t* sample_size)
{
    return guarded([&] {
        if (rng == nullptr || sample_size == nullptr ||
            (dimension != 0 && (probabilities == nullptr || columns == nullptr ||
                                multiplicities == nullptr ||
                                inverse_probabilities == nullptr))) {
            fail(UHA_INVALID_ARGUMENT, "sampling arguments must not be null");
        }
        // Columns are validated in order while drawing, as the reference
        // does, so a failed call has consumed the draws of the columns
        // before the invalid one.
        uint64_t k = 0;
        for (uint64_t column = 0; column < dimension; ++column) {
            const double p = probabilities[column];
            if (!std::isfinite(p)) {
                fail(UHA_DOMAIN_ERROR, "sampling probability must be finite");
            }
            if (p < 0.0 || p > 1.0) {
                fail(UHA_DOMAIN_ERROR, "invalid sampling probability");
            }
            if (p == 0.0 || repetitions == 0) {
                continue;
            }
            std::binomial_distribution<std::size_t> trials(
                static_cast<std::size_t>(repetitions), p);
            const std::size_t m = trials(rng->engine);
            if (m != 0) {
                columns[k] = column;
                multiplicities[k] = m;
                inverse_probabilities[k] = 1.0 / p;
                ++k;
            }
        }
        *sample_size = k;
    });
}

namespace {

void validate_sample_weights(const uint64_t* multiplicities,
                             const double* inverse_probabilities, uint64_t k)
{
    for (uint64_t i = 0; i < k; ++i) {
        if (multiplicities[i] == 0 || !std::isfinite(inverse_probabilities[i]) ||
            inverse_probabilities[i] <= 0.0) {
            fail(UHA_INVALID_ARGUMENT,
                 "sampled columns require positive finite weights");
        }
    }
}

}  // namespace

extern "C" uha_status uha_jl_matrix(const uint64_t* multiplicities,
                                    const double* inverse_probabilities,
                                    uint64_t sample_size,
                                    uint64_t projection_dimension,
                                    uha_rng* rng, double* out)
{
    return guarded([&] {
        if (rng == nullptr ||
            (sample_size != 0 && projection_dimension != 0 &&
             (multiplicities == nullptr || inverse_probabilities == nullptr ||
              out == nullptr))) {
            fail(UHA_INVALID_ARGUMENT, "projection arguments must not be null");
        }
        if (projection_dimension == 0) {
            fail(UHA_INVALID_ARGUMENT,
                 "projection_dimension has to be a positive integer");
        }
        uha::checked_mul(projection_dimension, sample_size, "JL matrix");
        validate_sample_weights(multiplicities, inverse_probabilities,
                                sample_size);
        const double row_scaling =
            1.0 / std::sqrt(static_cast<double>(projection_dimension));
        uint64_t index = 0;
        for (uint64_t row = 0; row < projection_dimension; ++row) {
            for (uint64_t i = 0; i < sample_size; ++i) {
                std::binomial_distribution<std::size_t> positive_signs(
                    static_cast<std::size_t>(multiplicities[i]), 0.5);
                const std::size_t positives = positive_signs(rng->engine);
                const double signed_sum =
                    2.0 * static_cast<double>(positives) -
                    static_cast<double>(multiplicities[i]);
                const double coefficient = signed_sum *
                                           std::sqrt(inverse_probabilities[i]) *
                                           row_scaling;
                if (!std::isfinite(coefficient)) {
                    fail(UHA_OVERFLOW_ERROR,
                         "JL projection coefficient is not finite");
                }
                out[index++] = coefficient;
            }
        }
    });
}

extern "C" uha_status uha_cauchy_matrix(const uint64_t* multiplicities,
                                        const double* inverse_probabilities,
                                        uint64_t sample_size,
                                        uint64_t projection_dimension,
                                        uha_rng* rng, double* out)
{
    return guarded([&] {
        if (rng == nullptr ||
            (sample_size != 0 && projection_dimension != 0 &&
             (multiplicities == nullptr || inverse_probabilities == nullptr ||
              out == nullptr))) {
            fail(UHA_INVALID_ARGUMENT, "projection arguments must not be null");
        }
        if (projection_dimension == 0) {
            fail(UHA_INVALID_ARGUMENT,
                 "projection_dimension has to be a positive integer");
        }
        uha::checked_mul(projection_dimension, sample_size, "Cauchy matrix");
        validate_sample_weights(multiplicities, inverse_probabilities,
                                sample_size);
        std::cauchy_distribution<double> cauchy(0.0, 1.0);
        uint64_t index = 0;
        for (uint64_t row = 0; row < projection_dimension; ++row) {
            for (uint64_t i = 0; i < sample_size; ++i) {
                const double coefficient =
                    cauchy(rng->engine) * inverse_probabilities[i] *
                    static_cast<double>(multiplicities[i]);
                if (!std::isfinite(coefficient)) {
                    fail(UHA_OVERFLOW_ERROR,
                         "Cauchy projection coefficient is not finite");
                }
                out[index++] = coefficient;
            }
        }
    });
}

// Gaussian JL entries with the variance of the aggregated Rademacher entries,
// rounded to binary32 (the matrix is a binary32 matrix held in binary64, so the
// binary64 projection path is exact with respect to it).
extern "C" uha_status uha_gaussian_jl_matrix(const uint64_t* multiplicities,
                                             const double* inverse_probabilities,
                                             uint64_t sample_size,
                                             uint64_t projection_dimension,
                                             uha_rng* rng, double* out)
{
    return guarded([&] {
        if (rng == nullptr ||
            (sample_size != 0 && projection_dimension != 0 &&
             (multiplicities == nullptr || inverse_probabilities == nullptr ||
              out == nullptr))) {
            fail(UHA_INVALID_ARGUMENT, "projection arguments must not be null");
        }
        if (projection_dimension == 0) {
            fail(UHA_INVALID_ARGUMENT,
                 "projection_dimension has to be a positive integer");
        }
        uha::checked_mul(projection_dimension, sample_size, "Gaussian JL matrix");
        validate_sample_weights(multiplicities, inverse_probabilities,
                                sample_size);
        std::vector<double> scale(sample_size);
        for (uint64_t i = 0; i < sample_size; ++i) {
            scale[i] = std::sqrt(static_cast<double>(multiplicities[i]) *
                                 inverse_probabilities[i] /
                                 static_cast<double>(projection_dimension));
        }
        std::normal_distribution<double> normal(0.0, 1.0);
        uint64_t index = 0;
        for (uint64_t row = 0; row < projection_dimension; ++row) {
            for (uint64_t i = 0; i < sample_size; ++i) {
                const float coefficient =
                    static_cast<float>(normal(rng->engine) * scale[i]);
                if (!std::isfinite(coefficient)) {
                    fail(UHA_OVERFLOW_ERROR,
                         "Gaussian JL projection coefficient is not finite");
                }
                out[index++] = coefficient;
            }
        }
    });
}

// Importance probabilities on the host cores with the reference CPU policies'
// arithmetic (src/hnsvw25/l2/importance_sampling.cpp:19-45,
// src/hnsvw25/l1/importance_sampling.cpp:19-47): binary64 pair distances (L2
// sequential sum of squares; L1 in std::transform_reduce's grouping of four),
// then the per-column maximum of min(1, d_j^2 / ||a-b||^2) or |d_j| / ||a-b||_1.
// First rows are split over `threads` threads with private maxima; the maximum
// is exact, so the result is bit-identical to the sequential loop.

namespace {

double pair_l2(const float* a, const float* b, uint64_t d)
{
    double s = 0.0;
    for (uint64_t i = 0; i < d; ++i) {
        const double diff = static_cast<double>(a[i]) - static_cast<double>(b[i]);
        s += diff * diff;
    }
    return s;
}

double pair_l1(const float* a, const float* b, uint64_t d)
{
    auto t = [&](uint64_t i) {
        return std::abs(static_cast<double>(a[i]) - static_cast<double>(b[i]));
    };
    double init = 0.0;
    uint64_t i = 0;
    for (; d - i >= 4; i += 4) {
        const double v1 = t(i) + t(i + 1);
        const double v2 = t(i + 2) + t(i + 3);
        init = init + (v1 + v2);
    }
    for (; i < d; ++i) {
        init = init + t(i);
    }
    return init;
}

}  // namespace

extern "C" uha_status uha_importance_probabilities_host(
    uha_metric metric, const float* rows, uint64_t row_count,
    uint64_t dimension, int threads, double* out)
{
    return guarded([&] {
        if (metric != UHA_L2 && metric != UHA_L1) {
            fail(UHA_INVALID_ARGUMENT, "unknown metric");
        }
        if ((rows == nullptr && row_count * dimension != 0) ||
            (out == nullptr && dimension != 0)) {
            fail(UHA_INVALID_ARGUMENT, "matrix and output must not be null");
        }
        uha::checked_mul(row_count, dimension, "representative matrix");
        for (uint64_t i = 0; i < row_count * dimension; ++i) {
            if (!std::isfinite(rows[i])) {
                fail(UHA_INVALID_ARGUMENT, "representatives must be finite");
            }
        }
        std::fill(out, out + dimension, 0.0);
        if (row_count < 2 || dimension == 0) {
            return;
        }
        const int workers = static_cast<int>(std::max<uint64_t>(
            1, std::min<uint64_t>(static_cast<uint64_t>(std::max(1, threads)),
                                  row_count - 1)));
        std::vector<std::vector<double>> local(workers,
                                               std::vector<double>(dimension, 0.0));
        std::vector<std::thread> pool;
        for (int w = 0; w < workers; ++w) {
            pool.emplace_back([&, w] {
                std::vector<double>& m = local[w];
                for (uint64_t a = w; a + 1 < row_count; a += workers) {
                    const float* ra = rows + a * dimension;
                    for (uint64_t b = a + 1; b < row_count; ++b) {
                        const float* rb = rows + b * dimension;
                        const double dist = metric == UHA_L2
                                                ? pair_l2(ra, rb, dimension)
                                                : pair_l1(ra, rb, dimension);
                        if (dist == 0.0) {
                            continue;
                        }
                        const double inv = 1.0 / dist;
                        for (uint64_t j = 0; j < dimension; ++j) {
                            const double diff = static_cast<double>(ra[j]) -
                                                static_cast<double>(rb[j]);
                            const double v = metric == UHA_L2
                                                 ? std::min(1.0, diff * diff * inv)
                                                 : std::abs(diff) * inv;
                            m[j] = std::max(m[j], v);
                        }
                    }
                }
            });
        }
        for (auto& t : pool) {
            t.join();
        }
        for (const auto& m : local) {
            for (uint64_t j = 0; j < dimension; ++j) {
                out[j] = std::max(out[j], m[j]);
            }
        }
    });
}
