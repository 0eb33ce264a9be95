// ORACLE — test infrastructure only. A C wrapper over the reference's own CPU
// classes, compiled by oracle/Makefile against the reference's headers and
// linked with its CPU sources into oracle/_ref/libref.so. Tests use it to pin
// the oracle restatement (oracle/uha_oracle.cpp) and the engine; bench.py's
// reference arm times it on the host cores. Nothing here runs on a GPU.
#include "ultrahigh_ann/coordinate_sampling/coordinate_sampling.hpp"
#include "ultrahigh_ann/coordinate_sampling/sampled_coordinate_l1_ann_index.hpp"
#include "ultrahigh_ann/coordinate_sampling/sampled_coordinate_l2_ann_index.hpp"
#include "ultrahigh_ann/core/dense_l2_scan_index.hpp"
#include "ultrahigh_ann/exact/l1/exact_l1_index.hpp"
#include "ultrahigh_ann/exact/l2/exact_l2_index.hpp"
#include "ultrahigh_ann/hnsvw25/l1/hierarchical/hierarchical_l1_ann_index.hpp"
#include "ultrahigh_ann/hnsvw25/l1/importance_sampling.hpp"
#include "ultrahigh_ann/hnsvw25/l2/hierarchical/hierarchical_l2_ann_index.hpp"
#include "ultrahigh_ann/hnsvw25/l2/importance_sampling.hpp"
#include "hnsvw25/l1/hierarchical/l1_hierarchical_projection.hpp"
#include "hnsvw25/l2/hierarchical/l2_hierarchical_projection.hpp"
#include "ultrahigh_ann/datasets/representative_query_dataset.hpp"
#include "ultrahigh_ann/io/importance_probability_io.hpp"
#include "ultrahigh_ann/io/sha256.hpp"
#include "benchmarks/benchmark_setup.hpp"

#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <memory>
#include <cstring>
#include <exception>
#include <mutex>
#include <random>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

using namespace ultrahigh_ann;

namespace {

thread_local std::string g_error;

// 0 ok; 1 invalid_argument; 2 length_error; 3 runtime_error;
// 4 overflow_error; 5 out_of_range; 6 domain_error; 7 other
template <typename F>
int guarded(F&& f)
{
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return 1;
    } catch (const std::length_error& e) {
        g_error = e.what();
        return 2;
    } catch (const std::overflow_error& e) {
        g_error = e.what();
        return 4;
    } catch (const std::out_of_range& e) {
        g_error = e.what();
        return 5;
    } catch (const std::domain_error& e) {
        g_error = e.what();
        return 6;
    } catch (const std::runtime_error& e) {
        g_error = e.what();
        return 3;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 7;
    }
}

DenseMatrix matrix(const float* v, uint64_t r, uint64_t d)
{
    return DenseMatrix(std::vector<float>(v, v + r * d), r, d);
}

CoordinateSample sample_of(const uint64_t* cols, const uint64_t* mult,
                           const double* invp, uint64_t k)
{
    CoordinateSample s;
    for (uint64_t i = 0; i < k; ++i) {
        s.columns.push_back(SampledColumn{cols[i], mult[i], invp[i]});
    }
    return s;
}

// Runs body(begin, end) over [0, n) on `threads` std::threads.
template <typename F>
void split(uint64_t n, int threads, F body)
{
    threads = std::max(1, threads);
    std::vector<std::thread> pool;
    std::exception_ptr error;
    std::mutex m;
    const uint64_t per = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const uint64_t b = std::min(n, t * per);
        const uint64_t e = std::min(n, b + per);
        if (b >= e) {
            break;
        }
        pool.emplace_back([&, b, e] {
            try {
                body(b, e);
            } catch (...) {
                std::lock_guard<std::mutex> g(m);
                error = std::current_exception();
            }
        });
    }
    for (auto& th : pool) {
        th.join();
    }
    if (error) {
        std::rethrow_exception(error);
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void)
{
    return g_error.c_str();
}

// A persistent reference exact index (for timing: the matrix copy stays out of
// the timed calls). metric 0: ExactL2Index, 1: ExactL1Index.
struct RefExact {
    DenseMatrix matrix;
    std::unique_ptr<ExactL2Index> l2;
    std::unique_ptr<ExactL1Index> l1;
};

void* ref_exact_create(int metric, const float* rows, uint64_t r, uint64_t d)
{
    try {
        auto h = std::make_unique<RefExact>();
        h->matrix = matrix(rows, r, d);
        if (metric == 0) {
            h->l2 = std::make_unique<ExactL2Index>(h->matrix);
        } else {
            h->l1 = std::make_unique<ExactL1Index>(h->matrix);
        }
        return h.release();
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void ref_exact_destroy(void* handle)
{
    delete static_cast<RefExact*>(handle);
}

// L2: query_batch with parallel_queries on `threads` OpenMP threads (sequential
// when threads == 1); L1: query() on `threads` std::threads.
int ref_exact_query(void* handle, const float* queries, uint64_t n,
                    int threads, uint64_t* out)
{
    return guarded([&] {
        auto* h = static_cast<RefExact*>(handle);
        const uint64_t d = h->matrix.cols();
        if (h->l2) {
            omp_set_num_threads(std::max(1, threads));
            std::vector<std::size_t> o(n);
            h->l2->query_batch(std::span<const float>(queries, n * d), n, o,
                               threads > 1 ? CpuDenseL2QueryStrategy::parallel_queries
                                           : CpuDenseL2QueryStrategy::sequential);
            std::copy(o.begin(), o.end(), out);
        } else {
            split(n, threads, [&](uint64_t b, uint64_t e) {
                for (uint64_t q = b; q < e; ++q) {
                    out[q] = h->l1->query(std::span<const float>(queries + q * d, d));
                }
            });
        }
    });
}

// L2 only: the queries in calls of `batch` queries each, every call a
// query_batch with CpuDenseL2QueryStrategy::automatic on `threads` OpenMP
// threads -- the reference's own choice of parallel dimension for that batch
// size (src/core/dense_l2_scan_index.cpp:82-101: parallel_representatives for
// one query, parallel_queries once the batch reaches half the threads).
int ref_exact_query_batched(void* handle, const float* queries, uint64_t n,
                            uint64_t batch, int threads, uint64_t* out)
{
    return guarded([&] {
        auto* h = static_cast<RefExact*>(handle);
        if (!h->l2) {
            throw std::invalid_argument("ref_exact_query_batched serves L2 indexes");
        }
        const uint64_t d = h->matrix.cols();
        omp_set_num_threads(std::max(1, threads));
        const uint64_t b = std::max<uint64_t>(1, batch);
        std::vector<std::size_t> o(b);
        for (uint64_t s = 0; s < n; s += b) {
            const uint64_t m = std::min(b, n - s);
            h->l2->query_batch(std::span<const float>(queries + s * d, m * d), m,
                               std::span<std::size_t>(o.data(), m),
                               CpuDenseL2QueryStrategy::automatic);
            std::copy(o.begin(), o.begin() + m, out + s);
        }
    });
}

// build_coordinate_sample; engine state after sampling is written to state_out.
int ref_sample(const double* probs, uint64_t d, uint64_t repetitions,
               uint64_t seed, uint64_t* cols, uint64_t* mult, double* invp,
               uint64_t* k, char* state_out, uint64_t state_capacity)
{
    return guarded([&] {
        std::mt19937_64 engine(seed);
        const CoordinateSample s = build_coordinate_sample(
            std::span<const double>(probs, d), repetitions, engine);
        *k = s.columns.size();
        for (uint64_t i = 0; i < s.columns.size(); ++i) {
            cols[i] = s.columns[i].source_column;
            mult[i] = s.columns[i].multiplicity;
            invp[i] = s.columns[i].inverse_probability;
        }
        if (state_out != nullptr) {
            std::ostringstream os;
            os << engine;
            const std::string st = os.str();
            if (st.size() + 1 <= state_capacity) {
                std::memcpy(state_out, st.c_str(), st.size() + 1);
            }
        }
    });
}

// policy: 0 sequential, 1 cpu_parallel
int ref_probabilities(int metric, const float* rows, uint64_t r, uint64_t d,
                      int policy, double* out)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        const ExecutionPolicy p =
            policy == 0 ? ExecutionPolicy::sequential : ExecutionPolicy::cpu_parallel;
        const std::vector<double> v = metric == 0
                                          ? compute_l2_importance_probabilities(m, p)
                                          : compute_l1_importance_probabilities(m, p);
        std::copy(v.begin(), v.end(), out);
    });
}

// ExactL2Index::query_batch; strategy: 0 sequential, 1 parallel_queries
int ref_exact_l2(const float* rows, uint64_t r, uint64_t d,
                 const float* queries, uint64_t n, int strategy, uint64_t* out)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        const ExactL2Index index(m);
        std::vector<std::size_t> o(n);
        index.query_batch(std::span<const float>(queries, n * d), n, o,
                          strategy == 0 ? CpuDenseL2QueryStrategy::sequential
                                        : CpuDenseL2QueryStrategy::parallel_queries);
        std::copy(o.begin(), o.end(), out);
    });
}

// ExactL1Index::query from `threads` threads over disjoint query ranges
int ref_exact_l1(const float* rows, uint64_t r, uint64_t d,
                 const float* queries, uint64_t n, int threads, uint64_t* out)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        const ExactL1Index index(m);
        split(n, threads, [&](uint64_t b, uint64_t e) {
            for (uint64_t q = b; q < e; ++q) {
                out[q] = index.query(std::span<const float>(queries + q * d, d));
            }
        });
    });
}

// SampledCoordinateL2AnnIndex(input, CoordinateSample)::query_batch
int ref_sampled_l2(const float* rows, uint64_t r, uint64_t d,
                   const uint64_t* cols, const uint64_t* mult,
                   const double* invp, uint64_t k, const float* queries,
                   uint64_t n, int strategy, uint64_t* out)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        const SampledCoordinateL2AnnIndex index(m, sample_of(cols, mult, invp, k));
        std::vector<std::size_t> o(n);
        index.query_batch(std::span<const float>(queries, n * d), n, o,
                          strategy == 0 ? CpuDenseL2QueryStrategy::sequential
                                        : CpuDenseL2QueryStrategy::parallel_queries);
        std::copy(o.begin(), o.end(), out);
    });
}

// SampledCoordinateL1AnnIndex(input, CoordinateSample)::query on threads
int ref_sampled_l1(const float* rows, uint64_t r, uint64_t d,
                   const uint64_t* cols, const uint64_t* mult,
                   const double* invp, uint64_t k, const float* queries,
                   uint64_t n, int threads, uint64_t* out)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        const SampledCoordinateL1AnnIndex index(m, sample_of(cols, mult, invp, k));
        split(n, threads, [&](uint64_t b, uint64_t e) {
            for (uint64_t q = b; q < e; ++q) {
                out[q] = index.query(std::span<const float>(queries + q * d, d));
            }
        });
    });
}

// Hierarchical{L2,L1}AnnIndex(input, probabilities, repetitions, p, engine)
// seeded with `seed`; queries answered with query() on `threads` threads.
// The engine state after construction is written to state_out.
int ref_hierarchical(int metric, const float* rows, uint64_t r, uint64_t d,
                     const double* probs, uint64_t repetitions, uint64_t p,
                     uint64_t seed, const float* queries, uint64_t n,
                     int threads, uint64_t* out, char* state_out,
                     uint64_t state_capacity)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        std::mt19937_64 engine(seed);
        const std::span<const double> pr(probs, d);
        auto run = [&](const auto& index) {
            split(n, threads, [&](uint64_t b, uint64_t e) {
                auto ws = index.make_query_workspace();
                for (uint64_t q = b; q < e; ++q) {
                    out[q] =
                        index.query(std::span<const float>(queries + q * d, d), ws);
                }
            });
        };
        if (metric == 0) {
            const HierarchicalL2AnnIndex index(m, pr, repetitions, p, engine);
            run(index);
        } else {
            const HierarchicalL1AnnIndex index(m, pr, repetitions, p, engine);
            run(index);
        }
        if (state_out != nullptr) {
            std::ostringstream os;
            os << engine;
            const std::string st = os.str();
            if (st.size() + 1 <= state_capacity) {
                std::memcpy(state_out, st.c_str(), st.size() + 1);
            }
        }
    });
}

// detail::build_l{2,1}_hierarchical_projection: the binary64 projection matrix
// (p x k) and projected representatives (r x p).
int ref_projection(int metric, const float* rows, uint64_t r, uint64_t d,
                   const uint64_t* cols, const uint64_t* mult,
                   const double* invp, uint64_t k, uint64_t p,
                   const char* state, uint64_t seed, double* matrix_out,
                   double* reps_out)
{
    return guarded([&] {
        const DenseMatrix m = matrix(rows, r, d);
        std::mt19937_64 engine(seed);
        if (state != nullptr) {
            std::istringstream is{std::string(state)};
            is >> engine;
        }
        if (metric == 0) {
            auto proj = detail::build_l2_hierarchical_projection(
                m, sample_of(cols, mult, invp, k), p, engine);
            std::copy(proj.jl_matrix.values().begin(), proj.jl_matrix.values().end(),
                      matrix_out);
            std::copy(proj.projected_representatives.values().begin(),
                      proj.projected_representatives.values().end(), reps_out);
        } else {
            auto proj = detail::build_l1_hierarchical_projection(
                m, sample_of(cols, mult, invp, k), p, engine);
            std::copy(proj.cauchy_matrix.values().begin(),
                      proj.cauchy_matrix.values().end(), matrix_out);
            std::copy(proj.projected_representatives.values().begin(),
                      proj.projected_representatives.values().end(), reps_out);
        }
    });
}

// ---- data files (src/io/*.cpp, src/datasets/representative_query_dataset.cpp)

int ref_sha256_file(const char* path, uint8_t* out)
{
    return guarded([&] {
        const auto d = ultrahigh_ann::io::sha256_file(path);
        std::memcpy(out, d.data(), d.size());
    });
}

// kind: 0 = L2, 1 = L1 (the engine's uha_metric values)
int ref_probabilities_save(const char* path, int kind, uint64_t reps, const uint8_t* sha,
                           const double* probs, uint64_t n)
{
    return guarded([&] {
        ultrahigh_ann::io::Sha256Digest d{};
        std::memcpy(d.data(), sha, d.size());
        ultrahigh_ann::io::save_importance_probabilities(
            path,
            kind == 1 ? ultrahigh_ann::io::ImportanceProbabilityKind::l1
                      : ultrahigh_ann::io::ImportanceProbabilityKind::l2,
            reps, d, std::span<const double>(probs, n));
    });
}

int ref_probabilities_load(const char* path, int* kind, uint64_t* reps, uint8_t* sha,
                           double* probs, uint64_t capacity, uint64_t* n)
{
    return guarded([&] {
        const auto f = ultrahigh_ann::io::load_importance_probabilities(path);
        *kind = f.kind == ultrahigh_ann::io::ImportanceProbabilityKind::l1 ? 1 : 0;
        *reps = f.representative_count;
        std::memcpy(sha, f.representatives_sha256.data(), 32);
        *n = f.probabilities.size();
        if (probs != nullptr) {
            if (capacity < f.probabilities.size()) {
                throw std::length_error("capacity");
            }
            std::memcpy(probs, f.probabilities.data(), f.probabilities.size() * sizeof(double));
        }
    });
}

int ref_npy_f32(const char* path, float* out, uint64_t capacity, uint64_t* rows,
                uint64_t* cols)
{
    return guarded([&] {
        const DenseMatrix m = ultrahigh_ann::load_float_matrix_npy(path);
        *rows = m.rows();
        *cols = m.cols();
        if (out != nullptr) {
            if (capacity < m.rows() * m.cols()) {
                throw std::length_error("capacity");
            }
            const auto v = m.values();
            std::copy(v.begin(), v.end(), out);
        }
    });
}

int ref_npy_u16(const char* path, uint64_t* out, uint64_t capacity, uint64_t* count)
{
    return guarded([&] {
        const auto v = ultrahigh_ann::load_label_vector_npy(path);
        *count = v.size();
        if (out != nullptr) {
            if (capacity < v.size()) {
                throw std::length_error("capacity");
            }
            for (size_t i = 0; i < v.size(); ++i) {
                out[i] = v[i];
            }
        }
    });
}

// ---- benchmark setup v2 (src/benchmarks/benchmark_setup.cpp): the parsed
// setup as JSON text
namespace {
std::string json_str(const std::string& v)
{
    std::string o = "\"";
    for (char c : v) {
        if (c == '"' || c == '\\') {
            o.push_back('\\');
        }
        o.push_back(c);
    }
    return o + "\"";
}
}  // namespace

int ref_parse_setup(const char* path, char* out, uint64_t capacity, uint64_t* length)
{
    return guarded([&] {
        namespace b = ultrahigh_ann::benchmark;
        const b::BenchmarkSetup s = b::load_benchmark_setup(path);
        std::ostringstream o;
        o << "{\"setup_path\":" << json_str(s.setup_path.string())
          << ",\"dataset_directory\":" << json_str(s.dataset_directory.string())
          << ",\"representatives_path\":" << json_str(s.representatives_path.string())
          << ",\"representative_labels_path\":"
          << json_str(s.representative_labels_path.string())
          << ",\"queries_path\":" << json_str(s.queries_path.string())
          << ",\"query_labels_path\":" << json_str(s.query_labels_path.string())
          << ",\"json_output_path\":" << json_str(s.json_output_path.string())
          << ",\"csv_output_path\":" << json_str(s.csv_output_path.string())
          << ",\"probabilities_path\":"
          << (s.probabilities_path ? json_str(s.probabilities_path->string()) : "null")
          << ",\"distance\":" << json_str(std::string(b::distance_name(s.distance)))
          << ",\"probability_policy\":"
          << json_str(std::string(b::probability_policy_name(s.probability_policy)))
          << ",\"diagnostics\":"
          << json_str(std::string(b::diagnostic_mode_name(s.diagnostics)))
          << ",\"maximum_queries\":" << s.maximum_queries << ",\"warmups\":" << s.warmups
          << ",\"trials\":" << s.trials << ",\"batch_sizes\":[";
        for (size_t i = 0; i < s.batch_sizes.size(); ++i) {
            o << (i ? "," : "") << s.batch_sizes[i];
        }
        o << "],\"device\":" << s.device << ",\"reference_run\":" << json_str(s.reference_run)
          << ",\"runs\":[";
        for (size_t r = 0; r < s.runs.size(); ++r) {
            const b::BenchmarkRun& run = s.runs[r];
            o << (r ? "," : "") << "{\"name\":" << json_str(run.name)
              << ",\"index\":" << json_str(std::string(b::index_name(run.index)))
              << ",\"backend\":" << json_str(std::string(b::backend_name(run.backend)))
              << ",\"strategy\":" << json_str(std::string(b::strategy_name(run.strategy)))
              << ",\"repetitions\":" << run.repetitions << ",\"seed\":" << run.seed
              << ",\"projection_dimension\":" << run.projection_dimension
              << ",\"batch_sizes\":[";
            for (size_t i = 0; i < run.batch_sizes.size(); ++i) {
                o << (i ? "," : "") << run.batch_sizes[i];
            }
            o << "],\"warmups\":" << run.warmups << ",\"trials\":" << run.trials << "}";
        }
        o << "]}";
        const std::string text = o.str();
        *length = text.size();
        if (out != nullptr && capacity > text.size()) {
            std::memcpy(out, text.c_str(), text.size() + 1);
        }
    });
}

}  // extern "C"
