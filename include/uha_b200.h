/*
 * uha_b200.h — C ABI of the B200 query engine for the HNSVW importance-sampling
 * nearest-neighbour indexes (flat, hierarchical and exact; L1 and L2).
 *
 * Plain pointers and sizes only. Every entry point returns a uha_status; on
 * failure uha_last_error() holds a message for the calling thread. Status codes
 * map one-to-one onto the C++ exception types the reference API throws, so a
 * C++ binding can rethrow exactly what the reference would have thrown.
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the reference project root).
 */
#ifndef UHA_B200_H
#define UHA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Reference exception mapping:
 *   UHA_INVALID_ARGUMENT -> std::invalid_argument (shapes, capacity, foreign
 *                           workspace, non-finite rows or sampled query values)
 *   UHA_LENGTH_ERROR     -> std::length_error     (size overflow, grid limits)
 *   UHA_RUNTIME_ERROR    -> std::runtime_error    (CUDA failure, no device)
 *   UHA_OVERFLOW_ERROR   -> std::overflow_error   (non-finite projected results)
 *   UHA_OUT_OF_RANGE     -> std::out_of_range     (sampled column >= dimension)
 *   UHA_DOMAIN_ERROR     -> std::domain_error     (invalid sampling probability)
 *   UHA_LOGIC_ERROR      -> std::logic_error
 * (src/core/cuda_dense_l2_scan_index.cu:26-32 check_cuda; src/core/finite_values.hpp:12-66) */
typedef enum uha_status {
    UHA_OK = 0,
    UHA_INVALID_ARGUMENT = 1,
    UHA_LENGTH_ERROR = 2,
    UHA_RUNTIME_ERROR = 3,
    UHA_OVERFLOW_ERROR = 4,
    UHA_OUT_OF_RANGE = 5,
    UHA_DOMAIN_ERROR = 6,
    UHA_LOGIC_ERROR = 7
} uha_status;

typedef enum uha_metric {
    UHA_L2 = 0,
    UHA_L1 = 1
} uha_metric;

/* Query strategies. The first two keep the reference enumerator values of
 * CudaDenseL2QueryStrategy / CudaSampledCoordinateL2QueryStrategy /
 * CudaHierarchicalL{1,2}QueryStrategy (include/ultrahigh_ann/core/
 * cuda_dense_l2_scan_index.hpp:17-23); the precision forms are appended.
 *   UHA_DIRECT: binary32 scan on CUDA cores with a certified error bound per
 *     distance; queries whose winner is not certified are re-scored by
 *     replaying the reference CPU's binary64 operation sequence, so the
 *     returned index equals the reference CPU index on every query.
 *   UHA_GEMM: the reference's unrefined binary32 norm identity
 *     ||r||^2 + ||q||^2 - 2 r.q (L2 only; L1 treats it as DIRECT).
 *   UHA_GEMM_BF16_RERANK, UHA_GEMM_FP8_RERANK (exact, flat and
 *     hierarchical L2 indexes): rows and queries rounded to BF16, or to
 *     FP8-E4M3 with one scale per row and per query; the score matrix runs
 *     on the tensor cores with FP32 accumulation; the k rows with the
 *     smallest estimate ||r~||^2 - 2 r~.q~ (uha_workspace_set_candidates) are
 *     re-scored from the original rows (the reference CPU's binary64 terms,
 *     added in parallel, with a certified bound; near-ties replay the CPU's
 *     order). Hierarchies also project the queries on the tensor cores (the
 *     rounded p x k projection times the batch) and re-score by the
 *     reference's binary64 projected distance. The answer equals the
 *     reference CPU index whenever that row is among the k candidates. The
 *     low-precision copies are built on the first query that needs them.
 *   UHA_GEMM_BF16_RERANK_FP32, UHA_GEMM_FP8_RERANK_FP32 (exact and flat L2
 *     indexes): the same scores and candidates, re-scored in binary32 from
 *     the original rows with a certified bound; a query whose candidates'
 *     bounds overlap is settled without FP64 instructions (float-float
 *     distances, then emulated binary64 for the candidates they cannot
 *     separate), so the answer is again the reference CPU's whenever its
 *     row is among the candidates. */
typedef enum uha_strategy {
    UHA_DIRECT = 0,
    UHA_GEMM = 1,
    UHA_GEMM_BF16_RERANK = 2,
    UHA_GEMM_FP8_RERANK = 3,
    UHA_GEMM_BF16_RERANK_FP32 = 4,
    UHA_GEMM_FP8_RERANK_FP32 = 5
} uha_strategy;

typedef struct uha_index uha_index;
typedef struct uha_workspace uha_workspace;
typedef struct uha_rng uha_rng;

/* include/ultrahigh_ann/core/index_space_usage.hpp:9-14 */
typedef struct uha_space_usage {
    uint64_t index_payload_bytes;
    uint64_t query_workspace_payload_bytes;
    uint64_t unique_query_coordinates;
    uint64_t sampled_multiplicity;
} uha_space_usage;

/* include/ultrahigh_ann/core/cuda_runtime_info.hpp:9-18 */
typedef struct uha_device_info {
    int device;
    char device_name[256];
    int compute_capability_major;
    int compute_capability_minor;
    uint64_t total_global_memory_bytes;
    int compiled_runtime_version;
    int runtime_version;
    int driver_version;
} uha_device_info;

/* Per-query diagnostics of the last uha_query call on a workspace. */
typedef struct uha_query_stats {
    uint64_t query_count;
    uint64_t certified_queries;   /* winner certified by the binary32 bound */
    uint64_t replayed_queries;    /* winner settled by the binary64 replay */
    uint64_t kernel_launches;     /* kernels this library launched for the call */
    double scan_ms;               /* device time of the timed scan kernels */
    double device_ms;             /* device time from first enqueue to results */
    uint64_t timed_scans;         /* scan launches scan_ms covers */
} uha_query_stats;

/* GPU probability-build report (include/ultrahigh_ann/hnsvw25/l2/
 * importance_sampling.hpp:23-41, l1/importance_sampling.hpp:22-40). */
typedef struct uha_probability_report {
    uint64_t pair_count;
    uint64_t pair_chunks;     /* launches the pairs were split into */
    uint64_t device_working_set_bytes;
    double host_to_device_ms;
    double inverse_distance_ms;
    double coordinate_maximum_ms;
    double device_to_host_ms;
    double total_ms;
} uha_probability_report;

/* Message of the calling thread's last failed call ("" when none). */
const char* uha_last_error(void);

/* 1 when a usable CUDA device is visible, else 0.
 * Replaces cuda_dense_l2_scan_available() and its siblings
 * (include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:14). */
int uha_cuda_available(void);

/* Replaces cuda_runtime_info(int) (include/ultrahigh_ann/core/
 * cuda_runtime_info.hpp:22-23; src/core/cuda_runtime_info.cu:11-38).
 * UHA_RUNTIME_ERROR when the device is not usable. */
uha_status uha_device_info_get(int device, uha_device_info* out);

/* ---------------------------------------------------------------- indexes */

/* Exact (full-coordinate) scan over an r x d row-major float matrix.
 * Replaces CudaDenseL2ScanIndex(const DenseMatrix&, int)
 * (include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:47-48),
 * CudaDenseL1ScanIndex(const DenseMatrix&, int)
 * (include/ultrahigh_ann/core/cuda_dense_l1_scan_index.hpp:39-40) and the
 * CudaExactL{1,2}Index facades (include/ultrahigh_ann/exact/l2/
 * cuda_exact_l2_index.hpp:27-28, exact/l1/cuda_exact_l1_index.hpp:25-26).
 * The rows are copied; the caller keeps ownership of `rows`. */
uha_status uha_exact_index_create(int device, uha_metric metric,
                                  const float* rows, uint64_t row_count,
                                  uint64_t dimension, uha_index** out);

/* Weighted L1 scan sum_j w_j |r_j - q_j| with binary32 weights.
 * Replaces CudaDenseL1ScanIndex(const DenseMatrix&, std::span<const float>,
 * int) (include/ultrahigh_ann/core/cuda_dense_l1_scan_index.hpp:41-43). */
uha_status uha_weighted_l1_index_create(int device, const float* rows,
                                        uint64_t row_count, uint64_t dimension,
                                        const float* weights,
                                        uha_index** out);

/* Sampled-coordinate (flat) index from a coordinate sample
 * {columns[i], multiplicities[i], inverse_probabilities[i]}, i < k, kept in
 * ascending column order. The embedding (L2: rows scaled by
 * float(sqrt(mult * inv_p)); L1: unscaled rows and weights mult * inv_p) is
 * built on the device. Replaces CudaSampledCoordinateL{1,2}AnnIndex(
 * const DenseMatrix&, CoordinateSample, int)
 * (include/ultrahigh_ann/coordinate_sampling/cuda_sampled_coordinate_l2_ann_index.hpp:54-56,
 *  cuda_sampled_coordinate_l1_ann_index.hpp:48-50). */
uha_status uha_sampled_index_create(int device, uha_metric metric,
                                    const float* rows, uint64_t row_count,
                                    uint64_t dimension,
                                    const uint64_t* columns,
                                    const uint64_t* multiplicities,
                                    const double* inverse_probabilities,
                                    uint64_t sample_size, uha_index** out);

/* Hierarchical index: sampled coordinates plus a p x k binary64 projection
 * (Rademacher-JL for L2, Cauchy for L1) drawn on the host with the
 * reference's random sequence (uha_jl_matrix / uha_cauchy_matrix). Projected
 * rows are formed on the device in binary64 with the reference's summation
 * order. Replaces CudaHierarchicalL{1,2}AnnIndex(const DenseMatrix&,
 * CoordinateSample, std::size_t, std::mt19937_64&, int)
 * (include/ultrahigh_ann/hnsvw25/l2/hierarchical/cuda_hierarchical_l2_ann_index.hpp:70-73,
 *  l1/hierarchical/cuda_hierarchical_l1_ann_index.hpp:74-77). */
uha_status uha_hierarchical_index_create(int device, uha_metric metric,
                                         const float* rows,
                                         uint64_t row_count,
                                         uint64_t dimension,
                                         const uint64_t* columns,
                                         const uint64_t* multiplicities,
                                         const double* inverse_probabilities,
                                         uint64_t sample_size,
                                         const double* projection,
                                         uint64_t projection_dimension,
                                         uha_index** out);

/* A row-major matrix already resident on the index's device: row i starts
 * at element i * row_stride of `data` (row_stride >= columns). BF16 values
 * are decoded exactly to binary32, so an index built from them equals one
 * built from the host binary32 matrix of the decoded values. */
typedef enum uha_value_type {
    UHA_VALUES_F32 = 0,
    UHA_VALUES_BF16 = 1
} uha_value_type;

typedef struct uha_device_matrix {
    const void* data;
    uha_value_type type;
    uint64_t rows;
    uint64_t columns;
    uint64_t row_stride;
} uha_device_matrix;

/* The three index constructors above with the representative matrix read
 * on the device (no host copy of it is made or needed): only the sampled
 * columns are read for sampled and hierarchical indexes. Same validation,
 * errors and resulting index as the host forms; in addition `data` must be
 * device memory of `device`, aligned to its element size. No reference
 * counterpart (the reference's constructors take a host DenseMatrix); it
 * builds indexes whose host matrix would not fit host memory (for example
 * 65,536 x 262,144 values). */
uha_status uha_exact_index_create_device(int device, uha_metric metric,
                                         const uha_device_matrix* rows,
                                         uha_index** out);
uha_status uha_sampled_index_create_device(int device, uha_metric metric,
                                           const uha_device_matrix* rows,
                                           const uint64_t* columns,
                                           const uint64_t* multiplicities,
                                           const double* inverse_probabilities,
                                           uint64_t sample_size, uha_index** out);
uha_status uha_hierarchical_index_create_device(
    int device, uha_metric metric, const uha_device_matrix* rows,
    const uint64_t* columns, const uint64_t* multiplicities,
    const double* inverse_probabilities, uint64_t sample_size,
    const double* projection, uint64_t projection_dimension, uha_index** out);

void uha_index_destroy(uha_index* index);

/* Replaces space_usage() of every CUDA index class, with the reference byte
 * formulas (e.g. include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:85). */
uha_status uha_index_space_usage(const uha_index* index, uha_space_usage* out);

/* device() / device_name() of every CUDA index class. */
uha_status uha_index_device(const uha_index* index, int* device,
                            char* name, uint64_t name_capacity);

/* --------------------------------------------------------------- queries */

/* Replaces make_query_workspace(std::size_t) (e.g. include/ultrahigh_ann/
 * core/cuda_dense_l2_scan_index.hpp:56-57). A workspace belongs to one index
 * and one caller thread; it owns a CUDA stream and its scratch buffers. */
uha_status uha_workspace_create(const uha_index* index,
                                uint64_t maximum_batch_size,
                                uha_workspace** out);
void uha_workspace_destroy(uha_workspace* workspace);

/* maximum_batch_size() and payload_bytes() (the reference's logical payload
 * formula, e.g. tests/exact/l2/cuda_exact_l2_index_test.cpp:96-108). */
uha_status uha_workspace_info(const uha_workspace* workspace,
                              uint64_t* maximum_batch_size,
                              uint64_t* payload_bytes);

/* Answer query_count queries, a row-major query_count x dimension float
 * matrix in ORIGINAL coordinates. queries_on_device != 0 means `queries` is a
 * device pointer on the index's device (query_device_batch,
 * include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:73-79); otherwise it
 * is host memory and the host-to-device copy is part of the call
 * (query_batch, e.g. cuda_dense_l2_scan_index.hpp:62-66 and
 * coordinate_sampling/cuda_sampled_coordinate_l2_ann_index.hpp:70-82).
 * out_indices (host, query_count entries) receives the row index per query;
 * out_distances (host, nullable) the distance that selected it (squared L2,
 * L1 or median |diff|). Only sampled coordinates are read or validated. */
uha_status uha_query(const uha_index* index, uha_workspace* workspace,
                     const float* queries, uint64_t query_count,
                     int queries_on_device, uha_strategy strategy,
                     uint64_t* out_indices, double* out_distances);

/* Certified query of at most 8 device-resident queries against an exact or
 * flat index that allocates no memory: no workspace, no cudaMalloc/cudaFree, no allocating library call.
 * It has no counterpart in the reference; it exists for callers that cannot
 * allocate while they answer queries (a server whose device memory is
 * reserved up front by its own pool, code that must not allocate while other
 * threads capture CUDA graphs, embedded callers with a fixed footprint).
 * `queries` is a device pointer to query_count x dimension floats on the
 * index's device; out_indices (uint64_t) and out_distances (double, nullable)
 * are device pointers with query_count entries; `stream` is the cudaStream_t
 * to run on (NULL: the legacy default stream). The call returns after the
 * results are written (it synchronises `stream`). Results and errors equal
 * uha_query's with UHA_DIRECT.
 * Scratch: one static 32 MiB device array per GPU that loads the library,
 * held until the process exits. The first call on a device resolves its
 * address (cudaGetSymbolAddress) and keeps it; make that first call before
 * any stream capture. Batches whose scratch would exceed 32 MiB, or more than
 * 8 queries, fail with UHA_LENGTH_ERROR. All calls share the array: calls
 * that overlap on the GPU (other threads, other streams) race and must be
 * serialised by the caller. */
uha_status uha_query_noalloc(const uha_index* index, const float* queries,
                             uint64_t query_count, uint64_t* out_indices,
                             double* out_distances, void* stream);

/* query_count queries in consecutive batches of `batch` (at most the
 * workspace capacity), each batch answered exactly as one uha_query call
 * would answer it. All batches are enqueued back to back on the workspace
 * stream and the call synchronises once; host queries are copied batch by
 * batch. A non-finite (sampled) query value anywhere fails the whole call.
 * uha_query is uha_query_many with one batch. (No reference counterpart:
 * the reference's benchmark loops over query_batch per chunk,
 * src/benchmarks/nearest_neighbor_benchmark.cpp:386-413.) */
uha_status uha_query_many(const uha_index* index, uha_workspace* workspace,
                          const float* queries, uint64_t query_count,
                          uint64_t batch, int queries_on_device,
                          uha_strategy strategy, uint64_t* out_indices,
                          double* out_distances);

/* Diagnostics of the last uha_query on this workspace. */
uha_status uha_workspace_last_stats(const uha_workspace* workspace,
                                    uha_query_stats* out);

/* The CUDA stream (cudaStream_t) the workspace enqueues its work on, so a
 * caller can order its own work or record timing events against it. */
void* uha_workspace_stream(const uha_workspace* workspace);

/* With enabled != 0, queries on this workspace record CUDA events on the
 * workspace stream around the whole device pipeline (device_ms) and around
 * the scan kernel of every enabled-th batch of a call (scan_ms, summed over
 * timed_scans launches): 1 times every batch, larger values sample batches
 * so that the events cost less in long calls of small batches. */
uha_status uha_workspace_set_timing(uha_workspace* workspace, int enabled);

/* Candidates per query of the precision strategies (1 to 64; default 32).
 * No reference counterpart. */
uha_status uha_workspace_set_candidates(uha_workspace* workspace,
                                        uint32_t candidates);

/* Arithmetic of the replay that settles uncertified queries of the certified
 * (UHA_DIRECT) path on exact and flat indexes: UHA_REPLAY_BINARY64 (default)
 * replays the reference CPU's operations on the FP64 units;
 * UHA_REPLAY_EMULATED uses no FP64 instruction (float-float distances with a
 * stated bound, then emulated binary64 for candidates they cannot separate).
 * Both return the reference CPU's row. Hierarchical indexes always replay in
 * binary64. No reference counterpart. */
typedef enum uha_replay_arithmetic {
    UHA_REPLAY_BINARY64 = 0,
    UHA_REPLAY_EMULATED = 1
} uha_replay_arithmetic;
uha_status uha_workspace_set_replay(uha_workspace* workspace,
                                    uha_replay_arithmetic arithmetic);

/* Diagnostic of the precision strategies (no reference counterpart): for
 * query_count host queries (at most the workspace capacity), out_scores
 * (host, query_count x row_count, query-major) receives the tensor-core
 * scores r~.q~ of every row (FP8: times both scales), and out_norms (host,
 * row_count, nullable) the squared norms ||r~||^2 of the rounded rows. */
uha_status uha_precision_scores(const uha_index* index, uha_workspace* workspace,
                                const float* queries, uint64_t query_count,
                                uha_strategy strategy, float* out_scores,
                                float* out_norms);

/* ------------------------------------------- autotuning and batches
 * (no reference counterparts) */

/* The scan shape the autotuner chose: kernel 0 = streaming scan
 * (queries_per_pass queries per pass over the rows), 1 = register-tiled scan
 * (64 queries per tile), 2 = tensor-core score kernel (tile_queries per
 * tile); `splits` column / K splits; 3 = the L1 hierarchy's median passes
 * (queries_per_pass queries per pruning-count CTA, `splits` rows whose exact
 * medians set the pruning threshold). best_ms is its median event-timed
 * duration, default_ms that of the built-in heuristic's shape. */
typedef struct uha_tune_report {
    uint32_t candidates;
    uint32_t kernel;
    uint32_t queries_per_pass;
    uint32_t tile_queries;
    uint32_t splits;
    double best_ms;
    double default_ms;
} uha_tune_report;

/* Times every candidate scan shape for batches of exactly `batch` queries with
 * `strategy` on this workspace (CUDA events, median of 3 launches) and keeps
 * the fastest: later queries of that batch size on this workspace use it.
 * Answers do not change (the certification bound follows the shape).
 * L1 hierarchies time their median passes (sample, pruning count,
 * survivors) on stand-in queries, midpoints of pairs of the index's own
 * projected rows, since their cost depends on the data; the workspace's query
 * buffers are overwritten. Trivial indexes report zero candidates. report
 * may be NULL. */
uha_status uha_workspace_autotune(uha_workspace* workspace, uint64_t batch,
                                  uha_strategy strategy, uha_tune_report* report);

/* Many (index, query count, strategy) pairs on one device answered by one
 * CUDA graph launch: every pair's pipeline (preparation, projection, scan,
 * argmin or re-score, result copies) is captured once on its own graph branch.
 * With autotune != 0 each pair's scan shape is autotuned first. Each pair's
 * answers equal a uha_query of the same queries on that index. */
typedef struct uha_batch uha_batch;
typedef struct uha_batch_stats {
    uint64_t pairs;
    uint64_t queries;
    uint64_t graph_nodes;
    uint64_t kernel_launches;  /* kernels per run, all pairs */
    uint64_t replayed_queries;
    double device_ms;          /* graph launch to completion, last run */
} uha_batch_stats;

uha_status uha_batch_create(const uha_index* const* indexes,
                            const uint64_t* query_counts,
                            const uha_strategy* strategies, uint64_t count,
                            int autotune, uha_batch** out);
/* The same batch run as three persistent, cooperative kernel launches (the
 * gather and projection at 8 CTAs per SM, the tile scans and median samples
 * with the tile scan's register budget, then the late stages at 4 CTAs per
 * SM; captured in the batch's graph with the result copies). Each kernel drains a device work queue of units from all pairs
 * (gather, projection, L2 tile scan or median sample / count / survivor
 * passes, certified argmin with replay, reported distances), ordered stage by
 * stage: a CTA takes the next unit and waits only until that unit's pair has
 * completed its earlier stages, so pairs overlap across stages with no
 * grid-wide barrier. A wait gives up after about two seconds (the run then
 * fails with UHA_RUNTIME_ERROR). Each unit runs the device code of the standalone
 * kernel it replaces, so each pair's answers equal a uha_query of the same
 * queries. Serves hierarchical indexes with the certified direct strategy
 * (projection dimension up to 256; L2 hierarchies with more than 8 queries;
 * up to 32 pairs);
 * other pairs fail with UHA_INVALID_ARGUMENT. No reference counterpart. */
uha_status uha_batch_create_persistent(const uha_index* const* indexes,
                                       const uint64_t* query_counts, uint64_t count,
                                       int autotune, uha_batch** out);
/* Device buffer (query_counts[pair] x dimension floats) that the graph reads
 * pair `pair`'s queries from; NULL for an unknown pair. */
float* uha_batch_query_buffer(uha_batch* batch, uint64_t pair);
/* queries: NULL (use the query buffers as they are) or one pointer per pair,
 * host or device (queries_on_device), copied into the query buffers before
 * the graph launch. out_indices / out_distances (nullable): the pairs'
 * answers concatenated in pair order. */
uha_status uha_batch_run(uha_batch* batch, const float* const* queries,
                         int queries_on_device, uint64_t* out_indices,
                         double* out_distances);
uha_status uha_batch_stats_get(const uha_batch* batch, uha_batch_stats* out);
/* Stage times of the last run of a persistent batch, in ms (%globaltimer):
 * stage s from the time all units of the earlier stages had completed to the
 * time all units up to stage s had (stages of different pairs overlap; the
 * sum is the run's kernel time). The first `count` of them into out_ms, zero
 * past the last stage. *stages = number of stages (0 for a batch that is not
 * persistent). No reference counterpart. */
uha_status uha_batch_stage_times(const uha_batch* batch, double* out_ms, uint64_t count,
                                 uint64_t* stages);
uha_status uha_batch_tuning(const uha_batch* batch, uint64_t pair,
                            uha_tune_report* out);
void uha_batch_destroy(uha_batch* batch);

/* ------------------------------------------------------- request loop
 * (no reference counterpart)
 *
 * A serving loop over device-resident indexes on one GPU. Requests (one
 * query each, tagged with an index) are queued per index; a dispatcher thread
 * forms a batch from an index's queue as soon as one of `slots` in-flight
 * batches is free (continuous batching: queries that arrive while others are
 * on the GPU go into the next batch), so batches of different indexes overlap
 * on the device. Every in-flight batch holds a pooled query workspace of its
 * index; a new workspace is admitted only while the pooled workspaces' device
 * bytes stay within hbm_budget_bytes (idle workspaces of other indexes are
 * released to make room; otherwise the batch waits for one to finish). Each
 * answer equals a uha_query of that query alone on its index. */
typedef struct uha_server uha_server;

typedef struct uha_server_config {
    uint64_t hbm_budget_bytes;  /* device bytes of pooled workspaces, at most */
    uint32_t max_batch;         /* queries per batch, at most */
    uint32_t slots;             /* batches in flight, at most */
    int queries_on_device;      /* request query pointers are device pointers */
} uha_server_config;

typedef struct uha_server_result {
    uint64_t tag;
    uint32_t index_id;
    uint32_t status;     /* uha_status of this query */
    uint64_t row;
    double distance;
    double latency_us;   /* submission to completion seen by the loop */
} uha_server_result;

typedef struct uha_server_stats {
    uint64_t submitted;
    uint64_t completed;
    uint64_t failed;
    uint64_t batches;
    double mean_batch;
    double p50_us;
    double p99_us;
    double max_us;
    double throughput_qps;        /* completed / (last completion - first submission) */
    uint64_t workspace_bytes;     /* pooled workspaces now */
    uint64_t peak_workspace_bytes;
    uint64_t admission_waits;     /* dispatches deferred by the budget */
    uint64_t evictions;           /* idle workspaces released for another index */
    uint32_t peak_in_flight;
} uha_server_stats;

uha_status uha_server_create(int device, const uha_server_config* config,
                             uha_server** out);
/* Registers an index (its workspace is sized and warmed at max_batch here);
 * fails with UHA_LENGTH_ERROR when one workspace exceeds the budget. The
 * index must outlive the server. */
uha_status uha_server_add_index(uha_server* server, const uha_index* index,
                                uha_strategy strategy, uint32_t* out_id);
/* Creates pooled workspaces of index `index_id` until it holds `count` (within
 * the budget; *held receives how many it holds), so that a later burst does
 * not wait for workspace creation. */
uha_status uha_server_reserve(uha_server* server, uint32_t index_id, uint32_t count,
                              uint32_t* held);
/* Queues one query (dimension floats at `query`, host or device per the
 * config; the memory must stay valid until its result is polled).
 * Thread-safe. */
uha_status uha_server_submit(uha_server* server, uint32_t index_id,
                             const float* query, uint64_t tag);
/* Open-loop load: submits request i at arrival_us[i] microseconds after the
 * call (ascending), from the calling thread. */
uha_status uha_server_replay(uha_server* server, uint64_t count,
                             const uint32_t* index_ids,
                             const float* const* queries,
                             const double* arrival_us, const uint64_t* tags);
/* Waits until every submitted request has completed. */
uha_status uha_server_drain(uha_server* server);
/* Moves up to `capacity` completed results into `out`; *count receives how
 * many. */
uha_status uha_server_poll(uha_server* server, uha_server_result* out,
                           uint64_t capacity, uint64_t* count);
uha_status uha_server_stats_get(uha_server* server, uha_server_stats* out);
/* Clears the latency record and counters (the pool stays). */
uha_status uha_server_reset_stats(uha_server* server);
void uha_server_destroy(uha_server* server);

/* ---------------------------------------------------------- index build */

/* Pair-distance method of the device probability build. DIRECT sums squared
 * (or absolute) differences per pair; GRAM (L2 only) forms the r x r Gram
 * matrix and recomputes cancellation-prone pairs directly, as the reference's
 * cuBLAS backend does (src/hnsvw25/l2/cuda_importance_sampling.cu:332-364). */
typedef enum uha_pair_backend {
    UHA_PAIRS_DIRECT = 0,
    UHA_PAIRS_GRAM = 1,
    /* the same binary64 pair distances, the per-column maxima formed in
     * binary32 (within 3e-7 relative of the binary64 maxima, inside the
     * reference GPU path's 1e-6): for full-size builds, which the binary64
     * pipe would otherwise bound. No reference counterpart. */
    UHA_PAIRS_DIRECT_MAX32 = 2,
    UHA_PAIRS_GRAM_MAX32 = 3
} uha_pair_backend;

/* Importance probabilities on the device. L2: p_j = max over row pairs of
 * min(1, (a_j-b_j)^2 / ||a-b||^2); L1: p_j = max over pairs of
 * |a_j-b_j| / ||a-b||_1; pairs at distance zero are skipped. Pair distances
 * and the normalisation are binary64. The per-column maxima are folded in
 * min(pair_chunks, pairs) launches over consecutive pair ranges, which bounds
 * the duration of each kernel (pair_chunks must be positive). Replaces
 * compute_l2_importance_probabilities_gpu (include/ultrahigh_ann/hnsvw25/l2/
 * importance_sampling.hpp:49-52) and compute_l1_importance_probabilities_gpu
 * (include/ultrahigh_ann/hnsvw25/l1/importance_sampling.hpp:45-48). */
uha_status uha_importance_probabilities(int device, uha_metric metric,
                                        const float* rows, uint64_t row_count,
                                        uint64_t dimension,
                                        uha_pair_backend backend,
                                        uint64_t pair_chunks,
                                        double* out_probabilities,
                                        uha_probability_report* report);

/* The same from a representative matrix already on `device` (row-major,
 * `dimension` floats per row, at device_rows): no host copy, for matrices
 * that the host cannot hold or that were built on the device. The values are
 * checked for finiteness on the device. No reference counterpart. */
uha_status uha_importance_probabilities_device(int device, uha_metric metric,
                                               const float* device_rows,
                                               uint64_t row_count, uint64_t dimension,
                                               uha_pair_backend backend,
                                               uint64_t pair_chunks,
                                               double* out_probabilities,
                                               uha_probability_report* report);

/* The same probabilities on the host cores with the reference CPU policies'
 * binary64 arithmetic, bit-identical to its sequential loop for any thread
 * count. Replaces the sequential / cpu_parallel policies of
 * compute_l{1,2}_importance_probabilities (src/hnsvw25/l2/
 * importance_sampling.cpp:126-144, src/hnsvw25/l1/importance_sampling.cpp:115-134). */
uha_status uha_importance_probabilities_host(uha_metric metric,
                                             const float* rows,
                                             uint64_t row_count,
                                             uint64_t dimension, int threads,
                                             double* out_probabilities);

/* ------------------------------------------------------------ data files */

/* SHA-256 (FIPS 180-4) of a buffer or of a file's bytes, 32 bytes out.
 * Replaces ultrahigh_ann::io::sha256_file (include/ultrahigh_ann/io/
 * sha256.hpp:14). */
uha_status uha_sha256(const void* data, uint64_t size, uint8_t* out);
uha_status uha_sha256_file(const char* path, uint8_t* out);

/* Versioned importance-probability file ("UHANNPR2", kind, representative
 * count, SHA-256 of the representative-matrix file, binary64 probabilities),
 * bound to the matrix it was computed from. Replaces
 * save_importance_probabilities / load_importance_probabilities
 * (include/ultrahigh_ann/io/importance_probability_io.hpp:27-35); malformed
 * files fail with UHA_RUNTIME_ERROR and the reference's messages. load: with
 * probabilities NULL only the header fields and *count are returned;
 * otherwise capacity must hold *count values (UHA_LENGTH_ERROR). */
uha_status uha_probabilities_save(const char* path, uha_metric kind,
                                  uint64_t representative_count,
                                  const uint8_t* representatives_sha256,
                                  const double* probabilities, uint64_t count);
uha_status uha_probabilities_load(const char* path, uha_metric* kind,
                                  uint64_t* representative_count,
                                  uint8_t* representatives_sha256,
                                  double* probabilities, uint64_t capacity,
                                  uint64_t* count);

/* Little-endian NPY files of the transformed datasets: a two-dimensional
 * C-order float32 matrix (finite values) and a one-dimensional uint16 label
 * vector. Replace load_float_matrix_npy / load_label_vector_npy
 * (include/ultrahigh_ann/datasets/representative_query_dataset.hpp:19-25);
 * with out NULL only the shape is returned. */
uha_status uha_npy_load_f32(const char* path, float* out, uint64_t capacity,
                            uint64_t* rows, uint64_t* cols);
uha_status uha_npy_load_u16(const char* path, uint64_t* out, uint64_t capacity,
                            uint64_t* count);

/* std::mt19937_64 engine shared by the host-side draws below, so that one
 * engine passes through sampling and projection in the reference order. */
uha_status uha_rng_create(uint64_t seed, uha_rng** out);
void uha_rng_destroy(uha_rng* rng);
/* Textual engine state (operator<< of std::mt19937_64). *length receives the
 * size needed including the terminating zero. */
uha_status uha_rng_state(const uha_rng* rng, char* buffer, uint64_t capacity,
                         uint64_t* length);
uha_status uha_rng_set_state(uha_rng* rng, const char* state);

/* Coordinate sample: for each j with p_j > 0, multiplicity ~ Binomial(
 * repetitions, p_j); kept when positive, in ascending j. Same engine draws as
 * build_coordinate_sample (include/ultrahigh_ann/coordinate_sampling/
 * coordinate_sampling.hpp:13-16). Outputs need room for `dimension` entries;
 * *sample_size receives k. */
uha_status uha_sample_coordinates(const double* probabilities,
                                  uint64_t dimension, uint64_t repetitions,
                                  uha_rng* rng, uint64_t* columns,
                                  uint64_t* multiplicities,
                                  double* inverse_probabilities,
                                  uint64_t* sample_size);

/* Row-major p x k Rademacher-JL matrix (aggregated signs per sampled column)
 * in the reference's draw order (src/hnsvw25/l2/hierarchical/
 * l2_hierarchical_projection.cpp:53-77). */
uha_status uha_jl_matrix(const uint64_t* multiplicities,
                         const double* inverse_probabilities,
                         uint64_t sample_size, uint64_t projection_dimension,
                         uha_rng* rng, double* out);

/* Row-major p x k Cauchy matrix in the reference's draw order
 * (src/hnsvw25/l1/hierarchical/l1_hierarchical_projection.cpp:54-77). */
uha_status uha_cauchy_matrix(const uint64_t* multiplicities,
                             const double* inverse_probabilities,
                             uint64_t sample_size,
                             uint64_t projection_dimension, uha_rng* rng,
                             double* out);

/* Row-major p x k Gaussian JL matrix, a seeded binary32 matrix for L2
 * hierarchies (passed to uha_hierarchical_index_create like the Rademacher
 * one): entry (row, i) = float(Z * sqrt(m_i * (1/p_i) / p)) with Z a standard
 * normal draw (std::normal_distribution<double> on the engine, row-major
 * order). The variance per entry, m_i (1/p_i) / p, is that of the
 * aggregated Rademacher entry it replaces (a sum of m_i independent
 * N(0, 1) is N(0, m_i)), so both estimate the same squared distance.
 * No counterpart in the reference, whose L2 hierarchy is Rademacher-only
 * (src/hnsvw25/l2/hierarchical/l2_hierarchical_projection.cpp:53-77). */
uha_status uha_gaussian_jl_matrix(const uint64_t* multiplicities,
                                  const double* inverse_probabilities,
                                  uint64_t sample_size,
                                  uint64_t projection_dimension, uha_rng* rng,
                                  double* out);

#ifdef __cplusplus
}
#endif

#endif /* UHA_B200_H */
