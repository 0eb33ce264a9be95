// Launch interface of the engine's CUDA kernels (host side). Each launcher
// enqueues on the given stream and returns without synchronising.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace uha {

// What a scan accumulates per (query, row) over the sampled/projected columns.
enum class ScanOp : int {
    l2 = 0,        // sum (q - r)^2
    l1 = 1,        // sum |q - r|
    l1_weighted = 2,  // sum w * |q - r|
    dot = 3,       // sum q * r  (binary32 norm-identity strategy)
};

// How the certifying replay reproduces the reference CPU sum.
enum class ReplayOp : int {
    l2_sequential = 0,       // s += (double(q) - double(r))^2, in column order
    l1_grouped4 = 1,         // std::transform_reduce grouping of |q - r|
    l1_weighted_sequential = 2,  // s += w64 * |double(q) - double(r)|
    l2_projected = 3,        // binary64 projected query vs binary64 rows
    median_projected = 4,    // median |double diff| (nth_element semantics)
};

// Device view of the per-(chunk, query, row) partial sums of a scan.
struct PartialView {
    float* partials;      // [chunks][batch][rows]
    uint32_t chunks;
    uint32_t batch;
    uint32_t rows;
};

// Certification parameters. For a binary32 distance D of row `row` and query
// `q` the reference CPU's binary64 distance lies in
//   plain:        [D - (rel D + abs), D + (rel D + abs)]
//   projected_l2: [((sqrt(D (1 - rel)) - E)+)^2 (1 - cpu_rel) - abs,
//                  (sqrt(D (1 + rel)) + E)^2 (1 + cpu_rel) + abs]
//   median:       [D - (rel D + E + abs), D + (rel D + E + abs)]
// with E = row_err[row] + query_err[q]: the Euclidean (projected_l2) or
// maximum (median) norm of the binary32-vs-binary64 error of the projected
// row and the projected query.
enum class BoundMode : int { plain = 0, projected_l2 = 1, median = 2 };

struct Bound {
    float rel;
    float abs;
    BoundMode mode = BoundMode::plain;
    const float* row_err = nullptr;
    const float* query_err = nullptr;
    float cpu_rel = 0.f;
    // median mode (nullable): per (query, row) error of a computed median,
    // pair_err[q * pair_rows + row], used in place of row_err + query_err
    const float* pair_err = nullptr;
    uint32_t pair_rows = 0;
    float row_err_max = 0.f;  // largest row_err (hierarchical modes)
};

struct Result {
    uint32_t row;
    float distance;
};

// ---- query preparation (gather / copy + finiteness validation)
void launch_prepare_dense(const float* queries, uint64_t batch, uint64_t dim,
                          float* out, uint64_t padded_dim, int* error_flag,
                          cudaStream_t stream);
void launch_prepare_sampled(const float* queries, uint64_t batch, uint64_t dim,
                            const uint32_t* columns, const float* scales,
                            uint64_t sample_size, float* out,
                            uint64_t padded_dim, int* error_flag,
                            cudaStream_t stream);
// out[q] = sources[q] (count device vectors of dim floats, gathered into
// one contiguous batch).
void launch_gather_vectors(const float* const* sources, uint64_t count, uint64_t dim,
                           float* out, cudaStream_t stream);
void launch_query_norms(const float* prepared, uint64_t batch,
                        uint64_t padded_dim, float* norms, cudaStream_t stream);

// ---- scans: write partial sums for every (chunk, query, row)
// Returns the number of chunks used (stored in PartialView.chunks by the
// caller) and the accumulation depth for the error bound.
struct ScanPlan {
    uint32_t chunks;
    uint32_t depth;        // longest chain of binary32 additions per distance
    int kernel;            // 0 = stream kernel, 1 = tile kernel
    uint32_t k_per_split;  // tile kernel: columns per split
    int queries_per_pass;  // stream kernel: queries per CTA (1, 2, 4 or 8)
};
ScanPlan plan_scan(uint64_t rows, uint64_t padded_dim, uint64_t batch,
                   int sm_count);
// The stream kernel with `queries_per_pass` (1, 2, 4, 8) queries per pass; the
// tile kernel with about `splits` column splits.
ScanPlan stream_plan(uint64_t padded_dim, int queries_per_pass);
ScanPlan tile_plan(uint64_t padded_dim, uint64_t splits);
// Plans the autotuner times for one (index, batch): the heuristic plan first.
std::vector<ScanPlan> scan_candidates(uint64_t rows, uint64_t padded_dim,
                                      uint64_t batch, int sm_count);
void launch_scan(const ScanPlan& plan, ScanOp op, const float* rows,
                 uint64_t row_count, uint64_t padded_dim, const float* weights,
                 const float* queries, uint64_t batch, float* partials,
                 cudaStream_t stream);

// ---- certification
// Everything the binary64 replay of a query needs: the reference CPU's
// operation sequence (`op`) and the operands it reads.
struct ReplayInputs {
    ReplayOp op;
    const float* rows;         // [rows][padded_dim]
    const float* queries;      // [batch][padded_dim] (projected ops: the
                               // gathered sampled values)
    const double* weights64;   // l1_weighted_sequential
    uint64_t dim;              // columns to replay (projected ops: k)
    uint64_t padded_dim;
    const double* rows64 = nullptr;        // projected ops: [rows][proj_dim]
    const double* projection64 = nullptr;  // projected ops: [proj_dim][dim]
    uint64_t proj_dim = 0;
    // Replay without the FP64 units (exact and flat ops): a float-float
    // distance per candidate, within ff_rel * S + ff_abs of the reference
    // CPU's binary64 value (its own rounding included), decides unless two
    // candidates' intervals overlap; those are replayed in emulated binary64
    // (exact64.h). weights_ff: the binary64 weights as float pairs hi, lo.
    bool emulated = false;
    float ff_rel = 0.f;
    float ff_abs = 0.f;
    const float* weights_ff = nullptr;
};
// ff_rel / ff_abs of the emulated replay of `dim` terms.
void emulated_replay_bound(uint64_t dim, float* rel, float* abs);

// Scratch of the argmin (per-query merge state, layout fixed by the workspace
// capacity). It must be zero when the workspace is created; the argmin leaves
// its counters at zero after every call.
uint64_t finalize_scratch_bytes(uint64_t batch, uint64_t rows);
// Certified argmin with lowest-index tie-break of every query of the view;
// uncertified queries are settled in the same kernel by the binary64 replay.
// results[q] receives the row; exact_distances[q] the replayed distance or
// NaN when the query was certified. *replay_count counts replayed queries.
void launch_argmin(PartialView view, Bound bound, ReplayInputs in,
                   Result* results, double* exact_distances, void* scratch,
                   uint64_t capacity, uint32_t* replay_count,
                   cudaStream_t stream);
// Indexes small enough for one CTA per query (rows <= 4096, padded columns
// <= 8192, rows x padded columns <= 65536): gather, scan and certified argmin
// (with replay) in one launch.
constexpr uint64_t kSmallRows = 4096;
constexpr uint64_t kSmallColumns = 8192;
constexpr uint64_t kSmallCells = 65536;
struct SmallQuery {
    const float* queries;     // [batch][dim] raw queries
    uint64_t dim;
    const uint32_t* columns;  // sampled columns (null: all columns)
    const float* scales;      // sampled L2 scales (nullable)
    uint64_t sample_size;
    const float* rows;        // [row_count][padded_dim]
    uint32_t row_count;
    uint64_t padded_dim;
    const float* weights32;   // weighted L1
    int op;                   // ScanOp: l2, l1 or l1_weighted
};
bool small_query_fits(uint64_t rows, uint64_t padded_dim);
uint32_t small_query_depth(uint64_t padded_dim);
void launch_small_query(const SmallQuery& sq, uint32_t batch, Bound bound, ReplayInputs in,
                        Result* results, double* exact_distances, uint32_t* replay_count,
                        int* error_flag, cudaStream_t stream);
// Flat and small exact indexes (padded columns <= kFlatColumns) at batches of
// at most kFlatBatch queries: gather, scan and certified argmin (with replay)
// in one launch with many CTAs per query, the last CTA of a query merging.
// Launched with programmatic stream serialization outside stream capture:
// consecutive launches on one stream alternate between that stream's two
// slots of the scratch (slot = 2 lane + 0, 1, 0, ...), and each one's gather
// and scan overlap the end of the previous one.
constexpr uint64_t kFlatColumns = 8192;
constexpr uint64_t kFlatBatch = 8;
// streams a call's flat launches are spread over (independent launch chains)
constexpr int kFlatLanes = 3;
struct FlatPlan {
    uint32_t lanes;       // lanes per row: 8, 16 or 32
    uint32_t span;        // rows per CTA
    uint32_t blocks;      // CTAs per query
    uint32_t depth;       // longest chain of binary32 additions per distance
    uint32_t chunk_rows;  // rows per bulk copy into shared memory
    uint32_t buffers;     // copy buffers per CTA (1 when a span is one chunk)
};
bool flat_query_fits(uint64_t rows, uint64_t padded_dim, uint64_t batch);
FlatPlan plan_flat_query(uint64_t rows, uint64_t padded_dim, uint64_t batch,
                         int sm_count);
// Scratch for a workspace of `capacity` queries, `slots` slots (two per
// stream lane); zero when created, left with its counters at zero by every
// launch.
uint64_t flat_query_scratch_bytes(uint64_t capacity, uint64_t rows, uint32_t slots);
void launch_flat_query(const SmallQuery& sq, const FlatPlan& plan, uint32_t batch,
                       Bound bound, ReplayInputs in, void* scratch, uint64_t capacity,
                       uint32_t slot, Result* results, double* exact_distances,
                       uint32_t* replay_count, int* error_flag, cudaStream_t stream);
// Binary32 norm identity (no certification), lowest index on ties.
void launch_finalize_gemm(PartialView view, const float* row_norms,
                          const float* query_norms, Result* results,
                          cudaStream_t stream);

// Reference binary64 distance of each query's selected row (projected replay
// ops only), for the queries that the argmin did not replay and whose
// certified interval is wider than 1e-5 relative.
void launch_refine_winners(ReplayInputs in, Bound bound, const Result* results,
                           uint32_t batch, double* exact_distances,
                           cudaStream_t stream);

// ---- precision form: low-precision scores on the tensor cores, top-k,
// binary32 re-score of the candidates
enum class LowpType : int { bf16 = 0, fp8_e4m3 = 1 };
// Elements per stored low-precision vector (a multiple of one 128-byte K
// slice; zero past the scanned columns).
uint64_t lowp_pitch(LowpType type, uint64_t dim);
// Vectors a low-precision buffer holds for `count` rows or queries.
uint64_t lowp_padded_count(uint64_t count);
uint64_t lowp_element_bytes(LowpType type);
// Rounds `count` binary32 vectors (src_pitch apart, `dim` used) into `out`
// (pitch apart): BF16, or E4M3 with scales[i] = max|x| / 448. norms[i]
// (nullable) = squared norm of the rounded (dequantized) vector.
void launch_lowp_convert(LowpType type, const float* src, uint64_t count,
                         uint64_t src_pitch, uint64_t dim, void* out,
                         uint64_t pitch, float* scales, float* norms,
                         cudaStream_t stream);
// Rounds `count` zero-padded binary32 query vectors (src_pitch apart, a
// multiple of 4) like launch_lowp_convert, without norms, with many blocks
// per vector. amax_scratch: `count` words (FP8).
void launch_lowp_queries(LowpType type, const float* src, uint64_t count,
                         uint64_t src_pitch, void* out, uint64_t pitch,
                         float* scales, unsigned int* amax_scratch,
                         cudaStream_t stream);
struct LowpPlan {
    int bn;                      // queries per tile (UMMA N)
    uint32_t splits;             // K splits (partial-score slabs)
    uint32_t kblocks;            // 128-byte K slices per vector
    uint32_t kblocks_per_split;
};
LowpPlan plan_lowp(LowpType type, uint64_t rows, uint64_t pitch, uint64_t batch,
                   int sm_count);
// Query tile width `bn` (16, 32, 64, 128, 256) and about `splits` K splits.
LowpPlan lowp_plan(LowpType type, uint64_t pitch, int bn, uint64_t splits);
// Plans the autotuner times for one (index, batch): the heuristic plan first.
std::vector<LowpPlan> lowp_candidates(LowpType type, uint64_t rows, uint64_t pitch,
                                      uint64_t batch, int sm_count);
// The candidate filter fused into the score kernel (plans of one K split):
// keys (e, row) of the rows whose estimate e = ||v~||^2 - 2 S is at most
// tau[q] are appended to keys[q][0 .. cap); count[q] (zero before) counts
// them all.
struct FilterArgs {
    const float* norms;        // rounded-row norms ||v~||^2
    const float* tau;          // per query
    unsigned long long* keys;  // batch x cap
    uint32_t* count;           // batch
    uint32_t cap;
};
// partials[split][q][row] = q~ . v~ over the split's K slices (FP8: times the
// row and query scales), or with `filter` (one K split) the filter's keys in
// place of the slab. error_flag |= 8 when a pipeline wait ran out.
// With sample_rows (a multiple of 128, below row_count) only that many rows
// are scored: whole tiles spread evenly over the index (sample_tile_stride),
// written as rows 0 .. sample_rows of the slab.
void launch_lowp_scores(const LowpPlan& plan, LowpType type, const void* rows_lp,
                        const float* row_scale, uint64_t row_count,
                        const void* queries_lp, const float* query_scale,
                        uint64_t batch, uint64_t pitch, float* partials,
                        int* error_flag, cudaStream_t stream,
                        const FilterArgs* filter = nullptr, uint64_t sample_rows = 0);
uint32_t sample_tile_stride(uint64_t rows, uint64_t sample_rows);
// The fused selection: sample rows (whole tiles spread over the index) whose
// k-th smallest estimate bounds each query's threshold, and the list
// capacity.
// A query whose list overflows sets error bit kCandidateOverflow; the call
// is then answered again by the slab path.
constexpr uint64_t kFilterMinRows = 16384;
constexpr int kCandidateOverflow = 32;
uint64_t filter_sample_rows(uint64_t rows);
uint32_t filter_capacity(uint64_t rows, uint32_t k);
// out[i] = norms[the index row sample row i stands for] (a sample of
// sample_rows over an index of `rows` rows, as launch_lowp_scores scores it).
void launch_gather_sample_norms(const float* norms, uint64_t rows, uint32_t sample_rows,
                                float* out, cudaStream_t stream);
// tau[q] = the estimate of sample_candidates[q * k + k - 1] over the sample's
// one-slab partials, with the sample's norms (+inf when the sample has fewer
// than k rows).
void launch_lowp_threshold(const float* partials, uint32_t batch, uint32_t sample_rows,
                           const float* sample_norms, uint32_t k,
                           const uint32_t* sample_candidates, float* tau,
                           cudaStream_t stream);
// candidates[q * k + i]: the k smallest keys of the query's list (the same
// rows and order as launch_lowp_topk over the whole slab); count[q] > cap
// sets error bit kCandidateOverflow.
void launch_lowp_select(const unsigned long long* keys, const uint32_t* count, uint32_t cap,
                        uint32_t batch, uint32_t k, uint32_t* candidates, int* error_flag,
                        cudaStream_t stream);
// candidates[q * k + i]: the k rows with the smallest ||v~||^2 - 2 S
// (ascending, lowest row on ties; 0xffffffff past the index's rows).
void launch_lowp_topk(const float* partials, uint32_t splits, uint32_t batch,
                      uint32_t rows, const float* norms, uint32_t k,
                      uint32_t* candidates, cudaStream_t stream);
// Precision form of the L2 hierarchy: out[q][j] = sum over the slabs of
// partials[s][q][j] for j < rows, zeros up to out_pitch.
void launch_sum_slabs(const float* partials, uint32_t splits, uint64_t batch,
                      uint64_t rows, float* out, uint64_t out_pitch, cudaStream_t stream);
// The reference's binary64 projection of gathered queries, y[q][j] =
// sum_i double(x[q][i]) * P[j][i] in i order (proj_t = P transposed,
// [k][p]); error_flag |= 4 for a non-finite result.
void launch_project_queries64(const float* x, uint64_t batch, uint64_t padded_k,
                              uint64_t k, const double* proj_t, uint64_t p, double* y,
                              int* error_flag, cudaStream_t stream);
// Per query, the candidate with the smallest (reference binary64 squared
// distance of the projected row rows64[row] to y64[q], row): results[q] and
// exact_distances[q]. Candidates 0xffffffff are skipped.
void launch_rescore_projected(const uint32_t* candidates, uint32_t k, uint32_t batch,
                              const double* rows64, const double* y64, uint32_t p,
                              Result* results, double* exact_distances,
                              cudaStream_t stream);
// Binary64 certification interval [S (1 - rel) - abs, S (1 + rel) + abs] of
// a parallel binary64 sum S of the reference CPU's own terms.
struct Bound64 {
    double rel;
    double abs;
};
// Accumulation depth of the re-score's binary64 distances (for the bound);
// the binary32 re-score has the same structure and depth.
uint32_t rescore_depth(uint64_t padded_dim);
uint32_t max_rerank_candidates();
// Certified argmin of each query over its k candidates (ReplayInputs as for
// the plain L2 scan): cand_dist holds batch x k doubles, done batch counters
// that are zero before and after the launch. results / exact distances /
// replay count as launch_argmin; exact[q] is the answer's binary64 distance.
void launch_rescore(Bound64 bound, ReplayInputs in, const uint32_t* candidates,
                    uint32_t k, uint32_t batch, uint32_t rows, double* cand_dist,
                    uint32_t* done, Result* results, double* exact_distances,
                    uint32_t* replay_count, cudaStream_t stream);

// The FP32 re-score of the precision strategies: each candidate's binary32
// distance from the original rows (bound: make_bound(rescore_depth, k, 2)),
// certified per query; uncertified queries are settled by the emulated replay
// (in.emulated must be set). cand_dist: batch x k floats; done as above.
void launch_rescore32(Bound bound, ReplayInputs in, const uint32_t* candidates,
                      uint32_t k, uint32_t batch, uint32_t rows, float* cand_dist,
                      uint32_t* done, Result* results, double* exact_distances,
                      uint32_t* replay_count, cudaStream_t stream);
// ---- hierarchical index (projection)
// Binary64 projected rows reps[row][j] = sum_i double(sampled[row][i]) *
// projection[j][i] in i order; `bad` is set when a result is not finite.
void launch_project_rows64(const float* sampled, uint64_t row_count,
                           uint64_t padded_k, uint64_t k,
                           const double* projection, uint64_t p, double* reps,
                           int* bad, cudaStream_t stream);
// reps64 -> binary32 padded rows and the per-row error norm
// (euclidean: 2-norm, else max-norm) of float(reps) - reps.
void launch_narrow_rows(const double* reps, uint64_t row_count, uint64_t p,
                        float* out, uint64_t padded_p, float* row_err,
                        bool euclidean, int* bad, cudaStream_t stream);
// Binary32 projection of gathered queries with its certified error norm:
// y[b][j] = sum_i x[b][i] proj32[j][i]; query_err[b] bounds the distance
// between y[b] and the reference's binary64 projection (2-norm if
// euclidean, else max-norm); coord_err (nullable) receives the bound of each
// coordinate, [batch][padded_p]. error_flag |= 4 for a non-finite projection.
void launch_project_queries(const float* gathered, uint64_t batch,
                            uint64_t padded_k, uint64_t k,
                            const float* proj32, uint64_t p, float* out,
                            uint64_t padded_p, float* query_err, float* coord_err,
                            double err_per_abs, bool euclidean,
                            int* error_flag, cudaStream_t stream);
// Median of |rows[row][j] - queries[q][j]| over j < p per (query, row),
// written as one chunk of partials. Rows that provably cannot be a query's
// argmin (their median is above a threshold derived from the exact medians of
// 32-256 spread rows and the median bound: relative `rel`, absolute
// `abs_err`, row errors up to row_err_max, query_err[q]) store minus that
// threshold: a lower bound with no upper bound. min_bits: one word per query.
// rows_t (nullable): the same rows transposed, [padded_p][r_pitch], for the
// register-tiled pruning count.
// Every pair whose median is computed also gets pair_err[q][row]: a bound on
// |median - reference median| from the coordinates near the median only
// (coord_err[q][j]: the projected query's per-coordinate error; rows carry
// their binary32 rounding), in place of the max-norm errors.
//
// The shape of the three passes (answers do not depend on it): `samples` rows
// whose exact medians set the threshold, `count_queries` queries per CTA of
// the pruning count (1, 2, 4 or 8, at most the batch).
struct MedianPlan {
    uint32_t samples;
    uint32_t count_queries;
};
MedianPlan default_median_plan(uint64_t row_count, uint64_t batch);
// The default first, then the autotuner's other candidates.
std::vector<MedianPlan> median_candidates(uint64_t row_count, uint64_t batch);
void launch_median_scan(const MedianPlan& plan, const float* rows, const float* rows_t,
                        uint64_t r_pitch, uint64_t row_count, uint64_t padded_p,
                        uint64_t p, const float* queries, uint64_t batch,
                        const float* query_err, const float* coord_err,
                        float row_err_max, float rel,
                        float abs_err, unsigned int* min_bits, float* partials,
                        float* pair_err, cudaStream_t stream);
// Stand-in queries for timing the median passes: query q is the midpoint of
// two rows of the index (rows a = (7919 q + 1) mod r, b = (104729 q + 3) mod r),
// zero past column p; written as batch x padded_p.
void launch_median_tuning_queries(const float* rows, uint64_t row_count, uint64_t padded_p,
                                  uint64_t p, uint64_t batch, float* queries,
                                  cudaStream_t stream);
// out[j][row] = rows[row][j] for j < padded_p (build time).
void launch_transpose_rows(const float* rows, uint64_t row_count, uint64_t padded_p,
                           float* out, uint64_t r_pitch, cudaStream_t stream);

// ---- build-time helpers
void launch_gather_rows(const float* source, uint64_t row_count, uint64_t dim,
                        const uint32_t* columns, const float* scales,
                        uint64_t sample_size, float* out, uint64_t padded_dim,
                        cudaStream_t stream);
// Gather from a device-resident binary32 or BF16 matrix with a row stride
// (columns == nullptr: column i); first_bad (nullable, two entries preset to
// ~0) receives the first non-finite source / scaled value's r * k + i.
void launch_gather_device_rows(const void* source, bool bf16, uint64_t stride,
                               uint64_t row_count, const uint32_t* columns,
                               const float* scales, uint64_t sample_size,
                               float* out, uint64_t padded_dim,
                               unsigned long long* first_bad, cudaStream_t stream);
void launch_row_norms(const float* rows, uint64_t row_count,
                      uint64_t padded_dim, float* norms, cudaStream_t stream);

// ---- importance probabilities (binary64 pair distances and normalisation)
void launch_pair_distances(int metric, const float* rows, uint64_t row_count,
                           uint64_t dim, double* inverse_distances,
                           cudaStream_t stream);
// L2 pair distances through the binary64 Gram identity with direct
// recomputation of cancellation-prone pairs; `gram` holds r x r doubles.
void launch_gram_inverse_distances(const float* rows, uint64_t row_count,
                                   uint64_t dim, double* gram,
                                   double* inverse_distances,
                                   cudaStream_t stream);
// Folds the pairs [pair_begin, pair_end) of the row-major order of pairs
// a < b into the per-column maxima (one launch per chunk of pairs); `single`:
// the contributions in binary32 (within 3e-7 relative).
void launch_coordinate_maxima(int metric, const float* rows,
                              uint64_t row_count, uint64_t dim,
                              const double* inverse_distances,
                              unsigned long long* maxima_bits,
                              uint64_t pair_begin, uint64_t pair_end,
                              cudaStream_t stream, bool single = false);
// flag |= 1 when any of the `count` values is not finite
void launch_finite_check(const float* values, uint64_t count, int* flag,
                         cudaStream_t stream);

}  // namespace uha
