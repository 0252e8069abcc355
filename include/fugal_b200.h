/*
 * fugal_b200.h -- C ABI of the B200 (sm_100a) FUGAL alignment kernels.
 *
 * Plain pointers and sizes only: every matrix/vector argument is a DEVICE
 * pointer owned by the caller (row-major, leading dimension in elements), every
 * call is asynchronous on the given CUDA stream and returns a fugal_status.
 * No entry point synchronises the device or allocates device memory; kernels
 * that need scratch take a caller-provided workspace whose size is returned by
 * the matching *_workspace_size() query.  A non-OK status leaves a message in
 * fugal_last_error().
 *
 * The first group mirrors, one entry point each, the pybind11 module
 * `cuda_kernels` of cuGAL (cuda_kernels/kernels.cpp:4-30, bound at :32-70) that
 * cugal/*.py calls.  The second group is the fused path that replaces the
 * Python-level Frank-Wolfe step (cugal/pred.py:89-148) with three calls:
 * gradient -> Sinkhorn solve -> update.
 */
#ifndef FUGAL_B200_H
#define FUGAL_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* fugal_stream_t; /* == cudaStream_t; NULL = legacy default stream */

typedef enum {
    FUGAL_OK = 0,
    FUGAL_BAD_SHAPE = 1,        /* size, leading dimension or alignment not supported */
    FUGAL_BAD_ARGUMENT = 2,     /* null pointer, bad enum value, bad parameter */
    FUGAL_CUDA_ERROR = 3,       /* a CUDA runtime call failed (launch, attribute, event) */
    FUGAL_ITER_LIMIT = 4,       /* an iteration cap was hit where that is an error */
    FUGAL_NONFINITE = 5,        /* NaN / Inf detected */
    FUGAL_DEVICE_TIMEOUT = 6,   /* a bounded device-side wait gave up (kernel returned early) */
    FUGAL_WORKSPACE_TOO_SMALL = 7,
    FUGAL_UNSUPPORTED = 8
} fugal_status;

typedef enum { FUGAL_F32 = 0, FUGAL_BF16 = 1, FUGAL_F16 = 2 } fugal_dtype;

typedef enum {
    FUGAL_LAP_GREEDY = 0,          /* cugal/greedy_lap.py:10-19 */
    FUGAL_LAP_DOUBLE_GREEDY = 1,   /* cugal/greedy_lap.py:50-63 */
    FUGAL_LAP_PARALLEL_GREEDY = 2, /* cugal/greedy_lap.py:65-85 */
    FUGAL_LAP_ORDERED = 3          /* RAND: rows in a caller-given order, cugal/greedy_lap.py:21-32 */
} fugal_lap_method;

/* Kernel families counted / timed by the instrumentation below. */
typedef enum {
    FUGAL_KERNEL_SWEEP = 0,       /* fused Sinkhorn sweep over the BF16/FP16 cost copy */
    FUGAL_KERNEL_SWEEP_F32 = 1,   /* fused Sinkhorn sweep over the FP32 cost (warm-up, polish, FP32 stream) */
    FUGAL_KERNEL_ABSORB = 2,      /* FP32 sweep that also writes the reduced-precision copy */
    FUGAL_KERNEL_FINALIZE = 3,    /* per-sweep column reduction + convergence decision */
    FUGAL_KERNEL_COLUMN_PASS = 4, /* column LSE of the first iteration of a solve */
    FUGAL_KERNEL_GRADIENT = 5,    /* both SpMM kernels of the gradient */
    FUGAL_KERNEL_UPDATE = 6,
    FUGAL_KERNEL_OTHER = 7,
    FUGAL_KERNEL_FAMILIES = 8
} fugal_kernel_family;

#define FUGAL_MAX_RECORDED_ERRORS 256

const char* fugal_status_string(int status);
const char* fugal_last_error(void);
int fugal_version(void);

/* ======================= mirrors of cuda_kernels (kernels.cpp:4-30) ======= */

/* adjacency_matmul (kernels.cpp:5-7; cuda_kernels/adjacency.cu:77-150).
 * out = (negate ? -A : A) @ M for the n x n CSR matrix A (int32 indices).
 * m_transposed == 0: M row-major (ldm), out row-major (ldo).
 * m_transposed == 1: M is the transpose of a row-major Q (M = Q^T, Q has leading
 *   dimension ldm) and out is written column-major, i.e. out^T row-major with
 *   leading dimension ldo -- the strides torch.empty_like(M) gives a transposed
 *   view, which is what the reference's cuSPARSE call writes (adjacency.cu:93,116). */
fugal_status fugal_adjacency_matmul(const int32_t* col_indices, const int32_t* row_pointers, int64_t n,
                                    const float* M, int64_t ldm, int m_transposed, float* out, int64_t ldo,
                                    int negate, fugal_stream_t stream);

/* create_adjacency (kernels.cpp:8; cuda_kernels/adjacency.cu:228-259).
 * edges: edge_count int32 pairs (x, y) as cugal/adjacency.py:68-69 flattens
 * them; row y of the CSR receives column x, columns ascending within a row.
 * Every row pointer is written, including rows without edges. */
fugal_status fugal_create_adjacency_workspace_size(int64_t edge_count, int64_t node_count, size_t* bytes);
fugal_status fugal_create_adjacency(const int32_t* edges, int64_t edge_count, int64_t node_count,
                                    int32_t* col_indices, int32_t* row_pointers, void* workspace,
                                    size_t workspace_bytes, fugal_stream_t stream);

/* graph_features (kernels.cpp:11; cuda_kernels/feature_extraction.cu:67-84).
 * degrees[v] = deg(v); clustering[v] = t(v) / (deg (deg-1)) with
 * t(v) = sum_{u in N(v)} |N(v) & N(u)| (integer), 0 when t == 0 or deg < 2.
 * Optional integer outputs: degree_counts (int32) and triangle_counts (t, int64). */
fugal_status fugal_graph_features(const int32_t* col_indices, const int32_t* row_pointers, int64_t n,
                                  float* clustering, float* degrees, int32_t* degree_counts,
                                  int64_t* triangle_counts, fugal_stream_t stream);

/* average_neighbor_features (kernels.cpp:12-14; feature_extraction.cu:108-125).
 * averages[v] = (FP32 sum of features over N(v) in CSR order) / deg(v), 0 if deg == 0. */
fugal_status fugal_average_neighbor_features(const int32_t* col_indices, const int32_t* row_pointers,
                                             int64_t n, const float* features, float* averages,
                                             fugal_stream_t stream);

/* sinkhorn_log_step (kernels.cpp:17; cuda_kernels/sinkhorn_log.cu:100-114).
 * out[r] = (1 - w) out[r] - w * LSE_c(K[r, c] + add[c]); |w - 1| < 1e-4 writes -LSE. */
fugal_status fugal_sinkhorn_log_step(const float* K, int64_t rows, int64_t cols, int64_t ldk,
                                     const float* add, float* out, float momentum, fugal_stream_t stream);

/* sinkhorn_log_marginal (kernels.cpp:18; cuda_kernels/sinkhorn_log.cu:88-98).
 * *result = sum over rows (axis 1, as the reference kernel) or columns (axis 0,
 * as cugal/sinkhorn.py:67-76) of |sum exp(K + u_r + v_c) - 1|, accumulated in FP64
 * into the DEVICE double `result`. */
fugal_status fugal_sinkhorn_log_marginal(const float* K, int64_t n, int64_t ldk, const float* u,
                                         const float* v, int axis, double* result, fugal_stream_t stream);

/* add_distance (kernels.cpp:21; cuda_kernels/distance.cu:35-53).
 * out[x][y] += ||source[x] - target[y]||_2 over the 4 feature columns (direct differences). */
fugal_status fugal_add_distance(const float* source, const float* target, int64_t n, float* out,
                                int64_t ldo, fugal_stream_t stream);

/* regularize (kernels.cpp:24; cuda_kernels/regularize.cu:24-39): G += it - 2 it P. */
fugal_status fugal_regularize(float* gradient, int64_t ldg, const float* P, int64_t ldp, int64_t n,
                              int iteration, fugal_stream_t stream);

/* update_quasi_permutation_log (kernels.cpp:27; update_quasi_permutation.cu:37-56).
 * q = exp(K + u_r + v_c); P += alpha (q - P); *gap = sum (q - P)(-reg K) in FP64
 * (DEVICE double; the reference returns |gap| to the host). */
fugal_status fugal_update_quasi_permutation_log(float* P, int64_t ldp, const float* K, int64_t ldk,
                                                const float* u, const float* v, int64_t n, float alpha,
                                                float regularization, double* gap, fugal_stream_t stream);

/* Greedy rounding (replaces cugal/greedy_lap.py:7-85, which the reference runs
 * as n sequential torch launches with a host read each; dense_hungarian,
 * kernels.cpp:30, is exported but never called by cugal).  columns_out[r] is the
 * column of row r; with mutate != 0, P is changed as the reference changes it
 * (row r multiplied by the columns still free when r was processed). order: the
 * row order for FUGAL_LAP_ORDERED (int64 device array), else ignored. */
fugal_status fugal_greedy_lap_workspace_size(int64_t n, int candidates, size_t* bytes);
fugal_status fugal_greedy_lap(float* P, int64_t ldp, int64_t n, int method, const int64_t* order,
                              int candidates, int mutate, int64_t* columns_out, void* workspace,
                              size_t workspace_bytes, fugal_stream_t stream);

/* MORE_RAND rounding (cugal/greedy_lap.py:34-48, a Python loop of n launches with
 * a host draw each): rows in the caller's order order[k]; row r is masked by the
 * columns still free (row *= taken, written back when mutate != 0) and takes the
 * first column j whose running sum of the masked row reaches total * uniforms[k]
 * (uniforms[k]: the k-th random.random() draw, so total * uniforms[k] is the
 * reference's random.uniform(0, cumsum[-1])).  Sums in FP64.  order: int64
 * device array, uniforms: double device array, both of length n; n <= 2^19. */
fugal_status fugal_sampled_lap(float* P, int64_t ldp, int64_t n, const int64_t* order, const double* uniforms,
                               int mutate, int64_t* columns_out, fugal_stream_t stream);

/* Exact assignment with the same mapping as scipy.optimize.linear_sum_assignment
 * (the reference's HungarianMethod.SCIPY rounding, cugal/pred.py:151-158): cost
 * c = -P (maximize != 0) or P, converted to double; Crouse's shortest augmenting
 * path with scipy's candidate order and tie rules, so ties resolve as scipy
 * resolves them.  columns_out[r] = column of row r (int64, device).  The search
 * stops after max_steps Dijkstra steps in total.  *status_out (device int32)
 * receives FUGAL_OK, FUGAL_ITER_LIMIT (cap hit; columns_out not written),
 * FUGAL_NONFINITE (NaN, or -inf cost) or FUGAL_BAD_ARGUMENT (infeasible);
 * *steps_out (device int64, nullable) the steps taken. */
fugal_status fugal_exact_lap_workspace_size(int64_t n, size_t* bytes);
fugal_status fugal_exact_lap(const float* P, int64_t ldp, int64_t n, int maximize, int64_t max_steps,
                             int64_t* columns_out, int64_t* steps_out, int32_t* status_out, void* workspace,
                             size_t workspace_bytes, fugal_stream_t stream);

/* count of entries of P (n x n) that are <= threshold (cugal/pred.py:152-153), into a DEVICE int64. */
fugal_status fugal_count_le(const float* P, int64_t ldp, int64_t n, float threshold, int64_t* count,
                            fugal_stream_t stream);

/* Overlap of an alignment with the planted one, the integer behind the
 * reference's EC / ICS / S3 metrics (benchmark/experiment.py:115-144):
 *   *overlap = |{(i, j) : A[answer_i][answer_j] = 1 and B[truth_i][truth_j] = 1}|
 * over the stored entries of the CSR graphs A and B (columns sorted per row).
 * answer and truth are int64 device arrays of length n.  *not_permutation
 * (device int32) gets bit 0 when answer is not a permutation of 0..n-1 (overlap
 * not computed; use the dense definition) and bit 1 when truth has an entry
 * outside 0..n-1. */
fugal_status fugal_alignment_overlap_workspace_size(int64_t n, size_t* bytes);
fugal_status fugal_alignment_overlap(const int32_t* a_row_pointers, const int32_t* a_col_indices,
                                     const int32_t* b_row_pointers, const int32_t* b_col_indices, int64_t n,
                                     const int64_t* answer, const int64_t* truth, uint64_t* overlap,
                                     int32_t* not_permutation, void* workspace, size_t workspace_bytes,
                                     fugal_stream_t stream);

/* Scaling-form Sinkhorn, SinkhornState.solve_standard (cugal/sinkhorn.py:122-144),
 * on K = exp(-C/reg) (FP32, n x n, ldk): per iteration
 *   v <- v^(1-w) (1 / (u K + 1e-16))^w,  u <- u^(1-w) (1 / (K v + 1e-16))^w,
 * the column-marginal error sum_j |sum_i u_i K_ij v_j - 1| at iterations 0,
 * eval_freq, 2 eval_freq, ... (stop below threshold, Lehmann momentum from
 * momentum_start, < 0 for none), at most max_iterations iterations.  u, v (FP32,
 * device) are read and written in place (warm start).  record: optional DEVICE
 * fugal_solve_record.  fugal_exp_scale writes out = exp(scale * C) (K from C with
 * scale = -1/reg); fugal_fw_update_standard is the update of cugal/pred.py:77-86
 * for this method: q = K v u, P += alpha (q - P), *gap = sum C (q - P) in FP64. */
fugal_status fugal_sinkhorn_standard_workspace_size(int64_t n, size_t* bytes);
fugal_status fugal_sinkhorn_standard_solve(const float* K, int64_t ldk, int64_t n, float* u, float* v,
                                           int max_iterations, double threshold, int eval_freq, int momentum_start,
                                           void* record, void* workspace, size_t workspace_bytes,
                                           fugal_stream_t stream);
fugal_status fugal_exp_scale(const float* C, int64_t ldc, int64_t n, double scale, float* out, int64_t ldo,
                             fugal_stream_t stream);
fugal_status fugal_fw_update_standard(int64_t n, float* P, int64_t ldp, const float* K, int64_t ldk, const float* u,
                                      const float* v, const float* C, int64_t ldc, double alpha, double* gap,
                                      fugal_stream_t stream);

/* Differentiation of the log-domain solve (no counterpart in the reference, which
 * has no backward pass; the torch autograd of its solve_log is the check).
 * fugal_sinkhorn_plan: P = exp(cost32 + u_i + v_j).  fugal_plan_matvec: with
 * M = P (W == NULL) or P o W, Py = M y and Ptx = M^T x (FP64 vectors, one pass
 * over M).  fugal_sinkhorn_adjoint: out = scale * P o (G - alpha_i - beta_j), the
 * cost gradient of the implicit adjoint (scale = -1/reg) once alpha, beta solve
 * [I P; P^T I][alpha; beta] = [(P o G) 1; (P o G)^T 1]. */
fugal_status fugal_sinkhorn_plan(const float* cost32, int64_t ld32, int64_t n, const float* u, const float* v,
                                 float* P, int64_t ldp, fugal_stream_t stream);
fugal_status fugal_plan_matvec_workspace_size(int64_t n, size_t* bytes);
fugal_status fugal_plan_matvec(const float* P, int64_t ldp, const float* W, int64_t ldw, int64_t n,
                               const double* x, const double* y, double* Ptx, double* Py, void* workspace,
                               size_t workspace_bytes, fugal_stream_t stream);
fugal_status fugal_sinkhorn_adjoint(const float* P, int64_t ldp, const float* G, int64_t ldg, int64_t n,
                                    const double* alpha, const double* beta, double scale, float* out, int64_t ldo,
                                    fugal_stream_t stream);
/* Unrolled backward of one half step of the log-domain iteration (no momentum),
 * for the checkpointed unrolled adjoint.  axis 1: out = -LSE_j(K_ij + other_j)
 * (row update); axis 0: out = -LSE_i(K_ij + other_i) (column update).  With
 * E = exp(K + other + out) in that orientation and g = dL/d(out) (FP64):
 * gK -= g o E (FP32, in place) and g_other -= the reduction of g o E over the
 * LSE axis (FP64, accumulated).  Workspace as fugal_plan_matvec_workspace_size. */
fugal_status fugal_sinkhorn_unrolled_step_backward(const float* K, int64_t ldk, int64_t n, const float* out_dual,
                                                   const float* other_dual, const double* g, int axis, float* gK,
                                                   int64_t ldg, double* g_other, void* workspace,
                                                   size_t workspace_bytes, fugal_stream_t stream);

/* ======================= fused Frank-Wolfe step (cugal/pred.py:89-148) ===== */

/* Gradient with the Sinkhorn kernel matrix fused into its epilogue
 * (cugal/pred.py:54-74 sparse_gradient + add_feature_distance :30-35 +
 * regularize + K = -C/reg at cugal/sinkhorn.py:98), for symmetric A and B:
 *   C[i][j]   = -2 (A P B)[i][j] + ||Fs_i - Ft_j|| + lambda_scale * lambda * (1 - 2 P[i][j])   (FP32)
 *   out[i][j] = out_scale * C[i][j] + U[i] + V[j]          (FP64 arithmetic, FP32 store)
 * out_scale = -1/reg with U, V the accumulated duals gives the absorbed Sinkhorn
 * input; out_scale = 1, U = V = NULL gives the plain gradient.  Features are the
 * n x 4 mu-scaled feature rows; alternatively D (n x n, ldd) is a stored distance
 * matrix read instead (the reference's recompute_distance=False input); with
 * neither there is no distance term.  lambda_scale is 1 for
 * the sparse reference path and 2 for its dense path (cugal/pred.py:46-50). */
fugal_status fugal_gradient_workspace_size(int64_t n, size_t* bytes);
fugal_status fugal_fw_gradient(int64_t n, const int32_t* a_row_pointers, const int32_t* a_col_indices,
                               const int32_t* b_row_pointers, const int32_t* b_col_indices, const float* P,
                               int64_t ldp, const float* source_features, const float* target_features,
                               const float* D, int64_t ldd, double lambda, double lambda_scale,
                               double out_scale, const double* U, const double* V, float* out, int64_t ldo,
                               void* workspace, size_t workspace_bytes, fugal_stream_t stream);

/* fugal_fw_gradient that also hands the Sinkhorn solve its first column update
 * (cugal/sinkhorn.py:105, v = -logsumexp over rows of K + u, u = 0 in the
 * absorbed frame), so the solve does not read the cost for it: for every panel
 * c of 128 output rows (c < chunks, fugal_gradient_column_chunks) and column j,
 * column_partials[c * ldc + j] = (M, S) as two floats, M = max of out_ij log2 e
 * over the panel's rows, S = sum of 2^(out_ij log2 e - M).  Pass the same
 * buffer, chunks and ldc to fugal_sinkhorn_solve (column_partials fields). */
fugal_status fugal_gradient_column_chunks(int64_t n, int32_t* chunks);
fugal_status fugal_fw_gradient_column_stats(int64_t n, const int32_t* a_row_pointers,
                                            const int32_t* a_col_indices, const int32_t* b_row_pointers,
                                            const int32_t* b_col_indices, const float* P, int64_t ldp,
                                            const float* source_features, const float* target_features,
                                            const float* D, int64_t ldd, double lambda, double lambda_scale,
                                            double out_scale, const double* U, const double* V, float* out,
                                            int64_t ldo, void* workspace, size_t workspace_bytes,
                                            float* column_partials, int64_t ldc, fugal_stream_t stream);

/* No counterpart in the reference.  fugal_fw_gradient for callers that cannot
 * allocate device memory (a host whose device memory belongs to a pool allocator
 * every allocation must go through, or a binding that only passes input and
 * output pointers): same arguments and result, minus the workspace, which comes
 * from one FUGAL_FIXED_SCRATCH_BYTES array compiled into the library.  Every GPU
 * on which the library's device code is loaded holds that array until the
 * process exits.  n above FUGAL_FIXED_SCRATCH_MAX_N is rejected with
 * FUGAL_BAD_SHAPE.  The call allocates nothing.  Its first call on a device (that
 * device current) looks up the array's device address; make that first call
 * before any stream capture.  The address is kept per device for the runtime's
 * primary context: after a cudaDeviceReset, or from another driver context, the
 * kept address is stale, so such callers must not use this entry point.  All
 * calls on a device share the array and it keeps the last call's contents
 * (nothing in it needs to start at zero); calls whose kernels overlap on the GPU
 * race on it, so order them on one stream. */
#define FUGAL_FIXED_SCRATCH_BYTES (16 * 1024 * 1024)
#define FUGAL_FIXED_SCRATCH_MAX_N 2048
fugal_status fugal_fw_gradient_fixed_scratch(int64_t n, const int32_t* a_row_pointers,
                                             const int32_t* a_col_indices, const int32_t* b_row_pointers,
                                             const int32_t* b_col_indices, const float* P, int64_t ldp,
                                             const float* source_features, const float* target_features,
                                             const float* D, int64_t ldd, double lambda, double lambda_scale,
                                             double out_scale, const double* U, const double* V, float* out,
                                             int64_t ldo, fugal_stream_t stream);

/* Log-domain Sinkhorn solve (cugal/sinkhorn.py:90-120) on the absorbed cost
 * cost32 = K + U_i + V_j, warm-started at u = v = 0 relative to that frame.
 * Same iteration as the reference: per iteration a column then a row update
 * (Lehmann momentum from sinkhorn_momentum_start), the column-marginal L1 error
 * checked after iterations eval_freq, 2 eval_freq, ... against threshold, at most
 * max_iterations iterations.  Each sweep reads the cost once: the row update and
 * the next column update's sums are fused.  With stream_dtype BF16/F16 the solve
 * switches, after fp32_warmup_sweeps, to the reduced-precision copy `cost16`
 * (which it writes, refreshed every reabsorb_every sweeps), then runs
 * polish_sweeps FP32 sweeps.  Outputs: u_out / v_out (FP32, n) in the frame of
 * cost32, and an optional DEVICE fugal_solve_record.  Padding columns [n, ld)
 * of cost32 and cost16 must hold finite values (zero them once). */
typedef struct {
    int64_t n;
    const float* cost32;
    int64_t ld32;
    void* cost16;
    int64_t ld16;
    int stream_dtype;
    int max_iterations;
    double threshold;
    int eval_freq;
    int momentum_start; /* < 0: no momentum (Config.sinkhorn_momentum_start = None) */
    int fp32_warmup_sweeps;
    int reabsorb_every;
    int polish_sweeps;
    float* u_out;
    float* v_out;
    void* record; /* fugal_solve_record* in device memory, or NULL */
    /* Optional (NULL: the solve reads cost32 for it): base-2 column (max, sum)
     * partials of cost32 from fugal_fw_gradient_column_stats, chunks x ldc
     * float pairs, merged into the first column update. */
    const float* column_partials;
    int32_t column_partial_chunks;
    int64_t column_partial_ld;
} fugal_solve_params;

typedef struct {
    int32_t iteration_count; /* iterations of the main phase (SinkhornProfile.iteration_count) */
    int32_t n_errors;        /* entries of errors[] (SinkhornProfile.errors) */
    int32_t status;          /* FUGAL_OK or FUGAL_DEVICE_TIMEOUT */
    int32_t polish_count;
    double last_error;       /* column-marginal L1 error after the last main-phase sweep */
    double polish_error;     /* after the polish sweeps (FP32 cost) */
    double errors[FUGAL_MAX_RECORDED_ERRORS];
} fugal_solve_record;

fugal_status fugal_sinkhorn_workspace_size(int64_t n, int stream_dtype, size_t* bytes);
/* Launch shape of the sweeps over an n-column cost of stream_dtype on the
 * current device: info = {threads per CTA, CTAs per cluster, clusters in the
 * grid, pipeline stages, dynamic shared memory bytes, rows per batch}. */
fugal_status fugal_sinkhorn_plan_info(int64_t n, int stream_dtype, int32_t* info);
fugal_status fugal_sinkhorn_solve(const fugal_solve_params* params, void* workspace, size_t workspace_bytes,
                                  fugal_stream_t stream);

/* Frank-Wolfe update (cugal/pred.py:133-141 and update_quasi_permutation.cu:7-35)
 * on the absorbed cost: q = exp(cost32 + u_i + v_j), P += alpha (q - P),
 * *gap = sum (q - P) C with C = -reg (cost32 - U_i - V_j) (FP64, DEVICE double).
 * commit != 0 then folds the duals into the frame: U += u, V += v. */
fugal_status fugal_fw_update(int64_t n, float* P, int64_t ldp, const float* cost32, int64_t ld32,
                             const float* u, const float* v, double* U, double* V, double alpha,
                             double regularization, double* gap, int commit, fugal_stream_t stream);

/* ============ structural term kept across Frank-Wolfe steps ==============
 * No counterpart in the reference, which forms -A P B from scratch with two
 * SpMMs every step (cugal/pred.py:54-74).  With the fixed step of
 * cugal/pred.py:133-141, P' = (1 - alpha) P + alpha q, so M = A P B follows
 *   M' = (1 - alpha) M + alpha A q B,
 * and once the Sinkhorn plan q has few nonzero entries per row (one per row
 * for a converged solve at small regularization) A q B is a sparse product.
 * The gradient then reads a stored M instead of gathering P through A and B.
 *
 * M is kept as int64 fixed point: M[i][j] = Mq[i][j] * 2^-frac_bits * scale,
 * with scale (the product of the (1 - alpha) factors since the last refresh)
 * and frac_bits held by the caller.  A step only adds to the entries that A q B
 * touches; integer addition is associative, so the sums do not depend on the
 * order of the atomic adds and reruns are bit-identical.  Choose frac_bits so
 * that d_max * FUGAL_PLAN_ROW_SUM_MAX * 2^frac_bits / scale < 2^52, d_max the
 * largest degree of A, for every scale used between refreshes.
 *
 * flags: two device int32, zeroed by the caller.  flags[0] != 0: the scatter
 * met a plan row with more than `slots` nonzero entries or a row sum above
 * FUGAL_PLAN_ROW_SUM_MAX (that row is not added: Mq is stale until the next
 * refresh).  flags[1] != 0: a refresh met a value outside the fixed-point range
 * (Mq unusable). */
#define FUGAL_PLAN_ROW_SUM_MAX 32.0f
typedef struct {
    int32_t column;
    float value;
} fugal_plan_entry;

/* rows[e] = the row of edge e of an n-row CSR matrix, e < nnz = row_pointers[n]. */
fugal_status fugal_csr_edge_rows(const int32_t* row_pointers, int64_t n, int64_t nnz, int32_t* rows,
                                 fugal_stream_t stream);

/* Mq[i][j] = round((A P B)[i][j] * 2^frac_bits) for i, j < n (the SpMM pair of
 * fugal_fw_gradient, same workspace); flags[1] is set on a value >= 2^52. */
fugal_status fugal_structural_refresh(int64_t n, const int32_t* a_row_pointers, const int32_t* a_col_indices,
                                      const int32_t* b_row_pointers, const int32_t* b_col_indices, const float* P,
                                      int64_t ldp, int64_t* Mq, int64_t ldm, int32_t frac_bits, void* workspace,
                                      size_t workspace_bytes, int32_t* flags, fugal_stream_t stream);

/* fugal_fw_update that also records the plan's nonzero entries: for each row k,
 * plan_counts[k] = the number of j with q_kj > 0, and min(count, slots) of them
 * as (j, q_kj) at plan_entries[k * slots ...], in no particular order. */
fugal_status fugal_fw_update_collect(int64_t n, float* P, int64_t ldp, const float* cost32, int64_t ld32,
                                     const float* u, const float* v, double* U, double* V, double alpha,
                                     double regularization, double* gap, int commit, int32_t* plan_counts,
                                     fugal_plan_entry* plan_entries, int32_t slots, fugal_stream_t stream);

/* Mq[i][j] += round(q_kl * increment_scale) for every recorded plan entry
 * (k, l, q_kl), i in N_A(k), j in N_B(l) (A, B symmetric, so this adds
 * round(increment_scale q) through A q B); a_edge_rows from fugal_csr_edge_rows
 * on A, a_nnz its edge count.  Does nothing when flags[0] or flags[1] is set on
 * entry; sets flags[0] (and skips the row) for a row whose count exceeds slots
 * or whose entries sum above FUGAL_PLAN_ROW_SUM_MAX. */
fugal_status fugal_structural_scatter(int64_t n, const int32_t* a_col_indices, const int32_t* a_edge_rows,
                                      int64_t a_nnz, const int32_t* b_row_pointers,
                                      const int32_t* b_col_indices, const int32_t* plan_counts,
                                      const fugal_plan_entry* plan_entries, int32_t slots, double increment_scale,
                                      int64_t* Mq, int64_t ldm, const int32_t* flags, fugal_stream_t stream);

/* The gradient of fugal_fw_gradient (column_partials != NULL: of
 * fugal_fw_gradient_column_stats) with (A P B)[i][j] = (float)(Mq[i][j] * m_scale)
 * in place of the SpMM pair.  shift > 0 also rescales Mq in place by 2^-shift
 * (rounded), for the caller to multiply its scale by 2^shift. */
fugal_status fugal_fw_gradient_structural(int64_t n, int64_t* Mq, int64_t ldm, double m_scale, int32_t shift,
                                          const float* P, int64_t ldp, const float* source_features,
                                          const float* target_features, const float* D, int64_t ldd,
                                          double lambda, double lambda_scale, double out_scale, const double* U,
                                          const double* V, float* out, int64_t ldo, float* column_partials,
                                          int64_t ldc, fugal_stream_t stream);

/* Exact line search, opt-in (Config.line_search).  No counterpart in the
 * reference, which steps with alpha = 2/(2+it) (cugal/pred.py:133-141).  On the
 * objective f(P) = -<P, A P B> + <D, P> + lam' <P, 1 - P>, whose gradient is the
 * one fugal_fw_gradient builds, f(P + a d) - f(P) = a g + a^2 Q exactly, with
 * d = q - P, g = <G, d>, Q = -<d, A d B> - lam' <d, d>.  Three calls:
 *
 * fugal_fw_direction: dir = q - P (FP32, columns [0, n) written) and, in FP64,
 * sums[0] = g, sums[1] = <d, d>, sums[2] = 0 (sums: 3 DEVICE doubles).  Log form
 * (K == NULL): q = exp(cost32 + u_i + v_j), G = -reg (cost32 - U_i - V_j), and
 * commit != 0 folds the duals as fugal_fw_update does.  Scaling form: q =
 * (K_ij v_j) u_i, G = cost32 (the plain gradient), U = V = NULL, commit = 0.
 *
 * fugal_fw_gradient with P := dir, no features or distance, lambda = 0,
 * out_scale = 1, U = V = NULL gives W = -2 A d B.
 *
 * fugal_fw_line_search_update: sums[2] = <d, W>, then a = argmin over [0, 1] of
 * a g + a^2 Q with Q = sums[2]/2 - lambda_eff sums[1] (Q > 0: -g/2Q clipped;
 * else 1 if g + Q < 0, else 0), P += a dir, *alpha = a and *gap = g (DEVICE
 * doubles; either may be NULL).  lambda_eff = lambda * lambda_scale of the
 * gradient.  Nothing is read back to the host. */
fugal_status fugal_fw_direction(int64_t n, const float* P, int64_t ldp, const float* cost32, int64_t ld32,
                                const float* K, int64_t ldk, const float* u, const float* v, double* U, double* V,
                                double regularization, float* dir, int64_t ldd, double* sums, int commit,
                                fugal_stream_t stream);
fugal_status fugal_fw_line_search_update(int64_t n, float* P, int64_t ldp, const float* dir, int64_t ldd,
                                         const float* W, int64_t ldw, double lambda_eff, double* sums,
                                         double* alpha, double* gap, fugal_stream_t stream);

/* ======================= instrumentation ================================== */
/* When enabled, every kernel of the families above is bracketed by CUDA events
 * on its launch stream; totals are accumulated when a solve polls its progress
 * or on fugal_timing_query(), which synchronises the recorded events. */
void fugal_timing_enable(int on);
void fugal_timing_reset(void);
fugal_status fugal_timing_query(int family, int64_t* launches, double* milliseconds);
/* Kernels launched by this library since load (all families). */
int64_t fugal_launch_count(void);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* FUGAL_B200_H */
