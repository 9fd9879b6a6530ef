/* vajra_pdhg.h -- C ABI of the B200 (sm_100a) restarted-PDHG LP backend.
 *
 * The library (libvajra_pdhg.so) replaces the reference's src/solvers/gpu/ backend:
 * gpu_context.cpp (probe + dispatch), pdhg_cuda.cu (host driver) and spmv_kernels.cuh
 * (device kernels).  All entry points are plain C: POD structs, host or device pointers
 * with explicit sizes, an int32 status, and no exceptions across the boundary.  A C++20
 * shim (vajra-opt_b200/shim/indus_gpu_dropin.cpp) maps the reference's C++ surface
 * indus::gpu::{solve_pdhg_gpu, probe_device, is_cuda_available, get_last_gpu_timing}
 * (include/indus/gpu.hpp:49-59) onto these functions.
 *
 * Conventions (same as the reference Model, include/indus/model.hpp:16-55):
 *   - A is m x n in CSC: col_ptr[n+1] (int64), row_idx[nnz] (int32, ascending within a
 *     column, no duplicates), values[nnz] (double).
 *   - Infinite bounds are +-1e20 (or beyond).
 *   - row_dual uses the verifier's sign convention (<= row: y <= 0, >= row: y >= 0),
 *     col_dual = c - A^T row_dual, row_value = A x, objective includes objective_offset.
 *   - status values are indus::SolveStatus (include/indus/types.hpp:34-47).
 * There is no CPU fallback: without a usable CUDA device every solve returns
 * VAJRA_ERR_NO_DEVICE and status UNSUPPORTED.
 */
#ifndef VAJRA_PDHG_H
#define VAJRA_PDHG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Layout version of the structs below.  A caller compiled against one version must not call
 * a library of another: compare with vajra_abi_version() before the first call. */
#define VAJRA_ABI_VERSION 8

typedef int32_t vajra_status;
enum {
    VAJRA_OK = 0,
    VAJRA_ERR_INVALID_ARGUMENT = 1,
    VAJRA_ERR_NO_DEVICE = 2,
    VAJRA_ERR_CUDA = 3,
    VAJRA_ERR_OUT_OF_MEMORY = 4,
    VAJRA_ERR_WAIT_TIMEOUT = 5,  /* reserved: no entry point waits on the device today      */
    VAJRA_ERR_INTERNAL = 6
};

/* indus::SolveStatus values (include/indus/types.hpp:34-47). */
enum {
    VAJRA_SOLVE_NOT_SOLVED = 0,
    VAJRA_SOLVE_OPTIMAL = 1,
    VAJRA_SOLVE_UNBOUNDED = 3,
    VAJRA_SOLVE_FEASIBLE = 5,
    VAJRA_SOLVE_ITERATION_LIMIT = 6,
    VAJRA_SOLVE_TIME_LIMIT = 7,
    VAJRA_SOLVE_NUMERICAL_ERROR = 9,
    VAJRA_SOLVE_MODEL_ERROR = 10,
    VAJRA_SOLVE_UNSUPPORTED = 11
};

/* Algorithms. */
enum {
    /* CpuPdhgSolver::solve semantics (src/solvers/pdhg/pdhg.cpp:70-440) in FP64 on the
     * device, evaluated in the reference's operation order: Ruiz (10 passes), power-
     * iteration norm, tau = sigma = 0.95/||A||, checks every check_frequency, tau/sigma
     * rebalancing, stagnation restart, best-iterate return.  Bit-identical to the
     * reference CPU solver on the same input. */
    VAJRA_ALGO_REFERENCE = 0,
    /* Restarted reflected Halpern PDHG with KKT-based adaptive restarts and primal-weight
     * updates, terminated on the FP64 relative KKT error of the original problem. */
    VAJRA_ALGO_HALPERN = 1
};

/* Precision of VAJRA_ALGO_HALPERN (VAJRA_ALGO_REFERENCE is always FP64). */
enum {
    VAJRA_PREC_FP64 = 0,   /* "plain" form: FP64 values, iterates and accumulation       */
    VAJRA_PREC_MIXED = 1,  /* FP32 values/iterates/SpMV accumulation, FP64 KKT, gap,
                              restart and primal-weight decisions, then an FP64 polish
                              restarted from the FP32 iterate                            */
    VAJRA_PREC_FP32 = 2    /* vajra_pdhg_unrolled only: the FP32 map and reverse pass    */
};

/* The reference Model (include/indus/model.hpp:16-55) as CSC host arrays. */
typedef struct vajra_lp {
    int32_t num_rows;
    int32_t num_cols;
    int64_t nnz;
    const int64_t* col_ptr;
    const int32_t* row_idx;
    const double* values;
    const double* c;
    const double* col_lower;
    const double* col_upper;
    const double* row_lower;
    const double* row_upper;
    int32_t sense;             /* 0 minimise, 1 maximise (ObjSense)                     */
    double objective_offset;
} vajra_lp;

/* Solver options: the PDHG keys of indus::Options (include/indus/options.hpp:10-41,
 * read at src/solvers/pdhg/pdhg.cpp:58-68) plus this backend's own settings. */
typedef struct vajra_opts {
    int32_t algorithm;          /* VAJRA_ALGO_*                                          */
    int32_t precision;          /* VAJRA_PREC_* (HALPERN only)                           */
    double tolerance;           /* REFERENCE: max-abs primal and dual residual
                                   ("tolerance"); HALPERN: relative KKT target           */
    double gap_tolerance;       /* REFERENCE: relative gap ("gap_tolerance")             */
    double time_limit;          /* seconds (Options::time_limit)                         */
    int64_t iteration_limit;    /* Options::iteration_limit                              */
    int32_t check_frequency;    /* REFERENCE: "check_frequency" (100); HALPERN: KKT /
                                   restart evaluation interval (64)                      */
    int32_t enable_scaling;     /* Options::enable_scaling                               */
    int32_t pock_chambolle;     /* HALPERN: 1 = Pock-Chambolle (alpha = 1) after Ruiz     */
    int32_t ruiz_iterations;    /* 10 (tol::kMaxRuizIterations)                          */
    double reflection;          /* HALPERN: reflection coefficient of the Halpern step   */
    double mixed_switch_tolerance; /* MIXED: FP32 phase hands over to FP64 below this
                                      relative KKT (2e-6), or when FP32 stalls            */
    int32_t device;             /* CUDA device ordinal                                   */
    int32_t autotune;           /* 1 = time SpMV variants at set-up and keep the fastest */
    int32_t verbose;            /* 1 = one line per check on stderr                      */
    int32_t mixed_stall_checks; /* MIXED: hand over when the relative KKT gained < 2 % over
                                   this many checks (20; 0 = never; at most 31)          */
    /* HALPERN restart and step parameters */
    double restart_sufficient;  /* restart when weighted KKT <= this x its restart value (0.2) */
    double restart_necessary;   /* ... or <= this x and rising (0.8)                     */
    double restart_artificial;  /* ... or inner iterations >= this x total (0.36)        */
    double primal_weight_smoothing; /* theta of omega <- exp(theta log(dy/dx) + (1-theta) log omega) (0.5) */
    double step_safety;         /* eta = step_safety / ||A||_2 (0.99)                    */
    int32_t restart_metric;     /* 0: primal-weighted KKT of T(z); 1: fixed-point residual
                                   sqrt(omega ||x+ - x||^2 + ||y+ - y||^2 / omega)          */
    int32_t spmv_shape_a;       /* HALPERN launch shape of the A x SpMV: 0 autotune (>= 2^20
                                   entries) or the set-up heuristic, -1 row-block kernel,
                                   -2 row-block kernel with two load groups per thread,
                                   -3 sliced ELL (degree-ordered LPs; else the row-block
                                   kernel), -4 sliced ELL with the first vector entries in
                                   shared memory, 1..32 lanes per row (1, 2, 4, 8, 16, 32)   */
    int32_t spmv_shape_at;      /* the same for the A^T y SpMV                           */
    double mixed_reflection;    /* MIXED: reflection coefficient of the FP32 phase once its
                                   relative KKT is within 10x of mixed_switch_tolerance (0.8);
                                   above that, and in the FP64 phase, `reflection` applies.
                                   Below 1 the reflected step is averaged, which keeps FP32
                                   rounding noise from building up within a restart epoch  */
    int32_t degree_order;       /* HALPERN: renumber rows and columns by descending entry
                                   count on the device, so that the vector entries the SpMVs
                                   gather most often share cache lines; results come back in
                                   the caller's numbering.  0 auto (on from 2^20 entries),
                                   1 on, -1 off                                            */
    int32_t pow2_scaling;       /* HALPERN: 1 = round the final row / column scale factors to
                                   the nearest power of two, so that scaling is exact: a
                                   matrix whose values fit FP32 still fits it once scaled (0) */
    int32_t fp64_value_storage; /* HALPERN FP64 iterations and every FP64 check: where each
                                   scaled value is exactly an FP32 number, read the FP32 copy
                                   of the matrix (4 bytes an entry instead of 8; FP64 vectors
                                   and sums, so every result is bit-identical).  0 auto (MIXED:
                                   on when exact; FP64 form: off), 1 FP64 copy always, 2 the
                                   FP32 copy when exact in either precision                  */
    int32_t handover_mode;      /* MIXED: 0 = the FP64 phase restarts from the FP32 candidate
                                   (a new Halpern epoch anchored there); 1 = it continues the
                                   FP32 phase's epoch (iterate, anchor, counter and restart
                                   references carried over); -1 (default) = 1 for LPs of 2^20
                                   entries or more, else 0.  The batched solver restarts.     */
    double max_violation;       /* HALPERN: > 0 also requires, before OPTIMAL, the maxima that
                                   the engine's status guard checks (Solution::recompute_quality,
                                   src/engine/model.cpp:203-374) to be at most this on the
                                   original LP: each row violation over 1 + |its bound|, each
                                   reduced-cost sign violation of a column off its bound, each
                                   row-dual sign violation (0 = relative KKT only)          */
    double max_abs_violation;   /* HALPERN: > 0 also requires every row violation of the
                                   original LP to be at most this in absolute terms (the
                                   reference verifier's check, src/engine/verifier.cpp)      */
} vajra_opts;

/* Caller-owned result.  Vector pointers may be NULL (not copied).  Sizes: col_value and
 * col_dual n, row_value and row_dual m. */
typedef struct vajra_result {
    double* col_value;
    double* row_value;
    double* row_dual;
    double* col_dual;
    int32_t status;             /* VAJRA_SOLVE_*                                         */
    int64_t iterations;
    double objective_value;
    double dual_objective;
    /* PdhgDiagnostics surface (include/indus/pdhg.hpp:30-43); HALPERN reports as the residuals
     * the largest absolute row violation and the largest reduced-cost / row-dual sign
     * violation on the original LP (the status guard's quantities) */
    int32_t restart_count;
    double primal_residual;
    double dual_residual;
    double duality_gap;
    double spectral_norm_estimate;
    double tau;
    double sigma;
    int32_t converged;
    /* FP64 relative KKT of the returned point on the original problem */
    double rel_primal;
    double rel_dual;
    double rel_gap;
    double rel_kkt;
    double primal_weight;
    int64_t fp32_iterations;
    int64_t fp64_iterations;
    /* GpuTimingDiagnostics surface (include/indus/gpu.hpp:37-46) */
    double upload_time_sec;
    double setup_time_sec;
    double iteration_time_sec;
    double download_time_sec;
    double total_time_sec;
    int64_t host_device_transfers;
    int32_t spmv_group_a;       /* SpMV shape chosen for A x: 1..32 lanes per row, 0 the
                                   shared-memory row-block kernel, 64 the same with two load
                                   groups per thread, 128 sliced ELL, 129 sliced ELL with the
                                   hot vector prefix in shared memory, -1 the exact in-order
                                   kernel of VAJRA_ALGO_REFERENCE                            */
    int32_t spmv_group_at;      /* same for A^T y                                           */
    /* Live kernel timing (HALPERN): CUDA-event durations of the fused iteration kernels,
     * sampled on the solve's stream once per check interval, for the precision that ran
     * most iterations, with the algorithmic bytes one launch must move. */
    double primal_kernel_us;    /* v = A^T y + primal prox / Halpern (stored transpose)   */
    double dual_kernel_us;      /* w = A x_bar + dual prox / Halpern (CSR)                 */
    double primal_kernel_bytes;
    double dual_kernel_bytes;
    int64_t kernel_samples;
    int64_t kernel_launches;    /* kernels this solve launched (graph nodes counted per replay) */
    double device_time_sec;     /* CUDA-event time on the solve's stream from the start of the
                                   device set-up to the end of post-processing (no downloads) */
    char status_message[256];
} vajra_result;

/* GpuDeviceInfo (include/indus/gpu.hpp:16-24). */
typedef struct vajra_device_info {
    int32_t available;
    char device_name[256];
    uint64_t total_vram_bytes;
    uint64_t free_vram_bytes;
    int32_t compute_capability_major;
    int32_t compute_capability_minor;
    int32_t multi_processor_count;
} vajra_device_info;

/* GpuTimingDiagnostics (include/indus/gpu.hpp:37-46), per calling thread. */
typedef struct vajra_timing {
    double upload_time_sec;
    double iteration_time_sec;
    double download_time_sec;
    double total_time_sec;
    int64_t host_device_transfers;
    int64_t iterations;
    char device_name[256];
    char kernel_mode[64];
} vajra_timing;

/* DeviceDiagnostics (include/indus/gpu.hpp:27-34). */
typedef struct vajra_device_diagnostics {
    double primal_residual;
    double dual_residual;
    double objective;
    double duality_gap;
    int32_t converged;
    int32_t numerical_error;
} vajra_device_diagnostics;

typedef struct vajra_pdhg vajra_pdhg;  /* opaque: one LP resident on one device */

/* ---- solver ------------------------------------------------------------------ */

/* Fills the defaults (HALPERN, MIXED, tolerance 1e-6, check every 64, ...). */
void vajra_default_opts(vajra_opts* opts);

/* Replaces indus::gpu::solve_pdhg_gpu (include/indus/gpu.hpp:59;
 * src/solvers/gpu/gpu_context.cpp:65-80 -> src/solvers/gpu/pdhg_cuda.cu:109-375):
 * upload, device set-up, iterate, download, all in one call.  Host buffers in and out. */
vajra_status vajra_pdhg_solve(const vajra_lp* lp, const vajra_opts* opts, vajra_result* result);

/* Split form of vajra_pdhg_solve for callers that solve the same LP repeatedly
 * (pdhg_cuda.cu:187-227 upload once): create uploads the LP to the device; run does the
 * device set-up and the solve from the resident copy; destroy frees it. */
vajra_status vajra_pdhg_create(const vajra_lp* lp, const vajra_opts* opts, vajra_pdhg** handle);
/* Batched form: `count` independent LPs solved together (VAJRA_ALGO_HALPERN), packed
 * block-diagonally into one device problem with per-instance scaling (each instance's Ruiz
 * passes end on its own stopping test, as if it were solved alone), step sizes, primal
 * weights, restarts and termination.  VAJRA_PREC_MIXED runs an FP32 pass first (FP32 values,
 * iterates and sums, FP64 checks), in which each instance either reaches the tolerance or -- at
 * mixed_switch_tolerance or on a stall -- hands over to an FP64 pass that restarts it from its
 * FP32 candidate; VAJRA_PREC_FP64 runs the FP64 pass alone.  Each pass runs on the device in
 * graph launches of many chunks; time_limit is checked after each (the first launch of a pass
 * runs 2048 iterations, later ones what fits in the time left at the measured rate).  Replaces a host loop of solve_pdhg_gpu calls (gpu.hpp:59), as
 * the reference's benchmark Suite 2 issues them (apps/benchmark_runner.cpp:936-944).
 * results[i] receives instance i; every result's device_time_sec is the whole batch's. */
vajra_status vajra_pdhg_solve_batch(int32_t count, const vajra_lp* lps, const vajra_opts* opts,
                                    vajra_result* results);
vajra_status vajra_pdhg_run(vajra_pdhg* handle, vajra_result* result);
vajra_status vajra_pdhg_destroy(vajra_pdhg* handle);

/* The device set-up's scaling of one LP, exported so that it can be checked against the
 * reference's host scaling: Ruiz equilibration exactly as RuizScaler::compute_and_scale
 * (src/linalg/scaling.cpp:7-153; opts->ruiz_iterations passes, tolerance 0.05), then -- with
 * opts->pock_chambolle -- the Pock-Chambolle diagonal preconditioner of
 * PockChambollePreconditioner::compute (scaling.cpp:179-220, alpha = 1) applied symmetrically:
 * A <- diag(sqrt(d_row)) A diag(sqrt(d_col)) on the Ruiz-scaled A, which is the same saddle
 * problem as PDHG with the step matrices diag(d_col), diag(d_row).  Outputs (host, any may be
 * NULL): the cumulative row_scale[m] and col_scale[n], the scaled values[nnz] in CSC order, the
 * scaled c[n] (negated for maximisation), col_lower/col_upper[n] and row_lower/row_upper[m]. */
vajra_status vajra_scale_lp(const vajra_lp* lp, const vajra_opts* opts, double* row_scale, double* col_scale,
                            double* values, double* c, double* col_lower, double* col_upper, double* row_lower,
                            double* row_upper);

/* The library keeps released device blocks in a per-device cache (up to 16 GiB, or
 * VAJRA_BLOCK_CACHE_MB megabytes read at the first allocation) so that repeated solves reuse
 * them without driver calls.  This returns every cached block of `device` (every device for a
 * negative ordinal) to the driver and reports the bytes freed; blocks in use by a live solve or
 * handle are not touched.  No counterpart in the reference (it allocates and frees per solve). */
int64_t vajra_release_cached_memory(int32_t device);

/* ---- differentiation: adjoint of the unrolled PDHG map ---------------------------
 * No counterpart in the reference (it has no derivatives); the forward map is the plain
 * PDHG iteration of src/solvers/pdhg/pdhg.cpp:196-241 (primal first, fixed steps
 * tau = sigma = step_safety / ||A_i||_2 after Ruiz + Pock-Chambolle scaling). */
typedef struct vajra_unrolled_opts {
    int32_t iterations;         /* unrolled iterations K (2000)                          */
    int32_t checkpoint_every;   /* forward checkpoint interval (100); segments between
                                   checkpoints are recomputed in the reverse pass         */
    int32_t precision;          /* VAJRA_PREC_MIXED (default): the FP64 map -- forward pass,
                                   checkpoints and the active sets recomputed per segment --
                                   with the reverse pass (cotangents, transposed SpMVs) in
                                   FP32; VAJRA_PREC_FP64: FP64 throughout; VAJRA_PREC_FP32:
                                   the FP32 map and reverse pass                          */
    int32_t enable_scaling;     /* Ruiz + Pock-Chambolle (constants of A)                */
    double step_safety;         /* 0.95                                                   */
    int32_t device;
    int32_t reserved[5];
} vajra_unrolled_opts;

void vajra_default_unrolled_opts(vajra_unrolled_opts* opts);

/* `count` minimisation LPs; vectors are packed over the instances in order (N = sum n_i,
 * M = sum m_i).  Loss of instance i: sum_j (weights_j + c_j) x_j(K), x(K) in original units.
 * loss[count] and x_final[N] are outputs (x_final may be NULL); grad_c[N],
 * grad_row_lower[M], grad_row_upper[M] (any may be NULL; all NULL = forward only) receive
 * dL_i/d(c, row_lower, row_upper) of the unrolled map (an equality row's right-hand side
 * gradient is grad_row_lower + grad_row_upper). */
vajra_status vajra_pdhg_unrolled(int32_t count, const vajra_lp* lps, const vajra_unrolled_opts* opts,
                                 const double* weights, double* loss, double* x_final, double* grad_c,
                                 double* grad_row_lower, double* grad_row_upper);

/* ---- device probe and telemetry ------------------------------------------------ */

/* Replaces indus::gpu::probe_device (gpu.hpp:49; gpu_context.cpp:16-59). */
vajra_status vajra_probe_device(int32_t device, vajra_device_info* info);
/* Replaces indus::gpu::is_cuda_available (gpu.hpp:52; gpu_context.cpp:61-63). */
int32_t vajra_is_cuda_available(void);
/* Replaces indus::gpu::get_last_gpu_timing (gpu.hpp:55; pdhg_cuda.cu:101-107);
 * thread-local instead of the reference's process-global g_last_gpu_timing. */
void vajra_last_timing(vajra_timing* out);
/* Human-readable text for a vajra_status. */
const char* vajra_status_string(vajra_status status);
/* VAJRA_ABI_VERSION the library was built with (no counterpart in the reference). */
int32_t vajra_abi_version(void);

/* ---- kernel-level entry points (device pointers, caller's stream; NULL = default) --
 * Each mirrors one kernel of src/solvers/gpu/spmv_kernels.cuh; the _f32 forms are the
 * mixed-precision variants.  Row pointers are int64 as in the reference CSR/CSC. */

/* spmv_csr_warp_kernel (spmv_kernels.cuh:39-76): y = A x over CSR. */
vajra_status vajra_csr_spmv_f64(int32_t rows, const int64_t* row_ptr, const int32_t* col_idx,
                                const double* values, const double* x, double* y, void* stream);
vajra_status vajra_csr_spmv_f32(int32_t rows, const int64_t* row_ptr, const int32_t* col_idx,
                                const float* values, const float* x, float* y, void* stream);
/* spmv_csc_transpose_warp_kernel (spmv_kernels.cuh:101-138): v = A^T y over CSC. */
vajra_status vajra_csc_spmv_transpose_f64(int32_t cols, const int64_t* col_ptr,
                                          const int32_t* row_idx, const double* values,
                                          const double* y, double* v, void* stream);
vajra_status vajra_csc_spmv_transpose_f32(int32_t cols, const int64_t* col_ptr,
                                          const int32_t* row_idx, const float* values,
                                          const float* y, float* v, void* stream);
/* dual_update_kernel (spmv_kernels.cuh:163-180). */
vajra_status vajra_dual_prox_f64(int32_t rows, double sigma, const double* ax,
                                 const double* row_lower, const double* row_upper, double* y,
                                 void* stream);
/* primal_update_kernel (spmv_kernels.cuh:185-206). */
vajra_status vajra_primal_prox_f64(int32_t cols, double tau, const double* aty, const double* c,
                                   const double* col_lower, const double* col_upper, double* x,
                                   double* x_bar, void* stream);
/* compute_diagnostics_device_kernel (spmv_kernels.cuh:210-278); out is a device pointer.
 * A grid of CTAs with a deterministic two-stage reduction instead of the reference's CAS
 * atomics; the block partials come from the stream-ordered pool (cudaMallocAsync) on `stream`. */
vajra_status vajra_device_diagnostics_f64(int32_t rows, int32_t cols, const double* ax,
                                          const double* row_lower, const double* row_upper,
                                          const double* aty, const double* c, const double* x,
                                          const double* y, const double* col_lower,
                                          const double* col_upper,
                                          vajra_device_diagnostics* out, void* stream);
/* One fused PDHG iteration (the 4-launch loop body of pdhg_cuda.cu:261-279 as 2 kernels):
 * w = A x_bar with the dual prox fused into its epilogue, then v = A^T y with the primal
 * prox and extrapolation fused.  CSR of A and CSC of A (= CSR of A^T). */
vajra_status vajra_pdhg_step_f64(int32_t rows, int32_t cols,
                                 const int64_t* row_ptr, const int32_t* col_idx,
                                 const double* csr_values, const int64_t* col_ptr,
                                 const int32_t* row_idx, const double* csc_values,
                                 const double* row_lower, const double* row_upper,
                                 const double* c, const double* col_lower,
                                 const double* col_upper, double sigma, double tau,
                                 double* x, double* x_bar, double* y, double* w, double* v,
                                 void* stream);

/* Measurement probe, no counterpart in the reference: partial sums of x[idx[k]] for k < count
 * over a grid of resident CTAs (every SM full), 4 independent gathers in flight per thread --
 * the random gathers of the dense vector that bound the iteration kernels, without their
 * matrix value stream and epilogue.  Timing it on the iteration kernels' own index stream gives
 * the gather floor their durations are compared with.  *threads (in: capacity of partials,
 * out: the number the launch writes); a capacity below that returns INVALID_ARGUMENT with
 * *threads set to the size needed (count = 0 with NULL arrays queries it). */
vajra_status vajra_gather_probe_f32(int64_t count, const int32_t* idx, const float* x, float* partials,
                                    int32_t* threads, void* stream);

/* FP64 relative KKT (the definition the solver's checks use) of a point (x, y) of an LP whose
 * data the caller already holds on the device: A as CSR and as CSC, c, bounds, the column
 * values x and the row duals y in the verifier's sign convention of the minimisation form.
 * out (device, 6 doubles) = rel_primal, rel_dual, rel_gap, rel_kkt, primal and dual
 * objective (minimisation form, offset included).
 * No counterpart in the reference.  It allocates nothing, for callers that cannot call
 * cudaMalloc: its scratch is a fixed 2 MiB device array inside the library, which limits
 * rows and columns to 8,388,608 each (larger sizes return VAJRA_ERR_INVALID_ARGUMENT).  Each
 * call outside a stream capture looks up that array's address on the current device; a call
 * inside a capture reuses the address the last such call found, so make the first call on a
 * device -- and the first after a cudaDeviceReset or primary-context reset -- outside any
 * capture.  An LP without rows (rows = 0) is accepted; its row-side pointers may then be NULL.
 * Nothing has to start at zero: each call writes every partial sum it later reads.  All calls
 * on a device share the array: calls that overlap on the GPU race. */
vajra_status vajra_relative_kkt_noalloc_f64(int32_t rows, int32_t cols, const int64_t* row_ptr,
                                            const int32_t* col_idx, const double* csr_values,
                                            const int64_t* col_ptr, const int32_t* row_idx,
                                            const double* csc_values, const double* c,
                                            const double* col_lower, const double* col_upper,
                                            const double* row_lower, const double* row_upper,
                                            const double* x, const double* y, int32_t sense,
                                            double objective_offset, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VAJRA_PDHG_H */
