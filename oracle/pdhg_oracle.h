/* Test infrastructure (oracle): a plain-C restatement of the reference's CPU PDHG path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this, as the
 * checker.  The product library (libvajra_pdhg.so) never links or calls it.
 *
 * Parity is pinned two ways (tests/test_oracle.py):
 *   1. the golden vectors of the reference's tests/test_cuda_kernels.cu:75-359 and
 *      tests/test_pdhg.cpp:443-562, and
 *   2. bit-for-bit agreement with the reference's own CPU code compiled from its sources
 *      (oracle/Makefile -> oracle/_ref/libindus_ref.so) on seeded LPs.
 *
 * Every floating-point operation follows the reference's evaluation order (no FMA
 * contraction: built with -ffp-contract=off), so results are bit-identical, not merely close.
 */
#ifndef VAJRA_PDHG_ORACLE_H
#define VAJRA_PDHG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same memory layout as ref_lp (oracle/ref_capi.cpp) and vajra_lp (include/vajra_pdhg.h):
 * the reference Model (include/indus/model.hpp:16-55) as CSC host arrays. */
typedef struct {
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
    int32_t sense;
    double objective_offset;
} orc_lp;

typedef struct {
    double tolerance;        /* Options "tolerance": primal and dual (pdhg.cpp:62-63)      */
    double gap_tolerance;    /* Options "gap_tolerance" (pdhg.cpp:64)                      */
    double time_limit;       /* unused by the oracle (no wall clock in a restatement)      */
    int64_t iteration_limit; /* Options::iteration_limit (pdhg.cpp:60)                     */
    int32_t check_frequency; /* Options "check_frequency" (pdhg.cpp:65)                    */
    int32_t enable_scaling;  /* Options::enable_scaling (pdhg.cpp:66)                      */
} orc_opts;

/* Mirrors ref_result's numeric fields (status values are indus::SolveStatus). */
typedef struct {
    double* col_value;
    double* row_value;
    double* row_dual;
    double* col_dual;
    int32_t status;
    int64_t iterations;
    double objective_value;
    int32_t restart_count;
    double primal_residual;
    double dual_residual;
    double duality_gap;
    double spectral_norm_estimate;
    double tau;
    double sigma;
    int32_t converged;
    double max_primal_violation;
    double max_dual_violation;
    int32_t is_primal_feasible;
    int32_t is_dual_feasible;
} orc_result;

/* Reference GPU diagnostics record (include/indus/gpu.hpp:27-34). */
typedef struct {
    double primal_residual;
    double dual_residual;
    double objective;
    double duality_gap;
    int32_t converged;
    int32_t numerical_error;
} orc_device_diagnostics;

/* y = A x over CSC, skipping |x_j| <= 1e-11 (sparse.cpp:196-217). */
void orc_csc_multiply(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                      const double* values, const double* x, double* y);
/* v = A^T y over CSC, one in-order dot per column (sparse.cpp:219-238). */
void orc_csc_multiply_transpose(int32_t m, int32_t n, const int64_t* col_ptr,
                                const int32_t* row_idx, const double* values,
                                const double* y, double* v);
/* y = A x over CSR, in-order dot per row (spmv_kernels.cuh:39-76 arithmetic). */
void orc_csr_multiply(int32_t m, const int64_t* row_ptr, const int32_t* col_idx,
                      const double* values, const double* x, double* y);
/* CSC -> CSR (sparse.cpp:147-184). row_ptr: m+1, col_idx/values: nnz. */
void orc_to_csr(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                const double* values, int64_t* row_ptr, int32_t* col_idx, double* csr_values);
/* Dual Moreau step y <- (y + s w) - s clamp((y + s w)/s, l, u) (spmv_kernels.cuh:163-180). */
void orc_dual_prox(int32_t m, double sigma, const double* w, const double* row_lower,
                   const double* row_upper, double* y);
/* Primal step x+ = clamp(x - t (v + c)), xbar = 2 x+ - x (spmv_kernels.cuh:185-206). */
void orc_primal_prox(int32_t n, double tau, const double* v, const double* c,
                     const double* col_lower, const double* col_upper, double* x, double* x_bar);
/* Reference GPU diagnostics kernel semantics (spmv_kernels.cuh:210-278). */
void orc_device_diagnostics_eval(int32_t m, int32_t n, const double* ax, const double* row_lower,
                                 const double* row_upper, const double* aty, const double* c,
                                 const double* x, const double* y, const double* col_lower,
                                 const double* col_upper, orc_device_diagnostics* out);
/* Ruiz l-inf equilibration in place (scaling.cpp:7-153).  Returns 1 if scaled. */
int32_t orc_ruiz(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                 double* values, double* c, double* row_lower, double* row_upper,
                 double* col_lower, double* col_upper, int32_t max_iters, double tol,
                 double* row_scale, double* col_scale);
/* Power iteration on A^T A returning sqrt(||A^T A v||) (pdhg.cpp:11-56). */
double orc_spectral_norm(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                         const double* values, int32_t max_iter, double tol);
/* CpuPdhgSolver::solve (pdhg.cpp:70-440) including Solution::recompute_quality's LP part
 * (model.cpp:203-374).  Returns 0 on success, nonzero on allocation failure. */
int32_t orc_pdhg_solve(const orc_lp* lp, const orc_opts* opts, orc_result* out);

#ifdef __cplusplus
}
#endif

#endif
