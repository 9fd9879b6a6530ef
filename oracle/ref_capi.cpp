// Test infrastructure (oracle only): plain C entry points over the REFERENCE's own CPU code.
//
// oracle/Makefile compiles this file together with the reference's sources, read in place
// from the reference tree, into oracle/_ref/libindus_ref.so.  Nothing in the product links
// or loads it: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline and
// `--impl reference` legs do, as the checker and as the timed CPU baseline.
//
// Entry points wrap (reference paths):
//   ref_solve           -> indus::pdhg::solve_pdhg_cpu            src/solvers/pdhg/pdhg.cpp:448-453
//                          or indus::solve (status guard)         src/engine/model.cpp:376-667
//   ref_spectral_norm   -> indus::pdhg::estimate_spectral_norm    src/solvers/pdhg/pdhg.cpp:11-56
//   ref_ruiz            -> indus::la::RuizScaler::compute_and_scale src/linalg/scaling.cpp:7-153
//   ref_pock_chambolle  -> indus::la::PockChambollePreconditioner::compute src/linalg/scaling.cpp:179-220
//   ref_csc_multiply(_transpose) -> SparseMatrixCSC::multiply(_transpose) src/linalg/sparse.cpp:196-238
//   ref_verify          -> indus::verifier::verify_solution       src/engine/verifier.cpp:25-330
//
// The Options "algorithm" key is assigned by FIELD: Options::set(key, "literal") binds to the
// bool overload (include/indus/options.hpp:14-17) and would silently select dual simplex.
#include "indus/model.hpp"
#include "indus/options.hpp"
#include "indus/pdhg.hpp"
#include "indus/verifier.hpp"
#include "src/linalg/scaling.hpp"

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

extern "C" {

typedef struct {
    int32_t num_rows;
    int32_t num_cols;
    int64_t nnz;
    const int64_t* col_ptr;   // n + 1
    const int32_t* row_idx;   // nnz, ascending within each column, no duplicates
    const double* values;     // nnz
    const double* c;          // n
    const double* col_lower;  // n
    const double* col_upper;  // n
    const double* row_lower;  // m
    const double* row_upper;  // m
    int32_t sense;            // 0 minimise, 1 maximise
    double objective_offset;
} ref_lp;

typedef struct {
    const char* algorithm;    // "pdhg_cpu", "dual_simplex", "primal_simplex", ...
    double tolerance;
    double gap_tolerance;
    double time_limit;
    int64_t iteration_limit;
    int32_t check_frequency;
    int32_t enable_scaling;
    int32_t enable_presolve;
    int32_t through_solve;    // 1: indus::solve (validate, presolve, status guard); 0: solve_pdhg_cpu
} ref_opts;

typedef struct {
    double* col_value;        // n   (caller buffers; NULL to skip)
    double* row_value;        // m
    double* row_dual;         // m
    double* col_dual;         // n
    int32_t status;           // indus::SolveStatus
    int64_t iterations;
    double objective_value;
    int64_t diag_iterations;
    int32_t restart_count;
    double primal_residual;
    double dual_residual;
    double duality_gap;
    double spectral_norm_estimate;
    double tau;
    double sigma;
    double setup_time_sec;
    double iteration_time_sec;
    double total_time_sec;
    int32_t converged;
    double max_primal_violation;
    double max_dual_violation;
    int32_t is_primal_feasible;
    int32_t is_dual_feasible;
    char status_message[256];
} ref_result;

typedef struct {
    int32_t passed;
    int32_t primal_feasible;
    int32_t dual_feasible;
    int32_t objective_matches;
    double max_primal_violation;
    double max_bound_violation;
    double max_row_violation;
    double max_dual_violation;
    double max_complementarity_violation;
    double objective_discrepancy;
    char summary[512];
} ref_verify_out;

}  // extern "C"

namespace {

indus::Model make_model(const ref_lp* lp) {
    indus::Model model;
    const int m = lp->num_rows;
    const int n = lp->num_cols;
    model.num_rows = m;
    model.num_cols = n;
    model.sense = lp->sense ? indus::ObjSense::kMaximize : indus::ObjSense::kMinimize;
    model.objective_offset = lp->objective_offset;
    model.A.m = m;
    model.A.n = n;
    model.A.col_ptr.assign(lp->col_ptr, lp->col_ptr + n + 1);
    model.A.row_idx.assign(lp->row_idx, lp->row_idx + lp->nnz);
    model.A.values.assign(lp->values, lp->values + lp->nnz);
    model.c.assign(lp->c, lp->c + n);
    model.col_lower.assign(lp->col_lower, lp->col_lower + n);
    model.col_upper.assign(lp->col_upper, lp->col_upper + n);
    model.row_lower.assign(lp->row_lower, lp->row_lower + m);
    model.row_upper.assign(lp->row_upper, lp->row_upper + m);
    return model;
}

void copy_out(const std::vector<double>& v, double* dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(double));
}

}  // namespace

extern "C" {

int ref_solve(const ref_lp* lp, const ref_opts* o, ref_result* r) {
    try {
        indus::Model model = make_model(lp);
        indus::Options opts;
        opts.algorithm = o->algorithm ? o->algorithm : "pdhg_cpu";   // field assignment (see header)
        opts.enable_presolve = o->enable_presolve != 0;
        opts.enable_scaling = o->enable_scaling != 0;
        opts.iteration_limit = o->iteration_limit;
        opts.time_limit = o->time_limit;
        opts.set("tolerance", o->tolerance);
        opts.set("gap_tolerance", o->gap_tolerance);
        opts.set("check_frequency", static_cast<int64_t>(o->check_frequency));

        indus::Solution sol = o->through_solve ? indus::solve(model, opts)
                                               : indus::pdhg::solve_pdhg_cpu(model, opts);
        const auto& d = indus::pdhg::get_last_cpu_pdhg_diagnostics();
        copy_out(sol.col_value, r->col_value);
        copy_out(sol.row_value, r->row_value);
        copy_out(sol.row_dual, r->row_dual);
        copy_out(sol.col_dual, r->col_dual);
        r->status = static_cast<int32_t>(sol.status);
        r->iterations = sol.iterations;
        r->objective_value = sol.objective_value;
        r->diag_iterations = d.iterations;
        r->restart_count = d.restart_count;
        r->primal_residual = d.primal_residual;
        r->dual_residual = d.dual_residual;
        r->duality_gap = d.duality_gap;
        r->spectral_norm_estimate = d.spectral_norm_estimate;
        r->tau = d.tau;
        r->sigma = d.sigma;
        r->setup_time_sec = d.setup_time_sec;
        r->iteration_time_sec = d.iteration_time_sec;
        r->total_time_sec = d.total_time_sec;
        r->converged = d.converged ? 1 : 0;
        r->max_primal_violation = sol.quality.max_primal_violation;
        r->max_dual_violation = sol.quality.max_dual_violation;
        r->is_primal_feasible = sol.quality.is_primal_feasible ? 1 : 0;
        r->is_dual_feasible = sol.quality.is_dual_feasible ? 1 : 0;
        std::strncpy(r->status_message, sol.status_message.c_str(), sizeof(r->status_message) - 1);
        r->status_message[sizeof(r->status_message) - 1] = '\0';
        return 0;
    } catch (const std::exception& e) {
        std::strncpy(r->status_message, e.what(), sizeof(r->status_message) - 1);
        r->status_message[sizeof(r->status_message) - 1] = '\0';
        return 1;
    }
}

double ref_spectral_norm(const ref_lp* lp, int32_t max_iter, double tol) {
    indus::Model model = make_model(lp);
    return indus::pdhg::estimate_spectral_norm(model.A, max_iter, tol);
}

// Ruiz equilibration in place on copies; outputs are the scaled matrix values (CSC order),
// scaled c / bounds, and the cumulative row and column scales.
int ref_ruiz(const ref_lp* lp, int32_t max_iters, double tol,
             double* values_out, double* c_out, double* rl_out, double* ru_out,
             double* cl_out, double* cu_out, double* row_scale_out, double* col_scale_out) {
    indus::Model model = make_model(lp);
    std::vector<double> c = model.c;
    std::vector<double> rl = model.row_lower, ru = model.row_upper;
    std::vector<double> cl = model.col_lower, cu = model.col_upper;
    auto sf = indus::la::RuizScaler::compute_and_scale(model.A, c, rl, ru, cl, cu, max_iters, tol);
    copy_out(model.A.values, values_out);
    copy_out(c, c_out);
    copy_out(rl, rl_out);
    copy_out(ru, ru_out);
    copy_out(cl, cl_out);
    copy_out(cu, cu_out);
    copy_out(sf.row_scale, row_scale_out);
    copy_out(sf.col_scale, col_scale_out);
    return sf.is_scaled ? 1 : 0;
}

// Pock-Chambolle diagonal preconditioners of the LP's matrix as given (the caller passes the
// Ruiz-scaled values to compose the two, as the device set-up does): d_row[m], d_col[n].
void ref_pock_chambolle(const ref_lp* lp, double alpha, double* d_row_out, double* d_col_out) {
    indus::Model model = make_model(lp);
    std::vector<double> d_row, d_col;
    indus::la::PockChambollePreconditioner::compute(model.A, d_row, d_col, alpha);
    copy_out(d_row, d_row_out);
    copy_out(d_col, d_col_out);
}

void ref_csc_multiply(const ref_lp* lp, const double* x, double* y) {
    indus::Model model = make_model(lp);
    model.A.multiply(std::span<const double>(x, static_cast<size_t>(lp->num_cols)),
                     std::span<double>(y, static_cast<size_t>(lp->num_rows)));
}

void ref_csc_multiply_transpose(const ref_lp* lp, const double* y, double* v) {
    indus::Model model = make_model(lp);
    model.A.multiply_transpose(std::span<const double>(y, static_cast<size_t>(lp->num_rows)),
                               std::span<double>(v, static_cast<size_t>(lp->num_cols)));
}

int ref_verify(const ref_lp* lp, const double* col_value, const double* row_dual,
               double objective_value, int32_t status, double tol, ref_verify_out* out) {
    try {
        indus::Model model = make_model(lp);
        indus::Solution sol;
        sol.status = static_cast<indus::SolveStatus>(status);
        sol.objective_value = objective_value;
        sol.col_value.assign(col_value, col_value + lp->num_cols);
        if (row_dual) sol.row_dual.assign(row_dual, row_dual + lp->num_rows);
        auto v = indus::verifier::verify_solution(model, sol, tol);
        out->passed = v.passed ? 1 : 0;
        out->primal_feasible = v.primal_feasible ? 1 : 0;
        out->dual_feasible = v.dual_feasible ? 1 : 0;
        out->objective_matches = v.objective_matches ? 1 : 0;
        out->max_primal_violation = v.max_primal_violation;
        out->max_bound_violation = v.max_bound_violation;
        out->max_row_violation = v.max_row_violation;
        out->max_dual_violation = v.max_dual_violation;
        out->max_complementarity_violation = v.max_complementarity_violation;
        out->objective_discrepancy = v.objective_discrepancy;
        std::strncpy(out->summary, v.summary.c_str(), sizeof(out->summary) - 1);
        out->summary[sizeof(out->summary) - 1] = '\0';
        return 0;
    } catch (const std::exception& e) {
        std::strncpy(out->summary, e.what(), sizeof(out->summary) - 1);
        out->summary[sizeof(out->summary) - 1] = '\0';
        return 1;
    }
}

}  // extern "C"
