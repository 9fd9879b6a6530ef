/* Test infrastructure (oracle): C restatement of the reference's CPU PDHG path.
 * See pdhg_oracle.h for what pins it.  Reference paths are relative to the reference
 * project root.  Only tests/, smoke() and bench.py's cpu_baseline leg call this code. */
#include "pdhg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_ZERO_DROP 1e-11      /* tol::kZeroDrop            tolerances.hpp:28 */
#define ORC_PRIMAL_FEAS 1e-7     /* tol::kPrimalFeasibility   tolerances.hpp:7  */
#define ORC_DUAL_FEAS 1e-7       /* tol::kDualFeasibility     tolerances.hpp:10 */

/* indus::SolveStatus values (types.hpp:34-47) */
enum { ST_NOT_SOLVED = 0, ST_OPTIMAL = 1, ST_UNBOUNDED = 3, ST_FEASIBLE = 5,
       ST_ITERATION_LIMIT = 6, ST_TIME_LIMIT = 7, ST_NODE_LIMIT = 8, ST_NUMERICAL_ERROR = 9 };

static int claims_a_point(int32_t s) { /* types.hpp:49-61 */
    return s == ST_OPTIMAL || s == ST_FEASIBLE || s == ST_UNBOUNDED || s == ST_ITERATION_LIMIT ||
           s == ST_TIME_LIMIT || s == ST_NODE_LIMIT;
}

void orc_csc_multiply(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                      const double* values, const double* x, double* y) {
    for (int32_t i = 0; i < m; ++i) y[i] = 0.0;
    for (int32_t j = 0; j < n; ++j) {
        const double xj = x[j];
        if (fabs(xj) <= ORC_ZERO_DROP) continue;          /* sparse.cpp:207 */
        for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) y[row_idx[k]] += xj * values[k];
    }
}

void orc_csc_multiply_transpose(int32_t m, int32_t n, const int64_t* col_ptr,
                                const int32_t* row_idx, const double* values,
                                const double* y, double* v) {
    (void)m;
    for (int32_t j = 0; j < n; ++j) {
        double dot = 0.0;
        for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) dot += values[k] * y[row_idx[k]];
        v[j] = 0.0 + dot;                                  /* y filled with 0, then += 1.0*dot */
    }
}

void orc_csr_multiply(int32_t m, const int64_t* row_ptr, const int32_t* col_idx,
                      const double* values, const double* x, double* y) {
    for (int32_t i = 0; i < m; ++i) {
        double s = 0.0;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += values[k] * x[col_idx[k]];
        y[i] = s;
    }
}

void orc_to_csr(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                const double* values, int64_t* row_ptr, int32_t* col_idx, double* csr_values) {
    for (int32_t i = 0; i <= m; ++i) row_ptr[i] = 0;
    const int64_t nnz = col_ptr[n];
    for (int64_t k = 0; k < nnz; ++k) row_ptr[row_idx[k] + 1]++;
    for (int32_t i = 0; i < m; ++i) row_ptr[i + 1] += row_ptr[i];
    int64_t* cursor = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
    memcpy(cursor, row_ptr, sizeof(int64_t) * (size_t)(m + 1));
    for (int32_t j = 0; j < n; ++j) {
        for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
            const int64_t dst = cursor[row_idx[k]]++;
            col_idx[dst] = j;
            csr_values[dst] = values[k];
        }
    }
    free(cursor);
}

static double dual_prox_one(double y, double w, double sigma, double l, double u) {
    const double y_hat = y + sigma * w;                    /* pdhg.cpp:204-209 */
    const double val = y_hat / sigma;
    const double clamped = (val < l) ? l : ((val > u) ? u : val);
    return y_hat - sigma * clamped;
}

void orc_dual_prox(int32_t m, double sigma, const double* w, const double* row_lower,
                   const double* row_upper, double* y) {
    for (int32_t i = 0; i < m; ++i) y[i] = dual_prox_one(y[i], w[i], sigma, row_lower[i], row_upper[i]);
}

void orc_primal_prox(int32_t n, double tau, const double* v, const double* c,
                     const double* col_lower, const double* col_upper, double* x, double* x_bar) {
    for (int32_t j = 0; j < n; ++j) {                      /* pdhg.cpp:228-241 */
        const double x_old = x[j];
        const double grad = v[j] + c[j];
        double x_new = x_old - tau * grad;
        if (x_new < col_lower[j]) x_new = col_lower[j];
        if (x_new > col_upper[j]) x_new = col_upper[j];
        x[j] = x_new;
        x_bar[j] = 2.0 * x_new - x_old;
    }
}

void orc_device_diagnostics_eval(int32_t m, int32_t n, const double* ax, const double* row_lower,
                                 const double* row_upper, const double* aty, const double* c,
                                 const double* x, const double* y, const double* col_lower,
                                 const double* col_upper, orc_device_diagnostics* out) {
    memset(out, 0, sizeof(*out));
    for (int32_t i = 0; i < m; ++i) {                      /* spmv_kernels.cuh:228-243 */
        if (isnan(ax[i]) || isinf(ax[i]) || isnan(y[i]) || isinf(y[i])) out->numerical_error = 1;
        double viol = 0.0;
        if (ax[i] < row_lower[i]) viol = row_lower[i] - ax[i];
        if (ax[i] > row_upper[i]) viol = ax[i] - row_upper[i];
        if (viol > out->primal_residual) out->primal_residual = viol;
    }
    for (int32_t j = 0; j < n; ++j) {                      /* spmv_kernels.cuh:246-277 */
        const double xj = x[j], cj = c[j], atyj = aty[j];
        if (isnan(xj) || isinf(xj) || isnan(cj) || isinf(cj) || isnan(atyj) || isinf(atyj))
            out->numerical_error = 1;
        const double lj = col_lower[j], uj = col_upper[j];
        double p_viol = 0.0;
        if (xj < lj) p_viol = lj - xj;
        if (xj > uj) p_viol = xj - uj;
        if (p_viol > out->primal_residual) out->primal_residual = p_viol;
        const double dj = cj + atyj;
        double d_viol = 0.0;
        if (xj > lj + 1e-5 && dj > 1e-6) d_viol = dj;
        if (xj < uj - 1e-5 && dj < -1e-6) d_viol = -dj;
        if (lj <= -1e20 && uj >= 1e20) d_viol = fabs(dj);
        if (d_viol > out->dual_residual) out->dual_residual = d_viol;
        out->objective += cj * xj;
    }
}

int32_t orc_ruiz(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                 double* values, double* c, double* row_lower, double* row_upper,
                 double* col_lower, double* col_upper, int32_t max_iters, double tol,
                 double* row_scale, double* col_scale) {
    if (m <= 0 || n <= 0) return 0;                        /* scaling.cpp:20-22 */
    double* r_k = (double*)malloc(sizeof(double) * (size_t)m);
    double* c_k = (double*)malloc(sizeof(double) * (size_t)n);
    double* row_inf = (double*)malloc(sizeof(double) * (size_t)m);
    double* col_inf = (double*)malloc(sizeof(double) * (size_t)n);
    for (int32_t i = 0; i < m; ++i) { row_scale[i] = 1.0; r_k[i] = 1.0; }
    for (int32_t j = 0; j < n; ++j) { col_scale[j] = 1.0; c_k[j] = 1.0; }

    for (int32_t it = 0; it < max_iters; ++it) {          /* scaling.cpp:32-101 */
        for (int32_t i = 0; i < m; ++i) row_inf[i] = 0.0;
        for (int32_t j = 0; j < n; ++j) {
            double cm = 0.0;
            for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
                const double a = fabs(values[k]);
                if (a > row_inf[row_idx[k]]) row_inf[row_idx[k]] = a;   /* std::max keeps first on tie */
                if (a > cm) cm = a;
            }
            col_inf[j] = cm;
        }
        double max_row_err = 0.0, max_col_err = 0.0;
        for (int32_t i = 0; i < m; ++i)
            if (row_inf[i] > ORC_ZERO_DROP && fabs(1.0 - row_inf[i]) > max_row_err)
                max_row_err = fabs(1.0 - row_inf[i]);
        for (int32_t j = 0; j < n; ++j)
            if (col_inf[j] > ORC_ZERO_DROP && fabs(1.0 - col_inf[j]) > max_col_err)
                max_col_err = fabs(1.0 - col_inf[j]);
        if (max_row_err <= tol && max_col_err <= tol) break;
        for (int32_t i = 0; i < m; ++i) {
            r_k[i] = (row_inf[i] > ORC_ZERO_DROP) ? 1.0 / sqrt(row_inf[i]) : 1.0;
            row_scale[i] *= r_k[i];
        }
        for (int32_t j = 0; j < n; ++j) {
            c_k[j] = (col_inf[j] > ORC_ZERO_DROP) ? 1.0 / sqrt(col_inf[j]) : 1.0;
            col_scale[j] *= c_k[j];
        }
        for (int32_t j = 0; j < n; ++j)
            for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k)
                values[k] *= r_k[row_idx[k]] * c_k[j];
    }
    /* scaling.cpp:104-149: inverse column scales multiply the column bounds */
    for (int32_t j = 0; j < n; ++j) c[j] *= col_scale[j];
    for (int32_t i = 0; i < m; ++i) {
        if (row_lower[i] > -1e20) row_lower[i] *= row_scale[i];
        if (row_upper[i] < 1e20) row_upper[i] *= row_scale[i];
    }
    for (int32_t j = 0; j < n; ++j) {
        const double inv = 1.0 / col_scale[j];
        if (col_lower[j] > -1e20) col_lower[j] *= inv;
        if (col_upper[j] < 1e20) col_upper[j] *= inv;
    }
    free(r_k); free(c_k); free(row_inf); free(col_inf);
    return 1;
}

double orc_spectral_norm(int32_t m, int32_t n, const int64_t* col_ptr, const int32_t* row_idx,
                         const double* values, int32_t max_iter, double tol) {
    if (m == 0 || n == 0 || col_ptr[n] == 0) return 1.0;   /* pdhg.cpp:14-16 */
    double* v = (double*)malloc(sizeof(double) * (size_t)n);
    double* w = (double*)malloc(sizeof(double) * (size_t)m);
    double* u = (double*)malloc(sizeof(double) * (size_t)n);
    const double v0 = 1.0 / sqrt((double)n);
    for (int32_t j = 0; j < n; ++j) v[j] = v0;
    double lambda_prev = 0.0, lambda = 1.0, result = -1.0;
    for (int32_t it = 0; it < max_iter; ++it) {            /* pdhg.cpp:25-52 */
        orc_csc_multiply(m, n, col_ptr, row_idx, values, v, w);
        orc_csc_multiply_transpose(m, n, col_ptr, row_idx, values, w, u);
        double norm_sq = 0.0;
        for (int32_t j = 0; j < n; ++j) norm_sq += u[j] * u[j];
        const double norm = sqrt(norm_sq);
        if (norm < 1e-15 || isnan(norm) || isinf(norm)) {
            result = (lambda > 1e-6) ? sqrt(lambda) : 1e-3;
            break;
        }
        lambda = norm;
        if (it > 0 && fabs(lambda - lambda_prev) <= tol * lambda) break;
        lambda_prev = lambda;
        const double inv_norm = 1.0 / norm;
        for (int32_t j = 0; j < n; ++j) v[j] = u[j] * inv_norm;
    }
    if (result < 0.0) {
        const double sigma_max = sqrt(lambda);
        result = (sigma_max > 1e-12) ? sigma_max : 1e-6;
    }
    free(v); free(w); free(u);
    return result;
}

/* Solution::recompute_quality, LP part (model.cpp:203-374): refreshes row_value and
 * col_dual and the primal / dual feasibility verdicts on the ORIGINAL model. */
static void recompute_quality(const orc_lp* lp, orc_result* r, double* x, double* row_value,
                              double* row_dual, double* col_dual) {
    r->max_primal_violation = 0.0;
    r->max_dual_violation = 0.0;
    r->is_primal_feasible = 0;
    r->is_dual_feasible = 0;
    if (!claims_a_point(r->status)) return;
    const int32_t m = lp->num_rows, n = lp->num_cols;
    double max_rel = 0.0;
    for (int32_t j = 0; j < n; ++j) {
        const double xj = x[j], lj = lp->col_lower[j], uj = lp->col_upper[j];
        if (xj < lj) {
            const double viol = lj - xj;
            if (viol > r->max_primal_violation) r->max_primal_violation = viol;
            if (viol / (1.0 + fabs(lj)) > max_rel) max_rel = viol / (1.0 + fabs(lj));
        }
        if (xj > uj) {
            const double viol = xj - uj;
            if (viol > r->max_primal_violation) r->max_primal_violation = viol;
            if (viol / (1.0 + fabs(uj)) > max_rel) max_rel = viol / (1.0 + fabs(uj));
        }
    }
    orc_csc_multiply(m, n, lp->col_ptr, lp->row_idx, lp->values, x, row_value);
    for (int32_t i = 0; i < m; ++i) {
        const double ax = row_value[i], li = lp->row_lower[i], ui = lp->row_upper[i];
        if (ax < li) {
            const double viol = li - ax;
            const double denom = 1.0 + (li > -1e19 ? fabs(li) : 1.0);
            if (viol > r->max_primal_violation) r->max_primal_violation = viol;
            if (viol / denom > max_rel) max_rel = viol / denom;
        }
        if (ax > ui) {
            const double viol = ax - ui;
            const double denom = 1.0 + (ui < 1e19 ? fabs(ui) : 1.0);
            if (viol > r->max_primal_violation) r->max_primal_violation = viol;
            if (viol / denom > max_rel) max_rel = viol / denom;
        }
    }
    r->is_primal_feasible = (r->max_primal_violation <= ORC_PRIMAL_FEAS || max_rel <= ORC_PRIMAL_FEAS);
    double* aty = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    orc_csc_multiply_transpose(m, n, lp->col_ptr, lp->row_idx, lp->values, row_dual, aty);
    const double sense_factor = lp->sense ? -1.0 : 1.0;
    for (int32_t j = 0; j < n; ++j) {
        const double dj = sense_factor * lp->c[j] - aty[j];
        col_dual[j] = lp->sense ? -dj : dj;
        const double xj = x[j], lj = lp->col_lower[j], uj = lp->col_upper[j];
        if (xj < uj - ORC_PRIMAL_FEAS && dj < -ORC_DUAL_FEAS && -dj > r->max_dual_violation)
            r->max_dual_violation = -dj;
        if (xj > lj + ORC_PRIMAL_FEAS && dj > ORC_DUAL_FEAS && dj > r->max_dual_violation)
            r->max_dual_violation = dj;
    }
    for (int32_t i = 0; i < m; ++i) {
        const double yi = row_dual[i], li = lp->row_lower[i], ui = lp->row_upper[i];
        if (li <= -1e20 && ui < 1e20) {
            if (yi > ORC_DUAL_FEAS && yi > r->max_dual_violation) r->max_dual_violation = yi;
        } else if (li > -1e20 && ui >= 1e20) {
            if (yi < -ORC_DUAL_FEAS && -yi > r->max_dual_violation) r->max_dual_violation = -yi;
        }
    }
    r->is_dual_feasible = r->max_dual_violation <= ORC_DUAL_FEAS;
    free(aty);
}

static void store(double* dst, const double* src, int32_t k) {
    if (dst && k > 0) memcpy(dst, src, sizeof(double) * (size_t)k);
}

int32_t orc_pdhg_solve(const orc_lp* lp, const orc_opts* o, orc_result* r) {
    const int32_t m = lp->num_rows, n = lp->num_cols;
    const int is_max = lp->sense != 0;
    const int64_t nnz = lp->col_ptr[n];
    r->status = ST_NOT_SOLVED;
    r->iterations = 0;
    r->restart_count = 0;
    r->primal_residual = r->dual_residual = r->duality_gap = 0.0;
    r->spectral_norm_estimate = r->tau = r->sigma = 0.0;
    r->converged = 0;

    /* Output vectors start at zero (pdhg.cpp:80-83). */
    double* out_x = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double* out_rv = (double*)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    double* out_y = (double*)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    double* out_d = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));

    if (n == 0) {                                          /* pdhg.cpp:88-94 */
        r->status = ST_OPTIMAL;
        r->objective_value = lp->objective_offset;
        r->converged = 1;
        goto done_no_quality;
    }
    if (m == 0) {                                          /* pdhg.cpp:96-127 */
        double obj = lp->objective_offset;
        for (int32_t j = 0; j < n; ++j) {
            const double cj = is_max ? -lp->c[j] : lp->c[j];
            const double lj = lp->col_lower[j], uj = lp->col_upper[j];
            if (cj > ORC_DUAL_FEAS) {
                if (lj <= -1e20) { r->status = ST_UNBOUNDED; goto done_no_quality; }
                out_x[j] = lj;
            } else if (cj < -ORC_DUAL_FEAS) {
                if (uj >= 1e20) { r->status = ST_UNBOUNDED; goto done_no_quality; }
                out_x[j] = uj;
            } else {
                out_x[j] = (lj > 0.0) ? lj : ((uj < 0.0) ? uj : 0.0);
            }
            obj += lp->c[j] * out_x[j];
        }
        r->status = ST_OPTIMAL;
        r->objective_value = obj;
        r->converged = 1;
        goto done_no_quality;
    }

    {
        /* Working copies (pdhg.cpp:129-149) */
        double* A = (double*)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
        memcpy(A, lp->values, sizeof(double) * (size_t)nnz);
        double* wc = (double*)malloc(sizeof(double) * (size_t)n);
        double* wrl = (double*)malloc(sizeof(double) * (size_t)m);
        double* wru = (double*)malloc(sizeof(double) * (size_t)m);
        double* wcl = (double*)malloc(sizeof(double) * (size_t)n);
        double* wcu = (double*)malloc(sizeof(double) * (size_t)n);
        double* rs = (double*)malloc(sizeof(double) * (size_t)m);
        double* cs = (double*)malloc(sizeof(double) * (size_t)n);
        for (int32_t j = 0; j < n; ++j) wc[j] = is_max ? -lp->c[j] : lp->c[j];
        memcpy(wrl, lp->row_lower, sizeof(double) * (size_t)m);
        memcpy(wru, lp->row_upper, sizeof(double) * (size_t)m);
        memcpy(wcl, lp->col_lower, sizeof(double) * (size_t)n);
        memcpy(wcu, lp->col_upper, sizeof(double) * (size_t)n);
        int32_t scaled = 0;
        if (o->enable_scaling)
            scaled = orc_ruiz(m, n, lp->col_ptr, lp->row_idx, A, wc, wrl, wru, wcl, wcu, 10, 0.05, rs, cs);

        const double spectral_norm = orc_spectral_norm(m, n, lp->col_ptr, lp->row_idx, A, 25, 1e-4);
        r->spectral_norm_estimate = spectral_norm;
        const double safety = 0.95;                        /* clamp(0.95, 0.5, 0.99) */
        double tau = safety / spectral_norm;
        double sigma = safety / spectral_norm;
        r->tau = tau;
        r->sigma = sigma;

        double* x = (double*)malloc(sizeof(double) * (size_t)n);
        double* xb = (double*)malloc(sizeof(double) * (size_t)n);
        double* y = (double*)calloc((size_t)m, sizeof(double));
        double* w = (double*)calloc((size_t)m, sizeof(double));
        double* v = (double*)calloc((size_t)n, sizeof(double));
        double* ax = (double*)calloc((size_t)m, sizeof(double));
        double* best_x = (double*)malloc(sizeof(double) * (size_t)n);
        double* best_y = (double*)calloc((size_t)m, sizeof(double));
        for (int32_t j = 0; j < n; ++j) {                  /* pdhg.cpp:167-175 */
            double val = 0.0;
            if (val < wcl[j]) val = wcl[j];
            if (val > wcu[j]) val = wcu[j];
            x[j] = val;
            xb[j] = val;
        }
        memcpy(best_x, x, sizeof(double) * (size_t)n);
        double best_infeas = 1e20;
        int64_t stagnation = 0;
        int converged = 0;
        const int64_t max_iter = o->iteration_limit;
        const int32_t check_freq = o->check_frequency > 1 ? o->check_frequency : 1;
        int64_t iter;
        for (iter = 1; iter <= max_iter; ++iter) {         /* pdhg.cpp:196-366 */
            orc_csc_multiply(m, n, lp->col_ptr, lp->row_idx, A, xb, w);
            int has_nan = 0;
            for (int32_t i = 0; i < m; ++i) {
                const double yn = dual_prox_one(y[i], w[i], sigma, wrl[i], wru[i]);
                if (isnan(yn) || isinf(yn)) has_nan = 1;
                y[i] = yn;
            }
            if (has_nan) { r->status = ST_NUMERICAL_ERROR; break; }
            orc_csc_multiply_transpose(m, n, lp->col_ptr, lp->row_idx, A, y, v);
            for (int32_t j = 0; j < n; ++j) {
                const double x_old = x[j];
                const double grad = v[j] + wc[j];
                double x_new = x_old - tau * grad;
                if (x_new < wcl[j]) x_new = wcl[j];
                if (x_new > wcu[j]) x_new = wcu[j];
                if (isnan(x_new) || isinf(x_new)) has_nan = 1;
                x[j] = x_new;
                xb[j] = 2.0 * x_new - x_old;
            }
            if (has_nan) { r->status = ST_NUMERICAL_ERROR; break; }

            if (iter % check_freq == 0 || iter == max_iter) {
                orc_csc_multiply(m, n, lp->col_ptr, lp->row_idx, A, x, ax);
                double prim = 0.0, dual = 0.0, dual_obj = 0.0, primal_obj = 0.0;
                for (int32_t i = 0; i < m; ++i) {          /* pdhg.cpp:261-268 */
                    if (ax[i] < wrl[i] && wrl[i] - ax[i] > prim) prim = wrl[i] - ax[i];
                    if (ax[i] > wru[i] && ax[i] - wru[i] > prim) prim = ax[i] - wru[i];
                }
                for (int32_t j = 0; j < n; ++j) {          /* pdhg.cpp:269-275 */
                    if (x[j] < wcl[j] && wcl[j] - x[j] > prim) prim = wcl[j] - x[j];
                    if (x[j] > wcu[j] && x[j] - wcu[j] > prim) prim = x[j] - wcu[j];
                }
                for (int32_t i = 0; i < m; ++i) {          /* pdhg.cpp:281-290 */
                    const double yi = y[i];
                    if (yi > 1e-12 && wru[i] < 1e20) dual_obj -= yi * wru[i];
                    else if (yi < -1e-12 && wrl[i] > -1e20) dual_obj -= yi * wrl[i];
                }
                for (int32_t j = 0; j < n; ++j) {          /* pdhg.cpp:292-313 */
                    const double dj = wc[j] + v[j];
                    const double xj = x[j], lj = wcl[j], uj = wcu[j];
                    if (xj > lj + 1e-5 && dj > 1e-6 && dj > dual) dual = dj;
                    if (xj < uj - 1e-5 && dj < -1e-6 && -dj > dual) dual = -dj;
                    if (lj <= -1e20 && uj >= 1e20 && fabs(dj) > dual) dual = fabs(dj);
                    if (dj > 1e-12 && lj > -1e20) dual_obj += dj * lj;
                    else if (dj < -1e-12 && uj < 1e20) dual_obj += dj * uj;
                }
                for (int32_t j = 0; j < n; ++j) primal_obj += wc[j] * x[j];
                const double gap = fabs(primal_obj - dual_obj) / (1.0 + fabs(primal_obj) + fabs(dual_obj));
                r->primal_residual = prim;
                r->dual_residual = dual;
                r->duality_gap = gap;
                const double total = prim + dual;
                if (total < best_infeas) {                 /* pdhg.cpp:327-335 */
                    best_infeas = total;
                    memcpy(best_x, x, sizeof(double) * (size_t)n);
                    memcpy(best_y, y, sizeof(double) * (size_t)m);
                    stagnation = 0;
                } else {
                    stagnation += check_freq;
                }
                if (prim <= o->tolerance && dual <= o->tolerance && gap <= o->gap_tolerance) {
                    converged = 1;
                    r->converged = 1;
                    memcpy(best_x, x, sizeof(double) * (size_t)n);
                    memcpy(best_y, y, sizeof(double) * (size_t)m);
                    r->status = ST_OPTIMAL;
                    break;
                }
                if (prim > 10.0 * dual && dual > 0.0) {    /* pdhg.cpp:351-357 */
                    sigma = (sigma * 1.3 < 1e6) ? sigma * 1.3 : 1e6;
                    tau = (safety * safety) / (spectral_norm * spectral_norm * sigma);
                } else if (dual > 10.0 * prim && prim > 0.0) {
                    tau = (tau * 1.3 < 1e6) ? tau * 1.3 : 1e6;
                    sigma = (safety * safety) / (spectral_norm * spectral_norm * tau);
                }
                if (stagnation >= 200) {                   /* pdhg.cpp:359-364 */
                    memcpy(xb, x, sizeof(double) * (size_t)n);
                    r->restart_count++;
                    stagnation = 0;
                }
            }
        }
        r->iterations = iter;
        if (!converged && r->status == ST_NOT_SOLVED && iter >= max_iter)   /* pdhg.cpp:373-378 */
            r->status = (best_infeas <= 1e-4) ? ST_FEASIBLE : ST_ITERATION_LIMIT;

        /* Unscale the best iterate and map to the original model (pdhg.cpp:380-433). */
        memcpy(out_x, best_x, sizeof(double) * (size_t)n);
        memcpy(out_y, best_y, sizeof(double) * (size_t)m);
        if (scaled) {
            for (int32_t j = 0; j < n; ++j) out_x[j] *= cs[j];
            for (int32_t i = 0; i < m; ++i) out_y[i] *= rs[i];
        }
        orc_csc_multiply(m, n, lp->col_ptr, lp->row_idx, lp->values, out_x, out_rv);
        double obj = lp->objective_offset;
        for (int32_t j = 0; j < n; ++j) obj += lp->c[j] * out_x[j];
        r->objective_value = obj;
        for (int32_t i = 0; i < m; ++i) out_y[i] = is_max ? out_y[i] : -out_y[i];
        orc_csc_multiply_transpose(m, n, lp->col_ptr, lp->row_idx, lp->values, out_y, out_d);
        for (int32_t j = 0; j < n; ++j) out_d[j] = lp->c[j] - out_d[j];

        free(A); free(wc); free(wrl); free(wru); free(wcl); free(wcu); free(rs); free(cs);
        free(x); free(xb); free(y); free(w); free(v); free(ax); free(best_x); free(best_y);
    }
    recompute_quality(lp, r, out_x, out_rv, out_y, out_d);
    goto finish;

done_no_quality:
    /* the m == 0 / n == 0 closed forms return before recompute_quality (pdhg.cpp:88-127) */
    r->max_primal_violation = r->max_dual_violation = 0.0;
    r->is_primal_feasible = r->is_dual_feasible = 0;
finish:
    store(r->col_value, out_x, n);
    store(r->row_value, out_rv, m);
    store(r->row_dual, out_y, m);
    store(r->col_dual, out_d, n);
    free(out_x); free(out_rv); free(out_y); free(out_d);
    return 0;
}
