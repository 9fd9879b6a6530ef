// VAJRA_ALGO_HALPERN: restarted reflected Halpern PDHG with KKT-driven adaptive restarts and
// primal-weight updates, terminated on the FP64 relative KKT error of the original LP.
//
// Operator T (primal first; same saddle form as the reference, pdhg.cpp:196-241):
//   x+ = proj_X(x - tau (c + A^T y)),   y+ = prox_{sigma h*}(y + sigma A (2 x+ - x))
// Halpern step with reflection gamma, inner index k since the last restart, anchor z0:
//   z_{k+1} = (k+1)/(k+2) ((1+gamma) T(z_k) - gamma z_k) + 1/(k+2) z0
// Two fused kernels per iteration:
//   primal: v = A^T y over the stored transpose -> x+, x_bar = 2x+ - x, x <- Halpern
//   dual  : w = A x_bar over CSR                -> y+, y <- Halpern
// Every check_frequency iterations (the chunk, captured once as a CUDA graph) the candidate
// T(z) is evaluated in FP64 with FP64 matrix values: A x+, A^T y+, then row / column passes
// with deterministic block partials and one control CTA that forms the relative KKT on the
// original problem, the primal-weighted KKT for restarts (sufficient 0.2 / necessary 0.8 +
// no progress / artificial 0.36 of total), the primal-weight update at restarts, and -- in
// mixed precision -- the FP32 phase's reflection coefficient and its hand-over to the FP64
// polish.  Large LPs are first renumbered by row / column length (degree ordering) and get
// sliced-ELL copies of both matrices; results go back to the caller's numbering.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "halpern_state.cuh"
#include "solver.cuh"

namespace vajra {
namespace {

// Per block of a check pass: kNS partial sums, then kNM maxima (NaN flag, then the status
// guard's violation maxima of Solution::recompute_quality, src/engine/model.cpp:203-374).
constexpr int kNS = 6;
constexpr int kNM = 4;
constexpr int kQ = kNS + kNM;
constexpr int kCheckBlocks = 148 * 4;
constexpr double kGuardTol = 1e-7;   // tol::kPrimalFeasibility / kDualFeasibility of the guard

__device__ __forceinline__ bool finite_lo(double l) { return l > -1e20; }
__device__ __forceinline__ bool finite_up(double u) { return u < 1e20; }

__device__ __forceinline__ void store_partials(double (&v)[kQ], double (&red)[kQ * 32], double* part) {
    block_reduce<OpSum, double, kNS>(*reinterpret_cast<double(*)[kNS]>(v), red);
    block_reduce<OpMax, double, kNM>(*reinterpret_cast<double(*)[kNM]>(v + kNS), red);
    if (threadIdx.x == 0)
        for (int q = 0; q < kQ; ++q) part[blockIdx.x * kQ + q] = v[q];
}

// Row pass: original- and scaled-space primal residual, row part of the dual objective,
// distance of y+ from the last restart point, NaN detection, and the guard's maxima: the
// row violation relative to 1 + |violated bound|, its absolute size, and the row dual's sign
// violation (verifier convention: y <= 0 on a <= row, y >= 0 on a >= row).
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_kkt_rows(int m, const double* __restrict__ ax, const T* __restrict__ yc, const T* __restrict__ yprev,
           const double* __restrict__ rl_s, const double* __restrict__ ru_s, const double* __restrict__ rl_o,
           const double* __restrict__ ru_o, const double* __restrict__ rs, const double* __restrict__ y_last,
           double* __restrict__ part, const HState* st, int phase) {
    if (st->stop || st->phase != phase) return;
    __shared__ double red[kQ * 32];
    // sums: rp_o^2, rp_s^2, dobj, dy^2 (restart), dy^2 (step), -; maxima: nan, p_rel, p_abs, d_abs
    double v[kQ] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const double a = ax[i];
        const double ys = static_cast<double>(yc[i]);
        if (!isfinite(a) || !isfinite(ys)) v[kNS] = 1.0;
        const double fy = ys - static_cast<double>(yprev[i]);
        v[4] += fy * fy;
        const double ps = a - fmin(fmax(a, rl_s[i]), ru_s[i]);
        const double ao = a / rs[i];
        const double lo = rl_o[i], up = ru_o[i];
        const double po = ao - fmin(fmax(ao, lo), up);
        const double yo = -ys * rs[i];          // verifier sign, original space
        double dt = 0.0;
        if (yo > 0.0 && finite_lo(lo)) dt = yo * lo;
        else if (yo < 0.0 && finite_up(up)) dt = yo * up;
        const double dy = ys - y_last[i];
        v[0] += po * po;
        v[1] += ps * ps;
        v[2] += dt;
        v[3] += dy * dy;
        if (po != 0.0) {
            const double bound = po < 0.0 ? (lo > -1e19 ? fabs(lo) : 1.0) : (up < 1e19 ? fabs(up) : 1.0);
            v[kNS + 1] = fmax(v[kNS + 1], fabs(po) / (1.0 + bound));
            v[kNS + 2] = fmax(v[kNS + 2], fabs(po));
        }
        if (!finite_lo(lo) && finite_up(up) && yo > 0.0) v[kNS + 3] = fmax(v[kNS + 3], yo);
        if (finite_lo(lo) && !finite_up(up) && yo < 0.0) v[kNS + 3] = fmax(v[kNS + 3], -yo);
    }
    store_partials(v, red, part);
}

// Column pass: reduced cost r = c + A^T y (min form), its bound-multiplier part lambda,
// dual residual r - lambda (original and scaled), primal objective, column part of the dual
// objective, distance of x+ from the last restart point, and the guard's reduced-cost sign
// violation (a column more than 1e-7 below its upper bound may not have r < 0, one more than
// 1e-7 above its lower bound may not have r > 0).
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_kkt_cols(int n, const double* __restrict__ aty, const T* __restrict__ xc, const T* __restrict__ xprev,
           const double* __restrict__ c_s, const double* __restrict__ cl_o, const double* __restrict__ cu_o,
           const double* __restrict__ cs, const double* __restrict__ x_last, double* __restrict__ part,
           const HState* st, int phase) {
    if (st->stop || st->phase != phase) return;
    __shared__ double red[kQ * 32];
    // sums: rd_o^2, rd_s^2, pobj, dobj, dx^2 (restart), dx^2 (step); maxima: nan, -, -, d_abs
    double v[kQ] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double at = aty[j];
        const double xs = static_cast<double>(xc[j]);
        if (!isfinite(at) || !isfinite(xs)) v[kNS] = 1.0;
        const double fx = xs - static_cast<double>(xprev[j]);
        v[5] += fx * fx;
        const double lo = cl_o[j], up = cu_o[j];
        const bool lf = finite_lo(lo), uf = finite_up(up);
        const double r_s = c_s[j] + at;
        const double r_o = r_s / cs[j];
        auto lam_of = [&](double r) { return (lf && uf) ? r : lf ? fmax(r, 0.0) : uf ? fmin(r, 0.0) : 0.0; };
        const double lo_lam = lam_of(r_o), ls = lam_of(r_s);
        const double ro = r_o - lo_lam, rsd = r_s - ls;
        double dt = 0.0;
        if (lo_lam > 0.0) dt = lo_lam * lo;
        else if (lo_lam < 0.0) dt = lo_lam * up;
        const double dx = xs - x_last[j];
        v[0] += ro * ro;
        v[1] += rsd * rsd;
        v[2] += c_s[j] * xs;
        v[3] += dt;
        v[4] += dx * dx;
        const double xo = xs * cs[j];
        if (xo < up - kGuardTol && r_o < 0.0) v[kNS + 3] = fmax(v[kNS + 3], -r_o);
        if (xo > lo + kGuardTol && r_o > 0.0) v[kNS + 3] = fmax(v[kNS + 3], r_o);
    }
    store_partials(v, red, part);
}

struct ControlParams {
    double tol;
    double switch_tol;
    double beta_sufficient;
    double beta_necessary;
    double beta_artificial;
    double pw_smoothing;
    int len;          // iterations in the chunk just finished
    int phase;
    double gamma32;   // reflection of the FP32 phase once its KKT is below early_tol
    double gamma64;   // reflection of the FP64 phase
    double early_tol; // FP32 phase: above this KKT it reflects with gamma64 (its noise is far below)
    int mixed;        // 1 when an FP32 phase hands over to FP64
    int stall_checks; // FP32 stall window in checks (0 = no stall test; at most kHist - 1)
    int metric;       // restart metric: 0 weighted KKT, 1 fixed-point residual
    double max_violation;       // > 0: also require the guard's maxima below this
    double max_abs_violation;   // > 0: also require every row violation below this (absolute)
    int handover_mode;          // 0: FP64 phase restarts from the FP32 candidate; 1: continues the epoch
};

constexpr int kS = 2 * kNS;   // sums the control CTA combines (rows, then columns)

__global__ void __launch_bounds__(1024)
k_halpern_control(const double* __restrict__ part_r, const double* __restrict__ part_c, ControlParams cp,
                  HState* st) {
    if (st->stop || st->phase != cp.phase) return;
    __shared__ double red[kS * 32];
    double s[kS];
#pragma unroll
    for (int q = 0; q < kS; ++q) s[q] = 0.0;
    for (int b = threadIdx.x; b < kCheckBlocks; b += blockDim.x) {
        for (int q = 0; q < kNS; ++q) { s[q] += part_r[b * kQ + q]; s[kNS + q] += part_c[b * kQ + q]; }
    }
    block_reduce<OpSum, double, kS>(s, red);
    // maxima: NaN flag, relative and absolute row violation, dual sign violation
    double f[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < kCheckBlocks; b += blockDim.x) {
        const double* r = part_r + b * kQ + kNS;
        const double* c = part_c + b * kQ + kNS;
        f[0] = fmax(f[0], fmax(r[0], c[0]));
        f[1] = fmax(f[1], r[1]);
        f[2] = fmax(f[2], r[2]);
        f[3] = fmax(f[3], fmax(r[3], c[3]));
    }
    block_reduce<OpMax, double, 4>(f, red);
    if (threadIdx.x != 0) return;
    const double rp_o2 = s[0], rp_s2 = s[1], dobj_r = s[2], dy2 = s[3], fy2 = s[4];
    const double rd_o2 = s[kNS], rd_s2 = s[kNS + 1], pobj_s = s[kNS + 2], dobj_c = s[kNS + 3], dx2 = s[kNS + 4],
                 fx2 = s[kNS + 5];
    st->total += cp.len;
    st->phase_iters[cp.phase] += cp.len;
    st->restart_flag = 0;
    st->switch_flag = 0;
    if (f[0] > 0.0 || isnan(rp_o2) || isnan(rd_o2)) {
        st->stop = 1;
        st->status = kStatusNumerical;
        st->stop_iter = st->total;
        return;
    }
    const double pobj = pobj_s + st->offset_min;
    const double dobj = dobj_r + dobj_c + st->offset_min;
    const double rel_p = sqrt(rp_o2) / (1.0 + st->bnorm);
    const double rel_d = sqrt(rd_o2) / (1.0 + st->cnorm);
    const double rel_gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double rel = fmax(rel_p, fmax(rel_d, rel_gap));
    st->rel_p = rel_p; st->rel_d = rel_d; st->rel_gap = rel_gap; st->rel_kkt = rel;
    st->pobj = pobj; st->dobj = dobj;
    st->viol_p_rel = f[1];
    st->viol_p_abs = f[2];
    st->viol_d_abs = f[3];
    // optimal: relative KKT within tolerance and, when asked, the status guard's maxima too
    const bool guard_ok = (cp.max_violation <= 0.0 || (f[1] <= cp.max_violation && f[3] <= cp.max_violation)) &&
                          (cp.max_abs_violation <= 0.0 || f[2] <= cp.max_abs_violation);
    if (rel <= cp.tol && guard_ok) {
        st->stop = 1;
        st->status = kStatusOptimal;
        st->stop_iter = st->total;
        return;
    }
    const double omega = st->omega;
    const double wk = cp.metric == 1 ? sqrt(omega * fx2 + fy2 / omega)
                                     : sqrt(omega * rp_s2 + rd_s2 / omega + rel_gap * rel_gap);
    if (cp.mixed && cp.phase == 0) {
        const int hn = st->hist_n;
        const int w = cp.stall_checks;
        bool stalled = false;
        if (w > 0 && hn >= w) {
            const double old = st->hist[(hn - w) % kHist];
            stalled = rel > 0.98 * old;
        }
        st->hist[hn % kHist] = rel;
        st->hist_n = hn + 1;
        if (rel <= cp.early_tol) st->gamma_now = cp.gamma32;
        if (rel <= cp.switch_tol || stalled) {
            st->switch_flag = 1;
            st->phase = 1;
            st->gamma_now = cp.gamma64;
            if (cp.handover_mode == 1) {   // the FP64 phase continues the FP32 phase's epoch
                st->k_base += cp.len;
            } else {                       // it restarts from the FP32 candidate
                st->k_base = 0;
                st->kkt_start = wk;
                st->kkt_prev = wk;
            }
            return;
        }
    }
    if (st->kkt_start < 0.0) { st->kkt_start = wk; st->kkt_prev = wk; }
    const long long k_in = st->k_base + cp.len;
    const bool restart = (wk <= cp.beta_sufficient * st->kkt_start) ||
                         (wk <= cp.beta_necessary * st->kkt_start && wk > st->kkt_prev) ||
                         (static_cast<double>(k_in) >= cp.beta_artificial * static_cast<double>(st->total));
    st->kkt_prev = wk;
    if (restart) {
        const double dx = sqrt(dx2), dy = sqrt(dy2);
        if (dx > 1e-10 && dy > 1e-10) {
            const double th = cp.pw_smoothing;
            st->omega = exp(th * log(dy / dx) + (1.0 - th) * log(omega));
            st->tau = st->eta / st->omega;
            st->sigma = st->eta * st->omega;
            st->inv_sigma = 1.0 / st->sigma;
        }
        st->k_base = 0;
        st->kkt_start = wk;
        st->kkt_prev = wk;
        st->restart_count += 1;
        st->restart_flag = 1;
    } else {
        st->k_base = k_in;
    }
}

template <typename T>
__global__ void k_halpern_restart(int m, int n, const T* __restrict__ xc, const T* __restrict__ yc, T* __restrict__ x,
                                  T* __restrict__ x0, T* __restrict__ y, T* __restrict__ y0, double* __restrict__ x_last,
                                  double* __restrict__ y_last, const HState* st, int len, double* __restrict__ hw) {
    if (blockIdx.x == 0) halpern_weights(st, len, hw, threadIdx.x, blockDim.x);   // for the next chunk
    if (!st->restart_flag) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { const T v = xc[i]; x[i] = v; x0[i] = v; x_last[i] = static_cast<double>(v); }
    if (i < m) { const T v = yc[i]; y[i] = v; y0[i] = v; y_last[i] = static_cast<double>(v); }
}

// FP32 -> FP64 hand-over that continues the FP32 phase's Halpern epoch: its iterate, anchor
// and candidate carried over as they are.
__global__ void k_handover_keep(int m, int n, const float* __restrict__ x32, const float* __restrict__ x032,
                                const float* __restrict__ xc32, const float* __restrict__ y32,
                                const float* __restrict__ y032, const float* __restrict__ yc32, double* __restrict__ x,
                                double* __restrict__ x0, double* __restrict__ xc, double* __restrict__ y,
                                double* __restrict__ y0, double* __restrict__ yc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { x[i] = x32[i]; x0[i] = x032[i]; xc[i] = xc32[i]; }
    if (i < m) { y[i] = y32[i]; y0[i] = y032[i]; yc[i] = yc32[i]; }
}

// FP32 -> FP64 hand-over: the FP32 candidate becomes the FP64 iterate and anchor.
__global__ void k_handover(int m, int n, const float* __restrict__ xc32, const float* __restrict__ yc32,
                           double* __restrict__ x, double* __restrict__ x0, double* __restrict__ xc,
                           double* __restrict__ y, double* __restrict__ y0, double* __restrict__ yc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { const double v = xc32[i]; x[i] = v; x0[i] = v; xc[i] = v; }
    if (i < m) { const double v = yc32[i]; y[i] = v; y0[i] = v; yc[i] = v; }
}

template <typename T>
__global__ void k_init_iterates(int m, int n, const double* __restrict__ cl, const double* __restrict__ cu,
                                T* __restrict__ x, T* __restrict__ x0, T* __restrict__ xb, T* __restrict__ xc,
                                T* __restrict__ y, T* __restrict__ y0, T* __restrict__ yc,
                                double* __restrict__ x_last, double* __restrict__ y_last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double v = fmin(fmax(0.0, cl[i]), cu[i]);
        x[i] = x0[i] = xb[i] = xc[i] = static_cast<T>(v);
        x_last[i] = static_cast<double>(static_cast<T>(v));
    }
    if (i < m) { y[i] = y0[i] = yc[i] = T(0); y_last[i] = 0.0; }
}

template <typename T>
__global__ void k_to_t(int64_t n, const double* __restrict__ s, T* __restrict__ d) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        d[k] = static_cast<T>(s[k]);
}

// ||b|| (finite row bounds, each equality row once), ||c||, scaled ||b||, ||c|| for the
// initial primal weight.
// ||b|| (every finite row bound, an equality row once) and ||c||, original and scaled:
// block partials over a fixed grid, then one CTA adds them in block order (deterministic).
__global__ void __launch_bounds__(kThreads)
k_norms_part(int m, int n, const double* __restrict__ rl_o, const double* __restrict__ ru_o,
             const double* __restrict__ c_o, const double* __restrict__ rl_s, const double* __restrict__ ru_s,
             const double* __restrict__ c_s, double* __restrict__ part) {
    __shared__ double red[4 * 32];
    double v[4] = {0, 0, 0, 0};
    auto b2 = [](double l, double u) {
        const bool lf = l > -1e20, uf = u < 1e20;
        if (lf && uf && l == u) return l * l;
        return (lf ? l * l : 0.0) + (uf ? u * u : 0.0);
    };
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        v[0] += b2(rl_o[i], ru_o[i]);
        v[2] += b2(rl_s[i], ru_s[i]);
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        v[1] += c_o[j] * c_o[j];
        v[3] += c_s[j] * c_s[j];
    }
    block_reduce<OpSum, double, 4>(v, red);
    if (threadIdx.x == 0) for (int q = 0; q < 4; ++q) part[blockIdx.x * 4 + q] = v[q];
}

__global__ void __launch_bounds__(1024)
k_norms_final(int nb, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double red[4 * 32];
    double v[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        for (int q = 0; q < 4; ++q) v[q] += part[b * 4 + q];
    block_reduce<OpSum, double, 4>(v, red);
    if (threadIdx.x == 0) for (int q = 0; q < 4; ++q) out[q] = sqrt(v[q]);
}

// Unscale and map to the verifier's conventions.  The row dual is the minimisation-form
// multiplier for both senses, which is what verifier::verify_solution and
// Solution::recompute_quality check (src/engine/verifier.cpp:172-262, model.cpp:286-364).
// (The reference PDHG returns +y for maximisation, pdhg.cpp:409-411, which its own verifier
// rejects; VAJRA_ALGO_REFERENCE keeps that for parity.)
__global__ void k_post_vectors(int m, int n, const double* __restrict__ xc, const double* __restrict__ yc,
                               const double* __restrict__ cs, const double* __restrict__ rs, int scaled,
                               double* __restrict__ x_out, double* __restrict__ y_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x_out[i] = scaled ? xc[i] * cs[i] : xc[i];
    if (i < m) { const double v = scaled ? yc[i] * rs[i] : yc[i]; y_out[i] = -v; }
}

template <typename T>
__global__ void k_widen(int k, const T* __restrict__ s, double* __restrict__ d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) d[i] = static_cast<double>(s[i]);
}

// offset + a.b, in the same two deterministic stages.
__global__ void __launch_bounds__(kThreads)
k_dot_part(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double red[32];
    double v[1] = {0.0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) v[0] += a[j] * b[j];
    block_reduce<OpSum, double, 1>(v, red);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(1024)
k_dot_final(int nb, const double* __restrict__ part, double offset, double* __restrict__ out) {
    __shared__ double red[32];
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] += part[b];
    block_reduce<OpSum, double, 1>(v, red);
    if (threadIdx.x == 0) *out = offset + v[0];
}

// Reduced costs as recompute_quality defines them (model.cpp:303-307): d = c - A^T y for
// minimisation, c + A^T y for maximisation (the sign-flipped min-form reduced cost).
__global__ void k_reduced_costs(int n, const double* __restrict__ c, int is_max, double* __restrict__ d) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) d[j] = is_max ? c[j] + d[j] : c[j] - d[j];
}

// One precision's iterate set, kernels and captured chunk graph.
template <typename T>
struct Phase {
    int m = 0, n = 0, phase = 0;
    DeviceBuffer<T> x, x0, xb, xc, xprev, y, y0, yc, yprev;
    DeviceBuffer<T> c, cl, cu, rl, ru;          // iteration copies in T (FP64: separate copies too)
    const T* csr_val = nullptr;
    const T* csc_val = nullptr;
    const T* sell_val_a = nullptr;    // the same values in sliced-ELL order (degree-ordered LPs)
    const T* sell_val_at = nullptr;
    // FP64 phase reading the FP32 copy of the matrix (every scaled value exactly an FP32
    // number): the same products and sums as with the FP64 copy, 4 bytes an entry less
    bool compact = false;
    const float* csr_val32 = nullptr;
    const float* csc_val32 = nullptr;
    const float* sell_val32_a = nullptr;
    const float* sell_val32_at = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};   // around the first iteration of a chunk
    double t_primal_ms = 0.0, t_dual_ms = 0.0;
    int64_t samples = 0;
    int64_t graph_kernels = 0;   // kernels captured in one chunk graph
    ~Phase() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& e : ev) if (e) cudaEventDestroy(e);
    }
    vajra_status alloc(int m_, int n_, const Prepared& p, cudaStream_t st) {
        m = m_; n = n_;
        for (auto& e : ev) VJ_CUDA(cudaEventCreate(&e));
        for (auto* b : {&x, &x0, &xb, &xc, &xprev, &c, &cl, &cu}) VJ_TRY(b->alloc(n));
        for (auto* b : {&y, &y0, &yc, &yprev, &rl, &ru}) VJ_TRY(b->alloc(m));
        const unsigned gn = grid_for(n, kThreads, 148 * 32), gm = grid_for(m, kThreads, 148 * 32);
        k_to_t<T><<<gn, kThreads, 0, st>>>(n, p.c.get(), c.get());
        k_to_t<T><<<gn, kThreads, 0, st>>>(n, p.col_lower.get(), cl.get());
        k_to_t<T><<<gn, kThreads, 0, st>>>(n, p.col_upper.get(), cu.get());
        k_to_t<T><<<gm, kThreads, 0, st>>>(m, p.row_lower.get(), rl.get());
        k_to_t<T><<<gm, kThreads, 0, st>>>(m, p.row_upper.get(), ru.get());
        VJ_LAUNCH_CHECK();
        note_launch(5);
        return VAJRA_OK;
    }
};

// `timed`: bracket the two kernels with event-record nodes (captured into the chunk graph).
// One SpMV of an iteration in shape v.group; the sliced-ELL shape reads its own copy of the
// values (`sell_val`), every other shape the CSR-order ones.
// VV: stored value type, T: vector and accumulation type.
template <typename VV, typename T, class Epi>
void launch_iter(const CsrView& v, const VV* csr_val, const VV* sell_val, const T* x, Epi epi, cudaStream_t st) {
    if (v.group == kSell && v.sell_off && sell_val) launch_sell<VV, T, T>(v, csr_val, sell_val, x, epi, st);
    else if (v.group == kSellHot && v.sell_off && sell_val) launch_sell_hot<VV, T, T>(v, csr_val, sell_val, x, epi, st);
    else launch_spmv_t<VV, T, T>(v, csr_val, x, epi, st);
}

// The two iteration SpMVs of a phase, from the phase's copy of the values (A^T y: stored
// transpose; A x: CSR).
template <typename T, class Epi>
void phase_spmv_at(const Phase<T>& ph, const CsrView& v, const T* x, Epi epi, cudaStream_t st) {
    if constexpr (sizeof(T) == 8) {
        if (ph.compact) { launch_iter<float, T>(v, ph.csc_val32, ph.sell_val32_at, x, epi, st); return; }
    }
    launch_iter<T, T>(v, ph.csc_val, ph.sell_val_at, x, epi, st);
}
template <typename T, class Epi>
void phase_spmv_a(const Phase<T>& ph, const CsrView& v, const T* x, Epi epi, cudaStream_t st) {
    if constexpr (sizeof(T) == 8) {
        if (ph.compact) { launch_iter<float, T>(v, ph.csr_val32, ph.sell_val32_a, x, epi, st); return; }
    }
    launch_iter<T, T>(v, ph.csr_val, ph.sell_val_a, x, epi, st);
}

// The check SpMVs of one phase (FP64 values -- or their exact FP32 copy -- and FP64 sums, the
// phase's iterate type as the vector).
template <typename VV, typename T>
void launch_check_spmv(const CsrView& v, const VV* csr_val, const VV* sell_val, const T* x, double* out,
                       const HState* S, int phase, cudaStream_t st) {
    const EpiStoreActive epi{out, S, phase};
    if (v.group == kSell && v.sell_off && sell_val) launch_sell<VV, T, double>(v, csr_val, sell_val, x, epi, st);
    else if (v.group == kSellHot && v.sell_off && sell_val)
        launch_sell_hot<VV, T, double>(v, csr_val, sell_val, x, epi, st);
    else launch_spmv_t<VV, T, double>(v, csr_val, x, epi, st);
}

// Shared-memory grants of the hot-prefix kernels a phase may launch (outside any capture).
template <typename T>
vajra_status prepare_hot_kernels() {
    VJ_CUDA((sell_hot_prepare<T, T, T, EpiHPrimal<T>>()));
    VJ_CUDA((sell_hot_prepare<T, T, T, EpiHDual<T>>()));
    VJ_CUDA((sell_hot_prepare<double, T, double, EpiStoreActive>()));
    VJ_CUDA((sell_hot_prepare<float, T, double, EpiStoreActive>()));
    if constexpr (sizeof(T) == 8) {
        VJ_CUDA((sell_hot_prepare<float, T, T, EpiHPrimal<T>>()));
        VJ_CUDA((sell_hot_prepare<float, T, T, EpiHDual<T>>()));
    }
    return VAJRA_OK;
}

template <typename T>
void enqueue_iteration(Phase<T>& ph, const CsrView& a, const CsrView& at, HState* S, const double* hw, int kk,
                       int write_cand, bool timed, cudaStream_t st) {
    if (timed) cudaEventRecordWithFlags(ph.ev[0], st, cudaEventRecordExternal);
    phase_spmv_at(ph, at, ph.y.get(),
                  EpiHPrimal<T>{ph.c.get(), ph.cl.get(), ph.cu.get(), ph.x0.get(), ph.x.get(), ph.xb.get(),
                                ph.xc.get(), ph.xprev.get(), S, hw, kk, ph.phase, write_cand}, st);
    if (timed) cudaEventRecordWithFlags(ph.ev[1], st, cudaEventRecordExternal);
    phase_spmv_a(ph, a, ph.xb.get(),
                 EpiHDual<T>{ph.rl.get(), ph.ru.get(), ph.y0.get(), ph.y.get(), ph.yc.get(), ph.yprev.get(), S, hw, kk,
                             ph.phase, write_cand}, st);
    if (timed) cudaEventRecordWithFlags(ph.ev[2], st, cudaEventRecordExternal);
}

struct CheckBuffers {
    DeviceBuffer<double> ax, aty, part_r, part_c, x_last, y_last;
    DeviceBuffer<double> hw;   // Halpern weights of the current chunk (2 per iteration)
    int hw_len = 0;            // iterations a chunk can hold
    bool compact_checks = false;   // check SpMVs read the exact FP32 copy of the values
};

template <typename T>
void enqueue_check(Phase<T>& ph, const CsrView& a64, const CsrView& at64, const Prepared& p, const DeviceLp& lp,
                   CheckBuffers& cb, HState* S, const ControlParams& cp, cudaStream_t st) {
    // FP64 values of the scaled A (their FP32 copy where that is exact); in sliced-ELL order
    // too when that is the FP64 shape
    if (cb.compact_checks) {
        launch_check_spmv<float, T>(a64, p.csr_val32.get(), p.sell_a.val32.get(), ph.xc.get(), cb.ax.get(), S,
                                    ph.phase, st);
        launch_check_spmv<float, T>(at64, p.csc_val32.get(), p.sell_at.val32.get(), ph.yc.get(), cb.aty.get(), S,
                                    ph.phase, st);
    } else {
        launch_check_spmv<double, T>(a64, p.csr_val.get(), p.sell_a.val64.get(), ph.xc.get(), cb.ax.get(), S,
                                     ph.phase, st);
        launch_check_spmv<double, T>(at64, p.csc_val.get(), p.sell_at.val64.get(), ph.yc.get(), cb.aty.get(), S,
                                     ph.phase, st);
    }
    k_kkt_rows<T><<<kCheckBlocks, kThreads, 0, st>>>(ph.m, cb.ax.get(), ph.yc.get(), ph.yprev.get(), p.row_lower.get(), p.row_upper.get(),
                                                     lp.row_lower.get(), lp.row_upper.get(), p.row_scale.get(),
                                                     cb.y_last.get(), cb.part_r.get(), S, ph.phase);
    k_kkt_cols<T><<<kCheckBlocks, kThreads, 0, st>>>(ph.n, cb.aty.get(), ph.xc.get(), ph.xprev.get(), p.c.get(), lp.col_lower.get(),
                                                     lp.col_upper.get(), p.col_scale.get(), cb.x_last.get(),
                                                     cb.part_c.get(), S, ph.phase);
    k_halpern_control<<<1, 1024, 0, st>>>(cb.part_r.get(), cb.part_c.get(), cp, S);
    const int mx = ph.m > ph.n ? ph.m : ph.n;
    k_halpern_restart<T><<<grid_for(mx), kThreads, 0, st>>>(ph.m, ph.n, ph.xc.get(), ph.yc.get(), ph.x.get(),
                                                            ph.x0.get(), ph.y.get(), ph.y0.get(), cb.x_last.get(),
                                                            cb.y_last.get(), S, cb.hw_len, cb.hw.get());
    note_launch(4);
}

template <typename T>
void enqueue_chunk(Phase<T>& ph, const CsrView& a, const CsrView& at, const CsrView& a64, const CsrView& at64,
                   const Prepared& p, const DeviceLp& lp, CheckBuffers& cb, HState* S, int len,
                   ControlParams cp, bool capturing, cudaStream_t st) {
    // Event-record nodes (cudaEventRecordExternal) exist only inside a stream capture.
    for (int kk = 0; kk < len; ++kk)
        enqueue_iteration(ph, a, at, S, cb.hw.get(), kk, kk == len - 1 ? 1 : 0, kk == 0 && capturing, st);
    cp.len = len;
    cp.phase = ph.phase;
    enqueue_check(ph, a64, at64, p, lp, cb, S, cp, st);
}

// Times every launch shape (row-block kernel with one or two load groups, 1..32 lanes per
// row, and sliced ELL where the set-up built it) of both iteration kernels with their real
// epilogues and keeps the fastest per matrix.  `tune_state` is a scratch state whose phase is
// the tuned one; the iterates it scribbles on are re-initialised after.
template <typename T>
vajra_status autotune_iteration(Phase<T>& ph, CsrView& a, CsrView& at, HState* tune_state, const CheckBuffers& cb,
                                cudaStream_t st) {
    const double* hw = cb.hw.get();
    k_halpern_weights<<<1, kThreads, 0, st>>>(tune_state, cb.hw_len, cb.hw.get());
    note_launch(1);
    cudaEvent_t e0, e1;
    VJ_CUDA(cudaEventCreate(&e0));
    VJ_CUDA(cudaEventCreate(&e1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } guard{e0, e1};
    // Every shape: one warm launch and three timed ones.  The three fastest then run three
    // more rounds of four launches each, taking turns (so a drift of the clock or of the
    // neighbours' load spreads over all of them), and the smallest total wins: shapes a few
    // per cent apart are not told apart by one three-launch sample.
    auto time_shapes = [&](CsrView& v, auto launch) -> vajra_status {
        if (v.rows <= 0) return VAJRA_OK;
        constexpr int kFinal = 3;
        // (the hot-prefix sliced-ELL shape is not a candidate: it measured 2x slower than plain
        // sliced ELL on every LP tried; callers can still force it)
        int shapes[9] = {0, kRowblock2, 1, 2, 4, 8, 16, 32, kSell};
        const int kShapes = v.sell_off ? 9 : 8;
        auto timed = [&](int g, int launches, float* ms) -> vajra_status {
            CsrView t = v;
            t.group = g;
            VJ_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < launches; ++r) launch(t);
            VJ_CUDA(cudaEventRecord(e1, st));
            VJ_CUDA(cudaEventSynchronize(e1));
            VJ_CUDA(cudaEventElapsedTime(ms, e0, e1));
            return VAJRA_OK;
        };
        float first[9];
        for (int i = 0; i < kShapes; ++i) {
            CsrView t = v;
            t.group = shapes[i];
            launch(t);   // warm
            VJ_TRY(timed(shapes[i], 3, &first[i]));
        }
        int order[9];
        for (int i = 0; i < kShapes; ++i) order[i] = i;
        std::sort(order, order + kShapes, [&](int a, int b) { return first[a] < first[b]; });
        float total[kFinal] = {0.f, 0.f, 0.f};
        for (int round = 0; round < 3; ++round)
            for (int f = 0; f < kFinal; ++f) {
                float ms = 0.f;
                VJ_TRY(timed(shapes[order[f]], 4, &ms));
                total[f] += ms;
            }
        int best = 0;
        for (int f = 1; f < kFinal; ++f)
            if (total[f] < total[best]) best = f;
        v.group = shapes[order[best]];
        return VAJRA_OK;
    };
    VJ_TRY(time_shapes(at, [&](const CsrView& t) {
        phase_spmv_at(ph, t, ph.y.get(),
                      EpiHPrimal<T>{ph.c.get(), ph.cl.get(), ph.cu.get(), ph.x0.get(), ph.x.get(), ph.xb.get(),
                                    ph.xc.get(), ph.xprev.get(), tune_state, hw, 0, ph.phase, 0}, st);
    }));
    VJ_TRY(time_shapes(a, [&](const CsrView& t) {
        phase_spmv_a(ph, t, ph.xb.get(),
                     EpiHDual<T>{ph.rl.get(), ph.ru.get(), ph.y0.get(), ph.y.get(), ph.yc.get(), ph.yprev.get(),
                                 tune_state, hw, 0, ph.phase, 0}, st);
    }));
    return VAJRA_OK;
}

template <typename T>
void init_iterates(Phase<T>& ph, const Prepared& p, CheckBuffers& cb, cudaStream_t st) {
    const int mx = ph.m > ph.n ? ph.m : ph.n;
    k_init_iterates<T><<<grid_for(mx), kThreads, 0, st>>>(ph.m, ph.n, p.col_lower.get(), p.col_upper.get(), ph.x.get(),
                                                          ph.x0.get(), ph.xb.get(), ph.xc.get(), ph.y.get(), ph.y0.get(),
                                                          ph.yc.get(), cb.x_last.get(), cb.y_last.get());
    note_launch(1);
}

// Launch shapes found by the autotuner, shared by every handle of the process whose LP has the
// same device, dimensions and number of entries (the shapes only change speed, never results),
// so repeated solves of one LP pay the timing runs once.
struct TuneKey {
    int device, m, n;
    int64_t nnz;
    int ordered;
    int compact;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, m, n, nnz, ordered, compact) < std::tie(o.device, o.m, o.n, o.nnz, o.ordered, o.compact);
    }
};
struct TuneEntry { int bits = 0, a32 = 8, at32 = 8, a64 = 8, at64 = 8; };
std::mutex g_tune_mutex;
std::map<TuneKey, TuneEntry> g_tune_cache;

}  // namespace

vajra_status run_halpern(vajra_pdhg* h, vajra_result* r) {
    const auto t_start = Clock::now();
    cudaStream_t st = h->stream;
    StreamTimer dev_timer;
    dev_timer.start(st);
    const vajra_opts& o = h->opts;
    const int m = h->m, n = h->n;
    const int64_t nnz = h->nnz;
    const bool is_max = h->sense != 0;
    const bool mixed = o.precision == VAJRA_PREC_MIXED;
    // Degree ordering (built once per handle); the result vectors go back to the caller's
    // numbering at the end.  Below ~1M entries the vectors stay in cache anyway.
    constexpr int64_t kOrderMinNnz = int64_t(1) << 20;
    const bool ordered = o.degree_order > 0 || (o.degree_order == 0 && nnz >= kOrderMinNnz);
    // verbose: host time of each set-up step (the stream drained at each mark)
    auto mark = [&](const char* what) {
        if (!o.verbose) return;
        cudaStreamSynchronize(st);
        std::fprintf(stderr, "[vajra] set-up %-14s %8.1f ms\n", what, 1e3 * seconds_since(t_start));
    };
    if (ordered && !h->ordered) {
        VJ_TRY(order_by_degree(h->lp, h->lp_ordered, h->order, st));
        h->ordered = true;
    }
    const DeviceLp& lp = ordered ? h->lp_ordered : h->lp;
    mark("ordering");

    Prepared p;
    DeviceBuffer<SetupState> sst;
    VJ_TRY(sst.alloc(1));
    VJ_TRY(build_csr(lp, p, st));
    mark("csr");
    ScalingOpts so;
    so.enable = o.enable_scaling != 0;
    so.ruiz_iterations = o.ruiz_iterations > 0 ? o.ruiz_iterations : 10;
    so.ruiz_tolerance = 0.05;
    so.pock_chambolle = o.pock_chambolle != 0;
    so.negate_c = is_max;
    so.pow2 = o.pow2_scaling != 0;
    VJ_TRY(prepare_scaled(lp, p, so, sst.get(), st));
    mark("scaling");
    VJ_TRY(plan_spmv(lp, p, st));
    mark("partitions");
    // FP64 iterations and checks on the FP32 copy of the values where that copy is exact
    const bool want_compact = o.fp64_value_storage == 2 || (o.fp64_value_storage == 0 && mixed);
    bool compact = false;
    if (want_compact) VJ_TRY(values_fit_fp32(p, nnz, &compact, st));
    if (mixed || compact) VJ_TRY(make_f32_values(p, nnz, st));
    // Sliced-ELL copies of both matrices (full slices need rows of similar length, which the
    // degree ordering provides): one more launch shape for the autotuner, and the power
    // iteration's SpMVs.  Without the ordering they are built only when a caller forces the
    // shape.
    if (ordered || o.spmv_shape_a <= -3 || o.spmv_shape_at <= -3) {
        VJ_TRY(build_sell(p.a, p.csr_val.get(), mixed || compact ? p.csr_val32.get() : nullptr, p.sell_a, st));
        VJ_TRY(build_sell(p.at, p.csc_val.get(), mixed || compact ? p.csc_val32.get() : nullptr, p.sell_at, st));
    }
    mark("sliced ell");
    if (p.a.sell_off || p.at.sell_off) {
        if (mixed) VJ_TRY(prepare_hot_kernels<float>());
        VJ_TRY(prepare_hot_kernels<double>());
    }
    VJ_TRY(spectral_norm_fast(p, m, n, 100, 1e-5, sst.get(), st));
    mark("norm estimate");
    SetupState hss{};
    VJ_CUDA(cudaMemcpyAsync(&hss, sst.get(), sizeof(hss), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    const double spectral_norm = hss.spectral_norm;
    if (!(spectral_norm > 1e-12) || !std::isfinite(spectral_norm)) {
        r->status = kStatusNumerical;
        std::snprintf(r->status_message, sizeof(r->status_message), "invalid spectral norm estimate %g", spectral_norm);
        return VAJRA_OK;
    }

    // Norms for the relative KKT and the initial primal weight.
    DeviceBuffer<double> norms;
    VJ_TRY(norms.alloc(4));
    DeviceBuffer<double> red_part;
    VJ_TRY(red_part.alloc(4 * static_cast<size_t>(kCheckBlocks)));
    k_norms_part<<<kCheckBlocks, kThreads, 0, st>>>(m, n, lp.row_lower.get(), lp.row_upper.get(), lp.c.get(),
                                                   p.row_lower.get(), p.row_upper.get(), p.c.get(), red_part.get());
    k_norms_final<<<1, 1024, 0, st>>>(kCheckBlocks, red_part.get(), norms.get());
    VJ_LAUNCH_CHECK();
    note_launch(2);
    double hn[4];
    VJ_CUDA(cudaMemcpyAsync(hn, norms.get(), sizeof(hn), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));

    Phase<float> p32;
    Phase<double> p64;
    p32.phase = 0;
    p64.phase = 1;
    if (mixed) {
        VJ_TRY(p32.alloc(m, n, p, st));
        p32.csr_val = p.csr_val32.get();
        p32.csc_val = p.csc_val32.get();
        p32.sell_val_a = p.a.sell_off ? p.sell_a.val32.get() : nullptr;
        p32.sell_val_at = p.at.sell_off ? p.sell_at.val32.get() : nullptr;
    }
    VJ_TRY(p64.alloc(m, n, p, st));
    p64.csr_val = p.csr_val.get();
    p64.csc_val = p.csc_val.get();
    p64.sell_val_a = p.a.sell_off ? p.sell_a.val64.get() : nullptr;
    p64.sell_val_at = p.at.sell_off ? p.sell_at.val64.get() : nullptr;
    if (compact) {
        p64.compact = true;
        p64.csr_val32 = p.csr_val32.get();
        p64.csc_val32 = p.csc_val32.get();
        p64.sell_val32_a = p.a.sell_off ? p.sell_a.val32.get() : nullptr;
        p64.sell_val32_at = p.at.sell_off ? p.sell_at.val32.get() : nullptr;
    }

    mark("iterate buffers");
    CheckBuffers cb;
    VJ_TRY(cb.ax.alloc(m));
    VJ_TRY(cb.aty.alloc(n));
    VJ_TRY(cb.part_r.alloc(kCheckBlocks * kQ));
    VJ_TRY(cb.part_c.alloc(kCheckBlocks * kQ));
    VJ_TRY(cb.x_last.alloc(n));
    VJ_TRY(cb.y_last.alloc(m));
    const int K = o.check_frequency > 0 ? o.check_frequency : 64;
    cb.hw_len = K;
    cb.compact_checks = compact;
    VJ_TRY(cb.hw.alloc(2 * static_cast<size_t>(K)));

    HState init{};
    const double eta = (o.step_safety > 0.0 && o.step_safety < 1.0 ? o.step_safety : 0.99) / spectral_norm;
    init.omega = (hn[2] > 1e-10 && hn[3] > 1e-10) ? hn[3] / hn[2] : 1.0;
    init.eta = eta;
    init.tau = eta / init.omega;
    init.sigma = eta * init.omega;
    init.inv_sigma = 1.0 / init.sigma;
    init.kkt_start = -1.0;
    init.kkt_prev = -1.0;
    init.bnorm = hn[0];
    init.cnorm = hn[1];
    init.offset_min = is_max ? -h->objective_offset : h->objective_offset;
    init.phase = mixed ? 0 : 1;
    init.rel_kkt = 1e30;
    DeviceBuffer<HState> dstate;
    VJ_TRY(dstate.alloc(1));

    // Launch shapes, tuned per precision with the real iteration kernels: (a32, at32) for the
    // FP32 phase, (a64, at64) for the FP64 iterations; every FP64 check uses (a64, at64) too.
    // A handle keeps its first tuning.
    const double gamma = o.reflection;
    const double gamma32 = (o.mixed_reflection > 0.0 && o.mixed_reflection <= 1.0) ? o.mixed_reflection : gamma;
    // The FP32 phase averages its reflection only near its noise floor: far above it (more
    // than kEarlyReflection x the hand-over tolerance) it takes the full FP64 step.
    constexpr double kEarlyReflection = 10.0;
    const double early_tol = kEarlyReflection * o.mixed_switch_tolerance;
    init.gamma_now = gamma;   // the FP32 phase starts with the full step too
    CsrView a64 = p.a, at64 = p.at;
    CsrView a32 = p.a, at32 = p.at;
    // Below ~1M entries a solve is launch-bound and the timing runs would cost more than any
    // shape saves: the set-up heuristic (lanes per row from the mean row length) stays.
    constexpr int64_t kAutotuneMinNnz = int64_t(1) << 20;
    const TuneKey tkey{h->device, m, n, nnz, ordered ? 1 : 0, compact ? 1 : 0};
    if (o.autotune) {   // shapes another handle already tuned for this LP
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(tkey);
        if (it != g_tune_cache.end()) {
            const TuneEntry& e = it->second;
            if ((e.bits & 1) && !(h->tuned & 1)) { h->tuned_a32 = e.a32; h->tuned_at32 = e.at32; h->tuned |= 1; }
            if ((e.bits & 2) && !(h->tuned & 2)) { h->tuned_a64 = e.a64; h->tuned_at64 = e.at64; h->tuned |= 2; }
        }
    }
    mark("shape lookup");
    if (o.autotune && nnz >= kAutotuneMinNnz && (!(h->tuned & 2) || (mixed && !(h->tuned & 1)))) {
        HState tune = init;
        if (mixed && !(h->tuned & 1)) {
            tune.phase = 0;
            VJ_CUDA(cudaMemcpyAsync(dstate.get(), &tune, sizeof(tune), cudaMemcpyHostToDevice, st));
            init_iterates(p32, p, cb, st);
            VJ_TRY(autotune_iteration<float>(p32, a32, at32, dstate.get(), cb, st));
            h->tuned_a32 = a32.group;
            h->tuned_at32 = at32.group;
            h->tuned |= 1;
        }
        if (!(h->tuned & 2)) {
            tune.phase = 1;
            VJ_CUDA(cudaMemcpyAsync(dstate.get(), &tune, sizeof(tune), cudaMemcpyHostToDevice, st));
            init_iterates(p64, p, cb, st);
            VJ_TRY(autotune_iteration<double>(p64, a64, at64, dstate.get(), cb, st));
            h->tuned_a64 = a64.group;
            h->tuned_at64 = at64.group;
            h->tuned |= 2;
        }
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        TuneEntry& e = g_tune_cache[tkey];
        if (h->tuned & 1) { e.a32 = h->tuned_a32; e.at32 = h->tuned_at32; }
        if (h->tuned & 2) { e.a64 = h->tuned_a64; e.at64 = h->tuned_at64; }
        e.bits |= h->tuned;
    }
    if (h->tuned & 1) {
        a32.group = h->tuned_a32;
        at32.group = h->tuned_at32;
    }
    if (h->tuned & 2) {
        a64.group = h->tuned_a64;
        at64.group = h->tuned_at64;
    }
    auto forced = [](int32_t shape, CsrView& v32, CsrView& v64) {   // caller-fixed shapes
        if (shape == -1 || shape == -2 || shape == 1 || shape == 2 || shape == 4 || shape == 8 || shape == 16 ||
            shape == 32)
            v32.group = v64.group = shape == -1 ? 0 : (shape == -2 ? kRowblock2 : shape);
        if (shape == -3) v32.group = v64.group = v32.sell_off ? kSell : 0;   // sliced ELL, else row block
        if (shape == -4) v32.group = v64.group = v32.sell_off ? kSellHot : 0;   // ... with the hot prefix
    };
    forced(o.spmv_shape_a, a32, a64);
    forced(o.spmv_shape_at, at32, at64);
    const CsrView& a_it = mixed ? a32 : a64;     // shapes reported for the dominant phase
    const CsrView& at_it = mixed ? at32 : at64;

    const int mx = m > n ? m : n;
    if (mixed) init_iterates(p32, p, cb, st);
    else init_iterates(p64, p, cb, st);
    VJ_LAUNCH_CHECK();
    VJ_CUDA(cudaMemcpyAsync(dstate.get(), &init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_halpern_weights<<<1, kThreads, 0, st>>>(dstate.get(), cb.hw_len, cb.hw.get());
    VJ_LAUNCH_CHECK();
    note_launch(1);
    VJ_CUDA(cudaStreamSynchronize(st));
    mark("launch shapes");
    const double setup_time = seconds_since(t_start);

    HState* S = dstate.get();
    HState* hs = nullptr;
    hs = static_cast<HState*>(pinned_scratch(sizeof(HState)));
    if (!hs) { set_error("page-locked host memory for the solver state"); return VAJRA_ERR_OUT_OF_MEMORY; }

    ControlParams cp{};
    cp.tol = o.tolerance;
    cp.switch_tol = o.mixed_switch_tolerance;
    cp.gamma32 = gamma32;
    cp.gamma64 = gamma;
    cp.early_tol = early_tol;
    cp.beta_sufficient = o.restart_sufficient;
    cp.beta_necessary = o.restart_necessary;
    cp.beta_artificial = o.restart_artificial;
    cp.pw_smoothing = o.primal_weight_smoothing;
    cp.mixed = mixed ? 1 : 0;
    cp.metric = o.restart_metric == 1 ? 1 : 0;
    cp.max_violation = o.max_violation;
    cp.max_abs_violation = o.max_abs_violation;
    // Hand-over to the FP64 phase: continue the FP32 phase's epoch on LPs of 2^20 entries or
    // more (the degree-ordering threshold), restart from the FP32 candidate below it, unless
    // the caller chose (1 / 0).  Measured: on four LPs of 3M-20M entries continuing was faster
    // (1M x 2M: 5.09 -> 4.94 s) or the same; on LPs of 40k-400k entries it was slower.
    const bool continue_epoch = o.handover_mode == 1 || (o.handover_mode < 0 && nnz >= kOrderMinNnz);
    cp.handover_mode = continue_epoch ? 1 : 0;
    cp.stall_checks = o.mixed_stall_checks < 0 ? 0 : (o.mixed_stall_checks > kHist - 1 ? kHist - 1 : o.mixed_stall_checks);
    const int64_t max_iter = o.iteration_limit;

    const auto t_iter = Clock::now();
    int64_t launched = 0;
    int cur_phase = mixed ? 0 : 1;
    int timed_out = 0;
    while (launched < max_iter) {
        const int64_t remaining = max_iter - launched;
        const int len = static_cast<int>(remaining < K ? remaining : K);
        auto run_chunk = [&](auto& ph) -> vajra_status {
            const CsrView& ia = ph.phase == 0 ? a32 : a64;
            const CsrView& iat = ph.phase == 0 ? at32 : at64;
            if (len == K) {
                if (!ph.exec) {
                    const auto t_graph = Clock::now();
                    const int64_t before = launch_count();
                    VJ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                    enqueue_chunk(ph, ia, iat, a64, at64, p, lp, cb, S, len, cp, true, st);
                    VJ_CUDA(cudaStreamEndCapture(st, &ph.graph));
                    VJ_CUDA(cudaGraphInstantiate(&ph.exec, ph.graph, 0));
                    ph.graph_kernels = launch_count() - before;
                    launch_count() = before;
                    if (o.verbose)
                        std::fprintf(stderr, "[vajra] chunk graph of phase %d (%lld kernels): capture + instantiate %.2f ms\n",
                                     ph.phase, static_cast<long long>(ph.graph_kernels), 1e3 * seconds_since(t_graph));
                }
                VJ_CUDA(cudaGraphLaunch(ph.exec, st));
                note_launch(ph.graph_kernels);
            } else {
                enqueue_chunk(ph, ia, iat, a64, at64, p, lp, cb, S, len, cp, false, st);
                VJ_LAUNCH_CHECK();
            }
            return VAJRA_OK;
        };
        if (cur_phase == 0) { VJ_TRY(run_chunk(p32)); } else { VJ_TRY(run_chunk(p64)); }
        launched += len;
        VJ_CUDA(cudaMemcpyAsync(hs, S, sizeof(HState), cudaMemcpyDeviceToHost, st));
        VJ_CUDA(cudaStreamSynchronize(st));
        h->transfers++;
        // Kernel durations of this chunk's first iteration, unless that phase had stopped
        // working before the chunk began (then its kernels returned at once).
        if (len > 1 && (hs->phase == cur_phase || hs->switch_flag) &&
            !(hs->stop && hs->stop_iter < launched - len + 1)) {
            float t01 = 0.f, t12 = 0.f;
            cudaEvent_t* ev = cur_phase == 0 ? p32.ev : p64.ev;
            if (cudaEventElapsedTime(&t01, ev[0], ev[1]) == cudaSuccess &&
                cudaEventElapsedTime(&t12, ev[1], ev[2]) == cudaSuccess) {
                auto& ph_t = cur_phase == 0 ? p32.t_primal_ms : p64.t_primal_ms;
                auto& ph_d = cur_phase == 0 ? p32.t_dual_ms : p64.t_dual_ms;
                auto& ph_n = cur_phase == 0 ? p32.samples : p64.samples;
                ph_t += t01;
                ph_d += t12;
                ph_n += 1;
            }
            cudaGetLastError();
        }
        if (hs->stop) break;
        if (hs->phase != cur_phase) {
            if (continue_epoch)
                k_handover_keep<<<grid_for(mx), kThreads, 0, st>>>(m, n, p32.x.get(), p32.x0.get(), p32.xc.get(),
                                                                   p32.y.get(), p32.y0.get(), p32.yc.get(), p64.x.get(),
                                                                   p64.x0.get(), p64.xc.get(), p64.y.get(), p64.y0.get(),
                                                                   p64.yc.get());
            else
                k_handover<<<grid_for(mx), kThreads, 0, st>>>(m, n, p32.xc.get(), p32.yc.get(), p64.x.get(),
                                                              p64.x0.get(), p64.xc.get(), p64.y.get(), p64.y0.get(),
                                                              p64.yc.get());
            VJ_LAUNCH_CHECK();
            note_launch(1);
            cur_phase = hs->phase;
        }
        if (o.verbose)
            std::fprintf(stderr, "[vajra] it %lld phase %d rel_kkt %.3e (p %.2e d %.2e gap %.2e) omega %.4g restarts %d\n",
                         hs->total, hs->phase, hs->rel_kkt, hs->rel_p, hs->rel_d, hs->rel_gap, hs->omega,
                         hs->restart_count);
        if (seconds_since(t_start) > o.time_limit) { timed_out = 1; break; }
    }
    const double iter_time = seconds_since(t_iter);
    if (o.verbose) std::fprintf(stderr, "[vajra] iterations %.2f ms (%lld host reads)\n", 1e3 * iter_time,
                                static_cast<long long>(h->transfers));

    // The returned point is the last evaluated candidate T(z) of the active precision.
    const auto t_post = Clock::now();
    DeviceBuffer<double> xc64, yc64, x_out, y_out, row_value, col_dual, obj;
    VJ_TRY(xc64.alloc(n));
    VJ_TRY(yc64.alloc(m));
    VJ_TRY(x_out.alloc(n));
    VJ_TRY(y_out.alloc(m));
    VJ_TRY(row_value.alloc(m));
    VJ_TRY(col_dual.alloc(n));
    VJ_TRY(obj.alloc(1));
    if (cur_phase == 0) {
        k_widen<float><<<grid_for(n), kThreads, 0, st>>>(n, p32.xc.get(), xc64.get());
        k_widen<float><<<grid_for(m), kThreads, 0, st>>>(m, p32.yc.get(), yc64.get());
    } else {
        VJ_CUDA(cudaMemcpyAsync(xc64.get(), p64.xc.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        VJ_CUDA(cudaMemcpyAsync(yc64.get(), p64.yc.get(), sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
    }
    k_post_vectors<<<grid_for(mx), kThreads, 0, st>>>(m, n, xc64.get(), yc64.get(), p.col_scale.get(), p.row_scale.get(),
                                                      p.scaled ? 1 : 0, x_out.get(), y_out.get());
    launch_spmv_t<double, double, double>(a64, p.csr_val_orig.get(), x_out.get(), EpiStore<double>{row_value.get()}, st);
    launch_spmv_t<double, double, double>(at64, lp.values.get(), y_out.get(), EpiStore<double>{col_dual.get()}, st);
    k_reduced_costs<<<grid_for(n), kThreads, 0, st>>>(n, lp.c.get(), is_max ? 1 : 0, col_dual.get());
    k_dot_part<<<kCheckBlocks, kThreads, 0, st>>>(n, lp.c.get(), x_out.get(), cb.part_r.get());
    k_dot_final<<<1, 1024, 0, st>>>(kCheckBlocks, cb.part_r.get(), h->objective_offset, obj.get());
    VJ_LAUNCH_CHECK();
    note_launch(cur_phase == 0 ? 6 : 4);
    const double* out_x = x_out.get();
    const double* out_row_value = row_value.get();
    const double* out_y = y_out.get();
    const double* out_col_dual = col_dual.get();
    DeviceBuffer<double> ux, urv, uy, ucd;   // the caller's numbering
    if (ordered) {
        VJ_TRY(ux.alloc(n));
        VJ_TRY(urv.alloc(m));
        VJ_TRY(uy.alloc(m));
        VJ_TRY(ucd.alloc(n));
        VJ_TRY(unorder(n, h->order.col_order.get(), x_out.get(), ux.get(), st));
        VJ_TRY(unorder(m, h->order.row_order.get(), row_value.get(), urv.get(), st));
        VJ_TRY(unorder(m, h->order.row_order.get(), y_out.get(), uy.get(), st));
        VJ_TRY(unorder(n, h->order.col_order.get(), col_dual.get(), ucd.get(), st));
        out_x = ux.get();
        out_row_value = urv.get();
        out_y = uy.get();
        out_col_dual = ucd.get();
    }
    double objective = 0.0;
    VJ_CUDA(cudaMemcpyAsync(&objective, obj.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hs, S, sizeof(HState), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    const double post_time = seconds_since(t_post);

    dev_timer.stop(st);
    r->device_time_sec = dev_timer.seconds();
    const auto t_dl = Clock::now();
    copy_out_vector(r->col_value, out_x, n, st);
    copy_out_vector(r->row_value, out_row_value, m, st);
    copy_out_vector(r->row_dual, out_y, m, st);
    copy_out_vector(r->col_dual, out_col_dual, n, st);
    VJ_CUDA(cudaStreamSynchronize(st));
    h->transfers += 4;

    int status = hs->status;
    if (!hs->stop) status = timed_out ? kStatusTimeLimit : kStatusIterLimit;
    r->status = status;
    r->iterations = hs->total;
    r->objective_value = objective;
    r->dual_objective = is_max ? -hs->dobj : hs->dobj;
    r->restart_count = hs->restart_count;
    r->primal_residual = hs->viol_p_abs;   // max-abs residuals, as PdhgDiagnostics reports them
    r->dual_residual = hs->viol_d_abs;
    r->duality_gap = hs->rel_gap;
    r->spectral_norm_estimate = spectral_norm;
    r->tau = hs->tau;
    r->sigma = hs->sigma;
    r->converged = status == kStatusOptimal ? 1 : 0;
    r->rel_primal = hs->rel_p;
    r->rel_dual = hs->rel_d;
    r->rel_gap = hs->rel_gap;
    r->rel_kkt = hs->rel_kkt;
    r->primal_weight = hs->omega;
    r->fp32_iterations = hs->phase_iters[0];
    r->fp64_iterations = hs->phase_iters[1];
    r->setup_time_sec = setup_time;
    r->iteration_time_sec = iter_time + post_time;
    r->download_time_sec = seconds_since(t_dl);
    r->spmv_group_a = a_it.group;
    r->spmv_group_at = at_it.group;
    {
        const bool use32 = mixed && hs->phase_iters[0] >= hs->phase_iters[1];
        const double vs = use32 ? 4.0 : 8.0;                        // vector bytes
        const double vb = (use32 || p64.compact) ? 4.0 : 8.0;       // matrix value bytes
        const double nn = static_cast<double>(nnz), dm = m, dn = n;
        const double t = use32 ? p32.t_primal_ms : p64.t_primal_ms, d = use32 ? p32.t_dual_ms : p64.t_dual_ms;
        const int64_t ns = use32 ? p32.samples : p64.samples;
        r->kernel_samples = ns;
        r->primal_kernel_us = ns ? 1e3 * t / ns : 0.0;
        r->dual_kernel_us = ns ? 1e3 * d / ns : 0.0;
        // primal: CSC pointers (int64), indices + values, y gathered once, c/l/u/x/x0 read,
        // x and x_bar written.  dual: CSR pointers, indices + values, x_bar gathered once,
        // l/u/y/y0 read, y written.
        r->primal_kernel_bytes = 8.0 * (dn + 1) + (4.0 + vb) * nn + vs * dm + 7.0 * vs * dn;
        r->dual_kernel_bytes = 8.0 * (dm + 1) + (4.0 + vb) * nn + vs * dn + 5.0 * vs * dm;
    }
    const char* msg = status == kStatusOptimal ? "relative KKT tolerance reached"
                    : status == kStatusNumerical ? "NaN/Inf in the KKT evaluation"
                    : status == kStatusTimeLimit ? "time limit reached" : "iteration limit reached";
    std::snprintf(r->status_message, sizeof(r->status_message), "%s", msg);
    return VAJRA_OK;
}

}  // namespace vajra
