// Device state of VAJRA_ALGO_HALPERN and the epilogues its two iteration kernels fuse into
// the SpMVs (x+ / x_bar / Halpern for the primal half, y+ / Halpern for the dual half).
#pragma once

#include "common.cuh"

namespace vajra {

constexpr int kHist = 32;

struct HState {
    double omega, eta, tau, sigma;
    double inv_sigma;   // 1 / sigma, kept with sigma so the dual prox multiplies
    double gamma_now;   // reflection coefficient of the running phase (set by the control)
    double kkt_start, kkt_prev;
    double rel_p, rel_d, rel_gap, rel_kkt, pobj, dobj;
    double bnorm, cnorm, offset_min;
    double viol_p_rel, viol_p_abs, viol_d_abs;   // status-guard maxima of the last check
    double hist[kHist];
    long long k_base;
    long long total;
    long long phase_iters[2];
    long long stop_iter;
    int hist_n;
    int phase;          // 0: FP32 phase of the mixed mode, 1: FP64
    int stop;
    int status;
    int restart_count;
    int restart_flag;
    int switch_flag;
    int pad;
};

constexpr int kStatusOptimal = 1;
constexpr int kStatusIterLimit = 6;
constexpr int kStatusTimeLimit = 7;
constexpr int kStatusNumerical = 9;

// At the last iteration of a chunk (write_cand) the epilogues also keep T(z) (xc, yc) and
// the point it was taken from (xprev, yprev) for the check.
// Both epilogues are two-phase (see spmv.cuh): pre() issues every load that does not need
// the row sum -- the read-only vectors and the device scalars through the read-only path
// (they are written only by other kernels) -- before the SpMV's own loads.
template <typename T>
struct EpiHPrimal {
    const T* c; const T* cl; const T* cu; const T* x0;
    T* x; T* xb; T* xc; T* xprev;
    const HState* st;
    const double* hw;   // Halpern weights of this chunk: hw[2kk] = (k+1)/(k+2), hw[2kk+1] = 1/(k+2)
    int kk, phase, write_cand;
    struct Pre { T xo, c, cl, cu, x0, tau, w1, w0, g; };
    __device__ bool active() const { return st->stop == 0 && st->phase == phase; }
    __device__ Pre pre(int j) const {
        Pre p;
        p.w1 = static_cast<T>(__ldg(hw + 2 * kk));
        p.w0 = static_cast<T>(__ldg(hw + 2 * kk + 1));
        p.tau = static_cast<T>(__ldg(&st->tau));
        p.g = static_cast<T>(__ldg(&st->gamma_now));
        p.xo = x[j];
        p.c = __ldg(c + j);
        p.cl = __ldg(cl + j);
        p.cu = __ldg(cu + j);
        p.x0 = __ldg(x0 + j);
        return p;
    }
    template <typename Acc>
    __device__ void operator()(int j, Acc v, const Pre& p) const {
        const T g = p.g;
        T xp = p.xo - p.tau * (p.c + static_cast<T>(v));
        xp = xp < p.cl ? p.cl : (xp > p.cu ? p.cu : xp);
        xb[j] = xp + xp - p.xo;
        x[j] = p.w1 * ((T(1) + g) * xp - g * p.xo) + p.w0 * p.x0;
        if (write_cand) { xc[j] = xp; xprev[j] = p.xo; }
    }
    template <typename Acc>
    __device__ void operator()(int j, Acc v) const { (*this)(j, v, pre(j)); }
};

template <typename T>
struct EpiHDual {
    const T* rl; const T* ru; const T* y0;
    T* y; T* yc; T* yprev;
    const HState* st;
    const double* hw;   // Halpern weights of this chunk (as in EpiHPrimal)
    int kk, phase, write_cand;
    struct Pre { T yo, rl, ru, y0, sigma, inv_sigma, w1, w0, g; };
    __device__ bool active() const { return st->stop == 0 && st->phase == phase; }
    __device__ Pre pre(int i) const {
        Pre p;
        p.w1 = static_cast<T>(__ldg(hw + 2 * kk));
        p.w0 = static_cast<T>(__ldg(hw + 2 * kk + 1));
        p.sigma = static_cast<T>(__ldg(&st->sigma));
        p.inv_sigma = static_cast<T>(__ldg(&st->inv_sigma));
        p.g = static_cast<T>(__ldg(&st->gamma_now));
        p.yo = y[i];
        p.rl = __ldg(rl + i);
        p.ru = __ldg(ru + i);
        p.y0 = __ldg(y0 + i);
        return p;
    }
    template <typename Acc>
    __device__ void operator()(int i, Acc w, const Pre& p) const {
        const T g = p.g;
        const T yh = p.yo + p.sigma * static_cast<T>(w);
        T q = yh * p.inv_sigma;
        q = q < p.rl ? p.rl : (q > p.ru ? p.ru : q);
        const T yp = yh - p.sigma * q;
        y[i] = p.w1 * ((T(1) + g) * yp - g * p.yo) + p.w0 * p.y0;
        if (write_cand) { yc[i] = yp; yprev[i] = p.yo; }
    }
    template <typename Acc>
    __device__ void operator()(int i, Acc w) const { (*this)(i, w, pre(i)); }
};

// The Halpern weights of the next chunk from the current inner counter: one thread per step.
__device__ __forceinline__ void halpern_weights(const HState* st, int len, double* hw, int t, int stride) {
    const long long kb = st->k_base;
    for (int kk = t; kk < len; kk += stride) {
        const double k = static_cast<double>(kb + kk);
        hw[2 * kk] = (k + 1.0) / (k + 2.0);
        hw[2 * kk + 1] = 1.0 / (k + 2.0);
    }
}

__global__ void k_halpern_weights(const HState* st, int len, double* hw) {
    halpern_weights(st, len, hw, threadIdx.x, blockDim.x);
}

struct EpiStoreActive {
    double* out;
    const HState* st;
    int phase;
    __device__ bool active() const { return st->stop == 0 && st->phase == phase; }
    template <typename Acc> __device__ void operator()(int i, Acc s) const { out[i] = static_cast<double>(s); }
};

}  // namespace vajra
