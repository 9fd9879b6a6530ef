// Batched restarted Halpern PDHG: many independent LPs of uneven sizes packed
// block-diagonally into one device problem.  In mixed precision an FP32 pass (FP32 values,
// iterates and sums; FP64 checks) comes first, and each instance either finishes there or
// hands over to the FP64 pass, which restarts it from its FP32 candidate -- the single-LP
// solver's precision split, decided per instance.
//
// The packed matrix diag(A_1, ..., A_B) is one CSC / CSR, so each iteration is still two
// fused SpMV launches over all instances.  Every instance keeps its own step sizes, primal
// weight, Halpern counter, restart state and termination flag in device arrays (struct of
// arrays below); the epilogues look up a row's / column's instance.  Row blocks and rows that
// belong only to finished instances are skipped before any load, so the work shrinks as
// instances converge.  Every check interval one CTA per instance reduces that instance's KKT
// terms, one thread per instance runs the restart / primal-weight / termination logic
// (same rules as the single-LP solver), and one thread counts the active instances.  A pass
// is one CUDA graph whose WHILE node repeats the chunk (iterations plus check) on the device
// while an instance is active, up to a chunk budget per launch; the host reads the
// counters once per launch.  No kernel waits on another kernel, so nothing in this path can
// spin, and the loop's chunk budget ends every launch.
//
// Scaling is per instance: Ruiz and Pock-Chambolle factors are local to a row or column, and
// each instance ends its Ruiz passes on its own stopping test, so every instance is scaled
// exactly as it would be alone.  Difference from solving the instances one by one: the power
// iteration runs a fixed 60 rounds for every instance.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "solver.cuh"

namespace vajra {
namespace {

constexpr int kBQ = 10;   // per-instance check sums

struct BatchArrays {      // device struct of arrays, B entries each
    double* omega; double* eta; double* tau; double* sigma;
    double* kkt_start; double* kkt_prev;
    double* rel_p; double* rel_d; double* rel_gap; double* rel_kkt; double* pobj; double* dobj;
    double* bnorm; double* cnorm; double* offset_min; double* lambda;
    double* inv_sigma;    // 1 / sigma
    double* gamma;        // reflection of the instance's current phase
    double* hw;           // Halpern weights of the current chunk, 2 hw_len per instance:
    int hw_len;           // hw[i 2 hw_len + 2 kk] = (k+1)/(k+2), [.. + 1] = 1/(k+2), k = k_base + kk
    double* hist;         // FP32 pass: the last kBHist relative KKT values per instance (stall test)
    long long* k_base; long long* total;
    long long* total32;   // iterations the instance spent in the FP32 pass
    int* done; int* status; int* restart_count; int* restart_flag; int* hist_n;
};

constexpr int kBHist = 32;
// Status of an instance that left the FP32 pass for the FP64 one (internal, never reported).
constexpr int kBHandover = 100;

// Read by the host after every launch of the pass graph.  `left` bounds the chunks one launch
// may run (the host writes it before the launch, the loop counts it down); `chunks` counts the
// chunks the loop ran.
struct BatchCounters {
    int active;
    int left;
    long long chunks;
};

// Chunks one launch of a pass graph may run before the host looks at the counters again.
// The first launch of a pass runs kFirstLaunchChunks; later ones as many as the time left
// allows at the chunk rate the host has measured (all of the pass, up to kMaxLaunchChunks,
// without a time limit), so a pass without a time limit takes one or two launches.
constexpr int kFirstLaunchChunks = 32;
constexpr int kMaxLaunchChunks = 4096;

__device__ __forceinline__ void instance_weights(const BatchArrays& S, int i) {
    const long long kb = S.k_base[i];
    double* w = S.hw + static_cast<size_t>(i) * 2 * S.hw_len;
    for (int kk = 0; kk < S.hw_len; ++kk) {
        const double k = static_cast<double>(kb + kk);
        w[2 * kk] = (k + 1.0) / (k + 2.0);
        w[2 * kk + 1] = 1.0 / (k + 2.0);
    }
}

__device__ __forceinline__ bool any_active(const int* done, const int* inst, int r0, int r1) {
    const int a = inst[r0], b = inst[r1 - 1];
    for (int i = a; i <= b; ++i)
        if (!done[i]) return true;
    return false;
}

template <typename T>
struct EpiBPrimal {
    const T* c; const T* cl; const T* cu; const T* x0;
    T* x; T* xb; T* xc;
    const int* col_inst;
    BatchArrays S;
    int kk, write_cand;
    // two-phase (spmv.cuh): the instance lookups and vector loads go out before the SpMV's
    struct Pre { T w1, w0, tau, g, xo, c, cl, cu, x0; int done; };
    __device__ bool active() const { return true; }
    __device__ bool skip_rows(int r0, int r1) const { return !any_active(S.done, col_inst, r0, r1); }
    __device__ Pre pre(int j) const {
        const int i = __ldg(col_inst + j);
        Pre p;
        p.done = S.done[i];
        const double* w = S.hw + static_cast<size_t>(i) * 2 * S.hw_len + 2 * kk;
        p.w1 = static_cast<T>(w[0]);
        p.w0 = static_cast<T>(w[1]);
        p.tau = static_cast<T>(S.tau[i]);
        p.g = static_cast<T>(S.gamma[i]);
        p.xo = x[j];
        p.c = __ldg(c + j);
        p.cl = __ldg(cl + j);
        p.cu = __ldg(cu + j);
        p.x0 = __ldg(x0 + j);
        return p;
    }
    template <typename Acc>
    __device__ void operator()(int j, Acc v, const Pre& p) const {
        if (p.done) return;
        T xp = p.xo - p.tau * (p.c + static_cast<T>(v));
        xp = xp < p.cl ? p.cl : (xp > p.cu ? p.cu : xp);
        xb[j] = xp + xp - p.xo;
        x[j] = p.w1 * ((T(1) + p.g) * xp - p.g * p.xo) + p.w0 * p.x0;
        if (write_cand) xc[j] = xp;
    }
    template <typename Acc>
    __device__ void operator()(int j, Acc v) const { (*this)(j, v, pre(j)); }
};

template <typename T>
struct EpiBDual {
    const T* rl; const T* ru; const T* y0;
    T* y; T* yc;
    const int* row_inst;
    BatchArrays S;
    int kk, write_cand;
    struct Pre { T w1, w0, sigma, inv_sigma, g, yo, rl, ru, y0; int done; };
    __device__ bool active() const { return true; }
    __device__ bool skip_rows(int r0, int r1) const { return !any_active(S.done, row_inst, r0, r1); }
    __device__ Pre pre(int r) const {
        const int i = __ldg(row_inst + r);
        Pre p;
        p.done = S.done[i];
        const double* w = S.hw + static_cast<size_t>(i) * 2 * S.hw_len + 2 * kk;
        p.w1 = static_cast<T>(w[0]);
        p.w0 = static_cast<T>(w[1]);
        p.sigma = static_cast<T>(S.sigma[i]);
        p.inv_sigma = static_cast<T>(S.inv_sigma[i]);
        p.g = static_cast<T>(S.gamma[i]);
        p.yo = y[r];
        p.rl = __ldg(rl + r);
        p.ru = __ldg(ru + r);
        p.y0 = __ldg(y0 + r);
        return p;
    }
    template <typename Acc>
    __device__ void operator()(int r, Acc w, const Pre& p) const {
        if (p.done) return;
        const T sg = p.sigma;
        const T yh = p.yo + sg * static_cast<T>(w);
        T q = yh * p.inv_sigma;
        q = q < p.rl ? p.rl : (q > p.ru ? p.ru : q);
        const T yp = yh - sg * q;
        y[r] = p.w1 * ((T(1) + p.g) * yp - p.g * p.yo) + p.w0 * p.y0;
        if (write_cand) yc[r] = yp;
    }
    template <typename Acc>
    __device__ void operator()(int r, Acc w) const { (*this)(r, w, pre(r)); }
};

struct EpiBStore {
    double* out;
    const int* inst;
    const int* done;
    __device__ bool active() const { return true; }
    __device__ bool skip_rows(int r0, int r1) const { return !any_active(done, inst, r0, r1); }
    __device__ void operator()(int r, double s) const {
        if (!done[inst[r]]) out[r] = s;
    }
};

struct EpiStorePlain {
    double* out;
    __device__ bool active() const { return true; }
    __device__ void operator()(int r, double s) const { out[r] = s; }
};

// Blocks of one launch shape that hold at least one row of an unfinished instance (order
// irrelevant: every row's result is independent of which CTA computes it).
__global__ void k_active_blocks(int nblocks, int rows, int rows_per_block, const int32_t* __restrict__ block_rows,
                                const int* __restrict__ inst, const int* __restrict__ done,
                                int32_t* __restrict__ list, int* __restrict__ count) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    int r0, r1;
    if (block_rows) {
        r0 = block_rows[b];
        r1 = block_rows[b + 1];
    } else {
        r0 = b * rows_per_block;
        r1 = r0 + rows_per_block < rows ? r0 + rows_per_block : rows;
    }
    if (r0 < r1 && any_active(done, inst, r0, r1)) list[atomicAdd(count, 1)] = b;
}

// The active-block list of one iteration view (list mode of spmv.cuh).
struct BlockList {
    DeviceBuffer<int32_t> list;
    DeviceBuffer<int> count;
    int nblocks = 0, rows = 0, rows_per_block = 0;
    const int32_t* block_rows = nullptr;
    const int* inst = nullptr;
    // Builds the shape description for `v` (as tuned) and switches `v` to list mode.
    vajra_status attach(CsrView& v, const int* inst_, int sms) {
        inst = inst_;
        rows = v.rows;
        int cap;
        if (is_rowblock_shape(v.group) && v.block_rows) {
            nblocks = v.nb;
            block_rows = v.block_rows;
            cap = sms * 4;
        } else {
            int g = v.group;
            if (g != 1 && g != 2 && g != 4 && g != 8 && g != 16) g = g == 0 ? 8 : 32;   // launch_spmv_t's dispatch
            rows_per_block = kThreads / g;
            nblocks = vec_block_count(v.rows, g);
            cap = sms * 8;
        }
        VJ_TRY(list.alloc(static_cast<size_t>(nblocks > 0 ? nblocks : 1)));
        VJ_TRY(count.alloc(1));
        v.blk_list = list.get();
        v.blk_count = count.get();
        v.blk_grid = nblocks < cap ? (nblocks > 0 ? nblocks : 1) : cap;
        return VAJRA_OK;
    }
    void rebuild(const int* done, cudaStream_t st) {
        cudaMemsetAsync(count.get(), 0, sizeof(int), st);
        if (nblocks > 0)
            k_active_blocks<<<grid_for(nblocks), kThreads, 0, st>>>(nblocks, rows, rows_per_block, block_rows, inst, done,
                                                                   list.get(), count.get());
        note_launch(1);
    }
};

__device__ __forceinline__ bool lo_fin(double l) { return l > -1e20; }
__device__ __forceinline__ bool up_fin(double u) { return u < 1e20; }

// One CTA per instance: the same KKT terms as the single-LP row / column passes.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_bkkt(const int64_t* __restrict__ roff, const int64_t* __restrict__ coff, const double* __restrict__ ax,
       const double* __restrict__ aty, const T* __restrict__ xc, const T* __restrict__ yc,
       const double* __restrict__ rl_s, const double* __restrict__ ru_s, const double* __restrict__ rl_o,
       const double* __restrict__ ru_o, const double* __restrict__ rs, const double* __restrict__ c_s,
       const double* __restrict__ cl_o, const double* __restrict__ cu_o, const double* __restrict__ cs,
       const double* __restrict__ x_last, const double* __restrict__ y_last, double* __restrict__ part,
       BatchArrays S) {
    const int inst = blockIdx.x;
    if (S.done[inst]) return;
    __shared__ double red[kBQ * 32];
    double v[kBQ] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    // 0 rp_o^2, 1 rp_s^2, 2 dobj rows, 3 dy^2, 4 rd_o^2, 5 rd_s^2, 6 pobj, 7 dobj cols, 8 dx^2, 9 nan
    for (int64_t i = roff[inst] + threadIdx.x; i < roff[inst + 1]; i += blockDim.x) {
        const double a = ax[i], ys = static_cast<double>(yc[i]);
        if (!isfinite(a) || !isfinite(ys)) v[9] = 1.0;
        const double ps = a - fmin(fmax(a, rl_s[i]), ru_s[i]);
        const double ao = a / rs[i];
        const double po = ao - fmin(fmax(ao, rl_o[i]), ru_o[i]);
        const double yo = -ys * rs[i];
        double dt = 0.0;
        if (yo > 0.0 && lo_fin(rl_o[i])) dt = yo * rl_o[i];
        else if (yo < 0.0 && up_fin(ru_o[i])) dt = yo * ru_o[i];
        const double dy = ys - y_last[i];
        v[0] += po * po; v[1] += ps * ps; v[2] += dt; v[3] += dy * dy;
    }
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) {
        const double at = aty[j], xs = static_cast<double>(xc[j]);
        if (!isfinite(at) || !isfinite(xs)) v[9] = 1.0;
        const bool lf = lo_fin(cl_o[j]), uf = up_fin(cu_o[j]);
        const double r_s = c_s[j] + at, r_o = r_s / cs[j];
        auto lam_of = [&](double r) { return (lf && uf) ? r : lf ? fmax(r, 0.0) : uf ? fmin(r, 0.0) : 0.0; };
        const double lo = lam_of(r_o), ls = lam_of(r_s);
        double dt = 0.0;
        if (lo > 0.0) dt = lo * cl_o[j];
        else if (lo < 0.0) dt = lo * cu_o[j];
        const double dx = xs - x_last[j];
        v[4] += (r_o - lo) * (r_o - lo); v[5] += (r_s - ls) * (r_s - ls);
        v[6] += c_s[j] * xs; v[7] += dt; v[8] += dx * dx;
    }
    double f[1] = {v[9]};
    block_reduce<OpSum, double, kBQ - 1>(*reinterpret_cast<double(*)[kBQ - 1]>(v), red);
    block_reduce<OpMax, double, 1>(f, red);
    if (threadIdx.x == 0) {
        for (int q = 0; q < kBQ - 1; ++q) part[inst * kBQ + q] = v[q];
        part[inst * kBQ + kBQ - 1] = f[0];
    }
}

struct BControl {
    double tol, beta_sufficient, beta_necessary, beta_artificial, pw_smoothing;
    int len, count;
    // FP32 pass of a mixed batch (same rules as the single-LP FP32 phase, per instance):
    int pass32;            // 1 while the FP32 pass runs
    double switch_tol;     // hand over to FP64 at or below this relative KKT ...
    int stall_checks;      // ... or after this many checks with < 2 % gain (0 = never)
    double early_tol;      // below this the FP32 pass reflects with gamma32
    double gamma32;
};

// One thread per instance: the single-LP control rules (halpern_mode.cu) per instance.
__global__ void k_bcontrol(const double* __restrict__ part, BControl cp, BatchArrays S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cp.count || S.done[i]) return;
    const double* s = part + i * kBQ;
    S.total[i] += cp.len;
    S.restart_flag[i] = 0;
    if (s[9] > 0.0 || isnan(s[0]) || isnan(s[4])) {
        S.done[i] = 1;
        S.status[i] = 9;
        return;
    }
    const double pobj = s[6] + S.offset_min[i];
    const double dobj = s[2] + s[7] + S.offset_min[i];
    const double rel_p = sqrt(s[0]) / (1.0 + S.bnorm[i]);
    const double rel_d = sqrt(s[4]) / (1.0 + S.cnorm[i]);
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double rel = fmax(rel_p, fmax(rel_d, gap));
    S.rel_p[i] = rel_p; S.rel_d[i] = rel_d; S.rel_gap[i] = gap; S.rel_kkt[i] = rel;
    S.pobj[i] = pobj; S.dobj[i] = dobj;
    if (rel <= cp.tol) {
        S.done[i] = 1;
        S.status[i] = 1;
        return;
    }
    if (cp.pass32) {
        const int hn = S.hist_n[i];
        double* hist = S.hist + static_cast<size_t>(i) * kBHist;
        const int w = cp.stall_checks;
        const bool stalled = w > 0 && hn >= w && rel > 0.98 * hist[(hn - w) % kBHist];
        hist[hn % kBHist] = rel;
        S.hist_n[i] = hn + 1;
        if (rel <= cp.early_tol) S.gamma[i] = cp.gamma32;
        if (rel <= cp.switch_tol || stalled) {   // leaves the FP32 pass; the FP64 pass takes it over
            S.done[i] = 1;
            S.status[i] = kBHandover;
            return;
        }
    }
    const double omega = S.omega[i];
    const double wk = sqrt(omega * s[1] + s[5] / omega + gap * gap);
    if (S.kkt_start[i] < 0.0) { S.kkt_start[i] = wk; S.kkt_prev[i] = wk; }
    const long long k_in = S.k_base[i] + cp.len;
    const bool restart = (wk <= cp.beta_sufficient * S.kkt_start[i]) ||
                         (wk <= cp.beta_necessary * S.kkt_start[i] && wk > S.kkt_prev[i]) ||
                         (static_cast<double>(k_in) >= cp.beta_artificial * static_cast<double>(S.total[i]));
    S.kkt_prev[i] = wk;
    if (restart) {
        const double dx = sqrt(s[8]), dy = sqrt(s[3]);
        if (dx > 1e-10 && dy > 1e-10) {
            const double th = cp.pw_smoothing;
            S.omega[i] = exp(th * log(dy / dx) + (1.0 - th) * log(omega));
            S.tau[i] = S.eta[i] / S.omega[i];
            S.sigma[i] = S.eta[i] * S.omega[i];
            S.inv_sigma[i] = 1.0 / S.sigma[i];
        }
        S.k_base[i] = 0;
        S.kkt_start[i] = wk;
        S.kkt_prev[i] = wk;
        S.restart_count[i] += 1;
        S.restart_flag[i] = 1;
    } else {
        S.k_base[i] = k_in;
    }
    instance_weights(S, i);
}

// Counts the unfinished instances.  Inside the WHILE body of a pass graph (`loop` = 1) it also
// decides whether the body runs again: only while an instance is active and the launch's chunk
// budget is not spent, so every launch ends after at most `left` chunks whatever the iterates do.
__global__ void __launch_bounds__(1024) k_bcount(int count, const int* __restrict__ done, BatchCounters* out,
                                                 cudaGraphConditionalHandle again, int loop) {
    __shared__ double red[32];
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < count; i += blockDim.x) v[0] += done[i] ? 0.0 : 1.0;
    block_reduce<OpSum, double, 1>(v, red);
    if (threadIdx.x == 0) {
        const int active = static_cast<int>(v[0]);
        out->active = active;
        if (loop) {
            const int left = out->left - 1;
            out->left = left;
            out->chunks += 1;
            cudaGraphSetConditional(again, active > 0 && left > 0 ? 1u : 0u);
        }
    }
}

template <typename T>
__global__ void k_brestart(int m, int n, const int* __restrict__ row_inst, const int* __restrict__ col_inst,
                           const T* __restrict__ xc, const T* __restrict__ yc, T* __restrict__ x,
                           T* __restrict__ x0, T* __restrict__ y, T* __restrict__ y0,
                           double* __restrict__ x_last, double* __restrict__ y_last, BatchArrays S) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && S.restart_flag[col_inst[t]]) { const T v = xc[t]; x[t] = v; x0[t] = v; x_last[t] = v; }
    if (t < m && S.restart_flag[row_inst[t]]) { const T v = yc[t]; y[t] = v; y0[t] = v; y_last[t] = v; }
}

// End of the FP32 pass, vectors: every instance's FP32 candidate becomes its FP64 candidate
// (the point post-processing reports for instances that finished in FP32 or hit a limit), and
// an instance that was handed over also starts its FP64 pass there (iterate, anchor and last
// restart point), as the single-LP hand-over does.
__global__ void k_bhandover(int m, int n, const int* __restrict__ row_inst, const int* __restrict__ col_inst,
                            const float* __restrict__ xc32, const float* __restrict__ yc32, double* __restrict__ x,
                            double* __restrict__ x0, double* __restrict__ xc, double* __restrict__ x_last,
                            double* __restrict__ y, double* __restrict__ y0, double* __restrict__ yc,
                            double* __restrict__ y_last, const int* __restrict__ status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const double v = xc32[t];
        xc[t] = v;
        if (status[col_inst[t]] == kBHandover) { x[t] = v; x0[t] = v; x_last[t] = v; }
    }
    if (t < m) {
        const double v = yc32[t];
        yc[t] = v;
        if (status[row_inst[t]] == kBHandover) { y[t] = v; y0[t] = v; y_last[t] = v; }
    }
}

// End of the FP32 pass, per-instance state: its iterations are counted as FP32 ones, and a
// handed-over instance starts a fresh Halpern epoch with the FP64 reflection (primal weight
// and step sizes carry over).
__global__ void k_bhandover_state(int count, double gamma64, BatchArrays S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    S.total32[i] = S.total[i];
    if (S.status[i] != kBHandover) return;
    S.done[i] = 0;
    S.status[i] = 0;
    S.k_base[i] = 0;
    S.kkt_start[i] = -1.0;
    S.kkt_prev[i] = -1.0;
    S.gamma[i] = gamma64;
    S.restart_flag[i] = 0;
    instance_weights(S, i);
}

// Packing: an instance's column pointers (copied as they are, starting at 0) shifted by its
// first entry; then its row indices shifted by its first row (the pointers are final by then).
__global__ void k_bshift_cols(int n, const int* __restrict__ col_inst, const int64_t* __restrict__ zoff,
                              int64_t* __restrict__ col_ptr) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) col_ptr[j] += zoff[col_inst[j]];
}
__global__ void k_bshift_rows(int n, const int* __restrict__ col_inst, const int64_t* __restrict__ roff,
                              const int64_t* __restrict__ col_ptr, int32_t* __restrict__ row_idx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int32_t r0 = static_cast<int32_t>(roff[col_inst[j]]);
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) row_idx[k] += r0;
}
__global__ void k_bmin_c(int n, const int* __restrict__ col_inst, const int* __restrict__ sense,
                         const double* __restrict__ c, double* __restrict__ cmin) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) cmin[j] = sense[col_inst[j]] ? -c[j] : c[j];
}

template <typename To>
__global__ void k_bconvert(int64_t n, const double* __restrict__ src, To* __restrict__ dst) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[k] = static_cast<To>(src[k]);
}

// Per-instance norms (||b||, ||c|| original; ||b||, ||c|| scaled) and initial state.
__global__ void __launch_bounds__(kThreads)
k_binit(const int64_t* __restrict__ roff, const int64_t* __restrict__ coff, const double* __restrict__ rl_o,
        const double* __restrict__ ru_o, const double* __restrict__ c_o, const double* __restrict__ rl_s,
        const double* __restrict__ ru_s, const double* __restrict__ c_s, const int* __restrict__ sense,
        const double* __restrict__ offsets, double step_safety, double gamma0, BatchArrays S) {
    const int inst = blockIdx.x;
    __shared__ double red[4 * 32];
    double v[4] = {0, 0, 0, 0};
    auto b2 = [](double l, double u) {
        const bool lf = l > -1e20, uf = u < 1e20;
        if (lf && uf && l == u) return l * l;
        return (lf ? l * l : 0.0) + (uf ? u * u : 0.0);
    };
    for (int64_t i = roff[inst] + threadIdx.x; i < roff[inst + 1]; i += blockDim.x) {
        v[0] += b2(rl_o[i], ru_o[i]);
        v[2] += b2(rl_s[i], ru_s[i]);
    }
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) {
        v[1] += c_o[j] * c_o[j];
        v[3] += c_s[j] * c_s[j];
    }
    block_reduce<OpSum, double, 4>(v, red);
    if (threadIdx.x != 0) return;
    const double bn = sqrt(v[0]), cn = sqrt(v[1]), bs = sqrt(v[2]), csn = sqrt(v[3]);
    const double norm = S.lambda[inst] > 1e-12 ? S.lambda[inst] : 1.0;
    const double eta = step_safety / norm;
    const double omega = (bs > 1e-10 && csn > 1e-10) ? csn / bs : 1.0;
    S.bnorm[inst] = bn; S.cnorm[inst] = cn;
    S.eta[inst] = eta; S.omega[inst] = omega; S.tau[inst] = eta / omega; S.sigma[inst] = eta * omega;
    S.inv_sigma[inst] = 1.0 / (eta * omega);
    S.kkt_start[inst] = -1.0; S.kkt_prev[inst] = -1.0;
    S.offset_min[inst] = sense[inst] ? -offsets[inst] : offsets[inst];
    S.k_base[inst] = 0; S.total[inst] = 0;
    S.done[inst] = 0; S.status[inst] = 0; S.restart_count[inst] = 0; S.restart_flag[inst] = 0;
    S.hist_n[inst] = 0; S.total32[inst] = 0;
    S.gamma[inst] = gamma0;
    S.rel_kkt[inst] = 1e30;
    instance_weights(S, inst);
}

__global__ void k_binit_iterates(int m, int n, const double* __restrict__ cl, const double* __restrict__ cu,
                                 double* x, double* x0, double* xb, double* xc, double* x_last,
                                 double* y, double* y0, double* yc, double* y_last) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const double v = fmin(fmax(0.0, cl[t]), cu[t]);
        x[t] = x0[t] = xb[t] = xc[t] = x_last[t] = v;
    }
    if (t < m) { y[t] = y0[t] = yc[t] = y_last[t] = 0.0; }
}

// Batched power iteration, one CTA per instance: ||u_i||, then v_i = u_i / ||u_i||.
__global__ void __launch_bounds__(kThreads)
k_bpower(const int64_t* __restrict__ coff, const double* __restrict__ u, double* __restrict__ v, BatchArrays S) {
    const int inst = blockIdx.x;
    __shared__ double red[32];
    __shared__ double inv;
    double s[1] = {0.0};
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) s[0] += u[j] * u[j];
    block_reduce<OpSum, double, 1>(s, red);
    if (threadIdx.x == 0) {
        const double nrm = sqrt(s[0]);
        S.lambda[inst] = sqrt(nrm);                 // sigma_max estimate = sqrt(||A^T A v||)
        inv = nrm > 1e-300 ? 1.0 / nrm : 0.0;
    }
    __syncthreads();
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) v[j] = u[j] * inv;
}

__global__ void k_bpower_init(int n, const int* __restrict__ col_inst, const int64_t* __restrict__ coff,
                              double* __restrict__ v) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = col_inst[j];
    v[j] = 1.0 / sqrt(static_cast<double>(coff[i + 1] - coff[i]));
}

__global__ void k_bpost(int m, int n, const int* __restrict__ col_inst, const int* __restrict__ sense,
                        const double* __restrict__ xc, const double* __restrict__ yc, const double* __restrict__ cs,
                        const double* __restrict__ rs, int scaled, double* __restrict__ x_out,
                        double* __restrict__ y_out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x_out[t] = scaled ? xc[t] * cs[t] : xc[t];
    if (t < m) y_out[t] = -(scaled ? yc[t] * rs[t] : yc[t]);
    (void)col_inst; (void)sense;
}

__global__ void k_breduced(int n, const int* __restrict__ col_inst, const int* __restrict__ sense,
                           const double* __restrict__ c, double* __restrict__ d) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) d[j] = sense[col_inst[j]] ? c[j] + d[j] : c[j] - d[j];
}

__global__ void __launch_bounds__(kThreads)
k_bobjective(const int64_t* __restrict__ coff, const double* __restrict__ c, const double* __restrict__ x,
             const double* __restrict__ offsets, double* __restrict__ out) {
    const int inst = blockIdx.x;
    __shared__ double red[32];
    double s[1] = {0.0};
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) s[0] += c[j] * x[j];
    block_reduce<OpSum, double, 1>(s, red);
    if (threadIdx.x == 0) out[inst] = offsets[inst] + s[0];
}

__global__ void k_fill_inst(int64_t total, const int64_t* __restrict__ off, int count, int* __restrict__ inst) {
    const int i = blockIdx.x;   // one CTA per instance
    if (i >= count) return;
    for (int64_t t = off[i] + threadIdx.x; t < off[i + 1]; t += blockDim.x) inst[t] = i;
    (void)total;
}

template <typename T>
vajra_status up(DeviceBuffer<T>& d, const std::vector<T>& h, cudaStream_t st) {
    VJ_TRY(d.alloc(h.size()));
    if (!h.empty()) VJ_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return VAJRA_OK;
}

}  // namespace

vajra_status run_batch(int count, const vajra_lp* lps, const vajra_opts& o, vajra_result* results,
                       cudaStream_t st, double* device_time) {
    const auto t_start = Clock::now();
    // ---- packing (block-diagonal CSC), straight into the device buffers ----------------------
    // Each instance's arrays are copied to their slots of the packed arrays as they are; two
    // kernels then shift its column pointers by its first entry and its row indices by its
    // first row.  No host copy of the entries is made.
    std::vector<int64_t> roff(count + 1, 0), coff(count + 1, 0), zoff(count + 1, 0);
    for (int i = 0; i < count; ++i) {
        roff[i + 1] = roff[i] + lps[i].num_rows;
        coff[i + 1] = coff[i] + lps[i].num_cols;
        zoff[i + 1] = zoff[i] + lps[i].nnz;
    }
    const int64_t M = roff[count], N = coff[count], NNZ = zoff[count];
    if (M >= (1LL << 31) || N >= (1LL << 31)) { set_error("packed batch exceeds 2^31 rows or columns"); return VAJRA_ERR_INVALID_ARGUMENT; }
    const int m = static_cast<int>(M), n = static_cast<int>(N);
    std::vector<double> offsets(count);
    std::vector<int> sense(count);
    for (int i = 0; i < count; ++i) {
        sense[i] = lps[i].sense;
        offsets[i] = lps[i].objective_offset;
    }
    auto mark = [&](const char* what) {
        if (!o.verbose) return;
        cudaStreamSynchronize(st);
        std::fprintf(stderr, "[vajra] batch %-22s %8.1f ms\n", what, 1e3 * seconds_since(t_start));
    };

    StreamTimer timer;
    timer.start(st);
    DeviceLp lp;
    lp.m = m;
    lp.n = n;
    lp.nnz = NNZ;
    VJ_TRY(lp.col_ptr.alloc(static_cast<size_t>(n) + 1));
    VJ_TRY(lp.row_idx.alloc(static_cast<size_t>(NNZ)));
    VJ_TRY(lp.values.alloc(static_cast<size_t>(NNZ)));
    for (auto* b : {&lp.c, &lp.col_lower, &lp.col_upper}) VJ_TRY(b->alloc(n));
    for (auto* b : {&lp.row_lower, &lp.row_upper}) VJ_TRY(b->alloc(m));
    auto put = [&](auto* dst, const auto* src, int64_t k) -> vajra_status {
        if (k > 0) VJ_CUDA(cudaMemcpyAsync(dst, src, sizeof(*src) * k, cudaMemcpyHostToDevice, st));
        return VAJRA_OK;
    };
    for (int i = 0; i < count; ++i) {
        const vajra_lp& L = lps[i];
        const int64_t c0 = coff[i], r0 = roff[i], z0 = zoff[i];
        VJ_TRY(put(lp.col_ptr.get() + c0, L.col_ptr, L.num_cols));
        VJ_TRY(put(lp.row_idx.get() + z0, L.row_idx, L.nnz));
        VJ_TRY(put(lp.values.get() + z0, L.values, L.nnz));
        VJ_TRY(put(lp.c.get() + c0, L.c, L.num_cols));
        VJ_TRY(put(lp.col_lower.get() + c0, L.col_lower, L.num_cols));
        VJ_TRY(put(lp.col_upper.get() + c0, L.col_upper, L.num_cols));
        VJ_TRY(put(lp.row_lower.get() + r0, L.row_lower, L.num_rows));
        VJ_TRY(put(lp.row_upper.get() + r0, L.row_upper, L.num_rows));
    }
    VJ_TRY(put(lp.col_ptr.get() + n, &NNZ, 1));
    DeviceBuffer<int64_t> d_roff, d_coff, d_zoff;
    DeviceBuffer<int> d_sense, row_inst, col_inst;
    DeviceBuffer<double> d_offsets, d_cmin;
    VJ_TRY(up(d_roff, roff, st));
    VJ_TRY(up(d_coff, coff, st));
    VJ_TRY(up(d_zoff, zoff, st));
    VJ_TRY(up(d_sense, sense, st));
    VJ_TRY(up(d_offsets, offsets, st));
    VJ_TRY(row_inst.alloc(m));
    VJ_TRY(col_inst.alloc(n));
    VJ_TRY(d_cmin.alloc(n));
    k_fill_inst<<<count, kThreads, 0, st>>>(M, d_roff.get(), count, row_inst.get());
    k_fill_inst<<<count, kThreads, 0, st>>>(N, d_coff.get(), count, col_inst.get());
    k_bshift_cols<<<grid_for(n), kThreads, 0, st>>>(n, col_inst.get(), d_zoff.get(), lp.col_ptr.get());
    k_bshift_rows<<<grid_for(n), kThreads, 0, st>>>(n, col_inst.get(), d_roff.get(), lp.col_ptr.get(),
                                                    lp.row_idx.get());
    // the packed problem is a minimisation: maximisation instances' objectives are negated
    k_bmin_c<<<grid_for(n), kThreads, 0, st>>>(n, col_inst.get(), d_sense.get(), lp.c.get(), d_cmin.get());
    VJ_LAUNCH_CHECK();
    note_launch(5);
    mark("packed on the device");

    // ---- set-up on the packed problem --------------------------------------------------
    Prepared p;
    DeviceBuffer<SetupState> sst;
    VJ_TRY(sst.alloc(1));
    VJ_TRY(build_csr(lp, p, st));
    ScalingOpts so;
    so.enable = o.enable_scaling != 0;
    so.ruiz_iterations = o.ruiz_iterations > 0 ? o.ruiz_iterations : 10;
    so.pock_chambolle = o.pock_chambolle != 0;
    so.negate_c = false;
    // each instance stops its Ruiz passes on its own test, as it would alone
    so.instances = count;
    so.roff = d_roff.get();
    so.coff = d_coff.get();
    so.row_inst = row_inst.get();
    so.col_inst = col_inst.get();
    {
        // Upload the min-form c as the raw c for scaling, keep the caller's c for reporting.
        DeviceBuffer<double> c_raw;
        std::swap(c_raw, lp.c);
        std::swap(lp.c, d_cmin);
        VJ_TRY(prepare_scaled(lp, p, so, sst.get(), st));
        std::swap(d_cmin, lp.c);
        std::swap(lp.c, c_raw);   // lp.c = caller's c again, d_cmin = min-form c
    }
    VJ_TRY(plan_spmv(lp, p, st));

    // ---- per-instance state -------------------------------------------------------------
    DeviceBuffer<double> dd;
    DeviceBuffer<long long> dl;
    DeviceBuffer<int> di;
    VJ_TRY(dd.alloc(18 * static_cast<size_t>(count)));
    const int K = o.check_frequency > 0 ? o.check_frequency : 64;
    DeviceBuffer<double> d_hw, d_hist;
    VJ_TRY(d_hw.alloc(2 * static_cast<size_t>(K) * count));
    VJ_TRY(d_hist.alloc(static_cast<size_t>(kBHist) * count));
    VJ_TRY(dl.alloc(3 * static_cast<size_t>(count)));
    VJ_TRY(di.alloc(5 * static_cast<size_t>(count)));
    BatchArrays S;
    double** fields[] = {&S.omega, &S.eta, &S.tau, &S.sigma, &S.kkt_start, &S.kkt_prev, &S.rel_p, &S.rel_d,
                         &S.rel_gap, &S.rel_kkt, &S.pobj, &S.dobj, &S.bnorm, &S.cnorm, &S.offset_min, &S.lambda,
                         &S.inv_sigma, &S.gamma};
    for (int q = 0; q < 18; ++q) *fields[q] = dd.get() + static_cast<size_t>(q) * count;
    S.hw = d_hw.get();
    S.hw_len = K;
    S.hist = d_hist.get();
    S.k_base = dl.get(); S.total = dl.get() + count; S.total32 = dl.get() + 2 * count;
    S.done = di.get(); S.status = di.get() + count; S.restart_count = di.get() + 2 * count;
    S.restart_flag = di.get() + 3 * count;
    S.hist_n = di.get() + 4 * count;
    VJ_CUDA(cudaMemsetAsync(di.get(), 0, sizeof(int) * 5 * count, st));   // done = 0 for the power iteration

    // batched power iteration (fixed 60 rounds)
    {
        DeviceBuffer<double> v, w, u;
        VJ_TRY(v.alloc(n));
        VJ_TRY(w.alloc(m));
        VJ_TRY(u.alloc(n));
        k_bpower_init<<<grid_for(n), kThreads, 0, st>>>(n, col_inst.get(), d_coff.get(), v.get());
        note_launch(1);
        for (int it = 0; it < 60; ++it) {
            launch_spmv_t<double, double, double>(p.a, p.csr_val.get(), v.get(), EpiStorePlain{w.get()}, st);
            launch_spmv_t<double, double, double>(p.at, p.csc_val.get(), w.get(), EpiStorePlain{u.get()}, st);
            k_bpower<<<count, kThreads, 0, st>>>(d_coff.get(), u.get(), v.get(), S);
            note_launch(1);
        }
        VJ_LAUNCH_CHECK();
        VJ_CUDA(cudaStreamSynchronize(st));
    }
    const double safety = (o.step_safety > 0.0 && o.step_safety < 1.0) ? o.step_safety : 0.99;
    k_binit<<<count, kThreads, 0, st>>>(d_roff.get(), d_coff.get(), lp.row_lower.get(), lp.row_upper.get(), d_cmin.get(),
                                        p.row_lower.get(), p.row_upper.get(), p.c.get(), d_sense.get(), d_offsets.get(),
                                        safety, o.reflection, S);
    note_launch(1);

    // iterates
    DeviceBuffer<double> x, x0, xb, xc, y, y0, yc, x_last, y_last, ax, aty, part;
    for (auto* b : {&x, &x0, &xb, &xc, &x_last, &aty}) VJ_TRY(b->alloc(n));
    for (auto* b : {&y, &y0, &yc, &y_last, &ax}) VJ_TRY(b->alloc(m));
    VJ_TRY(part.alloc(static_cast<size_t>(count) * kBQ));
    const int mx = m > n ? m : n;
    k_binit_iterates<<<grid_for(mx), kThreads, 0, st>>>(m, n, p.col_lower.get(), p.col_upper.get(), x.get(), x0.get(),
                                                        xb.get(), xc.get(), x_last.get(), y.get(), y0.get(), yc.get(),
                                                        y_last.get());
    note_launch(1);
    VJ_LAUNCH_CHECK();
    // Mixed precision: an FP32 pass (FP32 values, iterates and sums, FP64 checks) runs first;
    // each instance finishes there or hands over to the FP64 pass.
    const bool mixed = o.precision == VAJRA_PREC_MIXED;
    DeviceBuffer<float> x32, x0_32, xb32, xc32, y32, y0_32, yc32, c32, cl32, cu32, rl32, ru32;
    if (mixed) {
        VJ_TRY(make_f32_values(p, NNZ, st));
        for (auto* b : {&x32, &x0_32, &xb32, &xc32, &c32, &cl32, &cu32}) VJ_TRY(b->alloc(n));
        for (auto* b : {&y32, &y0_32, &yc32, &rl32, &ru32}) VJ_TRY(b->alloc(m));
        const unsigned gn = grid_for(n, kThreads, 148 * 32), gm = grid_for(m, kThreads, 148 * 32);
        k_bconvert<float><<<gn, kThreads, 0, st>>>(n, p.c.get(), c32.get());
        k_bconvert<float><<<gn, kThreads, 0, st>>>(n, p.col_lower.get(), cl32.get());
        k_bconvert<float><<<gn, kThreads, 0, st>>>(n, p.col_upper.get(), cu32.get());
        k_bconvert<float><<<gm, kThreads, 0, st>>>(m, p.row_lower.get(), rl32.get());
        k_bconvert<float><<<gm, kThreads, 0, st>>>(m, p.row_upper.get(), ru32.get());
        for (auto* b : {&x32, &x0_32, &xb32, &xc32})
            k_bconvert<float><<<gn, kThreads, 0, st>>>(n, x.get(), b->get());
        for (auto* b : {&y32, &y0_32, &yc32})
            k_bconvert<float><<<gm, kThreads, 0, st>>>(m, y.get(), b->get());
        note_launch(12);
        VJ_LAUNCH_CHECK();
    }

    // autotune the packed SpMVs (store epilogue, no skipping)
    CsrView a = p.a, at = p.at;
    if (o.autotune) {
        cudaEvent_t e0, e1;
        VJ_CUDA(cudaEventCreate(&e0));
        VJ_CUDA(cudaEventCreate(&e1));
        for (CsrView* v : {&a, &at}) {
            const double* xin = (v == &a) ? xb.get() : y.get();
            double* out = (v == &a) ? ax.get() : aty.get();
            const double* val = (v == &a) ? p.csr_val.get() : p.csc_val.get();
            float best = 1e30f;
            int best_g = v->group;
            for (int g : {0, kRowblock2, 1, 2, 4, 8, 16, 32}) {
                CsrView t = *v;
                t.group = g;
                launch_spmv_t<double, double, double>(t, val, xin, EpiStorePlain{out}, st);
                VJ_CUDA(cudaEventRecord(e0, st));
                for (int r = 0; r < 3; ++r) launch_spmv_t<double, double, double>(t, val, xin, EpiStorePlain{out}, st);
                VJ_CUDA(cudaEventRecord(e1, st));
                VJ_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                VJ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best) { best = ms; best_g = g; }
            }
            v->group = best_g;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }

    mark("set-up");
    // Iteration views in list mode: only blocks of unfinished instances run (rebuilt at the
    // start of every chunk, after the previous check decided which instances are done).
    int sms = 148;
    {
        int dev = 0;
        VJ_CUDA(cudaGetDevice(&dev));
        VJ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    CsrView a_it = a, at_it = at;
    BlockList list_a, list_at;
    VJ_TRY(list_a.attach(a_it, row_inst.get(), sms));
    VJ_TRY(list_at.attach(at_it, col_inst.get(), sms));

    DeviceBuffer<BatchCounters> counters;
    VJ_TRY(counters.alloc(1));
    VJ_CUDA(cudaMemsetAsync(counters.get(), 0, sizeof(BatchCounters), st));
    BatchCounters* hc = nullptr;
    hc = static_cast<BatchCounters*>(pinned_scratch(sizeof(BatchCounters)));
    if (!hc) { set_error("page-locked host memory for the batch counters"); return VAJRA_ERR_OUT_OF_MEMORY; }
    std::memset(hc, 0, sizeof(BatchCounters));
    struct Guard {
        cudaGraph_t g[2] = {nullptr, nullptr}; cudaGraphExec_t e[2] = {nullptr, nullptr};
        ~Guard() {
            for (int k = 0; k < 2; ++k) { if (e[k]) cudaGraphExecDestroy(e[k]); if (g[k]) cudaGraphDestroy(g[k]); }
        }
    } guard;

    BControl bc{};
    bc.tol = o.tolerance;
    bc.beta_sufficient = o.restart_sufficient;
    bc.beta_necessary = o.restart_necessary;
    bc.beta_artificial = o.restart_artificial;
    bc.pw_smoothing = o.primal_weight_smoothing;
    bc.count = count;
    bc.switch_tol = o.mixed_switch_tolerance;
    bc.stall_checks = o.mixed_stall_checks < 0 ? 0 : (o.mixed_stall_checks > kBHist - 1 ? kBHist - 1 : o.mixed_stall_checks);
    bc.early_tol = 10.0 * o.mixed_switch_tolerance;   // as the single-LP FP32 phase
    bc.gamma32 = (o.mixed_reflection > 0.0 && o.mixed_reflection <= 1.0) ? o.mixed_reflection : o.reflection;
    int64_t graph_kernels[2] = {0, 0};

    // One chunk of a pass in precision T (its iterates, values and bounds in T; the checks read
    // the FP64 values).  Pass 0 is the FP32 pass, pass 1 the FP64 one.
    struct PassBuffers {
        const void* csr; const void* csc;
        const void* c; const void* cl; const void* cu; const void* rl; const void* ru;
        void* x; void* x0; void* xb; void* xc; void* y; void* y0; void* yc;
    };
    const PassBuffers pb64{p.csr_val.get(), p.csc_val.get(), p.c.get(), p.col_lower.get(), p.col_upper.get(),
                           p.row_lower.get(), p.row_upper.get(), x.get(), x0.get(), xb.get(), xc.get(), y.get(),
                           y0.get(), yc.get()};
    const PassBuffers pb32{p.csr_val32.get(), p.csc_val32.get(), c32.get(), cl32.get(), cu32.get(), rl32.get(),
                           ru32.get(), x32.get(), x0_32.get(), xb32.get(), xc32.get(), y32.get(), y0_32.get(),
                           yc32.get()};
    auto chunk = [&](auto tag, int len, cudaGraphConditionalHandle again, int loop) {
        using T = decltype(tag);
        const PassBuffers& b = sizeof(T) == 4 ? pb32 : pb64;
        const T* csr = static_cast<const T*>(b.csr);
        const T* csc = static_cast<const T*>(b.csc);
        T* xv = static_cast<T*>(b.x); T* x0v = static_cast<T*>(b.x0); T* xbv = static_cast<T*>(b.xb);
        T* xcv = static_cast<T*>(b.xc); T* yv = static_cast<T*>(b.y); T* y0v = static_cast<T*>(b.y0);
        T* ycv = static_cast<T*>(b.yc);
        list_a.rebuild(S.done, st);
        list_at.rebuild(S.done, st);
        for (int kk = 0; kk < len; ++kk) {
            const int wc = kk == len - 1 ? 1 : 0;
            launch_spmv_t<T, T, T>(at_it, csc, yv,
                                   EpiBPrimal<T>{static_cast<const T*>(b.c), static_cast<const T*>(b.cl),
                                                 static_cast<const T*>(b.cu), x0v, xv, xbv, xcv, col_inst.get(), S,
                                                 kk, wc}, st);
            launch_spmv_t<T, T, T>(a_it, csr, xbv,
                                   EpiBDual<T>{static_cast<const T*>(b.rl), static_cast<const T*>(b.ru), y0v, yv, ycv,
                                               row_inst.get(), S, kk, wc}, st);
        }
        launch_spmv_t<double, T, double>(a_it, p.csr_val.get(), xcv, EpiBStore{ax.get(), row_inst.get(), S.done}, st);
        launch_spmv_t<double, T, double>(at_it, p.csc_val.get(), ycv, EpiBStore{aty.get(), col_inst.get(), S.done}, st);
        k_bkkt<T><<<count, kThreads, 0, st>>>(d_roff.get(), d_coff.get(), ax.get(), aty.get(), xcv, ycv,
                                              p.row_lower.get(), p.row_upper.get(), lp.row_lower.get(),
                                              lp.row_upper.get(), p.row_scale.get(), p.c.get(), lp.col_lower.get(),
                                              lp.col_upper.get(), p.col_scale.get(), x_last.get(), y_last.get(),
                                              part.get(), S);
        BControl c2 = bc;
        c2.len = len;
        c2.pass32 = sizeof(T) == 4 ? 1 : 0;
        k_bcontrol<<<(count + 127) / 128, 128, 0, st>>>(part.get(), c2, S);
        k_brestart<T><<<grid_for(mx), kThreads, 0, st>>>(m, n, row_inst.get(), col_inst.get(), xcv, ycv, xv, x0v, yv,
                                                         y0v, x_last.get(), y_last.get(), S);
        k_bcount<<<1, 1024, 0, st>>>(count, S.done, counters.get(), again, loop);
        note_launch(4);
    };

    const int64_t max_iter = o.iteration_limit;
    int64_t launched = 0;
    bool time_out = false;
    // Runs one pass until no instance is left in it or a limit is reached.  Full chunks run in
    // the pass graph: a WHILE node whose body is one chunk, repeated on the device while an
    // instance is active, at most `left` times a launch.  A last partial chunk (iteration
    // limit not a multiple of K) is launched directly.
    auto run_pass = [&](auto tag) -> vajra_status {
        using T = decltype(tag);
        const int k = sizeof(T) == 4 ? 0 : 1;
        long long pass_chunks = 0;   // chunks this pass has run, and the host time they took
        double pass_seconds = 0.0;
        while (launched < max_iter) {
            const int64_t remaining = max_iter - launched;
            if (remaining >= K) {
                if (!guard.e[k]) {
                    VJ_CUDA(cudaGraphCreate(&guard.g[k], 0));
                    cudaGraphConditionalHandle again;
                    VJ_CUDA(cudaGraphConditionalHandleCreate(&again, guard.g[k], 1, cudaGraphCondAssignDefault));
                    cudaGraphNodeParams np{};
                    np.type = cudaGraphNodeTypeConditional;
                    np.conditional.handle = again;
                    np.conditional.type = cudaGraphCondTypeWhile;
                    np.conditional.size = 1;
                    cudaGraphNode_t loop_node;
                    VJ_CUDA(cudaGraphAddNode(&loop_node, guard.g[k], nullptr, 0, &np));
                    const int64_t before = launch_count();
                    VJ_CUDA(cudaStreamBeginCaptureToGraph(st, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                          cudaStreamCaptureModeThreadLocal));
                    chunk(tag, K, again, 1);
                    cudaGraph_t body = nullptr;
                    VJ_CUDA(cudaStreamEndCapture(st, &body));
                    VJ_CUDA(cudaGraphInstantiate(&guard.e[k], guard.g[k], 0));
                    graph_kernels[k] = launch_count() - before;
                    launch_count() = before;
                }
                int64_t budget = kFirstLaunchChunks;
                if (pass_chunks > 0) {
                    // chunks that fit in the time left at this pass's measured rate (at least one)
                    const double per_chunk = pass_seconds / static_cast<double>(pass_chunks);
                    const double left_s = o.time_limit - seconds_since(t_start);
                    const double fit = per_chunk > 0.0 ? left_s / per_chunk : static_cast<double>(kMaxLaunchChunks);
                    budget = fit >= kMaxLaunchChunks ? kMaxLaunchChunks : (fit < 1.0 ? 1 : static_cast<int64_t>(fit));
                }
                if (remaining / K < budget) budget = remaining / K;
                const long long chunks_before = hc->chunks;
                const auto t_launch = Clock::now();
                hc->left = static_cast<int>(budget);
                VJ_CUDA(cudaMemcpyAsync(&counters.get()->left, &hc->left, sizeof(int), cudaMemcpyHostToDevice, st));
                VJ_CUDA(cudaGraphLaunch(guard.e[k], st));
                VJ_CUDA(cudaMemcpyAsync(hc, counters.get(), sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
                VJ_CUDA(cudaStreamSynchronize(st));
                const long long ran = hc->chunks - chunks_before;
                pass_chunks += ran;
                pass_seconds += seconds_since(t_launch);
                note_launch(graph_kernels[k] * ran);
                launched += ran * K;
                if (o.verbose)
                    std::fprintf(stderr, "[vajra] batch %s pass: %lld chunks to iteration %lld, %d active, %.1f ms\n",
                                 k == 0 ? "FP32" : "FP64", ran, static_cast<long long>(launched), hc->active,
                                 1e3 * seconds_since(t_start));
                if (ran < 1 || ran > budget) return VAJRA_ERR_INTERNAL;   // the loop runs 1..budget chunks
            } else {
                chunk(tag, static_cast<int>(remaining), cudaGraphConditionalHandle{}, 0);
                VJ_LAUNCH_CHECK();
                launched += remaining;
                VJ_CUDA(cudaMemcpyAsync(hc, counters.get(), sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
                VJ_CUDA(cudaStreamSynchronize(st));
            }
            if (hc->active == 0) break;
            if (seconds_since(t_start) > o.time_limit) { time_out = true; break; }
        }
        return VAJRA_OK;
    };
    if (mixed) {
        VJ_TRY(run_pass(float{}));
        k_bhandover<<<grid_for(mx), kThreads, 0, st>>>(m, n, row_inst.get(), col_inst.get(), xc32.get(), yc32.get(),
                                                       x.get(), x0.get(), xc.get(), x_last.get(), y.get(), y0.get(),
                                                       yc.get(), y_last.get(), S.status);
        k_bhandover_state<<<(count + 127) / 128, 128, 0, st>>>(count, o.reflection, S);
        k_bcount<<<1, 1024, 0, st>>>(count, S.done, counters.get(), cudaGraphConditionalHandle{}, 0);
        VJ_LAUNCH_CHECK();
        note_launch(3);
        VJ_CUDA(cudaMemcpyAsync(hc, counters.get(), sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
        VJ_CUDA(cudaStreamSynchronize(st));
    }
    if (!time_out && (!mixed || hc->active > 0)) VJ_TRY(run_pass(double{}));
    mark("iterations");

    // ---- post-processing -------------------------------------------------------------------
    DeviceBuffer<double> x_out, y_out, row_value, col_dual, objs;
    VJ_TRY(x_out.alloc(n));
    VJ_TRY(y_out.alloc(m));
    VJ_TRY(row_value.alloc(m));
    VJ_TRY(col_dual.alloc(n));
    VJ_TRY(objs.alloc(count));
    k_bpost<<<grid_for(mx), kThreads, 0, st>>>(m, n, col_inst.get(), d_sense.get(), xc.get(), yc.get(),
                                               p.col_scale.get(), p.row_scale.get(), p.scaled ? 1 : 0, x_out.get(),
                                               y_out.get());
    launch_spmv_t<double, double, double>(a, p.csr_val_orig.get(), x_out.get(), EpiStorePlain{row_value.get()}, st);
    launch_spmv_t<double, double, double>(at, lp.values.get(), y_out.get(), EpiStorePlain{col_dual.get()}, st);
    k_breduced<<<grid_for(n), kThreads, 0, st>>>(n, col_inst.get(), d_sense.get(), lp.c.get(), col_dual.get());
    k_bobjective<<<count, kThreads, 0, st>>>(d_coff.get(), lp.c.get(), x_out.get(), d_offsets.get(), objs.get());
    note_launch(3);
    VJ_LAUNCH_CHECK();
    timer.stop(st);
    std::vector<double> hx(n), hy(m), hrv(m), hcd(n), hobj(count), hd(18 * static_cast<size_t>(count));
    std::vector<long long> hl(3 * static_cast<size_t>(count));
    std::vector<int> hi(5 * static_cast<size_t>(count));
    VJ_CUDA(cudaMemcpyAsync(hx.data(), x_out.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hy.data(), y_out.get(), sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hrv.data(), row_value.get(), sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hcd.data(), col_dual.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hobj.data(), objs.get(), sizeof(double) * count, cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hd.data(), dd.get(), sizeof(double) * hd.size(), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hl.data(), dl.get(), sizeof(long long) * hl.size(), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaMemcpyAsync(hi.data(), di.get(), sizeof(int) * hi.size(), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    if (device_time) *device_time = timer.seconds();
    mark("post-processing, copies");
    auto field = [&](int q, int i) { return hd[static_cast<size_t>(q) * count + i]; };
    for (int i = 0; i < count; ++i) {
        vajra_result* r = &results[i];
        const int64_t r0 = roff[i], c0 = coff[i];
        const int mi = lps[i].num_rows, ni = lps[i].num_cols;
        if (r->col_value) std::memcpy(r->col_value, &hx[c0], sizeof(double) * ni);
        if (r->col_dual) std::memcpy(r->col_dual, &hcd[c0], sizeof(double) * ni);
        if (r->row_value) std::memcpy(r->row_value, &hrv[r0], sizeof(double) * mi);
        if (r->row_dual) std::memcpy(r->row_dual, &hy[r0], sizeof(double) * mi);
        const int status = hi[static_cast<size_t>(count) + i];
        r->status = status ? status : (time_out ? 7 : 6);
        r->iterations = hl[static_cast<size_t>(count) + i];
        r->objective_value = hobj[i];
        r->dual_objective = sense[i] ? -field(11, i) : field(11, i);
        r->restart_count = hi[2 * static_cast<size_t>(count) + i];
        r->rel_primal = r->primal_residual = field(6, i);
        r->rel_dual = r->dual_residual = field(7, i);
        r->rel_gap = r->duality_gap = field(8, i);
        r->rel_kkt = field(9, i);
        r->primal_weight = field(0, i);
        r->tau = field(2, i);
        r->sigma = field(3, i);
        r->spectral_norm_estimate = field(15, i);
        r->converged = r->status == 1 ? 1 : 0;
        r->fp32_iterations = hl[2 * static_cast<size_t>(count) + i];
        r->fp64_iterations = r->iterations - r->fp32_iterations;
        r->spmv_group_a = a.group;
        r->spmv_group_at = at.group;
        std::snprintf(r->status_message, sizeof(r->status_message), "%s",
                      r->status == 1 ? "relative KKT tolerance reached (batched)"
                      : r->status == 9 ? "NaN/Inf in the KKT evaluation (batched)"
                      : "limit reached before this instance converged (batched)");
    }
    return VAJRA_OK;
}

}  // namespace vajra
