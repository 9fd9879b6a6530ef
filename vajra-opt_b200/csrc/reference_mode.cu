// VAJRA_ALGO_REFERENCE: the reference CPU PDHG (CpuPdhgSolver::solve,
// src/solvers/pdhg/pdhg.cpp:70-440) executed on the device in FP64 with the reference's
// evaluation order, so results are bit-identical to the CPU solver on the same input.
//
// Per iteration two fused kernels (the reference GPU loop uses four launches,
// src/solvers/gpu/pdhg_cuda.cu:261-279):
//   dual   : w = A x_bar (CSR, in-order, |x|<=1e-11 skipped) -> y = prox_sigma(y + sigma w)
//   primal : v = A^T y (CSC = CSR of A^T, in-order)          -> x+ = clamp(x - tau (v + c)),
//                                                              x_bar = 2 x+ - x
// Every check_frequency iterations: A x, then one CTA evaluates the residuals, gap, best
// iterate, stopping test, tau/sigma rebalancing and stagnation restart (pdhg.cpp:250-365)
// and a commit kernel applies the copies it decided.  tau, sigma and all decisions stay in
// device memory; the host reads one small state record per chunk.  A chunk of
// check_frequency iterations plus its check is captured once as a CUDA graph.
#include <cmath>
#include <cstring>
#include <vector>

#include "solver.cuh"

namespace vajra {
namespace {

struct RefState {
    double tau;
    double sigma;
    double spectral_norm;
    double best_infeas;
    double prim, dual, gap;
    double objective;
    long long iter_base;     // iterations finished before the current chunk
    long long stop_iter;     // iteration at which the loop stopped (1-based)
    long long stagnation;
    int stop;                // no further iteration work
    int status;              // SolveStatus decided on the device (0 = undecided)
    int restart_count;
    int converged;
    int commit_best;         // copy x, y -> best_x, best_y at the next commit
    int commit_restart;      // copy x -> x_bar at the next commit
    int pad[2];
};

constexpr int kStatusOptimal = 1;
constexpr int kStatusFeasible = 5;
constexpr int kStatusIterLimit = 6;
constexpr int kStatusTimeLimit = 7;
constexpr int kStatusNumerical = 9;

__device__ __forceinline__ void flag_nan(RefState* st, long long iter) {
    st->stop = 1;
    st->status = kStatusNumerical;
    st->stop_iter = iter;
    st->commit_best = 0;
    st->commit_restart = 0;
}

struct EpiRefDual {
    const double* rl;
    const double* ru;
    double* y;
    RefState* st;
    int kk;   // 0-based iteration index within the chunk
    __device__ bool active() const { return st->stop == 0; }
    __device__ void operator()(int i, double w) const {
        const double yn = dual_prox_exact(y[i], w, st->sigma, rl[i], ru[i]);
        y[i] = yn;
        if (isnan(yn) || isinf(yn)) flag_nan(st, st->iter_base + kk + 1);
    }
};

struct EpiRefPrimal {
    const double* c;
    const double* cl;
    const double* cu;
    double* x;
    double* xb;
    RefState* st;
    int kk;
    __device__ bool active() const { return st->stop == 0; }
    __device__ void operator()(int j, double v) const {
        const double x_old = x[j];
        const double x_new = primal_prox_exact(x_old, v, c[j], st->tau, cl[j], cu[j]);
        x[j] = x_new;
        xb[j] = extrapolate_exact(x_new, x_old);
        if (isnan(x_new) || isinf(x_new)) flag_nan(st, st->iter_base + kk + 1);
    }
};

struct EpiStoreRef {
    double* out;
    const RefState* st;
    __device__ bool active() const { return st->stop == 0; }
    __device__ void operator()(int i, double s) const { out[i] = s; }
};

// Convergence check (pdhg.cpp:259-364).  Maxima in parallel (order-free), the two sums by
// thread 0 in index order as the reference accumulates them.
__global__ void __launch_bounds__(1024)
k_ref_check(int m, int n, const double* __restrict__ ax, const double* __restrict__ x,
            const double* __restrict__ y, const double* __restrict__ v, const double* __restrict__ c,
            const double* __restrict__ rl, const double* __restrict__ ru, const double* __restrict__ cl,
            const double* __restrict__ cu, int chunk_len, int check_freq, double tol, double gap_tol,
            double safety, RefState* st) {
    if (st->stop) return;
    __shared__ double red[2 * 32];
    double mx[2] = {0.0, 0.0};   // prim, dual
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double a = ax[i];
        if (a < rl[i]) { const double d = rl[i] - a; if (d > mx[0]) mx[0] = d; }
        if (a > ru[i]) { const double d = a - ru[i]; if (d > mx[0]) mx[0] = d; }
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double xj = x[j], lj = cl[j], uj = cu[j];
        if (xj < lj) { const double d = lj - xj; if (d > mx[0]) mx[0] = d; }
        if (xj > uj) { const double d = xj - uj; if (d > mx[0]) mx[0] = d; }
        const double dj = __dadd_rn(c[j], v[j]);
        if (xj > __dadd_rn(lj, 1e-5) && dj > 1e-6 && dj > mx[1]) mx[1] = dj;
        if (xj < __dsub_rn(uj, 1e-5) && dj < -1e-6 && -dj > mx[1]) mx[1] = -dj;
        if (lj <= -1e20 && uj >= 1e20 && fabs(dj) > mx[1]) mx[1] = fabs(dj);
    }
    block_reduce<OpMax, double, 2>(mx, red);
    if (threadIdx.x != 0) return;
    const double prim = mx[0], dual = mx[1];
    double dual_obj = 0.0;
    for (int i = 0; i < m; ++i) {
        const double yi = y[i];
        if (yi > 1e-12 && ru[i] < 1e20) dual_obj = __dsub_rn(dual_obj, __dmul_rn(yi, ru[i]));
        else if (yi < -1e-12 && rl[i] > -1e20) dual_obj = __dsub_rn(dual_obj, __dmul_rn(yi, rl[i]));
    }
    for (int j = 0; j < n; ++j) {
        const double dj = __dadd_rn(c[j], v[j]);
        if (dj > 1e-12 && cl[j] > -1e20) dual_obj = __dadd_rn(dual_obj, __dmul_rn(dj, cl[j]));
        else if (dj < -1e-12 && cu[j] < 1e20) dual_obj = __dadd_rn(dual_obj, __dmul_rn(dj, cu[j]));
    }
    double primal_obj = 0.0;
    for (int j = 0; j < n; ++j) primal_obj = __dadd_rn(primal_obj, __dmul_rn(c[j], x[j]));
    const double gap = __ddiv_rn(fabs(__dsub_rn(primal_obj, dual_obj)),
                                 __dadd_rn(__dadd_rn(1.0, fabs(primal_obj)), fabs(dual_obj)));
    st->prim = prim;
    st->dual = dual;
    st->gap = gap;
    const long long iter = st->iter_base + chunk_len;
    st->commit_best = 0;
    st->commit_restart = 0;
    const double total = __dadd_rn(prim, dual);
    if (total < st->best_infeas) {
        st->best_infeas = total;
        st->commit_best = 1;
        st->stagnation = 0;
    } else {
        st->stagnation += check_freq;
    }
    if (prim <= tol && dual <= tol && gap <= gap_tol) {
        st->converged = 1;
        st->commit_best = 1;
        st->status = kStatusOptimal;
        st->stop = 1;
        st->stop_iter = iter;
        st->iter_base = iter;
        return;
    }
    const double norm = st->spectral_norm;
    const double ss = __dmul_rn(safety, safety);
    if (prim > __dmul_rn(10.0, dual) && dual > 0.0) {
        const double s13 = __dmul_rn(st->sigma, 1.3);
        st->sigma = (s13 < 1e6) ? s13 : 1e6;
        st->tau = __ddiv_rn(ss, __dmul_rn(__dmul_rn(norm, norm), st->sigma));
    } else if (dual > __dmul_rn(10.0, prim) && prim > 0.0) {
        const double t13 = __dmul_rn(st->tau, 1.3);
        st->tau = (t13 < 1e6) ? t13 : 1e6;
        st->sigma = __ddiv_rn(ss, __dmul_rn(__dmul_rn(norm, norm), st->tau));
    }
    if (st->stagnation >= 200) {
        st->commit_restart = 1;
        st->restart_count += 1;
        st->stagnation = 0;
    }
    st->iter_base = iter;
}

__global__ void k_ref_commit(int m, int n, const double* __restrict__ x, const double* __restrict__ y,
                             double* __restrict__ best_x, double* __restrict__ best_y,
                             double* __restrict__ xb, const RefState* st) {
    const int b = st->commit_best, r = st->commit_restart;
    if (!b && !r) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        if (b) best_x[i] = x[i];
        if (r) xb[i] = x[i];
    }
    if (b && i < m) best_y[i] = y[i];
}

__global__ void k_init_x(int n, const double* __restrict__ cl, const double* __restrict__ cu,
                         double* __restrict__ x, double* __restrict__ xb, double* __restrict__ best_x) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double val = 0.0;                 // pdhg.cpp:167-175
    if (val < cl[j]) val = cl[j];
    if (val > cu[j]) val = cu[j];
    x[j] = val;
    xb[j] = val;
    best_x[j] = val;
}

__global__ void k_ref_status(long long max_iter, int timed_out, RefState* st) {
    if (st->stop) return;            // converged or NaN: status and stop_iter already set
    if (timed_out) {
        st->status = kStatusTimeLimit;
        st->stop_iter = st->iter_base;
        return;
    }
    st->stop_iter = st->iter_base + 1;   // loop variable after the last iteration
    st->status = (st->stop_iter >= max_iter && st->best_infeas <= 1e-4) ? kStatusFeasible : kStatusIterLimit;
}

// Unscale (pdhg.cpp:381-387) and flip the dual sign (:409-411).
__global__ void k_ref_unscale(int m, int n, const double* __restrict__ bx, const double* __restrict__ by,
                              const double* __restrict__ cs, const double* __restrict__ rs, int scaled,
                              int is_max, double* __restrict__ x_out, double* __restrict__ y_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x_out[i] = scaled ? __dmul_rn(bx[i], cs[i]) : bx[i];
    if (i < m) {
        const double yv = scaled ? __dmul_rn(by[i], rs[i]) : by[i];
        y_out[i] = is_max ? yv : -yv;
    }
}

__global__ void k_objective_seq(int n, const double* __restrict__ c, const double* __restrict__ x, double offset,
                                RefState* st) {
    double obj = offset;               // pdhg.cpp:396-399
    for (int j = 0; j < n; ++j) obj = __dadd_rn(obj, __dmul_rn(c[j], x[j]));
    st->objective = obj;
}

__global__ void k_reduced_cost(int n, const double* __restrict__ c, double* __restrict__ d) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) d[j] = __dsub_rn(c[j], d[j]);   // d = c - A^T y (pdhg.cpp:416-418)
}

}  // namespace

vajra_status run_reference(vajra_pdhg* h, vajra_result* r) {
    const auto t_start = Clock::now();
    cudaStream_t st = h->stream;
    StreamTimer dev_timer;
    dev_timer.start(st);
    const vajra_opts& o = h->opts;
    const int m = h->m, n = h->n;
    const int64_t nnz = h->nnz;
    const bool is_max = h->sense != 0;
    const DeviceLp& lp = h->lp;

    Prepared p;
    DeviceBuffer<SetupState> sst;
    VJ_TRY(sst.alloc(1));
    VJ_TRY(build_csr(lp, p, st));
    ScalingOpts so;
    so.enable = o.enable_scaling != 0;
    so.ruiz_iterations = 10;          // pdhg.cpp:143-148 passes 10 regardless of options
    so.ruiz_tolerance = 0.05;
    so.pock_chambolle = false;
    so.negate_c = is_max;
    VJ_TRY(prepare_scaled(lp, p, so, sst.get(), st));
    double spectral_norm = 1.0;       // pdhg.cpp:14-16: nnz == 0 -> 1.0
    if (nnz > 0) {
        VJ_TRY(spectral_norm_exact(p, m, n, 25, 1e-4, sst.get(), st));
        SetupState hs{};
        VJ_CUDA(cudaMemcpyAsync(&hs, sst.get(), sizeof(hs), cudaMemcpyDeviceToHost, st));
        VJ_CUDA(cudaStreamSynchronize(st));
        spectral_norm = hs.spectral_norm;
    }
    const double safety = 0.95;       // clamp(0.95, 0.5, 0.99), pdhg.cpp:156
    RefState init{};
    init.tau = safety / spectral_norm;
    init.sigma = safety / spectral_norm;
    init.spectral_norm = spectral_norm;
    init.best_infeas = 1e20;
    DeviceBuffer<RefState> dst;
    VJ_TRY(dst.alloc(1));
    VJ_CUDA(cudaMemcpyAsync(dst.get(), &init, sizeof(init), cudaMemcpyHostToDevice, st));

    DeviceBuffer<double> x, xb, y, best_x, best_y, ax;
    VJ_TRY(x.alloc(n));
    VJ_TRY(xb.alloc(n));
    VJ_TRY(best_x.alloc(n));
    VJ_TRY(y.alloc(m));
    VJ_TRY(best_y.alloc(m));
    VJ_TRY(ax.alloc(m));
    VJ_CUDA(cudaMemsetAsync(y.get(), 0, sizeof(double) * m, st));
    VJ_CUDA(cudaMemsetAsync(best_y.get(), 0, sizeof(double) * m, st));
    k_init_x<<<grid_for(n), kThreads, 0, st>>>(n, p.col_lower.get(), p.col_upper.get(), x.get(), xb.get(), best_x.get());
    VJ_LAUNCH_CHECK();
    VJ_CUDA(cudaStreamSynchronize(st));
    const double setup_time = seconds_since(t_start);

    // exact (in-order) views of A and A^T
    CsrView a = p.a, at = p.at;
    a.group = 1;
    at.group = 1;
    RefState* S = dst.get();
    const int check_freq = o.check_frequency > 1 ? o.check_frequency : 1;
    const int64_t max_iter = o.iteration_limit;
    const double tol = o.tolerance, gap_tol = o.gap_tolerance;
    const int mx = m > n ? m : n;

    auto enqueue_chunk = [&](int len) {
        for (int kk = 0; kk < len; ++kk) {
            launch_spmv_exact<double, true>(a, p.csr_val.get(), xb.get(),
                                            EpiRefDual{p.row_lower.get(), p.row_upper.get(), y.get(), S, kk}, st);
            launch_spmv_exact<double, false>(at, p.csc_val.get(), y.get(),
                                             EpiRefPrimal{p.c.get(), p.col_lower.get(), p.col_upper.get(), x.get(),
                                                          xb.get(), S, kk}, st);
        }
        // The primal SpMV output v (A^T y) is needed by the check; recompute it in order.
        launch_spmv_exact<double, true>(a, p.csr_val.get(), x.get(), EpiStoreRef{ax.get(), S}, st);
    };
    DeviceBuffer<double> v;
    VJ_TRY(v.alloc(n));
    auto enqueue_check = [&](int len) {
        launch_spmv_exact<double, false>(at, p.csc_val.get(), y.get(), EpiStoreRef{v.get(), S}, st);
        note_launch(2);
        k_ref_check<<<1, 1024, 0, st>>>(m, n, ax.get(), x.get(), y.get(), v.get(), p.c.get(), p.row_lower.get(),
                                        p.row_upper.get(), p.col_lower.get(), p.col_upper.get(), len, check_freq,
                                        tol, gap_tol, safety, S);
        k_ref_commit<<<grid_for(mx), kThreads, 0, st>>>(m, n, x.get(), y.get(), best_x.get(), best_y.get(),
                                                        xb.get(), S);
    };

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    RefState* hs = nullptr;
    hs = static_cast<RefState*>(pinned_scratch(sizeof(RefState)));
    if (!hs) { set_error("page-locked host memory for the solver state"); return VAJRA_ERR_OUT_OF_MEMORY; }
    struct Cleanup {
        cudaGraph_t* g; cudaGraphExec_t* e;
        ~Cleanup() { if (*e) cudaGraphExecDestroy(*e); if (*g) cudaGraphDestroy(*g); }
    } cleanup{&graph, &exec};

    const auto t_iter = Clock::now();
    int64_t done_iters = 0;
    int timed_out = 0;
    int64_t before = 0, graph_kernels = 0;
    while (done_iters < max_iter) {
        const int64_t remaining = max_iter - done_iters;
        const int len = static_cast<int>(remaining < check_freq ? remaining : check_freq);
        if (len == check_freq) {
            if (!exec) {
                before = launch_count();
                VJ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                enqueue_chunk(len);
                enqueue_check(len);
                VJ_CUDA(cudaStreamEndCapture(st, &graph));
                VJ_CUDA(cudaGraphInstantiate(&exec, graph, 0));
                graph_kernels = launch_count() - before;
                launch_count() = before;
            }
            VJ_CUDA(cudaGraphLaunch(exec, st));
            note_launch(graph_kernels);
        } else {
            enqueue_chunk(len);
            enqueue_check(len);
            VJ_LAUNCH_CHECK();
        }
        done_iters += len;
        VJ_CUDA(cudaMemcpyAsync(hs, S, sizeof(RefState), cudaMemcpyDeviceToHost, st));
        VJ_CUDA(cudaStreamSynchronize(st));
        h->transfers++;
        if (hs->stop) break;
        if (seconds_since(t_start) > o.time_limit) { timed_out = 1; break; }
    }
    k_ref_status<<<1, 1, 0, st>>>(max_iter, timed_out, S);

    // Post-processing on the original model (pdhg.cpp:380-418).
    DeviceBuffer<double> x_out, y_out, row_value, col_dual;
    VJ_TRY(x_out.alloc(n));
    VJ_TRY(y_out.alloc(m));
    VJ_TRY(row_value.alloc(m));
    VJ_TRY(col_dual.alloc(n));
    k_ref_unscale<<<grid_for(mx), kThreads, 0, st>>>(m, n, best_x.get(), best_y.get(), p.col_scale.get(),
                                                     p.row_scale.get(), p.scaled ? 1 : 0, is_max ? 1 : 0,
                                                     x_out.get(), y_out.get());
    CsrView a_orig = a;
    launch_spmv_exact<double, true>(a_orig, p.csr_val_orig.get(), x_out.get(), EpiStore<double>{row_value.get()}, st);
    k_objective_seq<<<1, 1, 0, st>>>(n, lp.c.get(), x_out.get(), h->objective_offset, S);
    launch_spmv_exact<double, false>(at, lp.values.get(), y_out.get(), EpiStore<double>{col_dual.get()}, st);
    k_reduced_cost<<<grid_for(n), kThreads, 0, st>>>(n, lp.c.get(), col_dual.get());
    VJ_LAUNCH_CHECK();
    VJ_CUDA(cudaMemcpyAsync(hs, S, sizeof(RefState), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    const double iter_time = seconds_since(t_iter);

    dev_timer.stop(st);
    r->device_time_sec = dev_timer.seconds();
    const auto t_dl = Clock::now();
    copy_out_vector(r->col_value, x_out.get(), n, st);
    copy_out_vector(r->row_value, row_value.get(), m, st);
    copy_out_vector(r->row_dual, y_out.get(), m, st);
    copy_out_vector(r->col_dual, col_dual.get(), n, st);
    VJ_CUDA(cudaStreamSynchronize(st));
    h->transfers += 4;
    r->status = hs->status;
    r->iterations = hs->stop_iter;
    r->objective_value = hs->objective;
    r->dual_objective = hs->objective;   // best_dual_bound = objective (pdhg.cpp:401)
    r->restart_count = hs->restart_count;
    r->primal_residual = hs->prim;
    r->dual_residual = hs->dual;
    r->duality_gap = hs->gap;
    r->spectral_norm_estimate = spectral_norm;
    r->tau = init.tau;                   // PdhgDiagnostics reports the initial steps
    r->sigma = init.sigma;
    r->converged = hs->converged;
    r->fp64_iterations = hs->stop_iter;
    r->fp32_iterations = 0;
    r->setup_time_sec = setup_time;
    r->iteration_time_sec = iter_time;
    r->download_time_sec = seconds_since(t_dl);
    r->spmv_group_a = -1;
    r->spmv_group_at = -1;
    const char* msg = "";
    switch (hs->status) {
        case kStatusOptimal: msg = "PDHG converged to optimal primal and dual tolerance"; break;
        case kStatusNumerical: msg = "PDHG iterate encountered NaN/Inf"; break;
        case kStatusTimeLimit: msg = "PDHG time limit reached"; break;
        default: msg = "PDHG reached iteration limit"; break;
    }
    std::snprintf(r->status_message, sizeof(r->status_message), "%s", msg);
    return VAJRA_OK;
}

}  // namespace vajra
