// Reverse-mode derivative of the unrolled PDHG map (plain PDHG, primal first, fixed steps)
// for many LPs at once, packed block-diagonally.
//
// Forward, per instance i with tau_i = sigma_i = step_safety / ||A_i||_2 (constants of A):
//   pre   = x - tau (c + A^T y)          x+ = clip(pre, l, u)        x_bar = 2 x+ - x
//   q     = y + sigma A x_bar            y+ = q - sigma clamp(q / sigma, row_l, row_u)
// Loss of instance i: L_i = sum_j (w_j + c_j) x_j(K) in original units (the weighted final
// iterate plus its objective).  Scaling (Ruiz + Pock-Chambolle) depends on A only, so it is
// a constant of the map.
//
// Reverse pass, per step k (masks of step k: P = [l < pre < u] per column, and per row
// 1 = below row_l, 2 = above row_u, 0 = inside):
//   q^ = y^ [code != 0];  row_l^ -= sigma y^ [code == 1];  row_u^ -= sigma y^ [code == 2]
//   xbar^ = sigma A^T q^
//   pre^ = (x^ + 2 xbar^) P;  c^ -= tau pre^;  x^ <- pre^ - xbar^;  y^ <- q^ - tau A pre^
// Checkpoints (x, y) every `checkpoint_every` iterates; each segment is recomputed from its
// checkpoint, storing one byte per row / column per step, then reversed.
#include <cmath>
#include <cstring>
#include <vector>

#include "batch_common.cuh"
#include "solver.cuh"

namespace vajra {
namespace {

template <typename T>
struct EpiFwdPrimal {
    const T* c; const T* cl; const T* cu;
    T* x; T* xb;
    const int* col_inst; const double* step;
    uint8_t* mask;   // may be null
    __device__ bool active() const { return true; }
    template <typename Acc> __device__ void operator()(int j, Acc v) const {
        const T tau = static_cast<T>(step[col_inst[j]]);
        const T xo = x[j];
        const T pre = xo - tau * (c[j] + static_cast<T>(v));
        const T xn = pre < cl[j] ? cl[j] : (pre > cu[j] ? cu[j] : pre);
        if (mask) mask[j] = (pre > cl[j] && pre < cu[j]) ? 1 : 0;
        xb[j] = xn + xn - xo;
        x[j] = xn;
    }
};

template <typename T>
struct EpiFwdDual {
    const T* rl; const T* ru;
    T* y;
    const int* row_inst; const double* step;
    uint8_t* mask;
    __device__ bool active() const { return true; }
    template <typename Acc> __device__ void operator()(int i, Acc w) const {
        const T sg = static_cast<T>(step[row_inst[i]]);
        const T q = y[i] + sg * static_cast<T>(w);
        const T t = q / sg;
        const uint8_t code = t < rl[i] ? 1 : (t > ru[i] ? 2 : 0);
        const T cl = code == 1 ? rl[i] : (code == 2 ? ru[i] : t);
        if (mask) mask[i] = code;
        y[i] = q - sg * cl;
    }
};

// Rows, elementwise: q^ and the bound adjoints of step k; w^ = sigma q^ for the next SpMV.
template <typename T>
__global__ void k_bwd_rows(int m, const uint8_t* __restrict__ mask, const int* __restrict__ row_inst,
                           const double* __restrict__ step, T* __restrict__ yh, T* __restrict__ wh,
                           double* __restrict__ g_rl, double* __restrict__ g_ru) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint8_t code = mask[i];
    const double sg = step[row_inst[i]];
    const T y = yh[i];
    if (code == 1) g_rl[i] -= sg * static_cast<double>(y);
    if (code == 2) g_ru[i] -= sg * static_cast<double>(y);
    const T q = code != 0 ? y : T(0);
    yh[i] = q;
    wh[i] = static_cast<T>(sg) * q;
}

template <typename T>
struct EpiBwdPrimal {
    T* xh; T* preh;
    double* g_c;
    const uint8_t* mask;
    const int* col_inst; const double* step;
    __device__ bool active() const { return true; }
    template <typename Acc> __device__ void operator()(int j, Acc v) const {
        const T xbh = static_cast<T>(v);
        const T p = mask[j] ? xh[j] + xbh + xbh : T(0);
        g_c[j] -= step[col_inst[j]] * static_cast<double>(p);
        xh[j] = p - xbh;
        preh[j] = p;
    }
};

template <typename T>
struct EpiBwdDual {
    T* yh;
    const int* row_inst; const double* step;
    __device__ bool active() const { return true; }
    template <typename Acc> __device__ void operator()(int i, Acc s) const {
        yh[i] = yh[i] - static_cast<T>(step[row_inst[i]]) * static_cast<T>(s);
    }
};

template <typename T>
__global__ void k_adj_init(int m, int n, const double* __restrict__ cl, const double* __restrict__ cu,
                           T* __restrict__ x, T* __restrict__ xb, T* __restrict__ y) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) { const T v = static_cast<T>(fmin(fmax(0.0, cl[t]), cu[t])); x[t] = v; xb[t] = v; }
    if (t < m) y[t] = T(0);
}

// Loss per instance and the final iterate in original units.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_adj_loss(const int64_t* __restrict__ coff, const T* __restrict__ x, const double* __restrict__ cs,
           const double* __restrict__ w, const double* __restrict__ c, double* __restrict__ x_out,
           double* __restrict__ loss) {
    const int inst = blockIdx.x;
    __shared__ double red[32];
    double s[1] = {0.0};
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) {
        const double xo = static_cast<double>(x[j]) * cs[j];
        if (x_out) x_out[j] = xo;
        s[0] += ((w ? w[j] : 0.0) + c[j]) * xo;
    }
    block_reduce<OpSum, double, 1>(s, red);
    if (threadIdx.x == 0) loss[inst] = s[0];
}

template <typename T>
__global__ void k_adj_seed(int m, int n, const double* __restrict__ cs, const double* __restrict__ w,
                           const double* __restrict__ c, T* __restrict__ xh, T* __restrict__ yh,
                           double* __restrict__ g_c, double* __restrict__ g_rl, double* __restrict__ g_ru) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) { xh[t] = static_cast<T>(cs[t] * ((w ? w[t] : 0.0) + c[t])); g_c[t] = 0.0; }
    if (t < m) { yh[t] = T(0); g_rl[t] = 0.0; g_ru[t] = 0.0; }
}

// Scaled-space adjoints -> original units; c also gets the direct term x(K).
template <typename T>
__global__ void k_adj_finish(int m, int n, const double* __restrict__ cs, const double* __restrict__ rs,
                             const T* __restrict__ x, double* __restrict__ g_c, double* __restrict__ g_rl,
                             double* __restrict__ g_ru, const double* __restrict__ rl_o, const double* __restrict__ ru_o) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) g_c[t] = cs[t] * g_c[t] + cs[t] * static_cast<double>(x[t]);
    if (t < m) {
        g_rl[t] = rl_o[t] > -1e20 ? rs[t] * g_rl[t] : 0.0;
        g_ru[t] = ru_o[t] < 1e20 ? rs[t] * g_ru[t] : 0.0;
    }
}

template <typename T>
__global__ void k_convert_to(int64_t n, const double* __restrict__ s, T* __restrict__ d) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        d[k] = static_cast<T>(s[k]);
}

__global__ void k_steps(int count, const double* __restrict__ sigma_max, double safety, double* __restrict__ step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) step[i] = safety / (sigma_max[i] > 1e-12 ? sigma_max[i] : 1.0);
}

// TF: type of the forward map (values, iterates, checkpoints, masks come from it); TB: type
// of the reverse pass (cotangents and the transposed SpMVs).
template <typename TF, typename TB>
struct Unrolled {
    int m = 0, n = 0;
    CsrView a, at;
    const TF* csr_val = nullptr;
    const TF* csc_val = nullptr;
    const TB* csr_val_b = nullptr;
    const TB* csc_val_b = nullptr;
    DeviceBuffer<TF> c, cl, cu, rl, ru, x, xb, y, ckpt;
    DeviceBuffer<TB> xh, yh, wh, preh;
    DeviceBuffer<uint8_t> pmask, dmask;
    const int* row_inst = nullptr;
    const int* col_inst = nullptr;
    const double* step = nullptr;

    void forward_step(uint8_t* pm, uint8_t* dm, cudaStream_t st) {
        launch_spmv_t<TF, TF, TF>(at, csc_val, y.get(),
                                  EpiFwdPrimal<TF>{c.get(), cl.get(), cu.get(), x.get(), xb.get(), col_inst, step, pm}, st);
        launch_spmv_t<TF, TF, TF>(a, csr_val, xb.get(), EpiFwdDual<TF>{rl.get(), ru.get(), y.get(), row_inst, step, dm}, st);
    }
    void backward_step(const uint8_t* pm, const uint8_t* dm, double* g_c, double* g_rl, double* g_ru,
                       cudaStream_t st) {
        k_bwd_rows<TB><<<grid_for(m), kThreads, 0, st>>>(m, dm, row_inst, step, yh.get(), wh.get(), g_rl, g_ru);
        note_launch(1);
        launch_spmv_t<TB, TB, TB>(at, csc_val_b, wh.get(),
                                  EpiBwdPrimal<TB>{xh.get(), preh.get(), g_c, pm, col_inst, step}, st);
        launch_spmv_t<TB, TB, TB>(a, csr_val_b, preh.get(), EpiBwdDual<TB>{yh.get(), row_inst, step}, st);
    }
};

template <typename T>
void values_of(Prepared& p, const T** csr, const T** csc) {
    if constexpr (sizeof(T) == 4) {
        *csr = p.csr_val32.get();
        *csc = p.csc_val32.get();
    } else {
        *csr = p.csr_val.get();
        *csc = p.csc_val.get();
    }
}

template <typename TF, typename TB>
vajra_status run_unrolled_t(const PackedHost& P, const vajra_unrolled_opts& o, Prepared& p, const DeviceLp& lp,
                            const int* row_inst, const int* col_inst, const int64_t* d_coff, const double* step,
                            const DeviceBuffer<double>& d_w, const double* c_orig_dev, double* h_loss, double* h_x,
                            double* h_gc, double* h_grl, double* h_gru, cudaStream_t st) {
    const int m = P.m, n = P.n, count = P.count;
    const int K = o.iterations;
    const int C = o.checkpoint_every > 0 ? o.checkpoint_every : 100;
    const int nseg = (K + C - 1) / C;
    const bool want_grad = h_gc || h_grl || h_gru;
    Unrolled<TF, TB> U;
    U.m = m; U.n = n;
    U.a = p.a; U.at = p.at;
    U.row_inst = row_inst; U.col_inst = col_inst; U.step = step;
    if (sizeof(TF) == 4 || sizeof(TB) == 4) VJ_TRY(make_f32_values(p, P.nnz, st));
    values_of<TF>(p, &U.csr_val, &U.csc_val);
    values_of<TB>(p, &U.csr_val_b, &U.csc_val_b);
    for (auto* b : {&U.c, &U.cl, &U.cu, &U.x, &U.xb}) VJ_TRY(b->alloc(n));
    for (auto* b : {&U.rl, &U.ru, &U.y}) VJ_TRY(b->alloc(m));
    for (auto* b : {&U.xh, &U.preh}) VJ_TRY(b->alloc(n));
    for (auto* b : {&U.yh, &U.wh}) VJ_TRY(b->alloc(m));
    auto conv = [&](const double* s, TF* d, int k) {
        if (k > 0) { k_convert_to<TF><<<grid_for(k, kThreads, 148 * 32), kThreads, 0, st>>>(k, s, d); note_launch(1); }
    };
    conv(p.c.get(), U.c.get(), n);
    conv(p.col_lower.get(), U.cl.get(), n);
    conv(p.col_upper.get(), U.cu.get(), n);
    conv(p.row_lower.get(), U.rl.get(), m);
    conv(p.row_upper.get(), U.ru.get(), m);
    const int mx = m > n ? m : n;
    k_adj_init<TF><<<grid_for(mx), kThreads, 0, st>>>(m, n, p.col_lower.get(), p.col_upper.get(), U.x.get(), U.xb.get(),
                                                     U.y.get());
    note_launch(1);
    if (want_grad) {
        VJ_TRY(U.ckpt.alloc(static_cast<size_t>(nseg) * (static_cast<size_t>(n) + m)));
        VJ_TRY(U.pmask.alloc(static_cast<size_t>(C) * n));
        VJ_TRY(U.dmask.alloc(static_cast<size_t>(C) * m));
    }
    VJ_LAUNCH_CHECK();
    auto ck_x = [&](int s) { return U.ckpt.get() + static_cast<size_t>(s) * (static_cast<size_t>(n) + m); };
    auto ck_y = [&](int s) { return ck_x(s) + n; };
    // forward, with checkpoints
    for (int s = 0; s < nseg; ++s) {
        const int len = (s + 1) * C <= K ? C : K - s * C;
        if (want_grad) {
            VJ_CUDA(cudaMemcpyAsync(ck_x(s), U.x.get(), sizeof(TF) * n, cudaMemcpyDeviceToDevice, st));
            VJ_CUDA(cudaMemcpyAsync(ck_y(s), U.y.get(), sizeof(TF) * m, cudaMemcpyDeviceToDevice, st));
        }
        for (int k = 0; k < len; ++k) U.forward_step(nullptr, nullptr, st);
    }
    DeviceBuffer<double> loss, x_out, g_c, g_rl, g_ru;
    VJ_TRY(loss.alloc(count));
    VJ_TRY(x_out.alloc(n));
    k_adj_loss<TF><<<count, kThreads, 0, st>>>(d_coff, U.x.get(), p.col_scale.get(), d_w.get(), c_orig_dev, x_out.get(),
                                               loss.get());
    note_launch(1);
    VJ_LAUNCH_CHECK();
    if (want_grad) {
        VJ_TRY(g_c.alloc(n));
        VJ_TRY(g_rl.alloc(m));
        VJ_TRY(g_ru.alloc(m));
        DeviceBuffer<TF> x_final;
        VJ_TRY(x_final.alloc(n));
        VJ_CUDA(cudaMemcpyAsync(x_final.get(), U.x.get(), sizeof(TF) * n, cudaMemcpyDeviceToDevice, st));
        k_adj_seed<TB><<<grid_for(mx), kThreads, 0, st>>>(m, n, p.col_scale.get(), d_w.get(), c_orig_dev, U.xh.get(),
                                                         U.yh.get(), g_c.get(), g_rl.get(), g_ru.get());
        note_launch(1);
        for (int s = nseg - 1; s >= 0; --s) {
            const int len = (s + 1) * C <= K ? C : K - s * C;
            VJ_CUDA(cudaMemcpyAsync(U.x.get(), ck_x(s), sizeof(TF) * n, cudaMemcpyDeviceToDevice, st));
            VJ_CUDA(cudaMemcpyAsync(U.y.get(), ck_y(s), sizeof(TF) * m, cudaMemcpyDeviceToDevice, st));
            for (int k = 0; k < len; ++k)
                U.forward_step(U.pmask.get() + static_cast<size_t>(k) * n, U.dmask.get() + static_cast<size_t>(k) * m, st);
            for (int k = len - 1; k >= 0; --k)
                U.backward_step(U.pmask.get() + static_cast<size_t>(k) * n, U.dmask.get() + static_cast<size_t>(k) * m,
                                g_c.get(), g_rl.get(), g_ru.get(), st);
        }
        k_adj_finish<TF><<<grid_for(mx), kThreads, 0, st>>>(m, n, p.col_scale.get(), p.row_scale.get(), x_final.get(),
                                                           g_c.get(), g_rl.get(), g_ru.get(), lp.row_lower.get(),
                                                           lp.row_upper.get());
        note_launch(1);
        VJ_LAUNCH_CHECK();
        if (h_gc) VJ_CUDA(cudaMemcpyAsync(h_gc, g_c.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        if (h_grl) VJ_CUDA(cudaMemcpyAsync(h_grl, g_rl.get(), sizeof(double) * m, cudaMemcpyDeviceToHost, st));
        if (h_gru) VJ_CUDA(cudaMemcpyAsync(h_gru, g_ru.get(), sizeof(double) * m, cudaMemcpyDeviceToHost, st));
        VJ_CUDA(cudaStreamSynchronize(st));
    }
    if (h_loss) VJ_CUDA(cudaMemcpyAsync(h_loss, loss.get(), sizeof(double) * count, cudaMemcpyDeviceToHost, st));
    if (h_x) VJ_CUDA(cudaMemcpyAsync(h_x, x_out.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

}  // namespace

vajra_status run_unrolled(int count, const vajra_lp* lps, const vajra_unrolled_opts& o, const double* weights,
                          double* h_loss, double* h_x, double* h_gc, double* h_grl, double* h_gru, cudaStream_t st) {
    PackedHost P;
    VJ_TRY(pack_lps(count, lps, P));
    for (int i = 0; i < count; ++i)
        if (P.sense[i]) { set_error("instance %d: the unrolled map is defined for minimisation", i); return VAJRA_ERR_INVALID_ARGUMENT; }
    DeviceLp lp;
    VJ_TRY(upload_lp(&P.view, lp, st));
    DeviceBuffer<int64_t> d_roff, d_coff;
    DeviceBuffer<int> row_inst, col_inst;
    VJ_TRY(upload_vec(d_roff, P.roff, st));
    VJ_TRY(upload_vec(d_coff, P.coff, st));
    VJ_TRY(row_inst.alloc(P.m));
    VJ_TRY(col_inst.alloc(P.n));
    k_fill_instance_map<<<count, kThreads, 0, st>>>(d_roff.get(), count, row_inst.get());
    k_fill_instance_map<<<count, kThreads, 0, st>>>(d_coff.get(), count, col_inst.get());
    note_launch(2);
    DeviceBuffer<double> d_w;
    if (weights) {
        VJ_TRY(d_w.alloc(P.n));
        VJ_CUDA(cudaMemcpyAsync(d_w.get(), weights, sizeof(double) * P.n, cudaMemcpyHostToDevice, st));
    }
    Prepared p;
    DeviceBuffer<SetupState> sst;
    VJ_TRY(sst.alloc(1));
    VJ_TRY(build_csr(lp, p, st));
    ScalingOpts so;
    so.enable = o.enable_scaling != 0;
    so.ruiz_iterations = 10;
    so.pock_chambolle = true;
    VJ_TRY(prepare_scaled(lp, p, so, sst.get(), st));
    VJ_TRY(plan_spmv(lp, p, st));
    DeviceBuffer<double> sigma_max, step;
    VJ_TRY(sigma_max.alloc(count));
    VJ_TRY(step.alloc(count));
    VJ_TRY(batched_spectral_norms(p, P.m, P.n, count, col_inst.get(), d_coff.get(), sigma_max.get(), 60, st));
    const double safety = (o.step_safety > 0.0 && o.step_safety < 1.0) ? o.step_safety : 0.95;
    k_steps<<<(count + 127) / 128, 128, 0, st>>>(count, sigma_max.get(), safety, step.get());
    note_launch(1);
    VJ_LAUNCH_CHECK();
    // the weight pointer handed to the kernels is null when no weights were given
    DeviceBuffer<double> none;
    const DeviceBuffer<double>& w = weights ? d_w : none;
    // FP64: FP64 map and reverse pass.  MIXED: the FP64 map (forward, checkpoints and the
    // recomputed active sets), reverse pass in FP32.  FP32: the FP32 map and reverse pass.
    if (o.precision == VAJRA_PREC_FP64)
        return run_unrolled_t<double, double>(P, o, p, lp, row_inst.get(), col_inst.get(), d_coff.get(), step.get(), w,
                                              lp.c.get(), h_loss, h_x, h_gc, h_grl, h_gru, st);
    if (o.precision == VAJRA_PREC_FP32)
        return run_unrolled_t<float, float>(P, o, p, lp, row_inst.get(), col_inst.get(), d_coff.get(), step.get(), w,
                                            lp.c.get(), h_loss, h_x, h_gc, h_grl, h_gru, st);
    return run_unrolled_t<double, float>(P, o, p, lp, row_inst.get(), col_inst.get(), d_coff.get(), step.get(), w,
                                         lp.c.get(), h_loss, h_x, h_gc, h_grl, h_gru, st);
}

}  // namespace vajra
