// Device set-up passes: upload, CSC -> CSR, Ruiz / Pock-Chambolle scaling, power iteration.
// The reference runs all of this single-threaded on the host before the first iteration
// (src/solvers/gpu/pdhg_cuda.cu:136-171); here it stays on the device.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <cmath>

#include "problem.cuh"

namespace vajra {

// ---------------------------------------------------------------------------------------
// upload
// ---------------------------------------------------------------------------------------
template <typename T>
static vajra_status upload(DeviceBuffer<T>& d, const T* h, size_t n, cudaStream_t st) {
    VJ_TRY(d.alloc(n));
    if (n) VJ_CUDA(cudaMemcpyAsync(d.get(), h, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return VAJRA_OK;
}

vajra_status upload_lp(const vajra_lp* lp, DeviceLp& d, cudaStream_t st) {
    d.m = lp->num_rows;
    d.n = lp->num_cols;
    d.nnz = lp->col_ptr[lp->num_cols];
    d.sense = lp->sense;
    d.objective_offset = lp->objective_offset;
    VJ_TRY(upload(d.col_ptr, lp->col_ptr, static_cast<size_t>(d.n) + 1, st));
    VJ_TRY(upload(d.row_idx, lp->row_idx, static_cast<size_t>(d.nnz), st));
    VJ_TRY(upload(d.values, lp->values, static_cast<size_t>(d.nnz), st));
    VJ_TRY(upload(d.c, lp->c, static_cast<size_t>(d.n), st));
    VJ_TRY(upload(d.col_lower, lp->col_lower, static_cast<size_t>(d.n), st));
    VJ_TRY(upload(d.col_upper, lp->col_upper, static_cast<size_t>(d.n), st));
    VJ_TRY(upload(d.row_lower, lp->row_lower, static_cast<size_t>(d.m), st));
    VJ_TRY(upload(d.row_upper, lp->row_upper, static_cast<size_t>(d.m), st));
    return VAJRA_OK;
}

// ---------------------------------------------------------------------------------------
// CSC -> CSR
// ---------------------------------------------------------------------------------------
__global__ void k_expand_cols(int n, const int64_t* __restrict__ col_ptr, int32_t* __restrict__ col_of) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) col_of[k] = j;
}

__global__ void k_iota64(int64_t nnz, int64_t* __restrict__ v) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[k] = k;
}

// row_ptr[r] = first k with keys[k] >= r (keys sorted ascending); each r written once.
__global__ void k_row_ptr_from_sorted(int64_t nnz, int m, const int32_t* __restrict__ keys,
                                      int64_t* __restrict__ row_ptr) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k <= nnz;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int lo = (k == 0) ? -1 : keys[k - 1];
        const int hi = (k == nnz) ? m : keys[k];
        for (int r = lo + 1; r <= hi; ++r) row_ptr[r] = k;
    }
}

template <typename T>
__global__ void k_gather(int64_t nnz, const int64_t* __restrict__ perm, const T* __restrict__ src,
                         T* __restrict__ dst) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[k] = src[perm[k]];
}

template <typename Ti, typename To>
__global__ void k_convert(int64_t n, const Ti* __restrict__ src, To* __restrict__ dst) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[k] = static_cast<To>(src[k]);
}

static unsigned grid_stride_blocks(int64_t work) { return grid_for(work, kThreads, 148 * 32); }

vajra_status build_csr(const DeviceLp& lp, Prepared& p, cudaStream_t st) {
    const int m = lp.m, n = lp.n;
    const int64_t nnz = lp.nnz;
    VJ_TRY(p.csr_ptr.alloc(static_cast<size_t>(m) + 1));
    VJ_TRY(p.csr_idx.alloc(static_cast<size_t>(nnz)));
    VJ_TRY(p.perm.alloc(static_cast<size_t>(nnz)));
    DeviceBuffer<int32_t> col_of, keys_out;
    DeviceBuffer<int64_t> iota;
    VJ_TRY(col_of.alloc(static_cast<size_t>(nnz)));
    VJ_TRY(keys_out.alloc(static_cast<size_t>(nnz)));
    VJ_TRY(iota.alloc(static_cast<size_t>(nnz)));
    if (n > 0) k_expand_cols<<<grid_for(n), kThreads, 0, st>>>(n, lp.col_ptr.get(), col_of.get());
    k_iota64<<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, iota.get());
    VJ_LAUNCH_CHECK();
    if (nnz > 0) {
        int end_bit = 1;
        while (end_bit < 31 && (1LL << end_bit) < m) ++end_bit;
        size_t temp_bytes = 0;
        VJ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, lp.row_idx.get(), keys_out.get(),
                                                iota.get(), p.perm.get(), nnz, 0, end_bit, st));
        DeviceBuffer<unsigned char> temp;
        VJ_TRY(temp.alloc(temp_bytes));
        VJ_CUDA(cub::DeviceRadixSort::SortPairs(temp.get(), temp_bytes, lp.row_idx.get(), keys_out.get(),
                                                iota.get(), p.perm.get(), nnz, 0, end_bit, st));
        k_gather<int32_t><<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, p.perm.get(), col_of.get(), p.csr_idx.get());
    }
    k_row_ptr_from_sorted<<<grid_stride_blocks(nnz + 1), kThreads, 0, st>>>(nnz, m, keys_out.get(), p.csr_ptr.get());
    VJ_LAUNCH_CHECK();
    note_launch(3 + (nnz > 0 ? 1 + 4 : 0));   // expand, iota, row_ptr; gather + radix-sort passes
    // Keep the temporaries alive until the work that reads them has run.
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

// ---------------------------------------------------------------------------------------
// scaling (Ruiz: src/linalg/scaling.cpp:7-153, in its evaluation order)
// ---------------------------------------------------------------------------------------
// The per-row / per-column l-inf norms, plus each block's max |1 - norm| over norms > 1e-11
// folded into the pass-wide maximum with one atomicMax per block on the bit pattern (for
// non-negative doubles the bit order is the value order, so the result is the exact maximum
// whatever the block order).
__global__ void k_col_inf(int n, const int64_t* __restrict__ col_ptr, const double* __restrict__ v,
                          double* __restrict__ col_inf, SetupState* sst) {
    if (sst->ruiz_done) return;
    __shared__ double red[32];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double e[1] = {0.0};
    if (j < n) {
        double mx = 0.0;
        for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
            const double a = fabs(v[k]);
            if (a > mx) mx = a;
        }
        col_inf[j] = mx;
        if (mx > kZeroDrop) e[0] = fabs(1.0 - mx);
    }
    block_reduce<OpMax, double, 1>(e, red);
    if (threadIdx.x == 0) atomicMax(&sst->col_err_bits, static_cast<unsigned long long>(__double_as_longlong(e[0])));
}

__global__ void k_row_inf(int m, const int64_t* __restrict__ csr_ptr, const int64_t* __restrict__ perm,
                          const double* __restrict__ v, double* __restrict__ row_inf, SetupState* sst) {
    if (sst->ruiz_done) return;
    __shared__ double red[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e[1] = {0.0};
    if (i < m) {
        double mx = 0.0;
        for (int64_t k = csr_ptr[i]; k < csr_ptr[i + 1]; ++k) {
            const double a = fabs(v[perm[k]]);
            if (a > mx) mx = a;
        }
        row_inf[i] = mx;
        if (mx > kZeroDrop) e[0] = fabs(1.0 - mx);
    }
    block_reduce<OpMax, double, 1>(e, red);
    if (threadIdx.x == 0) atomicMax(&sst->row_err_bits, static_cast<unsigned long long>(__double_as_longlong(e[0])));
}

// The Ruiz convergence test of the pass (scaling.cpp:54-70), then reset for the next pass.
__global__ void k_ruiz_err(double tol, SetupState* sst) {
    if (sst->ruiz_done) return;
    const double re = __longlong_as_double(static_cast<long long>(sst->row_err_bits));
    const double ce = __longlong_as_double(static_cast<long long>(sst->col_err_bits));
    sst->ruiz_row_err = re;
    sst->ruiz_col_err = ce;
    if (re <= tol && ce <= tol) sst->ruiz_done = 1;
    sst->row_err_bits = 0ull;
    sst->col_err_bits = 0ull;
}

// r = 1/sqrt(norm) (1 where norm <= 1e-11); cumulative scale *= r.
__global__ void k_scale_factors(int k_count, const double* __restrict__ norm, double* __restrict__ step,
                                double* __restrict__ scale, const SetupState* sst, int respect_done) {
    if (respect_done && sst->ruiz_done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k_count) return;
    const double r = (norm[i] > kZeroDrop) ? __ddiv_rn(1.0, __dsqrt_rn(norm[i])) : 1.0;
    step[i] = r;
    scale[i] = __dmul_rn(scale[i], r);
}

// A_ij *= r_i * c_j (scaling.cpp:92-100: the product of the two factors first), one entry
// per thread (col_of: the column of every CSC entry).
__global__ void k_scale_matrix(int64_t nnz, const int32_t* __restrict__ col_of, const int32_t* __restrict__ row_idx,
                               double* __restrict__ v, const double* __restrict__ r, const double* __restrict__ cs,
                               const SetupState* sst, int respect_done) {
    if (respect_done && sst->ruiz_done) return;
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[k] = __dmul_rn(v[k], __dmul_rn(r[row_idx[k]], cs[col_of[k]]));
}

// The Ruiz convergence test of one instance of a block-diagonal LP (one CTA each): the same
// maxima as k_row_inf / k_col_inf and k_ruiz_err over the instance's own rows and columns.
// An instance that passes keeps factor 1 from this pass on (sticky `inst_done`).
__global__ void __launch_bounds__(kThreads)
k_ruiz_err_inst(const int64_t* __restrict__ roff, const int64_t* __restrict__ coff, const double* __restrict__ row_inf,
                const double* __restrict__ col_inf, double tol, int* __restrict__ inst_done, const SetupState* sst) {
    if (sst->ruiz_done) return;
    const int inst = blockIdx.x;
    if (inst_done[inst]) return;
    __shared__ double red[2 * 32];   // block_reduce needs 32 slots per reduced value
    double e[2] = {0.0, 0.0};
    for (int64_t i = roff[inst] + threadIdx.x; i < roff[inst + 1]; i += blockDim.x)
        if (row_inf[i] > kZeroDrop) e[0] = fmax(e[0], fabs(1.0 - row_inf[i]));
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x)
        if (col_inf[j] > kZeroDrop) e[1] = fmax(e[1], fabs(1.0 - col_inf[j]));
    block_reduce<OpMax, double, 2>(e, red);
    if (threadIdx.x == 0 && e[0] <= tol && e[1] <= tol) inst_done[inst] = 1;
}

// k_scale_factors for a block-diagonal LP: factor 1 for the rows / columns of instances whose
// Ruiz test has passed.
__global__ void k_scale_factors_inst(int k_count, const double* __restrict__ norm, double* __restrict__ step,
                                     double* __restrict__ scale, const int* __restrict__ inst,
                                     const int* __restrict__ inst_done, const SetupState* sst) {
    if (sst->ruiz_done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k_count) return;
    if (inst_done[inst[i]]) { step[i] = 1.0; return; }
    const double r = (norm[i] > kZeroDrop) ? __ddiv_rn(1.0, __dsqrt_rn(norm[i])) : 1.0;
    step[i] = r;
    scale[i] = __dmul_rn(scale[i], r);
}

// Pock-Chambolle (alpha = 1) norms: sum |a| per column / per row, in storage order.
__global__ void k_col_abs_sum(int n, const int64_t* __restrict__ col_ptr, const double* __restrict__ v,
                              double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) s += fabs(v[k]);
    out[j] = s;
}

__global__ void k_row_abs_sum(int m, const int64_t* __restrict__ csr_ptr, const int64_t* __restrict__ perm,
                              const double* __restrict__ v, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double s = 0.0;
    for (int64_t k = csr_ptr[i]; k < csr_ptr[i + 1]; ++k) s += fabs(v[perm[k]]);
    out[i] = s;
}

// The cumulative factors rounded to the nearest power of two (in log2): scaling by them is
// exact in binary floating point, so a matrix whose values fit FP32 still fits it after
// scaling, and the scaled LP is the original one up to exact exponent shifts.
__global__ void k_round_pow2(int64_t n, double* __restrict__ s) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = s[k];
        if (v > 0.0 && isfinite(v)) s[k] = ldexp(1.0, static_cast<int>(rint(log2(v))));
    }
}

// Raises *flag when a scaled value does not survive a round trip through FP32.
__global__ void k_fp32_exact(int64_t nnz, const double* __restrict__ v, int* __restrict__ flag) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (static_cast<double>(static_cast<float>(v[k])) != v[k]) { *flag = 1; return; }
}

// c *= C; finite row bounds *= R; finite column bounds *= C^-1 (scaling.cpp:104-149).
__global__ void k_scale_vectors(int m, int n, double* c, double* rl, double* ru, double* cl, double* cu,
                                const double* __restrict__ rs, const double* __restrict__ cs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        c[i] = __dmul_rn(c[i], cs[i]);
        const double inv = __ddiv_rn(1.0, cs[i]);
        if (cl[i] > -kInf) cl[i] = __dmul_rn(cl[i], inv);
        if (cu[i] < kInf) cu[i] = __dmul_rn(cu[i], inv);
    }
    if (i < m) {
        if (rl[i] > -kInf) rl[i] = __dmul_rn(rl[i], rs[i]);
        if (ru[i] < kInf) ru[i] = __dmul_rn(ru[i], rs[i]);
    }
}

__global__ void k_fill(int64_t n, double* v, double val) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[k] = val;
}

__global__ void k_negate(int n, double* v) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) v[j] = -v[j];
}

vajra_status prepare_scaled(const DeviceLp& lp, Prepared& p, const ScalingOpts& o, SetupState* sst,
                            cudaStream_t st) {
    const int m = lp.m, n = lp.n;
    const int64_t nnz = lp.nnz;
    auto copy = [&](DeviceBuffer<double>& dst, const DeviceBuffer<double>& src, size_t cnt) -> vajra_status {
        VJ_TRY(dst.alloc(cnt));
        if (cnt) VJ_CUDA(cudaMemcpyAsync(dst.get(), src.get(), cnt * sizeof(double), cudaMemcpyDeviceToDevice, st));
        return VAJRA_OK;
    };
    VJ_TRY(copy(p.csc_val, lp.values, static_cast<size_t>(nnz)));
    VJ_TRY(copy(p.c, lp.c, static_cast<size_t>(n)));
    VJ_TRY(copy(p.col_lower, lp.col_lower, static_cast<size_t>(n)));
    VJ_TRY(copy(p.col_upper, lp.col_upper, static_cast<size_t>(n)));
    VJ_TRY(copy(p.row_lower, lp.row_lower, static_cast<size_t>(m)));
    VJ_TRY(copy(p.row_upper, lp.row_upper, static_cast<size_t>(m)));
    VJ_TRY(p.row_scale.alloc(static_cast<size_t>(m)));
    VJ_TRY(p.col_scale.alloc(static_cast<size_t>(n)));
    k_fill<<<grid_stride_blocks(m), kThreads, 0, st>>>(m, p.row_scale.get(), 1.0);
    k_fill<<<grid_stride_blocks(n), kThreads, 0, st>>>(n, p.col_scale.get(), 1.0);
    if (o.negate_c && n > 0) k_negate<<<grid_for(n), kThreads, 0, st>>>(n, p.c.get());
    VJ_LAUNCH_CHECK();
    note_launch(2 + (o.negate_c && n > 0 ? 1 : 0));
    p.scaled = false;
    if (o.enable && m > 0 && n > 0) {
        DeviceBuffer<double> row_norm, col_norm, r_k, c_k;
        VJ_TRY(row_norm.alloc(static_cast<size_t>(m)));
        VJ_TRY(col_norm.alloc(static_cast<size_t>(n)));
        VJ_TRY(r_k.alloc(static_cast<size_t>(m)));
        VJ_TRY(c_k.alloc(static_cast<size_t>(n)));
        DeviceBuffer<int32_t> col_of;
        VJ_TRY(col_of.alloc(static_cast<size_t>(nnz)));
        k_expand_cols<<<grid_for(n), kThreads, 0, st>>>(n, lp.col_ptr.get(), col_of.get());
        note_launch(1);
        VJ_CUDA(cudaMemsetAsync(sst, 0, sizeof(SetupState), st));
        const bool per_instance = o.instances > 0;
        DeviceBuffer<int> inst_done;
        if (per_instance) {
            VJ_TRY(inst_done.alloc(static_cast<size_t>(o.instances)));
            VJ_CUDA(cudaMemsetAsync(inst_done.get(), 0, sizeof(int) * o.instances, st));
        }
        for (int it = 0; it < o.ruiz_iterations; ++it) {
            k_col_inf<<<grid_for(n), kThreads, 0, st>>>(n, lp.col_ptr.get(), p.csc_val.get(), col_norm.get(), sst);
            k_row_inf<<<grid_for(m), kThreads, 0, st>>>(m, p.csr_ptr.get(), p.perm.get(), p.csc_val.get(),
                                                        row_norm.get(), sst);
            if (per_instance) {
                // per-instance tests first; the global one after it only ends the passes early
                // once every instance has passed (then every factor below would be 1)
                k_ruiz_err_inst<<<o.instances, kThreads, 0, st>>>(o.roff, o.coff, row_norm.get(), col_norm.get(),
                                                                   o.ruiz_tolerance, inst_done.get(), sst);
                k_ruiz_err<<<1, 1, 0, st>>>(o.ruiz_tolerance, sst);
                k_scale_factors_inst<<<grid_for(m), kThreads, 0, st>>>(m, row_norm.get(), r_k.get(), p.row_scale.get(),
                                                                       o.row_inst, inst_done.get(), sst);
                k_scale_factors_inst<<<grid_for(n), kThreads, 0, st>>>(n, col_norm.get(), c_k.get(), p.col_scale.get(),
                                                                       o.col_inst, inst_done.get(), sst);
                note_launch(1);
            } else {
                k_ruiz_err<<<1, 1, 0, st>>>(o.ruiz_tolerance, sst);
                k_scale_factors<<<grid_for(m), kThreads, 0, st>>>(m, row_norm.get(), r_k.get(), p.row_scale.get(), sst, 1);
                k_scale_factors<<<grid_for(n), kThreads, 0, st>>>(n, col_norm.get(), c_k.get(), p.col_scale.get(), sst, 1);
            }
            k_scale_matrix<<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, col_of.get(), lp.row_idx.get(),
                                                                          p.csc_val.get(), r_k.get(), c_k.get(), sst, 1);
            VJ_LAUNCH_CHECK();
            note_launch(6);
        }
        if (o.pock_chambolle) {
            k_col_abs_sum<<<grid_for(n), kThreads, 0, st>>>(n, lp.col_ptr.get(), p.csc_val.get(), col_norm.get());
            k_row_abs_sum<<<grid_for(m), kThreads, 0, st>>>(m, p.csr_ptr.get(), p.perm.get(), p.csc_val.get(), row_norm.get());
            k_scale_factors<<<grid_for(m), kThreads, 0, st>>>(m, row_norm.get(), r_k.get(), p.row_scale.get(), sst, 0);
            k_scale_factors<<<grid_for(n), kThreads, 0, st>>>(n, col_norm.get(), c_k.get(), p.col_scale.get(), sst, 0);
            k_scale_matrix<<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, col_of.get(), lp.row_idx.get(),
                                                                          p.csc_val.get(), r_k.get(), c_k.get(), sst, 0);
            VJ_LAUNCH_CHECK();
            note_launch(5);
        }
        if (o.pow2) {
            // round the cumulative factors and scale the original values by them once
            k_round_pow2<<<grid_stride_blocks(m), kThreads, 0, st>>>(m, p.row_scale.get());
            k_round_pow2<<<grid_stride_blocks(n), kThreads, 0, st>>>(n, p.col_scale.get());
            VJ_CUDA(cudaMemcpyAsync(p.csc_val.get(), lp.values.get(), sizeof(double) * nnz, cudaMemcpyDeviceToDevice, st));
            k_scale_matrix<<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, col_of.get(), lp.row_idx.get(),
                                                                          p.csc_val.get(), p.row_scale.get(),
                                                                          p.col_scale.get(), sst, 0);
            VJ_LAUNCH_CHECK();
            note_launch(3);
        }
        const int mx = m > n ? m : n;
        k_scale_vectors<<<grid_for(mx), kThreads, 0, st>>>(m, n, p.c.get(), p.row_lower.get(), p.row_upper.get(),
                                                           p.col_lower.get(), p.col_upper.get(),
                                                           p.row_scale.get(), p.col_scale.get());
        VJ_LAUNCH_CHECK();
        note_launch(1);
        VJ_CUDA(cudaStreamSynchronize(st));   // temporaries above go out of scope
        p.scaled = true;
    }
    VJ_TRY(p.csr_val.alloc(static_cast<size_t>(nnz)));
    VJ_TRY(p.csr_val_orig.alloc(static_cast<size_t>(nnz)));
    if (nnz > 0) {
        k_gather<double><<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, p.perm.get(), p.csc_val.get(), p.csr_val.get());
        k_gather<double><<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, p.perm.get(), lp.values.get(), p.csr_val_orig.get());
        VJ_LAUNCH_CHECK();
        note_launch(2);
    }
    // CSR views: A over csr_*, A^T over the raw CSC structure.
    p.a.rows = m; p.a.cols = n; p.a.nnz = nnz; p.a.ptr = p.csr_ptr.get(); p.a.idx = p.csr_idx.get();
    p.at.rows = n; p.at.cols = m; p.at.nnz = nnz; p.at.ptr = lp.col_ptr.get(); p.at.idx = lp.row_idx.get();
    return VAJRA_OK;
}

vajra_status values_fit_fp32(const Prepared& p, int64_t nnz, bool* exact, cudaStream_t st) {
    *exact = false;
    if (nnz <= 0) { *exact = true; return VAJRA_OK; }
    DeviceBuffer<int> flag;
    VJ_TRY(flag.alloc(1));
    VJ_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), st));
    k_fp32_exact<<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, p.csc_val.get(), flag.get());
    VJ_LAUNCH_CHECK();
    note_launch(1);
    int h = 1;
    VJ_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    *exact = h == 0;
    return VAJRA_OK;
}

vajra_status make_f32_values(Prepared& p, int64_t nnz, cudaStream_t st) {
    VJ_TRY(p.csc_val32.alloc(static_cast<size_t>(nnz)));
    VJ_TRY(p.csr_val32.alloc(static_cast<size_t>(nnz)));
    if (nnz > 0) {
        k_convert<double, float><<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, p.csc_val.get(), p.csc_val32.get());
        k_convert<double, float><<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, p.csr_val.get(), p.csr_val32.get());
        VJ_LAUNCH_CHECK();
        note_launch(2);
    }
    return VAJRA_OK;
}

// ---------------------------------------------------------------------------------------
// power iteration (src/solvers/pdhg/pdhg.cpp:11-56)
// ---------------------------------------------------------------------------------------
struct EpiStoreUnlessDone {
    double* out;
    const int* done;
    __device__ bool active() const { return *done == 0; }
    __device__ void operator()(int row, double s) const { out[row] = s; }
};

// Sequential: the reference sums u_j^2 in index order.
__global__ void k_power_step_exact(int n, const double* __restrict__ u, double tol, SetupState* sst) {
    if (sst->power_done) return;
    double norm_sq = 0.0;
    for (int j = 0; j < n; ++j) norm_sq = __dadd_rn(norm_sq, __dmul_rn(u[j], u[j]));
    const double norm = __dsqrt_rn(norm_sq);
    const int it = sst->power_iter;
    if (norm < 1e-15 || isnan(norm) || isinf(norm)) {
        sst->spectral_norm = (sst->lambda > 1e-6) ? __dsqrt_rn(sst->lambda) : 1e-3;
        sst->power_done = 2;   // 2: result already final
        return;
    }
    sst->lambda = norm;
    if (it > 0 && fabs(__dsub_rn(norm, sst->lambda_prev)) <= __dmul_rn(tol, norm)) {
        sst->power_done = 1;
        return;
    }
    sst->lambda_prev = norm;
    sst->inv_norm = __ddiv_rn(1.0, norm);
    sst->power_iter = it + 1;
}

__global__ void k_power_scale(int n, const double* __restrict__ u, double* __restrict__ v, const SetupState* sst) {
    if (sst->power_done) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) v[j] = __dmul_rn(u[j], sst->inv_norm);
}

__global__ void k_power_final(SetupState* sst) {
    if (sst->power_done == 2) return;
    const double s = __dsqrt_rn(sst->lambda);
    sst->spectral_norm = (s > 1e-12) ? s : 1e-6;
}

static vajra_status power_init(int n, DeviceBuffer<double>& v, DeviceBuffer<double>& w, DeviceBuffer<double>& u,
                               int m, SetupState* sst, cudaStream_t st) {
    VJ_TRY(v.alloc(static_cast<size_t>(n)));
    VJ_TRY(w.alloc(static_cast<size_t>(m)));
    VJ_TRY(u.alloc(static_cast<size_t>(n)));
    const double v0 = 1.0 / std::sqrt(static_cast<double>(n));
    k_fill<<<grid_stride_blocks(n), kThreads, 0, st>>>(n, v.get(), v0);
    SetupState init{};
    init.lambda = 1.0;
    VJ_CUDA(cudaMemcpyAsync(sst, &init, sizeof(SetupState), cudaMemcpyHostToDevice, st));
    VJ_CUDA(cudaStreamSynchronize(st));   // `init` lives on this stack frame
    return VAJRA_OK;
}

vajra_status spectral_norm_exact(const Prepared& p, int m, int n, int max_iter, double tol, SetupState* sst,
                                 cudaStream_t st) {
    DeviceBuffer<double> v, w, u;
    VJ_TRY(power_init(n, v, w, u, m, sst, st));
    const int* done = &sst->power_done;
    for (int it = 0; it < max_iter; ++it) {
        launch_spmv_exact<double, true>(p.a, p.csr_val.get(), v.get(), EpiStoreUnlessDone{w.get(), done}, st);
        launch_spmv_exact<double, false>(p.at, p.csc_val.get(), w.get(), EpiStoreUnlessDone{u.get(), done}, st);
        k_power_step_exact<<<1, 1, 0, st>>>(n, u.get(), tol, sst);
        k_power_scale<<<grid_for(n), kThreads, 0, st>>>(n, u.get(), v.get(), sst);
        VJ_LAUNCH_CHECK();
        note_launch(2);
    }
    k_power_final<<<1, 1, 0, st>>>(sst);
    VJ_LAUNCH_CHECK();
    note_launch(2);   // final + the initial fill
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

// Fast form: deterministic two-stage sum of squares.
__global__ void k_sumsq_partial(int n, const double* __restrict__ u, double* __restrict__ part, const SetupState* sst) {
    if (sst->power_done) return;
    __shared__ double red[32];
    double v[1] = {0.0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) v[0] += u[j] * u[j];
    block_reduce<OpSum, double, 1>(v, red);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void k_power_step_fast(int nparts, const double* __restrict__ part, double tol, SetupState* sst) {
    if (sst->power_done) return;
    __shared__ double red[32];
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) v[0] += part[b];
    block_reduce<OpSum, double, 1>(v, red);
    if (threadIdx.x != 0) return;
    const double norm = sqrt(v[0]);
    const int it = sst->power_iter;
    if (norm < 1e-15 || isnan(norm) || isinf(norm)) {
        sst->spectral_norm = (sst->lambda > 1e-6) ? sqrt(sst->lambda) : 1e-3;
        sst->power_done = 2;
        return;
    }
    sst->lambda = norm;
    if (it > 0 && fabs(norm - sst->lambda_prev) <= tol * norm) { sst->power_done = 1; return; }
    sst->lambda_prev = norm;
    sst->inv_norm = 1.0 / norm;
    sst->power_iter = it + 1;
}

vajra_status spectral_norm_fast(const Prepared& p, int m, int n, int max_iter, double tol, SetupState* sst,
                                cudaStream_t st) {
    DeviceBuffer<double> v, w, u, part;
    VJ_TRY(power_init(n, v, w, u, m, sst, st));
    const int nparts = 148 * 4;
    VJ_TRY(part.alloc(nparts));
    const int* done = &sst->power_done;
    // Once the estimate has converged every later launch returns at once, so the loop stops at
    // the first look (every kPowerLook rounds) that finds the flag set: the same result without
    // the remaining launches (about 5 us each on a small LP, where 100 rounds took 2 ms).
    constexpr int kPowerLook = 16;
    for (int it = 0; it < max_iter; ++it) {
        if (it > 0 && it % kPowerLook == 0) {
            int flag = 0;
            VJ_CUDA(cudaMemcpyAsync(&flag, done, sizeof(int), cudaMemcpyDeviceToHost, st));
            VJ_CUDA(cudaStreamSynchronize(st));
            if (flag) break;
        }
        // sliced-ELL copies, where the set-up built them, are the faster form of both SpMVs
        if (p.a.sell_off)
            launch_sell<double, double, double>(p.a, p.csr_val.get(), p.sell_a.val64.get(), v.get(),
                                                EpiStoreUnlessDone{w.get(), done}, st);
        else
            launch_spmv<double, double>(p.a, p.csr_val.get(), v.get(), EpiStoreUnlessDone{w.get(), done}, st);
        if (p.at.sell_off)
            launch_sell<double, double, double>(p.at, p.csc_val.get(), p.sell_at.val64.get(), w.get(),
                                                EpiStoreUnlessDone{u.get(), done}, st);
        else
            launch_spmv<double, double>(p.at, p.csc_val.get(), w.get(), EpiStoreUnlessDone{u.get(), done}, st);
        k_sumsq_partial<<<nparts, kThreads, 0, st>>>(n, u.get(), part.get(), sst);
        k_power_step_fast<<<1, kThreads, 0, st>>>(nparts, part.get(), tol, sst);
        k_power_scale<<<grid_for(n), kThreads, 0, st>>>(n, u.get(), v.get(), sst);
        VJ_LAUNCH_CHECK();
        note_launch(3);
    }
    k_power_final<<<1, 1, 0, st>>>(sst);
    VJ_LAUNCH_CHECK();
    note_launch(2);
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

// ---------------------------------------------------------------------------------------
// SpMV plan: group size from the mean row length, long-row lists
// ---------------------------------------------------------------------------------------
__global__ void k_collect_long(int rows, const int64_t* __restrict__ ptr, int64_t long_len,
                               int32_t* __restrict__ out, int* __restrict__ count) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    if (ptr[r + 1] - ptr[r] > long_len) out[atomicAdd(count, 1)] = r;
}

static int default_group(double mean_len) {
    int g = 1;
    while (g < 32 && g * 2 <= mean_len) g *= 2;   // ~2 products per lane
    return g;
}

// block_rows[b] = first row whose first entry is at or after b * tile (binary search over
// ptr[0..rows]); block_rows[nb] = rows.
__global__ void k_rowblock_partition(int rows, const int64_t* __restrict__ ptr, int64_t tile, int nb,
                                     int32_t* __restrict__ block_rows) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nb) return;
    if (b == nb) { block_rows[b] = rows; return; }
    const int64_t target = static_cast<int64_t>(b) * tile;
    int lo = 0, hi = rows;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (ptr[mid] < target) lo = mid + 1; else hi = mid;
    }
    block_rows[b] = lo;
}

__global__ void k_tile_desc(int nb, const int64_t* __restrict__ ptr, const int32_t* __restrict__ block_rows,
                            int64_t tile, TileDesc* __restrict__ tiles) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int r0 = block_rows[b], r1 = block_rows[b + 1];
    int r_end = r1;
    if (r1 > r0 && ptr[r1] - ptr[r1 - 1] > tile) r_end = r1 - 1;
    TileDesc d;
    d.r0 = r0;
    d.r_end = r_end > r0 ? r_end : r0;
    d.e0 = r_end > r0 ? ptr[r0] : 0;
    d.e1 = r_end > r0 ? ptr[r_end] : 0;
    tiles[b] = d;
}

static vajra_status collect_long(const CsrView& v, int64_t long_len, DeviceBuffer<int32_t>& list, int* count,
                                 cudaStream_t st) {
    VJ_TRY(list.alloc(static_cast<size_t>(v.rows > 0 ? v.rows : 1)));
    DeviceBuffer<int> cnt;
    VJ_TRY(cnt.alloc(1));
    VJ_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int), st));
    if (v.rows > 0) k_collect_long<<<grid_for(v.rows), kThreads, 0, st>>>(v.rows, v.ptr, long_len, list.get(), cnt.get());
    VJ_LAUNCH_CHECK();
    note_launch(v.rows > 0 ? 1 : 0);
    int h = 0;
    VJ_CUDA(cudaMemcpyAsync(&h, cnt.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    *count = h;
    return VAJRA_OK;
}

vajra_status build_row_partition(const CsrView& v, int64_t tile, DeviceBuffer<int32_t>& blocks,
                                 DeviceBuffer<TileDesc>& tiles, DeviceBuffer<int32_t>& long_rows, int* nb,
                                 int* n_long, cudaStream_t st) {
    int64_t nb64 = (v.nnz + tile - 1) / tile;
    if (nb64 < 1) nb64 = 1;
    if (nb64 > (1LL << 30)) { set_error("matrix too large for the row-block partition"); return VAJRA_ERR_INVALID_ARGUMENT; }
    *nb = static_cast<int>(nb64);
    VJ_TRY(blocks.alloc(static_cast<size_t>(*nb) + 1));
    k_rowblock_partition<<<grid_for(static_cast<int64_t>(*nb) + 1), kThreads, 0, st>>>(v.rows, v.ptr, tile, *nb,
                                                                                       blocks.get());
    VJ_LAUNCH_CHECK();
    VJ_TRY(tiles.alloc(static_cast<size_t>(*nb)));
    k_tile_desc<<<grid_for(*nb), kThreads, 0, st>>>(*nb, v.ptr, blocks.get(), tile, tiles.get());
    VJ_LAUNCH_CHECK();
    note_launch(2);
    return collect_long(v, tile, long_rows, n_long, st);
}

static vajra_status plan_one(CsrView& v, DeviceBuffer<int32_t>& list, DeviceBuffer<int32_t>& blocks,
                             DeviceBuffer<TileDesc>& tiles, DeviceBuffer<int32_t>& rb_list, cudaStream_t st) {
    const double mean = v.rows > 0 ? static_cast<double>(v.nnz) / v.rows : 0.0;
    v.group = default_group(mean);
    int64_t long_len = static_cast<int64_t>(8.0 * mean);
    if (long_len < 256) long_len = 256;
    v.long_len = long_len;
    VJ_TRY(collect_long(v, long_len, list, &v.n_long, st));
    v.long_rows = list.get();
    VJ_TRY(build_row_partition(v, kTile, blocks, tiles, rb_list, &v.nb, &v.rb_n_long, st));
    v.block_rows = blocks.get();
    v.tiles = tiles.get();
    v.rb_long_rows = rb_list.get();
    return VAJRA_OK;
}

vajra_status plan_spmv(const DeviceLp& lp, Prepared& p, cudaStream_t st) {
    (void)lp;
    VJ_TRY(plan_one(p.a, p.long_rows_a, p.rb_blocks_a, p.rb_tiles_a, p.rb_long_a, st));
    VJ_TRY(plan_one(p.at, p.long_rows_at, p.rb_blocks_at, p.rb_tiles_at, p.rb_long_at, st));
    return VAJRA_OK;
}

// ---------------------------------------------------------------------------------------
// degree ordering
// ---------------------------------------------------------------------------------------
// Sort keys: descending entry count as an ascending unsigned key (the stable radix sort keeps
// equal counts in index order).
__global__ void k_col_count_keys(int n, const int64_t* __restrict__ col_ptr, uint32_t* __restrict__ keys,
                                 int32_t* __restrict__ idx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    keys[j] = 0xffffffffu - static_cast<uint32_t>(col_ptr[j + 1] - col_ptr[j]);
    idx[j] = j;
}

__global__ void k_row_counts(int64_t nnz, const int32_t* __restrict__ row_idx, uint32_t* __restrict__ counts) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        atomicAdd(&counts[row_idx[k]], 1u);
}

__global__ void k_row_count_keys(int m, uint32_t* __restrict__ keys, int32_t* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    keys[i] = 0xffffffffu - keys[i];
    idx[i] = i;
}

__global__ void k_invert(int count, const int32_t* __restrict__ order, int32_t* __restrict__ inv) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) inv[order[k]] = k;
}

// New column pointers: counts in the new order, then a running sum (one block).
__global__ void k_ordered_counts(int n, const int64_t* __restrict__ col_ptr, const int32_t* __restrict__ col_order,
                                 int64_t* __restrict__ counts) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) counts[k] = col_ptr[col_order[k] + 1] - col_ptr[col_order[k]];
}

// One warp per new column: its entries in the original order, rows renumbered.
__global__ void k_copy_columns(int n, const int64_t* __restrict__ src_ptr, const int32_t* __restrict__ src_row,
                               const double* __restrict__ src_val, const int32_t* __restrict__ col_order,
                               const int32_t* __restrict__ row_inv, const int64_t* __restrict__ dst_ptr,
                               int32_t* __restrict__ dst_row, double* __restrict__ dst_val) {
    const int64_t w = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const int j = col_order[w];
    const int64_t s = src_ptr[j], len = src_ptr[j + 1] - s, d = dst_ptr[w];
    for (int64_t t = lane; t < len; t += 32) {
        dst_row[d + t] = row_inv[src_row[s + t]];
        dst_val[d + t] = src_val[s + t];
    }
}

template <typename T>
__global__ void k_take(int count, const int32_t* __restrict__ order, const T* __restrict__ src, T* __restrict__ dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[k] = src[order[k]];
}

template <typename T>
__global__ void k_put(int count, const int32_t* __restrict__ order, const T* __restrict__ src, T* __restrict__ dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[order[k]] = src[k];
}

static vajra_status sort_order(int count, const uint32_t* keys, DeviceBuffer<int32_t>& idx,
                               DeviceBuffer<int32_t>& order, cudaStream_t st) {
    DeviceBuffer<uint32_t> keys_out;
    VJ_TRY(keys_out.alloc(static_cast<size_t>(count)));
    size_t temp_bytes = 0;
    VJ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_out.get(), idx.get(), order.get(), count,
                                            0, 32, st));
    DeviceBuffer<unsigned char> temp;
    VJ_TRY(temp.alloc(temp_bytes));
    VJ_CUDA(cub::DeviceRadixSort::SortPairs(temp.get(), temp_bytes, keys, keys_out.get(), idx.get(), order.get(),
                                            count, 0, 32, st));
    note_launch(4);
    VJ_CUDA(cudaStreamSynchronize(st));   // temporaries die here
    return VAJRA_OK;
}

vajra_status order_by_degree(const DeviceLp& src, DeviceLp& dst, LpOrder& ord, cudaStream_t st) {
    const int m = src.m, n = src.n;
    const int64_t nnz = src.nnz;
    dst.m = m;
    dst.n = n;
    dst.nnz = nnz;
    dst.sense = src.sense;
    dst.objective_offset = src.objective_offset;
    VJ_TRY(ord.col_order.alloc(static_cast<size_t>(n)));
    VJ_TRY(ord.row_order.alloc(static_cast<size_t>(m)));
    DeviceBuffer<uint32_t> keys;
    DeviceBuffer<int32_t> idx, row_inv;
    // columns
    VJ_TRY(keys.alloc(static_cast<size_t>(n)));
    VJ_TRY(idx.alloc(static_cast<size_t>(n)));
    if (n > 0) {
        k_col_count_keys<<<grid_for(n), kThreads, 0, st>>>(n, src.col_ptr.get(), keys.get(), idx.get());
        VJ_LAUNCH_CHECK();
        note_launch(1);
        VJ_TRY(sort_order(n, keys.get(), idx, ord.col_order, st));
    }
    // rows
    VJ_TRY(keys.alloc(static_cast<size_t>(m)));
    VJ_TRY(idx.alloc(static_cast<size_t>(m)));
    VJ_TRY(row_inv.alloc(static_cast<size_t>(m)));
    if (m > 0) {
        VJ_CUDA(cudaMemsetAsync(keys.get(), 0, sizeof(uint32_t) * m, st));
        if (nnz > 0) k_row_counts<<<grid_stride_blocks(nnz), kThreads, 0, st>>>(nnz, src.row_idx.get(), keys.get());
        k_row_count_keys<<<grid_for(m), kThreads, 0, st>>>(m, keys.get(), idx.get());
        VJ_LAUNCH_CHECK();
        note_launch(nnz > 0 ? 2 : 1);
        VJ_TRY(sort_order(m, keys.get(), idx, ord.row_order, st));
        k_invert<<<grid_for(m), kThreads, 0, st>>>(m, ord.row_order.get(), row_inv.get());
        VJ_LAUNCH_CHECK();
        note_launch(1);
    }
    // matrix: new column pointers, then the columns' entries with renumbered rows
    VJ_TRY(dst.col_ptr.alloc(static_cast<size_t>(n) + 1));
    VJ_TRY(dst.row_idx.alloc(static_cast<size_t>(nnz)));
    VJ_TRY(dst.values.alloc(static_cast<size_t>(nnz)));
    {
        DeviceBuffer<int64_t> counts;
        VJ_TRY(counts.alloc(static_cast<size_t>(n) + 1));
        VJ_CUDA(cudaMemsetAsync(counts.get(), 0, sizeof(int64_t) * (static_cast<size_t>(n) + 1), st));
        if (n > 0) {
            k_ordered_counts<<<grid_for(n), kThreads, 0, st>>>(n, src.col_ptr.get(), ord.col_order.get(), counts.get());
            VJ_LAUNCH_CHECK();
            note_launch(1);
        }
        // exclusive sum over n + 1 slots (the last count is 0): col_ptr[0] = 0, col_ptr[n] = nnz
        size_t temp_bytes = 0;
        VJ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, counts.get(), dst.col_ptr.get(), n + 1, st));
        DeviceBuffer<unsigned char> temp;
        VJ_TRY(temp.alloc(temp_bytes));
        VJ_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), temp_bytes, counts.get(), dst.col_ptr.get(), n + 1, st));
        note_launch(2);
        if (n > 0 && nnz > 0) {
            k_copy_columns<<<grid_for(static_cast<int64_t>(n) * 32), kThreads, 0, st>>>(
                n, src.col_ptr.get(), src.row_idx.get(), src.values.get(), ord.col_order.get(), row_inv.get(),
                dst.col_ptr.get(), dst.row_idx.get(), dst.values.get());
            VJ_LAUNCH_CHECK();
            note_launch(1);
        }
        VJ_CUDA(cudaStreamSynchronize(st));   // temporaries die here
    }
    // vectors
    VJ_TRY(dst.c.alloc(static_cast<size_t>(n)));
    VJ_TRY(dst.col_lower.alloc(static_cast<size_t>(n)));
    VJ_TRY(dst.col_upper.alloc(static_cast<size_t>(n)));
    VJ_TRY(dst.row_lower.alloc(static_cast<size_t>(m)));
    VJ_TRY(dst.row_upper.alloc(static_cast<size_t>(m)));
    if (n > 0) {
        k_take<double><<<grid_for(n), kThreads, 0, st>>>(n, ord.col_order.get(), src.c.get(), dst.c.get());
        k_take<double><<<grid_for(n), kThreads, 0, st>>>(n, ord.col_order.get(), src.col_lower.get(), dst.col_lower.get());
        k_take<double><<<grid_for(n), kThreads, 0, st>>>(n, ord.col_order.get(), src.col_upper.get(), dst.col_upper.get());
        note_launch(3);
    }
    if (m > 0) {
        k_take<double><<<grid_for(m), kThreads, 0, st>>>(m, ord.row_order.get(), src.row_lower.get(), dst.row_lower.get());
        k_take<double><<<grid_for(m), kThreads, 0, st>>>(m, ord.row_order.get(), src.row_upper.get(), dst.row_upper.get());
        note_launch(2);
    }
    VJ_LAUNCH_CHECK();
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

// ---------------------------------------------------------------------------------------
// sliced ELL
// ---------------------------------------------------------------------------------------
// is_long / is_vlong: rows of kSellWidth..kSellCtaRow entries / above (0 for sliced rows),
// and the one-byte length the slices read (kSellLong for the listed rows).
__global__ void k_sell_classify(int rows, const int64_t* __restrict__ ptr, uint8_t* __restrict__ is_long,
                                uint8_t* __restrict__ is_vlong, uint8_t* __restrict__ len8) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int64_t len = ptr[r + 1] - ptr[r];
    is_long[r] = (len > kSellWidth && len <= kSellCtaRow) ? 1 : 0;
    is_vlong[r] = len > kSellCtaRow ? 1 : 0;
    len8[r] = len > kSellWidth ? kSellLong : static_cast<uint8_t>(len);
}

// Slice s holds 32 x (its longest sliced row's length, rounded up to kSellPack) slots;
// sizes[slices] = 0 closes the scan.
__global__ void k_sell_sizes(int rows, int slices, const int64_t* __restrict__ ptr, int64_t* __restrict__ sizes) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > slices) return;
    if (s == slices) { sizes[s] = 0; return; }
    int64_t w = 0;
    const int r1 = 32 * s + 32 < rows ? 32 * s + 32 : rows;
    for (int r = 32 * s; r < r1; ++r) {
        const int64_t len = ptr[r + 1] - ptr[r];
        if (len <= kSellWidth && len > w) w = len;
    }
    sizes[s] = 32 * ((w + kSellPack - 1) / kSellPack * kSellPack);
}

// One thread per sliced row: its entries to their slots (kSellPack entries of a row side by
// side, then the next lane's).
__global__ void k_sell_fill(int rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const double* __restrict__ v64, const float* __restrict__ v32,
                            const int64_t* __restrict__ off, int32_t* __restrict__ sidx, double* __restrict__ s64,
                            float* __restrict__ s32) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int64_t b = ptr[r], len = ptr[r + 1] - b;
    if (len > kSellWidth) return;
    const int s = r >> 5, lane = r & 31;
    const int64_t o = off[s] + kSellPack * lane;
    for (int64_t k = 0; k < len; ++k) {
        const int64_t q = o + 32 * kSellPack * (k / kSellPack) + k % kSellPack;
        sidx[q] = idx[b + k];
        s64[q] = v64[b + k];
        if (v32) s32[q] = v32[b + k];
    }
}

// The rows whose flag is set, in row order.
static vajra_status select_rows(int rows, const uint8_t* flags, DeviceBuffer<int32_t>& out, int* count, cudaStream_t st) {
    DeviceBuffer<int> n_sel;
    VJ_TRY(n_sel.alloc(1));
    VJ_TRY(out.alloc(static_cast<size_t>(rows)));
    thrust::counting_iterator<int32_t> first(0);
    size_t temp_bytes = 0;
    VJ_CUDA(cub::DeviceSelect::Flagged(nullptr, temp_bytes, first, flags, out.get(), n_sel.get(), rows, st));
    DeviceBuffer<unsigned char> temp;
    VJ_TRY(temp.alloc(temp_bytes));
    VJ_CUDA(cub::DeviceSelect::Flagged(temp.get(), temp_bytes, first, flags, out.get(), n_sel.get(), rows, st));
    note_launch(1);
    VJ_CUDA(cudaMemcpyAsync(count, n_sel.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));   // temporaries die here
    return VAJRA_OK;
}

vajra_status build_sell(CsrView& v, const double* val64, const float* val32, SellData& out, cudaStream_t st) {
    v.sell_off = nullptr;
    v.sell_idx = nullptr;
    v.sell_len = nullptr;
    v.sell_long_rows = v.sell_vlong_rows = nullptr;
    v.sell_slices = v.sell_n_long = v.sell_n_vlong = 0;
    if (v.rows <= 0) return VAJRA_OK;
    int n_long = 0, n_vlong = 0;
    {
        DeviceBuffer<uint8_t> is_long, is_vlong;
        VJ_TRY(is_long.alloc(static_cast<size_t>(v.rows)));
        VJ_TRY(is_vlong.alloc(static_cast<size_t>(v.rows)));
        VJ_TRY(out.len.alloc(static_cast<size_t>(v.rows)));
        k_sell_classify<<<grid_for(v.rows), kThreads, 0, st>>>(v.rows, v.ptr, is_long.get(), is_vlong.get(),
                                                               out.len.get());
        VJ_LAUNCH_CHECK();
        note_launch(1);
        VJ_TRY(select_rows(v.rows, is_long.get(), out.long_rows, &n_long, st));
        VJ_TRY(select_rows(v.rows, is_vlong.get(), out.vlong_rows, &n_vlong, st));
    }
    const int slices = (v.rows + 31) / 32;
    VJ_TRY(out.off.alloc(static_cast<size_t>(slices) + 1));
    {
        DeviceBuffer<int64_t> sizes;
        VJ_TRY(sizes.alloc(static_cast<size_t>(slices) + 1));
        k_sell_sizes<<<grid_for(static_cast<int64_t>(slices) + 1), kThreads, 0, st>>>(v.rows, slices, v.ptr, sizes.get());
        VJ_LAUNCH_CHECK();
        size_t temp_bytes = 0;
        VJ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, sizes.get(), out.off.get(), slices + 1, st));
        DeviceBuffer<unsigned char> temp;
        VJ_TRY(temp.alloc(temp_bytes));
        VJ_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), temp_bytes, sizes.get(), out.off.get(), slices + 1, st));
        note_launch(3);
        VJ_CUDA(cudaStreamSynchronize(st));   // temporaries die here
    }
    int64_t total = 0;
    VJ_CUDA(cudaMemcpyAsync(&total, out.off.get() + slices, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    VJ_CUDA(cudaStreamSynchronize(st));
    VJ_TRY(out.idx.alloc(static_cast<size_t>(total)));
    VJ_TRY(out.val64.alloc(static_cast<size_t>(total)));
    if (val32) VJ_TRY(out.val32.alloc(static_cast<size_t>(total)));
    k_sell_fill<<<grid_for(v.rows), kThreads, 0, st>>>(v.rows, v.ptr, v.idx, val64, val32, out.off.get(), out.idx.get(),
                                                       out.val64.get(), val32 ? out.val32.get() : nullptr);
    VJ_LAUNCH_CHECK();
    note_launch(1);
    v.sell_off = out.off.get();
    v.sell_idx = out.idx.get();
    v.sell_len = out.len.get();
    v.sell_slices = slices;
    v.sell_long_rows = out.long_rows.get();
    v.sell_n_long = n_long;
    v.sell_vlong_rows = out.vlong_rows.get();
    v.sell_n_vlong = n_vlong;
    return VAJRA_OK;
}

vajra_status unorder(int count, const int32_t* order, const double* src, double* dst, cudaStream_t st) {
    if (count <= 0) return VAJRA_OK;
    k_put<double><<<grid_for(count), kThreads, 0, st>>>(count, order, src, dst);
    VJ_LAUNCH_CHECK();
    note_launch(1);
    return VAJRA_OK;
}

}  // namespace vajra
