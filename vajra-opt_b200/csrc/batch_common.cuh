// Shared pieces of the multi-instance paths (batched solver, unrolled adjoint): host-side
// block-diagonal packing of many LPs into one, instance maps, and the batched power
// iteration that gives every instance its own ||A_i||_2 estimate.
#pragma once

#include <cmath>
#include <cstring>
#include <vector>

#include "problem.cuh"

namespace vajra {

// Host arrays of diag(A_1, ..., A_B) in CSC, with every instance's rows / columns / entries
// at offsets roff / coff / zoff.  c_min is c negated for maximisation instances.
struct PackedHost {
    int count = 0;
    int m = 0, n = 0;
    int64_t nnz = 0;
    std::vector<int64_t> roff, coff, zoff, col_ptr;
    std::vector<int32_t> row_idx;
    std::vector<double> values, c, c_min, cl, cu, rl, ru, offsets;
    std::vector<int> sense;
    vajra_lp view{};   // points into the vectors above
};

inline vajra_status pack_lps(int count, const vajra_lp* lps, PackedHost& P) {
    P.count = count;
    P.roff.assign(count + 1, 0);
    P.coff.assign(count + 1, 0);
    P.zoff.assign(count + 1, 0);
    for (int i = 0; i < count; ++i) {
        P.roff[i + 1] = P.roff[i] + lps[i].num_rows;
        P.coff[i + 1] = P.coff[i] + lps[i].num_cols;
        P.zoff[i + 1] = P.zoff[i] + lps[i].nnz;
    }
    if (P.roff[count] >= (1LL << 31) || P.coff[count] >= (1LL << 31)) {
        set_error("packed problem exceeds 2^31 rows or columns");
        return VAJRA_ERR_INVALID_ARGUMENT;
    }
    P.m = static_cast<int>(P.roff[count]);
    P.n = static_cast<int>(P.coff[count]);
    P.nnz = P.zoff[count];
    P.col_ptr.assign(static_cast<size_t>(P.n) + 1, 0);
    P.row_idx.resize(static_cast<size_t>(P.nnz));
    P.values.resize(static_cast<size_t>(P.nnz));
    P.c.resize(P.n); P.cl.resize(P.n); P.cu.resize(P.n);
    P.rl.resize(P.m); P.ru.resize(P.m);
    P.offsets.resize(count);
    P.sense.resize(count);
    for (int i = 0; i < count; ++i) {
        const vajra_lp& L = lps[i];
        const int64_t c0 = P.coff[i], r0 = P.roff[i], z0 = P.zoff[i];
        for (int j = 0; j < L.num_cols; ++j) P.col_ptr[c0 + j] = z0 + L.col_ptr[j];
        for (int64_t k = 0; k < L.nnz; ++k) P.row_idx[z0 + k] = static_cast<int32_t>(r0 + L.row_idx[k]);
        if (L.nnz) std::memcpy(&P.values[z0], L.values, sizeof(double) * L.nnz);
        if (L.num_cols) {
            std::memcpy(&P.c[c0], L.c, sizeof(double) * L.num_cols);
            std::memcpy(&P.cl[c0], L.col_lower, sizeof(double) * L.num_cols);
            std::memcpy(&P.cu[c0], L.col_upper, sizeof(double) * L.num_cols);
        }
        if (L.num_rows) {
            std::memcpy(&P.rl[r0], L.row_lower, sizeof(double) * L.num_rows);
            std::memcpy(&P.ru[r0], L.row_upper, sizeof(double) * L.num_rows);
        }
        P.sense[i] = L.sense;
        P.offsets[i] = L.objective_offset;
    }
    P.col_ptr[P.n] = P.nnz;
    P.c_min = P.c;
    for (int i = 0; i < count; ++i)
        if (P.sense[i]) for (int64_t j = P.coff[i]; j < P.coff[i + 1]; ++j) P.c_min[j] = -P.c_min[j];
    P.view = vajra_lp{};
    P.view.num_rows = P.m; P.view.num_cols = P.n; P.view.nnz = P.nnz;
    P.view.col_ptr = P.col_ptr.data(); P.view.row_idx = P.row_idx.data(); P.view.values = P.values.data();
    P.view.c = P.c.data(); P.view.col_lower = P.cl.data(); P.view.col_upper = P.cu.data();
    P.view.row_lower = P.rl.data(); P.view.row_upper = P.ru.data();
    return VAJRA_OK;
}

template <typename T>
inline vajra_status upload_vec(DeviceBuffer<T>& d, const std::vector<T>& h, cudaStream_t st) {
    VJ_TRY(d.alloc(h.size()));
    if (!h.empty()) VJ_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return VAJRA_OK;
}

namespace {

// inst[t] = i for t in [off[i], off[i+1]); one CTA per instance.
__global__ void k_fill_instance_map(const int64_t* __restrict__ off, int count, int* __restrict__ inst) {
    const int i = blockIdx.x;
    if (i >= count) return;
    for (int64_t t = off[i] + threadIdx.x; t < off[i + 1]; t += blockDim.x) inst[t] = i;
}

__global__ void k_power_init_batched(int n, const int* __restrict__ col_inst, const int64_t* __restrict__ coff,
                                     double* __restrict__ v) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = col_inst[j];
    v[j] = 1.0 / sqrt(static_cast<double>(coff[i + 1] - coff[i]));
}

// One CTA per instance: ||u_i||, sigma_max_i = sqrt(||A_i^T A_i v_i||), v_i = u_i / ||u_i||.
__global__ void __launch_bounds__(kThreads)
k_power_step_batched(const int64_t* __restrict__ coff, const double* __restrict__ u, double* __restrict__ v,
                     double* __restrict__ sigma_max) {
    const int inst = blockIdx.x;
    __shared__ double red[32];
    __shared__ double inv;
    double s[1] = {0.0};
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) s[0] += u[j] * u[j];
    block_reduce<OpSum, double, 1>(s, red);
    if (threadIdx.x == 0) {
        const double nrm = sqrt(s[0]);
        sigma_max[inst] = sqrt(nrm);
        inv = nrm > 1e-300 ? 1.0 / nrm : 0.0;
    }
    __syncthreads();
    for (int64_t j = coff[inst] + threadIdx.x; j < coff[inst + 1]; j += blockDim.x) v[j] = u[j] * inv;
}

struct EpiStoreAll {
    double* out;
    __device__ bool active() const { return true; }
    __device__ void operator()(int r, double s) const { out[r] = s; }
};

}  // namespace

// Fixed-round batched power iteration on the scaled packed matrix; sigma_max[count] on device.
inline vajra_status batched_spectral_norms(const Prepared& p, int m, int n, int count, const int* col_inst,
                                           const int64_t* coff, double* sigma_max, int rounds, cudaStream_t st) {
    DeviceBuffer<double> v, w, u;
    VJ_TRY(v.alloc(n));
    VJ_TRY(w.alloc(m));
    VJ_TRY(u.alloc(n));
    k_power_init_batched<<<grid_for(n), kThreads, 0, st>>>(n, col_inst, coff, v.get());
    note_launch(1);
    for (int it = 0; it < rounds; ++it) {
        launch_spmv_t<double, double, double>(p.a, p.csr_val.get(), v.get(), EpiStoreAll{w.get()}, st);
        launch_spmv_t<double, double, double>(p.at, p.csc_val.get(), w.get(), EpiStoreAll{u.get()}, st);
        k_power_step_batched<<<count, kThreads, 0, st>>>(coff, u.get(), v.get(), sigma_max);
        note_launch(1);
    }
    VJ_LAUNCH_CHECK();
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

}  // namespace vajra
