// vajra_relative_kkt_noalloc_f64: the FP64 relative-KKT evaluation of the solver's checks
// (k_kkt_rows / k_kkt_cols + their combine in halpern_mode.cu, whose block partials live in
// memory the solver allocates) as an entry point that allocates nothing.
//
// Who needs it: callers that cannot call cudaMalloc / cudaFree at this point -- an
// application whose device memory is owned by another allocator (a framework's caching pool
// that has already reserved the free memory, so a plain cudaMalloc fails), a latency-critical
// loop in which cudaMalloc / cudaFree would synchronise the device and stall other streams,
// and code that must not be able to fail on allocation in the middle of a run.
//
// The per-block partial sums go to a file-scope device array of fixed size (2 MiB, loaded
// with the library and held by every device that uses it until the process exits), which
// limits an LP to 8,388,608 rows and columns here; larger sizes are rejected.  Host code
// cannot use the array's name as a device address, so each call looks up the current
// device's address with cudaGetSymbolAddress (with that device current) whenever its stream
// is not being captured, and keeps it per device.  A call made during a stream capture uses
// the address kept by the last call outside a capture on that device, so make the first call
// on a device before any capture -- and, after a cudaDeviceReset or a reset of the primary
// context (which reloads the library's module, so the array may move), make one call outside
// a capture before capturing again.
// Every call on a device shares the one array and overwrites it: calls that overlap on the
// GPU (different streams, or host threads without ordering) race and give wrong results.
// Each call writes every partial it later reads, so nothing needs clearing between calls.
#include <mutex>

#include "common.cuh"

// 2 partial-sum tables (row pass, column pass) x 32768 blocks x 4 doubles = 2 MiB.
static __device__ __align__(256) double g_noalloc_scratch[2 * 32768 * 4];

namespace vajra {
namespace {

constexpr int kNaRowsPerBlock = 256;                 // 8 warps x 32 rows
constexpr int kNaMaxBlocks = 32768;                  // per pass
constexpr int kNaQ = 4;                              // partial sums per block
constexpr size_t kNoAllocScratchDoubles = 2ull * kNaMaxBlocks * kNaQ;
static_assert(sizeof(g_noalloc_scratch) == kNoAllocScratchDoubles * sizeof(double), "scratch layout");
constexpr int64_t kNaMaxExtent = static_cast<int64_t>(kNaMaxBlocks) * kNaRowsPerBlock;   // 8,388,608

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Row pass: one warp per row; primal residual A x - proj(A x), ||b||^2 (finite bounds, an
// equality row once) and the row part of the dual objective.
__global__ void __launch_bounds__(kThreads)
k_na_rows(int m, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const double* __restrict__ val,
          const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ rl,
          const double* __restrict__ ru, double* __restrict__ part) {
    __shared__ double red[kNaQ * 32];
    double v[kNaQ] = {0, 0, 0, 0};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r0 = blockIdx.x * kNaRowsPerBlock;
    for (int r = r0 + warp; r < r0 + kNaRowsPerBlock && r < m; r += kThreads / 32) {
        double s = 0.0;
        for (int64_t k = ptr[r] + lane; k < ptr[r + 1]; k += 32) s += val[k] * x[idx[k]];
        s = warp_reduce<OpSum>(s);
        if (lane == 0) {
            const double l = rl[r], u = ru[r];
            const bool lf = l > -1e20, uf = u < 1e20;
            const double p = s - fmin(fmax(s, l), u);
            const double yi = y[r];
            v[0] += p * p;
            v[1] += (lf && uf && l == u) ? l * l : (lf ? l * l : 0.0) + (uf ? u * u : 0.0);
            if (yi > 0.0 && lf) v[2] += yi * l;
            else if (yi < 0.0 && uf) v[2] += yi * u;
        }
    }
    block_reduce<OpSum, double, kNaQ>(v, red);
    if (threadIdx.x == 0)
        for (int q = 0; q < kNaQ; ++q) part[blockIdx.x * kNaQ + q] = v[q];
}

// Column pass: one warp per column of the CSC; reduced cost r = c - A^T y (minimisation
// form), its bound-multiplier part, primal objective, ||c||^2, column part of the dual
// objective.
__global__ void __launch_bounds__(kThreads)
k_na_cols(int n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const double* __restrict__ val,
          const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ c,
          const double* __restrict__ cl, const double* __restrict__ cu, int sense, double* __restrict__ part) {
    __shared__ double red[kNaQ * 32];
    double v[kNaQ] = {0, 0, 0, 0};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j0 = blockIdx.x * kNaRowsPerBlock;
    for (int j = j0 + warp; j < j0 + kNaRowsPerBlock && j < n; j += kThreads / 32) {
        double s = 0.0;
        for (int64_t k = ptr[j] + lane; k < ptr[j + 1]; k += 32) s += val[k] * y[idx[k]];
        s = warp_reduce<OpSum>(s);
        if (lane == 0) {
            const double cm = sense ? -c[j] : c[j];
            const double r = cm - s;
            const bool lf = cl[j] > -1e20, uf = cu[j] < 1e20;
            const double lam = (lf && uf) ? r : lf ? fmax(r, 0.0) : uf ? fmin(r, 0.0) : 0.0;
            v[0] += (r - lam) * (r - lam);
            v[1] += c[j] * c[j];
            v[2] += cm * x[j];
            if (lam > 0.0) v[3] += lam * cl[j];
            else if (lam < 0.0) v[3] += lam * cu[j];
        }
    }
    block_reduce<OpSum, double, kNaQ>(v, red);
    if (threadIdx.x == 0)
        for (int q = 0; q < kNaQ; ++q) part[blockIdx.x * kNaQ + q] = v[q];
}

// out = [rel_primal, rel_dual, rel_gap, rel_kkt, primal objective, dual objective] in the
// minimisation form (the objective offset included, negated for maximisation).
__global__ void __launch_bounds__(1024)
k_na_final(int nb_r, int nb_c, const double* __restrict__ part_r, const double* __restrict__ part_c,
           double offset_min, double* __restrict__ out) {
    __shared__ double red[7 * 32];
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nb_r; b += blockDim.x)
        for (int q = 0; q < 3; ++q) s[q] += part_r[b * kNaQ + q];
    for (int b = threadIdx.x; b < nb_c; b += blockDim.x)
        for (int q = 0; q < 4; ++q) s[3 + q] += part_c[b * kNaQ + q];
    block_reduce<OpSum, double, 7>(s, red);
    if (threadIdx.x != 0) return;
    const double rel_p = sqrt(s[0]) / (1.0 + sqrt(s[1]));
    const double rel_d = sqrt(s[3]) / (1.0 + sqrt(s[4]));
    const double pobj = s[5] + offset_min;
    const double dobj = s[2] + s[6] + offset_min;
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    out[0] = rel_p;
    out[1] = rel_d;
    out[2] = gap;
    out[3] = fmax(rel_p, fmax(rel_d, gap));
    out[4] = pobj;
    out[5] = dobj;
}

// The current device's address of g_noalloc_scratch.  Looked up afresh on every call whose
// stream is not capturing (a reset context reloads the module, and the array can move); a
// call inside a capture cannot make that lookup and uses the address the last such call kept.
vajra_status scratch_address(cudaStream_t st, double** out) {
    int dev = 0;
    VJ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) { set_error("device ordinal %d beyond %d", dev, kMaxDevices); return VAJRA_ERR_INVALID_ARGUMENT; }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    const cudaError_t ce = cudaStreamIsCapturing(st, &cap);
    const bool capturing = ce != cudaSuccess || cap != cudaStreamCaptureStatusNone;
    if (ce != cudaSuccess) cudaGetLastError();   // e.g. the legacy stream while another captures
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!capturing) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_scratch_addr[dev] = static_cast<double*>(p);
    } else if (!g_scratch_addr[dev]) {
        set_error("vajra_relative_kkt_noalloc_f64: first call on device %d made inside a stream capture; "
                  "make one call outside a capture first", dev);
        return VAJRA_ERR_INVALID_ARGUMENT;
    }
    *out = g_scratch_addr[dev];
    return VAJRA_OK;
}

}  // namespace
}  // namespace vajra

using namespace vajra;

extern "C" vajra_status vajra_relative_kkt_noalloc_f64(
    int32_t rows, int32_t cols, const int64_t* row_ptr, const int32_t* col_idx, const double* csr_values,
    const int64_t* col_ptr, const int32_t* row_idx, const double* csc_values, const double* c,
    const double* col_lower, const double* col_upper, const double* row_lower, const double* row_upper,
    const double* x, const double* y, int32_t sense, double objective_offset, double* out, void* stream) {
    // An LP without rows (column bounds only) is allowed: its row-side arrays may be NULL.
    const bool has_rows = rows > 0;
    if (rows < 0 || cols < 1 || !col_ptr || !c || !col_lower || !col_upper || !x || !out ||
        (has_rows && (!row_ptr || !col_idx || !csr_values || !row_idx || !csc_values || !row_lower || !row_upper ||
                      !y))) {
        set_error("vajra_relative_kkt_noalloc_f64: negative row count, no columns, or a NULL pointer");
        return VAJRA_ERR_INVALID_ARGUMENT;
    }
    if (rows > kNaMaxExtent || cols > kNaMaxExtent) {
        set_error("vajra_relative_kkt_noalloc_f64: %d rows / %d columns exceed the no-allocation limit of %lld "
                  "(its fixed 2 MiB scratch); use the allocating solver path for larger LPs",
                  rows, cols, static_cast<long long>(kNaMaxExtent));
        return VAJRA_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* scratch = nullptr;
    VJ_TRY(scratch_address(st, &scratch));
    const int nb_r = (rows + kNaRowsPerBlock - 1) / kNaRowsPerBlock;
    const int nb_c = (cols + kNaRowsPerBlock - 1) / kNaRowsPerBlock;
    double* part_r = scratch;
    double* part_c = scratch + static_cast<size_t>(kNaMaxBlocks) * kNaQ;
    if (has_rows)
        k_na_rows<<<nb_r, kThreads, 0, st>>>(rows, row_ptr, col_idx, csr_values, x, y, row_lower, row_upper, part_r);
    k_na_cols<<<nb_c, kThreads, 0, st>>>(cols, col_ptr, row_idx, csc_values, x, y, c, col_lower, col_upper, sense,
                                         part_c);
    k_na_final<<<1, 1024, 0, st>>>(nb_r, nb_c, part_r, part_c, sense ? -objective_offset : objective_offset, out);
    note_launch(has_rows ? 3 : 2);
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}
