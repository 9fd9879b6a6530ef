// Device-resident LP data and the set-up passes that turn the caller's CSC into what the
// iteration kernels read.
//
// HBM layout (one LP, one device):
//   raw (uploaded once by vajra_pdhg_create, never modified):
//     col_ptr int64[n+1] | row_idx int32[nnz] | values f64[nnz] | c, col_lo, col_up f64[n]
//     | row_lo, row_up f64[m]
//   prepared (rebuilt by every run; the reference does this on the host, pdhg_cuda.cu:136-171):
//     CSR of A: csr_ptr int64[m+1] | csr_idx int32[nnz] | perm int64[nnz] (CSR slot -> CSC slot)
//     scaled values in both orders (f64; plus f32 copies for the mixed-precision path)
//     scaled c (negated for maximisation), bounds, cumulative row / column scales.
#pragma once

#include "common.cuh"
#include "spmv.cuh"

namespace vajra {

struct DeviceLp {
    int m = 0, n = 0;
    int64_t nnz = 0;
    int sense = 0;
    double objective_offset = 0.0;
    DeviceBuffer<int64_t> col_ptr;
    DeviceBuffer<int32_t> row_idx;
    DeviceBuffer<double> values;
    DeviceBuffer<double> c, col_lower, col_upper, row_lower, row_upper;
};

// Sliced-ELL copy of a matrix whose rows are sorted by descending length (spmv.cuh, kSell):
// slice offsets, indices, and the values in FP64 and (mixed precision) FP32.
struct SellData {
    DeviceBuffer<int64_t> off;
    DeviceBuffer<int32_t> idx;
    DeviceBuffer<double> val64;
    DeviceBuffer<float> val32;
    DeviceBuffer<int32_t> long_rows, vlong_rows;   // rows kept in CSR (row order)
    DeviceBuffer<uint8_t> len;                     // row lengths, kSellLong for listed rows
};

struct Prepared {
    // structure
    DeviceBuffer<int64_t> csr_ptr;
    DeviceBuffer<int32_t> csr_idx;
    DeviceBuffer<int64_t> perm;
    // scaled data (CSC order = stored transpose, CSR order = A)
    DeviceBuffer<double> csc_val, csr_val;
    DeviceBuffer<float> csc_val32, csr_val32;
    DeviceBuffer<double> csr_val_orig;       // unscaled A in CSR order (post-processing)
    DeviceBuffer<double> c, col_lower, col_upper, row_lower, row_upper;
    DeviceBuffer<double> row_scale, col_scale;
    // per-row / per-column lists of long rows for the fast SpMV
    DeviceBuffer<int32_t> long_rows_a, long_rows_at;
    // row-block partitions (block boundaries) and their rows longer than kTile
    DeviceBuffer<int32_t> rb_blocks_a, rb_blocks_at, rb_long_a, rb_long_at;
    DeviceBuffer<TileDesc> rb_tiles_a, rb_tiles_at;
    // sliced-ELL copies (degree-ordered LPs only)
    SellData sell_a, sell_at;
    bool scaled = false;
    CsrView a, at;                            // A (rows = m) and A^T (rows = n)
};

// Scalars that set-up passes hand to one another on the device.
struct SetupState {
    int ruiz_done;
    int power_done;
    double ruiz_row_err;
    double ruiz_col_err;
    double lambda;
    double lambda_prev;
    double inv_norm;
    double spectral_norm;
    int power_iter;
    int pad;
    unsigned long long row_err_bits;   // this Ruiz pass's max |1 - row norm| (bit pattern, atomicMax)
    unsigned long long col_err_bits;
};

vajra_status upload_lp(const vajra_lp* lp, DeviceLp& d, cudaStream_t st);

// CSC -> CSR structure (stable radix sort by row keeps columns ascending within a row).
vajra_status build_csr(const DeviceLp& lp, Prepared& p, cudaStream_t st);

struct ScalingOpts {
    bool enable = true;
    int ruiz_iterations = 10;
    double ruiz_tolerance = 0.05;
    bool pock_chambolle = false;
    bool negate_c = false;     // maximisation
    bool pow2 = false;         // round the final factors to powers of two (exact scaling)
    // Block-diagonal LPs (the batched solver): with instances > 0, each instance runs the Ruiz
    // stopping test on its own rows and columns and keeps factor 1 once it has passed, so every
    // instance is scaled exactly as it would be alone.  Offsets: instances + 1 entries each;
    // row_inst / col_inst: the instance of every row / column.
    int instances = 0;
    const int64_t* roff = nullptr;
    const int64_t* coff = nullptr;
    const int* row_inst = nullptr;
    const int* col_inst = nullptr;
};

// Copies the raw data into the working buffers and applies Ruiz (exactly as
// src/linalg/scaling.cpp:7-153) and optionally Pock-Chambolle (alpha = 1) scaling, then
// fills the CSR-ordered values.  `sst` is a device SetupState.
vajra_status prepare_scaled(const DeviceLp& lp, Prepared& p, const ScalingOpts& o,
                            SetupState* sst, cudaStream_t st);

// True when every scaled value is exactly representable in FP32 (one host synchronisation).
vajra_status values_fit_fp32(const Prepared& p, int64_t nnz, bool* exact, cudaStream_t st);

// f32 copies of the scaled values (mixed-precision path).
vajra_status make_f32_values(Prepared& p, int64_t nnz, cudaStream_t st);

// Reference power iteration (src/solvers/pdhg/pdhg.cpp:11-56) evaluated in its order:
// sequential sums, zero-drop skip.  Result in sst->spectral_norm.
vajra_status spectral_norm_exact(const Prepared& p, int m, int n, int max_iter, double tol,
                                 SetupState* sst, cudaStream_t st);

// Fast power iteration on the scaled A (fp64, deterministic tree sums).
vajra_status spectral_norm_fast(const Prepared& p, int m, int n, int max_iter, double tol,
                                SetupState* sst, cudaStream_t st);

// Long-row lists and group sizes for the fast SpMV (a heuristic; the solver's autotuner
// may override `group`).
vajra_status plan_spmv(const DeviceLp& lp, Prepared& p, cudaStream_t st);

// Degree ordering: columns and rows renumbered in descending order of their entry counts
// (equal counts keep index order).  The entries of x and y that the two SpMVs gather most
// often then sit together in a few cache lines instead of one line each, and the rows of a
// row-block tile have similar lengths.  Within a column the entries keep their order.
struct LpOrder {
    DeviceBuffer<int32_t> col_order;   // new column -> caller's column
    DeviceBuffer<int32_t> row_order;   // new row -> caller's row
};
vajra_status order_by_degree(const DeviceLp& src, DeviceLp& dst, LpOrder& ord, cudaStream_t st);

// Sliced-ELL copy (SellData) of `v`: builds `out` from v's CSR-order values (val32 may be
// null) and sets v's sell_* fields.
vajra_status build_sell(CsrView& v, const double* val64, const float* val32, SellData& out, cudaStream_t st);

// dst[order[k]] = src[k] for k < count: a result vector back in the caller's numbering.
vajra_status unorder(int count, const int32_t* order, const double* src, double* dst, cudaStream_t st);

// Row-block partition of `v` at `tile` entries per block: nb + 1 block boundaries, the nb
// block descriptors, and the rows longer than `tile` (one CTA each).
vajra_status build_row_partition(const CsrView& v, int64_t tile, DeviceBuffer<int32_t>& blocks,
                                 DeviceBuffer<TileDesc>& tiles, DeviceBuffer<int32_t>& long_rows, int* nb,
                                 int* n_long, cudaStream_t st);

}  // namespace vajra
