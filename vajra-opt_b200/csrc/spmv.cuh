// Sparse matrix-vector kernels over CSR (A) and over the stored transpose (the CSC of A,
// i.e. the CSR of A^T).  Each kernel hands every finished row sum to an epilogue functor,
// which is where the dual / primal prox, Halpern and KKT work is fused, so a row sum never
// makes a round trip through HBM.
//
// Kernel families:
//   k_spmv_seq       one thread per row, products added in storage order with explicit _rn
//                    intrinsics (no FMA contraction).  Over a CSR whose rows are sorted by
//                    column this reproduces the reference's CSC scatter SpMV
//                    (src/linalg/sparse.cpp:196-217) and in-order dot (:219-238) bit for bit,
//                    including the |x_j| <= 1e-11 skip.
//   k_spmv_vec       G lanes per row (G = 1..32), coalesced strided loads with streaming
//                    (evict-first) cache hints for the matrix and cached gathers for the dense
//                    vector, xor-butterfly reduction (deterministic), and trailing CTAs that
//                    take the rows longer than `long_len` one CTA per row.
//   k_spmv_rowblock  blocks of consecutive rows holding ~2048 entries, products staged in
//                    shared memory, then summed per row (one or two load groups per thread).
//   k_spmv_sell      sliced ELL: 32 rows a slice, a thread per row, the row's entries in pairs
//                    laid out so that every load is coalesced across the warp (the fastest
//                    form on rows numbered by length, as the degree-ordered LP has them).
// The autotuner of each solver picks the family and shape per matrix and precision.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace vajra {

// ----- round-to-nearest arithmetic without contraction --------------------------------
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }

template <typename T> __device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }
template <typename T> __device__ __forceinline__ T ld_cached(const T* p) { return __ldg(p); }

// ----- the reference's elementwise updates, in its evaluation order --------------------
// Dual Moreau step (src/solvers/pdhg/pdhg.cpp:204-209, spmv_kernels.cuh:173-178).
template <typename T>
__device__ __forceinline__ T dual_prox_exact(T y, T w, T sigma, T l, T u) {
    const T y_hat = rn_add(y, rn_mul(sigma, w));
    const T val = rn_div(y_hat, sigma);
    const T clamped = (val < l) ? l : ((val > u) ? u : val);
    return rn_sub(y_hat, rn_mul(sigma, clamped));
}

// Primal projected step (pdhg.cpp:229-235, spmv_kernels.cuh:197-202); returns x_new.
template <typename T>
__device__ __forceinline__ T primal_prox_exact(T x_old, T aty, T c, T tau, T l, T u) {
    const T grad = rn_add(aty, c);
    T x_new = rn_sub(x_old, rn_mul(tau, grad));
    if (x_new < l) x_new = l;
    if (x_new > u) x_new = u;
    return x_new;
}

template <typename T>
__device__ __forceinline__ T extrapolate_exact(T x_new, T x_old) {   // 2 x_new - x_old
    return rn_sub(rn_mul(T(2), x_new), x_old);
}

// ----- optional row-skip hook ----------------------------------------------------------
// An epilogue may define `bool skip_rows(int r0, int r1) const`: true when none of the rows
// [r0, r1) needs a result (the batched solver's finished instances).  The kernels then skip
// those rows' loads entirely.  Epilogues without the member never skip.
template <class E>
__device__ __forceinline__ auto skip_rows_impl(const E& e, int r0, int r1, int) -> decltype(e.skip_rows(r0, r1)) {
    return e.skip_rows(r0, r1);
}
template <class E>
__device__ __forceinline__ bool skip_rows_impl(const E&, int, int, long) { return false; }

// ----- optional two-phase epilogue ----------------------------------------------------
// An epilogue may define `Pre pre(int row) const` -- every load it needs that does not
// depend on the row sum -- and `void operator()(int row, Acc sum, const Pre&) const`.  The
// fast kernels call pre() before the row's matrix loads, so the epilogue's vector loads are
// in flight together with the SpMV's instead of after it (the epilogue's loads are otherwise
// ordered behind its own stores).  Epilogues without pre() are called as epi(row, sum).
struct NoPre {};
template <class E>
__device__ __forceinline__ auto epi_pre(const E& e, int row, int) -> decltype(e.pre(row)) { return e.pre(row); }
template <class E>
__device__ __forceinline__ NoPre epi_pre(const E&, int, long) { return NoPre{}; }
template <class E, class Acc, class P>
__device__ __forceinline__ auto epi_fin(const E& e, int row, Acc s, const P& p, int) -> decltype(e(row, s, p)) {
    return e(row, s, p);
}
template <class E, class Acc, class P>
__device__ __forceinline__ void epi_fin(const E& e, int row, Acc s, const P&, long) { e(row, s); }
template <class E>
using PreOf = decltype(epi_pre(*static_cast<const E*>(nullptr), 0, 0));

// ----- epilogues usable by both families ---------------------------------------------
template <typename T>
struct EpiStore {
    T* out;
    __device__ bool active() const { return true; }
    template <typename Acc> __device__ void operator()(int row, Acc s) const { out[row] = static_cast<T>(s); }
};

// ----- exact family -----------------------------------------------------------------
// ZERO_DROP: skip products whose dense operand has |x_j| <= 1e-11, as the reference's CSC
// multiply does (sparse.cpp:207).  Adding +0.0 instead of skipping is identical because a
// sum that starts at +0.0 never becomes -0.0.
template <typename V, bool ZERO_DROP, class Epi>
__global__ void __launch_bounds__(kThreads)
k_spmv_seq(int rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
           const V* __restrict__ val, const V* __restrict__ x, Epi epi) {
    pdl_enter();
    if (!epi.active()) return;
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= rows) return;
    const int64_t s = ptr[row], e = ptr[row + 1];
    V sum = V(0);
    for (int64_t k = s; k < e; ++k) {
        const V xv = x[idx[k]];
        if (ZERO_DROP && fabs(xv) <= V(kZeroDrop)) continue;
        sum = rn_add(sum, rn_mul(val[k], xv));
    }
    epi(row, sum);
}

// ----- fast family --------------------------------------------------------------------
// The rows of lane-group block b: 256 / G consecutive rows, G lanes each.
template <typename VV, typename VX, typename Acc, int G, class Epi>
__device__ __forceinline__ void vec_block(int b, int rows, const int64_t* __restrict__ ptr,
                                          const int32_t* __restrict__ idx, const VV* __restrict__ val,
                                          const VX* __restrict__ x, int64_t long_len, const Epi& epi) {
    const int lane = threadIdx.x & (G - 1);
    const int row = (b * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x)) / G;
    bool valid = row < rows;
    int64_t s = 0, e = 0;
    PreOf<Epi> pre{};
    if (valid && lane == 0) pre = epi_pre(epi, row, 0);   // ahead of the row pointers
    if (valid) {
        s = ptr[row];
        e = ptr[row + 1];
        if (e - s > long_len || skip_rows_impl(epi, row, row + 1, 0)) valid = false;
    }
    Acc acc = Acc(0);
    if (valid) {
#pragma unroll 4
        for (int64_t k = s + lane; k < e; k += G)
            acc = fma(static_cast<Acc>(ld_stream(val + k)), static_cast<Acc>(ld_cached(x + ld_stream(idx + k))), acc);
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (valid && lane == 0) epi_fin(epi, row, acc, pre, 0);
}

// VV: stored value type, VX: dense-vector type, Acc: accumulation type.
// CTAs [0, vec_blocks) take lane-group blocks: block blockIdx.x, or -- in list mode
// (blk_list != null) -- blocks blk_list[t] for t = blockIdx.x, + vec_blocks, ... < *blk_count.
// CTAs from vec_blocks on take one long row each.
template <typename VV, typename VX, typename Acc, int G, class Epi>
__global__ void __launch_bounds__(kThreads)
k_spmv_vec(int rows, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
           const VV* __restrict__ val, const VX* __restrict__ x, int64_t long_len,
           const int32_t* __restrict__ long_rows, int vec_blocks, const int32_t* __restrict__ blk_list,
           const int* __restrict__ blk_count, Epi epi) {
    pdl_enter();
    if (!epi.active()) return;
    if (static_cast<int>(blockIdx.x) >= vec_blocks) {
        // One CTA per long row.
        __shared__ Acc red[32];
        const int row = long_rows[blockIdx.x - vec_blocks];
        if (skip_rows_impl(epi, row, row + 1, 0)) return;
        const int64_t s = ptr[row], e = ptr[row + 1];
        Acc acc = Acc(0);
        for (int64_t k = s + threadIdx.x; k < e; k += blockDim.x)
            acc = fma(static_cast<Acc>(ld_stream(val + k)), static_cast<Acc>(ld_cached(x + ld_stream(idx + k))), acc);
        Acc v[1] = {acc};
        block_reduce<OpSum, Acc, 1>(v, red);
        if (threadIdx.x == 0) epi(row, v[0]);
        return;
    }
    if (blk_list == nullptr) {
        vec_block<VV, VX, Acc, G>(blockIdx.x, rows, ptr, idx, val, x, long_len, epi);
        return;
    }
    const int cnt = *blk_count;
    for (int t = blockIdx.x; t < cnt; t += vec_blocks)
        vec_block<VV, VX, Acc, G>(blk_list[t], rows, ptr, idx, val, x, long_len, epi);
}

// ----- row-block family (shared-memory staging) ----------------------------------------
// The rows are cut into blocks of consecutive rows: block b holds the rows whose first entry
// lies in [b*kTile, (b+1)*kTile) (a binary search per block at set-up).  A CTA streams its
// block's indices and values with 128-bit vector loads (aligned groups of four; the partial
// groups at both ends are masked), issues every gather of the dense vector independently,
// and stages the products in shared memory.  Then each short row is summed by one thread in
// storage order and rows longer than kMediumRow by one warp (fixed butterfly), and the
// epilogue runs on consecutive rows, so its vector loads and stores coalesce.  A row longer
// than kTile is necessarily the last row starting in its block; it is taken by one of the
// trailing CTAs of the same launch.  A block's staged entries never exceed 2 kTile - 1.
constexpr int kTile = 2048;
constexpr int kMediumRow = 48;

__device__ __forceinline__ void load4(const int32_t* p, int (&v)[4]) {
    const int4 t = __ldcs(reinterpret_cast<const int4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load4(const float* p, float (&v)[4]) {
    const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// A row block as the kernel reads it: rows [r0, r_end) and their entries [e0, e1) (the
// block's last row is left out when it is longer than kTile).  Precomputed at set-up so a CTA
// starts its stream loads after one dependent load instead of two.
struct TileDesc {
    long long e0, e1;
    int r0, r_end;
};

// Resident CTAs per SM the row-block kernel is compiled for: with 4-byte values six (40
// registers a thread) measured fastest; with 8-byte values four (64 registers; six spills).
template <typename VV>
constexpr int rowblock_min_blocks() { return sizeof(VV) == 4 ? 6 : 4; }

// One row block (tile b).  Every exit before the first barrier is uniform over the CTA.
// U: groups of four entries a thread loads before it gathers (all U groups' loads in flight).
// PRE: issue the epilogue's early loads (two-phase epilogues) for the thread's first row.
template <typename VV, typename VX, typename Acc, int U, int KT, int MR, bool PRE, class Epi>
__device__ __forceinline__ void rowblock_tile(int b, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                              const VV* __restrict__ val, const VX* __restrict__ x,
                                              const TileDesc* __restrict__ tiles, Acc* prod, int* med_rows,
                                              int& n_med, const Epi& epi) {
    const TileDesc td = tiles[b];
    const int r0 = td.r0, r_end = td.r_end;
    if (r0 >= r_end || skip_rows_impl(epi, r0, r_end, 0)) return;
    const int64_t e0 = td.e0, e1 = td.e1;
    // this thread's first row (the row it sums below): epilogue inputs and row bounds load
    // now, alongside the block's stream
    const int my_row = r0 + static_cast<int>(threadIdx.x);
    PreOf<Epi> pre{};
    int my_s = 0, my_e = 0;
    if (my_row < r_end) {
        if constexpr (PRE) pre = epi_pre(epi, my_row, 0);
        my_s = static_cast<int>(ptr[my_row] - e0);
        my_e = static_cast<int>(ptr[my_row + 1] - e0);
    }
    const int64_t qstride = 4 * static_cast<int64_t>(blockDim.x);
    for (int64_t q0 = (e0 & ~int64_t(3)) + 4 * static_cast<int64_t>(threadIdx.x); q0 < e1; q0 += U * qstride) {
        int ii[U][4];
        VV vv[U][4];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t q = q0 + u * qstride;
            if (q < e1) {
                load4(idx + q, ii[u]);
                load4(val + q, vv[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t q = q0 + u * qstride;
            Acc pr[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int64_t k = q + t;
                pr[t] = (k >= e0 && k < e1) ? static_cast<Acc>(vv[u][t]) * static_cast<Acc>(ld_cached(x + ii[u][t]))
                                            : Acc(0);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int64_t k = q + t;
                if (k >= e0 && k < e1) prod[k - e0] = pr[t];
            }
        }
    }
    if (threadIdx.x == 0) n_med = 0;
    __syncthreads();
    for (int r = my_row; r < r_end; r += blockDim.x) {
        const int s = r == my_row ? my_s : static_cast<int>(ptr[r] - e0);
        const int e = r == my_row ? my_e : static_cast<int>(ptr[r + 1] - e0);
        if (e - s > MR) {
            med_rows[atomicAdd(&n_med, 1)] = r;
            continue;
        }
        Acc acc = Acc(0);
        for (int k = s; k < e; ++k) acc += prod[k];
        if (PRE && r == my_row) epi_fin(epi, r, acc, pre, 0);
        else epi(r, acc);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int w = warp; w < n_med; w += blockDim.x >> 5) {
        const int r = med_rows[w];
        const int s = static_cast<int>(ptr[r] - e0), e = static_cast<int>(ptr[r + 1] - e0);
        Acc acc = Acc(0);
        for (int k = s + lane; k < e; k += 32) acc += prod[k];
        acc = warp_reduce<OpSum>(acc);
        if (lane == 0) epi(r, acc);
    }
}

// CTAs [0, nb) take row blocks: block blockIdx.x, or -- in list mode (blk_list != null) --
// blocks blk_list[t] for t = blockIdx.x, + nb, ... < *blk_count.  CTAs from nb on take one
// row longer than kTile each.
template <typename VV, typename VX, typename Acc, class Epi, int MB = rowblock_min_blocks<VV>(), int U = 1,
          int KT = kTile, int MR = kMediumRow, bool PRE = true>
__global__ void __launch_bounds__(kThreads, MB)
k_spmv_rowblock(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const VV* __restrict__ val,
                const VX* __restrict__ x, const TileDesc* __restrict__ tiles, int nb,
                const int32_t* __restrict__ long_rows, const int32_t* __restrict__ blk_list,
                const int* __restrict__ blk_count, Epi epi) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Acc* prod = reinterpret_cast<Acc*>(smem_raw);
    __shared__ int med_rows[(2 * KT) / MR + 1];
    __shared__ int n_med;
    __shared__ Acc red[32];
    pdl_enter();
    if (!epi.active()) return;
    if (static_cast<int>(blockIdx.x) >= nb) {
        const int row = long_rows[blockIdx.x - nb];
        if (skip_rows_impl(epi, row, row + 1, 0)) return;
        const int64_t s = ptr[row], e = ptr[row + 1];
        Acc acc = Acc(0);
        for (int64_t k = s + threadIdx.x; k < e; k += blockDim.x)
            acc = fma(static_cast<Acc>(ld_stream(val + k)), static_cast<Acc>(ld_cached(x + ld_stream(idx + k))), acc);
        Acc v[1] = {acc};
        block_reduce<OpSum, Acc, 1>(v, red);
        if (threadIdx.x == 0) epi(row, v[0]);
        return;
    }
    if (blk_list == nullptr) {
        rowblock_tile<VV, VX, Acc, U, KT, MR, PRE>(blockIdx.x, ptr, idx, val, x, tiles, prod, med_rows, n_med, epi);
        return;
    }
    const int cnt = *blk_count;
    for (int t = blockIdx.x; t < cnt; t += nb) {
        rowblock_tile<VV, VX, Acc, U, KT, MR, PRE>(blk_list[t], ptr, idx, val, x, tiles, prod, med_rows, n_med, epi);
        __syncthreads();   // the tile's shared state is reused by the next one
    }
}

// ----- sliced-ELL family ---------------------------------------------------------------
// The rows are cut into slices of 32 consecutive rows; slice s stores entries 2j and 2j + 1 of
// its row `lane` side by side at sell_off[s] + 64 j + 2 lane (kSellPack = 2; with 1, entry k at
// sell_off[s] + 32 k + lane).  One warp takes a slice, a thread its row, and every load of
// indices and values is coalesced across the warp; a row's sum is formed in storage order, so
// no shared memory, barrier or cross-lane reduction is needed.  A slice's width is the length
// of its longest row (rounded up to even); the padding is never gathered.  Rows longer than
// kSellWidth stay in CSR and are listed: one warp each, one CTA each above kSellCtaRow
// entries.  The layout pays off when the rows of a slice have similar lengths -- the
// degree-ordered LP numbers its rows by descending length, so there the long rows are a prefix
// and the slices are nearly full.
constexpr int kSellWidth = 128;
constexpr int kSellCtaRow = 4096;
constexpr int kSellPack = 2;
template <typename T> struct Pack2;
template <> struct Pack2<float> { using type = float2; };
template <> struct Pack2<double> { using type = double2; };

// Where a kernel reads the dense vector's entries from: global memory through the read-only
// path, or -- for the entries [0, hot) of the hot-prefix kernel -- a copy in shared memory.
template <typename VX>
struct GatherGlobal {
    const VX* __restrict__ x;
    __device__ __forceinline__ VX operator()(int j) const { return ld_cached(x + j); }
};
// Global load through the read-only path that only the lanes with `pred` issue (predicated
// in PTX, so no branch splits the warp and the loads of an unrolled loop stay in flight
// together); the other lanes keep `v`.
__device__ __forceinline__ void ld_nc_if(float& v, const float* p, bool pred) {
    asm("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q ld.global.nc.f32 %0, [%1];\n\t}"
        : "+f"(v) : "l"(p), "r"(static_cast<int>(pred)));
}
__device__ __forceinline__ void ld_nc_if(double& v, const double* p, bool pred) {
    asm("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q ld.global.nc.f64 %0, [%1];\n\t}"
        : "+d"(v) : "l"(p), "r"(static_cast<int>(pred)));
}
template <typename VX>
struct GatherHot {
    const VX* __restrict__ x;
    const VX* xs;   // shared-memory copy of x[0, hot)
    int hot;
    __device__ __forceinline__ VX operator()(int j) const {
        const bool cold = j >= hot;
        VX g = VX(0);
        ld_nc_if(g, x + j, cold);             // only the cold lanes make an L1/L2 request
        const VX s = xs[cold ? 0 : j];        // every lane reads shared memory (cold lanes: entry 0)
        return cold ? g : s;
    }
};

template <typename VV, typename VX, typename Acc, class Epi, class G>
__device__ __forceinline__ void sell_warp_row(int row, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                              const VV* __restrict__ val, const G& gx, const Epi& epi) {
    const int lane = threadIdx.x & 31;
    PreOf<Epi> pre{};
    if (lane == 0) pre = epi_pre(epi, row, 0);
    const int64_t s = ptr[row], e = ptr[row + 1];
    Acc acc = Acc(0);
#pragma unroll 4
    for (int64_t k = s + lane; k < e; k += 32)
        acc = fma(static_cast<Acc>(ld_stream(val + k)), static_cast<Acc>(gx(ld_stream(idx + k))), acc);
    acc = warp_reduce<OpSum>(acc);
    if (lane == 0) epi_fin(epi, row, acc, pre, 0);
}

// The rows of slice `sl` (one per lane) that are not listed as long.  No warp collectives.
// sell_len[row]: the row's length, kSellLong for a listed row (one byte instead of two 8-byte
// row pointers per row).
constexpr uint8_t kSellLong = 0xFF;
static_assert(kSellWidth < kSellLong, "row lengths of the slices must fit one byte below the marker");

template <typename VV, typename VX, typename Acc, class Epi, class G>
__device__ __forceinline__ void sell_slice(int sl, int rows, const uint8_t* __restrict__ sell_len,
                                           const int64_t* __restrict__ sell_off, const int32_t* __restrict__ sell_idx,
                                           const VV* __restrict__ sell_val, const G& gx, const Epi& epi) {
    const int lane = threadIdx.x & 31;
    const int row = sl * 32 + lane;
    if (row >= rows) return;
    const int len = __ldg(sell_len + row);
    if (len == kSellLong) return;
    const PreOf<Epi> pre = epi_pre(epi, row, 0);
    Acc acc = Acc(0);
    if constexpr (kSellPack == 1) {
        const int64_t base = sell_off[sl] + lane;
#pragma unroll 4
        for (int k = 0; k < len; ++k) {
            const int64_t q = base + 32 * static_cast<int64_t>(k);
            acc = fma(static_cast<Acc>(ld_stream(sell_val + q)), static_cast<Acc>(gx(ld_stream(sell_idx + q))), acc);
        }
    } else {
        // one 8-byte index load and one 8- or 16-byte value load per pair (the slot after an
        // odd row's last entry is not gathered)
        using VV2 = typename Pack2<VV>::type;
        const int64_t base = sell_off[sl] + 2 * lane;
        const int pairs = (len + 1) >> 1;
#pragma unroll 4
        for (int j = 0; j < pairs; ++j) {
            const int64_t q = base + 64 * static_cast<int64_t>(j);
            const int2 ii = __ldcs(reinterpret_cast<const int2*>(sell_idx + q));
            const VV2 vv = __ldcs(reinterpret_cast<const VV2*>(sell_val + q));
            acc = fma(static_cast<Acc>(vv.x), static_cast<Acc>(gx(ii.x)), acc);
            if (2 * j + 1 < len) acc = fma(static_cast<Acc>(vv.y), static_cast<Acc>(gx(ii.y)), acc);
        }
    }
    epi_fin(epi, row, acc, pre, 0);
}

// CTAs [0, n_vlong): the listed rows above kSellCtaRow entries, one CTA each.  The next
// ceil(n_long / 8) CTAs: the listed rows of kSellWidth..kSellCtaRow entries, one warp each.
// The remaining CTAs: 8 slices each, a warp per slice.  Long rows come first so that they
// start first.
template <typename VV, typename VX, typename Acc, class Epi, int MB>
__global__ void __launch_bounds__(kThreads, MB)
k_spmv_sell(int rows, int slices, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
            const VV* __restrict__ val, const int32_t* __restrict__ vlong_rows, int n_vlong,
            const int32_t* __restrict__ long_rows, int n_long, const uint8_t* __restrict__ sell_len,
            const int64_t* __restrict__ sell_off,
            const int32_t* __restrict__ sell_idx, const VV* __restrict__ sell_val, const VX* __restrict__ x, Epi epi) {
    pdl_enter();
    if (!epi.active()) return;
    int b = static_cast<int>(blockIdx.x);
    if (b < n_vlong) {
        __shared__ Acc red[32];
        const int row = vlong_rows[b];
        if (skip_rows_impl(epi, row, row + 1, 0)) return;
        const int64_t s = ptr[row], e = ptr[row + 1];
        Acc acc = Acc(0);
        for (int64_t k = s + threadIdx.x; k < e; k += blockDim.x)
            acc = fma(static_cast<Acc>(ld_stream(val + k)), static_cast<Acc>(ld_cached(x + ld_stream(idx + k))), acc);
        Acc v[1] = {acc};
        block_reduce<OpSum, Acc, 1>(v, red);
        if (threadIdx.x == 0) epi(row, v[0]);
        return;
    }
    b -= n_vlong;
    const int warp = static_cast<int>(threadIdx.x >> 5);
    constexpr int kWarps = kThreads / 32;
    const int long_ctas = (n_long + kWarps - 1) / kWarps;
    if (b < long_ctas) {
        const int w = b * kWarps + warp;
        if (w < n_long) {
            const int row = long_rows[w];
            if (!skip_rows_impl(epi, row, row + 1, 0))
                sell_warp_row<VV, VX, Acc>(row, ptr, idx, val, GatherGlobal<VX>{x}, epi);
        }
        return;
    }
    const int sl = (b - long_ctas) * kWarps + warp;
    if (sl < slices) sell_slice<VV, VX, Acc>(sl, rows, sell_len, sell_off, sell_idx, sell_val, GatherGlobal<VX>{x}, epi);
}

// ----- sliced ELL with the hot prefix of the dense vector in shared memory ---------------
// On the degree-ordered LP the vector entries gathered most often are the first ones: the
// 28,672 longest columns of the 1M x 2M LP hold 40 % of A's entries.  Every CTA of this
// persistent kernel first copies x[0, hot) into shared memory, and the gathers below `hot` are
// then served from there -- a shared-memory access instead of an L1/L2 request, which is
// what bounds the plain kernel.  Persistent CTAs (kSellHotCtasPerSm per SM, kSellHotThreads
// threads) amortise the copy; the CTAs walk the very long rows (one CTA each), then their
// warps take the listed long rows and the slices in an interleaved order (slice widths fall
// along the order, so interleaving balances the warps).  Sums and epilogues are the plain
// kernel's, so results are bit-identical to it.
constexpr int kSellHotThreads = 768;
constexpr int kSellHotCtasPerSm = 2;
constexpr int kSellHotBytes = 112 * 1024;   // shared memory per CTA (two CTAs fill an SM's 228 KB)

template <typename VV, typename VX, typename Acc, class Epi>
__global__ void __launch_bounds__(kSellHotThreads, kSellHotCtasPerSm)
k_spmv_sell_hot(int rows, int slices, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                const VV* __restrict__ val, const int32_t* __restrict__ vlong_rows, int n_vlong,
                const int32_t* __restrict__ long_rows, int n_long, const uint8_t* __restrict__ sell_len,
                const int64_t* __restrict__ sell_off, const int32_t* __restrict__ sell_idx,
                const VV* __restrict__ sell_val, const VX* __restrict__ x, int hot, Epi epi) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Acc red[32];
    VX* xs = reinterpret_cast<VX*>(smem_raw);
    pdl_enter();
    if (!epi.active()) return;   // uniform over the grid (device state)
    // x[0, hot): 16-byte loads (x is a device allocation, 256-byte aligned; hot is a multiple
    // of the vector width), written by the previous kernel, so a plain load
    constexpr int kVec = 16 / sizeof(VX);
    for (int k = threadIdx.x * kVec; k < hot; k += kSellHotThreads * kVec) {
        if constexpr (sizeof(VX) == 4) *reinterpret_cast<float4*>(xs + k) = *reinterpret_cast<const float4*>(x + k);
        else *reinterpret_cast<double2*>(xs + k) = *reinterpret_cast<const double2*>(x + k);
    }
    __syncthreads();
    const GatherHot<VX> gx{x, xs, hot};
    for (int i = blockIdx.x; i < n_vlong; i += gridDim.x) {   // uniform over the CTA
        const int row = vlong_rows[i];
        const int64_t s = ptr[row], e = ptr[row + 1];
        Acc acc = Acc(0);
        // the plain kernel's split of the row over kThreads threads (the other warps add zeros),
        // so that the row sum has the same bits
        if (threadIdx.x < kThreads)
            for (int64_t k = s + threadIdx.x; k < e; k += kThreads)
                acc = fma(static_cast<Acc>(ld_stream(val + k)), static_cast<Acc>(gx(ld_stream(idx + k))), acc);
        Acc v[1] = {acc};
        block_reduce<OpSum, Acc, 1>(v, red);
        if (threadIdx.x == 0) epi(row, v[0]);
    }
    constexpr int kWarps = kSellHotThreads / 32;
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const int items = n_long + slices;
    for (int w = blockIdx.x * kWarps + warp; w < items; w += gridDim.x * kWarps) {
        if (w < n_long) sell_warp_row<VV, VX, Acc>(long_rows[w], ptr, idx, val, gx, epi);
        else sell_slice<VV, VX, Acc>(w - n_long, rows, sell_len, sell_off, sell_idx, sell_val, gx, epi);
    }
}

// Host-side description of one SpMV operand (a CSR, possibly the stored transpose) and the
// launch shape the autotuner chose for it.
struct CsrView {
    int rows = 0;
    int cols = 0;
    int64_t nnz = 0;
    const int64_t* ptr = nullptr;
    const int32_t* idx = nullptr;
    int group = 8;                      // lanes per row (1,2,4,...,32); 0 / kRowblock2 = row-block kernel
    int64_t long_len = 1 << 30;         // grouped-lane kernel: rows longer than this go one CTA per row
    const int32_t* long_rows = nullptr; // device list of those rows
    int n_long = 0;
    const int32_t* block_rows = nullptr;  // row-block kernel: nb + 1 block boundaries
    const TileDesc* tiles = nullptr;      // and the nb blocks as the kernel reads them
    int nb = 0;
    const int32_t* rb_long_rows = nullptr;  // rows longer than kTile
    int rb_n_long = 0;
    // List mode (the batched solver): only the blocks blk_list[0, *blk_count) -- lane-group
    // blocks of `group`, or row blocks for group 0 -- are computed, by blk_grid persistent CTAs.
    const int32_t* blk_list = nullptr;
    const int* blk_count = nullptr;
    int blk_grid = 0;
    // Sliced-ELL structure (null where none was built): sell_slices slices of 32 rows, and the
    // rows longer than kSellWidth listed (sell_long_rows: one warp each, sell_vlong_rows: above
    // kSellCtaRow entries, one CTA each).  The values in slice order are per precision and
    // are passed to launch_sell by the caller.
    const int64_t* sell_off = nullptr;
    const int32_t* sell_idx = nullptr;
    const uint8_t* sell_len = nullptr;
    int sell_slices = 0;
    const int32_t* sell_long_rows = nullptr;
    int sell_n_long = 0;
    const int32_t* sell_vlong_rows = nullptr;
    int sell_n_vlong = 0;
};

// Launch-shape code of the sliced-ELL kernel.
constexpr int kSell = 128;

// Slice blocks (8 slices, one CTA) of the sliced-ELL kernel.
inline int sell_block_count(const CsrView& a) { return (a.sell_slices + kThreads / 32 - 1) / (kThreads / 32); }

template <typename VV, typename VX, typename Acc, class Epi>
inline void launch_sell(const CsrView& a, const VV* csr_val, const VV* sell_val, const VX* x, Epi epi, cudaStream_t st) {
    constexpr int MB = sizeof(VV) == 4 ? 6 : 4;
    constexpr int kWarps = kThreads / 32;
    const int blocks = a.sell_n_vlong + (a.sell_n_long + kWarps - 1) / kWarps + sell_block_count(a);
    if (blocks <= 0) return;
    launch_chained(k_spmv_sell<VV, VX, Acc, Epi, MB>, blocks, kThreads, 0, st,
                   a.rows, a.sell_slices, a.ptr, a.idx, csr_val, a.sell_vlong_rows, a.sell_n_vlong, a.sell_long_rows,
                   a.sell_n_long, a.sell_len, a.sell_off, a.sell_idx, sell_val, x, epi);
    note_launch();
}

// Launch-shape code of the hot-prefix sliced-ELL kernel.
constexpr int kSellHot = 129;

// Streaming multiprocessors of the current device (read once per device).
int sm_count();

// Entries of the dense vector the hot-prefix kernel keeps in shared memory.
template <typename VX>
inline int sell_hot_extent(int cols) {
    const int cap = kSellHotBytes / static_cast<int>(sizeof(VX));
    return cols < cap ? (cols + 3) / 4 * 4 : cap;   // a multiple of four: whole 16-byte loads
}

// The kernel needs more than 48 KB of dynamic shared memory, which is granted per kernel and
// device.  Called outside any stream capture (the solver's set-up does) before the first
// launch; idempotent.
template <typename VV, typename VX, typename Acc, class Epi>
inline cudaError_t sell_hot_prepare() {
    return cudaFuncSetAttribute(k_spmv_sell_hot<VV, VX, Acc, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSellHotBytes);
}

template <typename VV, typename VX, typename Acc, class Epi>
inline void launch_sell_hot(const CsrView& a, const VV* csr_val, const VV* sell_val, const VX* x, Epi epi,
                            cudaStream_t st) {
    constexpr int kWarps = kSellHotThreads / 32;
    const int items = a.sell_n_long + a.sell_slices;
    int grid = sm_count() * kSellHotCtasPerSm;
    const int need = std::max(a.sell_n_vlong, (items + kWarps - 1) / kWarps);
    if (need < grid) grid = need;
    if (grid <= 0) return;
    const int hot = sell_hot_extent<VX>(a.cols);
    // a vector shorter than the 16-byte padding of its allocation is still read whole (the
    // buffers carry 16 spare elements, so the rounded-up extent stays inside the allocation)
    launch_chained(k_spmv_sell_hot<VV, VX, Acc, Epi>, grid, kSellHotThreads, static_cast<size_t>(hot) * sizeof(VX), st,
                   a.rows, a.sell_slices, a.ptr, a.idx, csr_val, a.sell_vlong_rows, a.sell_n_vlong, a.sell_long_rows,
                   a.sell_n_long, a.sell_len, a.sell_off, a.sell_idx, sell_val, x, hot, epi);
    note_launch();
}

// Launch-shape code of the row-block kernel with two groups of four entries in flight per
// thread (U = 2).  With 4-byte values it keeps six CTAs per SM by leaving the epilogue's loads
// to the end (they would not fit in 40 registers); with 8-byte values it keeps them early at
// four CTAs per SM.  Group 0 is U = 1 with early epilogue loads.
constexpr int kRowblock2 = 64;
inline bool is_rowblock_shape(int group) { return group == 0 || group == kRowblock2; }

template <typename VV, typename VX, typename Acc, int U = 1, class Epi>
inline void launch_rowblock(const CsrView& a, const VV* val, const VX* x, Epi epi, cudaStream_t st) {
    const size_t smem = sizeof(Acc) * 2 * kTile;
    const int nb = a.blk_list ? a.blk_grid : a.nb;
    constexpr int MB = U == 1 ? rowblock_min_blocks<VV>() : (sizeof(VV) == 4 ? 6 : 4);
    constexpr bool PRE = U == 1 || sizeof(VV) != 4;
    launch_chained(k_spmv_rowblock<VV, VX, Acc, Epi, MB, U, kTile, kMediumRow, PRE>, nb + a.rb_n_long, kThreads, smem,
                   st, a.ptr, a.idx, val, x, a.tiles, nb, a.rb_long_rows, a.blk_list, a.blk_count, epi);
    note_launch();
}

// Lane-group blocks of the grouped-lane kernel at G lanes per row.
inline int vec_block_count(int rows, int G) { return static_cast<int>(grid_for(static_cast<int64_t>(rows) * G)); }

template <typename VV, typename VX, typename Acc, int G, class Epi>
inline void launch_vec_g(const CsrView& a, const VV* val, const VX* x, Epi epi, cudaStream_t st) {
    const int vec_blocks = a.blk_list ? a.blk_grid : vec_block_count(a.rows, G);
    launch_chained(k_spmv_vec<VV, VX, Acc, G, Epi>, vec_blocks + a.n_long, kThreads, 0, st,
                   a.rows, a.ptr, a.idx, val, x, a.long_len, a.long_rows, vec_blocks, a.blk_list, a.blk_count, epi);
    note_launch();
}

// group 0 / kRowblock2 select the row-block kernel; other lane-group sizes than 1..16 dispatch to 32.
// kSell needs the values in sliced-ELL order (launch_sell); given CSR values only, it runs as
// the row-block kernel.
template <typename VV, typename VX, typename Acc, class Epi>
inline void launch_spmv_t(const CsrView& a, const VV* val, const VX* x, Epi epi, cudaStream_t st) {
    if (a.rows <= 0) return;
    switch (a.group) {
        case kSell:
        case kSellHot:
        case 0:
            if (a.tiles) { launch_rowblock<VV, VX, Acc, 1>(a, val, x, epi, st); break; }
            launch_vec_g<VV, VX, Acc, 8>(a, val, x, epi, st);
            break;
        case kRowblock2:
            if (a.tiles) { launch_rowblock<VV, VX, Acc, 2>(a, val, x, epi, st); break; }
            launch_vec_g<VV, VX, Acc, 8>(a, val, x, epi, st);
            break;
        case 1: launch_vec_g<VV, VX, Acc, 1>(a, val, x, epi, st); break;
        case 2: launch_vec_g<VV, VX, Acc, 2>(a, val, x, epi, st); break;
        case 4: launch_vec_g<VV, VX, Acc, 4>(a, val, x, epi, st); break;
        case 8: launch_vec_g<VV, VX, Acc, 8>(a, val, x, epi, st); break;
        case 16: launch_vec_g<VV, VX, Acc, 16>(a, val, x, epi, st); break;
        default: launch_vec_g<VV, VX, Acc, 32>(a, val, x, epi, st); break;
    }
}

template <typename V, typename Acc, class Epi>
inline void launch_spmv(const CsrView& a, const V* val, const V* x, Epi epi, cudaStream_t st) {
    launch_spmv_t<V, V, Acc>(a, val, x, epi, st);
}

template <typename V, bool ZERO_DROP, class Epi>
inline void launch_spmv_exact(const CsrView& a, const V* val, const V* x, Epi epi, cudaStream_t st) {
    if (a.rows <= 0) return;
    launch_chained(k_spmv_seq<V, ZERO_DROP, Epi>, grid_for(a.rows), kThreads, 0, st, a.rows, a.ptr, a.idx, val, x, epi);
    note_launch();
}

}  // namespace vajra
