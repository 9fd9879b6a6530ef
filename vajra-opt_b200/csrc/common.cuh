// Shared infrastructure for libvajra_pdhg: status plumbing (no exception ever crosses the C
// ABI), owning device buffers, and deterministic reductions (fixed order, no atomics on
// floating-point values, so every run repeats bit for bit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>

#include "vajra_pdhg.h"

namespace vajra {

// Last error text of the calling thread (copied into vajra_result::status_message).
void set_error(const char* fmt, ...);
const char* last_error();

// Kernels launched by the calling thread (graph replays count every captured node).
int64_t& launch_count();
inline void note_launch(int64_t k = 1) { launch_count() += k; }

vajra_status cuda_status(cudaError_t e, const char* what, const char* file, int line);

#define VJ_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t vj_e_ = (call);                                                    \
        if (vj_e_ != cudaSuccess) return ::vajra::cuda_status(vj_e_, #call, __FILE__, __LINE__); \
    } while (0)

#define VJ_TRY(call)                                                                   \
    do {                                                                               \
        vajra_status vj_s_ = (call);                                                   \
        if (vj_s_ != VAJRA_OK) return vj_s_;                                           \
    } while (0)

#define VJ_LAUNCH_CHECK() VJ_CUDA(cudaGetLastError())

constexpr int kThreads = 256;           // default CTA size of elementwise / SpMV kernels
constexpr double kInf = 1e20;           // reference infinity convention (model.hpp)
constexpr double kZeroDrop = 1e-11;     // tol::kZeroDrop (tolerances.hpp:28)

inline unsigned grid_for(int64_t work, int threads = kThreads, int64_t cap = 1 << 30) {
    int64_t g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<unsigned>(g);
}

// Page-locked host memory for the small state record a solve reads back after every chunk
// (at least `bytes`, 16-byte aligned): one block per host thread, allocated on its first use
// and kept for the life of the process.  Freeing page-locked memory (cudaFreeHost) took from
// 5 ms to over a second a call on a shared machine, more than a small LP's whole solve, when
// every solve allocated and freed its own.  A thread runs one solve at a time, and a solve
// uses one record, so the block is never shared.  The block is checked before each use: after a
// reset of the context that allocated it (cudaDeviceReset), a new one is taken.  nullptr if the
// allocation fails.
void* pinned_scratch(size_t bytes);

// Programmatic dependent launch.  The SpMV kernels are launched with programmatic stream
// serialization: the next kernel's CTAs may be scheduled while the previous kernel in the
// stream is still draining, which hides most of the launch gap between the two SpMVs of an
// iteration when the SpMVs themselves take a few microseconds.  Every kernel launched that way
// runs pdl_enter() before anything else: griddepcontrol.wait returns once the previous kernel
// has completed and its writes are visible, so nothing is read or written early, and a kernel
// that then returns at once has still waited (the kernel after it sees everything before it).
// launch_dependents then lets the next kernel be scheduled.  In a kernel launched without the
// attribute both instructions return at once.  VAJRA_PDL=0 in the environment launches the
// SpMV kernels without it.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// False when VAJRA_PDL=0 (read once per process).
bool pdl_enabled();

// <<<grid, block, smem, st>>> with programmatic stream serialization; errors are left for
// cudaGetLastError, as with <<<>>>.
template <typename... Params, typename... Args>
inline void launch_chained(void (*kernel)(Params...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                           Args&&... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Device blocks go through a process-wide cache keyed by (device, context, size class): a
// released block is handed out again only after the work queued before its release has
// finished (the ordering cudaFree gives; see ReleaseStreamScope) and is kept for the next
// request of its size class on that device, which then needs no driver call.  A solve
// allocates and releases the same few dozen buffers every run; on shared machines those driver
// calls were where the occasional multi-second host stalls of a solve showed up.  At most
// block_cache_limit() bytes are kept; beyond that blocks are freed.  Cached blocks keep their
// old contents (so does fresh cudaMalloc memory: nothing may assume zeros).
//
// The context is the driver's unique id of the device's current context (`ctx` below).  A
// reset of the device (cudaDeviceReset) ends that context and frees every block it held: the
// cache then drops, without freeing or reusing, every block of an older context of the device,
// and a buffer released after the reset that was allocated before it is dropped as well (its
// address may already belong to a new allocation).
cudaError_t cached_alloc(void** p, size_t bytes, int* device, unsigned long long* ctx);
void cached_release(void* p, size_t bytes, int device, unsigned long long ctx);
// The driver's id of the calling thread's current context (0 if it cannot be read).
unsigned long long current_context_id();
// While alive, blocks the calling thread releases on `device` are ordered after the work
// queued so far on `st` (the stream every kernel of the current solve runs on) by an event,
// instead of by a device-wide synchronisation.
class ReleaseStreamScope {
public:
    ReleaseStreamScope(cudaStream_t st, int device);
    ~ReleaseStreamScope();
    ReleaseStreamScope(const ReleaseStreamScope&) = delete;
    ReleaseStreamScope& operator=(const ReleaseStreamScope&) = delete;
private:
    cudaStream_t prev_stream_;
    int prev_device_;
};
size_t block_cache_limit();
size_t release_cached_blocks(int device);

// Owning device allocation.  Moves only; releases on destruction.
template <typename T>
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    ~DeviceBuffer() { reset(); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_), dev_(o.dev_), ctx_(o.ctx_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) { reset(); p_ = o.p_; n_ = o.n_; dev_ = o.dev_; ctx_ = o.ctx_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    // Every allocation carries kPad spare elements, so 128-bit vector loads of the last
    // aligned group of four never leave the allocation (their extra lanes are masked).
    static constexpr size_t kPad = 16;
    vajra_status alloc(size_t n) {
        reset();
        if (n == 0) n = 1;   // keep a valid pointer for empty extents
        void* p = nullptr;
        cudaError_t e = cached_alloc(&p, (n + kPad) * sizeof(T), &dev_, &ctx_);
        if (e != cudaSuccess) { p_ = nullptr; return cuda_status(e, "cudaMalloc", __FILE__, __LINE__); }
        p_ = static_cast<T*>(p);
        n_ = n;
        return VAJRA_OK;
    }
    void reset() noexcept {
        if (p_) cached_release(p_, (n_ + kPad) * sizeof(T), dev_, ctx_);
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const noexcept { return p_; }
    size_t size() const noexcept { return n_; }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
    int dev_ = 0;
    unsigned long long ctx_ = 0;   // the context the block was allocated in
};

// ---------------------------------------------------------------------------------------
// Deterministic reductions.  A warp reduces with an xor butterfly, a block combines its
// warps in warp order through shared memory, and a grid combines per-block partials in
// block order in a second single-CTA pass.  Same inputs -> same bits on every run.
// ---------------------------------------------------------------------------------------
struct OpSum {
    template <typename T> __device__ static T apply(T a, T b) { return a + b; }
    template <typename T> __device__ static T identity() { return T(0); }
};
struct OpMax {   // ignores NaN like `if (v > cur) cur = v`
    template <typename T> __device__ static T apply(T a, T b) { return (b > a) ? b : a; }
    template <typename T> __device__ static T identity() { return T(0); }
};

template <class Op, typename T>
__device__ __forceinline__ T warp_reduce(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = Op::apply(v, __shfl_xor_sync(0xffffffffu, v, off));
    return v;
}

// Reduces NV values per thread across the block; the result is valid in thread 0.
// `smem` holds 32 slots per value (checked at compile time).  All threads of the block must
// call it.
template <class Op, typename T, int NV, int S>
__device__ __forceinline__ void block_reduce(T (&v)[NV], T (&smem)[S]) {
    static_assert(S >= NV * 32, "block_reduce needs 32 shared slots per reduced value");
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_reduce<Op>(v[q]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) smem[q * 32 + warp] = v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            T acc = smem[q * 32];
            for (int w = 1; w < nwarps; ++w) acc = Op::apply(acc, smem[q * 32 + w]);
            v[q] = acc;
        }
    }
    __syncthreads();
}

}  // namespace vajra
