// C ABI of libvajra_pdhg (include/vajra_pdhg.h).  Every entry point returns a status and
// never lets an exception escape.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "solver.cuh"

namespace vajra {

namespace {
thread_local char g_error[512] = "";
thread_local vajra_timing g_last_timing = {};
thread_local int64_t g_launches = 0;
}  // namespace

int64_t& launch_count() { return g_launches; }

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

const char* last_error() { return g_error; }

vajra_status cuda_status(cudaError_t e, const char* what, const char* file, int line) {
    set_error("CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
    if (e == cudaErrorMemoryAllocation) return VAJRA_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return VAJRA_ERR_NO_DEVICE;
    return VAJRA_ERR_CUDA;
}

// ----- device block cache (common.cuh) -------------------------------------------------
namespace {
// A cached block and, when it was released while a solve's stream was current, an event
// recorded on that stream at release: the block is handed out again only once the event has
// completed (every kernel queued before the release has finished).  Without an event the
// release waited for the whole device instead.
struct CachedBlock {
    void* p;
    cudaEvent_t ready;
};
// (device, context id, size class)
using BlockKey = std::tuple<int, unsigned long long, size_t>;
struct BlockCache {
    std::mutex mu;
    std::map<BlockKey, std::vector<CachedBlock>> free_blocks;
    std::map<int, unsigned long long> device_ctx;   // the newest context seen per device
    size_t cached_bytes = 0;
};
BlockCache& block_cache() {
    static BlockCache* c = new BlockCache();   // never destroyed: blocks live until exit
    return *c;
}
// Size classes: powers of two up to 1 MiB, whole MiB above.
size_t size_class(size_t bytes) {
    constexpr size_t kMiB = size_t(1) << 20;
    if (bytes >= kMiB) return (bytes + kMiB - 1) / kMiB * kMiB;
    size_t c = 512;
    while (c < bytes) c <<= 1;
    return c;
}
thread_local cudaStream_t g_release_stream = nullptr;
thread_local int g_release_device = -1;
}  // namespace

ReleaseStreamScope::ReleaseStreamScope(cudaStream_t st, int device)
    : prev_stream_(g_release_stream), prev_device_(g_release_device) {
    g_release_stream = st;
    g_release_device = device;
}
ReleaseStreamScope::~ReleaseStreamScope() {
    g_release_stream = prev_stream_;
    g_release_device = prev_device_;
}

// 16 GiB unless VAJRA_BLOCK_CACHE_MB says otherwise (0 keeps no blocks: every release frees).
size_t block_cache_limit() {
    static const size_t limit = [] {
        const char* v = std::getenv("VAJRA_BLOCK_CACHE_MB");
        if (v && *v) {
            char* end = nullptr;
            const unsigned long long mb = std::strtoull(v, &end, 10);
            if (end && *end == '\0') return static_cast<size_t>(mb) << 20;
        }
        return size_t(16) << 30;
    }();
    return limit;
}

unsigned long long current_context_id() {
    // cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (CUDA 12.0 forms),
    // so the library needs no link against the driver library
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx) {
        cudaFree(nullptr);   // makes the current device's primary context current
        cudaGetLastError();
        if (get_current(&ctx) != 0 || !ctx) return 0;
    }
    unsigned long long id = 0;
    return get_id(ctx, &id) == 0 ? id : 0;
}

namespace {
// Drops the cached blocks of `device` that belong to a context other than `ctx` (caller holds
// the lock).  Only a reset replaces a device's context, and the reset freed those blocks and
// ended their events, so they are forgotten, neither freed nor waited on.
void forget_old_contexts(BlockCache& c, int device, unsigned long long ctx) {
    auto seen = c.device_ctx.find(device);
    if (seen != c.device_ctx.end() && seen->second == ctx) return;
    c.device_ctx[device] = ctx;
    for (auto it = c.free_blocks.begin(); it != c.free_blocks.end();) {
        if (std::get<0>(it->first) == device && std::get<1>(it->first) != ctx) {
            c.cached_bytes -= std::get<2>(it->first) * it->second.size();
            it = c.free_blocks.erase(it);
        } else {
            ++it;
        }
    }
}
}  // namespace

// Frees every cached block of `device` (all devices for device < 0); returns the bytes freed.
size_t release_cached_blocks(int device) {
    BlockCache& c = block_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    size_t freed = 0;
    int cur = 0;
    const bool have_cur = cudaGetDevice(&cur) == cudaSuccess;
    for (auto it = c.free_blocks.begin(); it != c.free_blocks.end();) {
        const int dev = std::get<0>(it->first);
        const size_t cls = std::get<2>(it->first);
        if (device >= 0 && dev != device) { ++it; continue; }
        cudaSetDevice(dev);
        if (std::get<1>(it->first) == current_context_id()) {
            for (const CachedBlock& b : it->second) {
                if (b.ready) { cudaEventSynchronize(b.ready); cudaEventDestroy(b.ready); }
                cudaFree(b.p);
                freed += cls;
            }
        }   // else: a context that a reset ended; its blocks are gone already
        c.cached_bytes -= cls * it->second.size();
        it = c.free_blocks.erase(it);
    }
    if (have_cur) cudaSetDevice(cur);
    return freed;
}

cudaError_t cached_alloc(void** p, size_t bytes, int* device, unsigned long long* ctx) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    *device = dev;
    const unsigned long long id = current_context_id();
    *ctx = id;
    const size_t cls = size_class(bytes);
    if (id == 0) return cudaMalloc(p, cls);   // context unknown: no caching (see cached_release)
    CachedBlock b{nullptr, nullptr};
    {
        BlockCache& c = block_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        forget_old_contexts(c, dev, id);
        auto it = c.free_blocks.find(BlockKey{dev, id, cls});
        if (it != c.free_blocks.end() && !it->second.empty()) {
            b = it->second.back();
            it->second.pop_back();
            c.cached_bytes -= cls;
        }
    }
    if (b.p) {
        if (b.ready) {   // usually complete already; otherwise wait for the releasing stream
            cudaError_t w = cudaEventSynchronize(b.ready);
            cudaEventDestroy(b.ready);
            if (w != cudaSuccess) { cudaFree(b.p); return w; }
        }
        *p = b.p;
        return cudaSuccess;
    }
    return cudaMalloc(p, cls);
}

void cached_release(void* p, size_t bytes, int device, unsigned long long ctx) {
    const size_t cls = size_class(bytes);
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return;
    if (cur != device) cudaSetDevice(device);
    if (ctx == 0) {   // allocated while the context id could not be read: not cached
        cudaFree(p);
        cudaGetLastError();
        if (cur != device) cudaSetDevice(cur);
        return;
    }
    if (current_context_id() != ctx) {
        // allocated in a context that a reset has ended: the block was freed with it, and its
        // address may belong to a new allocation by now
        if (cur != device) cudaSetDevice(cur);
        return;
    }
    // Nothing still queued on the device may touch the block once it is handed out again:
    // an event on the releasing solve's stream (all of a solve's kernels use it), else the
    // whole device.  Not inside a stream capture, where neither works: the block is freed.
    cudaEvent_t ready = nullptr;
    bool usable = false;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (g_release_stream && g_release_device == device &&
        cudaStreamIsCapturing(g_release_stream, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone &&
        cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) == cudaSuccess) {
        usable = cudaEventRecord(ready, g_release_stream) == cudaSuccess;
        if (!usable) { cudaEventDestroy(ready); ready = nullptr; }
    }
    if (!usable) {
        cudaGetLastError();
        usable = cudaDeviceSynchronize() == cudaSuccess;
    }
    bool kept = false;
    if (usable) {
        BlockCache& c = block_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        forget_old_contexts(c, device, ctx);
        if (c.cached_bytes + cls <= block_cache_limit()) {
            c.free_blocks[BlockKey{device, ctx, cls}].push_back(CachedBlock{p, ready});
            c.cached_bytes += cls;
            kept = true;
        }
    }
    if (!kept) {
        if (ready) cudaEventDestroy(ready);
        cudaFree(p);
    }
    if (cur != device) cudaSetDevice(cur);
}

int sm_count() {
    static std::mutex mu;
    static std::map<int, int> counts;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    auto it = counts.find(dev);
    if (it != counts.end()) return it->second;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    counts.emplace(dev, sms);
    return sms;
}

void* pinned_scratch(size_t bytes) {
    struct Block { void* p = nullptr; size_t size = 0; };
    thread_local Block b;   // never freed: see the declaration
    if (b.p) {
        // A reset of the context that allocated it (cudaDeviceReset) releases the block: then
        // the address is no longer page-locked host memory and a new block is taken.
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, b.p) != cudaSuccess || a.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            b = Block{};
        }
    }
    if (b.size < bytes) {
        const size_t want = bytes < 4096 ? 4096 : bytes;
        void* p = nullptr;
        if (cudaHostAlloc(&p, want, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        if (b.p) cudaFreeHost(b.p);   // only when a larger record is asked for
        b.p = p;
        b.size = want;
    }
    return b.p;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("VAJRA_PDL");
        return !(e && std::strcmp(e, "0") == 0);
    }();
    return on;
}

void copy_out_vector(double* dst, const double* dev, int count, cudaStream_t st) {
    if (dst && count > 0) cudaMemcpyAsync(dst, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, st);
}

// Closed forms (no device work): n == 0 and m == 0 follow pdhg.cpp:88-127.
bool solve_trivial(const vajra_pdhg* h, vajra_result* r) {
    const int m = h->m, n = h->n;
    const bool is_max = h->sense != 0;
    if (n != 0 && m != 0) return false;
    auto fill = [](double* p, int k) { if (p) for (int i = 0; i < k; ++i) p[i] = 0.0; };
    fill(r->col_value, n);
    fill(r->row_value, m);
    fill(r->row_dual, m);
    fill(r->col_dual, n);
    r->iterations = 0;
    r->converged = 1;
    r->status = VAJRA_SOLVE_OPTIMAL;
    if (n == 0) {
        r->objective_value = h->objective_offset;
        std::snprintf(r->status_message, sizeof(r->status_message), "no columns: closed form");
        return true;
    }
    double obj = h->objective_offset;
    for (int j = 0; j < n; ++j) {
        const double cj = is_max ? -h->h_c[j] : h->h_c[j];
        const double lj = h->h_cl[j], uj = h->h_cu[j];
        double xj;
        if (cj > 1e-7) {
            if (lj <= -1e20) { r->status = VAJRA_SOLVE_UNBOUNDED; r->converged = 0; break; }
            xj = lj;
        } else if (cj < -1e-7) {
            if (uj >= 1e20) { r->status = VAJRA_SOLVE_UNBOUNDED; r->converged = 0; break; }
            xj = uj;
        } else {
            xj = (lj > 0.0) ? lj : ((uj < 0.0) ? uj : 0.0);
        }
        if (r->col_value) r->col_value[j] = xj;
        if (r->col_dual) r->col_dual[j] = h->h_c[j];
        obj += h->h_c[j] * xj;
    }
    r->objective_value = obj;
    r->dual_objective = obj;
    std::snprintf(r->status_message, sizeof(r->status_message), "no rows: closed form");
    return true;
}

// Device validation of the index array: every row index in [0, m), ascending within a
// column.  col_ptr has already been checked on the host, so every access is in bounds.
__global__ void k_validate_rows(int n, int m, const int64_t* __restrict__ col_ptr,
                                const int32_t* __restrict__ row_idx, int* __restrict__ bad) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int prev = -1;
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
        const int r = row_idx[k];
        if (r < 0 || r >= m) { atomicOr(bad, 1); return; }
        if (r <= prev) { atomicOr(bad, 2); return; }
        prev = r;
    }
}

static vajra_status validate_host(const vajra_lp* lp) {
    if (!lp) { set_error("lp is NULL"); return VAJRA_ERR_INVALID_ARGUMENT; }
    const int m = lp->num_rows, n = lp->num_cols;
    if (m < 0 || n < 0) { set_error("negative dimensions"); return VAJRA_ERR_INVALID_ARGUMENT; }
    if (!lp->col_ptr || (n > 0 && (!lp->c || !lp->col_lower || !lp->col_upper)) ||
        (m > 0 && (!lp->row_lower || !lp->row_upper))) {
        set_error("NULL array in vajra_lp");
        return VAJRA_ERR_INVALID_ARGUMENT;
    }
    if (lp->col_ptr[0] != 0) { set_error("col_ptr[0] != 0"); return VAJRA_ERR_INVALID_ARGUMENT; }
    for (int j = 0; j < n; ++j)
        if (lp->col_ptr[j + 1] < lp->col_ptr[j]) { set_error("col_ptr decreases at column %d", j); return VAJRA_ERR_INVALID_ARGUMENT; }
    if (lp->col_ptr[n] != lp->nnz) { set_error("col_ptr[n] != nnz"); return VAJRA_ERR_INVALID_ARGUMENT; }
    if (lp->nnz > 0 && (!lp->row_idx || !lp->values)) { set_error("NULL row_idx / values"); return VAJRA_ERR_INVALID_ARGUMENT; }
    if (lp->nnz > 0 && m == 0) { set_error("nonzeros in a matrix without rows"); return VAJRA_ERR_INVALID_ARGUMENT; }
    // Model::validate (src/engine/model.cpp:35-150): NaN or crossed bounds are model errors.
    for (int j = 0; j < n; ++j) {
        const double l = lp->col_lower[j], u = lp->col_upper[j];
        if (std::isnan(l) || std::isnan(u) || l > u + 1e-11) { set_error("column %d has NaN or crossed bounds", j); return VAJRA_ERR_INVALID_ARGUMENT; }
    }
    for (int i = 0; i < m; ++i) {
        const double l = lp->row_lower[i], u = lp->row_upper[i];
        if (std::isnan(l) || std::isnan(u) || l > u + 1e-11) { set_error("row %d has NaN or crossed bounds", i); return VAJRA_ERR_INVALID_ARGUMENT; }
    }
    return VAJRA_OK;
}

static vajra_status validate_device(const vajra_pdhg* h) {
    if (h->nnz == 0 || h->n == 0) return VAJRA_OK;
    DeviceBuffer<int> bad;
    VJ_TRY(bad.alloc(1));
    VJ_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), h->stream));
    k_validate_rows<<<grid_for(h->n), kThreads, 0, h->stream>>>(h->n, h->m, h->lp.col_ptr.get(), h->lp.row_idx.get(), bad.get());
    VJ_LAUNCH_CHECK();
    int hb = 0;
    VJ_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    VJ_CUDA(cudaStreamSynchronize(h->stream));
    if (hb & 1) { set_error("row index out of range"); return VAJRA_ERR_INVALID_ARGUMENT; }
    if (hb & 2) { set_error("row indices not strictly ascending within a column (duplicates or unsorted)"); return VAJRA_ERR_INVALID_ARGUMENT; }
    return VAJRA_OK;
}

static void fail_result(vajra_result* r, vajra_status s) {
    if (!r) return;
    r->status = (s == VAJRA_ERR_NO_DEVICE) ? VAJRA_SOLVE_UNSUPPORTED
              : (s == VAJRA_ERR_INVALID_ARGUMENT) ? VAJRA_SOLVE_MODEL_ERROR : VAJRA_SOLVE_NUMERICAL_ERROR;
    std::snprintf(r->status_message, sizeof(r->status_message), "%s: %s", vajra_status_string(s), last_error());
}

}  // namespace vajra

using namespace vajra;

extern "C" {

int32_t vajra_abi_version(void) { return VAJRA_ABI_VERSION; }

const char* vajra_status_string(vajra_status s) {
    switch (s) {
        case VAJRA_OK: return "ok";
        case VAJRA_ERR_INVALID_ARGUMENT: return "invalid argument";
        case VAJRA_ERR_NO_DEVICE: return "no CUDA device";
        case VAJRA_ERR_CUDA: return "CUDA error";
        case VAJRA_ERR_OUT_OF_MEMORY: return "out of device memory";
        case VAJRA_ERR_WAIT_TIMEOUT: return "device wait timed out (reserved)";
        case VAJRA_ERR_INTERNAL: return "internal error";
        default: return "unknown status";
    }
}

void vajra_default_opts(vajra_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->algorithm = VAJRA_ALGO_HALPERN;
    o->precision = VAJRA_PREC_MIXED;
    o->tolerance = 1e-6;
    o->gap_tolerance = 1e-6;
    o->time_limit = 1e20;
    o->iteration_limit = 1000000;
    o->check_frequency = 64;
    o->enable_scaling = 1;
    o->pock_chambolle = 1;
    o->ruiz_iterations = 10;
    o->reflection = 1.0;
    o->mixed_switch_tolerance = 2e-6;
    o->mixed_reflection = 0.8;
    o->device = 0;
    o->autotune = 1;
    o->verbose = 0;
    o->mixed_stall_checks = 20;
    o->restart_sufficient = 0.2;
    o->restart_necessary = 0.8;
    o->restart_artificial = 0.36;
    o->primal_weight_smoothing = 0.5;
    o->step_safety = 0.99;
    o->handover_mode = -1;
}

// Static properties of `device`, read once per device (cudaGetDeviceProperties takes
// milliseconds).  VAJRA_ERR_NO_DEVICE when the ordinal names no device.
static vajra_status cached_props(int32_t device, cudaDeviceProp* prop) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0 || device < 0 || device >= count) {
        cudaGetLastError();
        return VAJRA_ERR_NO_DEVICE;
    }
    static std::mutex props_mu;
    static std::map<int, cudaDeviceProp> props_cache;
    std::lock_guard<std::mutex> lock(props_mu);
    auto it = props_cache.find(device);
    if (it == props_cache.end()) {
        if (cudaGetDeviceProperties(prop, device) != cudaSuccess) {
            cudaGetLastError();
            return VAJRA_ERR_CUDA;
        }
        props_cache.emplace(device, *prop);
    } else {
        *prop = it->second;
    }
    return VAJRA_OK;
}

// The check every solve entry makes: the ordinal names a device whose properties can be read.
// Unlike vajra_probe_device it asks the driver for no free-memory figure, which took from
// 0.2 to 7 ms a call, a fifth of a small LP's whole solve.
static vajra_status device_usable(int32_t device, cudaDeviceProp* prop) {
    return cached_props(device, prop);
}

vajra_status vajra_probe_device(int32_t device, vajra_device_info* info) {
    if (!info) return VAJRA_ERR_INVALID_ARGUMENT;
    std::memset(info, 0, sizeof(*info));
    cudaDeviceProp prop;
    const vajra_status ps = cached_props(device, &prop);
    if (ps == VAJRA_ERR_NO_DEVICE) {
        std::snprintf(info->device_name, sizeof(info->device_name), "None (No CUDA devices found)");
        return ps;
    }
    if (ps != VAJRA_OK) {
        std::snprintf(info->device_name, sizeof(info->device_name), "Error querying CUDA device");
        return ps;
    }
    info->available = 1;
    std::snprintf(info->device_name, sizeof(info->device_name), "%s", prop.name);
    info->compute_capability_major = prop.major;
    info->compute_capability_minor = prop.minor;
    info->multi_processor_count = prop.multiProcessorCount;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
        info->free_vram_bytes = fr;
        info->total_vram_bytes = tot;
    } else {
        info->total_vram_bytes = prop.totalGlobalMem;
    }
    cudaSetDevice(prev);
    return VAJRA_OK;
}

int32_t vajra_is_cuda_available(void) {
    vajra_device_info info;
    return vajra_probe_device(0, &info) == VAJRA_OK ? 1 : 0;
}

void vajra_last_timing(vajra_timing* out) {
    if (out) *out = g_last_timing;
}

vajra_status vajra_pdhg_create(const vajra_lp* lp, const vajra_opts* opts, vajra_pdhg** handle) {
    if (!handle) return VAJRA_ERR_INVALID_ARGUMENT;
    *handle = nullptr;
    vajra_status s = validate_host(lp);
    if (s != VAJRA_OK) return s;
    vajra_opts o;
    if (opts) o = *opts; else vajra_default_opts(&o);
    if (o.algorithm != VAJRA_ALGO_REFERENCE && o.algorithm != VAJRA_ALGO_HALPERN) {
        set_error("unknown algorithm %d", o.algorithm);
        return VAJRA_ERR_INVALID_ARGUMENT;
    }
    const auto t_probe = Clock::now();
    cudaDeviceProp prop;
    s = device_usable(o.device, &prop);
    if (s != VAJRA_OK) { set_error("no usable CUDA device %d (no CPU fallback)", o.device); return VAJRA_ERR_NO_DEVICE; }
    if (o.verbose) std::fprintf(stderr, "[vajra] create: device probe %.1f ms\n", 1e3 * seconds_since(t_probe));
    auto t0 = Clock::now();
    vajra_pdhg* h = new (std::nothrow) vajra_pdhg();
    if (!h) return VAJRA_ERR_INTERNAL;
    h->opts = o;
    h->device = o.device;
    h->m = lp->num_rows;
    h->n = lp->num_cols;
    h->nnz = lp->nnz;
    h->sense = lp->sense;
    h->objective_offset = lp->objective_offset;
    auto fail = [&](vajra_status st) { vajra_pdhg_destroy(h); return st; };
    if (cudaSetDevice(o.device) != cudaSuccess) return fail(cuda_status(cudaGetLastError(), "cudaSetDevice", __FILE__, __LINE__));
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_status(e, "cudaStreamCreate", __FILE__, __LINE__));
    ReleaseStreamScope release_scope(h->stream, o.device);
    if (h->m == 0 || h->n == 0 || (h->nnz == 0 && o.algorithm == VAJRA_ALGO_HALPERN)) {
        h->h_c.assign(lp->c, lp->c + h->n);
        h->h_cl.assign(lp->col_lower, lp->col_lower + h->n);
        h->h_cu.assign(lp->col_upper, lp->col_upper + h->n);
        h->h_rl.assign(lp->row_lower, lp->row_lower + h->m);
        h->h_ru.assign(lp->row_upper, lp->row_upper + h->m);
    }
    if (h->m > 0 && h->n > 0) {
        s = upload_lp(lp, h->lp, h->stream);
        if (s != VAJRA_OK) return fail(s);
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return fail(cuda_status(e, "upload", __FILE__, __LINE__));
        h->transfers = 8;
        s = validate_device(h);
        if (s != VAJRA_OK) return fail(s);
    }
    h->upload_time_sec = seconds_since(t0);
    if (o.verbose) std::fprintf(stderr, "[vajra] create: stream, upload, checks %.1f ms\n", 1e3 * h->upload_time_sec);
    *handle = h;
    return VAJRA_OK;
}

vajra_status vajra_pdhg_destroy(vajra_pdhg* h) {
    if (!h) return VAJRA_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    ReleaseStreamScope release_scope(h->stream, h->device);
    {
        vajra::DeviceLp empty, empty_ordered;
        vajra::LpOrder empty_order;
        std::swap(h->lp, empty);   // frees device memory before the stream goes
        std::swap(h->lp_ordered, empty_ordered);
        std::swap(h->order, empty_order);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return VAJRA_OK;
}

// Closed form for nnz == 0 (HALPERN): rows decouple; a row is feasible iff 0 in [l, u].
static vajra_status solve_no_nonzeros(vajra_pdhg* h, vajra_result* r) {
    const int m = h->m, n = h->n;
    for (int i = 0; i < m; ++i) {
        if (h->h_rl[i] > 1e-7 || h->h_ru[i] < -1e-7) {
            r->status = 2;   // INFEASIBLE
            std::snprintf(r->status_message, sizeof(r->status_message), "row %d: 0 outside its bounds", i);
            return VAJRA_OK;
        }
    }
    vajra_pdhg tmp;
    tmp.m = 0; tmp.n = n; tmp.sense = h->sense; tmp.objective_offset = h->objective_offset;
    tmp.h_c = h->h_c; tmp.h_cl = h->h_cl; tmp.h_cu = h->h_cu;
    double* rv = r->row_value; double* rd = r->row_dual;
    r->row_value = nullptr; r->row_dual = nullptr;
    solve_trivial(&tmp, r);
    r->row_value = rv; r->row_dual = rd;
    if (rv) for (int i = 0; i < m; ++i) rv[i] = 0.0;
    if (rd) for (int i = 0; i < m; ++i) rd[i] = 0.0;
    return VAJRA_OK;
}

vajra_status vajra_pdhg_run(vajra_pdhg* h, vajra_result* r) {
    if (!h || !r) return VAJRA_ERR_INVALID_ARGUMENT;
    const auto t0 = Clock::now();
    r->status = VAJRA_SOLVE_NOT_SOLVED;
    r->status_message[0] = '\0';
    vajra_status s = VAJRA_OK;
    const int64_t launches0 = launch_count();
    ReleaseStreamScope release_scope(h->stream, h->device);
    if (cudaSetDevice(h->device) != cudaSuccess) {
        s = cuda_status(cudaGetLastError(), "cudaSetDevice", __FILE__, __LINE__);
    } else if (solve_trivial(h, r)) {
        s = VAJRA_OK;
    } else if (h->nnz == 0 && h->opts.algorithm == VAJRA_ALGO_HALPERN) {
        s = solve_no_nonzeros(h, r);
    } else if (h->opts.algorithm == VAJRA_ALGO_REFERENCE) {
        s = run_reference(h, r);
    } else {
        s = run_halpern(h, r);
    }
    if (s != VAJRA_OK) {
        fail_result(r, s);
        cudaGetLastError();
        if (h->stream) cudaStreamSynchronize(h->stream);
    }
    r->kernel_launches = launch_count() - launches0;
    r->upload_time_sec = h->upload_time_sec;
    r->total_time_sec = seconds_since(t0) + h->upload_time_sec;
    r->host_device_transfers = h->transfers;
    g_last_timing.upload_time_sec = r->upload_time_sec;
    g_last_timing.iteration_time_sec = r->iteration_time_sec;
    g_last_timing.download_time_sec = r->download_time_sec;
    g_last_timing.total_time_sec = r->total_time_sec;
    g_last_timing.host_device_transfers = r->host_device_transfers;
    g_last_timing.iterations = r->iterations;
    cudaDeviceProp prop;
    if (cached_props(h->device, &prop) == VAJRA_OK)
        std::snprintf(g_last_timing.device_name, sizeof(g_last_timing.device_name), "%s", prop.name);
    std::snprintf(g_last_timing.kernel_mode, sizeof(g_last_timing.kernel_mode), "%s",
                  h->opts.algorithm == VAJRA_ALGO_REFERENCE ? "sm100_exact_fp64"
                  : h->opts.precision == VAJRA_PREC_MIXED ? "sm100_halpern_mixed" : "sm100_halpern_fp64");
    return s;
}

vajra_status vajra_pdhg_solve(const vajra_lp* lp, const vajra_opts* opts, vajra_result* r) {
    if (!r) return VAJRA_ERR_INVALID_ARGUMENT;
    const auto t0 = Clock::now();
    vajra_pdhg* h = nullptr;
    vajra_status s = vajra_pdhg_create(lp, opts, &h);
    if (s != VAJRA_OK) {
        fail_result(r, s);
        return s;
    }
    const double t_create = seconds_since(t0);
    s = vajra_pdhg_run(h, r);
    const double t_run = seconds_since(t0);
    const bool verbose = h->opts.verbose != 0;
    vajra_pdhg_destroy(h);
    r->total_time_sec = seconds_since(t0);
    if (verbose)
        std::fprintf(stderr, "[vajra] solve: create %.1f ms, run %.1f ms, destroy %.1f ms\n", 1e3 * t_create,
                     1e3 * (t_run - t_create), 1e3 * (r->total_time_sec - t_run));
    g_last_timing.total_time_sec = r->total_time_sec;
    return s;
}

vajra_status vajra_scale_lp(const vajra_lp* lp, const vajra_opts* opts, double* row_scale, double* col_scale,
                            double* values, double* c, double* col_lower, double* col_upper, double* row_lower,
                            double* row_upper) {
    vajra_opts o;
    if (opts) o = *opts; else vajra_default_opts(&o);
    o.algorithm = VAJRA_ALGO_HALPERN;
    vajra_pdhg* h = nullptr;
    vajra_status s = vajra_pdhg_create(lp, &o, &h);
    if (s != VAJRA_OK) return s;
    struct Guard { vajra_pdhg* h; ~Guard() { vajra_pdhg_destroy(h); } } guard{h};
    const int m = h->m, n = h->n;
    if (m == 0 || n == 0) { set_error("vajra_scale_lp: an LP without rows or columns is not scaled"); return VAJRA_ERR_INVALID_ARGUMENT; }
    cudaStream_t st = h->stream;
    Prepared p;
    DeviceBuffer<SetupState> sst;
    VJ_TRY(sst.alloc(1));
    VJ_TRY(build_csr(h->lp, p, st));
    ScalingOpts so;
    so.enable = o.enable_scaling != 0;
    so.ruiz_iterations = o.ruiz_iterations > 0 ? o.ruiz_iterations : 10;
    so.ruiz_tolerance = 0.05;
    so.pock_chambolle = o.pock_chambolle != 0;
    so.negate_c = h->sense != 0;
    VJ_TRY(prepare_scaled(h->lp, p, so, sst.get(), st));
    auto out = [&](double* dst, const DeviceBuffer<double>& src, int64_t k) -> vajra_status {
        if (dst && k > 0) VJ_CUDA(cudaMemcpyAsync(dst, src.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, st));
        return VAJRA_OK;
    };
    VJ_TRY(out(row_scale, p.row_scale, m));
    VJ_TRY(out(col_scale, p.col_scale, n));
    VJ_TRY(out(values, p.csc_val, h->nnz));
    VJ_TRY(out(c, p.c, n));
    VJ_TRY(out(col_lower, p.col_lower, n));
    VJ_TRY(out(col_upper, p.col_upper, n));
    VJ_TRY(out(row_lower, p.row_lower, m));
    VJ_TRY(out(row_upper, p.row_upper, m));
    VJ_CUDA(cudaStreamSynchronize(st));
    return VAJRA_OK;
}

int64_t vajra_release_cached_memory(int32_t device) {
    return static_cast<int64_t>(release_cached_blocks(device));
}

void vajra_default_unrolled_opts(vajra_unrolled_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->iterations = 2000;
    o->checkpoint_every = 100;
    o->precision = VAJRA_PREC_MIXED;
    o->enable_scaling = 1;
    o->step_safety = 0.95;
    o->device = 0;
}

vajra_status vajra_pdhg_unrolled(int32_t count, const vajra_lp* lps, const vajra_unrolled_opts* opts,
                                 const double* weights, double* loss, double* x_final, double* grad_c,
                                 double* grad_row_lower, double* grad_row_upper) {
    if (count <= 0 || !lps || !loss) { set_error("empty batch or NULL arrays"); return VAJRA_ERR_INVALID_ARGUMENT; }
    for (int i = 0; i < count; ++i) {
        vajra_status s = validate_host(&lps[i]);
        if (s == VAJRA_OK && (lps[i].num_rows == 0 || lps[i].num_cols == 0)) {
            set_error("instance %d has no rows or no columns", i);
            s = VAJRA_ERR_INVALID_ARGUMENT;
        }
        if (s != VAJRA_OK) return s;
    }
    vajra_unrolled_opts o;
    if (opts) o = *opts; else vajra_default_unrolled_opts(&o);
    if (o.iterations < 0) { set_error("negative iteration count"); return VAJRA_ERR_INVALID_ARGUMENT; }
    cudaDeviceProp prop;
    if (device_usable(o.device, &prop) != VAJRA_OK) {
        set_error("no usable CUDA device %d (no CPU fallback)", o.device);
        return VAJRA_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(o.device) != cudaSuccess) return cuda_status(cudaGetLastError(), "cudaSetDevice", __FILE__, __LINE__);
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamCreate", __FILE__, __LINE__);
    vajra_status s;
    {
        ReleaseStreamScope release_scope(st, o.device);
        s = run_unrolled(count, lps, o, weights, loss, x_final, grad_c, grad_row_lower, grad_row_upper, st);
    }
    if (s != VAJRA_OK) cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return s;
}

vajra_status vajra_pdhg_solve_batch(int32_t count, const vajra_lp* lps, const vajra_opts* opts,
                                    vajra_result* results) {
    if (count <= 0 || !lps || !results) { set_error("empty batch or NULL arrays"); return VAJRA_ERR_INVALID_ARGUMENT; }
    const auto t0 = Clock::now();
    for (int i = 0; i < count; ++i) {
        vajra_status s = validate_host(&lps[i]);
        if (s == VAJRA_OK && (lps[i].num_rows == 0 || lps[i].num_cols == 0)) {
            set_error("instance %d has no rows or no columns (solve it with vajra_pdhg_solve)", i);
            s = VAJRA_ERR_INVALID_ARGUMENT;
        }
        if (s != VAJRA_OK) {
            for (int k = 0; k < count; ++k) fail_result(&results[k], s);
            return s;
        }
    }
    vajra_opts o;
    if (opts) o = *opts; else vajra_default_opts(&o);
    cudaDeviceProp prop;
    if (device_usable(o.device, &prop) != VAJRA_OK) {
        set_error("no usable CUDA device %d (no CPU fallback)", o.device);
        for (int k = 0; k < count; ++k) fail_result(&results[k], VAJRA_ERR_NO_DEVICE);
        return VAJRA_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(o.device) != cudaSuccess) return cuda_status(cudaGetLastError(), "cudaSetDevice", __FILE__, __LINE__);
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamCreate", __FILE__, __LINE__);
    const int64_t launches0 = launch_count();
    double dev_time = 0.0;
    vajra_status s;
    {
        ReleaseStreamScope release_scope(st, o.device);
        s = run_batch(count, lps, o, results, st, &dev_time);
    }
    if (s != VAJRA_OK) {
        for (int k = 0; k < count; ++k) fail_result(&results[k], s);
        cudaGetLastError();
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    const double total = seconds_since(t0);
    const int64_t launches = launch_count() - launches0;
    for (int k = 0; k < count; ++k) {
        results[k].total_time_sec = total;
        results[k].device_time_sec = dev_time;
        results[k].kernel_launches = launches;
    }
    return s;
}

// ---------------------------------------------------------------------------------------
// kernel-level entry points
// ---------------------------------------------------------------------------------------
}  // extern "C"

namespace vajra {
namespace {

template <typename T>
struct EpiPlain {
    T* out;
    __device__ bool active() const { return true; }
    __device__ void operator()(int i, T s) const { out[i] = s; }
};

__global__ void k_dual_prox(int m, double sigma, const double* __restrict__ w, const double* __restrict__ rl,
                            const double* __restrict__ ru, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) y[i] = dual_prox_exact(y[i], w[i], sigma, rl[i], ru[i]);
}

__global__ void k_primal_prox(int n, double tau, const double* __restrict__ v, const double* __restrict__ c,
                              const double* __restrict__ cl, const double* __restrict__ cu, double* __restrict__ x,
                              double* __restrict__ xb) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double x_old = x[j];
    const double x_new = primal_prox_exact(x_old, v[j], c[j], tau, cl[j], cu[j]);
    x[j] = x_new;
    xb[j] = extrapolate_exact(x_new, x_old);
}

struct EpiStepDual {
    const double* rl; const double* ru; double* y; double* w; double sigma;
    __device__ bool active() const { return true; }
    __device__ void operator()(int i, double s) const {
        w[i] = s;
        y[i] = dual_prox_exact(y[i], s, sigma, rl[i], ru[i]);
    }
};

struct EpiStepPrimal {
    const double* c; const double* cl; const double* cu; double* x; double* xb; double* v; double tau;
    __device__ bool active() const { return true; }
    __device__ void operator()(int j, double s) const {
        v[j] = s;
        const double x_old = x[j];
        const double x_new = primal_prox_exact(x_old, s, c[j], tau, cl[j], cu[j]);
        x[j] = x_new;
        xb[j] = extrapolate_exact(x_new, x_old);
    }
};

// compute_diagnostics_device_kernel semantics (spmv_kernels.cuh:210-278) over a grid of CTAs
// with a deterministic two-stage reduction: each CTA writes its maxima (primal, dual, NaN flag)
// and its objective partial in a fixed order, then one CTA combines the partials in CTA order.
constexpr int kDiagQ = 4;
constexpr int kDiagMaxBlocks = 148 * 4;

__global__ void __launch_bounds__(kThreads)
k_diag_part(int m, int n, const double* __restrict__ ax, const double* __restrict__ rl, const double* __restrict__ ru,
            const double* __restrict__ aty, const double* __restrict__ c, const double* __restrict__ x,
            const double* __restrict__ y, const double* __restrict__ cl, const double* __restrict__ cu,
            double* __restrict__ part) {
    __shared__ double red_max[3 * 32];
    __shared__ double red_sum[32];
    double mx[3] = {0.0, 0.0, 0.0};   // primal, dual, nan flag
    double sm[1] = {0.0};
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double a = ax[i], yi = y[i];
        if (isnan(a) || isinf(a) || isnan(yi) || isinf(yi)) mx[2] = 1.0;
        double viol = 0.0;
        if (a < rl[i]) viol = rl[i] - a;
        if (a > ru[i]) viol = a - ru[i];
        if (viol > mx[0]) mx[0] = viol;
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const double xj = x[j], cj = c[j], atyj = aty[j];
        if (isnan(xj) || isinf(xj) || isnan(cj) || isinf(cj) || isnan(atyj) || isinf(atyj)) mx[2] = 1.0;
        const double lj = cl[j], uj = cu[j];
        double p = 0.0;
        if (xj < lj) p = lj - xj;
        if (xj > uj) p = xj - uj;
        if (p > mx[0]) mx[0] = p;
        const double dj = cj + atyj;
        double d = 0.0;
        if (xj > lj + 1e-5 && dj > 1e-6) d = dj;
        if (xj < uj - 1e-5 && dj < -1e-6) d = -dj;
        if (lj <= -1e20 && uj >= 1e20) d = fabs(dj);
        if (d > mx[1]) mx[1] = d;
        sm[0] += cj * xj;
    }
    block_reduce<OpMax, double, 3>(mx, red_max);
    block_reduce<OpSum, double, 1>(sm, red_sum);
    if (threadIdx.x == 0) {
        double* q = part + static_cast<size_t>(blockIdx.x) * kDiagQ;
        q[0] = mx[0]; q[1] = mx[1]; q[2] = mx[2]; q[3] = sm[0];
    }
}

__global__ void __launch_bounds__(1024)
k_diag_final(int nb, const double* __restrict__ part, vajra_device_diagnostics* out) {
    __shared__ double red_max[3 * 32];
    __shared__ double red_sum[32];
    double mx[3] = {0.0, 0.0, 0.0};
    double sm[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const double* q = part + static_cast<size_t>(b) * kDiagQ;
        for (int k = 0; k < 3; ++k) mx[k] = q[k] > mx[k] ? q[k] : mx[k];
        sm[0] += q[3];
    }
    block_reduce<OpMax, double, 3>(mx, red_max);
    block_reduce<OpSum, double, 1>(sm, red_sum);
    if (threadIdx.x == 0) {
        out->primal_residual = mx[0];
        out->dual_residual = mx[1];
        out->objective = sm[0];
        out->duality_gap = 0.0;
        out->converged = 0;
        out->numerical_error = mx[2] > 0.0 ? 1 : 0;
    }
}

// Gather-rate probe: sum of x[idx[k]] over all k, 4 independent gathers in flight per thread,
// grid-stride over a grid of resident CTAs; one partial per thread.  The iteration kernels'
// random gathers of the dense vector, without their value stream and epilogue.
__global__ void __launch_bounds__(kThreads)
k_gather_sum(int64_t n, const int32_t* __restrict__ idx, const float* __restrict__ x, float* __restrict__ out) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    int64_t k = t;
    for (; k + 3 * stride < n; k += 4 * stride) {
        const int i0 = __ldcs(idx + k), i1 = __ldcs(idx + k + stride), i2 = __ldcs(idx + k + 2 * stride),
                  i3 = __ldcs(idx + k + 3 * stride);
        a0 += __ldg(x + i0); a1 += __ldg(x + i1); a2 += __ldg(x + i2); a3 += __ldg(x + i3);
    }
    for (; k < n; k += stride) a0 += __ldg(x + __ldcs(idx + k));
    out[t] = (a0 + a1) + (a2 + a3);
}

CsrView exact_view(int rows, const int64_t* ptr, const int32_t* idx) {
    CsrView v;
    v.rows = rows;
    v.ptr = ptr;
    v.idx = idx;
    v.group = 1;
    return v;
}

}  // namespace
}  // namespace vajra

extern "C" {

#define VJ_STREAM(s) static_cast<cudaStream_t>(s)

vajra_status vajra_csr_spmv_f64(int32_t rows, const int64_t* row_ptr, const int32_t* col_idx, const double* values,
                                const double* x, double* y, void* stream) {
    if (rows < 0 || (rows > 0 && (!row_ptr || !col_idx || !values || !x || !y))) return VAJRA_ERR_INVALID_ARGUMENT;
    launch_spmv_exact<double, false>(exact_view(rows, row_ptr, col_idx), values, x, EpiPlain<double>{y}, VJ_STREAM(stream));
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}

vajra_status vajra_csr_spmv_f32(int32_t rows, const int64_t* row_ptr, const int32_t* col_idx, const float* values,
                                const float* x, float* y, void* stream) {
    if (rows < 0 || (rows > 0 && (!row_ptr || !col_idx || !values || !x || !y))) return VAJRA_ERR_INVALID_ARGUMENT;
    launch_spmv_exact<float, false>(exact_view(rows, row_ptr, col_idx), values, x, EpiPlain<float>{y}, VJ_STREAM(stream));
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}

vajra_status vajra_csc_spmv_transpose_f64(int32_t cols, const int64_t* col_ptr, const int32_t* row_idx,
                                          const double* values, const double* y, double* v, void* stream) {
    return vajra_csr_spmv_f64(cols, col_ptr, row_idx, values, y, v, stream);
}

vajra_status vajra_csc_spmv_transpose_f32(int32_t cols, const int64_t* col_ptr, const int32_t* row_idx,
                                          const float* values, const float* y, float* v, void* stream) {
    return vajra_csr_spmv_f32(cols, col_ptr, row_idx, values, y, v, stream);
}

vajra_status vajra_dual_prox_f64(int32_t rows, double sigma, const double* ax, const double* row_lower,
                                 const double* row_upper, double* y, void* stream) {
    if (rows < 0 || (rows > 0 && (!ax || !row_lower || !row_upper || !y))) return VAJRA_ERR_INVALID_ARGUMENT;
    if (rows > 0) k_dual_prox<<<grid_for(rows), kThreads, 0, VJ_STREAM(stream)>>>(rows, sigma, ax, row_lower, row_upper, y);
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}

vajra_status vajra_primal_prox_f64(int32_t cols, double tau, const double* aty, const double* c,
                                   const double* col_lower, const double* col_upper, double* x, double* x_bar,
                                   void* stream) {
    if (cols < 0 || (cols > 0 && (!aty || !c || !col_lower || !col_upper || !x || !x_bar))) return VAJRA_ERR_INVALID_ARGUMENT;
    if (cols > 0) k_primal_prox<<<grid_for(cols), kThreads, 0, VJ_STREAM(stream)>>>(cols, tau, aty, c, col_lower, col_upper, x, x_bar);
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}

vajra_status vajra_device_diagnostics_f64(int32_t rows, int32_t cols, const double* ax, const double* row_lower,
                                          const double* row_upper, const double* aty, const double* c,
                                          const double* x, const double* y, const double* col_lower,
                                          const double* col_upper, vajra_device_diagnostics* out, void* stream) {
    if (rows < 0 || cols < 0 || !out) return VAJRA_ERR_INVALID_ARGUMENT;
    cudaStream_t st = VJ_STREAM(stream);
    const int64_t work = rows > cols ? rows : cols;
    const int nb = static_cast<int>(grid_for(work > 0 ? work : 1, kThreads, kDiagMaxBlocks));
    // The block partials come from the stream-ordered pool on the caller's stream (no device
    // synchronisation, and usable inside a stream capture).
    double* part = nullptr;
    VJ_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * kDiagQ * nb, st));
    k_diag_part<<<nb, kThreads, 0, st>>>(rows, cols, ax, row_lower, row_upper, aty, c, x, y, col_lower, col_upper,
                                          part);
    k_diag_final<<<1, 1024, 0, st>>>(nb, part, out);
    const cudaError_t le = cudaGetLastError();
    VJ_CUDA(cudaFreeAsync(part, st));
    VJ_CUDA(le);
    note_launch(2);
    return VAJRA_OK;
}

vajra_status vajra_gather_probe_f32(int64_t count, const int32_t* idx, const float* x, float* partials,
                                    int32_t* threads, void* stream) {
    if (count < 0 || !threads || (count > 0 && (!idx || !x || !partials))) return VAJRA_ERR_INVALID_ARGUMENT;
    const int grid = sm_count() * (2048 / kThreads);
    if (*threads < grid * kThreads) { *threads = grid * kThreads; return VAJRA_ERR_INVALID_ARGUMENT; }
    *threads = grid * kThreads;
    k_gather_sum<<<grid, kThreads, 0, VJ_STREAM(stream)>>>(count, idx, x, partials);
    note_launch(1);
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}

vajra_status vajra_pdhg_step_f64(int32_t rows, int32_t cols, const int64_t* row_ptr, const int32_t* col_idx,
                                 const double* csr_values, const int64_t* col_ptr, const int32_t* row_idx,
                                 const double* csc_values, const double* row_lower, const double* row_upper,
                                 const double* c, const double* col_lower, const double* col_upper, double sigma,
                                 double tau, double* x, double* x_bar, double* y, double* w, double* v,
                                 void* stream) {
    if (rows < 0 || cols < 0) return VAJRA_ERR_INVALID_ARGUMENT;
    cudaStream_t st = VJ_STREAM(stream);
    launch_spmv_exact<double, false>(exact_view(rows, row_ptr, col_idx), csr_values, x_bar,
                                     EpiStepDual{row_lower, row_upper, y, w, sigma}, st);
    launch_spmv_exact<double, false>(exact_view(cols, col_ptr, row_idx), csc_values, y,
                                     EpiStepPrimal{c, col_lower, col_upper, x, x_bar, v, tau}, st);
    VJ_LAUNCH_CHECK();
    return VAJRA_OK;
}

}  // extern "C"
