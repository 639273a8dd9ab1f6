// s512_runtime.cu -- per-device context, scratch pool, configuration,
// statistics and error reporting for libsort512cuda.
#include "s512_runtime.cuh"

namespace s512 {

// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

static s512_config g_cfg = {S512_SPLIT_PLAIN, 0, 3.0, 0x5EEDull, 0, 0};
s512_config& config() { return g_cfg; }

static thread_local s512_stats g_stats;
s512_stats& thread_stats() { return g_stats; }

// ---------------------------------------------------------------------------
PhaseTimer::~PhaseTimer() {
    for (auto e : ev_) cudaEventDestroy(e);
}

int PhaseTimer::mark() {
    if (!on_) return -1;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    cudaEventRecord(e, st_);
    ev_.push_back(e);
    return (int)ev_.size() - 1;
}

double PhaseTimer::ms(int a, int b) {
    if (!on_ || a < 0 || b < 0) return 0.0;
    cudaEventSynchronize(ev_[b]);
    float v = 0.f;
    cudaEventElapsedTime(&v, ev_[a], ev_[b]);
    return (double)v;
}

// ---------------------------------------------------------------------------
void* DevCtx::get(const char* name, size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (g_cfg.fault_inject & S512_FAULT_ALLOC) {
        set_error("injected allocation failure (scratch '%s')", name);
        return nullptr;
    }
    auto it = bufs.find(name);
    if (it != bufs.end()) {
        if (it->second.second >= bytes) return it->second.first;
        cudaFree(it->second.first);
        bufs.erase(it);
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc of %zu bytes for scratch '%s' failed", bytes, name);
        return nullptr;
    }
    bufs[name] = {p, bytes};
    return p;
}

void* DevCtx::host_pinned(size_t bytes) {
    if (pinned_bytes >= bytes) return pinned;
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    pinned_bytes = 0;
    if (cudaMallocHost(&pinned, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMallocHost of %zu bytes failed", bytes);
        return nullptr;
    }
    pinned_bytes = bytes;
    return pinned;
}

void DevCtx::release_all() {
    for (auto& kv : bufs) cudaFree(kv.second.first);
    bufs.clear();
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    pinned_bytes = 0;
}

cudaError_t DevCtx::prepare(const void* fn, size_t smem) {
    auto it = smem_set.find(fn);
    if (it != smem_set.end() && it->second >= smem) return cudaSuccess;
    // the 48 KB default covers static + dynamic shared memory together
    cudaFuncAttributes fa;
    cudaError_t ea = cudaFuncGetAttributes(&fa, fn);
    if (ea != cudaSuccess) return ea;
    if (smem + fa.sharedSizeBytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        // prefer the largest shared-memory carveout so that several such
        // blocks can be resident on one SM
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
    }
    smem_set[fn] = smem;
    occ.erase(fn);
    return cudaSuccess;
}

int DevCtx::persistent_grid(const void* fn, int threads, size_t smem) {
    auto it = occ.find(fn);
    int per_sm;
    if (it != occ.end()) {
        per_sm = it->second;
    } else {
        per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
            cudaGetLastError();
            per_sm = 1;
        }
        if (per_sm < 1) per_sm = 1;
        occ[fn] = per_sm;
    }
    return per_sm * sms;
}

static std::mutex g_ctx_mu;
static std::map<int, DevCtx*> g_ctx;

DevCtx* current_ctx(int* status) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("no CUDA device");
        *status = S512_ERR_UNSUPPORTED;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(dev);
    if (it != g_ctx.end()) {
        *status = S512_OK;
        return it->second;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaGetDeviceProperties failed");
        *status = S512_ERR_CUDA;
        return nullptr;
    }
    if (prop.major < 10) {
        set_error("device %d (%s, sm_%d%d) is not an sm_100 part; this library is built for sm_100a only", dev,
                  prop.name, prop.major, prop.minor);
        *status = S512_ERR_UNSUPPORTED;
        return nullptr;
    }
    DevCtx* c = new DevCtx();
    c->dev = dev;
    c->sms = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    g_ctx[dev] = c;
    *status = S512_OK;
    return c;
}

CallGuard::CallGuard(DevCtx* c, cudaStream_t st) : c_(c), st_(st), lk_(c->mu) {
    if (c_->last_done) cudaStreamWaitEvent(st_, c_->last_done, 0);
}

void CallGuard::finish() {
    if (!c_->last_done) cudaEventCreateWithFlags(&c_->last_done, cudaEventDisableTiming);
    cudaEventRecord(c_->last_done, st_);
}

CallGuard::~CallGuard() {}

int pointer_kind(const void* p, int flags) {
    if (flags & S512_PTR_HOST) return 1;
    if (flags & S512_PTR_DEVICE) return 2;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    if (at.type == cudaMemoryTypeManaged) return 2;
    if (at.type != cudaMemoryTypeDevice) return 1;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (at.device != dev) {
        set_error("pointer %p is memory of device %d, the current device is %d", p, at.device, dev);
        return 0;
    }
    return 2;
}

}  // namespace s512

// ---------------------------------------------------------------------------
extern "C" {

int s512_set_config(const s512_config* cfg) {
    if (!cfg) return S512_ERR_ARG;
    if (cfg->splitter_mode != S512_SPLIT_PLAIN && cfg->splitter_mode != S512_SPLIT_LEARNED) return S512_ERR_ARG;
    if (!(cfg->max_imbalance >= 1.0)) return S512_ERR_ARG;
    s512::config() = *cfg;
    return S512_OK;
}

int s512_get_config(s512_config* cfg) {
    if (!cfg) return S512_ERR_ARG;
    *cfg = s512::config();
    return S512_OK;
}

int s512_get_stats(s512_stats* out) {
    if (!out) return S512_ERR_ARG;
    *out = s512::thread_stats();
    return S512_OK;
}

const char* s512_last_error_string(void) { return s512::g_err; }

int s512_release_scratch(void) {
    int st = 0;
    s512::DevCtx* c = s512::current_ctx(&st);
    if (!c) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaDeviceSynchronize();
    c->release_all();
    return S512_OK;
}

int s512_version(void) { return 100; }

int s512_popcount(unsigned mask) { return __builtin_popcount(mask & 0xFFFFu); }

}  // extern "C"
