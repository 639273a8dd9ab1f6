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
        // the old buffer may still be read by this stream's queued work
        cudaStreamSynchronize(stream);
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

void* DevCtx::stage_pinned(int k, size_t bytes) {
    if (stage_bytes[k] >= bytes) return stage[k];
    if (stage[k]) {
        cudaStreamSynchronize(stream);
        cudaFreeHost(stage[k]);
    }
    stage[k] = nullptr;
    stage_bytes[k] = 0;
    if (cudaMallocHost(&stage[k], bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMallocHost of %zu bytes for the streamed sort failed", bytes);
        return nullptr;
    }
    stage_bytes[k] = bytes;
    return stage[k];
}

void* DevCtx::host_pinned(size_t bytes) {
    if (pinned_bytes >= bytes) return pinned;
    if (pinned) {
        cudaStreamSynchronize(stream);
        cudaFreeHost(pinned);
    }
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
    for (int k = 0; k < 2; ++k) {
        if (stage[k]) cudaFreeHost(stage[k]);
        stage[k] = nullptr;
        stage_bytes[k] = 0;
    }
    for (auto e : events) cudaEventDestroy(e);
    events.clear();
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
}

cudaError_t DevCtx::copy_resources(size_t n) {
    if (!copy_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            copy_stream = nullptr;
            return e;
        }
    }
    while (events.size() < n) {
        cudaEvent_t ev;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
        events.push_back(ev);
    }
    return cudaSuccess;
}

cudaError_t DevCtx::prepare(const void* fn, size_t smem) {
    std::lock_guard<std::mutex> lk(sh->mu);
    auto it = sh->smem_set.find(fn);
    if (it != sh->smem_set.end() && it->second >= smem) return cudaSuccess;
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
    sh->smem_set[fn] = smem;
    sh->occ.erase(fn);
    return cudaSuccess;
}

int DevCtx::persistent_grid(const void* fn, int threads, size_t smem) {
    std::lock_guard<std::mutex> lk(sh->mu);
    auto it = sh->occ.find(fn);
    int per_sm;
    if (it != sh->occ.end()) {
        per_sm = it->second;
    } else {
        per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
            cudaGetLastError();
            per_sm = 1;
        }
        if (per_sm < 1) per_sm = 1;
        sh->occ[fn] = per_sm;
    }
    return per_sm * sms;
}

static std::mutex g_ctx_mu;
static std::map<int, DevShared*> g_dev;
static std::map<std::pair<int, cudaStream_t>, DevCtx*> g_ctx;

DevCtx* current_ctx(int* status, cudaStream_t st) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("no CUDA device");
        *status = S512_ERR_UNSUPPORTED;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find({dev, st});
    if (it != g_ctx.end()) {
        *status = S512_OK;
        return it->second;
    }
    DevShared* sh;
    auto dit = g_dev.find(dev);
    if (dit != g_dev.end()) {
        sh = dit->second;
    } else {
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
        sh = new DevShared();
        sh->dev = dev;
        sh->sms = prop.multiProcessorCount;
        sh->smem_optin = prop.sharedMemPerBlockOptin;
        g_dev[dev] = sh;
    }
    DevCtx* c = new DevCtx();
    c->sh = sh;
    c->dev = dev;
    c->sms = sh->sms;
    c->smem_optin = sh->smem_optin;
    c->stream = st;
    g_ctx[{dev, st}] = c;
    *status = S512_OK;
    return c;
}

// every pool of the current device
static void release_device_pools() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    std::vector<DevCtx*> mine;
    {
        std::lock_guard<std::mutex> lk(g_ctx_mu);
        for (auto& kv : g_ctx)
            if (kv.first.first == dev) mine.push_back(kv.second);
    }
    cudaDeviceSynchronize();
    for (DevCtx* c : mine) {
        std::lock_guard<std::mutex> lk(c->mu);
        c->release_all();
    }
}

CallGuard::CallGuard(DevCtx* c, cudaStream_t) : lk_(c->mu) {}

CallGuard::~CallGuard() {}

int pointer_kind(const void* p, int flags) {
    if (flags & S512_PTR_DEVICE) return PTR_DEVICE_MEM;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return PTR_PAGEABLE;
    }
    if (at.type == cudaMemoryTypeHost) return at.devicePointer ? PTR_PINNED : PTR_PAGEABLE;
    if (flags & S512_PTR_HOST) return PTR_PAGEABLE;
    if (at.type == cudaMemoryTypeManaged) return PTR_DEVICE_MEM;
    if (at.type != cudaMemoryTypeDevice) return PTR_PAGEABLE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return PTR_OTHER_DEVICE;
    }
    if (at.device != dev) {
        set_error("pointer %p is memory of device %d, the current device is %d", p, at.device, dev);
        return PTR_OTHER_DEVICE;
    }
    return PTR_DEVICE_MEM;
}

const void* mapped_host_address(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
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
    s512::DevCtx* c = s512::current_ctx(&st, nullptr);
    if (!c) return st;
    s512::release_device_pools();
    return S512_OK;
}

int s512_version(void) { return 100; }

int s512_popcount(unsigned mask) { return __builtin_popcount(mask & 0xFFFFu); }

}  // extern "C"
