// s512_segsort.cu -- batched segmented sort: C-ABI entry points, the
// CUDA-graph plan and the launch-shape autotuner.
//
// A batch is many independent arrays stored back to back (segment s is
// data[offsets[s], offsets[s+1])).  The reference sorts such a batch with a
// loop of SmallSort16V / Sort calls (sort512perf.cpp:612-709 timeSmall).
// Here: one classification kernel, one persistent launch for every segment
// that fits a block (segsort_small_kernel), and the partition levels for the
// few longer segments, all on one stream.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "s512_pipeline.cuh"
#include "s512_segsort.cuh"

namespace s512 {

// ---------------------------------------------------------------------------
// launch shapes of the persistent kernel (the autotuner's search space)
struct SegShape {
    int threads, ept;
};
static const SegShape kSegShapes[] = {{256, 16}, {512, 8}, {512, 16}, {1024, 8}};
constexpr int kNumSegShapes = 4;
constexpr int kDefaultSegShape = 2;  // 512 x 16: blocks of up to 8192 keys

enum { DT_I32 = 0, DT_F64 = 1, DT_KV = 2, NUM_DT = 3 };
static int g_seg_shape[NUM_DT] = {-1, -1, -1};
static std::mutex g_tune_mu;

static const char* dt_name(int dt) { return dt == DT_I32 ? "i32" : dt == DT_F64 ? "f64" : "kv_i32"; }

static std::string tune_cache_path() {
    const char* p = getenv("S512_TUNE_CACHE");
    if (p && *p) return p;
    return "";
}

// Cache file: one line per entry, "<device name>|<dtype>|<shape index>".
static void load_tune_cache() {
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return;
    cudaDeviceProp prop;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&prop, dev);
    char line[512];
    while (fgets(line, sizeof(line), f)) {
        char name[256] = {0}, dts[32] = {0};
        int idx = -1;
        if (sscanf(line, "%255[^|]|%31[^|]|%d", name, dts, &idx) == 3 && std::string(name) == prop.name &&
            idx >= 0 && idx < kNumSegShapes) {
            for (int d = 0; d < NUM_DT; ++d)
                if (std::string(dts) == dt_name(d) && g_seg_shape[d] < 0) g_seg_shape[d] = idx;
        }
    }
    fclose(f);
}

static void save_tune_cache(int dt, int idx) {
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    cudaDeviceProp prop;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&prop, dev);
    FILE* f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s|%s|%d\n", prop.name, dt_name(dt), idx);
    fclose(f);
}

static int seg_shape_for(int dt) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_seg_shape[dt] < 0) load_tune_cache();
    return g_seg_shape[dt] >= 0 ? g_seg_shape[dt] : kDefaultSegShape;
}

// ---------------------------------------------------------------------------
// prepare_only: set the kernel's attributes and size its grid without
// launching (done before a stream capture, where those calls do not belong)
template <typename Codec, int T, int E>
static int launch_small(DevCtx& C, Codec io, const SegItem* wi, const SegItem* bi, SegCtl* ctl, cudaStream_t st,
                        bool prepare_only) {
    using K = typename Codec::Key;
    auto fn = segsort_small_kernel<Codec, T, E>;
    const size_t block_bytes = SlotSmem<K, T, E>::bytes;
    const size_t warp_bytes = (size_t)(T / 32) * WARP_REGION * sizeof(K);
    const size_t smem = block_bytes > warp_bytes ? block_bytes : warp_bytes;
    int grid = 0;
    S512_CUDA_TRY(launch_persistent(C, fn, T, smem, st, 0, &grid));
    if (prepare_only) return S512_OK;
    fn<<<grid, T, smem, st>>>(io, wi, bi, ctl);
    S512_LAUNCH_CHECK();
    return S512_OK;
}

template <typename Codec>
static int launch_small_shape(DevCtx& C, int shape, Codec io, const SegItem* wi, const SegItem* bi, SegCtl* ctl,
                              cudaStream_t st, bool prepare_only = false) {
    switch (shape) {
        case 0: return launch_small<Codec, 256, 16>(C, io, wi, bi, ctl, st, prepare_only);
        case 1: return launch_small<Codec, 512, 8>(C, io, wi, bi, ctl, st, prepare_only);
        case 2: return launch_small<Codec, 512, 16>(C, io, wi, bi, ctl, st, prepare_only);
        default: return launch_small<Codec, 1024, 8>(C, io, wi, bi, ctl, st, prepare_only);
    }
}

static uint32_t shape_cap(int shape) { return (uint32_t)(kSegShapes[shape].threads * kSegShapes[shape].ept); }

// Work lists of one batch (device memory).
struct SegLists {
    SegItem* warp_items = nullptr;
    SegItem* block_items = nullptr;
    SegDesc* big = nullptr;
    SegCtl* ctl = nullptr;
};

static int seg_lists_pool(DevCtx& C, size_t nseg, SegLists* L) {
    L->warp_items = (SegItem*)C.get("seg_warp", (nseg + 1) * sizeof(SegItem));
    L->block_items = (SegItem*)C.get("seg_block", (nseg + 1) * sizeof(SegItem));
    L->big = (SegDesc*)C.get("seg_big", (nseg + 1) * sizeof(SegDesc));
    L->ctl = (SegCtl*)C.get("seg_ctl", sizeof(SegCtl));
    return (L->warp_items && L->block_items && L->big && L->ctl) ? S512_OK : S512_ERR_ALLOC;
}

static int classify(const size_t* d_off, size_t nseg, uint32_t cap, const SegLists& L, cudaStream_t st) {
    S512_CUDA_TRY(cudaMemsetAsync(L.ctl, 0, sizeof(SegCtl), st));
    const int grid = (int)std::min<size_t>((nseg + 255) / 256, 4096);
    segsort_classify_kernel<<<grid > 0 ? grid : 1, 256, 0, st>>>(d_off, nseg, cap, L.warp_items, L.block_items,
                                                                  L.big, L.ctl);
    S512_LAUNCH_CHECK();
    return S512_OK;
}

// Segments longer than a block: the partition levels, from the device list.
template <typename K, typename Codec>
static int sort_big(DevCtx& C, Codec io, const SegLists& L, uint32_t n_big, uint64_t big_keys, cudaStream_t st,
                    PhaseTimer& tm, s512_stats& S) {
    if (n_big == 0) return S512_OK;
    return run_levels<K, Codec, Codec>(C, io, io, L.big, n_big, big_keys, st, tm, S, false);
}

// The whole batch on the device: classify, persistent launch, long segments.
template <typename K, typename Codec>
static int segsort_device(DevCtx& C, Codec io, const size_t* d_off, size_t nseg, int dt, cudaStream_t st) {
    s512_stats& S = thread_stats();
    memset(&S, 0, sizeof(S));
    S.key_bytes = sizeof(K);
    PhaseTimer tm(st, config().collect_stats != 0);
    const int t0 = tm.mark();
    SegLists L;
    int rc = seg_lists_pool(C, nseg, &L);
    if (rc) return rc;
    const int shape = seg_shape_for(dt);
    rc = classify(d_off, nseg, shape_cap(shape), L, st);
    if (rc) return rc;
    rc = launch_small_shape<Codec>(C, shape, io, L.warp_items, L.block_items, L.ctl, st);
    if (rc) return rc;
    S.kernel_launches += 2;
    SegCtl* h = (SegCtl*)C.host_pinned(sizeof(SegCtl));
    if (!h) return S512_ERR_ALLOC;
    S512_CUDA_TRY(cudaMemcpyAsync(h, L.ctl, sizeof(SegCtl), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t n_big = h->n_big;
    const uint64_t big_keys = h->big_keys;
    const int t1 = tm.mark();
    rc = sort_big<K, Codec>(C, io, L, n_big, big_keys, st, tm, S);
    if (rc) return rc;
    const int t2 = tm.mark();
    if (tm.on()) {
        S.leaf_ms[0] = tm.ms(t0, t1);
        S.total_ms = tm.ms(t0, t2);
    }
    return S512_OK;
}

// ---------------------------------------------------------------------------
// entry points

template <typename K, typename MakeCodec>
static int segsort_entry(int dt, void* keys, void* values, size_t elem_bytes, const size_t* offsets, size_t nseg,
                         int flags, void* stream, MakeCodec make) {
    if (nseg == 0) return S512_OK;
    if (!keys || !offsets || (dt == DT_KV && !values)) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    CallGuard guard(C, st);
    S512_HOST_PTR(host, keys, flags);
    S512_HOST_PTR(off_host, offsets, (flags & S512_PTR_DEVICE) ? 0 : flags);
    const size_t* d_off = offsets;
    if (off_host) {
        size_t* o = (size_t*)C->get("seg_offsets", (nseg + 1) * sizeof(size_t));
        if (!o) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemcpyAsync(o, offsets, (nseg + 1) * sizeof(size_t), cudaMemcpyHostToDevice, st));
        d_off = o;
    }
    void* dk = keys;
    void* dv = values;
    size_t total = 0;
    if (host) {
        if (!off_host) {
            set_error("segmented sort: host data needs host offsets");
            return S512_ERR_ARG;
        }
        total = offsets[nseg];
        dk = C->get("stage0", total * elem_bytes + 16);
        if (!dk) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemcpyAsync(dk, keys, total * elem_bytes, cudaMemcpyHostToDevice, st));
        if (dt == DT_KV) {
            dv = C->get("stage1", total * sizeof(int) + 16);
            if (!dv) return S512_ERR_ALLOC;
            S512_CUDA_TRY(cudaMemcpyAsync(dv, values, total * sizeof(int), cudaMemcpyHostToDevice, st));
        }
    }
    int rc = segsort_device<K>(*C, make(dk, dv), d_off, nseg, dt, st);
    if (rc) return rc;
    if (host) {
        S512_CUDA_TRY(cudaMemcpyAsync(keys, dk, total * elem_bytes, cudaMemcpyDeviceToHost, st));
        if (dt == DT_KV)
            S512_CUDA_TRY(cudaMemcpyAsync(values, dv, total * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    guard.finish();
    if (host || !(flags & S512_ASYNC)) S512_CUDA_TRY(cudaStreamSynchronize(st));
    return S512_OK;
}

static CodecI32 make_i32(void* k, void*) { return CodecI32{(const int*)k, (int*)k}; }
static CodecF64 make_f64(void* k, void*) {
    return CodecF64{(const unsigned long long*)k, (unsigned long long*)k};
}
static CodecKV make_kv(void* k, void* v) { return CodecKV{(const int*)k, (const int*)v, (int*)k, (int*)v}; }

// ---------------------------------------------------------------------------
// autotuner: time every launch shape on random keys with the caller's
// segment layout and keep the fastest for the dtype

template <typename K, typename Codec>
static int tune_dtype(DevCtx& C, int dt, Codec io, uint64_t total, const size_t* d_off, size_t nseg, cudaStream_t st,
                      double* best_ms) {
    SegLists L;
    int rc = seg_lists_pool(C, nseg, &L);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = kDefaultSegShape;
    double bms = 1e30;
    for (int shape = 0; shape < kNumSegShapes; ++shape) {
        double ms_sum = 0;
        for (int rep = 0; rep < 3; ++rep) {
            segsort_fill_kernel<Codec><<<1024, 256, 0, st>>>(io, total, 0x7u + (uint64_t)rep);
            cudaEventRecord(e0, st);
            rc = classify(d_off, nseg, shape_cap(shape), L, st);
            if (!rc) rc = launch_small_shape<Codec>(C, shape, io, L.warp_items, L.block_items, L.ctl, st);
            SegCtl h;
            if (!rc) {
                cudaMemcpyAsync(&h, L.ctl, sizeof(SegCtl), cudaMemcpyDeviceToHost, st);
                cudaStreamSynchronize(st);
                PhaseTimer tm(st, false);
                s512_stats S;
                memset(&S, 0, sizeof(S));
                rc = sort_big<K, Codec>(C, io, L, h.n_big, h.big_keys, st, tm, S);
            }
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            if (rc) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) ms_sum += ms;  // the first run warms the shape up
        }
        if (rc) break;
        if (ms_sum < bms) {
            bms = ms_sum;
            best = shape;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_seg_shape[dt] = best;
    }
    save_tune_cache(dt, best);
    *best_ms = bms / 2.0;
    return S512_OK;
}

// ---------------------------------------------------------------------------
// graph plan: the classification is done once; the persistent launch (and the
// reset of its queue counters) is captured in a CUDA graph and replayed

struct Plan {
    int dt;
    void* keys;
    void* values;
    size_t nseg;
    int shape;
    SegItem* warp_items;
    SegItem* block_items;
    SegDesc* big;
    SegCtl* ctl;
    uint32_t n_big;
    uint64_t big_keys;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

}  // namespace s512

using namespace s512;

extern "C" {

int s512_segsort_i32(int* data, const size_t* offsets, size_t nseg, int flags, void* stream) {
    return segsort_entry<uint32_t>(DT_I32, data, nullptr, sizeof(int), offsets, nseg, flags, stream, make_i32);
}
int s512_segsort_f64(double* data, const size_t* offsets, size_t nseg, int flags, void* stream) {
    return segsort_entry<uint64_t>(DT_F64, data, nullptr, sizeof(double), offsets, nseg, flags, stream, make_f64);
}
int s512_segsort_kv_i32(int* keys, int* values, const size_t* offsets, size_t nseg, int flags, void* stream) {
    return segsort_entry<uint64_t>(DT_KV, keys, values, sizeof(int), offsets, nseg, flags, stream, make_kv);
}

int s512_segsort_tune(int dtype, const size_t* d_offsets, size_t nseg, double* best_ms, int* shape_index,
                      void* stream) {
    if (dtype < 0 || dtype >= NUM_DT || !d_offsets || nseg == 0) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    if (pointer_kind(d_offsets, 0) != 2) {
        set_error("s512_segsort_tune: offsets must be device memory");
        return S512_ERR_ARG;
    }
    size_t total = 0;
    S512_CUDA_TRY(cudaMemcpy(&total, d_offsets + nseg, sizeof(size_t), cudaMemcpyDeviceToHost));
    CallGuard guard(C, st);
    void* k = C->get("tune_keys", total * (dtype == DT_F64 ? 8 : 4) + 16);
    void* v = dtype == DT_KV ? C->get("tune_vals", total * 4 + 16) : nullptr;
    if (!k || (dtype == DT_KV && !v)) return S512_ERR_ALLOC;
    double ms = 0;
    int rc;
    if (dtype == DT_I32) rc = tune_dtype<uint32_t>(*C, dtype, make_i32(k, v), total, d_offsets, nseg, st, &ms);
    else if (dtype == DT_F64) rc = tune_dtype<uint64_t>(*C, dtype, make_f64(k, v), total, d_offsets, nseg, st, &ms);
    else rc = tune_dtype<uint64_t>(*C, dtype, make_kv(k, v), total, d_offsets, nseg, st, &ms);
    guard.finish();
    if (rc) return rc;
    if (best_ms) *best_ms = ms;
    if (shape_index) *shape_index = g_seg_shape[dtype];
    return S512_OK;
}

int s512_segsort_plan_create(s512_segsort_plan** out, int dtype, void* keys, void* values, const size_t* d_offsets,
                             size_t nseg, void* stream) {
    if (!out || dtype < 0 || dtype >= NUM_DT || !keys || !d_offsets || nseg == 0 || (dtype == DT_KV && !values))
        return S512_ERR_ARG;
    *out = nullptr;
    if (pointer_kind(keys, 0) != 2 || pointer_kind(d_offsets, 0) != 2) {
        set_error("s512_segsort_plan_create: keys, values and offsets must be device memory");
        return S512_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    Plan* p = new Plan();
    memset(p, 0, sizeof(Plan));
    p->dt = dtype;
    p->keys = keys;
    p->values = values;
    p->nseg = nseg;
    p->shape = seg_shape_for(dtype);
    // plan-owned lists (the shared scratch pool may be resized by other calls)
    if (cudaMalloc(&p->warp_items, (nseg + 1) * sizeof(SegItem)) != cudaSuccess ||
        cudaMalloc(&p->block_items, (nseg + 1) * sizeof(SegItem)) != cudaSuccess ||
        cudaMalloc(&p->big, (nseg + 1) * sizeof(SegDesc)) != cudaSuccess ||
        cudaMalloc(&p->ctl, sizeof(SegCtl)) != cudaSuccess) {
        cudaGetLastError();
        s512_segsort_plan_destroy((s512_segsort_plan*)p);
        set_error("s512_segsort_plan_create: allocation failed");
        return S512_ERR_ALLOC;
    }
    SegLists L{p->warp_items, p->block_items, p->big, p->ctl};
    int rc;
    {
        CallGuard guard(C, st);
        rc = classify(d_offsets, nseg, shape_cap(p->shape), L, st);
        SegCtl h;
        if (!rc) {
            S512_CUDA_TRY(cudaMemcpyAsync(&h, p->ctl, sizeof(SegCtl), cudaMemcpyDeviceToHost, st));
            S512_CUDA_TRY(cudaStreamSynchronize(st));
            p->n_big = h.n_big;
            p->big_keys = h.big_keys;
        }
        // kernel attributes and grid size are settled before the capture
        if (!rc) {
            if (dtype == DT_I32) rc = launch_small_shape(*C, p->shape, make_i32(keys, values), p->warp_items,
                                                         p->block_items, p->ctl, st, true);
            else if (dtype == DT_F64) rc = launch_small_shape(*C, p->shape, make_f64(keys, values), p->warp_items,
                                                              p->block_items, p->ctl, st, true);
            else rc = launch_small_shape(*C, p->shape, make_kv(keys, values), p->warp_items, p->block_items,
                                         p->ctl, st, true);
        }
        // capture: reset the queue counters, then the persistent launch
        cudaStream_t cs = nullptr;
        if (!rc && cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) rc = S512_ERR_CUDA;
        if (!rc) {
            if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = S512_ERR_CUDA;
            if (!rc) {
                cudaMemsetAsync(&p->ctl->ctr_block, 0, 2 * sizeof(uint32_t), cs);
                if (dtype == DT_I32) rc = launch_small_shape(*C, p->shape, make_i32(keys, values), p->warp_items,
                                                             p->block_items, p->ctl, cs);
                else if (dtype == DT_F64) rc = launch_small_shape(*C, p->shape, make_f64(keys, values),
                                                                  p->warp_items, p->block_items, p->ctl, cs);
                else rc = launch_small_shape(*C, p->shape, make_kv(keys, values), p->warp_items, p->block_items,
                                             p->ctl, cs);
                cudaGraph_t g = nullptr;
                if (cudaStreamEndCapture(cs, &g) != cudaSuccess) rc = rc ? rc : S512_ERR_CUDA;
                p->graph = g;
                if (!rc && cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) rc = S512_ERR_CUDA;
            }
            cudaStreamDestroy(cs);
        }
        guard.finish();
    }
    if (rc) {
        cudaGetLastError();
        set_error("s512_segsort_plan_create: capture of the persistent launch failed");
        s512_segsort_plan_destroy((s512_segsort_plan*)p);
        return rc;
    }
    *out = (s512_segsort_plan*)p;
    return S512_OK;
}

int s512_segsort_plan_launch(s512_segsort_plan* plan, void* stream) {
    Plan* p = (Plan*)plan;
    if (!p || !p->exec) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    CallGuard guard(C, st);
    s512_stats& S = thread_stats();
    memset(&S, 0, sizeof(S));
    S512_CUDA_TRY(cudaGraphLaunch(p->exec, st));
    S.kernel_launches = 1;
    if (p->n_big) {
        PhaseTimer tm(st, false);
        SegLists L{p->warp_items, p->block_items, p->big, p->ctl};
        int rc;
        if (p->dt == DT_I32) rc = sort_big<uint32_t>(*C, make_i32(p->keys, p->values), L, p->n_big, p->big_keys, st,
                                                     tm, S);
        else if (p->dt == DT_F64) rc = sort_big<uint64_t>(*C, make_f64(p->keys, p->values), L, p->n_big,
                                                          p->big_keys, st, tm, S);
        else rc = sort_big<uint64_t>(*C, make_kv(p->keys, p->values), L, p->n_big, p->big_keys, st, tm, S);
        if (rc) return rc;
    }
    guard.finish();
    return S512_OK;
}

int s512_segsort_plan_destroy(s512_segsort_plan* plan) {
    Plan* p = (Plan*)plan;
    if (!p) return S512_OK;
    cudaDeviceSynchronize();
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    cudaFree(p->warp_items);
    cudaFree(p->block_items);
    cudaFree(p->big);
    cudaFree(p->ctl);
    delete p;
    return S512_OK;
}

}  // extern "C"
