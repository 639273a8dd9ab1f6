// s512_segsort.cu -- batched segmented sort: C-ABI entry points, the
// CUDA-graph plan and the launch-shape autotuner.
//
// A batch is many independent arrays stored back to back (segment s is
// data[offsets[s], offsets[s+1])).  The reference sorts such a batch with a
// loop of SmallSort16V / Sort calls (sort512perf.cpp:612-709 timeSmall).
// Here: one classification kernel, one persistent launch for the warp-sized
// segments and one per block size class (1K..16K keys) that has segments,
// and the partition levels for the few longer segments, all on one stream.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "s512_pipeline.cuh"
#include "s512_segsort.cuh"

namespace s512 {

// ---------------------------------------------------------------------------
// The autotuner's search space: the largest block class used (segments above
// it run the partition levels).  Shape i uses classes 0..kSegShapeTop[i].
static const int kSegShapeTop[] = {1, 2, 3, 4};
constexpr int kNumSegShapes = 4;
constexpr int kDefaultSegShape = 3;  // blocks of up to 16384 keys

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

static uint32_t shape_cap(int shape) { return seg_class_cap(kSegShapeTop[shape]); }

// Work lists of one batch (device memory).
struct SegLists {
    SegItem* warp_items = nullptr;
    SegItem* cls_items = nullptr;  // SEG_NCLASS lists of stride nseg + 1
    size_t stride = 0;
    SegDesc* big = nullptr;
    SegCtl* ctl = nullptr;
};

static int seg_lists_pool(DevCtx& C, size_t nseg, SegLists* L) {
    L->stride = nseg + 1;
    L->warp_items = (SegItem*)C.get("seg_warp", (nseg + 1) * sizeof(SegItem));
    L->cls_items = (SegItem*)C.get("seg_block", SEG_NCLASS * (nseg + 1) * sizeof(SegItem));
    L->big = (SegDesc*)C.get("seg_big", (nseg + 1) * sizeof(SegDesc));
    L->ctl = (SegCtl*)C.get("seg_ctl", sizeof(SegCtl));
    return (L->warp_items && L->cls_items && L->big && L->ctl) ? S512_OK : S512_ERR_ALLOC;
}

static int classify(const size_t* d_off, size_t nseg, uint32_t cap, const SegLists& L, cudaStream_t st) {
    S512_CUDA_TRY(cudaMemsetAsync(L.ctl, 0, sizeof(SegCtl), st));
    const int grid = (int)std::min<size_t>((nseg + 255) / 256, 4096);
    segsort_classify_kernel<<<grid > 0 ? grid : 1, 256, 0, st>>>(d_off, nseg, cap, L.warp_items, L.cls_items,
                                                                  L.stride, L.big, L.ctl);
    S512_LAUNCH_CHECK();
    return S512_OK;
}

// prepare_only: set the kernel's attributes without launching (done before a
// stream capture, where those calls do not belong).  n: the class's segment
// count (the grid is no larger).
template <typename Codec, int T, int E>
static int launch_block_class(DevCtx& C, Codec io, const SegItem* items, const uint32_t* d_n, uint32_t n,
                              cudaStream_t st, bool prepare_only) {
    using K = typename Codec::Key;
    auto fn = segsort_block_kernel<Codec, T, E>;
    const size_t smem = SlotSmem<K, T, E>::bytes;
    int grid = 0;
    S512_CUDA_TRY(launch_persistent(C, fn, T, smem, st, (int)n, &grid));
    if (prepare_only || n == 0) return S512_OK;
    fn<<<grid, T, smem, st>>>(io, items, d_n);
    S512_LAUNCH_CHECK();
    return S512_OK;
}

// Every segment of up to the shape's largest class, given the class counts
// read back after classification.
template <typename Codec>
static int launch_classes(DevCtx& C, int shape, Codec io, const SegLists& L, const SegCtl& h, cudaStream_t st,
                          uint32_t* launches, bool prepare_only = false) {
    {
        auto fn = segsort_warp_kernel<Codec>;
        int grid = 0;
        S512_CUDA_TRY(launch_persistent(C, fn, 256, 0, st, (int)((h.n_warp + 7) / 8), &grid));
        if (!prepare_only && h.n_warp) {
            fn<<<grid, 256, 0, st>>>(io, L.warp_items, L.ctl);
            S512_LAUNCH_CHECK();
            ++*launches;
        }
    }
    const int top = kSegShapeTop[shape];
    for (int c = top; c >= 0; --c) {  // the longest segments first
        const SegItem* items = L.cls_items + (size_t)c * L.stride;
        const uint32_t* d_n = &L.ctl->n_cls[c];
        const uint32_t n = h.n_cls[c];
        // 8 keys per thread where a class allows it: 64-bit keys with 16 per
        // thread (plus the inline block sort) run out of registers
        constexpr bool wide = sizeof(typename Codec::Key) == 8;
        int rc;
        switch (c) {
            case 0: rc = launch_block_class<Codec, 128, 8>(C, io, items, d_n, n, st, prepare_only); break;
            case 1: rc = launch_block_class<Codec, 256, 8>(C, io, items, d_n, n, st, prepare_only); break;
            case 2:
                rc = wide ? launch_block_class<Codec, 512, 8>(C, io, items, d_n, n, st, prepare_only)
                          : launch_block_class<Codec, 256, 16>(C, io, items, d_n, n, st, prepare_only);
                break;
            case 3:
                rc = wide ? launch_block_class<Codec, 1024, 8>(C, io, items, d_n, n, st, prepare_only)
                          : launch_block_class<Codec, 512, 16>(C, io, items, d_n, n, st, prepare_only);
                break;
            default: rc = launch_block_class<Codec, 1024, 16>(C, io, items, d_n, n, st, prepare_only); break;
        }
        if (rc) return rc;
        if (!prepare_only && n) ++*launches;
    }
    return S512_OK;
}

// Segments longer than a block: the partition levels, from the device list,
// on the pool's helper stream and with that stream's own scratch pool, so
// that these latency-bound launches (a read-back between levels) run beside
// the class launches queued on st.  `ready` (recorded on st before those
// launches) orders them after the caller's earlier work; st waits for them
// at the end, also after an error.
template <typename K, typename Codec>
static int sort_big_beside(DevCtx& C, Codec io, const SegLists& L, uint32_t n_big, uint64_t big_keys,
                           cudaStream_t st, cudaEvent_t ready, s512_stats& S) {
    if (n_big == 0) return S512_OK;
    cudaStream_t hs = C.copy_stream;
    S512_CUDA_TRY(cudaStreamWaitEvent(hs, ready, 0));
    int rc = S512_OK;
    DevCtx* H = current_ctx(&rc, hs);
    if (H) {
        CallGuard guard(H, hs);
        PhaseTimer tm(hs, false);
        rc = run_levels<K, Codec, Codec>(*H, io, io, L.big, n_big, big_keys, hs, tm, S, false);
    }
    S512_CUDA_TRY(cudaEventRecord(C.events[1], hs));
    S512_CUDA_TRY(cudaStreamWaitEvent(st, C.events[1], 0));
    return rc;
}

// The helper stream and two events when there are long segments; `ready` is
// recorded on st at once.
static int big_prologue(DevCtx& C, uint32_t n_big, cudaStream_t st) {
    if (n_big == 0) return S512_OK;
    S512_CUDA_TRY(C.copy_resources(2));
    S512_CUDA_TRY(cudaEventRecord(C.events[0], st));
    return S512_OK;
}

// The whole batch on the device: classify, the class launches, long segments.
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
    SegCtl* h = (SegCtl*)C.host_pinned(sizeof(SegCtl));
    if (!h) return S512_ERR_ALLOC;
    S512_CUDA_TRY(cudaMemcpyAsync(h, L.ctl, sizeof(SegCtl), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    const SegCtl counts = *h;
    S.kernel_launches += 1;
    rc = big_prologue(C, counts.n_big, st);
    if (rc) return rc;
    rc = launch_classes<Codec>(C, shape, io, L, counts, st, &S.kernel_launches);
    if (rc) return rc;
    const int t1 = tm.mark();
    rc = sort_big_beside<K, Codec>(C, io, L, counts.n_big, counts.big_keys, st, C.events.empty() ? nullptr : C.events[0], S);
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
            SegCtl h;
            if (!rc) {
                cudaMemcpyAsync(&h, L.ctl, sizeof(SegCtl), cudaMemcpyDeviceToHost, st);
                cudaStreamSynchronize(st);
                uint32_t launches = 0;
                rc = big_prologue(C, h.n_big, st);
                if (!rc) rc = launch_classes<Codec>(C, shape, io, L, h, st, &launches);
            }
            if (!rc) {
                s512_stats S;
                memset(&S, 0, sizeof(S));
                rc = sort_big_beside<K, Codec>(C, io, L, h.n_big, h.big_keys, st,
                                               C.events.empty() ? nullptr : C.events[0], S);
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
// graph plan: the classification is done once; the class launches are
// captured in a CUDA graph and replayed

struct Plan {
    int dt;
    void* keys;
    void* values;
    size_t nseg;
    int shape;
    SegItem* warp_items;
    SegItem* cls_items;
    SegDesc* big;
    SegCtl* ctl;
    SegCtl counts;       // the classification's counts (host copy)
    uint32_t launches;   // kernels in the graph
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

static SegLists plan_lists(const Plan* p) {
    SegLists L;
    L.warp_items = p->warp_items;
    L.cls_items = p->cls_items;
    L.stride = p->nseg + 1;
    L.big = p->big;
    L.ctl = p->ctl;
    return L;
}

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
        cudaMalloc(&p->cls_items, SEG_NCLASS * (nseg + 1) * sizeof(SegItem)) != cudaSuccess ||
        cudaMalloc(&p->big, (nseg + 1) * sizeof(SegDesc)) != cudaSuccess ||
        cudaMalloc(&p->ctl, sizeof(SegCtl)) != cudaSuccess) {
        cudaGetLastError();
        s512_segsort_plan_destroy((s512_segsort_plan*)p);
        set_error("s512_segsort_plan_create: allocation failed");
        return S512_ERR_ALLOC;
    }
    const SegLists L = plan_lists(p);
    int rc;
    {
        CallGuard guard(C, st);
        rc = classify(d_offsets, nseg, shape_cap(p->shape), L, st);
        if (!rc) {
            S512_CUDA_TRY(cudaMemcpyAsync(&p->counts, p->ctl, sizeof(SegCtl), cudaMemcpyDeviceToHost, st));
            S512_CUDA_TRY(cudaStreamSynchronize(st));
        }
        // kernel attributes and grid sizes are settled before the capture
        uint32_t launches = 0;
        if (!rc) {
            if (dtype == DT_I32) rc = launch_classes(*C, p->shape, make_i32(keys, values), L, p->counts, st, &launches,
                                                     true);
            else if (dtype == DT_F64) rc = launch_classes(*C, p->shape, make_f64(keys, values), L, p->counts, st,
                                                          &launches, true);
            else rc = launch_classes(*C, p->shape, make_kv(keys, values), L, p->counts, st, &launches, true);
        }
        // capture the class launches (the lists and counts stay on the device)
        cudaStream_t cs = nullptr;
        if (!rc && cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) rc = S512_ERR_CUDA;
        if (!rc) {
            if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = S512_ERR_CUDA;
            if (!rc) {
                if (dtype == DT_I32) rc = launch_classes(*C, p->shape, make_i32(keys, values), L, p->counts, cs,
                                                         &p->launches);
                else if (dtype == DT_F64) rc = launch_classes(*C, p->shape, make_f64(keys, values), L, p->counts, cs,
                                                              &p->launches);
                else rc = launch_classes(*C, p->shape, make_kv(keys, values), L, p->counts, cs, &p->launches);
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
        set_error("s512_segsort_plan_create: capture of the class launches failed");
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
    const uint32_t nb = p->counts.n_big;
    int rc = big_prologue(*C, nb, st);
    if (rc) return rc;
    S512_CUDA_TRY(cudaGraphLaunch(p->exec, st));
    S.kernel_launches = p->launches;
    if (nb) {
        const SegLists L = plan_lists(p);
        const uint64_t bk = p->counts.big_keys;
        cudaEvent_t ready = C->events[0];
        if (p->dt == DT_I32) rc = sort_big_beside<uint32_t>(*C, make_i32(p->keys, p->values), L, nb, bk, st, ready, S);
        else if (p->dt == DT_F64)
            rc = sort_big_beside<uint64_t>(*C, make_f64(p->keys, p->values), L, nb, bk, st, ready, S);
        else rc = sort_big_beside<uint64_t>(*C, make_kv(p->keys, p->values), L, nb, bk, st, ready, S);
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
    cudaFree(p->cls_items);
    cudaFree(p->big);
    cudaFree(p->ctl);
    delete p;
    return S512_OK;
}

}  // extern "C"
