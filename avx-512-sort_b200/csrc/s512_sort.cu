// s512_sort.cu -- the sort driver and the C-ABI entry points for Sort,
// SmallSort16V, CoreSmallSortN and Partition512.
//
// Reference call stack being replaced (sort512.hpp):
//   Sort (5960) -> CoreSort (5947) -> SmallSort16V (5312 / 2255) for ranges
//   under SortLimite, else CoreSortPivotPartition (5929) -> Partition512
//   (5730 / 5822) and recursion on both sides.
// Here: whole arrays of at most one leaf go straight to one warp / one block;
// larger arrays run partition levels (sample -> splitters -> multi-way
// partition -> plan) until every bucket fits a leaf, and the leaves are sorted
// into their final place.  Only one small read-back per level reaches the
// host (the level's item counts and error word).
#include "s512_pipeline.cuh"
#include "s512_partition2.cuh"
#include "s512_stream.cuh"

using namespace s512;

#define S512_ENTER(ctxvar, st)              \
    int status_ = S512_OK;                  \
    DevCtx* ctxvar = current_ctx(&status_, st); \
    if (!ctxvar) return status_;            \
    CallGuard guard_(ctxvar, st)

extern "C" {

// ---- Sort ------------------------------------------------------------------
int s512_sort_i32(int* data, size_t n, int flags, void* stream) {
    if (n == 0) return S512_OK;
    if (!data) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    S512_ENTER(C, st);
    S512_HOST_PTR(host, data, flags);
    if (host && stream_needed(n, sizeof(int))) {  // larger than the device budget
        int rc = stream_sort<int>(*C, data, n, st);
        if (rc) return rc;
        return finish_call(guard_, st, flags, host);
    }
    int* d = data;
    HostFeed feed;
    bool chunked = false;
    if (host) {
        d = (int*)C->get("stage0", n * sizeof(int));
        if (!d) return S512_ERR_ALLOC;
        void* hp[1] = {data};
        void* dp[1] = {d};
        S512_TRY_RC(copy_in<uint32_t>(*C, 1, hp, dp, sizeof(int), n, host_pinned, st, &feed, &chunked));
    }
    int rc = sort_device<uint32_t>(*C, CodecI32{d, d}, CodecI32{d, d}, n, st, use_learned(flags),
                                   chunked ? &feed : nullptr);
    if (rc) return rc;
    if (host) S512_CUDA_TRY(cudaMemcpyAsync(data, d, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    return finish_call(guard_, st, flags, host, host_pinned);
}

int s512_sort_f64(double* data, size_t n, int flags, void* stream) {
    if (n == 0) return S512_OK;
    if (!data) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    S512_ENTER(C, st);
    S512_HOST_PTR(host, data, flags);
    if (host && stream_needed(n, sizeof(double))) {  // larger than the device budget
        int rc = stream_sort<double>(*C, data, n, st);
        if (rc) return rc;
        return finish_call(guard_, st, flags, host);
    }
    unsigned long long* d = (unsigned long long*)data;
    HostFeed feed;
    bool chunked = false;
    if (host) {
        d = (unsigned long long*)C->get("stage0", n * sizeof(double));
        if (!d) return S512_ERR_ALLOC;
        void* hp[1] = {data};
        void* dp[1] = {d};
        S512_TRY_RC(copy_in<uint64_t>(*C, 1, hp, dp, sizeof(double), n, host_pinned, st, &feed, &chunked));
    }
    int rc = sort_device<uint64_t>(*C, CodecF64{d, d}, CodecF64{d, d}, n, st, use_learned(flags),
                                   chunked ? &feed : nullptr);
    if (rc) return rc;
    if (host) S512_CUDA_TRY(cudaMemcpyAsync(data, d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    return finish_call(guard_, st, flags, host, host_pinned);
}

int s512_sort_kv_i32(int* keys, int* values, size_t n, int flags, void* stream) {
    if (n == 0) return S512_OK;
    if (!keys || !values) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    S512_ENTER(C, st);
    S512_HOST_PTR(host, keys, flags);
    if (host && stream_needed(n, 2 * sizeof(int))) {  // larger than the device budget
        int rc = stream_sort_kv(*C, keys, values, n, st);
        if (rc) return rc;
        return finish_call(guard_, st, flags, host);
    }
    int* dk = keys;
    int* dv = values;
    HostFeed feed;
    bool chunked = false;
    bool pinned_both = false;
    if (host) {
        // both arrays are host memory; both must be page-locked to be fed in chunks
        S512_HOST_PTR(vhost, values, flags);
        pinned_both = host_pinned && vhost && vhost_pinned;
        dk = (int*)C->get("stage0", n * sizeof(int));
        dv = (int*)C->get("stage1", n * sizeof(int));
        if (!dk || !dv) return S512_ERR_ALLOC;
        void* hp[2] = {keys, values};
        void* dp[2] = {dk, dv};
        S512_TRY_RC(copy_in<uint64_t>(*C, 2, hp, dp, sizeof(int), n, pinned_both, st, &feed, &chunked));
    }
    int rc = sort_device<uint64_t>(*C, CodecKV{dk, dv, dk, dv}, CodecKV{dk, dv, dk, dv}, n, st, use_learned(flags),
                                   chunked ? &feed : nullptr);
    if (rc) return rc;
    if (host) {
        S512_CUDA_TRY(cudaMemcpyAsync(keys, dk, n * sizeof(int), cudaMemcpyDeviceToHost, st));
        S512_CUDA_TRY(cudaMemcpyAsync(values, dv, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    return finish_call(guard_, st, flags, host, pinned_both);
}

// ---- SmallSort16V / CoreSmallSortN ----------------------------------------
// Same kernels as Sort: an array of <= 256 keys is one warp's bitonic network.
int s512_smallsort_i32(int* data, size_t len, int flags, void* stream) {
    return s512_sort_i32(data, len, flags, stream);
}
int s512_smallsort_f64(double* data, size_t len, int flags, void* stream) {
    return s512_sort_f64(data, len, flags, stream);
}
int s512_smallsort_kv_i32(int* keys, int* values, size_t len, int flags, void* stream) {
    return s512_sort_kv_i32(keys, values, len, flags, stream);
}
int s512_core_small_sort_i32(int* data, int nvec, int flags, void* stream) {
    if (nvec < 1 || nvec > 16) return S512_ERR_ARG;
    return s512_sort_i32(data, (size_t)nvec * 16, flags, stream);
}
int s512_core_small_sort_f64(double* data, int nvec, int flags, void* stream) {
    if (nvec < 1 || nvec > 16) return S512_ERR_ARG;
    return s512_sort_f64(data, (size_t)nvec * 8, flags, stream);
}
int s512_core_small_sort_kv_i32(int* keys, int* values, int nvec, int flags, void* stream) {
    if (nvec < 1 || nvec > 16) return S512_ERR_ARG;
    return s512_sort_kv_i32(keys, values, (size_t)nvec * 16, flags, stream);
}

}  // extern "C"

// ---- Partition512 -----------------------------------------------------------
namespace s512 {

template <typename T, bool KV>
static int partition_entry(T* data, int* values, size_t left, size_t right, T pivot, size_t* boundary, int flags,
                           void* stream) {
    if (!boundary) return S512_ERR_ARG;
    if (right < left) {  // empty range
        *boundary = left;
        return S512_OK;
    }
    if (!data || (KV && !values)) return S512_ERR_ARG;
    const size_t n = right - left + 1;
    cudaStream_t st = (cudaStream_t)stream;
    S512_ENTER(C, st);
    S512_HOST_PTR(host, data, flags);
    T* dk = data + left;
    int* dv = KV ? values + left : nullptr;
    if (host) {
        dk = (T*)C->get("stage0", n * sizeof(T));
        if (!dk) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemcpyAsync(dk, data + left, n * sizeof(T), cudaMemcpyHostToDevice, st));
        if (KV) {
            dv = (int*)C->get("stage1", n * sizeof(int));
            if (!dv) return S512_ERR_ALLOC;
            S512_CUDA_TRY(cudaMemcpyAsync(dv, values + left, n * sizeof(int), cudaMemcpyHostToDevice, st));
        }
    }
    constexpr int THREADS = 256, IPT = sizeof(T) == 4 ? 16 : 8;
    constexpr int TILE = THREADS * IPT;
    const uint32_t ntiles = (uint32_t)((n + TILE - 1) / TILE);
    T* ok = (T*)C->get("p2_keys", n * sizeof(T));
    int* ov = KV ? (int*)C->get("p2_vals", n * sizeof(int)) : nullptr;
    unsigned long long* status = (unsigned long long*)C->get("p2_status", (size_t)ntiles * 2 * 8 + 16);
    Part2Ctl* ctl = (Part2Ctl*)C->get("p2_ctl", sizeof(Part2Ctl));
    Part2Ctl* hctl = (Part2Ctl*)C->host_pinned(sizeof(Part2Ctl));
    if (!ok || (KV && !ov) || !status || !ctl || !hctl) return S512_ERR_ALLOC;
    // (the spare pair of status words past the last tile is the never-written
    // predecessor of the failure-injection test)
    S512_CUDA_TRY(cudaMemsetAsync(status, 0, (size_t)(ntiles + 1) * 2 * 8, st));
    S512_CUDA_TRY(cudaMemsetAsync(ctl, 0, sizeof(Part2Ctl), st));
    auto fn = partition2_kernel<T, KV, THREADS, IPT>;
    int grid = 0;
    S512_CUDA_TRY(launch_persistent(*C, fn, THREADS, 0, st, (int)ntiles, &grid));
    fn<<<grid, THREADS, 0, st>>>(dk, dv, ok, ov, (uint64_t)n, pivot, status, ctl, ntiles,
                                 (config().fault_inject & S512_FAULT_TIMEOUT) ? ntiles : 0xFFFFFFFFu);
    S512_LAUNCH_CHECK();
    // the error word first: tiles that gave up wrote nothing, so on an error
    // the scratch holds stale keys and the caller's range stays as it was
    S512_CUDA_TRY(cudaMemcpyAsync(hctl, ctl, sizeof(Part2Ctl), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    if (hctl->err) {
        guard_.finish();
        set_error("partition look-back wait timed out");
        return S512_ERR_TIMEOUT;
    }
    T* dst = host ? dk : data + left;
    S512_CUDA_TRY(cudaMemcpyAsync(dst, ok, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    if (KV) S512_CUDA_TRY(cudaMemcpyAsync(host ? dv : values + left, ov, n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    if (host) {
        S512_CUDA_TRY(cudaMemcpyAsync(data + left, dk, n * sizeof(T), cudaMemcpyDeviceToHost, st));
        if (KV) S512_CUDA_TRY(cudaMemcpyAsync(values + left, dv, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    guard_.finish();
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    s512_stats& S = thread_stats();
    memset(&S, 0, sizeof(S));
    S.kernel_launches = 1;
    S.key_bytes = sizeof(T);
    *boundary = left + (size_t)hctl->total_low;
    return S512_OK;
}

}  // namespace s512

extern "C" {
int s512_partition_i32(int* data, size_t left, size_t right, int pivot, size_t* boundary, int flags, void* stream) {
    return partition_entry<int, false>(data, nullptr, left, right, pivot, boundary, flags, stream);
}
int s512_partition_f64(double* data, size_t left, size_t right, double pivot, size_t* boundary, int flags,
                       void* stream) {
    return partition_entry<double, false>(data, nullptr, left, right, pivot, boundary, flags, stream);
}
int s512_partition_kv_i32(int* keys, int* values, size_t left, size_t right, int pivot, size_t* boundary,
                          int flags, void* stream) {
    return partition_entry<int, true>(keys, values, left, right, pivot, boundary, flags, stream);
}
}  // extern "C"
