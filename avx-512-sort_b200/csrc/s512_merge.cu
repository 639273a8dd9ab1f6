// s512_merge.cu -- C-ABI entry points for merging sorted runs on the GPU and
// for the merge-based drivers (SortOmpMerge, SortOmpMergeDeps,
// SortOmpParMerge: sort512.hpp:6006-6174 with parallelInplace.hpp).
#include <vector>

#include "s512_merge.cuh"
#include "s512_runtime.cuh"

namespace s512 {

struct Run {
    uint64_t start, len;
};

// Merge neighbouring runs level by level (a pair of runs per merge; an odd
// last run passes through) until one run is left.  Ping-pong between `data`
// and `tmp`; the result ends in `data`.
template <typename T>
static int merge_tree(DevCtx& C, T* data, T* tmp, std::vector<Run> runs, cudaStream_t st, uint32_t* launches) {
    T* src = data;
    T* dst = tmp;
    std::vector<MergePair> pairs;
    while (runs.size() > 1) {
        pairs.clear();
        std::vector<Run> next;
        uint32_t tiles = 0;
        for (size_t r = 0; r < runs.size(); r += 2) {
            MergePair p;
            p.a0 = runs[r].start;
            p.la = runs[r].len;
            p.b0 = r + 1 < runs.size() ? runs[r + 1].start : runs[r].start + runs[r].len;
            p.lb = r + 1 < runs.size() ? runs[r + 1].len : 0;
            p.out0 = p.a0;
            p.tile0 = tiles;
            p.ntiles = (uint32_t)((p.la + p.lb + MERGE_TILE - 1) / MERGE_TILE);
            if (p.ntiles == 0) p.ntiles = 1;
            tiles += p.ntiles;
            pairs.push_back(p);
            next.push_back({p.out0, p.la + p.lb});
        }
        MergePair* dpairs = (MergePair*)C.get("merge_pairs", pairs.size() * sizeof(MergePair));
        uint64_t* cor = (uint64_t*)C.get("merge_corank", (size_t)tiles * sizeof(uint64_t));
        if (!dpairs || !cor) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemcpyAsync(dpairs, pairs.data(), pairs.size() * sizeof(MergePair),
                                      cudaMemcpyHostToDevice, st));
        corank_kernel<T><<<(tiles + 255) / 256, 256, 0, st>>>(src, dpairs, (uint32_t)pairs.size(), tiles, cor);
        S512_LAUNCH_CHECK();
        int grid = 0;
        S512_CUDA_TRY(launch_persistent(C, merge_kernel<T>, MERGE_THREADS, 0, st, (int)tiles, &grid));
        merge_kernel<T><<<grid, MERGE_THREADS, 0, st>>>(src, dst, dpairs, (uint32_t)pairs.size(), tiles, cor);
        S512_LAUNCH_CHECK();
        // the host vector is reused next level: the copy above must have read it
        S512_CUDA_TRY(cudaStreamSynchronize(st));
        *launches += 2;
        std::swap(src, dst);
        runs.swap(next);
    }
    if (src != data) {
        const uint64_t n = runs.empty() ? 0 : runs[0].start + runs[0].len;
        S512_CUDA_TRY(cudaMemcpyAsync(data, src, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    }
    return S512_OK;
}

template <typename T>
static int merge_entry(T* data, size_t n, size_t middle, int flags, void* stream) {
    if (n == 0 || middle == 0 || middle >= n) return S512_OK;  // nothing to merge
    if (!data) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    CallGuard guard(C, st);
    S512_HOST_PTR(host, data, flags);
    T* d = data;
    if (host) {
        d = (T*)C->get("stage0", n * sizeof(T));
        if (!d) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemcpyAsync(d, data, n * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    T* tmp = (T*)C->get("merge_tmp", n * sizeof(T));
    if (!tmp) return S512_ERR_ALLOC;
    s512_stats& S = thread_stats();
    memset(&S, 0, sizeof(S));
    S.key_bytes = sizeof(T);
    std::vector<Run> runs = {{0, middle}, {middle, n - middle}};
    int rc = merge_tree<T>(*C, d, tmp, runs, st, &S.kernel_launches);
    if (rc) return rc;
    if (host) S512_CUDA_TRY(cudaMemcpyAsync(data, d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    guard.finish();
    if (host || !(flags & S512_ASYNC)) S512_CUDA_TRY(cudaStreamSynchronize(st));
    return S512_OK;
}

template <typename T>
static int sort_by_chunks(T* data, size_t n, int nparts, int flags, void* stream,
                          int (*sort_fn)(T*, size_t, int, void*)) {
    if (n == 0) return S512_OK;
    if (!data || nparts < 1) return S512_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int status = S512_OK;
    DevCtx* C = current_ctx(&status, st);
    if (!C) return status;
    S512_HOST_PTR(host, data, flags);
    T* d = data;
    if (host) {
        CallGuard g(C, st);
        d = (T*)C->get("chunk_stage", n * sizeof(T));
        if (!d) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemcpyAsync(d, data, n * sizeof(T), cudaMemcpyHostToDevice, st));
        g.finish();
    }
    // 1. every chunk sorted on its own (the reference's per-thread CoreSort)
    const uint64_t chunk = (n + (uint64_t)nparts - 1) / (uint64_t)nparts;
    std::vector<Run> runs;
    for (uint64_t first = 0; first < n; first += chunk) {
        const uint64_t len = first + chunk <= n ? chunk : n - first;
        int rc = sort_fn(d + first, len, S512_PTR_DEVICE | S512_ASYNC, stream);
        if (rc) return rc;
        runs.push_back({first, len});
    }
    // 2. the merge tree, one merge-path pass per level
    CallGuard guard(C, st);
    T* tmp = (T*)C->get("merge_tmp", n * sizeof(T));
    if (!tmp) return S512_ERR_ALLOC;
    s512_stats& S = thread_stats();
    uint32_t launches = 0;
    int rc = merge_tree<T>(*C, d, tmp, runs, st, &launches);
    if (rc) return rc;
    S.kernel_launches += launches;
    if (host) S512_CUDA_TRY(cudaMemcpyAsync(data, d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    guard.finish();
    if (host || !(flags & S512_ASYNC)) S512_CUDA_TRY(cudaStreamSynchronize(st));
    return S512_OK;
}

static int sort_i32_fn(int* d, size_t n, int flags, void* st) { return s512_sort_i32(d, n, flags, st); }
static int sort_f64_fn(double* d, size_t n, int flags, void* st) { return s512_sort_f64(d, n, flags, st); }

}  // namespace s512

extern "C" {

int s512_merge_i32(int* data, size_t n, size_t middle, int flags, void* stream) {
    return s512::merge_entry<int>(data, n, middle, flags, stream);
}
int s512_merge_f64(double* data, size_t n, size_t middle, int flags, void* stream) {
    return s512::merge_entry<double>(data, n, middle, flags, stream);
}
int s512_sort_omp_merge_i32(int* data, size_t n, int nparts, int flags, void* stream) {
    return s512::sort_by_chunks<int>(data, n, nparts, flags, stream, s512::sort_i32_fn);
}
int s512_sort_omp_merge_f64(double* data, size_t n, int nparts, int flags, void* stream) {
    return s512::sort_by_chunks<double>(data, n, nparts, flags, stream, s512::sort_f64_fn);
}

}  // extern "C"
