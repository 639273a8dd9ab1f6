// s512_merge.cuh -- merge-path merging of sorted runs in global memory.
//
// The reference merges sorted runs in its OpenMP drivers: SortOmpMerge and
// SortOmpMergeDeps call std::inplace_merge on neighbouring chunks level by
// level (sort512.hpp:6045, 6092); SortOmpParMerge calls
// ParallelInplace::parallelMergeInPlace (parallelInplace.hpp:210-306), which
// splits a merge between threads with FindMedian (78-135) -- a binary search
// for where a diagonal of the merge crosses the two runs -- and rotates the
// middle parts into place (reorderShifting, 31-75).
//
// On the GPU the same split is the merge path: the output of a pair of runs
// is cut into tiles of TILE outputs; corank_kernel finds, for every tile
// boundary at once, how many of the first d outputs come from the left run
// (binary search); merge_kernel then loads each tile's two input slices into
// shared memory and every thread merges its own EPT outputs after a second,
// shared-memory co-rank search.  Comparisons use the element type's own `<`
// and take from the left run on ties, which is std::inplace_merge's (stable)
// result.
#pragma once

#include "s512_common.cuh"

namespace s512 {

// One pair of adjacent sorted runs to merge: a = src[a0, a0+la), b = src[b0, b0+lb)
// into dst[out0, out0+la+lb).  tile0 = first tile of this pair.
struct MergePair {
    uint64_t a0, la, b0, lb, out0;
    uint32_t tile0, ntiles;
};

constexpr int MERGE_THREADS = 256;
constexpr int MERGE_EPT = 16;
constexpr int MERGE_TILE = MERGE_THREADS * MERGE_EPT;  // 4096 outputs per tile

// smallest i in [max(0,d-lb), min(d,la)] such that a[i] > b[d-1-i] (ties -> a first)
template <typename T, typename AF, typename BF>
__device__ __forceinline__ uint64_t corank(uint64_t d, uint64_t la, uint64_t lb, AF a, BF b) {
    uint64_t lo = d > lb ? d - lb : 0;
    uint64_t hi = d < la ? d : la;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (b(d - 1 - mid) < a(mid)) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t pair_of_tile(const MergePair* pairs, uint32_t npairs, uint32_t t) {
    uint32_t lo = 0, hi = npairs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pairs[mid].tile0 <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// co-rank of every tile start; corank_out[t] = number of left-run keys among
// the pair's first (t - tile0) * TILE outputs
template <typename T>
__global__ void corank_kernel(const T* __restrict__ src, const MergePair* __restrict__ pairs, uint32_t npairs,
                              uint32_t ntiles, uint64_t* __restrict__ corank_out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const MergePair p = pairs[pair_of_tile(pairs, npairs, t)];
    const uint64_t d = (uint64_t)(t - p.tile0) * MERGE_TILE;
    const T* a = src + p.a0;
    const T* b = src + p.b0;
    corank_out[t] = corank<T>(d, p.la, p.lb, [&](uint64_t i) { return a[i]; }, [&](uint64_t j) { return b[j]; });
}

template <typename T>
__global__ void __launch_bounds__(MERGE_THREADS) merge_kernel(const T* __restrict__ src, T* __restrict__ dst,
                                                              const MergePair* __restrict__ pairs, uint32_t npairs,
                                                              uint32_t ntiles, const uint64_t* __restrict__ coranks) {
    // one tile's two input slices, left then right (na + nb <= MERGE_TILE);
    // each thread merges its outputs into registers, then writes them back
    // here for a coalesced store
    __shared__ T buf[MERGE_TILE + 1];
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const MergePair p = pairs[pair_of_tile(pairs, npairs, t)];
        const uint64_t total = p.la + p.lb;
        const uint64_t d0 = (uint64_t)(t - p.tile0) * MERGE_TILE;
        const uint64_t d1 = d0 + MERGE_TILE < total ? d0 + MERGE_TILE : total;
        const uint64_t i0 = coranks[t];
        const uint64_t i1 = (t + 1 < p.tile0 + p.ntiles) ? coranks[t + 1] : p.la;
        const uint64_t j0 = d0 - i0, j1 = d1 - i1;
        const uint32_t na = (uint32_t)(i1 - i0), nb = (uint32_t)(j1 - j0), nout = (uint32_t)(d1 - d0);
        T* sa = buf;
        T* sb = buf + na;
        for (uint32_t k = threadIdx.x; k < na; k += MERGE_THREADS) sa[k] = src[p.a0 + i0 + k];
        for (uint32_t k = threadIdx.x; k < nb; k += MERGE_THREADS) sb[k] = src[p.b0 + j0 + k];
        __syncthreads();
        const uint32_t o0 = threadIdx.x * MERGE_EPT;
        T out[MERGE_EPT];
        uint32_t cnt = 0;
        if (o0 < nout) {
            uint32_t ia = (uint32_t)corank<T>(o0, na, nb, [&](uint64_t i) { return sa[i]; },
                                              [&](uint64_t j) { return sb[j]; });
            uint32_t ib = o0 - ia;
            cnt = nout - o0 < (uint32_t)MERGE_EPT ? nout - o0 : (uint32_t)MERGE_EPT;
#pragma unroll
            for (int k = 0; k < MERGE_EPT; ++k) {
                if ((uint32_t)k < cnt) {
                    const bool take_a = ib >= nb || (ia < na && !(sb[ib] < sa[ia]));
                    out[k] = take_a ? sa[ia] : sb[ib];
                    ia += take_a ? 1u : 0u;
                    ib += take_a ? 0u : 1u;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < MERGE_EPT; ++k)
            if ((uint32_t)k < cnt) buf[o0 + k] = out[k];
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < nout; k += MERGE_THREADS) dst[p.out0 + d0 + k] = buf[k];
        __syncthreads();
    }
}

}  // namespace s512
