// s512_blocksort.cuh -- block-level sort of one bucket held in shared memory:
// bitonic leaves of 256 keys (one warp each, registers + __shfl_xor_sync, the
// SmallSort16V network of s512_bitonic.cuh) followed by merge-path merges of
// the sorted runs inside shared memory.
//
// This pairs the reference's two building blocks: the bitonic leaf
// (SmallSort16V, sort512.hpp:5312-5689) and the merge of sorted runs that its
// parallel drivers do (SortOmpMerge's std::inplace_merge, sort512.hpp:6045,
// and the median-split merge of parallelInplace.hpp:78-207, which is a merge
// path: FindMedian finds where a diagonal crosses two sorted runs).  Here every
// thread finds its own diagonal by binary search (the co-rank) and merges
// EPT outputs serially, so one merge level costs one read and one write of
// shared memory per key.
//
// Shared-memory layout: key e lives at e + e/8 (one pad slot every 8 keys), so
// that a warp reading "8 consecutive keys per lane" hits distinct banks.
#pragma once

#include "s512_bitonic.cuh"

namespace s512 {

constexpr int CHUNK_IPT = 8;             // keys per lane in a warp's bitonic leaf
constexpr int CHUNK = 32 * CHUNK_IPT;    // 256 keys per warp leaf

__host__ __device__ constexpr uint32_t padded_len(uint32_t n) { return n + n / 8 + 8; }
__device__ __forceinline__ uint32_t pidx(uint32_t e) { return e + (e >> 3); }

// Sort s[0..c) (padded layout) ascending.  s must hold padded_len(N) keys with
// N >= round_up(c, CHUNK) and N <= THREADS*EPT.  Keys [c, round_up(c,CHUNK))
// are filled with the maximum here.  All threads of the block must call it.
template <typename K, int THREADS, int EPT>
__device__ void block_merge_sort(K* s, uint32_t c) {
    constexpr int NW = THREADS / 32;
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t nch = (c + CHUNK - 1) / CHUNK;
    const uint32_t npad = nch * CHUNK;
    for (uint32_t i = c + threadIdx.x; i < npad; i += THREADS) s[pidx(i)] = KeyMax<K>::value;
    __syncthreads();

    // 1. bitonic leaves: one warp per 256-key chunk
    for (uint32_t ch = warp; ch < nch; ch += NW) {
        const uint32_t base = ch * CHUNK + lane * CHUNK_IPT;
        K x[CHUNK_IPT];
#pragma unroll
        for (int r = 0; r < CHUNK_IPT; ++r) x[r] = s[pidx(base + r)];
        warp_bitonic_sort<K, CHUNK_IPT>(x);
#pragma unroll
        for (int r = 0; r < CHUNK_IPT; ++r) s[pidx(base + r)] = x[r];
    }
    __syncthreads();

    // 2. merge-path merges: runs of L keys -> 2L, in place (read all, sync, write)
    for (uint32_t L = CHUNK; L < npad; L <<= 1) {
        K out[EPT];
        const uint32_t base = threadIdx.x * EPT;
        const bool active = base < npad;
        if (active) {
            const uint32_t pair0 = (base / (2 * L)) * (2 * L);
            const uint32_t a0 = pair0;
            const uint32_t la = min(L, npad - a0);
            const uint32_t b0 = a0 + la;
            const uint32_t lb = b0 < npad ? min(L, npad - b0) : 0u;
            const uint32_t d = base - pair0;
            // co-rank: smallest i with a[i] > b[d-1-i]
            uint32_t lo = d > lb ? d - lb : 0u;
            uint32_t hi = min(d, la);
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s[pidx(a0 + mid)] > s[pidx(b0 + d - 1 - mid)]) hi = mid;
                else lo = mid + 1;
            }
            uint32_t ai = a0 + lo, bi = b0 + (d - lo);
            const uint32_t ae = a0 + la, be = b0 + lb;
            K va = ai < ae ? s[pidx(ai)] : K(0);
            K vb = bi < be ? s[pidx(bi)] : K(0);
#pragma unroll
            for (int k = 0; k < EPT; ++k) {
                const bool take_a = bi >= be || (ai < ae && !(vb < va));
                out[k] = take_a ? va : vb;
                if (take_a) {
                    ++ai;
                    if (ai < ae) va = s[pidx(ai)];
                } else {
                    ++bi;
                    if (bi < be) vb = s[pidx(bi)];
                }
            }
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k = 0; k < EPT; ++k)
                if (base + k < npad) s[pidx(base + k)] = out[k];
        }
        __syncthreads();
    }
}

}  // namespace s512
