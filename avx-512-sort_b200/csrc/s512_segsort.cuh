// s512_segsort.cuh -- kernels of the batched segmented sort.
//
// The reference's analogue is a loop of SmallSort16V (or Sort) over
// independent arrays (sort512perf.cpp:612-709 timeSmall).  Here a batch of
// segments is classified once by length, then one persistent launch sorts
// every segment of up to a block's capacity: blocks first take "block"
// segments from an atomic queue (one block per segment: the slot sort of
// s512_slotsort.cuh, with the bitonic + merge-path block sort for segments
// whose values are unevenly spread), then every warp takes "warp" segments of
// at most 256 keys (one bitonic network per warp).  Longer segments run the partition levels.
#pragma once

#include "s512_blocksort.cuh"
#include "s512_sortpipe.cuh"

namespace s512 {

struct SegItem {
    uint64_t off;
    uint32_t count;
    uint32_t pad_;
};

struct SegCtl {
    uint32_t n_warp, n_block, n_big;
    uint32_t ctr_block, ctr_warp;
    uint32_t err;
    unsigned long long big_keys;
};

constexpr int WARP_SEG_MAX = 256;
constexpr uint32_t WARP_REGION = padded_len(WARP_SEG_MAX);  // keys of shared memory per warp

// one warp appends to a list: warp-aggregated slot reservation
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
    const unsigned m = __ballot_sync(0xFFFFFFFFu, pred);
    if (!m) return 0;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return base + __popc(m & ((1u << lane_id()) - 1u));
}

__global__ void segsort_classify_kernel(const size_t* __restrict__ offsets, size_t nseg, uint32_t block_cap,
                                        SegItem* __restrict__ warp_items, SegItem* __restrict__ block_items,
                                        SegDesc* __restrict__ big, SegCtl* __restrict__ ctl) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < nseg; base += stride) {
        const size_t i = base + threadIdx.x;
        uint64_t off = 0, len = 0;
        if (i < nseg) {
            off = offsets[i];
            len = offsets[i + 1] - off;
        }
        const bool w = len > 1 && len <= (uint64_t)WARP_SEG_MAX;
        const bool b = len > (uint64_t)WARP_SEG_MAX && len <= block_cap;
        const bool g = len > block_cap;
        const uint32_t sw = warp_append(&ctl->n_warp, w);
        const uint32_t sb = warp_append(&ctl->n_block, b);
        const uint32_t sg = warp_append(&ctl->n_big, g);
        if (w) warp_items[sw] = SegItem{off, (uint32_t)len, 0u};
        if (b) block_items[sb] = SegItem{off, (uint32_t)len, 0u};
        if (g) {
            SegDesc d;
            d.in_off = off;
            d.count = len;
            d.final_off = off;
            d.out_base = 0;
            d.tile_start = 0;
            d.ntiles = 0;
            big[sg] = d;
            atomicAdd(&ctl->big_keys, (unsigned long long)len);
        }
    }
}

// The persistent launch for warp and block segments.  io reads and writes the
// caller's layout in place.
template <typename Codec, int THREADS, int EPT>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) segsort_small_kernel(Codec io, const SegItem* __restrict__ warp_items,
                                                                const SegItem* __restrict__ block_items,
                                                                SegCtl* __restrict__ ctl) {
    using K = typename Codec::Key;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* s = reinterpret_cast<K*>(smem_raw);
    __shared__ uint32_t s_item;
    __shared__ SlotRed<K> red;
    const uint32_t nblock = ctl->n_block;
    const uint32_t nwarp = ctl->n_warp;

    // block segments
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(&ctl->ctr_block, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        __syncthreads();
        if (it >= nblock) break;
        const SegItem item = block_items[it];
        K key[EPT];
#pragma unroll
        for (int r = 0; r < EPT; ++r) {
            const uint32_t i = (uint32_t)r * THREADS + threadIdx.x;
            if (i < item.count) key[r] = io.load(item.off + i);
        }
        block_slot_sort<K, THREADS, EPT, true>(
            key, item.count, [&](uint32_t i, K x) { io.store(item.off + i, x); }, [] {}, [] {}, smem_raw, red);
    }

    // warp segments
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    K* sw = s + (size_t)warp * WARP_REGION;
    while (true) {
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(&ctl->ctr_warp, 1u);
        w = __shfl_sync(0xFFFFFFFFu, w, 0);
        if (w >= nwarp) break;
        const SegItem item = warp_items[w];
        for (uint32_t i = lane; i < (uint32_t)WARP_SEG_MAX; i += 32)
            sw[pidx(i)] = i < item.count ? io.load(item.off + i) : KeyMax<K>::value;
        __syncwarp();
        K x[CHUNK_IPT];
#pragma unroll
        for (int r = 0; r < CHUNK_IPT; ++r) x[r] = sw[pidx(lane * CHUNK_IPT + r)];
        warp_bitonic_sort<K, CHUNK_IPT>(x);
#pragma unroll
        for (int r = 0; r < CHUNK_IPT; ++r) sw[pidx(lane * CHUNK_IPT + r)] = x[r];
        __syncwarp();
        for (uint32_t i = lane; i < item.count; i += 32) io.store(item.off + i, sw[pidx(i)]);
        __syncwarp();
    }
}

// Random keys for the autotuner's timing runs.
template <typename Codec>
__global__ void segsort_fill_kernel(Codec io, uint64_t n, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        io.store(i, mix64(seed ^ i));
}

}  // namespace s512
