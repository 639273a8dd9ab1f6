// s512_segsort.cuh -- kernels of the batched segmented sort.
//
// The reference's analogue is a loop of SmallSort16V (or Sort) over
// independent arrays (sort512perf.cpp:612-709 timeSmall).  Here a batch of
// segments is classified once by length into size classes: segments of at
// most 256 keys are sorted one per warp (a bitonic network in registers);
// longer ones, up to the largest block class, one per block of the smallest
// class that holds them (the slot sort of s512_slotsort.cuh, with the
// bitonic + merge-path block sort for segments whose values are unevenly
// spread), each class by its own persistent launch sized for it, so that a
// 300-key segment does not pay for the counters of a 16K-key block.  Longer
// segments run the partition levels.
#pragma once

#include "s512_blocksort.cuh"
#include "s512_sortpipe.cuh"

namespace s512 {

struct SegItem {
    uint64_t off;
    uint32_t count;
    uint32_t pad_;
};

// Block classes: class c holds segments of up to 1024 << c keys.
constexpr int SEG_NCLASS = 5;
__host__ __device__ constexpr uint32_t seg_class_cap(int c) { return 1024u << c; }

struct SegCtl {
    uint32_t n_warp, n_big;
    uint32_t n_cls[SEG_NCLASS];
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

// Segments of 2..256 keys to the warp list, of up to max_cap keys to the list
// of the smallest block class that holds them (class c's list starts at
// cls_items + c * cls_stride), longer ones to the partition list.
__global__ void segsort_classify_kernel(const size_t* __restrict__ offsets, size_t nseg, uint32_t max_cap,
                                        SegItem* __restrict__ warp_items, SegItem* __restrict__ cls_items,
                                        size_t cls_stride, SegDesc* __restrict__ big, SegCtl* __restrict__ ctl) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < nseg; base += stride) {
        const size_t i = base + threadIdx.x;
        uint64_t off = 0, len = 0;
        if (i < nseg) {
            off = offsets[i];
            len = offsets[i + 1] - off;
        }
        const bool w = len > 1 && len <= (uint64_t)WARP_SEG_MAX;
        const bool blk = len > (uint64_t)WARP_SEG_MAX && len <= max_cap;
        const bool g = len > max_cap;
        int cls = -1;
        if (blk) {
            cls = 0;
            while (seg_class_cap(cls) < len) ++cls;
        }
        const uint32_t sw = warp_append(&ctl->n_warp, w);
        const uint32_t sg = warp_append(&ctl->n_big, g);
        if (w) warp_items[sw] = SegItem{off, (uint32_t)len, 0u};
#pragma unroll
        for (int c = 0; c < SEG_NCLASS; ++c) {
            const uint32_t sc = warp_append(&ctl->n_cls[c], cls == c);
            if (cls == c) cls_items[(size_t)c * cls_stride + sc] = SegItem{off, (uint32_t)len, 0u};
        }
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

// Warp segments: one warp per segment (8 warps per block), in place on the
// caller's layout.
template <typename Codec>
__global__ void __launch_bounds__(256) segsort_warp_kernel(Codec io, const SegItem* __restrict__ items,
                                                           const SegCtl* __restrict__ ctl) {
    using K = typename Codec::Key;
    __shared__ K stage[8][WARP_REGION];
    const uint32_t nitems = ctl->n_warp;
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    K* sw = stage[warp];
    for (uint32_t w = blockIdx.x * 8 + warp; w < nitems; w += gridDim.x * 8) {
        const SegItem item = items[w];
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

// One block class: one block per segment of at most THREADS * EPT keys; the
// next segment's keys are loaded into registers while the current one is
// ranked and written.
template <typename Codec, int THREADS, int EPT>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
    segsort_block_kernel(Codec io, const SegItem* __restrict__ items, const uint32_t* __restrict__ n_items) {
    using K = typename Codec::Key;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ SlotRed<K> red;
    const uint32_t nitems = *n_items;
    uint32_t it = blockIdx.x;
    if (it >= nitems) return;
    SegItem cur = items[it];
    K key[EPT];
    auto load = [&](const SegItem& item) {
#pragma unroll
        for (int r = 0; r < EPT; ++r) {
            const uint32_t i = (uint32_t)r * THREADS + threadIdx.x;
            if (i < item.count) key[r] = io.load(item.off + i);
        }
    };
    load(cur);
    for (; it < nitems; it += gridDim.x) {
        const uint32_t nx = it + gridDim.x;
        SegItem next;
        next.count = 0;
        if (nx < nitems) next = items[nx];
        const uint64_t off = cur.off;
        block_slot_sort<K, THREADS, EPT, true>(
            key, cur.count, [&](uint32_t i, K x) { io.store(off + i, x); }, [&]() { load(next); }, [] {}, smem_raw,
            red);
        cur = next;
    }
}

// Random keys for the autotuner's timing runs.
template <typename Codec>
__global__ void segsort_fill_kernel(Codec io, uint64_t n, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        io.store(i, mix64(seed ^ i));
}

}  // namespace s512
