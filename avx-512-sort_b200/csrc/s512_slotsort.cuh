// s512_slotsort.cuh -- one bucket sorted by distribution counting: keys are
// dealt into value slots by a monotone linear map of their offset from the
// bucket's minimum, the slots are laid out by an exclusive scan of their
// counts, the keys are dealt into their slots, and each slot that received
// more than one key (a few keys at most) is put in order in place by the
// thread that scanned it; the buffer is then the sorted bucket.
//
// A bucket that reaches the leaf stage holds the keys between two adjacent
// quantile splitters, so its values are close to evenly spread over
// [min, max]: with as many slots as the class has keys, a slot holds about
// one key and the whole sort costs a few shared-memory operations per key,
// where a comparison network costs one compare-exchange per key for every
// stage.  When the spread is uneven (a cluster, a run of repeated values, an
// outlier that stretches the range) the slot counts show it before any key
// moves: if the largest slot exceeds SLOT_MAX_RUN keys, or the ranking work
// (the sum of squared slot counts) exceeds SLOT_SUMSQ per key, the bucket is
// sorted by the bitonic + merge-path block sort instead (s512_blocksort.cuh).
//
// Equal keys are identical encoded words (see s512_common.cuh), so placing
// ties in any order gives the same output.
#pragma once

#include "s512_blocksort.cuh"

namespace s512 {

constexpr uint32_t SLOT_MAX_RUN = 32;  // largest slot put in order by one thread
constexpr uint32_t SLOT_SUMSQ = 4;     // in-slot ordering work (sum of squared counts) allowed per key

// Monotone map from a key in [lo, hi] to a slot in [0, nslots): the offset
// x - lo is cut to its 32 leading significant bits (shift sh), then either
// used as the slot itself (direct, when the cut range is below nslots) or
// scaled by mul / 2^32 with mul = floor(nslots * 2^32 / (range + 1)), which
// keeps the largest offset below nslots.
template <typename K>
struct SlotMap {
    K lo;
    uint32_t sh, mul, direct;
    __device__ __forceinline__ uint32_t operator()(K x) const {
        const uint32_t d = (uint32_t)((x - lo) >> sh);
        return direct ? d : __umulhi(d, mul);
    }
};

template <typename K>
__device__ __forceinline__ SlotMap<K> make_slot_map(K lo, K hi, uint32_t nslots) {
    SlotMap<K> f;
    f.lo = lo;
    const K range = hi - lo;
    int nb;
    if constexpr (sizeof(K) == 8) nb = 64 - __clzll((long long)range);
    else nb = 32 - __clz((int)range);
    f.sh = nb > 32 ? (uint32_t)(nb - 32) : 0u;
    const uint32_t dr = (uint32_t)(range >> f.sh);
    f.direct = dr < nslots ? 1u : 0u;
    f.mul = f.direct ? 0u : (uint32_t)(((uint64_t)nslots << 32) / ((uint64_t)dr + 1));
    return f;
}

// Per-warp partials of the block reductions.
template <typename K>
struct SlotRed {
    K wlo[32], whi[32];
    uint32_t wtot[32], wmax[32], wsq[32];
};

// Shared memory of block_slot_sort for a block of THREADS x IPT keys: the
// key buffer (padded for the block sort when that runs inline, INLINE) and
// the counters.
template <typename K, int THREADS, int IPT, bool INLINE = true>
struct SlotSmem {
    static constexpr uint32_t S = (uint32_t)THREADS * IPT;
    static constexpr size_t keys_bytes = ((size_t)(INLINE ? padded_len(S) : S) * sizeof(K) + 15) & ~(size_t)15;
    static constexpr size_t ctr_bytes = (size_t)S * sizeof(uint32_t);
    static constexpr size_t bytes = keys_bytes + ctr_bytes;
};

// Sort the c <= THREADS*IPT keys held striped in key[] (element
// r*THREADS + tid in key[r]; entries past c are ignored) into store(0..c).
// `smem` holds SlotSmem<K,THREADS,IPT>::bytes; `red` is the block's reduction
// scratch.  refill() is called exactly once, as soon as key[] is no longer
// needed, so that the caller can start loading the next bucket into it while
// this one is ranked and written.  Every thread of the block must call it; it
// ends with a barrier, so the caller may reuse the shared memory right after.
// Returns true when the bucket took the distribution-counting path.
//
// An uneven bucket is sorted here by the block sort when INLINE_FALLBACK is
// set; otherwise thread 0 calls uneven() (which hands the bucket to a
// separate launch) and nothing is written.  Keeping the block sort out of
// the kernel keeps the slot path's register budget for the keys.
template <typename K, int THREADS, int IPT, bool INLINE_FALLBACK, typename Store, typename Refill, typename Uneven>
__device__ bool block_slot_sort(K (&key)[IPT], uint32_t c, Store store, Refill refill, Uneven uneven,
                                unsigned char* smem, SlotRed<K>& red) {
    constexpr uint32_t S = (uint32_t)THREADS * IPT;
    constexpr int NW = THREADS / 32;
    static_assert(IPT % 4 == 0 && IPT <= 32, "counters are read four at a time, slot bits in one word");
    using SM = SlotSmem<K, THREADS, IPT, INLINE_FALLBACK>;
    K* s = reinterpret_cast<K*>(smem);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(smem + SM::keys_bytes);
    const unsigned tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;

    // 1. bounds of the bucket; counters zeroed
    K lo = KeyMax<K>::value, hi = K(0);
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        if ((uint32_t)r * THREADS + tid < c) {
            lo = kmin(lo, key[r]);
            hi = kmax(hi, key[r]);
        }
    }
#pragma unroll
    for (int r = 0; r < IPT; r += 4)
        *reinterpret_cast<uint4*>(&ctr[tid * IPT + r]) = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        lo = kmin(lo, shfl_xor(lo, d));
        hi = kmax(hi, shfl_xor(hi, d));
    }
    if (lane == 0) {
        red.wlo[warp] = lo;
        red.whi[warp] = hi;
    }
    __syncthreads();
    lo = lane < (unsigned)NW ? red.wlo[lane] : KeyMax<K>::value;
    hi = lane < (unsigned)NW ? red.whi[lane] : K(0);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        lo = kmin(lo, shfl_xor(lo, d));
        hi = kmax(hi, shfl_xor(hi, d));
    }

    if (lo == hi) {  // every key equal: already in order
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t i = (uint32_t)r * THREADS + tid;
            if (i < c) store(i, key[r]);
        }
        refill();
        __syncthreads();
        return true;
    }

    // 2. slot counts
    const SlotMap<K> f = make_slot_map<K>(lo, hi, S);
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        if ((uint32_t)r * THREADS + tid < c) atomicAdd(&ctr[f(key[r])], 1u);
    }
    __syncthreads();

    // 3. exclusive scan of the counts (IPT consecutive counters per thread)
    //    with the largest count and the sum of squared counts; one barrier:
    //    every warp scans the per-warp totals itself
    uint32_t sum = 0, mx = 0, sq = 0;
#pragma unroll
    for (int r = 0; r < IPT; r += 4) {
        const uint4 q = *reinterpret_cast<const uint4*>(&ctr[tid * IPT + r]);
        sum += q.x + q.y + q.z + q.w;
        mx = max(max(mx, max(q.x, q.y)), max(q.z, q.w));
        sq += q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    }
    uint32_t inc = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
        if (lane >= (unsigned)d) inc += o;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, d));
        sq += __shfl_xor_sync(0xFFFFFFFFu, sq, d);
    }
    if (lane == 31) red.wtot[warp] = inc;
    if (lane == 0) {
        red.wmax[warp] = mx;
        red.wsq[warp] = sq;
    }
    __syncthreads();
    uint32_t before = (lane < warp) ? red.wtot[lane] : 0u;
    mx = lane < (unsigned)NW ? red.wmax[lane] : 0u;
    sq = lane < (unsigned)NW ? red.wsq[lane] : 0u;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        before += __shfl_xor_sync(0xFFFFFFFFu, before, d);
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, d));
        sq += __shfl_xor_sync(0xFFFFFFFFu, sq, d);
    }
    const bool even = mx <= SLOT_MAX_RUN && sq <= SLOT_SUMSQ * c;

    if (even) {
        // counts -> slot starts (the counters are read again rather than kept
        // in registers across the barrier)
        uint32_t run = before + inc - sum;
        uint32_t mbits = 0;  // bit r: slot tid*IPT + r holds more than one key
#pragma unroll
        for (int r = 0; r < IPT; r += 4) {
            uint4 q = *reinterpret_cast<const uint4*>(&ctr[tid * IPT + r]);
            mbits |= ((q.x > 1u) ? 1u : 0u) << r | ((q.y > 1u) ? 1u : 0u) << (r + 1) |
                     ((q.z > 1u) ? 1u : 0u) << (r + 2) | ((q.w > 1u) ? 1u : 0u) << (r + 3);
            const uint32_t s0 = run, s1 = s0 + q.x, s2 = s1 + q.y, s3 = s2 + q.z;
            run = s3 + q.w;
            q = make_uint4(s0, s1, s2, s3);
            *reinterpret_cast<uint4*>(&ctr[tid * IPT + r]) = q;
        }
        __syncthreads();
        // 4. deal the keys into their slots; afterwards ctr[j] is the end of slot j
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            if ((uint32_t)r * THREADS + tid < c) s[atomicAdd(&ctr[f(key[r])], 1u)] = key[r];
        }
        refill();
        __syncthreads();
        // 5. the keys of a slot of several are in dealing order: the thread
        //    that scanned the slot puts them in key order, in place
        for (uint32_t bits = mbits; bits; bits &= bits - 1) {
            const uint32_t j = tid * IPT + (uint32_t)(__ffs(bits) - 1);
            const uint32_t a = j ? ctr[j - 1] : 0u;
            const uint32_t e = ctr[j];
            if (e - a == 2) {
                const K x0 = s[a], x1 = s[a + 1];
                if (x1 < x0) {
                    s[a] = x1;
                    s[a + 1] = x0;
                }
            } else {
                for (uint32_t q = a + 1; q < e; ++q) {
                    const K x = s[q];
                    uint32_t k = q;
                    for (; k > a; --k) {
                        const K y = s[k - 1];
                        if (!(x < y)) break;
                        s[k] = y;
                    }
                    s[k] = x;
                }
            }
        }
        __syncthreads();
        // 6. every key is in its final place
        for (uint32_t p = tid; p < c; p += THREADS) store(p, s[p]);
    } else if constexpr (INLINE_FALLBACK) {
        // uneven spread: bitonic leaves + merge path on the same keys
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t i = (uint32_t)r * THREADS + tid;
            if (i < c) s[pidx(i)] = key[r];
        }
        block_merge_sort<K, THREADS, IPT>(s, c);
        for (uint32_t i = tid; i < c; i += THREADS) store(i, s[pidx(i)]);
        refill();  // (after the merge, which needs the registers)
    } else {
        if (tid == 0) uneven();
        refill();
    }
    __syncthreads();
    return even;
}

}  // namespace s512
