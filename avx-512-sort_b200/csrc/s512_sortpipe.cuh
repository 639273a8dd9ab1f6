// s512_sortpipe.cuh -- partition-then-sort pipeline for one GPU.
//
// The reference sorts by recursive two-way partitioning (Partition512,
// sort512.hpp:5729-5912, driven by CoreSort 5947-5958 with the pseudo-median
// pivot of CoreSortGetPivot 5916-5927) down to leaves of at most 16 vectors
// (SortLimite = 16*64/sizeof(T), 5949), which SmallSort16V sorts with bitonic
// networks.  This file keeps that method and widens each step for a GPU:
//
//   * a pivot becomes up to 255 splitters drawn from a random sample of the
//     segment (sorted on the device), so one partition pass splits a segment
//     into up to 256 buckets instead of 2;
//   * splitter values that repeat in the sample get an equality bucket (keys
//     equal to that value need no further sorting), which removes the
//     reference's quadratic behaviour on few-distinct and sorted inputs;
//   * the partition pass is out of place and "one sweep": every tile of keys
//     computes its bucket histogram, reserves its share of each bucket's
//     output region with one atomic add per bucket, then scatters its keys
//     through shared memory so global writes are coalesced.  Bucket b of a
//     segment is written into a region whose capacity comes from the sample
//     (a 6-sigma bound); a bucket that outgrows it is reported and the level
//     is redone with exact counts;
//   * buckets at most a leaf's capacity are sorted in shared memory (one warp
//     and the bitonic networks of s512_bitonic.cuh up to 256 keys, one block
//     and the slot sort of s512_slotsort.cuh above, by size class) and written
//     to their final place; larger buckets become the segments of the next
//     partition level.
#pragma once

#include <cstddef>
#include <type_traits>

#include "s512_slotsort.cuh"

namespace s512 {

constexpr int NB = 256;            // buckets per segment per pass (max)
constexpr int SAMPLE_N = 16384;    // keys sampled per segment
constexpr int COPY_CHUNK = 16384;  // equality buckets are copied in chunks of this size
constexpr int SPLIT_SLOTS = 4096;  // value slots of the splitter lookup table

// A segment to partition at some level.
struct SegDesc {
    uint64_t in_off;     // first key in the level's input buffer
    uint64_t count;      // number of keys
    uint64_t final_off;  // where the segment's keys end in the final output
    uint64_t out_base;   // start of the segment's bucket regions in the level's output
    uint32_t tile_start; // first global tile index of the segment
    uint32_t ntiles;
};

// Splitters of one segment and the layout of its bucket regions.
template <typename K>
struct SplitSet {
    K tree[NB];            // Eytzinger tree of the unique splitters, nodes 1..255, padded with max
                           // (the exact-count fallback's search; the pass uses slot_tab)
    K uniq[NB];            // unique splitters in ascending order (padded with max)
    uint64_t region_off[NB];  // bucket region start, relative to SegDesc::out_base
    uint64_t region_cap[NB];  // bucket region capacity (keys)
    uint8_t range_b[NB];   // bucket of keys with lower_bound index j that are not equal to uniq[j]
    uint8_t eq_b[NB];      // bucket of keys equal to uniq[j] when splitter j has an equality bucket
    uint32_t eq_mask[NB / 32];     // splitter j has an equality bucket
    uint32_t bucket_eq[NB / 32];   // bucket b is an equality bucket
    uint32_t nbuckets;
    uint32_t has_eq;
    uint32_t nuniq;
    uint32_t pad_;
    // Lookup table over the sample's value range: keys are clamped to
    // [slot_map.lo, slot_hi] and mapped to SPLIT_SLOTS slots by slot_map.
    // Entry s packs lo | cnt << 8: lo = the number of unique splitters whose
    // slot is below s, cnt = how many share slot s.  A key of slot s has lo
    // splitters below it for sure and still has to be compared with
    // uniq[lo .. lo+cnt) -- none for most keys (255 splitters, 4096 slots).
    SlotMap<K> slot_map;
    K slot_hi;
    alignas(16) uint16_t slot_tab[SPLIT_SLOTS + 8];
};

// A bucket that a leaf kernel sorts (or copies) into its final place.
template <typename K>
struct LeafItem {
    const K* src;        // encoded keys in a level buffer
    uint64_t dst;        // index of the first key in the caller's output
    uint32_t count;
    uint32_t pad_;
};

// Leaf size classes.  Class 0 is one warp per bucket (a 256-key bitonic
// leaf); the others are one block per bucket (the slot sort of
// s512_slotsort.cuh, with the bitonic + merge-path block sort for uneven
// buckets).  A bucket's class is the smallest that holds it; the classes
// above 4096 are close together, because small blocks sort their keys faster
// (more buckets in flight per SM) and a bucket's keys should fill most of its
// class's slots.  The copy list holds equality buckets.
constexpr int NCLASS = 9;
constexpr int CLS_COPY = NCLASS;  // index of the copy list
__host__ __device__ constexpr int class_cap(int c) {
    return c == 0 ? 256 : c == 1 ? 1024 : c == 2 ? 2048 : c == 3 ? 4096 : c == 4 ? 4608 : c == 5 ? 5120
         : c == 6 ? 6144 : c == 7 ? 8192 : 16384;
}
__host__ __device__ constexpr uint32_t leaf_max(int /*key_bytes*/) { return 16384u; }
__host__ __device__ inline int class_of(int /*key_bytes*/, uint32_t count) {
    int c = 0;
    while (c < NCLASS - 1 && (uint32_t)class_cap(c) < count) ++c;
    return c;
}

// Number of buckets to aim for in a segment of `count` keys: enough that the
// average bucket is ~leaf_max/4, at most 256.
__host__ __device__ inline int target_buckets(int key_bytes, uint64_t count) {
    uint64_t want = (count * 4 + leaf_max(key_bytes) - 1) / leaf_max(key_bytes);
    if (want < 2) want = 2;
    if (want > NB) want = NB;
    return (int)want;
}

// Keys sampled from a segment that will be split into nb buckets: about 128
// per bucket (so a bucket's sample count is ~128 and its capacity bound ~1.6x
// its expected size), between 2048 and SAMPLE_N.
__host__ __device__ inline uint32_t sample_size(int nb) {
    uint32_t m = 128u * (uint32_t)nb;
    if (m < 2048u) m = 2048u;
    if (m > (uint32_t)SAMPLE_N) m = SAMPLE_N;
    return m;
}

// Upper bound of the total region capacity the splitter kernel may lay out
// for a segment of `count` keys (see splitter_kernel): 2.01*count + 4096.
__host__ __device__ inline uint64_t region_bound(uint64_t count) {
    return count * 2 + count / 100 + 4096;
}

// Level control block (device); read back by the host after each level.
struct LevelCtl {
    uint32_t tile_counter;
    uint32_t err;
    uint32_t n_next;          // segments for the next level
    uint32_t n_items[NCLASS + 1];
    uint32_t ntiles_next;
    uint64_t next_keys;       // keys in next-level segments
    uint64_t bound_next;      // region bound of the next level
    uint32_t max_bucket;      // largest bucket seen this level
    uint32_t nonempty;        // non-empty buckets this level
    uint64_t level_keys;      // keys partitioned this level
    uint32_t learned_used;    // segments routed by their learned model
    uint32_t plain_used;      // segments routed by the splitter tree
    uint32_t learned_fitted;  // segments whose learned model was trained
    uint32_t model_imb_bits;  // largest sample imbalance of a trained model (float bits)
    uint32_t n_uneven[NCLASS];  // leaves handed from the slot sort to the block sort
    uint32_t never_set;       // testing: a flag nothing writes (the injected wait)
    double bucket_sq;         // sum of squared non-empty bucket sizes this level
};

// ===========================================================================
// 1. Sampling: SAMPLE_N keys per segment at hashed positions (with replacement)

template <typename Codec>
__global__ void sample_kernel(Codec in, const SegDesc* __restrict__ segs, uint32_t nsegs,
                              typename Codec::Key* __restrict__ samples, uint64_t seed, int key_bytes) {
    const uint32_t s = blockIdx.x;
    if (s >= nsegs) return;
    const SegDesc sd = segs[s];
    const uint32_t m = sample_size(target_buckets(key_bytes, sd.count));
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
        const uint64_t h = mix64(seed ^ ((uint64_t)s << 32) ^ (uint64_t)i);
        const uint64_t pos = __umul64hi(h, sd.count);
        samples[(size_t)s * SAMPLE_N + i] = in.load(sd.in_off + pos);
    }
}

// 2. Sorting the samples: one block of 1024 threads per segment.
template <typename K>
__global__ void __launch_bounds__(1024) sample_sort_kernel(K* __restrict__ samples, const SegDesc* __restrict__ segs,
                                                           uint32_t nsegs, int key_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ SlotRed<K> red;
    constexpr int IPT = SAMPLE_N / 1024;
    const uint32_t m = sample_size(target_buckets(key_bytes, segs[blockIdx.x].count));
    K* p = samples + (size_t)blockIdx.x * SAMPLE_N;
    K key[IPT];
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const uint32_t i = (uint32_t)r * 1024 + threadIdx.x;
        if (i < m) key[r] = p[i];
    }
    // samples are spread like the segment's keys: distribution counting,
    // with the block sort for skewed samples (s512_slotsort.cuh)
    block_slot_sort<K, 1024, IPT, true>(
        key, m, [&](uint32_t i, K x) { p[i] = x; }, [] {}, [] {}, smem_raw, red);
}

// 3. Splitters and bucket regions: one block of 256 threads per segment.
template <typename K>
__device__ __forceinline__ uint32_t lower_bound_dev(const K* a, uint32_t n, K v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}
template <typename K>
__device__ __forceinline__ uint32_t upper_bound_dev(const K* a, uint32_t n, K v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (!(v < a[mid])) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <typename K>
__global__ void __launch_bounds__(256) splitter_kernel(const K* __restrict__ samples, const SegDesc* __restrict__ segs,
                                                       uint32_t nsegs, SplitSet<K>* __restrict__ splits,
                                                       int key_bytes) {
    const uint32_t s = blockIdx.x;
    if (s >= nsegs) return;
    __shared__ K cand[NB];
    __shared__ K uniq[NB];
    __shared__ uint32_t eqf[NB];
    __shared__ uint32_t wtot[8];
    __shared__ uint32_t total_u, total_eq;
    __shared__ uint64_t cap_s[NB];
    __shared__ uint64_t wtot64[8];
    __shared__ uint64_t cap_total;

    const K* smp = samples + (size_t)s * SAMPLE_N;
    const SegDesc sd = segs[s];
    SplitSet<K>* out = splits + s;
    const int t = threadIdx.x;
    const int nb = target_buckets(key_bytes, sd.count);
    const int ncand = nb - 1;
    const uint32_t m = sample_size(nb);

    // candidate splitters at the sample quantiles
    K c = KeyMax<K>::value;
    if (t < ncand) c = smp[(uint32_t)(((uint64_t)(t + 1) * m) / nb) - 1];
    cand[t] = c;
    __syncthreads();
    const bool valid = t < ncand;
    const bool first = valid && (t == 0 || cand[t] != cand[t - 1]);
    const bool dup = valid && ((t > 0 && cand[t] == cand[t - 1]) || (t + 1 < ncand && cand[t] == cand[t + 1]));
    uint32_t j = block_exclusive_scan_first<NB, uint32_t>(first ? 1u : 0u, wtot, &total_u);
    if (first) {
        uniq[j] = c;
        eqf[j] = dup ? 1u : 0u;
    }
    __syncthreads();
    const uint32_t K_u = total_u;
    if (t >= (int)K_u) {
        uniq[t] = KeyMax<K>::value;
        eqf[t] = 0;
    }
    __syncthreads();
    // splitter lookup table over [sample min, sample max]
    {
        __shared__ uint32_t sk[NB];
        const SlotMap<K> f = make_slot_map<K>(smp[0], smp[m - 1], (uint32_t)SPLIT_SLOTS);
        sk[t] = t < (int)K_u ? f(uniq[t]) : 0xFFFFFFFFu;
        if (t == 0) {
            out->slot_map = f;
            out->slot_hi = smp[m - 1];
        }
        __syncthreads();
        auto below = [&](uint32_t s) {  // splitters with slot < s
            uint32_t lo = 0, hi = K_u;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (sk[mid] < s) lo = mid + 1; else hi = mid;
            }
            return lo;
        };
        for (uint32_t s = t; s < (uint32_t)SPLIT_SLOTS + 8; s += NB) {
            const uint32_t lo = below(s);
            const uint32_t cnt = s < (uint32_t)SPLIT_SLOTS ? below(s + 1) - lo : 0u;
            out->slot_tab[s] = (uint16_t)(lo | (cnt << 8));
        }
    }
    // bucket ids: range_j, then eq_j if splitter j has one; the last range bucket is K_u
    const uint32_t my_eq = (t < (int)K_u) ? eqf[t] : 0u;
    const uint32_t eq_before = block_exclusive_scan_first<NB, uint32_t>(my_eq, wtot, &total_eq);
    const uint32_t range_id = (uint32_t)t + eq_before;  // valid for t <= K_u
    if (t <= (int)K_u) out->range_b[t] = (uint8_t)range_id;
    else out->range_b[t] = 0;
    out->eq_b[t] = (uint8_t)(my_eq ? range_id + 1 : 0);
    const uint32_t nbk = K_u + 1 + total_eq;

    // sample counts per bucket -> capacities
    // range bucket j (t <= K_u): keys in (uniq[j-1], uniq[j]] or (uniq[j-1], uniq[j]) if eq_j
    uint64_t cap_range = 0, cap_eq = 0;
    const double scale = (double)sd.count / (double)m;
    auto cap_of = [&](uint32_t cnt) -> uint64_t {
        double v = ((double)cnt + 6.0 * sqrt((double)cnt + 1.0) + 16.0) * scale;
        uint64_t cap = (uint64_t)ceil(v);
        if (cap > sd.count) cap = sd.count;
        return (cap + 15) & ~15ull;
    };
    if (t <= (int)K_u) {
        const uint32_t lo = (t == 0) ? 0u : upper_bound_dev<K>(smp, m, uniq[t - 1]);
        uint32_t hi;
        if (t == (int)K_u) hi = m;
        else hi = my_eq ? lower_bound_dev<K>(smp, m, uniq[t]) : upper_bound_dev<K>(smp, m, uniq[t]);
        cap_range = cap_of(hi > lo ? hi - lo : 0u);
        if (my_eq) {
            const uint32_t e0 = lower_bound_dev<K>(smp, m, uniq[t]);
            const uint32_t e1 = upper_bound_dev<K>(smp, m, uniq[t]);
            cap_eq = cap_of(e1 - e0);
        }
    }
    // scatter capacities into bucket order
    if (t < NB) cap_s[t] = 0;
    __syncthreads();
    if (t <= (int)K_u) {
        cap_s[range_id] = cap_range;
        if (my_eq) cap_s[range_id + 1] = cap_eq;
    }
    __syncthreads();
    const uint64_t my_cap = cap_s[t];
    const uint64_t off = block_exclusive_scan_first<NB, uint64_t>(my_cap, wtot64, &cap_total);
    out->region_off[t] = off;
    out->region_cap[t] = my_cap;
    // Eytzinger tree over uniq[0..254]: node i at depth d has in-order index
    // (2*(i - 2^d) + 1) * 2^(7-d) - 1.
    if (t >= 1 && t < NB) {
        const int d = 31 - __clz(t);
        const int io = (2 * (t - (1 << d)) + 1) * (1 << (7 - d)) - 1;
        out->tree[t] = uniq[io];
    } else {
        out->tree[0] = KeyMax<K>::value;
    }
    out->uniq[t] = uniq[t];
    // masks
    const unsigned bal_eq = __ballot_sync(0xFFFFFFFFu, my_eq != 0);
    if ((t & 31) == 0) out->eq_mask[t >> 5] = bal_eq;
    __shared__ uint32_t beq[NB / 32];
    if (t < NB / 32) beq[t] = 0;
    __syncthreads();
    if (my_eq) atomicOr(&beq[(range_id + 1) >> 5], 1u << ((range_id + 1) & 31));
    __syncthreads();
    if (t < NB / 32) out->bucket_eq[t] = beq[t];
    if (t == 0) {
        out->nbuckets = nbk;
        out->has_eq = total_eq ? 1u : 0u;
        out->nuniq = K_u;
    }
}

// Bucket of key x under a split set held in shared memory.
template <typename K>
__device__ __forceinline__ uint32_t find_bucket(const K* __restrict__ tree, K x, bool has_eq,
                                                const K* __restrict__ uniq, const uint8_t* __restrict__ range_b,
                                                const uint8_t* __restrict__ eq_b, const uint32_t* __restrict__ eq_mask) {
    uint32_t i = 1;
#pragma unroll
    for (int d = 0; d < 8; ++d) i = 2 * i + (tree[i] < x ? 1u : 0u);
    const uint32_t j = i - 256;  // number of unique splitters < x
    if (!has_eq) return j;
    if (j < 255 && ((eq_mask[j >> 5] >> (j & 31)) & 1u) && uniq[j] == x) return eq_b[j];
    return range_b[j];
}

// A split set's slot map held in registers for a run of lookups: keys are
// clamped to [lo, lo + range] (one compare: x - lo wraps above range when
// x < lo), cut to 32 bits by a funnel shift and scaled.  Same slots as
// SlotMap::operator() on the clamped key.
template <typename K>
struct SlotRegs {
    K lo, range;
    uint32_t sh, mul;
    bool direct;
    __device__ __forceinline__ SlotRegs(const SlotMap<K>& f, K hi)
        : lo(f.lo), range(hi - f.lo), sh(f.sh), mul(f.mul), direct(f.direct != 0) {}
    __device__ __forceinline__ uint32_t operator()(K x) const {
        K d = x - lo;
        if (d > range) d = x < lo ? K(0) : range;
        uint32_t d32;
        if constexpr (sizeof(K) == 8)
            d32 = __funnelshift_rc((uint32_t)d, (uint32_t)(d >> 32), sh);  // sh <= 32
        else
            d32 = (uint32_t)d >> sh;
        return direct ? d32 : __umulhi(d32, mul);
    }
};

// Bucket of key x given its slot entry (see SplitSet::slot_tab).
template <typename K>
__device__ __forceinline__ uint32_t bucket_from_slot(uint32_t e, K x, bool has_eq, const K* __restrict__ uniq,
                                                     const uint8_t* __restrict__ range_b,
                                                     const uint8_t* __restrict__ eq_b,
                                                     const uint32_t* __restrict__ eq_mask) {
    uint32_t lo = e & 0xFFu;
    const uint32_t cnt = e >> 8;
    if (cnt) {
        if (cnt == 1) {  // one splitter shares the key's slot
            lo += uniq[lo] < x ? 1u : 0u;
        } else {
            uint32_t hi = lo + cnt;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (uniq[mid] < x) lo = mid + 1; else hi = mid;
            }
        }
    }
    const uint32_t j = lo;  // number of unique splitters < x
    if (!has_eq) return j;
    if (j < 255 && ((eq_mask[j >> 5] >> (j & 31)) & 1u) && uniq[j] == x) return eq_b[j];
    return range_b[j];
}

}  // namespace s512

#include "s512_learned.cuh"

namespace s512 {

// ===========================================================================
// 4. The partition pass (persistent; tiles claimed in runs)
//
// Every tile of keys is classified, ranked within the tile by shared-memory
// atomics, staged in bucket order in shared memory and written out with
// coalesced stores.  Where a tile's keys of bucket b go inside the bucket's
// region is reserved with one global atomic add per (tile, bucket) on the
// segment's fill counter of b: the pass is not stable (a bucket's keys land in
// the order their tiles reserved, and the leaves sort them anyway), so no
// tile ever waits for another and tiles may be processed in any order.  The
// counters end as the bucket sizes.  A reservation past the region's
// capacity (the sample's 6-sigma bound) drops the tile's keys of that bucket
// and reports an overflow; the level is then redone with exact counts.
//
// Pipeline per block: the next tile travels into the second shared-memory
// buffer by a 1-D bulk copy (TMA, completing on an mbarrier) while the
// current one is ranked, staged and written; the buffer that held a tile's
// raw keys is reused to stage them in bucket order.  Three block barriers per
// tile: histogram complete | bucket starts known | staging complete.  Two
// blocks share an SM, so one block's barrier phases overlap the other's
// memory traffic.  When an input array is not 16-byte aligned the tiles are
// read with plain loads instead (a.tma == 0).
constexpr int SEG_SMEM = 256;  // segment tables up to this size are searched in shared memory
// Consecutive tiles a block claims at once: one segment's tables are loaded
// once per group, so levels with many segments take longer runs; a single
// segment takes short ones (a finer split of the last tiles among blocks).
constexpr uint32_t CLAIM_GROUP_ONE_SEG = 4;
constexpr uint32_t CLAIM_GROUP_MANY_SEGS = 16;
// Keys past the regions of a level buffer where a bucket that overflowed its
// region writes its keys of the tile (at most a tile's worth; tiles race
// there harmlessly: the level is redone with exact counts).
constexpr uint64_t JUNK_KEYS = 8192;

template <typename K>
struct PartArgs {
    const SegDesc* segs;
    uint32_t nsegs;               // segment count (host-known)
    const uint32_t* tile_seg;     // global tile -> segment (nullptr: single segment 0)
    const SplitSet<K>* splits;
    K* out;                       // level output buffer
    uint64_t junk;                // offset in out of the JUNK_KEYS overflow area
    unsigned long long* fill;     // nsegs * NB fill counters (zeroed); end as the bucket sizes
    LevelCtl* ctl;
    uint32_t ntiles;              // end of the launch's tiles (used when ntiles_dev is null)
    const uint32_t* ntiles_dev;   // tile count written by prepare_level_kernel
    uint32_t tile_first;          // first tile of the launch (a level fed in chunks launches per chunk)
    uint32_t* tile_counter;       // the launch's claim counter (zeroed)
    int tma;                      // tiles arrive by bulk copy
    const LearnedSet<K>* learned; // per segment learned model (nullptr: splitters only)
    int inject_timeout;           // testing: tile 1 waits, with a short bound, on a flag nothing sets
};

// The routing tables of a plain split set, as the partition pass keeps them.
template <typename K>
struct PlainTables {
    K uniq[NB];
    uint8_t range_b[NB];
    uint8_t eq_b[NB];
    uint32_t eq_mask[NB / 32];
    SlotMap<K> fmap;
    K fhi;
    alignas(16) uint16_t tab[SPLIT_SLOTS + 8];
};

// Bytes of a LearnedSet that inference reads (its leading fields).
template <typename K>
constexpr size_t learned_model_bytes() { return offsetof(LearnedSet<K>, region_off); }

template <typename K, int THREADS, int IPT>
struct PartSmem {
    static constexpr int TILE = THREADS * IPT;
    alignas(128) unsigned char buf[2][TILE * sizeof(K)];
    uint8_t bkt[TILE];
    uint64_t region_off[NB];
    uint64_t region_cap[NB];
    uint64_t gdelta[NB];
    uint32_t hist[NB];
    uint32_t loc[NB];
    uint32_t seg_tile_start[SEG_SMEM];
    uint64_t mbar[2];
    uint32_t tile_cur, has_eq, use_learned, abort;
    SegDesc sd;                   // segment of the tile being processed
    SegDesc iss_sd;               // thread 0: segment of the last tile it fetched
    uint32_t iss_seg;
    // a segment routes by its split set or by its learned model, never both
    union {
        PlainTables<K> P;
        alignas(16) unsigned char model[learned_model_bytes<K>()];
    } T;
};

template <typename K, typename InCodec, int THREADS, int IPT>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) partition_kernel(PartArgs<K> a, InCodec in) {
    extern __shared__ __align__(128) unsigned char smem_part[];
    using SM = PartSmem<K, THREADS, IPT>;
    SM& sm = *reinterpret_cast<SM*>(smem_part);
    constexpr int TILE = THREADS * IPT;
    constexpr int ESZ = InCodec::ESZ;
    constexpr int NARR = InCodec::NARR;
    static_assert(TILE < (1 << 24), "rank and bucket share a 32-bit word");
    static_assert(TILE <= (int)JUNK_KEYS, "an overflowed bucket's keys of a tile fit the overflow area");
    const int tid = threadIdx.x;
    const uint32_t ntiles = a.ntiles_dev ? *a.ntiles_dev : a.ntiles;
    const bool small_tab = a.tile_seg && a.nsegs <= (uint32_t)SEG_SMEM;
    uint32_t cached_seg = 0xFFFFFFFFu;

    if (tid == 0) {
        mbar_init(&sm.mbar[0], 1);
        mbar_init(&sm.mbar[1], 1);
        fence_mbar_init();
        sm.abort = 0;
        sm.iss_seg = 0xFFFFFFFFu;
    }
    for (int b = tid; b < NB; b += THREADS) sm.hist[b] = 0;
    if (small_tab)
        for (uint32_t i = tid; i < a.nsegs; i += THREADS) sm.seg_tile_start[i] = a.segs[i].tile_start;
    __syncthreads();

    auto seg_of = [&](uint32_t t) -> uint32_t {
        if (!a.tile_seg) return 0u;
        if (!small_tab) return a.tile_seg[t];
        uint32_t lo = 0, hi = a.nsegs;  // last segment whose tile_start <= t
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sm.seg_tile_start[mid] <= t) lo = mid; else hi = mid;
        }
        return lo;
    };
    // thread 0: start the bulk copy of tile t into buffer b
    auto issue = [&](uint32_t t, int b) {
        const uint32_t seg = seg_of(t);
        if (seg != sm.iss_seg) {  // (tiles come in runs of one segment)
            sm.iss_sd = a.segs[seg];
            sm.iss_seg = seg;
        }
        const SegDesc sd = sm.iss_sd;
        const uint32_t ti = t - sd.tile_start;
        const uint64_t first = sd.in_off + (uint64_t)ti * TILE;
        const uint64_t rem = sd.count - (uint64_t)ti * TILE;
        const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
        const uint32_t bytes = (cnt * ESZ) & ~15u;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&sm.mbar[b], bytes * NARR);
        if (bytes) {
#pragma unroll
            for (int k = 0; k < NARR; ++k)
                bulk_g2s(sm.buf[b] + (size_t)k * TILE * ESZ,
                         static_cast<const unsigned char*>(in.arr(k)) + first * ESZ, bytes, &sm.mbar[b]);
        }
    };

    // thread 0 claims claim_group consecutive tiles at a time, so that a block
    // works through a run of one segment before it loads another's tables
    const uint32_t claim_group = a.nsegs > 1 ? CLAIM_GROUP_MANY_SEGS : CLAIM_GROUP_ONE_SEG;
    uint32_t grp_next = 0, grp_end = 0;
    auto claim = [&]() -> uint32_t {
        if (grp_next == grp_end) {
            grp_next = a.tile_first + atomicAdd(a.tile_counter, claim_group);
            grp_end = grp_next + claim_group;
        }
        return grp_next++;
    };
    uint32_t t_next = 0;  // thread 0: the tile after the current one
    if (tid == 0) {
        const uint32_t t0 = claim();
        sm.tile_cur = t0;
        if (a.tma && t0 < ntiles) issue(t0, 0);
        t_next = claim();
    }
    __syncthreads();
    uint32_t phases = 0;  // bit b: the parity to wait for on buffer b's mbarrier
    int b = 0;

    while (true) {
        // tile_cur is rewritten by thread 0 only after the first barrier of
        // the iteration, and read again after the last one
        const uint32_t t = sm.tile_cur;
        if (t >= ntiles || sm.abort) break;
        const uint32_t seg = seg_of(t);
        const bool new_seg = seg != cached_seg;
        if (new_seg) {
            // the segment's descriptor and tables, read once per run of its
            // tiles (the previous tile's write-out reads none of them)
            if (tid < (int)(sizeof(SegDesc) / 4))
                reinterpret_cast<uint32_t*>(&sm.sd)[tid] = reinterpret_cast<const uint32_t*>(&a.segs[seg])[tid];
            const bool use_learned = a.learned && a.learned[seg].ok;
            if (use_learned) {
                const LearnedSet<K>& ls = a.learned[seg];
                const uint32_t* src = reinterpret_cast<const uint32_t*>(&ls);
                uint32_t* dst = reinterpret_cast<uint32_t*>(sm.T.model);
                for (uint32_t i = tid; i < learned_model_bytes<K>() / 4; i += THREADS) dst[i] = src[i];
                for (int i = tid; i < NB; i += THREADS) {
                    sm.region_off[i] = ls.region_off[i];
                    sm.region_cap[i] = ls.region_cap[i];
                }
            } else {
                const SplitSet<K>& ss = a.splits[seg];
                for (int i = tid; i < NB; i += THREADS) {
                    sm.T.P.uniq[i] = ss.uniq[i];
                    sm.region_off[i] = ss.region_off[i];
                    sm.region_cap[i] = ss.region_cap[i];
                    sm.T.P.range_b[i] = ss.range_b[i];
                    sm.T.P.eq_b[i] = ss.eq_b[i];
                }
                if (tid < NB / 32) sm.T.P.eq_mask[tid] = ss.eq_mask[tid];
                {
                    const uint4* src = reinterpret_cast<const uint4*>(ss.slot_tab);
                    uint4* dst = reinterpret_cast<uint4*>(sm.T.P.tab);
                    for (int i = tid; i < (SPLIT_SLOTS + 8) * 2 / 16; i += THREADS) dst[i] = src[i];
                }
                if (tid == 0) {
                    sm.has_eq = ss.has_eq;
                    sm.T.P.fmap = ss.slot_map;
                    sm.T.P.fhi = ss.slot_hi;
                }
            }
            if (tid == 0) sm.use_learned = use_learned ? 1u : 0u;
            cached_seg = seg;
        }
        bool data_ok = true;
        if (a.tma) {
            // every thread waits on the barrier itself: the bulk copy's data is
            // then visible to it without a block barrier
            data_ok = mbar_wait_bounded(&sm.mbar[b], (phases >> b) & 1u);
            phases ^= 1u << b;
            if (!data_ok) raise_error(&a.ctl->err, DEV_ERR_TIMEOUT);
        }
        if (a.inject_timeout && t == 1) {
            // injected failure: a wait on a flag that nothing sets, with a
            // short bound; the tile then gives up and writes nothing
            uint32_t spins = 0;
            while (!*(volatile uint32_t*)&a.ctl->never_set && ++spins < 1024u) __nanosleep(100);
            data_ok = false;
            raise_error(&a.ctl->err, DEV_ERR_TIMEOUT);
        }
        if (new_seg) __syncthreads();  // the segment's descriptor and tables in shared memory
        // (the descriptor stays in shared memory: registers hold the keys)
        const uint32_t ti = t - sm.sd.tile_start;
        const uint64_t base = sm.sd.in_off + (uint64_t)ti * TILE;
        const uint64_t rem = sm.sd.count - (uint64_t)ti * TILE;
        const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
        const uint32_t tma_elems = a.tma ? ((cnt * ESZ) & ~15u) / ESZ : 0u;
        const bool has_eq = sm.has_eq != 0;
        const bool learned = sm.use_learned != 0;
        const SlotRegs<K> fm(sm.T.P.fmap, sm.T.P.fhi);  // (meaningless for a learned segment: unused)

        // a whole tile from the bulk copy (no per-key range checks)
        const bool FULL = cnt == (uint32_t)TILE && tma_elems == (uint32_t)TILE;
        {
            // A. keys (striped: element r*THREADS + tid, from the bulk-copied
            // tile; tail elements past the copied bytes from global memory),
            // their buckets and their ranks within the tile
            K key[IPT];
            uint32_t br[IPT];  // bucket | rank << 8
#pragma unroll
            for (int r = 0; r < IPT; ++r) {
                const uint32_t idx = (uint32_t)(r * THREADS + tid);
                if (FULL) key[r] = in.decode(sm.buf[b], idx, TILE);
                else if (idx < cnt) key[r] = idx < tma_elems ? in.decode(sm.buf[b], idx, TILE) : in.load(base + idx);
            }
            // all IPT bucket lookups first: they are independent chains of
            // shared loads, so the scheduler can overlap them
            uint32_t bks[IPT];
            if (learned) {
#pragma unroll
                for (int r = 0; r < IPT; ++r) {
                    const uint32_t idx = (uint32_t)(r * THREADS + tid);
                    // (only the model prefix of the LearnedSet is in shared memory)
                    bks[r] = (FULL || idx < cnt)
                                 ? learned_bucket<K>(*reinterpret_cast<const LearnedSet<K>*>(sm.T.model), key[r])
                                 : (uint32_t)NB;  // lanes past the end carry the out-of-range bucket NB
                }
            } else {
#pragma unroll
                for (int r = 0; r < IPT; ++r) bks[r] = sm.T.P.tab[fm(key[r])];  // slot entries first
#pragma unroll
                for (int r = 0; r < IPT; ++r) {
                    const uint32_t idx = (uint32_t)(r * THREADS + tid);
                    bks[r] = (FULL || idx < cnt) ? bucket_from_slot<K>(bks[r], key[r], has_eq, sm.T.P.uniq,
                                                                       sm.T.P.range_b, sm.T.P.eq_b, sm.T.P.eq_mask)
                                                 : (uint32_t)NB;
                }
            }
            // A warp whose 32 keys share a bucket (sorted or constant runs)
            // ranks them with one atomic instead of 32 on one address.  Whether
            // to look for that is decided once per tile from the warp's first
            // 32 keys: on unsorted input the check would cost a shuffle and a
            // vote per key and never pay.
            const bool try_uni = __all_sync(0xFFFFFFFFu, bks[0] == __shfl_sync(0xFFFFFFFFu, bks[0], 0));
#pragma unroll
            for (int r = 0; r < IPT; ++r) {
                const uint32_t bk = bks[r];
                uint32_t b0 = bk;
                bool uni = false;
                if (try_uni) {
                    b0 = __shfl_sync(0xFFFFFFFFu, bk, 0);
                    uni = __all_sync(0xFFFFFFFFu, bk == b0);
                }
                uint32_t rank = 0;
                if (uni) {
                    if (FULL || b0 < (uint32_t)NB) {
                        uint32_t basev = 0;
                        if (lane_id() == 0) basev = atomicAdd(&sm.hist[b0], 32u);
                        rank = __shfl_sync(0xFFFFFFFFu, basev, 0) + lane_id();
                    }
                } else if (FULL || bk < (uint32_t)NB) {
                    rank = atomicAdd(&sm.hist[bk], 1u);
                }
                br[r] = bk | (rank << 8);
            }
            __syncthreads();  // (1) the tile's histogram is complete; the previous tile is written

            // B. reserve the tile's share of each bucket's region, and the
            // buckets' starts within the tile (exclusive scan by warp 0)
            uint32_t h = 0;
            unsigned long long off = 0;
            if (tid < NB) {
                h = sm.hist[tid];
                if (h) off = atomicAdd(&a.fill[(size_t)seg * NB + tid], (unsigned long long)h);
            }
            if (tid < 32) {
                uint32_t v[NB / 32];
                uint32_t run = 0;
#pragma unroll
                for (int i = 0; i < NB / 32; ++i) {
                    v[i] = run;
                    run += sm.hist[tid * (NB / 32) + i];
                }
                uint32_t inc = run;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
                    if (tid >= d) inc += o;
                }
                const uint32_t ex = inc - run;
#pragma unroll
                for (int i = 0; i < NB / 32; ++i) sm.loc[tid * (NB / 32) + i] = ex + v[i];
            }
            if (tid == 0) {
                // the next tile's keys into the other buffer: its last reader,
                // the previous tile's write-out, finished before barrier (1)
                if (a.tma && t_next < ntiles) issue(t_next, b ^ 1);
                sm.tile_cur = t_next;
                t_next = claim();
            }
            __syncthreads();  // (2) bucket starts within the tile

            // C. stage the keys in bucket order, reusing this tile's buffer
            K* stage = reinterpret_cast<K*>(sm.buf[b]);
#pragma unroll
            for (int r = 0; r < IPT; ++r) {
                const uint32_t idx = (uint32_t)(r * THREADS + tid);
                if (FULL || idx < cnt) {
                    const uint32_t bk = br[r] & 0xFFu;
                    const uint32_t p = sm.loc[bk] + (br[r] >> 8);
                    stage[p] = key[r];
                    sm.bkt[p] = (uint8_t)bk;
                }
            }
            if (tid < NB) {
                const unsigned long long end = off + h;
                const bool ovf = !data_ok || end > sm.region_cap[tid];
                if (ovf && h) raise_error(&a.ctl->err, data_ok ? DEV_ERR_OVERFLOW : DEV_ERR_TIMEOUT);
                sm.gdelta[tid] =
                    (ovf ? a.junk : sm.sd.out_base + sm.region_off[tid] + off) - (uint64_t)sm.loc[tid];
                sm.hist[tid] = 0;  // (next used after barrier (3))
            }
            if (tid == 0 && !data_ok) sm.abort = 1;
            __syncthreads();  // (3) staging complete

            // D. coalesced write-out (an overflowed bucket's keys go to the
            // overflow area past the regions: the level is redone)
#pragma unroll
            for (int r = 0; r < IPT; ++r) {
                const uint32_t i = (uint32_t)(r * THREADS + tid);
                if (FULL || i < cnt) {
                    const uint64_t g = sm.gdelta[sm.bkt[i]];
                    a.out[g + i] = stage[i];
                }
            }
        }
        b ^= 1;
    }
    // after an abort, let a copy still in flight land before the block exits
    if (a.tma && sm.abort && tid == 0 && sm.tile_cur < ntiles) mbar_wait_bounded(&sm.mbar[b], (phases >> b) & 1u);
}

// Testing: shrink every bucket capacity of segment 0 (forces an overflow).
template <typename K>
__global__ void inject_overflow_kernel(SplitSet<K>* splits, LearnedSet<K>* learned) {
    const int b = threadIdx.x;
    if (b < NB) {
        if (splits[0].region_cap[b] > 16) splits[0].region_cap[b] = 16;
        if (learned && learned[0].region_cap[b] > 16) learned[0].region_cap[b] = 16;
    }
}

// Testing: reject every learned model of the level.
template <typename K>
__global__ void inject_reject_kernel(LearnedSet<K>* learned, uint32_t nsegs) {
    for (uint32_t s = threadIdx.x; s < nsegs; s += blockDim.x) learned[s].ok = 0;
}

// Exact histogram of a level (the fallback after a capacity overflow).
template <typename K, typename InCodec, int THREADS, int IPT>
__global__ void __launch_bounds__(THREADS) count_kernel(PartArgs<K> a, InCodec in) {
    __shared__ K tree[NB];
    __shared__ K uniq[NB];
    __shared__ uint8_t range_b[NB], eq_b[NB];
    __shared__ uint32_t eq_mask[NB / 32];
    __shared__ uint32_t hist[NB];
    __shared__ uint32_t has_eq;
    constexpr int TILE = THREADS * IPT;
    const uint32_t ntiles = a.ntiles_dev ? *a.ntiles_dev : a.ntiles;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t seg = a.tile_seg ? a.tile_seg[t] : 0u;
        const SegDesc sd = a.segs[seg];
        const SplitSet<K>& ss = a.splits[seg];
        for (int b = threadIdx.x; b < NB; b += THREADS) {
            tree[b] = ss.tree[b];
            uniq[b] = ss.uniq[b];
            range_b[b] = ss.range_b[b];
            eq_b[b] = ss.eq_b[b];
            hist[b] = 0;
        }
        if (threadIdx.x < NB / 32) eq_mask[threadIdx.x] = ss.eq_mask[threadIdx.x];
        if (threadIdx.x == 0) has_eq = ss.has_eq;
        __syncthreads();
        const uint32_t ti = t - sd.tile_start;
        const uint64_t base = sd.in_off + (uint64_t)ti * TILE;
        const uint64_t rem = sd.count - (uint64_t)ti * TILE;
        const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
        for (uint32_t i = threadIdx.x; i < cnt; i += THREADS) {
            const K x = in.load(base + i);
            atomicAdd(&hist[find_bucket<K>(tree, x, has_eq != 0, uniq, range_b, eq_b, eq_mask)], 1u);
        }
        __syncthreads();
        for (int b = threadIdx.x; b < NB; b += THREADS)
            if (hist[b]) atomicAdd(&a.fill[(size_t)seg * NB + b], (unsigned long long)hist[b]);
        __syncthreads();
    }
}

// Re-lay the bucket regions of every segment from exact counts.
template <typename K>
__global__ void __launch_bounds__(NB) exact_regions_kernel(SplitSet<K>* splits, const uint64_t* bucket_counts,
                                                           uint32_t nsegs) {
    __shared__ uint64_t wtot64[8];
    const uint32_t s = blockIdx.x;
    if (s >= nsegs) return;
    const uint64_t c = bucket_counts[(size_t)s * NB + threadIdx.x];
    const uint64_t cap = (c + 15) & ~15ull;
    const uint64_t off = block_exclusive_scan_first<NB, uint64_t>(cap, wtot64, (uint64_t*)nullptr);
    splits[s].region_off[threadIdx.x] = off;
    splits[s].region_cap[threadIdx.x] = cap;
}

// ===========================================================================
// 5. Planning: classify each bucket of each segment (one block per segment)

template <typename K>
struct PlanArgs {
    const SegDesc* segs;
    const SplitSet<K>* splits;
    const LearnedSet<K>* learned;       // used for segments whose model was accepted
    const uint64_t* bucket_counts;
    const K* level_out;                 // the level's output buffer
    LeafItem<K>* items[NCLASS + 1];     // per class, plus the copy list
    uint32_t item_cap;
    SegDesc* next;                      // next-level segments (in_off into level_out)
    uint32_t next_cap;
    LevelCtl* ctl;
    int key_bytes;
};

template <typename K>
__global__ void __launch_bounds__(NB) plan_kernel(PlanArgs<K> a, uint32_t nsegs) {
    __shared__ uint64_t wtot64[8];
    const uint32_t s = blockIdx.x;
    if (s >= nsegs) return;
    const SegDesc sd = a.segs[s];
    const bool use_learned = a.learned && a.learned[s].ok;
    const uint32_t nbk = use_learned ? a.learned[s].nbuckets : a.splits[s].nbuckets;
    const uint64_t* region_off = use_learned ? a.learned[s].region_off : a.splits[s].region_off;
    const uint32_t* bucket_eq = use_learned ? a.learned[s].bucket_eq : a.splits[s].bucket_eq;
    const int b = threadIdx.x;
    if (b == 0) {
        atomicAdd(use_learned ? &a.ctl->learned_used : &a.ctl->plain_used, 1u);
        if (a.learned && a.learned[s].fitted) {
            atomicAdd(&a.ctl->learned_fitted, 1u);
            atomicMax(&a.ctl->model_imb_bits, __float_as_uint(a.learned[s].max_over_mean));  // (>= 0)
        }
    }
    const uint64_t c = (b < (int)nbk) ? a.bucket_counts[(size_t)s * NB + b] : 0ull;
    const uint64_t excl = block_exclusive_scan_first<NB, uint64_t>(c, wtot64, (uint64_t*)nullptr);
    // what the bucket becomes: a copy (equality bucket or single key, in
    // chunks), a leaf of some class, or a segment of the next level
    constexpr int LIST_NEXT = NCLASS + 1;  // lists 0..NCLASS-1 leaves, NCLASS copies, NCLASS+1 next level
    __shared__ uint32_t list_n[NCLASS + 2], list_base[NCLASS + 2];
    __shared__ uint32_t st_max, st_nonempty;
    __shared__ unsigned long long st_keys, st_next_keys;
    __shared__ double st_sq;
    if (b < NCLASS + 2) list_n[b] = 0;
    if (b == 0) {
        st_max = 0;
        st_nonempty = 0;
        st_keys = 0;
        st_next_keys = 0;
        st_sq = 0.0;
    }
    __syncthreads();
    const bool is_eq = (bucket_eq[b >> 5] >> (b & 31)) & 1u;
    int list = -1;
    uint32_t nslots = 0;
    if (c > 0) {
        if (is_eq || c == 1) {
            list = CLS_COPY;
            nslots = (uint32_t)((c + COPY_CHUNK - 1) / COPY_CHUNK);
        } else if (c <= leaf_max(a.key_bytes)) {
            list = class_of(a.key_bytes, (uint32_t)c);
            nslots = 1;
        } else {
            list = LIST_NEXT;
            nslots = 1;
        }
    }
    // the level's statistics and the list slots, gathered in the block: one
    // global atomic per block and counter instead of one per bucket
    const uint32_t local = list >= 0 ? atomicAdd(&list_n[list], nslots) : 0u;
    {
        uint32_t mx = (uint32_t)(c > 0xFFFFFFFFull ? 0xFFFFFFFFull : c), ne = c > 0 ? 1u : 0u;
        unsigned long long keys = c, nk = list == LIST_NEXT ? c : 0ull;
        double sq = (double)c * (double)c;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, d));
            ne += __shfl_xor_sync(0xFFFFFFFFu, ne, d);
            keys += __shfl_xor_sync(0xFFFFFFFFu, keys, d);
            nk += __shfl_xor_sync(0xFFFFFFFFu, nk, d);
            sq += __shfl_xor_sync(0xFFFFFFFFu, sq, d);
        }
        if ((b & 31) == 0 && ne) {
            atomicMax(&st_max, mx);
            atomicAdd(&st_nonempty, ne);
            atomicAdd(&st_keys, keys);
            atomicAdd(&st_next_keys, nk);
            atomicAdd(&st_sq, sq);
        }
    }
    __syncthreads();
    if (b < NCLASS + 2 && list_n[b]) {
        unsigned int* ctr = b == LIST_NEXT ? &a.ctl->n_next : &a.ctl->n_items[b];
        list_base[b] = atomicAdd(ctr, list_n[b]);
    }
    if (b == 0 && st_nonempty) {
        atomicMax(&a.ctl->max_bucket, st_max);
        atomicAdd(&a.ctl->nonempty, st_nonempty);
        atomicAdd((unsigned long long*)&a.ctl->level_keys, st_keys);
        atomicAdd(&a.ctl->bucket_sq, st_sq);
        if (st_next_keys) atomicAdd((unsigned long long*)&a.ctl->next_keys, st_next_keys);
    }
    __syncthreads();
    if (list < 0) return;
    const K* src = a.level_out + sd.out_base + region_off[b];
    const uint64_t dst = sd.final_off + excl;
    const uint32_t first = list_base[list] + local;
    if (list == CLS_COPY) {
        uint32_t slot = first;
        for (uint64_t o = 0; o < c; o += COPY_CHUNK, ++slot) {
            if (slot < a.item_cap) {
                LeafItem<K> it;
                it.src = src + o;
                it.dst = dst + o;
                it.count = (uint32_t)((c - o) < COPY_CHUNK ? (c - o) : COPY_CHUNK);
                it.pad_ = 0;
                a.items[CLS_COPY][slot] = it;
            } else {
                raise_error(&a.ctl->err, DEV_ERR_CAPACITY);
            }
        }
    } else if (list < NCLASS) {
        if (first < a.item_cap) {
            LeafItem<K> it;
            it.src = src;
            it.dst = dst;
            it.count = (uint32_t)c;
            it.pad_ = 0;
            a.items[list][first] = it;
        } else {
            raise_error(&a.ctl->err, DEV_ERR_CAPACITY);
        }
    } else {
        if (first < a.next_cap) {
            SegDesc n;
            n.in_off = sd.out_base + region_off[b];
            n.count = c;
            n.final_off = dst;
            n.out_base = 0;
            n.tile_start = 0;
            n.ntiles = 0;
            a.next[first] = n;
        } else {
            raise_error(&a.ctl->err, DEV_ERR_CAPACITY);
        }
    }
}

// Give the next level's segments their tiles and output regions (one block).
static __global__ void __launch_bounds__(1024) prepare_level_kernel(SegDesc* segs, uint32_t nsegs, uint32_t tile,
                                                             LevelCtl* ctl_next) {
    __shared__ uint64_t wt1[32], wt2[32];
    __shared__ uint64_t tot1, tot2;
    __shared__ uint64_t carry_tiles, carry_bound;
    if (threadIdx.x == 0) {
        carry_tiles = 0;
        carry_bound = 0;
    }
    __syncthreads();
    for (uint32_t base = 0; base < nsegs; base += 1024) {
        const uint32_t s = base + threadIdx.x;
        uint64_t nt = 0, bd = 0;
        if (s < nsegs) {
            nt = (segs[s].count + tile - 1) / tile;
            bd = (region_bound(segs[s].count) + 15) & ~15ull;
        }
        const uint64_t ex_t = block_exclusive_scan_first<1024, uint64_t>(nt, wt1, &tot1);
        const uint64_t ex_b = block_exclusive_scan_first<1024, uint64_t>(bd, wt2, &tot2);
        if (s < nsegs) {
            segs[s].tile_start = (uint32_t)(carry_tiles + ex_t);
            segs[s].ntiles = (uint32_t)nt;
            segs[s].out_base = carry_bound + ex_b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry_tiles += tot1;
            carry_bound += tot2;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctl_next->ntiles_next = (uint32_t)carry_tiles;
        ctl_next->bound_next = carry_bound;
    }
}

// tile -> segment map (one block per segment)
static __global__ void tile_map_kernel(const SegDesc* segs, uint32_t nsegs, uint32_t* tile_seg) {
    const uint32_t s = blockIdx.x;
    if (s >= nsegs) return;
    const SegDesc sd = segs[s];
    for (uint32_t i = threadIdx.x; i < sd.ntiles; i += blockDim.x) tile_seg[sd.tile_start + i] = s;
}

// ===========================================================================
// 6. Leaves

// One warp per bucket of at most 32*IPT keys (class 0).
template <typename K, typename OutCodec, int IPT>
__global__ void __launch_bounds__(256) leaf_warp_kernel(const LeafItem<K>* __restrict__ items, uint32_t nitems,
                                                        OutCodec out) {
    __shared__ K stage[8][32 * IPT];
    const unsigned warp = threadIdx.x >> 5, lane = lane_id();
    K* sw = stage[warp];
    for (uint32_t it = blockIdx.x * 8 + warp; it < nitems; it += gridDim.x * 8) {
        const LeafItem<K> item = items[it];
        for (uint32_t i = lane; i < 32 * IPT; i += 32) sw[i] = i < item.count ? item.src[i] : KeyMax<K>::value;
        __syncwarp();
        K x[IPT];
#pragma unroll
        for (int r = 0; r < IPT; ++r) x[r] = sw[lane * IPT + r];
        __syncwarp();
        warp_bitonic_sort<K, IPT>(x);
#pragma unroll
        for (int r = 0; r < IPT; ++r) sw[lane * IPT + r] = x[r];
        __syncwarp();
        for (uint32_t i = lane; i < item.count; i += 32) out.store(item.dst + i, sw[i]);
        __syncwarp();
    }
}

// Blocks per SM that the leaf kernel's register budget is sized for (the
// 384-thread class fits three, with its keys' shared memory unpadded).
__host__ __device__ constexpr int leaf_min_blocks(int threads) {
    return (threads == 288 || threads == 320 || threads == 384) ? 3 : 1024 / threads;
}

// One block per bucket of at most THREADS*EPT keys: distribution counting
// into value slots (s512_slotsort.cuh).  The next bucket's keys are loaded
// into registers while the current one is ranked and written.  A bucket whose
// slots come out uneven is appended to `uneven` (count in *n_uneven) for
// leaf_merge_kernel.
template <typename K, typename OutCodec, int THREADS, int EPT>
__global__ void __launch_bounds__(THREADS, leaf_min_blocks(THREADS))
    leaf_block_kernel(const LeafItem<K>* __restrict__ items, uint32_t nitems, OutCodec out, LeafItem<K>* uneven,
                      uint32_t* n_uneven) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ SlotRed<K> red;
    uint32_t it = blockIdx.x;
    if (it >= nitems) return;
    LeafItem<K> cur = items[it];
    K key[EPT];
    auto load = [&](const LeafItem<K>& item) {
#pragma unroll
        for (int r = 0; r < EPT; ++r) {
            const uint32_t i = (uint32_t)r * THREADS + threadIdx.x;
            if (i < item.count) key[r] = __ldg(item.src + i);
        }
    };
    load(cur);
    for (; it < nitems; it += gridDim.x) {
        const uint32_t nx = it + gridDim.x;
        LeafItem<K> next;
        next.count = 0;
        if (nx < nitems) next = items[nx];
        const size_t dst = cur.dst;
        block_slot_sort<K, THREADS, EPT, false>(
            key, cur.count, [&](uint32_t i, K x) { out.store(dst + i, x); }, [&]() { load(next); },
            [&]() { uneven[atomicAdd(n_uneven, 1u)] = cur; }, smem_raw, red);
        cur = next;
    }
}

// The buckets leaf_block_kernel found uneven: bitonic leaves + merge path.
template <typename K, typename OutCodec, int THREADS, int EPT>
__global__ void __launch_bounds__(THREADS) leaf_merge_kernel(const LeafItem<K>* __restrict__ items,
                                                             const uint32_t* n_items, OutCodec out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* s = reinterpret_cast<K*>(smem_raw);
    const uint32_t nitems = *n_items;
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const LeafItem<K> item = items[it];
        for (uint32_t i = threadIdx.x; i < item.count; i += THREADS) s[pidx(i)] = item.src[i];
        block_merge_sort<K, THREADS, EPT>(s, item.count);
        for (uint32_t i = threadIdx.x; i < item.count; i += THREADS) out.store(item.dst + i, s[pidx(i)]);
        __syncthreads();
    }
}

// Copy equality buckets (and single keys) to their final place.
template <typename K, typename OutCodec>
__global__ void __launch_bounds__(256) leaf_copy_kernel(const LeafItem<K>* __restrict__ items, uint32_t nitems,
                                                        OutCodec out) {
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const LeafItem<K> item = items[it];
        for (uint32_t i = threadIdx.x; i < item.count; i += 256) out.store(item.dst + i, item.src[i]);
    }
}

// ===========================================================================
// 7. Whole arrays that fit one leaf: sort straight from and to the caller's layout.

template <typename InCodec, typename OutCodec, int IPT>
__global__ void __launch_bounds__(32) small_warp_sort_kernel(InCodec in, OutCodec out, uint32_t n) {
    using K = typename InCodec::Key;
    __shared__ K sw[32 * IPT];
    const unsigned lane = lane_id();
    for (uint32_t i = lane; i < 32 * IPT; i += 32) sw[i] = i < n ? in.load(i) : KeyMax<K>::value;
    __syncwarp();
    K x[IPT];
#pragma unroll
    for (int r = 0; r < IPT; ++r) x[r] = sw[lane * IPT + r];
    __syncwarp();
    warp_bitonic_sort<K, IPT>(x);
#pragma unroll
    for (int r = 0; r < IPT; ++r) sw[lane * IPT + r] = x[r];
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) out.store(i, sw[i]);
}

template <typename InCodec, typename OutCodec, int THREADS, int EPT>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) small_block_sort_kernel(InCodec in, OutCodec out,
                                                                                   uint32_t n) {
    using K = typename InCodec::Key;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ SlotRed<K> red;
    K key[EPT];
#pragma unroll
    for (int r = 0; r < EPT; ++r) {
        const uint32_t i = (uint32_t)r * THREADS + threadIdx.x;
        if (i < n) key[r] = in.load(i);
    }
    block_slot_sort<K, THREADS, EPT, true>(
        key, n, [&](uint32_t i, K x) { out.store(i, x); }, [] {}, [] {}, smem_raw, red);
}
}  // namespace s512
