// s512_pipeline.cuh -- host driver of the partition-then-sort pipeline
// (included by the translation units that sort: s512_sort.cu, s512_segsort.cu).
#pragma once

#include "s512_runtime.cuh"
#include "s512_sortpipe.cuh"

namespace s512 {

// Tile shapes of the partition kernel per key size: levels with many segments
// (PartShape), and a level that is one whole array (PartShapeOne).  512
// threads and 24-32 KB of keys per tile: two blocks (2 x ~90 KB of shared
// memory) share an SM.
template <typename K> struct PartShape;
template <> struct PartShape<uint32_t> { static constexpr int THREADS = 512, IPT = 12; };
template <> struct PartShape<uint64_t> { static constexpr int THREADS = 512, IPT = 8; };
template <typename K> struct PartShapeOne;
template <> struct PartShapeOne<uint32_t> { static constexpr int THREADS = 512, IPT = 12; };
template <> struct PartShapeOne<uint64_t> { static constexpr int THREADS = 512, IPT = 8; };

// ---------------------------------------------------------------------------
// leaf launches per class

// Slot sort of a class's buckets, then the block sort of those it found
// uneven (the second launch reads the count on the device and exits at once
// when there are none).
template <typename K, typename OutCodec, int THREADS, int EPT>
static int launch_leaf_block(DevCtx& C, const LeafItem<K>* items, uint32_t n, OutCodec out, LeafItem<K>* uneven,
                             uint32_t* n_uneven, cudaStream_t st) {
    {
        auto fn = leaf_block_kernel<K, OutCodec, THREADS, EPT>;
        const size_t smem = SlotSmem<K, THREADS, EPT, false>::bytes;
        int grid = 0;
        S512_CUDA_TRY(launch_persistent(C, fn, THREADS, smem, st, (int)n, &grid));
        fn<<<grid, THREADS, smem, st>>>(items, n, out, uneven, n_uneven);
        S512_LAUNCH_CHECK();
    }
    {
        auto fn = leaf_merge_kernel<K, OutCodec, THREADS, EPT>;
        const size_t smem = (size_t)padded_len(THREADS * EPT) * sizeof(K);
        int grid = 0;
        S512_CUDA_TRY(launch_persistent(C, fn, THREADS, smem, st, (int)n, &grid));
        fn<<<grid, THREADS, smem, st>>>(uneven, n_uneven, out);
        S512_LAUNCH_CHECK();
    }
    return S512_OK;
}

// Launch the leaf kernels of one class.  `uneven` has room for n items.
template <typename K, typename OutCodec>
static int launch_leaf_class(DevCtx& C, int cls, const LeafItem<K>* items, uint32_t n, OutCodec out,
                             LeafItem<K>* uneven, uint32_t* n_uneven, cudaStream_t st) {
    if (n == 0) return S512_OK;
    switch (cls) {
        case 0: {
            auto fn = leaf_warp_kernel<K, OutCodec, 8>;
            int grid = 0;
            S512_CUDA_TRY(launch_persistent(C, fn, 256, 0, st, (int)((n + 7) / 8), &grid));
            fn<<<grid, 256, 0, st>>>(items, n, out);
            S512_LAUNCH_CHECK();
            return S512_OK;
        }
        case 1: return launch_leaf_block<K, OutCodec, 128, 8>(C, items, n, out, uneven, n_uneven, st);
        case 2: return launch_leaf_block<K, OutCodec, 256, 8>(C, items, n, out, uneven, n_uneven, st);
        case 3: return launch_leaf_block<K, OutCodec, 256, 16>(C, items, n, out, uneven, n_uneven, st);
        case 4: return launch_leaf_block<K, OutCodec, 288, 16>(C, items, n, out, uneven, n_uneven, st);
        case 5: return launch_leaf_block<K, OutCodec, 320, 16>(C, items, n, out, uneven, n_uneven, st);
        case 6: return launch_leaf_block<K, OutCodec, 384, 16>(C, items, n, out, uneven, n_uneven, st);
        case 7: return launch_leaf_block<K, OutCodec, 512, 16>(C, items, n, out, uneven, n_uneven, st);
        case 8: return launch_leaf_block<K, OutCodec, 1024, 16>(C, items, n, out, uneven, n_uneven, st);
        case CLS_COPY: {
            auto fn = leaf_copy_kernel<K, OutCodec>;
            int grid = 0;
            S512_CUDA_TRY(launch_persistent(C, fn, 256, 0, st, (int)n, &grid));
            fn<<<grid, 256, 0, st>>>(items, n, out);
            S512_LAUNCH_CHECK();
            return S512_OK;
        }
    }
    set_error("bad leaf class %d", cls);
    return S512_ERR_INTERNAL;
}

// Whole array in one leaf (n <= leaf_max).
template <typename InCodec, typename OutCodec, int THREADS, int EPT>
static int launch_small_block(DevCtx& C, InCodec in, OutCodec out, uint32_t n, cudaStream_t st) {
    using K = typename InCodec::Key;
    auto fn = small_block_sort_kernel<InCodec, OutCodec, THREADS, EPT>;
    const size_t smem = SlotSmem<K, THREADS, EPT>::bytes;
    S512_CUDA_TRY(C.prepare((const void*)fn, smem));
    fn<<<1, THREADS, smem, st>>>(in, out, n);
    S512_LAUNCH_CHECK();
    return S512_OK;
}

template <typename InCodec, typename OutCodec>
static int sort_one_leaf(DevCtx& C, InCodec in, OutCodec out, uint32_t n, cudaStream_t st) {
    using K = typename InCodec::Key;
    if (n <= 256) {
        small_warp_sort_kernel<InCodec, OutCodec, 8><<<1, 32, 0, st>>>(in, out, n);
        S512_LAUNCH_CHECK();
        return S512_OK;
    }
    switch (class_of(sizeof(K), n)) {
        case 1: return launch_small_block<InCodec, OutCodec, 128, 8>(C, in, out, n, st);
        case 2: return launch_small_block<InCodec, OutCodec, 256, 8>(C, in, out, n, st);
        case 3: return launch_small_block<InCodec, OutCodec, 512, 8>(C, in, out, n, st);
        case 4:
        case 5:
        case 6:
        case 7: return launch_small_block<InCodec, OutCodec, 512, 16>(C, in, out, n, st);
        default: return launch_small_block<InCodec, OutCodec, 1024, 16>(C, in, out, n, st);
    }
}

// The partition kernel fetches tiles by bulk copy when every input array is
// 16-byte aligned (segment and tile offsets keep that alignment).
template <typename C>
static bool codec_aligned(const C& c) {
    for (int k = 0; k < C::NARR; ++k)
        if (reinterpret_cast<uintptr_t>(c.arr(k)) & 15u) return false;
    return true;
}

// ---------------------------------------------------------------------------
// The first partition level of a host-pointer sort, fed while the caller's
// page-locked arrays are still being copied in: the sample is read from the
// host arrays themselves (through their device addresses), and the
// partition kernel runs once per chunk, each launch waiting for its chunk's
// copy.  Chunks are whole tiles of that level.
struct HostFeed {
    const void* mapped[2];      // device addresses of the caller's host arrays
    uint32_t nchunks;
    uint64_t chunk_keys;        // keys per chunk (a multiple of the level's tile)
    const cudaEvent_t* ready;   // ready[c]: chunk c is on the device
};

// The stream waits for every chunk (a sort that does not consume the feed).
static inline int wait_feed(const HostFeed* feed, cudaStream_t st) {
    if (!feed) return S512_OK;
    for (uint32_t c = 0; c < feed->nchunks; ++c) S512_CUDA_TRY(cudaStreamWaitEvent(st, feed->ready[c], 0));
    return S512_OK;
}

// ---------------------------------------------------------------------------
// One partition level: sample -> sort sample -> splitters -> partition -> plan.
template <typename K, typename InCodec>
struct Level {
    InCodec in;
    SegDesc* segs;
    uint32_t nsegs;
    const uint32_t* tile_seg;   // null for a single segment
    uint32_t ntiles_host;       // level 0
    const uint32_t* ntiles_dev; // levels >= 1
    uint32_t ntiles_bound;
    K* out;
    uint64_t junk;              // offset in out of JUNK_KEYS keys past every region (overflow writes)
    bool aligned;               // every tile starts 16-byte aligned (bulk copies allowed)
};

template <typename K, typename InCodec, typename UserOut, typename Shape = PartShape<K>>
static int run_level(DevCtx& C, Level<K, InCodec>& L, int level, UserOut uout, size_t n, cudaStream_t st,
                     LevelCtl* ctl, LevelCtl* next_ctl_dev, SegDesc* next_segs, uint32_t next_cap,
                     PhaseTimer& tm, s512_stats& S, LevelCtl* host_ctl, bool learned,
                     const HostFeed* feed = nullptr) {
    constexpr int KB = sizeof(K);
    const uint32_t nsegs = L.nsegs;
    int rc;

    // scratch for this level
    K* samples = (K*)C.get("samples", (size_t)nsegs * SAMPLE_N * KB);
    SplitSet<K>* splits = (SplitSet<K>*)C.get("splits", (size_t)nsegs * sizeof(SplitSet<K>));
    uint64_t* counts = (uint64_t*)C.get("counts", (size_t)nsegs * NB * sizeof(uint64_t));
    const uint32_t item_cap = nsegs * NB + (uint32_t)(n / COPY_CHUNK) + 16;
    LeafItem<K>* items[NCLASS + 1];
    {
        char* base = (char*)C.get("items", (size_t)(NCLASS + 1) * item_cap * sizeof(LeafItem<K>));
        if (!base) return S512_ERR_ALLOC;
        for (int c = 0; c <= NCLASS; ++c) items[c] = (LeafItem<K>*)(base + (size_t)c * item_cap * sizeof(LeafItem<K>));
    }
    LearnedSet<K>* lsets = learned ? (LearnedSet<K>*)C.get("lsets", (size_t)nsegs * sizeof(LearnedSet<K>)) : nullptr;
    if (!samples || !splits || !counts || (learned && !lsets)) return S512_ERR_ALLOC;

    const int t0 = tm.mark();
    S512_CUDA_TRY(cudaMemsetAsync(ctl, 0, sizeof(LevelCtl), st));
    S512_CUDA_TRY(cudaMemsetAsync(counts, 0, (size_t)nsegs * NB * sizeof(uint64_t), st));
    const uint64_t seed = config().seed + 0x9E3779B97F4A7C15ull * (uint64_t)(level + 1);
    if (feed)  // the caller's host arrays, read where they are
        sample_kernel<InCodec><<<nsegs, 256, 0, st>>>(L.in.rebased(feed->mapped), L.segs, nsegs, samples, seed, KB);
    else
        sample_kernel<InCodec><<<nsegs, 256, 0, st>>>(L.in, L.segs, nsegs, samples, seed, KB);
    S512_LAUNCH_CHECK();
    {
        auto fn = sample_sort_kernel<K>;
        const size_t smem = SlotSmem<K, 1024, SAMPLE_N / 1024>::bytes;
        S512_CUDA_TRY(C.prepare((const void*)fn, smem));
        fn<<<nsegs, 1024, smem, st>>>(samples, L.segs, nsegs, KB);
        S512_LAUNCH_CHECK();
    }
    splitter_kernel<K><<<nsegs, NB, 0, st>>>(samples, L.segs, nsegs, splits, KB);
    S512_LAUNCH_CHECK();
    S.kernel_launches += 3;
    int tfit0 = -1;
    if (learned) {
        // the model is fitted to the same sorted sample; the split set above
        // stays as its fallback and supplies the heavy keys
        uint32_t* lfirst = (uint32_t*)C.get("lr_first", (size_t)nsegs * (LR_LEAVES + 1) * sizeof(uint32_t));
        if (!lfirst) return S512_ERR_ALLOC;
        tfit0 = tm.mark();
        launch_learned_fit<K>(samples, L.segs, nsegs, splits, lsets, lfirst, KB, (float)config().max_imbalance, st);
        S512_LAUNCH_CHECK();
        S.kernel_launches += 3;
        if (config().fault_inject & S512_FAULT_REJECT_MODEL) {
            inject_reject_kernel<K><<<1, 256, 0, st>>>(lsets, nsegs);
            S512_LAUNCH_CHECK();
        }
    }
    const int fault = level == 0 ? config().fault_inject : 0;
    if (fault & S512_FAULT_OVERFLOW) {
        inject_overflow_kernel<K><<<1, NB, 0, st>>>(splits, lsets);
        S512_LAUNCH_CHECK();
    }
    const int t1 = tm.mark();

    PartArgs<K> pa;
    pa.segs = L.segs;
    pa.tile_seg = L.tile_seg;
    pa.splits = splits;
    pa.out = L.out;
    pa.junk = L.junk;
    pa.fill = (unsigned long long*)counts;
    pa.ctl = ctl;
    pa.ntiles = L.ntiles_host;
    pa.ntiles_dev = L.ntiles_dev;
    pa.tile_first = 0;
    pa.tile_counter = &ctl->tile_counter;
    pa.nsegs = nsegs;
    pa.tma = (L.aligned && codec_aligned(L.in)) ? 1 : 0;
    pa.learned = lsets;
    pa.inject_timeout = (fault & S512_FAULT_TIMEOUT) ? 1 : 0;
    auto pfn = partition_kernel<K, InCodec, Shape::THREADS, Shape::IPT>;
    const size_t psmem = sizeof(PartSmem<K, Shape::THREADS, Shape::IPT>);
    int pgrid = 0;
    S512_CUDA_TRY(launch_persistent(C, pfn, Shape::THREADS, psmem, st, 0, &pgrid));
    if (feed) {
        // one launch per chunk of the input, each after its chunk's copy
        constexpr uint32_t TILE = Shape::THREADS * Shape::IPT;
        uint32_t* cctr = (uint32_t*)C.get("chunk_ctr", (size_t)feed->nchunks * sizeof(uint32_t));
        if (!cctr) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemsetAsync(cctr, 0, (size_t)feed->nchunks * sizeof(uint32_t), st));
        const uint32_t tpc = (uint32_t)(feed->chunk_keys / TILE);
        for (uint32_t c = 0; c < feed->nchunks; ++c) {
            PartArgs<K> pc = pa;
            pc.tile_first = c * tpc;
            pc.ntiles = (c + 1) * tpc < L.ntiles_host ? (c + 1) * tpc : L.ntiles_host;
            pc.tile_counter = cctr + c;
            const uint32_t claims = (pc.ntiles - pc.tile_first + CLAIM_GROUP_ONE_SEG - 1) / CLAIM_GROUP_ONE_SEG;
            const int g = pgrid < (int)claims ? pgrid : (int)claims;
            S512_CUDA_TRY(cudaStreamWaitEvent(st, feed->ready[c], 0));
            pfn<<<g, Shape::THREADS, psmem, st>>>(pc, L.in);
            S512_LAUNCH_CHECK();
        }
        S.kernel_launches += feed->nchunks;
    } else {
        pfn<<<pgrid, Shape::THREADS, psmem, st>>>(pa, L.in);
        S512_LAUNCH_CHECK();
        S.kernel_launches += 1;
    }
    const int t2 = tm.mark();

    PlanArgs<K> pl;
    pl.segs = L.segs;
    pl.splits = splits;
    pl.learned = lsets;
    pl.bucket_counts = counts;
    pl.level_out = L.out;
    for (int c = 0; c <= NCLASS; ++c) pl.items[c] = items[c];
    pl.item_cap = item_cap;
    pl.next = next_segs;
    pl.next_cap = next_cap;
    pl.ctl = ctl;
    pl.key_bytes = KB;
    plan_kernel<K><<<nsegs, NB, 0, st>>>(pl, nsegs);
    S512_LAUNCH_CHECK();
    S512_CUDA_TRY(cudaMemcpyAsync(host_ctl, ctl, sizeof(LevelCtl), cudaMemcpyDeviceToHost, st));
    S512_CUDA_TRY(cudaStreamSynchronize(st));
    S.kernel_launches += 1;

    if (host_ctl->err & DEV_ERR_TIMEOUT) {
        set_error("partition wait timed out at level %d", level);
        return S512_ERR_TIMEOUT;
    }
    if (host_ctl->err & DEV_ERR_OVERFLOW) {
        // a bucket outgrew its sampled capacity: exact counts, exact regions,
        // redo with the splitters only
        S.fallbacks += 1;
        if (lsets) S.learned_rejected += host_ctl->learned_used;
        pa.learned = nullptr;
        pl.learned = nullptr;
        const uint32_t ntiles = L.ntiles_dev ? host_ctl->ntiles_next : L.ntiles_host;
        (void)ntiles;
        S512_CUDA_TRY(cudaMemsetAsync(counts, 0, (size_t)nsegs * NB * sizeof(uint64_t), st));
        // same tile shape as the partition kernel: tiles are numbered for it
        auto cfn = count_kernel<K, InCodec, Shape::THREADS, Shape::IPT>;
        int cgrid = 0;
        S512_CUDA_TRY(launch_persistent(C, cfn, Shape::THREADS, 0, st, 0, &cgrid));
        cfn<<<cgrid, Shape::THREADS, 0, st>>>(pa, L.in);
        S512_LAUNCH_CHECK();
        exact_regions_kernel<K><<<nsegs, NB, 0, st>>>(splits, counts, nsegs);
        S512_LAUNCH_CHECK();
        S512_CUDA_TRY(cudaMemsetAsync(ctl, 0, sizeof(LevelCtl), st));
        S512_CUDA_TRY(cudaMemsetAsync(counts, 0, (size_t)nsegs * NB * sizeof(uint64_t), st));
        pfn<<<pgrid, Shape::THREADS, psmem, st>>>(pa, L.in);
        S512_LAUNCH_CHECK();
        plan_kernel<K><<<nsegs, NB, 0, st>>>(pl, nsegs);
        S512_LAUNCH_CHECK();
        S512_CUDA_TRY(cudaMemcpyAsync(host_ctl, ctl, sizeof(LevelCtl), cudaMemcpyDeviceToHost, st));
        S512_CUDA_TRY(cudaStreamSynchronize(st));
        S.kernel_launches += 5;
    }
    if (host_ctl->err) {
        if (host_ctl->err & DEV_ERR_TIMEOUT) {
            set_error("partition wait timed out at level %d", level);
            return S512_ERR_TIMEOUT;
        }
        set_error("partition level %d reported device error 0x%x", level, host_ctl->err);
        return S512_ERR_INTERNAL;
    }

    // leaves of this level
    const int t3 = tm.mark();
    size_t n_block_items = 0;
    for (int c = 1; c < NCLASS; ++c) n_block_items += host_ctl->n_items[c];
    LeafItem<K>* uneven =
        n_block_items ? (LeafItem<K>*)C.get("uneven", n_block_items * sizeof(LeafItem<K>)) : nullptr;
    if (n_block_items && !uneven) return S512_ERR_ALLOC;
    for (int c = 0; c <= NCLASS; ++c) {
        if (host_ctl->n_items[c] == 0) continue;
        rc = launch_leaf_class<K, UserOut>(C, c, items[c], host_ctl->n_items[c], uout, uneven,
                                           c < NCLASS ? &ctl->n_uneven[c] : nullptr, st);
        if (rc) return rc;
        S.kernel_launches += (c >= 1 && c < NCLASS) ? 2 : 1;
        if (c >= 1 && c < NCLASS) uneven += host_ctl->n_items[c];
    }
    const int t4 = tm.mark();

    if (lsets && host_ctl->learned_used) S.learned_levels += 1;
    if (lsets) S.learned_rejected += host_ctl->plain_used;
    if (level < S512_MAX_LEVELS) {
        S.partition_keys[level] += (level == 0) ? (uint64_t)n : 0;
        S.partition_launches[level] += 1;
        if (lsets) {
            S.learned_segments[level] += host_ctl->learned_used;
            S.learned_fitted[level] += host_ctl->learned_fitted;
            float imb;
            memcpy(&imb, &host_ctl->model_imb_bits, sizeof(imb));
            if (host_ctl->learned_fitted && imb > S.model_max_over_mean[level]) S.model_max_over_mean[level] = imb;
        }
        if (tm.on()) {
            S.sample_ms[level] += tm.ms(t0, t1);
            if (tfit0 >= 0) S.fit_ms[level] += tm.ms(tfit0, t1);
            S.partition_ms[level] += tm.ms(t1, t2);
            S.leaf_ms[level] += tm.ms(t2, t4);
        }
        (void)t3;
        // imbalance: largest bucket over the mean non-empty bucket of the level
        if (host_ctl->nonempty && host_ctl->level_keys) {
            const double mean = (double)host_ctl->level_keys / (double)host_ctl->nonempty;
            S.max_bucket_over_mean[level] = (double)host_ctl->max_bucket / mean;
            const double var = host_ctl->bucket_sq / (double)host_ctl->nonempty - mean * mean;
            S.bucket_cv[level] = var > 0.0 ? sqrt(var) / mean : 0.0;
        }
    }
    (void)next_ctl_dev;
    return S512_OK;
}

// Partition levels starting from `nsegs0` segments of the caller's array
// (keys0 keys in all), described on the device by segs0 (in_off, count,
// final_off set).  A single segment starting at element 0 is laid out here;
// several segments are laid out by prepare_level_kernel.  Buckets that fit a
// leaf are sorted straight into their final place in the caller's array.
//
// `whole` says that segs0 is one segment covering the caller's array from
// element 0 with its tile fields set (sort_pipeline); any other list, even of
// one segment, is laid out on the device (a lone segment of a batch starts
// wherever the caller's segment starts, so its tiles need not be 16-byte
// aligned for the bulk copy).
template <typename K, typename UserIn, typename UserOut>
static int run_levels(DevCtx& C, UserIn uin, UserOut uout, SegDesc* segs0, uint32_t nsegs0, uint64_t keys0,
                      cudaStream_t st, PhaseTimer& tm, s512_stats& S, bool whole, bool learned = false,
                      const HostFeed* feed = nullptr) {
    constexpr int KB = sizeof(K);
    using Shape = PartShape<K>;
    constexpr int TILE = Shape::THREADS * Shape::IPT;
    constexpr int TILE_ONE = PartShapeOne<K>::THREADS * PartShapeOne<K>::IPT;
    const bool single = whole && nsegs0 == 1;

    // Level buffers T0 / T1 alternate as partition outputs.  A level's output
    // needs the sum over its segments of region_bound(count) rounded to 16
    // (prepare_level_kernel lays the segments out that way).
    K* T[2];
    // (plus JUNK_KEYS at the end, where a bucket that overflows its region
    // writes that tile's keys: the level is then redone)
    const size_t need0 = single ? region_bound(keys0) + 64
                                : 2 * keys0 + keys0 / 100 + (size_t)nsegs0 * (4096 + 16) + 64;
    T[0] = (K*)C.get("T0", (need0 + JUNK_KEYS) * KB);
    T[1] = nullptr;
    LevelCtl* ctls = (LevelCtl*)C.get("ctl", 2 * sizeof(LevelCtl));
    LevelCtl* host_ctl = (LevelCtl*)C.host_pinned(sizeof(LevelCtl));
    const uint32_t next_cap = (uint32_t)(keys0 / leaf_max(KB)) + 2;
    SegDesc* segbuf[2];
    segbuf[0] = (SegDesc*)C.get("segs0", (size_t)next_cap * sizeof(SegDesc));
    segbuf[1] = (SegDesc*)C.get("segs1", (size_t)next_cap * sizeof(SegDesc));
    if (!T[0] || !ctls || !host_ctl || !segbuf[0] || !segbuf[1]) return S512_ERR_ALLOC;

    // level 0 reads the caller's layout
    Level<K, UserIn> L0;
    L0.in = uin;
    L0.segs = segs0;
    L0.nsegs = nsegs0;
    L0.out = T[0];
    L0.junk = need0;
    if (single) {
        L0.tile_seg = nullptr;
        L0.ntiles_host = (uint32_t)((keys0 + TILE_ONE - 1) / TILE_ONE);
        L0.ntiles_dev = nullptr;
        L0.ntiles_bound = L0.ntiles_host;
        L0.aligned = true;
    } else {
        const uint32_t bound = (uint32_t)(keys0 / TILE) + nsegs0 + 1;
        uint32_t* tile_seg = (uint32_t*)C.get("tile_seg", (size_t)bound * sizeof(uint32_t));
        if (!tile_seg) return S512_ERR_ALLOC;
        S512_CUDA_TRY(cudaMemsetAsync(&ctls[1], 0, sizeof(LevelCtl), st));
        prepare_level_kernel<<<1, 1024, 0, st>>>(segs0, nsegs0, TILE, &ctls[1]);
        S512_LAUNCH_CHECK();
        tile_map_kernel<<<nsegs0, 256, 0, st>>>(segs0, nsegs0, tile_seg);
        S512_LAUNCH_CHECK();
        S.kernel_launches += 2;
        L0.tile_seg = tile_seg;
        L0.ntiles_host = 0;
        L0.ntiles_dev = &ctls[1].ntiles_next;
        L0.ntiles_bound = bound;
        L0.aligned = false;  // segment starts are wherever the caller's segments start
    }
    if (!single) S512_TRY_RC(wait_feed(feed, st));  // (only a whole array is fed chunk by chunk)
    int rc = single ? run_level<K, UserIn, UserOut, PartShapeOne<K>>(C, L0, 0, uout, keys0, st, &ctls[0], &ctls[1],
                                                                      segbuf[1], next_cap, tm, S, host_ctl, learned,
                                                                      feed)
                    : run_level<K, UserIn, UserOut>(C, L0, 0, uout, keys0, st, &ctls[0], &ctls[1], segbuf[1],
                                                    next_cap, tm, S, host_ctl, learned);
    if (rc) return rc;
    S.levels = 1;

    uint32_t nsegs = host_ctl->n_next;
    uint64_t next_keys = host_ctl->next_keys;
    int level = 1;
    while (nsegs > 0) {
        if (level >= 16) {
            set_error("partition did not converge after %d levels", level);
            return S512_ERR_INTERNAL;
        }
        SegDesc* cur = segbuf[level & 1];
        SegDesc* nxt = segbuf[(level + 1) & 1];
        K* in_buf = T[(level - 1) & 1];
        // grow (never shrink) this level's output buffer; its old contents
        // were consumed two levels ago
        const size_t need = 2 * next_keys + next_keys / 100 + (size_t)nsegs * (4096 + 16) + 64;
        T[level & 1] = (K*)C.get((level & 1) ? "T1" : "T0", (need + JUNK_KEYS) * KB);
        K* out_buf = T[level & 1];
        if (!out_buf) return S512_ERR_ALLOC;
        const uint32_t ntiles_bound = (uint32_t)(next_keys / TILE) + nsegs + 1;
        uint32_t* tile_seg = (uint32_t*)C.get("tile_seg", (size_t)ntiles_bound * sizeof(uint32_t));
        if (!tile_seg) return S512_ERR_ALLOC;
        LevelCtl* lctl = &ctls[level & 1];
        LevelCtl* tctl = &ctls[(level + 1) & 1];  // receives this level's tile count
        S512_CUDA_TRY(cudaMemsetAsync(tctl, 0, sizeof(LevelCtl), st));
        prepare_level_kernel<<<1, 1024, 0, st>>>(cur, nsegs, TILE, tctl);
        S512_LAUNCH_CHECK();
        tile_map_kernel<<<nsegs, 256, 0, st>>>(cur, nsegs, tile_seg);
        S512_LAUNCH_CHECK();
        S.kernel_launches += 2;
        Level<K, Raw<K>> Ln;
        Ln.in = Raw<K>{in_buf, nullptr};
        Ln.segs = cur;
        Ln.nsegs = nsegs;
        Ln.tile_seg = tile_seg;
        Ln.ntiles_host = 0;
        Ln.ntiles_dev = &tctl->ntiles_next;
        Ln.ntiles_bound = ntiles_bound;
        Ln.out = out_buf;
        Ln.junk = need;
        Ln.aligned = true;
        // the tile count lives in tctl, so the level's own control block is the other one
        rc = run_level<K, Raw<K>, UserOut>(C, Ln, level, uout, keys0, st, lctl, tctl, nxt, next_cap, tm, S,
                                           host_ctl, learned);
        if (rc) return rc;
        if (level < S512_MAX_LEVELS) S.partition_keys[level] += next_keys;
        nsegs = host_ctl->n_next;
        next_keys = host_ctl->next_keys;
        ++level;
        S.levels = level;
    }
    return S512_OK;
}

// The whole pipeline for one array of n > leaf_max keys.
template <typename K, typename UserIn, typename UserOut>
static int sort_pipeline(DevCtx& C, UserIn uin, UserOut uout, size_t n, cudaStream_t st, bool learned,
                         const HostFeed* feed = nullptr) {
    constexpr int TILE = PartShapeOne<K>::THREADS * PartShapeOne<K>::IPT;  // a single segment
    s512_stats& S = thread_stats();
    PhaseTimer tm(st, config().collect_stats != 0);
    const int tstart = tm.mark();
    SegDesc* seg0 = (SegDesc*)C.get("seg_whole", sizeof(SegDesc));
    if (!seg0) return S512_ERR_ALLOC;
    SegDesc s0;
    s0.in_off = 0;
    s0.count = n;
    s0.final_off = 0;
    s0.out_base = 0;
    s0.tile_start = 0;
    s0.ntiles = (uint32_t)((n + TILE - 1) / TILE);
    S512_CUDA_TRY(cudaMemcpyAsync(seg0, &s0, sizeof(SegDesc), cudaMemcpyHostToDevice, st));
    int rc = run_levels<K, UserIn, UserOut>(C, uin, uout, seg0, 1, n, st, tm, S, true, learned, feed);
    if (rc) return rc;
    const int tend = tm.mark();
    if (tm.on()) S.total_ms = tm.ms(tstart, tend);
    return S512_OK;
}

// ---------------------------------------------------------------------------
// Entry: sort `n` keys read through uin and written through uout (same
// positions; device memory).
template <typename K, typename UserIn, typename UserOut>
static int sort_device(DevCtx& C, UserIn uin, UserOut uout, size_t n, cudaStream_t st, bool learned = false,
                       const HostFeed* feed = nullptr) {
    s512_stats& S = thread_stats();
    memset(&S, 0, sizeof(S));
    S.key_bytes = sizeof(K);
    if (n <= leaf_max(sizeof(K))) S512_TRY_RC(wait_feed(feed, st));  // no partition level to feed
    if (n <= 1) {
        if (n == 1) {
            // still route through the codec so in != out works
            int rc = sort_one_leaf<UserIn, UserOut>(C, uin, uout, 1, st);
            S.kernel_launches = 1;
            return rc;
        }
        return S512_OK;
    }
    if (n <= leaf_max(sizeof(K))) {
        PhaseTimer tm(st, config().collect_stats != 0);
        const int a = tm.mark();
        int rc = sort_one_leaf<UserIn, UserOut>(C, uin, uout, (uint32_t)n, st);
        const int b = tm.mark();
        S.kernel_launches = 1;
        if (tm.on()) S.total_ms = tm.ms(a, b);
        return rc;
    }
    return sort_pipeline<K, UserIn, UserOut>(C, uin, uout, n, st, learned, feed);
}

// ---------------------------------------------------------------------------
// Host-pointer calls: the caller's arrays are copied to device buffers of the
// stream's pool, sorted there and copied back.

// Page-locked host arrays at least this large are copied in chunks that the
// first partition level consumes as they land.
constexpr size_t HOST_CHUNKED_MIN_BYTES = 16u << 20;
constexpr uint32_t HOST_CHUNKS = 32;

// Copy n elements of narr host arrays (esz bytes each) into the device
// buffers dev[].  Page-locked arrays that a sort of K keys would partition
// go in chunks on the pool's copy stream, with *feed describing them for the
// first level (*chunked set); anything else is one copy per array on st.
template <typename K>
static int copy_in(DevCtx& C, int narr, void* const* host, void* const* dev, size_t esz, size_t n, bool pinned,
                   cudaStream_t st, HostFeed* feed, bool* chunked) {
    *chunked = false;
    const void* mapped[2] = {nullptr, nullptr};
    bool can = pinned && n > leaf_max(sizeof(K)) && n * esz * narr >= HOST_CHUNKED_MIN_BYTES;
    for (int k = 0; can && k < narr; ++k) {
        mapped[k] = mapped_host_address(host[k]);
        can = mapped[k] != nullptr;
    }
    if (!can) {
        for (int k = 0; k < narr; ++k)
            S512_CUDA_TRY(cudaMemcpyAsync(dev[k], host[k], n * esz, cudaMemcpyHostToDevice, st));
        return S512_OK;
    }
    constexpr uint64_t TILE = (uint64_t)PartShapeOne<K>::THREADS * PartShapeOne<K>::IPT;
    const uint64_t per = (n + HOST_CHUNKS - 1) / HOST_CHUNKS;
    const uint64_t chunk = (per + TILE - 1) / TILE * TILE;
    const uint32_t nchunks = (uint32_t)((n + chunk - 1) / chunk);
    S512_CUDA_TRY(C.copy_resources(nchunks + 1));
    // the copies start after the work already queued on st (which may still
    // read the same device buffers)
    cudaEvent_t start = C.events[nchunks];
    S512_CUDA_TRY(cudaEventRecord(start, st));
    S512_CUDA_TRY(cudaStreamWaitEvent(C.copy_stream, start, 0));
    for (uint32_t c = 0; c < nchunks; ++c) {
        const uint64_t off = (uint64_t)c * chunk;
        const uint64_t len = n - off < chunk ? n - off : chunk;
        for (int k = 0; k < narr; ++k)
            S512_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(dev[k]) + off * esz,
                                          static_cast<const char*>(host[k]) + off * esz, len * esz,
                                          cudaMemcpyHostToDevice, C.copy_stream));
        S512_CUDA_TRY(cudaEventRecord(C.events[c], C.copy_stream));
    }
    feed->mapped[0] = mapped[0];
    feed->mapped[1] = mapped[1];
    feed->nchunks = nchunks;
    feed->chunk_keys = chunk;
    feed->ready = C.events.data();
    *chunked = true;
    return S512_OK;
}

// learned splitters for this call: the flag wins over the configuration
static inline bool use_learned(int flags) {
    if (flags & S512_SPLIT_LEARNED) return true;
    if (flags & S512_SPLIT_PLAIN) return false;
    return config().splitter_mode == S512_SPLIT_LEARNED;
}

// A call returns at once with S512_ASYNC when its data is device memory or
// page-locked host memory (the caller synchronises the stream before reading
// the result); pageable host memory is always waited for.
static int finish_call(CallGuard& g, cudaStream_t st, int flags, bool host, bool host_pinned = false) {
    g.finish();
    if (!(flags & S512_ASYNC) || (host && !host_pinned)) S512_CUDA_TRY(cudaStreamSynchronize(st));
    return S512_OK;
}

}  // namespace s512

