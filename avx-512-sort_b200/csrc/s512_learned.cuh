// s512_learned.cuh -- learned splitters: a small monotone CDF model per
// segment, fitted on the device to the segment's sorted sample, that maps a
// key to its bucket in a few arithmetic steps instead of the plain splitters'
// slot table and compares.  The plain splitters stay as the fallback.
//
// Model (all slopes non-negative, so the map is monotone by construction):
//   zr  = float(key - kmin) * R / float(kmax - kmin)       (saturating at 0)
//   p0  = c[s] + w[s] * min(zr - s, 1),   s = min(floor(zr), R - 1)   (root)
//   l   = clamp(floor(p0 * LEAVES))                           (leaf choice)
//   p   = clamp(a[l] + b[l] * float(key - base[l]), lo[l], hi[l])
//   r   = min(floor(p * nmodel), nmodel - 1)                  (model bucket)
// with w = theta^2 >= 0 (root slopes; each trimmed so that c[s] + w[s] <=
// c[s+1] in float arithmetic), c the running sum of w, b >= 0, and
// [lo[l], hi[l]] the sample-CDF range of leaf l, so that every leaf's outputs
// lie above the previous leaf's.  Each step is a non-decreasing function of
// the previous one, in IEEE arithmetic too, hence keys map to buckets in key
// order and a partition by model buckets is a valid sample-sort partition:
// the model only decides how balanced the buckets are, never the result.
// A "heavy" key (one that repeats among the sample quantiles, as for the plain
// splitters' equality buckets) splits its model bucket into below / equal /
// above, and its equal bucket needs no sort.
//
// Training (on the device, per segment): targets are the
// sample's empirical CDF y_i = (i + 0.5) / m.  The root starts from the
// sample histogram over its R pieces and takes ITERS full-batch Adam steps on
// theta with the analytic gradient
//   dL/dw_t = (2/m) * ( sum_{i: s_i > t} r_i + sum_{i: s_i = t} r_i * frac_i ),
//   dL/dtheta_t = dL/dw_t * 2 * theta_t,         r_i = p0(z_i) - y_i.
// Both sums are evaluated from six per-piece sums of the sample taken once
// (root_moments below), so the steps themselves never touch the sample.
// Each leaf starts from its least-squares line on the samples routed to it,
// which is already the optimum of its squared error when its slope is
// positive; a leaf whose least-squares slope was clipped to 0 takes
// LEAF_ITERS Adam steps on (a, beta) with b = beta^2.
//
// The fit is three launches: the roots (one block per segment), the leaves
// (one warp per (segment, leaf), all segments at once), and the bucket layout
// (one block per segment).  A segment is routed by its model only when the
// model passes the balance check AND the plain splitter table would have to
// search for many keys (more than LR_TABLE_SEARCH_FRAC of the sample falls in
// slots shared by several splitters, as with tightly clustered keys): where
// the table settles a key with one lookup the model has nothing to win.
#pragma once

#include "s512_blocksort.cuh"

// (included from s512_sortpipe.cuh after the split-set types)

namespace s512 {

// Segments below this many keys are not fitted: a partition pass over them
// is short next to the fit, and once the first level has split the clusters
// apart the splitter table rarely searches (the levels of many segments).
constexpr uint64_t LR_MIN_KEYS = 1ull << 23;
constexpr int LR_ROOT = 256;
constexpr int LR_LEAVES = 256;
constexpr int LR_THREADS = 512;
constexpr int LR_ITERS = 16;
constexpr int LR_LEAF_ITERS = 8;
constexpr float LR_STEP = 0.02f;  // Adam step, relative to the parameters' scale
constexpr float LR_TABLE_SEARCH_FRAC = 0.25f;

// A leaf: p = a + b * float(key - base) (0 below base), clamped to the
// leaf's sample-CDF range [lo, hi].
template <typename K>
struct LeafParam {
    K base;          // the leaf's first sample key
    float a, b;
    float lo, hi;
};

template <typename K>
struct LearnedSet {
    // the model: everything inference reads, first, so that the partition
    // pass can copy just this prefix (up to region_off) into shared memory
    K kmin;
    float zscale;        // LR_ROOT / float(kmax - kmin)
    uint32_t nmodel;     // model buckets
    float2 rcw[LR_ROOT]; // root piece: (value at its start, slope), normalised, monotone across pieces
    LeafParam<K> leaf[LR_LEAVES];
    K heavy[NB];         // per model bucket: its heavy key (if flagged)
    uint16_t bid[NB];    // per model bucket: first bucket id | 0x100 if it has a heavy key
    // bucket layout and diagnostics
    uint64_t region_off[NB];
    uint64_t region_cap[NB];
    uint32_t bucket_eq[NB / 32];
    uint32_t nbuckets;
    uint32_t ok;         // 1: the model routes the segment (balanced, and cheaper than the splitter table)
    uint32_t balanced;   // 1: imbalance within the bound
    uint32_t fitted;     // 1: trained (0: too small, or the splitter table needs no searches)
    uint32_t searches;   // 1: the splitter table would search for many of the segment's keys
    float loss_init, loss_root, loss_final;
    float max_over_mean;  // sample-count imbalance of the learned buckets (equal buckets aside)
};

// ---------------------------------------------------------------------------
// inference (every step is non-decreasing in its input, in IEEE arithmetic)

__device__ __forceinline__ float key_to_float(uint32_t d) { return __uint2float_rn(d); }
__device__ __forceinline__ float key_to_float(uint64_t d) { return __ull2float_rn(d); }

// The root's key map: pieces split [kmin, kmax] evenly.
template <typename K>
struct RootMap {
    K kmin;
    float zscale;
    __device__ __forceinline__ void init(K lo, K hi) {
        kmin = lo;
        zscale = hi > lo ? (float)LR_ROOT / key_to_float(hi - lo) : 0.f;
    }
    // piece of a key and its place inside the piece, in [0, 1]
    __device__ __forceinline__ int piece(K key, float* frac) const {
        const K d = key > kmin ? key - kmin : K(0);
        const float zr = key_to_float(d) * zscale;
        int s = (int)zr;
        s = s > LR_ROOT - 1 ? LR_ROOT - 1 : s;
        *frac = fminf(zr - (float)s, 1.f);
        return s;
    }
};

template <typename K>
__device__ __forceinline__ RootMap<K> root_map_of(const LearnedSet<K>& L) {
    RootMap<K> r;
    r.kmin = L.kmin;
    r.zscale = L.zscale;
    return r;
}

template <typename K>
__device__ __forceinline__ float root_p0(const RootMap<K>& rm, const float2* rcw, K key) {
    float frac;
    const int s = rm.piece(key, &frac);
    const float2 cw = rcw[s];
    return cw.x + cw.y * frac;
}

template <typename K>
__device__ __forceinline__ float root_p0(const LearnedSet<K>& L, K key) {
    return root_p0<K>(root_map_of<K>(L), L.rcw, key);
}

__device__ __forceinline__ int leaf_of(float p0) {
    const int l = (int)(p0 * (float)LR_LEAVES);
    return l < 0 ? 0 : (l > LR_LEAVES - 1 ? LR_LEAVES - 1 : l);
}

template <typename K>
__device__ __forceinline__ float leaf_p(const LeafParam<K>& lp, K key) {
    const K du = key > lp.base ? key - lp.base : K(0);
    return fminf(fmaxf(lp.a + lp.b * key_to_float(du), lp.lo), lp.hi);
}

__device__ __forceinline__ uint32_t model_bucket(float p, uint32_t nmodel) {
    int r = (int)(p * (float)nmodel);
    r = r < 0 ? 0 : r;
    return (uint32_t)r > nmodel - 1 ? nmodel - 1 : (uint32_t)r;
}

// bucket id of a key under a learned set held in shared memory
template <typename K>
__device__ __forceinline__ uint32_t learned_bucket(const LearnedSet<K>& L, K key) {
    const float p0 = root_p0<K>(L, key);
    const LeafParam<K>& lp = L.leaf[leaf_of(p0)];
    const uint32_t r = model_bucket(leaf_p<K>(lp, key), L.nmodel);
    const uint32_t e = L.bid[r];
    uint32_t id = e & 0xFFu;
    if (e >> 8) {
        const K h = L.heavy[r];
        id += key < h ? 0u : (key == h ? 1u : 2u);
    }
    return id;
}

// ---------------------------------------------------------------------------
// training

// Adam with b1 = 0.9, b2 = 0.999.  The bias corrections depend on the step
// only, so the caller keeps them (AdamBias) for all its parameters.
constexpr float ADAM_B1 = 0.9f, ADAM_B2 = 0.999f;
struct AdamBias {
    float p1 = 1.f, p2 = 1.f;  // b1^t, b2^t
    float c1 = 0.f, c2 = 0.f;  // 1 / (1 - b1^t), 1 / (1 - b2^t)
    __device__ __forceinline__ void next() {
        p1 *= ADAM_B1;
        p2 *= ADAM_B2;
        c1 = 1.f / (1.f - p1);
        c2 = 1.f / (1.f - p2);
    }
};
struct Adam {
    float m = 0.f, v = 0.f;
    __device__ __forceinline__ float step(float g, float lr, const AdamBias& bc) {
        m = ADAM_B1 * m + (1.f - ADAM_B1) * g;
        v = ADAM_B2 * v + (1.f - ADAM_B2) * g * g;
        return lr * (m * bc.c1) / (sqrtf(v * bc.c2) + 1e-8f);
    }
};

// The root's training data, gathered once.  A sample's piece s_i and its
// place f_i inside the piece depend on its key only (not on theta), so with
// p0_i = rc[s_i] + rw[s_i] * f_i, y_i = (i + 1/2) / m and r_i = p0_i - y_i,
// the loss (1/m) sum r_i^2 and the per-piece sums S0_t = sum r_i,
// S1_t = sum r_i f_i (over the samples of piece t) are quadratic in
// (rc_t, rw_t) with six fixed coefficients per piece:
//   n_t, sum f, sum f^2, sum y, sum y^2, sum y f.
// One pass over the sample collects them (in double: the loss is a small
// difference of these sums); a training step is then O(pieces) work in one
// warp.
constexpr int RM_N = 0, RM_F = 1, RM_FF = 2, RM_Y = 3, RM_YY = 4, RM_YF = 5, RM_COUNT = 6;
// Training runs in one warp, RP = LR_ROOT / 32 consecutive pieces a lane
// (lane t / RP holds piece t).  The sums of piece t sit at mom[mom_idx(t, c)]:
// consecutive lanes read consecutive words, free of bank conflicts.
constexpr int RP = LR_ROOT / 32;
__host__ __device__ constexpr int mom_idx(int t, int c) { return ((t % RP) * RM_COUNT + c) * 32 + t / RP; }

// Block-wide.  pstart[t] (LR_ROOT + 1 entries) receives the first sample of
// piece t (samples are sorted and the piece is monotone in the key).
template <typename K>
__device__ void root_moments(const K* smp, uint32_t m, const RootMap<K>& rm, uint32_t* pstart,
                             double* mom) {
    const int tid = threadIdx.x;
    for (int t = tid; t <= LR_ROOT; t += blockDim.x) pstart[t] = m;
    __syncthreads();
    for (uint32_t i = tid; i < m; i += blockDim.x) {
        float f;
        const int s = rm.piece(smp[i], &f);
        const int sp = i == 0 ? -1 : rm.piece(smp[i - 1], &f);
        for (int q = sp + 1; q <= s; ++q) pstart[q] = i;
    }
    __syncthreads();
    const int lane = tid & 31, nw = blockDim.x >> 5;
    const double inv_m = 1.0 / (double)m;
    for (int t = tid >> 5; t < LR_ROOT; t += nw) {
        double a[RM_COUNT] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (uint32_t i = pstart[t] + lane; i < pstart[t + 1]; i += 32) {
            float ff;
            (void)rm.piece(smp[i], &ff);
            const double f = (double)ff, y = ((double)i + 0.5) * inv_m;
            a[RM_N] += 1.0;
            a[RM_F] += f;
            a[RM_FF] += f * f;
            a[RM_Y] += y;
            a[RM_YY] += y * y;
            a[RM_YF] += y * f;
        }
#pragma unroll
        for (int k = 0; k < RM_COUNT; ++k) {
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) a[k] += __shfl_xor_sync(0xFFFFFFFFu, a[k], d);
        }
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < RM_COUNT; ++k) mom[mom_idx(t, k)] = a[k];
    }
    __syncthreads();
}

// One warp, RP = LR_ROOT / 32 consecutive pieces a lane (lane * RP + k): the
// loss of the root with w_t = theta_t^2 (rw = w, rc = exclusive running sum
// of w) and dL/dw_t,
//   dL/dw_t = (2/m) * (S1_t + sum_{u > t} S0_u).
__device__ __forceinline__ void root_eval_warp(const double* mom, uint32_t m, const float (&th)[RP],
                                               double* loss, double (&g)[RP]) {
    const int lane = threadIdx.x & 31;
    double w[RP], lane_w = 0.0;
#pragma unroll
    for (int k = 0; k < RP; ++k) {
        w[k] = (double)th[k] * th[k];
        lane_w += w[k];
    }
    double inc = lane_w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
        if (lane >= d) inc += o;
    }
    double rc = inc - lane_w;  // running sum before this lane's first piece
    double S0[RP], S1[RP], l = 0.0, lane_s0 = 0.0;
#pragma unroll
    for (int k = 0; k < RP; ++k) {
        const double* M = mom + k * RM_COUNT * 32 + lane;  // M[c * 32]: sum c of piece lane * RP + k
        const double A = rc, B = w[k];
        const double n = M[RM_N * 32], sf = M[RM_F * 32], sff = M[RM_FF * 32];
        const double sy = M[RM_Y * 32], syy = M[RM_YY * 32], syf = M[RM_YF * 32];
        S0[k] = n * A + B * sf - sy;
        S1[k] = A * sf + B * sff - syf;
        l += n * A * A + B * B * sff + syy + 2.0 * A * B * sf - 2.0 * A * sy - 2.0 * B * syf;
        lane_s0 += S0[k];
        rc += w[k];
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) l += __shfl_xor_sync(0xFFFFFFFFu, l, d);
    // S0 summed over the pieces after each piece: the later lanes' totals,
    // then this lane's later pieces
    double pre = lane_s0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double o = __shfl_up_sync(0xFFFFFFFFu, pre, d);
        if (lane >= d) pre += o;
    }
    double after = __shfl_sync(0xFFFFFFFFu, pre, 31) - pre;
    const double kk = 2.0 / (double)m;
#pragma unroll
    for (int k = RP - 1; k >= 0; --k) {
        g[k] = kk * (after + S1[k]);
        after += S0[k];
    }
    *loss = (l > 0.0 ? l : 0.0) / (double)m;
}

// --- fit, launch 1: the root of each segment (one block of LR_THREADS each).
// Also the first sample of each leaf (samples are sorted and routing is
// monotone, so each leaf owns a contiguous run of the sample), into
// lfirst[seg * (LR_LEAVES + 1) + l].
template <typename K>
__global__ void __launch_bounds__(LR_THREADS) learned_root_kernel(const K* __restrict__ samples,
                                                                  const SegDesc* __restrict__ segs, uint32_t nsegs,
                                                                  const SplitSet<K>* __restrict__ plain,
                                                                  LearnedSet<K>* __restrict__ out,
                                                                  uint32_t* __restrict__ lfirst, int key_bytes,
                                                                  int force) {
    const uint32_t sgi = blockIdx.x;
    if (sgi >= nsegs) return;
    __shared__ double mom[LR_ROOT * RM_COUNT];
    __shared__ uint32_t pstart[LR_ROOT + 1];
    __shared__ float2 rcw[LR_ROOT];
    __shared__ uint32_t search_s;
    const SegDesc sd = segs[sgi];
    const int tid = threadIdx.x;
    LearnedSet<K>& L = out[sgi];
    const int nb = target_buckets(key_bytes, sd.count);
    const uint32_t m = sample_size(nb);
    const K* smp = samples + (size_t)sgi * SAMPLE_N;
    // worth a fit?  Only for a large segment whose splitter table would have
    // to search for many keys (slots shared by several splitters)
    if (tid == 0) search_s = 0;
    __syncthreads();
    bool fit = sd.count >= LR_MIN_KEYS;
    bool searches = false;
    if (fit) {
        const SplitSet<K>& ps = plain[sgi];
        const SlotMap<K> fmap = ps.slot_map;
        uint32_t mine = 0;
        for (uint32_t i = tid; i < m; i += blockDim.x) {
            const K xc = kmin(kmax(smp[i], fmap.lo), ps.slot_hi);
            mine += (ps.slot_tab[fmap(xc)] >> 8) > 1u ? 1u : 0u;
        }
        atomicAdd(&search_s, mine);
        __syncthreads();
        searches = (float)search_s > LR_TABLE_SEARCH_FRAC * (float)m;
        fit = searches || force;
    }
    if (!fit) {  // the split set routes it
        if (tid == 0) {
            L.ok = 0;
            L.balanced = 0;
            L.fitted = 0;
            L.searches = searches ? 1u : 0u;
        }
        return;
    }
    const K kmin = smp[0], kmax = smp[m - 1];
    RootMap<K> rm;
    rm.init(kmin, kmax);

    // the training data (per-piece sums), then Adam on theta in warp 0, two
    // pieces a lane, from the histogram start theta = sqrt(n_t / m); the
    // parameters with the lowest loss seen are kept, so training never ends
    // worse than its start
    root_moments<K>(smp, m, rm, pstart, mom);
    static_assert(LR_ROOT % 32 == 0, "whole pieces per lane of warp 0");
    if (tid < 32) {
        float th[RP], best_th[RP];
        Adam opt[RP];
#pragma unroll
        for (int k = 0; k < RP; ++k) best_th[k] = th[k] = sqrtf((float)(mom[mom_idx(tid * RP + k, RM_N)] / (double)m));
        double best = 1e300, first = 0.0;
        AdamBias bc;
        for (int it = 0; it <= LR_ITERS; ++it) {
            double loss, g[RP];
            root_eval_warp(mom, m, th, &loss, g);
            if (it == 0) first = loss;
            if (loss < best) {
                best = loss;
#pragma unroll
                for (int k = 0; k < RP; ++k) best_th[k] = th[k];
            }
            if (it == LR_ITERS) break;
            bc.next();
#pragma unroll
            for (int k = 0; k < RP; ++k) th[k] -= opt[k].step((float)(g[k] * 2.0 * th[k]), LR_STEP * 0.125f, bc);
        }
        // the kept root, normalised so that it spans [0, 1]: piece ends
        // b_t = float(C_t / C_R) of the running sums C of w = theta^2, made
        // non-decreasing; piece t starts at b_{t-1} and its slope is the
        // largest float w with b_{t-1} + w <= b_t in float arithmetic, so p0
        // never decreases from the end of one piece to the start of the next
        double w[RP], lane_w = 0.0;
#pragma unroll
        for (int k = 0; k < RP; ++k) {
            w[k] = (double)(best_th[k] * best_th[k]);
            lane_w += w[k];
        }
        double inc = lane_w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
            if (tid >= d) inc += o;
        }
        const double tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
        const double inv = tot > 0.0 ? 1.0 / tot : 0.0;
        const double before = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
        double c = tid ? before : 0.0;
        float b[RP];
#pragma unroll
        for (int k = 0; k < RP; ++k) {
            c += w[k];
            b[k] = (float)(c * inv);
            if (k) b[k] = fmaxf(b[k], b[k - 1]);
        }
        if (tid == 31) b[RP - 1] = fmaxf(b[RP - 1], 1.f);
        float prev_end = b[RP - 1];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const float o = __shfl_up_sync(0xFFFFFFFFu, prev_end, d);
            if (tid >= d) prev_end = fmaxf(prev_end, o);
        }
        prev_end = __shfl_up_sync(0xFFFFFFFFu, prev_end, 1);  // largest end of the earlier lanes
        if (tid == 0) prev_end = 0.f;
        float start = prev_end;
#pragma unroll
        for (int k = 0; k < RP; ++k) {
            const float end = fmaxf(b[k], prev_end);
            float wk = fmaxf(__fsub_rn(end, start), 0.f);
            while (wk > 0.f && __fadd_rn(start, wk) > end) wk = nextafterf(wk, 0.f);
            rcw[tid * RP + k] = make_float2(start, wk);
            L.rcw[tid * RP + k] = make_float2(start, wk);
            start = end;
        }
        if (tid == 0) {
            L.kmin = rm.kmin;
            L.zscale = rm.zscale;
            L.loss_init = (float)first;
            L.loss_root = (float)best;
            L.fitted = 1;
            L.searches = searches ? 1u : 0u;
        }
    }
    __syncthreads();
    uint32_t* lf = lfirst + (size_t)sgi * (LR_LEAVES + 1);
    for (int l = tid; l <= LR_LEAVES; l += blockDim.x) lf[l] = m;
    __syncthreads();
    for (uint32_t i = tid; i < m; i += blockDim.x) {
        const int l = leaf_of(root_p0<K>(rm, rcw, smp[i]));
        const int lp = i == 0 ? -1 : leaf_of(root_p0<K>(rm, rcw, smp[i - 1]));
        for (int q = lp + 1; q <= l; ++q) lf[q] = i;  // leaves lp+1..l start at i
    }
}

// --- fit, launch 2: the leaves, one warp per (segment, leaf), 8 warps a
// block.  The lanes stride over the leaf's (contiguous) samples and every sum
// is reduced across the warp, so all lanes hold the same parameters.
template <typename K>
__global__ void __launch_bounds__(256) learned_leaf_kernel(const K* __restrict__ samples,
                                                           const SegDesc* __restrict__ segs, uint32_t nsegs,
                                                           LearnedSet<K>* __restrict__ out,
                                                           const uint32_t* __restrict__ lfirst, int key_bytes) {
    const uint32_t wg = blockIdx.x * 8 + (threadIdx.x >> 5);
    const uint32_t sgi = wg / LR_LEAVES;
    const int l = (int)(wg % LR_LEAVES);
    if (sgi >= nsegs) return;
    if (!out[sgi].fitted) return;
    const SegDesc sd = segs[sgi];
    const int lane = threadIdx.x & 31;
    const uint32_t m = sample_size(target_buckets(key_bytes, sd.count));
    const K* smp = samples + (size_t)sgi * SAMPLE_N;
    auto wsum = [&](float v) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
        return v;
    };
    // leaf l owns the samples [lfirst[l], lfirst[l+1])
    const uint32_t* lf = lfirst + (size_t)sgi * (LR_LEAVES + 1);
    const uint32_t f = lf[l];
    const uint32_t e = lf[l + 1];
    LeafParam<K> P;
    if (f < e && f < m) {
        const K base = smp[f];
        const K span = smp[e - 1] - base;
        const float inv_span = span ? 1.0f / key_to_float(span) : 0.f;
        // least squares on (u, y), u in [0, 1]
        float su = 0.f, sy = 0.f, suu = 0.f, suy = 0.f;
        const float cnt = (float)(e - f);
        for (uint32_t i = f + lane; i < e; i += 32) {
            const float u = key_to_float(smp[i] - base) * inv_span;
            const float y = ((float)i + 0.5f) / (float)m;
            su += u;
            sy += y;
            suu += u * u;
            suy += u * y;
        }
        su = wsum(su);
        sy = wsum(sy);
        suu = wsum(suu);
        suy = wsum(suy);
        const float mu = su / cnt, my = sy / cnt;
        const float var = suu / cnt - mu * mu, cov = suy / cnt - mu * my;
        float b = var > 1e-12f ? cov / var : 0.f;
        const bool clipped = !(b > 0.f);
        b = clipped ? 0.f : b;
        float a = my - b * mu;
        float beta = sqrtf(b);
        if (clipped) {
            // refine (a, beta), b = beta^2, by Adam on the leaf's squared
            // error (forward + backward per step); keep the best pair seen
            float best_a = a, best_beta = beta, best_l = 3.4e38f;
            Adam oa, ob;
            AdamBias bc;
            for (int it = 1; it <= LR_LEAF_ITERS + 1; ++it) {
                float ga = 0.f, gb = 0.f, l2 = 0.f;
                for (uint32_t i = f + lane; i < e; i += 32) {
                    const float u = key_to_float(smp[i] - base) * inv_span;
                    const float r = a + beta * beta * u - ((float)i + 0.5f) / (float)m;
                    l2 += r * r;
                    ga += r;
                    gb += r * u;
                }
                l2 = wsum(l2);
                ga = wsum(ga);
                gb = wsum(gb);
                if (l2 < best_l) {
                    best_l = l2;
                    best_a = a;
                    best_beta = beta;
                }
                if (it > LR_LEAF_ITERS) break;
                ga *= 2.f / cnt;
                gb *= 2.f / cnt * 2.f * beta;
                bc.next();
                a -= oa.step(ga, LR_STEP / (float)m, bc);
                beta -= ob.step(gb, LR_STEP / (float)m, bc);
            }
            a = best_a;
            beta = best_beta;
        }
        P.base = base;
        P.a = a;
        P.b = beta * beta * inv_span;  // slope per unit of (key - base)
        P.lo = ((float)f + 0.5f) / (float)m;
        P.hi = ((float)(e - 1) + 0.5f) / (float)m;
    } else {
        P.base = KeyMax<K>::value;
        P.a = 0.f;
        P.b = 0.f;
        P.lo = P.hi = -1.f;  // patched in launch 3: an empty leaf repeats its left neighbour's top
    }
    if (lane == 0) out[sgi].leaf[l] = P;
}

// --- fit, launch 3: per segment (one block of NB threads) the empty leaves
// patched, the heavy keys and bucket ids, the sample's bucket histogram, the
// balance check, the routing choice, the regions and the final loss.  The
// plain split set of the segment (computed from the same sorted sample)
// supplies the heavy keys and the table the routing choice compares with.
template <typename K>
__global__ void __launch_bounds__(NB) learned_finish_kernel(const K* __restrict__ samples,
                                                            const SegDesc* __restrict__ segs, uint32_t nsegs,
                                                            const SplitSet<K>* __restrict__ plain,
                                                            LearnedSet<K>* __restrict__ out, int key_bytes,
                                                            float max_imbalance, int report_loss) {
    const uint32_t sgi = blockIdx.x;
    if (sgi >= nsegs) return;
    if (!out[sgi].fitted) return;
    const SegDesc sd = segs[sgi];
    __shared__ LearnedSet<K> L;  // built here, copied out at the end
    __shared__ uint32_t hist[NB];
    __shared__ uint32_t first_heavy[NB];
    __shared__ uint32_t wt32[32];
    __shared__ uint64_t wt64[32];
    __shared__ uint32_t max_s, tot_ids_s, sorted_s;
    __shared__ float loss_s, top_w[NB / 32];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(out + sgi);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&L);
        for (uint32_t i = tid; i < sizeof(LearnedSet<K>) / 4; i += blockDim.x) dst[i] = src[i];
    }
    const int nb = target_buckets(key_bytes, sd.count);
    const uint32_t m = sample_size(nb);
    const K* smp = samples + (size_t)sgi * SAMPLE_N;
    if (tid == 0) {
        max_s = 0;
        sorted_s = 0;
        loss_s = 0.f;
    }
    __syncthreads();

    // empty leaves: lo = hi = a = the top of the nearest non-empty leaf to
    // their left (0 if none): a running maximum of the leaves' tops
    static_assert(LR_LEAVES == NB, "one thread per leaf");
    {
        const bool empty = L.leaf[tid].lo < 0.f;
        float run = empty ? 0.f : L.leaf[tid].hi;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const float o = __shfl_up_sync(0xFFFFFFFFu, run, d);
            if (lane >= d) run = fmaxf(run, o);
        }
        if (lane == 31) top_w[warp] = run;
        __syncthreads();
        for (int w = 0; w < warp; ++w) run = fmaxf(run, top_w[w]);
        __syncthreads();
        if (empty) {
            L.leaf[tid].lo = L.leaf[tid].hi = run;
            L.leaf[tid].a = run;
        }
    }
    __syncthreads();

    // heavy keys (splitters with an equality bucket in the plain split set):
    // a model bucket keeps its first heavy key
    const SplitSet<K>& ps = plain[sgi];
    first_heavy[tid] = 0xFFFFFFFFu;
    const bool heavy = tid < (int)ps.nuniq && ((ps.eq_mask[tid >> 5] >> (tid & 31)) & 1u);
    const uint32_t nheavy = (uint32_t)__syncthreads_count(heavy);
    uint32_t nmodel = NB - 2 * nheavy;
    if (nmodel > (uint32_t)(2 * nb)) nmodel = 2 * nb;  // no more model buckets than the plain path aims for
    if (nmodel < 2) nmodel = 2;
    if (heavy) {
        const K h = ps.uniq[tid];
        const float p0 = root_p0<K>(L, h);
        const uint32_t r = model_bucket(leaf_p<K>(L.leaf[leaf_of(p0)], h), nmodel);
        atomicMin(&first_heavy[r], (uint32_t)tid);
    }
    __syncthreads();
    const bool has_heavy = first_heavy[tid] != 0xFFFFFFFFu && (uint32_t)tid < nmodel;
    L.heavy[tid] = has_heavy ? ps.uniq[first_heavy[tid]] : K(0);
    // bucket ids: a model bucket is one id, or three (below / equal / above)
    // with a heavy key
    const uint32_t width = (uint32_t)tid < nmodel ? (has_heavy ? 3u : 1u) : 0u;
    const uint32_t id = block_exclusive_scan_first<NB, uint32_t>(width, wt32, &tot_ids_s);
    const uint32_t base_id = id < NB ? id : NB - 1;
    L.bid[tid] = (uint16_t)(base_id | (has_heavy ? 0x100u : 0u));
    if (tid == 0) {
        L.nmodel = nmodel;
        L.nbuckets = tot_ids_s;  // (the scan's total, written by one thread to shared memory)
    }
    hist[tid] = 0;
    __syncthreads();

    // the "equal" bucket of each heavy model bucket r is base_id[r] + 1
    if (tid < NB / 32) L.bucket_eq[tid] = 0;
    __syncthreads();
    if (has_heavy) {
        const uint32_t e = base_id + 1;
        atomicOr(&L.bucket_eq[e >> 5], 1u << (e & 31));
    }
    // the sample through the model: its bucket histogram, and the balance of
    // the buckets that are sorted further (an equal bucket holds one key
    // value, however many times it repeats, and is only copied)
    for (uint32_t i = tid; i < m; i += blockDim.x) atomicAdd(&hist[learned_bucket<K>(L, smp[i])], 1u);
    __syncthreads();
    const uint32_t c = hist[tid];
    if (c && !((L.bucket_eq[tid >> 5] >> (tid & 31)) & 1u)) {
        atomicMax(&max_s, c);
        atomicAdd(&sorted_s, c);
    }
    const double scale = (double)sd.count / (double)m;
    uint64_t cap = 0;
    if ((uint32_t)tid < L.nbuckets) {
        const double v = ((double)c + 6.0 * sqrt((double)c + 1.0) + 16.0) * scale;
        cap = (uint64_t)ceil(v);
        if (cap > sd.count) cap = sd.count;
        cap = (cap + 15) & ~15ull;
    }
    const uint64_t off = block_exclusive_scan_first<NB, uint64_t>(cap, wt64, (uint64_t*)nullptr);
    L.region_off[tid] = off;
    L.region_cap[tid] = cap;
    // final loss of the whole model on the sample (root + leaves), for the
    // fit's report only
    if (report_loss) {
        float lfs = 0.f;
        for (uint32_t i = tid; i < m; i += blockDim.x) {
            const float p0 = root_p0<K>(L, smp[i]);
            const float r = leaf_p<K>(L.leaf[leaf_of(p0)], smp[i]) - ((float)i + 0.5f) / (float)m;
            lfs += r * r;
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) lfs += __shfl_xor_sync(0xFFFFFFFFu, lfs, d);
        if (lane == 0) atomicAdd(&loss_s, lfs / (float)m);
    }
    __syncthreads();
    if (tid == 0) {
        // against the mean the model aims at: the sorted samples spread over
        // all nmodel model buckets (a model that sends the sample to a few
        // buckets is unbalanced, however even those few are)
        const float mean = sorted_s ? (float)sorted_s / (float)L.nmodel : 1.f;
        L.max_over_mean = (float)max_s / mean;
        L.balanced = (L.max_over_mean <= max_imbalance && L.nbuckets <= (uint32_t)NB) ? 1u : 0u;
        L.ok = (L.balanced && L.searches) ? 1u : 0u;
        L.loss_final = loss_s;
    }
    __syncthreads();
    uint32_t* dst = reinterpret_cast<uint32_t*>(out + sgi);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&L);
    for (uint32_t i = tid; i < sizeof(LearnedSet<K>) / 4; i += blockDim.x) dst[i] = src[i];
}

// The three launches of a fit (lfirst: nsegs * (LR_LEAVES + 1) words).
// force: train every large segment, also where the table would not search
// (the model is then reported but does not route), and compute the final
// loss for the report.
template <typename K>
static void launch_learned_fit(const K* samples, const SegDesc* segs, uint32_t nsegs, const SplitSet<K>* plain,
                               LearnedSet<K>* out, uint32_t* lfirst, int key_bytes, float max_imbalance,
                               cudaStream_t st, int force = 0) {
    learned_root_kernel<K><<<nsegs, LR_THREADS, 0, st>>>(samples, segs, nsegs, plain, out, lfirst, key_bytes,
                                                         force);
    learned_leaf_kernel<K><<<(nsegs * LR_LEAVES + 7) / 8, 256, 0, st>>>(samples, segs, nsegs, out, lfirst, key_bytes);
    learned_finish_kernel<K><<<nsegs, NB, 0, st>>>(samples, segs, nsegs, plain, out, key_bytes, max_imbalance,
                                                   force);
}

}  // namespace s512
