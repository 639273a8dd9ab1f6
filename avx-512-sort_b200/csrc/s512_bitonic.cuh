// s512_bitonic.cuh -- bitonic sorting networks in registers and across a
// warp with __shfl_xor_sync.
//
// This is the GPU form of the reference's leaf: SmallSort16V (sort512.hpp:
// 5312-5689 int, 2255-2634 double) loads up to 16 AVX-512 vectors, pads the
// tail with the type's maximum, runs the CoreSmallSortN network (permute +
// min/max + mask blend, e.g. CoreSmallSort 2637-2720, CoreExchangeSort2V
// 2727-2783, CoreSmallEnd 3873-4813) and stores the first `length` lanes.
// Here one warp holds 32*IPT keys, IPT per lane in registers; a stage whose
// partner is in the same lane is a register min/max, and a stage whose partner
// is in another lane is a __shfl_xor_sync exchange.  Longer runs are merged
// (s512_blocksort.cuh).
//
// Element layout ("blocked"): lane l of warp w holds elements
//   e = (w*32 + l)*IPT + r,  r = 0..IPT-1.
// The network is the "mirror" form of bitonic sort: for each merge size k the
// first stage compares e with e ^ (k-1) (both halves were sorted ascending),
// then half-cleaners compare e with e ^ j for j = k/4 .. 1.  Every comparator
// puts the minimum at the lower index, so no direction bits are needed.
#pragma once

#include "s512_common.cuh"

namespace s512 {

// Stage helpers ------------------------------------------------------------

// Register-local comparator stage: pairs (r, r ^ m) inside one lane.
template <typename K, int IPT>
__device__ __forceinline__ void reg_stage(K (&x)[IPT], int m) {
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const int p = r ^ m;
        if (p > r) cas(x[r], x[p]);
    }
}

// Mirror stage inside a lane (k <= IPT): pairs (r, r ^ (k-1)).
template <typename K, int IPT>
__device__ __forceinline__ void reg_mirror(K (&x)[IPT], int k) {
    reg_stage<K, IPT>(x, k - 1);
}

// Cross-lane half-cleaner: partner lane l ^ lm, same register.
template <typename K, int IPT>
__device__ __forceinline__ void lane_stage(K (&x)[IPT], int lm) {
    const bool upper = (lane_id() & (unsigned)lm) != 0;
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const K y = shfl_xor(x[r], lm);
        x[r] = keep_side(x[r], y, upper);
    }
}

// Cross-lane mirror: partner lane l ^ lm, register IPT-1-r.  `hb` is the
// lane bit that tells the upper half of the k-block.
template <typename K, int IPT>
__device__ __forceinline__ void lane_mirror(K (&x)[IPT], int lm, int hb) {
    const bool upper = (lane_id() & (unsigned)hb) != 0;
#pragma unroll
    for (int r = 0; r < IPT / 2; ++r) {
        const int q = IPT - 1 - r;
        const K yr = shfl_xor(x[q], lm);
        const K yq = shfl_xor(x[r], lm);
        x[r] = keep_side(x[r], yr, upper);
        x[q] = keep_side(x[q], yq, upper);
    }
    if (IPT == 1) {
        const K y = shfl_xor(x[0], lm);
        x[0] = keep_side(x[0], y, upper);
    }
}

// Half-cleaners j = jtop .. 1 restricted to one warp (jtop < 32*IPT).
template <typename K, int IPT>
__device__ __forceinline__ void warp_half_cleaners(K (&x)[IPT], int jtop) {
#pragma unroll
    for (int j = jtop; j > 0; j >>= 1) {
        if (j < IPT) reg_stage<K, IPT>(x, j);
        else lane_stage<K, IPT>(x, j / IPT);
    }
}

// Sort the 32*IPT keys held by one warp (blocked layout), ascending.
template <typename K, int IPT>
__device__ __forceinline__ void warp_bitonic_sort(K (&x)[IPT]) {
#pragma unroll
    for (int k = 2; k <= 32 * IPT; k <<= 1) {
        if (k <= IPT) {
            reg_mirror<K, IPT>(x, k);
        } else {
            lane_mirror<K, IPT>(x, k / IPT - 1, k / IPT / 2);
        }
        warp_half_cleaners<K, IPT>(x, k / 4);
    }
}

}  // namespace s512
