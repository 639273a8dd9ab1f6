// s512_partition2.cuh -- the two-way partition behind Partition512.
//
// Partition512 (sort512.hpp:5729-5819 int, 5821-5912 double; kv
// sort512kv.hpp:5959-6082) moves every element <= pivot before every element
// > pivot inside [left, right] and returns the first index of the > side.  The
// reference walks the range from both ends with compress-stores.  Here each
// tile of the range ranks its "low" and "high" elements with warp ballots,
// learns how many lows and highs all earlier tiles hold from a decoupled
// look-back (two counters per tile), and writes lows forward from the start
// and highs backward from the end of a scratch range, which the host copies
// back when the kernel reports no error.  The comparison is the reference's own: `x <= pivot` on the caller's
// type (so a NaN double goes to the high side, as with _CMP_LE_OQ).
#pragma once

#include "s512_common.cuh"

namespace s512 {

constexpr unsigned long long ST_INC_P2 = 1ull << 63;  // status: inclusive count
constexpr unsigned long long ST_AGG_P2 = 1ull << 62;  // status: tile count only
constexpr unsigned long long ST_VAL_P2 = (1ull << 62) - 1;

struct Part2Ctl {
    uint32_t tile_counter;
    uint32_t err;
    unsigned long long total_low;
};

template <typename T, bool KV, int THREADS, int IPT>
__global__ void __launch_bounds__(THREADS) partition2_kernel(const T* __restrict__ in, const int* __restrict__ vin,
                                                             T* __restrict__ out, int* __restrict__ vout, uint64_t n,
                                                             T pivot, unsigned long long* __restrict__ status,
                                                             Part2Ctl* ctl, uint32_t ntiles,
                                                             uint32_t inject_slot = 0xFFFFFFFFu) {
    constexpr int NW = THREADS / 32;
    constexpr int TILE = THREADS * IPT;
    constexpr int NC = IPT * NW;  // counters per tile, multiple of 32
    static_assert(NC % 32 == 0 && NC <= THREADS, "tile shape");
    __shared__ uint64_t cnt[NC];  // (lows << 32) | highs for (item r, warp w)
    __shared__ uint64_t wtot[32];
    __shared__ uint64_t tile_tot;
    __shared__ uint64_t pre[2];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x;
    const unsigned lane = lane_id(), warp = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;

    while (true) {
        if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter, 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles) break;
        const uint64_t base = (uint64_t)t * TILE;
        T x[IPT];
        int v[IPT];
        uint32_t mask_lo[IPT], mask_hi[IPT];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint64_t i = base + (uint64_t)r * THREADS + tid;
            const bool valid = i < n;
            x[r] = pivot;
            v[r] = 0;
            if (valid) {
                x[r] = in[i];
                if (KV) v[r] = vin[i];
            }
            const bool low = valid && (x[r] <= pivot);
            const bool high = valid && !(x[r] <= pivot);
            mask_lo[r] = __ballot_sync(0xFFFFFFFFu, low);
            mask_hi[r] = __ballot_sync(0xFFFFFFFFu, high);
            if (lane == 0) cnt[r * NW + warp] = ((uint64_t)__popc(mask_lo[r]) << 32) | (uint64_t)__popc(mask_hi[r]);
        }
        __syncthreads();
        uint64_t c = (tid < NC) ? cnt[tid] : 0ull;
        const uint64_t ex = block_exclusive_scan_first<NC, uint64_t>(c, wtot, &tile_tot);
        if (tid < NC) cnt[tid] = ex;
        __syncthreads();
        const uint64_t tlo = tile_tot >> 32, thi = tile_tot & 0xFFFFFFFFull;
        // look-back: thread 0 counts lows, thread 1 highs
        if (tid < 2) {
            const uint64_t mine = tid == 0 ? tlo : thi;
            unsigned long long* st = status + (size_t)t * 2 + tid;
            uint64_t prefix = 0;
            if (t == 0) {
                st_status(st, ST_INC_P2 | mine);
            } else if (t == 1 && inject_slot != 0xFFFFFFFFu) {
                // testing: a predecessor that never publishes (the spare
                // status slot past the last tile), waited for with a short
                // bound; the tile records the timeout and writes nothing
                st_status(st, ST_AGG_P2 | mine);
                uint32_t spins = 0;
                while (!(ld_status(status + (size_t)inject_slot * 2 + tid) & (ST_INC_P2 | ST_AGG_P2)) &&
                       ++spins < 1024u)
                    __nanosleep(100);
                raise_error(&ctl->err, DEV_ERR_TIMEOUT);
                prefix = ~0ull;
            } else {
                st_status(st, ST_AGG_P2 | mine);
                uint32_t p = t - 1;
                while (true) {
                    unsigned long long w;
                    uint32_t spins = 0;
                    while (true) {
                        w = ld_status(status + (size_t)p * 2 + tid);
                        if (w & (ST_INC_P2 | ST_AGG_P2)) break;
                        if (++spins > SPIN_LIMIT) break;
                        __nanosleep(spins < 64 ? 20 : 200);
                    }
                    if (!(w & (ST_INC_P2 | ST_AGG_P2))) {
                        raise_error(&ctl->err, DEV_ERR_TIMEOUT);
                        prefix = ~0ull;  // writes below are skipped
                        break;
                    }
                    prefix += w & ST_VAL_P2;
                    if (w & ST_INC_P2) break;
                    --p;
                }
                if (prefix != ~0ull) st_status(st, ST_INC_P2 | (prefix + mine));
            }
            pre[tid] = prefix;
            if (t == ntiles - 1 && tid == 0 && prefix != ~0ull) ctl->total_low = prefix + mine;
        }
        __syncthreads();
        const uint64_t plo = pre[0], phi = pre[1];
        if (plo != ~0ull && phi != ~0ull) {
#pragma unroll
            for (int r = 0; r < IPT; ++r) {
                const uint64_t off = cnt[r * NW + warp];
                if ((mask_lo[r] >> lane) & 1u) {
                    const uint64_t o = plo + (off >> 32) + __popc(mask_lo[r] & lt);
                    out[o] = x[r];
                    if (KV) vout[o] = v[r];
                } else if ((mask_hi[r] >> lane) & 1u) {
                    const uint64_t o = n - 1 - (phi + (off & 0xFFFFFFFFull) + __popc(mask_hi[r] & lt));
                    out[o] = x[r];
                    if (KV) vout[o] = v[r];
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace s512
