// s512_common.cuh -- key codecs, device utilities and error reporting shared by
// every kernel of libsort512cuda.
//
// All kernels sort unsigned integer keys ascending:
//   int32            -> uint32  k = x ^ 0x80000000            (signed order)
//   double           -> uint64  k = x<0 ? ~bits : bits|2^63    (IEEE total order;
//                                -0 sorts before +0, NaNs at the ends by sign)
//   int key + int value (two arrays) -> uint64 k = (ukey << 32) | uvalue
// The transform is applied where a kernel reads the caller's layout and undone
// where it writes the caller's layout; every buffer in between holds encoded
// keys.  The reference compares the same values with signed/ordered compares
// (sort512.hpp:5762 int, 5854 double), so for int and finite double inputs the
// sorted order is the same.
#pragma once

#include <cuda_runtime.h>
#include <cuda/atomic>
#include <stdint.h>

namespace s512 {

// ---------------------------------------------------------------------------
// status / error word written by kernels (never trap)
enum : uint32_t {
    DEV_ERR_NONE = 0,
    DEV_ERR_TIMEOUT = 1u << 0,   // a bounded spin gave up (lookback, queue)
    DEV_ERR_OVERFLOW = 1u << 1,  // a bucket outgrew its sample-based capacity
    DEV_ERR_BOUNDS = 1u << 2,    // a checked index fell outside its buffer
    DEV_ERR_CAPACITY = 1u << 3,  // a work item is larger than its kernel class
};

// Iteration cap for every spin on a flag another block writes.  With
// __nanosleep backoff this is well above any legitimate wait (a predecessor
// tile takes microseconds) and well below a second.
constexpr uint32_t SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ void raise_error(uint32_t* err, uint32_t code) {
    if (err) atomicOr(err, code);
}

// ---------------------------------------------------------------------------
// key traits
template <typename K> struct KeyMax;
template <> struct KeyMax<uint32_t> { static constexpr uint32_t value = 0xFFFFFFFFu; };
template <> struct KeyMax<uint64_t> { static constexpr uint64_t value = ~0ull; };

__device__ __forceinline__ uint32_t enc_i32(int x) { return (uint32_t)x ^ 0x80000000u; }
__device__ __forceinline__ int dec_i32(uint32_t k) { return (int)(k ^ 0x80000000u); }

__device__ __forceinline__ uint64_t enc_f64_bits(uint64_t u) {
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ uint64_t dec_f64_bits(uint64_t k) {
    return (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
}

// key in the high half, value in the low half, both in signed order, so that
// pairs sort by (key, value) in lexicographic order
__device__ __forceinline__ uint64_t enc_kv(int key, int val) {
    return ((uint64_t)enc_i32(key) << 32) | enc_i32(val);
}

// ---------------------------------------------------------------------------
// Codecs: how a kernel reads / writes the caller's layout.
//   load(i)      -> encoded key of element i of the source
//   store(i, k)  -> write encoded key k as element i of the destination
// `Raw` is the identity codec used on the library's own scratch buffers.

// Besides load/store, every input codec describes its raw arrays (NARR
// arrays of ESZ-byte elements, arr(k)) and decodes element i of a tile that a
// bulk copy placed in shared memory (array k of the tile at buf + k*tile*ESZ).
template <typename K>
struct Raw {
    using Key = K;
    static constexpr int NARR = 1;
    static constexpr int ESZ = sizeof(K);
    const K* __restrict__ in;
    K* __restrict__ out;
    __device__ __forceinline__ K load(size_t i) const { return __ldg(in + i); }
    __device__ __forceinline__ void store(size_t i, K k) const { out[i] = k; }
    __host__ __device__ const void* arr(int) const { return in; }
    // the same codec reading other arrays (e.g. the caller's page-locked host memory)
    Raw rebased(const void* const* a) const { return Raw{static_cast<const K*>(a[0]), out}; }
    __device__ __forceinline__ K decode(const unsigned char* buf, uint32_t i, uint32_t) const {
        return reinterpret_cast<const K*>(buf)[i];
    }
};

struct CodecI32 {
    using Key = uint32_t;
    static constexpr int NARR = 1;
    static constexpr int ESZ = 4;
    const int* __restrict__ in;
    int* __restrict__ out;
    __device__ __forceinline__ uint32_t load(size_t i) const { return enc_i32(__ldg(in + i)); }
    __device__ __forceinline__ void store(size_t i, uint32_t k) const { out[i] = dec_i32(k); }
    __host__ __device__ const void* arr(int) const { return in; }
    CodecI32 rebased(const void* const* a) const { return CodecI32{static_cast<const int*>(a[0]), out}; }
    __device__ __forceinline__ uint32_t decode(const unsigned char* buf, uint32_t i, uint32_t) const {
        return enc_i32(reinterpret_cast<const int*>(buf)[i]);
    }
};

struct CodecF64 {
    using Key = uint64_t;
    static constexpr int NARR = 1;
    static constexpr int ESZ = 8;
    const unsigned long long* __restrict__ in;
    unsigned long long* __restrict__ out;
    __device__ __forceinline__ uint64_t load(size_t i) const { return enc_f64_bits(__ldg(in + i)); }
    __device__ __forceinline__ void store(size_t i, uint64_t k) const { out[i] = dec_f64_bits(k); }
    __host__ __device__ const void* arr(int) const { return in; }
    CodecF64 rebased(const void* const* a) const {
        return CodecF64{static_cast<const unsigned long long*>(a[0]), out};
    }
    __device__ __forceinline__ uint64_t decode(const unsigned char* buf, uint32_t i, uint32_t) const {
        return enc_f64_bits(reinterpret_cast<const unsigned long long*>(buf)[i]);
    }
};

struct CodecKV {
    using Key = uint64_t;
    static constexpr int NARR = 2;
    static constexpr int ESZ = 4;
    const int* __restrict__ kin;
    const int* __restrict__ vin;
    int* __restrict__ kout;
    int* __restrict__ vout;
    __host__ __device__ const void* arr(int k) const { return k ? (const void*)vin : (const void*)kin; }
    CodecKV rebased(const void* const* a) const {
        return CodecKV{static_cast<const int*>(a[0]), static_cast<const int*>(a[1]), kout, vout};
    }
    __device__ __forceinline__ uint64_t decode(const unsigned char* buf, uint32_t i, uint32_t tile) const {
        return enc_kv(reinterpret_cast<const int*>(buf)[i], reinterpret_cast<const int*>(buf + (size_t)tile * 4)[i]);
    }
    __device__ __forceinline__ uint64_t load(size_t i) const { return enc_kv(__ldg(kin + i), __ldg(vin + i)); }
    __device__ __forceinline__ void store(size_t i, uint64_t k) const {
        kout[i] = dec_i32((uint32_t)(k >> 32));
        vout[i] = dec_i32((uint32_t)k);
    }
};

// int64 keys: uint64 k = x ^ 2^63 (signed order).
struct CodecI64 {
    using Key = uint64_t;
    static constexpr int NARR = 1;
    static constexpr int ESZ = 8;
    const unsigned long long* __restrict__ in;
    unsigned long long* __restrict__ out;
    __device__ __forceinline__ uint64_t load(size_t i) const { return __ldg(in + i) ^ 0x8000000000000000ull; }
    __device__ __forceinline__ void store(size_t i, uint64_t k) const { out[i] = k ^ 0x8000000000000000ull; }
    __host__ __device__ const void* arr(int) const { return in; }
    CodecI64 rebased(const void* const* a) const {
        return CodecI64{static_cast<const unsigned long long*>(a[0]), out};
    }
    __device__ __forceinline__ uint64_t decode(const unsigned char* buf, uint32_t i, uint32_t) const {
        return reinterpret_cast<const unsigned long long*>(buf)[i] ^ 0x8000000000000000ull;
    }
};

// int key + int value interleaved as pairs (int[2]: key first): one 64-bit
// word per pair (little-endian: key in the low half), encoded like CodecKV.
struct CodecKVPairs {
    using Key = uint64_t;
    static constexpr int NARR = 1;
    static constexpr int ESZ = 8;
    const unsigned long long* __restrict__ in;
    unsigned long long* __restrict__ out;
    static __device__ __forceinline__ uint64_t enc(unsigned long long w) {
        return enc_kv((int)(uint32_t)w, (int)(uint32_t)(w >> 32));
    }
    __device__ __forceinline__ uint64_t load(size_t i) const { return enc(__ldg(in + i)); }
    __device__ __forceinline__ void store(size_t i, uint64_t k) const {
        const uint32_t key = (uint32_t)dec_i32((uint32_t)(k >> 32));
        const uint32_t val = (uint32_t)dec_i32((uint32_t)k);
        out[i] = ((unsigned long long)val << 32) | key;
    }
    __host__ __device__ const void* arr(int) const { return in; }
    CodecKVPairs rebased(const void* const* a) const {
        return CodecKVPairs{static_cast<const unsigned long long*>(a[0]), out};
    }
    __device__ __forceinline__ uint64_t decode(const unsigned char* buf, uint32_t i, uint32_t) const {
        return enc(reinterpret_cast<const unsigned long long*>(buf)[i]);
    }
};

// Codec that reads the library's encoded scratch and writes the caller's layout.
template <typename K, typename OutCodec>
struct RawToUser {
    using Key = K;
    const K* __restrict__ in;
    OutCodec oc;
    __device__ __forceinline__ K load(size_t i) const { return __ldg(in + i); }
    __device__ __forceinline__ void store(size_t i, K k) const { oc.store(i, k); }
};

// ---------------------------------------------------------------------------
// small device helpers

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int mask) {
    return __shfl_xor_sync(0xFFFFFFFFu, v, mask);
}
template <>
__device__ __forceinline__ uint64_t shfl_xor<uint64_t>(uint64_t v, int mask) {
    uint32_t lo = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)v, mask);
    uint32_t hi = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)(v >> 32), mask);
    return ((uint64_t)hi << 32) | lo;
}

template <typename T>
__device__ __forceinline__ T kmin(T a, T b) { return a < b ? a : b; }
template <typename T>
__device__ __forceinline__ T kmax(T a, T b) { return a < b ? b : a; }

// compare-exchange: a <- min, b <- max (one comparison, two selects)
template <typename T>
__device__ __forceinline__ void cas(T& a, T& b) {
    const bool sw = b < a;
    const T lo = sw ? b : a;
    const T hi = sw ? a : b;
    a = lo;
    b = hi;
}

// One side of a comparator whose other key y lives in another lane: the lower
// side keeps the minimum, the upper side the maximum.
template <typename T>
__device__ __forceinline__ T keep_side(T x, T y, bool upper) {
    return ((y < x) != upper) ? y : x;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// 64-bit device-scope loads / stores of look-back status words.  A status
// word carries its flag and its count together, and nothing else is read
// through it, so relaxed atomics suffice; acquire loads would also serialise
// the look-back window's loads behind one another.
__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*const_cast<unsigned long long*>(p));
    return r.load(cuda::memory_order_relaxed);
}
__device__ __forceinline__ void st_status(unsigned long long* p, unsigned long long v) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_relaxed);
}

// ---------------------------------------------------------------------------
// 1-D bulk copies (TMA, no multicast) completing on a CTA mbarrier

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// order earlier generic-proxy accesses of shared memory before later
// async-proxy (bulk copy) writes to it
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// dst, src 16-byte aligned; bytes a positive multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// try_wait that suspends the thread in hardware until the phase completes or
// `ns` nanoseconds pass (instead of returning at once): a waiting warp takes
// no issue slots from the other warps of the SM
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t phase, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase), "r"(ns)
        : "memory");
    return ok != 0;
}
// Iterations of a suspending wait: at most about a second in all.
constexpr uint32_t SUSPEND_NS = 1000;
constexpr uint32_t SUSPEND_LIMIT = 1u << 20;

// bounded wait for a phase of an mbarrier; false if the limit was reached
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
    for (uint32_t i = 0; i < SUSPEND_LIMIT; ++i)
        if (mbar_try_wait_suspend(bar, phase, SUSPEND_NS)) return true;
    return false;
}

// splitmix64 finaliser: counter-based hashing for sample positions
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Block-wide exclusive scan of one value per thread for the first N threads
// (N <= blockDim.x, N multiple of 32).  `warp_tot` needs N/32 entries.
template <int N, typename T>
__device__ __forceinline__ T block_exclusive_scan_first(T v, T* warp_tot, T* total) {
    const unsigned lane = lane_id();
    const unsigned warp = threadIdx.x >> 5;
    T inc = v;
    if (threadIdx.x < N) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
            if (lane >= (unsigned)d) inc += o;
        }
        if (lane == 31) warp_tot[warp] = inc;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        T w = (threadIdx.x < (unsigned)(N / 32)) ? warp_tot[threadIdx.x] : T(0);
        T wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T o = __shfl_up_sync(0xFFFFFFFFu, wi, d);
            if (threadIdx.x >= (unsigned)d) wi += o;
        }
        if (threadIdx.x < (unsigned)(N / 32)) warp_tot[threadIdx.x] = wi - w;
        if (threadIdx.x == (unsigned)(N / 32 - 1) && total) *total = wi;
    }
    __syncthreads();
    T r = T(0);
    if (threadIdx.x < N) r = warp_tot[warp] + inc - v;
    return r;
}

}  // namespace s512
