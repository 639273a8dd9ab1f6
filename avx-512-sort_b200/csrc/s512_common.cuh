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

template <typename K>
struct Raw {
    using Key = K;
    const K* __restrict__ in;
    K* __restrict__ out;
    __device__ __forceinline__ K load(size_t i) const { return __ldg(in + i); }
    __device__ __forceinline__ void store(size_t i, K k) const { out[i] = k; }
};

struct CodecI32 {
    using Key = uint32_t;
    const int* __restrict__ in;
    int* __restrict__ out;
    __device__ __forceinline__ uint32_t load(size_t i) const { return enc_i32(__ldg(in + i)); }
    __device__ __forceinline__ void store(size_t i, uint32_t k) const { out[i] = dec_i32(k); }
};

struct CodecF64 {
    using Key = uint64_t;
    const unsigned long long* __restrict__ in;
    unsigned long long* __restrict__ out;
    __device__ __forceinline__ uint64_t load(size_t i) const { return enc_f64_bits(__ldg(in + i)); }
    __device__ __forceinline__ void store(size_t i, uint64_t k) const { out[i] = dec_f64_bits(k); }
};

struct CodecKV {
    using Key = uint64_t;
    const int* __restrict__ kin;
    const int* __restrict__ vin;
    int* __restrict__ kout;
    int* __restrict__ vout;
    __device__ __forceinline__ uint64_t load(size_t i) const { return enc_kv(__ldg(kin + i), __ldg(vin + i)); }
    __device__ __forceinline__ void store(size_t i, uint64_t k) const {
        kout[i] = dec_i32((uint32_t)(k >> 32));
        vout[i] = dec_i32((uint32_t)k);
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

// compare-exchange: a <- min, b <- max
template <typename T>
__device__ __forceinline__ void cas(T& a, T& b) {
    T lo = kmin(a, b), hi = kmax(a, b);
    a = lo;
    b = hi;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// 64-bit device-scope acquire / release for the lookback status words
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*const_cast<unsigned long long*>(p));
    return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_release);
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
