/*
 * sort512cuda.h -- C ABI of libsort512cuda, a B200 (sm_100a) implementation of
 * the sorting path of berenger-eu/avx-512-sort.
 *
 * Plain pointers and sizes only.  Every function returns an int status
 * (S512_OK == 0).  Pointers may be host or device memory: with S512_PTR_AUTO
 * (the default) the library asks the CUDA driver which one it is; host data is
 * copied to the device, sorted there and copied back.  Device data is sorted
 * in place on `stream` (a cudaStream_t, NULL = the default stream).  A call
 * waits for its result unless S512_ASYNC is set; with S512_ASYNC, device data
 * and page-locked host data (cudaHostAlloc / cudaHostRegister) are ready once
 * the stream has finished, pageable host data is always waited for.  A sort
 * of large page-locked host arrays copies them in by chunks on a second
 * stream and starts partitioning each chunk as it lands.
 *
 * Every operation is in place, like the reference.  Scratch memory comes from
 * one pool per (device, stream) that grows on demand and is kept until
 * s512_release_scratch() or process exit (the page-locked host staging array
 * of a streamed sort, below, too); calls on different streams use different
 * pools, so they may overlap on the device.
 *
 * Element types: int32 ("i32"), double ("f64") and int32 key + int32 value
 * pairs held in two arrays ("kv_i32").  Results:
 *   - i32: the sorted array (bit-exact with the reference's Sort);
 *   - f64: sorted by IEEE total order (-0.0 before +0.0, NaNs at the ends by
 *     sign bit); for finite inputs this is bit-exact with the reference
 *     except for the relative order of -0.0 and +0.0, which the reference
 *     leaves to min/max operand order;
 *   - kv: keys bit-exact, pairs ordered by (key, value).  The reference is
 *     not stable, so only the (key, value) multiset is comparable.
 */
#ifndef SORT512CUDA_H
#define SORT512CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define S512_API __attribute__((visibility("default")))
#else
#define S512_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    S512_OK = 0,
    S512_ERR_ARG = 1,         /* bad argument (null pointer with n > 0, left > right, ...) */
    S512_ERR_ALLOC = 2,       /* device or pinned allocation failed */
    S512_ERR_TIMEOUT = 3,     /* a bounded device-side wait gave up (look-back spin, bulk copy) */
    S512_ERR_CUDA = 4,        /* a CUDA runtime call failed; see s512_last_error_string() */
    S512_ERR_INTERNAL = 5,    /* an internal capacity check failed */
    S512_ERR_UNSUPPORTED = 6  /* no usable sm_100 device */
};

/* flags (bitwise or) */
enum {
    S512_PTR_AUTO = 0,        /* ask the driver whether pointers are host or device memory */
    S512_PTR_HOST = 1,        /* pointers are host memory (pageable or pinned) */
    S512_PTR_DEVICE = 2,      /* pointers are device memory */
    S512_SPLIT_AUTO = 0,      /* splitter mode from s512_config (default: plain) */
    S512_SPLIT_PLAIN = 4,     /* sampled splitters + binary search */
    S512_SPLIT_LEARNED = 8,   /* learned monotone CDF model, plain splitters as fallback */
    S512_ASYNC = 16           /* device or page-locked host data: return without waiting for the stream */
};

/* library configuration (process wide) */
typedef struct s512_config {
    int splitter_mode;        /* S512_SPLIT_PLAIN (default) or S512_SPLIT_LEARNED */
    int collect_stats;        /* 1: time every phase with CUDA events (s512_get_stats) */
    double max_imbalance;     /* learned model is rejected if max bucket > this x mean (default 3.0) */
    uint64_t seed;            /* sampling seed (default 0x5EED) */
    int fault_inject;         /* testing only: S512_FAULT_* bits, 0 in normal use */
    uint64_t device_budget;   /* host-pointer sorts: device bytes one call may use (0: 80% of the free
                                 memory); a host array larger than the budget allows is sorted in
                                 pieces streamed through the device (s512_sort_* below) */
} s512_config;

/* Failure injection (tests of the library's own error paths; 0 by default).
 * OVERFLOW shrinks the first level's bucket capacities so the partition pass
 * overflows and the level is redone with exact counts; REJECT_MODEL rejects
 * every learned model so the splitters route every level; ALLOC makes scratch
 * allocation fail; TIMEOUT makes one tile of the first partition level (or of
 * Partition512) wait on a device flag that is never set, with a short bound,
 * so the call returns S512_ERR_TIMEOUT while the device stays usable. */
enum {
    S512_FAULT_OVERFLOW = 1,
    S512_FAULT_REJECT_MODEL = 2,
    S512_FAULT_ALLOC = 4,
    S512_FAULT_TIMEOUT = 8
};

/* per-call statistics of the last call on this host thread */
#define S512_MAX_LEVELS 8
typedef struct s512_stats {
    double total_ms;                        /* device time of the whole call */
    double sample_ms[S512_MAX_LEVELS];      /* sampling + sample sort + splitters/model, per level */
    double partition_ms[S512_MAX_LEVELS];   /* the multi-way partition kernel, per level */
    double leaf_ms[S512_MAX_LEVELS];        /* planning + leaf sorts, per level */
    uint64_t partition_keys[S512_MAX_LEVELS]; /* keys moved by the partition kernel, per level */
    uint32_t partition_launches[S512_MAX_LEVELS];
    uint32_t levels;                        /* partition levels run */
    uint32_t fallbacks;                     /* levels redone with exact counts after an overflow */
    uint32_t learned_levels;                /* levels routed by the learned model */
    uint32_t learned_rejected;              /* learned models rejected (imbalance / overflow) */
    double max_bucket_over_mean[S512_MAX_LEVELS]; /* bucket imbalance per level */
    uint32_t kernel_launches;               /* kernels launched by the call */
    uint32_t key_bytes;                     /* 4 or 8 */
    double bucket_cv[S512_MAX_LEVELS];      /* std / mean of the non-empty bucket sizes, per level */
    double fit_ms[S512_MAX_LEVELS];         /* learned model fit (part of sample_ms), per level */
    uint32_t learned_segments[S512_MAX_LEVELS]; /* segments routed by their learned model, per level */
    uint32_t learned_fitted[S512_MAX_LEVELS];   /* segments whose model was trained, per level */
    double model_max_over_mean[S512_MAX_LEVELS]; /* worst sample imbalance of a trained model, per level */
} s512_stats;

/* --- configuration, errors, resources ---------------------------------- */
S512_API int s512_set_config(const s512_config* cfg);
S512_API int s512_get_config(s512_config* cfg);
S512_API int s512_get_stats(s512_stats* out);
S512_API const char* s512_last_error_string(void);
S512_API int s512_release_scratch(void);
S512_API int s512_version(void);

/* --- Sort512::Sort<T,IndexType>(T array[], IndexType size)   sort512.hpp:5960-5964
 *     Sort512::SortOmpPartition (sort512.hpp:5993-6004) maps here as well:
 *     on the GPU the parallel backend is the device itself. */
S512_API int s512_sort_i32(int* data, size_t n, int flags, void* stream);
S512_API int s512_sort_f64(double* data, size_t n, int flags, void* stream);

/* --- Sort512kv::Sort<T,IndexType>(T keys[], T values[], IndexType size)
 *     sort512kv.hpp:6132-6136 (and SortOmpPartition, sort512kv.hpp:6165) */
S512_API int s512_sort_kv_i32(int* keys, int* values, size_t n, int flags, void* stream);

/* --- 64-bit words the reference names but does not implement:
 *     int key/value pairs stored interleaved, pairs[2i] = key, pairs[2i+1] =
 *     value (the "int[2]" of the reference's README.md:6; its kv interface,
 *     Sort512kv::Sort at sort512kv.hpp:6133-6163, takes two arrays), sorted by
 *     (key, value); and int64 keys (no counterpart in the reference, which
 *     sorts int and double only).  Same pipeline and flags as above. */
S512_API int s512_sort_kv_pairs_i32(int* pairs, size_t n, int flags, void* stream);
S512_API int s512_sort_i64(long long* data, size_t n, int flags, void* stream);

/* --- Sort512::Partition512<IndexType>(array, left, right, pivot)
 *     int sort512.hpp:5729-5819, double 5821-5912; kv sort512kv.hpp:5959-6082.
 *     Inclusive range [left, right]; elements <= pivot first.  *boundary
 *     receives the index of the first element > pivot (right+1 if none). */
S512_API int s512_partition_i32(int* data, size_t left, size_t right, int pivot, size_t* boundary,
                       int flags, void* stream);
S512_API int s512_partition_f64(double* data, size_t left, size_t right, double pivot, size_t* boundary,
                       int flags, void* stream);
S512_API int s512_partition_kv_i32(int* keys, int* values, size_t left, size_t right, int pivot,
                          size_t* boundary, int flags, void* stream);

/* --- Sort512::SmallSort16V(ptr, length)   int sort512.hpp:5312, double 2255
 *     Sort512kv::SmallSort16V(keys, values, length)   sort512kv.hpp:5235
 *     Lengths up to 16 vectors (256 int / 128 double / 256 pairs) run as one
 *     warp; longer arrays (undefined in the reference) are fully sorted. */
S512_API int s512_smallsort_i32(int* data, size_t len, int flags, void* stream);
S512_API int s512_smallsort_f64(double* data, size_t len, int flags, void* stream);
S512_API int s512_smallsort_kv_i32(int* keys, int* values, size_t len, int flags, void* stream);

/* --- Sort512::CoreSmallSort / CoreSmallSort2..16 pointer forms
 *     (sort512.hpp:95-97, 212, 282, ... 2211 double; 2722-2724 ... 5230 int;
 *     sort512kv.hpp:179, 497, ... 5164): sort nvec consecutive vectors
 *     (16 ints / 8 doubles / 16 pairs each), nvec in 1..16. */
S512_API int s512_core_small_sort_i32(int* data, int nvec, int flags, void* stream);
S512_API int s512_core_small_sort_f64(double* data, int nvec, int flags, void* stream);
S512_API int s512_core_small_sort_kv_i32(int* keys, int* values, int nvec, int flags, void* stream);

/* --- Merge two sorted runs in place: data[0, middle) and data[middle, n).
 *     ParallelInplace::parallelMergeInPlace (parallelInplace.hpp:210-306) and
 *     std::inplace_merge as called by SortOmpMerge (sort512.hpp:6045).
 *     Stable: on equal keys the left run's element comes first. */
S512_API int s512_merge_i32(int* data, size_t n, size_t middle, int flags, void* stream);
S512_API int s512_merge_f64(double* data, size_t n, size_t middle, int flags, void* stream);

/* --- Sort512::SortOmpMerge / SortOmpMergeDeps / SortOmpParMerge
 *     (sort512.hpp:6006-6058, 6060-6102, 6104-6174): sort nparts chunks of
 *     ceil(n/nparts) keys each, then merge neighbouring runs level by level
 *     with merge-path merges.  Any nparts >= 1 (the reference needs a power
 *     of two <= 128). */
S512_API int s512_sort_omp_merge_i32(int* data, size_t n, int nparts, int flags, void* stream);
S512_API int s512_sort_omp_merge_f64(double* data, size_t n, int nparts, int flags, void* stream);

/* --- Batched segmented sort: segment s is data[offsets[s], offsets[s+1]),
 *     nseg segments, offsets has nseg+1 entries (host or device memory; host
 *     data needs host offsets).  Every segment is sorted in place.  The
 *     reference's analogue is a loop of SmallSort16V / Sort over independent
 *     arrays (sort512perf.cpp:612-709, timeSmall).  Segments of up to 256
 *     keys are sorted one per warp, longer ones one per block of the smallest
 *     size class that holds them (1K, 2K, 4K, 8K, 16K keys), one persistent
 *     launch per class; longer ones run the partition levels, on a helper
 *     stream beside the class launches (the call's stream waits for them). */
S512_API int s512_segsort_i32(int* data, const size_t* offsets, size_t nseg, int flags, void* stream);
S512_API int s512_segsort_f64(double* data, const size_t* offsets, size_t nseg, int flags, void* stream);
S512_API int s512_segsort_kv_i32(int* keys, int* values, const size_t* offsets, size_t nseg, int flags,
                                 void* stream);

/* Element types of the plan / tuning calls. */
enum { S512_DTYPE_I32 = 0, S512_DTYPE_F64 = 1, S512_DTYPE_KV_I32 = 2 };

/* Pick the largest block class used (shape 0..3: 2K, 4K, 8K or 16K keys;
 * longer segments run the partition levels) for a dtype by timing every
 * candidate on random keys with this segment layout (device offsets).  The
 * choice is kept for the process and, when the
 * environment variable S512_TUNE_CACHE names a file, appended to it and read
 * back by later processes. */
S512_API int s512_segsort_tune(int dtype, const size_t* d_offsets, size_t nseg, double* best_ms, int* shape_index,
                               void* stream);

/* A segmented sort captured in a CUDA graph for repeated use on the same
 * device buffers and layout: classification happens once at creation; each
 * launch replays the captured class launches and, beside them on a helper
 * stream, runs the partition levels for segments longer than the largest
 * class (not captured: their level structure depends on the data; the launch
 * stream waits for them).  values is used by S512_DTYPE_KV_I32 only. */
typedef struct s512_segsort_plan s512_segsort_plan;
S512_API int s512_segsort_plan_create(s512_segsort_plan** plan, int dtype, void* keys, void* values,
                                      const size_t* d_offsets, size_t nseg, void* stream);
S512_API int s512_segsort_plan_launch(s512_segsort_plan* plan, void* stream);
S512_API int s512_segsort_plan_destroy(s512_segsort_plan* plan);

/* --- Learned splitters (no counterpart in the reference; S512_SPLIT_LEARNED).
 *     Checking entry points of the model.  Keys are "encoded" keys: uint32
 *     (int32 ^ 0x80000000) or uint64 (IEEE total-order bits of a double, or
 *     (key,value) packed), ascending, in device memory.
 *     s512_learned_root_grad: loss and dL/dtheta of the root piecewise-linear
 *     CDF (256 pieces, slopes theta^2) for the given theta (host, 256 floats).
 *     s512_learned_fit: fit the whole model to a sorted sample of a segment of
 *     seg_count keys, as a partition level does (m must be the sample size the
 *     library draws for that segment); optional per-bucket sample histogram. */
#define S512_LEARNED_ROOT_PIECES 256
typedef struct s512_learned_report {
    float loss_init;      /* root loss at its histogram initialisation */
    float loss_root;      /* root loss after training */
    float loss_final;     /* loss of root + leaves */
    float max_over_mean;  /* largest bucket / mean bucket, sample counts (equal buckets aside) */
    uint32_t nbuckets, nmodel;
    uint32_t ok;          /* the model would route the segment: balanced, and the plain splitter table
                             would search for many keys (clustered keys) */
    uint32_t balanced;    /* max_over_mean within s512_config.max_imbalance */
} s512_learned_report;
S512_API int s512_learned_root_grad(int key_bytes, const void* d_sorted_keys, uint32_t m, const float* theta,
                                    float* loss, float* grad, void* stream);
S512_API int s512_learned_fit(int key_bytes, const void* d_sorted_keys, uint32_t m, uint64_t seg_count,
                              uint32_t* d_bucket_hist, s512_learned_report* report, void* stream);

/* --- Sort512::popcount(__mmask16)   sort512.hpp:5714-5725 */
S512_API int s512_popcount(unsigned mask);

/* --- No counterpart in the reference.  Partition512 on int32 device data for
 *     callers that must not allocate (a framework's allocator owns all device
 *     memory, a real-time host forbids allocations after start-up, ...):
 *     same kernel and result as s512_partition_i32 with S512_PTR_DEVICE, but
 *     its scratch is a fixed device array of S512_NOALLOC_MAX_ELEMS ints plus
 *     a few KB, held by every GPU that loads the library until exit.  Larger
 *     ranges return S512_ERR_ARG, and so does data that is not memory of the
 *     current device (managed memory is accepted).  The first call on a
 *     device does the set-up: it looks up that array, and since CUDA loads
 *     modules lazily by default, the driver reserves the array's memory then.
 *     Make that first call at start-up, before another allocator owns the
 *     device's memory and before any stream capture; a call with an empty
 *     range (right < left) does only the set-up.  Calls that overlap on the
 *     GPU share the array and race.  Waits for the result; on an error the
 *     caller's data is left as it was. */
#define S512_NOALLOC_MAX_ELEMS (1u << 20)
S512_API int s512_partition_i32_noalloc(int* data, size_t left, size_t right, int pivot, size_t* boundary,
                                        void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SORT512CUDA_H */
