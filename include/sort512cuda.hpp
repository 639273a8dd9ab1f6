// sort512cuda.hpp -- drop-in replacement for the sorting API of
// berenger-eu/avx-512-sort (sort512.hpp, sort512kv.hpp), backed by the B200
// library libsort512cuda (C ABI: sort512cuda.h).
//
// The function names, template parameters and argument meaning are the
// reference's.  Swapping `#include "sort512.hpp"` for
// `#include "sort512cuda.hpp"` and linking -lsort512cuda is the whole change.
//
//   Sort512::Sort<T,IndexType>(T array[], IndexType size)          sort512.hpp:5960
//   Sort512::SortOmpPartition / SortOmpMerge / SortOmpMergeDeps /
//            SortOmpParMerge<T,IndexType>(T array[], IndexType size) 5993/6007/6061/6105
//   Sort512::Partition512<IndexType>(int|double array[], left, right, pivot) 5730/5822
//   Sort512::SmallSort16V(int*|double*, size_t length)               5312/2255
//   Sort512::CoreSmallSort, CoreSmallSort2..16 (pointer forms)
//   Sort512::popcount(mask)                                          5714
//   ParallelInplace::parallelMergeInPlace(array, size, center)       parallelInplace.hpp:210
//   Sort512kv::Sort / SortOmpPartition<T,IndexType>(T keys[], T values[], IndexType size)  sort512kv.hpp:6133/6165
//   Sort512kv::Partition512<IndexType>(int keys[], int values[], left, right, pivot)       5960
//   Sort512kv::SmallSort16V(int*, int*, size_t)                                            5235
//   Sort512kv::CoreSmallSort, CoreSmallSort2..16(int* keys, int* values)
//
// Pointers may be host or device memory (the library asks the driver).  Extra
// overloads take a Sort512::DevicePtr<T> and a stream for asynchronous device
// use.  Where the reference is undefined (size 0, lengths over 16 vectors,
// thread counts that are not powers of two) these functions are defined:
// size 0 is a no-op and any length is sorted.  A failure of the device or of
// an allocation throws Sort512::Error (the reference has no error path).
// SortOmpPartition runs the partition sort; SortOmpMerge/MergeDeps/ParMerge
// keep the reference's method (chunk sorts, then a merge tree) with
// merge-path merges; all return the same sorted array.
#ifndef SORT512CUDA_HPP
#define SORT512CUDA_HPP

#include <cstddef>
#include <stdexcept>
#include <string>

#include "sort512cuda.h"

#ifndef __CUDA_RUNTIME_H__
typedef struct CUstream_st* cudaStream_t;
#endif

namespace Sort512 {

class Error : public std::runtime_error {
  public:
    Error(const char* fn, int code)
        : std::runtime_error(std::string(fn) + " failed (status " + std::to_string(code) +
                             "): " + s512_last_error_string()),
          code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

namespace detail {
inline void check(const char* fn, int rc) {
    if (rc != S512_OK) throw Error(fn, rc);
}
inline int call(int* a, size_t n, int flags, void* st) { return s512_sort_i32(a, n, flags, st); }
inline int call(double* a, size_t n, int flags, void* st) { return s512_sort_f64(a, n, flags, st); }
// 64-bit integer keys (an extension: the reference sorts int and double)
inline int call(long long* a, size_t n, int flags, void* st) { return s512_sort_i64(a, n, flags, st); }
inline int call(long* a, size_t n, int flags, void* st) {
    static_assert(sizeof(long) == sizeof(long long), "64-bit long expected");
    return s512_sort_i64(reinterpret_cast<long long*>(a), n, flags, st);
}
}  // namespace detail

// Tag for explicit device pointers (no pointer probe, optional async stream).
template <class T>
struct DevicePtr {
    T* ptr;
    explicit DevicePtr(T* p) : ptr(p) {}
};

template <class SortType, class IndexType = size_t>
inline void Sort(SortType array[], const IndexType size) {
    detail::check("Sort512::Sort", detail::call(array, (size_t)size, S512_PTR_AUTO, nullptr));
}

template <class SortType, class IndexType = size_t>
inline void Sort(DevicePtr<SortType> array, const IndexType size, cudaStream_t stream = nullptr,
                 bool async = false) {
    detail::check("Sort512::Sort",
                  detail::call(array.ptr, (size_t)size, S512_PTR_DEVICE | (async ? S512_ASYNC : 0), stream));
}

template <class SortType, class IndexType = size_t>
inline void SortOmpPartition(SortType array[], const IndexType size) {
    Sort<SortType, IndexType>(array, size);
}
namespace detail {
inline int call_merge_sort(int* a, size_t n, int parts) {
    return s512_sort_omp_merge_i32(a, n, parts, S512_PTR_AUTO, nullptr);
}
inline int call_merge_sort(double* a, size_t n, int parts) {
    return s512_sort_omp_merge_f64(a, n, parts, S512_PTR_AUTO, nullptr);
}
inline int call_merge(int* a, size_t n, size_t mid) { return s512_merge_i32(a, n, mid, S512_PTR_AUTO, nullptr); }
inline int call_merge(double* a, size_t n, size_t mid) { return s512_merge_f64(a, n, mid, S512_PTR_AUTO, nullptr); }
// chunks of the merge-based drivers: the reference uses one per OpenMP thread
constexpr int kMergeParts = 8;
}  // namespace detail

// Chunk sorts followed by a tree of merges, as in the reference; on the GPU
// every merge is a merge-path pass.
template <class SortType, class IndexType = size_t>
inline void SortOmpMerge(SortType array[], const IndexType size) {
    detail::check("Sort512::SortOmpMerge", detail::call_merge_sort(array, (size_t)size, detail::kMergeParts));
}
template <class SortType, class IndexType = size_t>
inline void SortOmpMergeDeps(SortType array[], const IndexType size) {
    detail::check("Sort512::SortOmpMergeDeps", detail::call_merge_sort(array, (size_t)size, detail::kMergeParts));
}
template <class SortType, class IndexType = size_t>
inline void SortOmpParMerge(SortType array[], const IndexType size) {
    detail::check("Sort512::SortOmpParMerge", detail::call_merge_sort(array, (size_t)size, detail::kMergeParts));
}

// The reference's README names SortOmp(); the real symbols are the four above.
template <class SortType, class IndexType = size_t>
inline void SortOmp(SortType array[], const IndexType size) {
    Sort<SortType, IndexType>(array, size);
}

template <class IndexType>
inline IndexType Partition512(int array[], IndexType left, IndexType right, const int pivot) {
    size_t b = 0;
    detail::check("Sort512::Partition512",
                  s512_partition_i32(array, (size_t)left, (size_t)right, pivot, &b, S512_PTR_AUTO, nullptr));
    return (IndexType)b;
}

template <class IndexType>
inline IndexType Partition512(double array[], IndexType left, IndexType right, const double pivot) {
    size_t b = 0;
    detail::check("Sort512::Partition512",
                  s512_partition_f64(array, (size_t)left, (size_t)right, pivot, &b, S512_PTR_AUTO, nullptr));
    return (IndexType)b;
}

inline void SmallSort16V(int* ptr, const size_t length) {
    detail::check("Sort512::SmallSort16V", s512_smallsort_i32(ptr, length, S512_PTR_AUTO, nullptr));
}
inline void SmallSort16V(double* ptr, const size_t length) {
    detail::check("Sort512::SmallSort16V", s512_smallsort_f64(ptr, length, S512_PTR_AUTO, nullptr));
}

inline int popcount(unsigned mask) { return s512_popcount(mask); }

// CoreSmallSortN pointer forms.  The reference takes one pointer per vector;
// the vectors are sorted as one sequence (pointer k holds elements 16k..16k+15
// of the network's input).  Consecutive vectors are the common (and tested)
// case; scattered vectors are gathered on the host.
namespace detail {
template <class T, int S>
inline void core_sort(T* const* ptrs, int nvec) {
    bool contiguous = true;
    for (int i = 1; i < nvec; ++i) contiguous = contiguous && (ptrs[i] == ptrs[0] + i * S);
    if (contiguous) {
        check("Sort512::CoreSmallSort", call(ptrs[0], (size_t)nvec * S, S512_PTR_AUTO, nullptr));
        return;
    }
    T buf[16 * S];
    for (int i = 0; i < nvec; ++i)
        for (int l = 0; l < S; ++l) buf[i * S + l] = ptrs[i][l];
    check("Sort512::CoreSmallSort", call(buf, (size_t)nvec * S, S512_PTR_HOST, nullptr));
    for (int i = 0; i < nvec; ++i)
        for (int l = 0; l < S; ++l) ptrs[i][l] = buf[i * S + l];
}
}  // namespace detail

#define S512_CORE_SMALL_SORT_OVERLOADS(T, S)                                                           \
    inline void CoreSmallSort(T* p1) { T* p[] = {p1}; detail::core_sort<T, S>(p, 1); }                  \
    inline void CoreSmallSort2(T* p1, T* p2) { T* p[] = {p1, p2}; detail::core_sort<T, S>(p, 2); }      \
    inline void CoreSmallSort3(T* p1, T* p2, T* p3) { T* p[] = {p1, p2, p3}; detail::core_sort<T, S>(p, 3); } \
    inline void CoreSmallSort4(T* p1, T* p2, T* p3, T* p4) {                                           \
        T* p[] = {p1, p2, p3, p4}; detail::core_sort<T, S>(p, 4);                                       \
    }                                                                                                   \
    inline void CoreSmallSort5(T* p1, T* p2, T* p3, T* p4, T* p5) {                                    \
        T* p[] = {p1, p2, p3, p4, p5}; detail::core_sort<T, S>(p, 5);                                   \
    }                                                                                                   \
    inline void CoreSmallSort6(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6) {                             \
        T* p[] = {p1, p2, p3, p4, p5, p6}; detail::core_sort<T, S>(p, 6);                               \
    }                                                                                                   \
    inline void CoreSmallSort7(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7) {                      \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7}; detail::core_sort<T, S>(p, 7);                           \
    }                                                                                                   \
    inline void CoreSmallSort8(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8) {               \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8}; detail::core_sort<T, S>(p, 8);                       \
    }                                                                                                   \
    inline void CoreSmallSort9(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9) {        \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9}; detail::core_sort<T, S>(p, 9);                   \
    }                                                                                                   \
    inline void CoreSmallSort10(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10) { \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10}; detail::core_sort<T, S>(p, 10);             \
    }                                                                                                   \
    inline void CoreSmallSort11(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10, \
                                T* p11) {                                                               \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10, p11}; detail::core_sort<T, S>(p, 11);        \
    }                                                                                                   \
    inline void CoreSmallSort12(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10, \
                                T* p11, T* p12) {                                                       \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10, p11, p12}; detail::core_sort<T, S>(p, 12);   \
    }                                                                                                   \
    inline void CoreSmallSort13(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10, \
                                T* p11, T* p12, T* p13) {                                               \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10, p11, p12, p13};                              \
        detail::core_sort<T, S>(p, 13);                                                                 \
    }                                                                                                   \
    inline void CoreSmallSort14(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10, \
                                T* p11, T* p12, T* p13, T* p14) {                                       \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10, p11, p12, p13, p14};                         \
        detail::core_sort<T, S>(p, 14);                                                                 \
    }                                                                                                   \
    inline void CoreSmallSort15(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10, \
                                T* p11, T* p12, T* p13, T* p14, T* p15) {                               \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10, p11, p12, p13, p14, p15};                    \
        detail::core_sort<T, S>(p, 15);                                                                 \
    }                                                                                                   \
    inline void CoreSmallSort16(T* p1, T* p2, T* p3, T* p4, T* p5, T* p6, T* p7, T* p8, T* p9, T* p10, \
                                T* p11, T* p12, T* p13, T* p14, T* p15, T* p16) {                       \
        T* p[] = {p1, p2, p3, p4, p5, p6, p7, p8, p9, p10, p11, p12, p13, p14, p15, p16};               \
        detail::core_sort<T, S>(p, 16);                                                                 \
    }

S512_CORE_SMALL_SORT_OVERLOADS(int, 16)
S512_CORE_SMALL_SORT_OVERLOADS(double, 8)
#undef S512_CORE_SMALL_SORT_OVERLOADS

}  // namespace Sort512

// ParallelInplace::parallelMergeInPlace (parallelInplace.hpp:210): merge the
// sorted runs array[0, centerPosition) and array[centerPosition, sizeArray).
// The OpenMP plumbing arguments of the reference (thread count, first thread,
// interval and barrier arrays) have no meaning on the GPU and are dropped.
namespace ParallelInplace {
template <class NumType>
inline void parallelMergeInPlace(NumType array[], const long sizeArray, const long centerPosition) {
    Sort512::detail::check("ParallelInplace::parallelMergeInPlace",
                           Sort512::detail::call_merge(array, (size_t)sizeArray, (size_t)centerPosition));
}
}  // namespace ParallelInplace

namespace Sort512kv {

using Sort512::DevicePtr;
using Sort512::Error;

template <class SortType, class IndexType = size_t>
inline void Sort(SortType array[], SortType values[], const IndexType size) {
    static_assert(sizeof(SortType) == sizeof(int), "Sort512kv sorts int keys with int values");
    Sort512::detail::check("Sort512kv::Sort",
                           s512_sort_kv_i32((int*)array, (int*)values, (size_t)size, S512_PTR_AUTO, nullptr));
}

template <class SortType, class IndexType = size_t>
inline void Sort(DevicePtr<SortType> array, DevicePtr<SortType> values, const IndexType size,
                 cudaStream_t stream = nullptr, bool async = false) {
    Sort512::detail::check("Sort512kv::Sort",
                           s512_sort_kv_i32((int*)array.ptr, (int*)values.ptr, (size_t)size,
                                            S512_PTR_DEVICE | (async ? S512_ASYNC : 0), stream));
}

template <class SortType, class IndexType = size_t>
inline void SortOmpPartition(SortType array[], SortType values[], const IndexType size) {
    Sort<SortType, IndexType>(array, values, size);
}

// int[2] pairs (key, value) stored interleaved, as the reference's README
// describes its kv sort; sorted by key, then value.
template <class IndexType = size_t>
inline void Sort(int (*pairs)[2], const IndexType size) {
    Sort512::detail::check("Sort512kv::Sort", s512_sort_kv_pairs_i32(&pairs[0][0], (size_t)size, S512_PTR_AUTO, nullptr));
}

template <class IndexType = size_t>
inline void Sort(DevicePtr<int[2]> pairs, const IndexType size, cudaStream_t stream = nullptr, bool async = false) {
    Sort512::detail::check("Sort512kv::Sort",
                           s512_sort_kv_pairs_i32(&pairs.ptr[0][0], (size_t)size,
                                                  S512_PTR_DEVICE | (async ? S512_ASYNC : 0), stream));
}

template <class IndexType>
inline IndexType Partition512(int array[], int values[], IndexType left, IndexType right, const int pivot) {
    size_t b = 0;
    Sort512::detail::check("Sort512kv::Partition512",
                           s512_partition_kv_i32(array, values, (size_t)left, (size_t)right, pivot, &b,
                                                 S512_PTR_AUTO, nullptr));
    return (IndexType)b;
}

inline void SmallSort16V(int* ptr, int* values, const size_t length) {
    Sort512::detail::check("Sort512kv::SmallSort16V",
                           s512_smallsort_kv_i32(ptr, values, length, S512_PTR_AUTO, nullptr));
}

inline int popcount(unsigned mask) { return s512_popcount(mask); }

// kv CoreSmallSortN(int* keys, int* values): N*16 consecutive pairs.
#define S512_KV_CORE(NAME, N)                                                                      \
    inline void NAME(int* keys, int* values) {                                                    \
        Sort512::detail::check("Sort512kv::" #NAME,                                                \
                               s512_core_small_sort_kv_i32(keys, values, N, S512_PTR_AUTO, nullptr)); \
    }
S512_KV_CORE(CoreSmallSort, 1)
S512_KV_CORE(CoreSmallSort2, 2)
S512_KV_CORE(CoreSmallSort3, 3)
S512_KV_CORE(CoreSmallSort4, 4)
S512_KV_CORE(CoreSmallSort5, 5)
S512_KV_CORE(CoreSmallSort6, 6)
S512_KV_CORE(CoreSmallSort7, 7)
S512_KV_CORE(CoreSmallSort8, 8)
S512_KV_CORE(CoreSmallSort9, 9)
S512_KV_CORE(CoreSmallSort10, 10)
S512_KV_CORE(CoreSmallSort11, 11)
S512_KV_CORE(CoreSmallSort12, 12)
S512_KV_CORE(CoreSmallSort13, 13)
S512_KV_CORE(CoreSmallSort14, 14)
S512_KV_CORE(CoreSmallSort15, 15)
S512_KV_CORE(CoreSmallSort16, 16)
#undef S512_KV_CORE

}  // namespace Sort512kv

#endif  // SORT512CUDA_HPP
