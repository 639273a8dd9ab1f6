// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI wrapper around the unmodified reference headers (sort512.hpp,
// sort512kv.hpp, parallelInplace.hpp), compiled from where they lie by
// oracle/Makefile into oracle/_ref/libsort512ref.so.  Used to pin the C
// restatement (sort512_oracle.c) and the golden fixtures, and as the timed CPU
// baseline.  Nothing in the product links it.
//
// Every function forwards to exactly one reference entry point:
//   ref_sort_*                 Sort512::Sort                sort512.hpp:5960
//   ref_sort_omp_partition_*   Sort512::SortOmpPartition    sort512.hpp:5993
//   ref_sort_omp_merge_*       Sort512::SortOmpMerge        sort512.hpp:6007
//   ref_sort_omp_merge_deps_*  Sort512::SortOmpMergeDeps    sort512.hpp:6061
//   ref_sort_omp_parmerge_*    Sort512::SortOmpParMerge     sort512.hpp:6105
//   ref_partition_*            Sort512::Partition512        sort512.hpp:5730 / 5822
//   ref_smallsort_*            Sort512::SmallSort16V        sort512.hpp:5312 / 2255
//   ref_core_small_sort_*      Sort512::CoreSmallSort{,2..16} (pointer forms)
//   ref_*_kv_i32               Sort512kv::{Sort 6133, SortOmpPartition 6165,
//                              Partition512 5960, SmallSort16V 5235,
//                              CoreSmallSort{,2..16} pointer forms}
#include <climits>
#include <cstddef>
#include <limits>
#include <omp.h>

#include "sort512.hpp"
#include "sort512kv.hpp"

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API void ref_set_threads(int n) { omp_set_num_threads(n); }
REF_API int ref_max_threads() { return omp_get_max_threads(); }
REF_API int ref_popcount(unsigned m) { return Sort512::popcount((__mmask16)m); }

REF_API void ref_sort_i32(int* a, size_t n) { Sort512::Sort<int, size_t>(a, n); }
REF_API void ref_sort_f64(double* a, size_t n) { Sort512::Sort<double, size_t>(a, n); }
REF_API void ref_sort_omp_partition_i32(int* a, size_t n) { Sort512::SortOmpPartition<int, size_t>(a, n); }
REF_API void ref_sort_omp_partition_f64(double* a, size_t n) { Sort512::SortOmpPartition<double, size_t>(a, n); }
REF_API void ref_sort_omp_merge_i32(int* a, size_t n) { Sort512::SortOmpMerge<int, size_t>(a, n); }
REF_API void ref_sort_omp_merge_f64(double* a, size_t n) { Sort512::SortOmpMerge<double, size_t>(a, n); }
REF_API void ref_sort_omp_merge_deps_i32(int* a, size_t n) { Sort512::SortOmpMergeDeps<int, size_t>(a, n); }
REF_API void ref_sort_omp_merge_deps_f64(double* a, size_t n) { Sort512::SortOmpMergeDeps<double, size_t>(a, n); }
REF_API void ref_sort_omp_parmerge_i32(int* a, size_t n) { Sort512::SortOmpParMerge<int, size_t>(a, n); }
REF_API void ref_sort_omp_parmerge_f64(double* a, size_t n) { Sort512::SortOmpParMerge<double, size_t>(a, n); }

REF_API size_t ref_partition_i32(int* a, size_t l, size_t r, int pivot) {
    return Sort512::Partition512<size_t>(a, l, r, pivot);
}
REF_API size_t ref_partition_f64(double* a, size_t l, size_t r, double pivot) {
    return Sort512::Partition512<size_t>(a, l, r, pivot);
}
REF_API void ref_smallsort_i32(int* a, size_t n) { Sort512::SmallSort16V(a, n); }
REF_API void ref_smallsort_f64(double* a, size_t n) { Sort512::SmallSort16V(a, n); }

// CoreSmallSortN pointer forms: nvec consecutive vectors starting at p.
REF_API int ref_core_small_sort_i32(int* p, int nvec) {
    const int S = 16;
    switch (nvec) {
    case 1: Sort512::CoreSmallSort(p); break;
    case 2: Sort512::CoreSmallSort2(p, p + S); break;
    case 3: Sort512::CoreSmallSort3(p, p + S, p + 2 * S); break;
    case 4: Sort512::CoreSmallSort4(p, p + S, p + 2 * S, p + 3 * S); break;
    case 5: Sort512::CoreSmallSort5(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S); break;
    case 6: Sort512::CoreSmallSort6(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S); break;
    case 7: Sort512::CoreSmallSort7(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S); break;
    case 8: Sort512::CoreSmallSort8(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S); break;
    case 9: Sort512::CoreSmallSort9(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S); break;
    case 10: Sort512::CoreSmallSort10(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S); break;
    case 11: Sort512::CoreSmallSort11(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S); break;
    case 12: Sort512::CoreSmallSort12(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S); break;
    case 13: Sort512::CoreSmallSort13(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S); break;
    case 14: Sort512::CoreSmallSort14(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S, p + 13 * S); break;
    case 15: Sort512::CoreSmallSort15(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S, p + 13 * S, p + 14 * S); break;
    case 16: Sort512::CoreSmallSort16(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S, p + 13 * S, p + 14 * S, p + 15 * S); break;
    default: return -1;
    }
    return 0;
}

REF_API int ref_core_small_sort_f64(double* p, int nvec) {
    const int S = 8;
    switch (nvec) {
    case 1: Sort512::CoreSmallSort(p); break;
    case 2: Sort512::CoreSmallSort2(p, p + S); break;
    case 3: Sort512::CoreSmallSort3(p, p + S, p + 2 * S); break;
    case 4: Sort512::CoreSmallSort4(p, p + S, p + 2 * S, p + 3 * S); break;
    case 5: Sort512::CoreSmallSort5(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S); break;
    case 6: Sort512::CoreSmallSort6(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S); break;
    case 7: Sort512::CoreSmallSort7(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S); break;
    case 8: Sort512::CoreSmallSort8(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S); break;
    case 9: Sort512::CoreSmallSort9(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S); break;
    case 10: Sort512::CoreSmallSort10(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S); break;
    case 11: Sort512::CoreSmallSort11(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S); break;
    case 12: Sort512::CoreSmallSort12(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S); break;
    case 13: Sort512::CoreSmallSort13(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S); break;
    case 14: Sort512::CoreSmallSort14(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S, p + 13 * S); break;
    case 15: Sort512::CoreSmallSort15(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S, p + 13 * S, p + 14 * S); break;
    case 16: Sort512::CoreSmallSort16(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S, p + 8 * S, p + 9 * S, p + 10 * S, p + 11 * S, p + 12 * S, p + 13 * S, p + 14 * S, p + 15 * S); break;
    default: return -1;
    }
    return 0;
}

REF_API void ref_sort_kv_i32(int* k, int* v, size_t n) { Sort512kv::Sort<int, size_t>(k, v, n); }
REF_API void ref_sort_omp_partition_kv_i32(int* k, int* v, size_t n) {
    Sort512kv::SortOmpPartition<int, size_t>(k, v, n);
}
REF_API size_t ref_partition_kv_i32(int* k, int* v, size_t l, size_t r, int pivot) {
    return Sort512kv::Partition512<size_t>(k, v, l, r, pivot);
}
REF_API void ref_smallsort_kv_i32(int* k, int* v, size_t n) { Sort512kv::SmallSort16V(k, v, n); }

REF_API int ref_core_small_sort_kv_i32(int* k, int* v, int nvec) {
    switch (nvec) {
    case 1: Sort512kv::CoreSmallSort(k, v); break;
    case 2: Sort512kv::CoreSmallSort2(k, v); break;
    case 3: Sort512kv::CoreSmallSort3(k, v); break;
    case 4: Sort512kv::CoreSmallSort4(k, v); break;
    case 5: Sort512kv::CoreSmallSort5(k, v); break;
    case 6: Sort512kv::CoreSmallSort6(k, v); break;
    case 7: Sort512kv::CoreSmallSort7(k, v); break;
    case 8: Sort512kv::CoreSmallSort8(k, v); break;
    case 9: Sort512kv::CoreSmallSort9(k, v); break;
    case 10: Sort512kv::CoreSmallSort10(k, v); break;
    case 11: Sort512kv::CoreSmallSort11(k, v); break;
    case 12: Sort512kv::CoreSmallSort12(k, v); break;
    case 13: Sort512kv::CoreSmallSort13(k, v); break;
    case 14: Sort512kv::CoreSmallSort14(k, v); break;
    case 15: Sort512kv::CoreSmallSort15(k, v); break;
    case 16: Sort512kv::CoreSmallSort16(k, v); break;
    default: return -1;
    }
    return 0;
}
