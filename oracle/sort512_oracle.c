/*
 * sort512_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain, scalar C restatement of the reference's sorting path
 * (berenger-eu/avx-512-sort: sort512.hpp, sort512kv.hpp, parallelInplace.hpp).
 * It exists so that the GPU library can be checked against the reference's
 * algorithm on machines where the reference itself cannot run (no AVX-512).
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
 * it, and only as the checker or the timed CPU baseline; the product path
 * (libsort512cuda) never links or calls it.
 *
 * Each function cites the reference lines it restates.  Where the reference
 * is a vector network (the SmallSort16V bitonic networks), the restatement
 * reproduces the network's *output* (sorted padded vectors, first `len`
 * lanes stored), not the permute sequence: for int and finite double keys the
 * output of any correct network on the same padded input is identical.
 * The key/value leaf is the exception: the reference's kv network is not
 * stable and drops values on INT_MAX keys, so the restatement sorts pairs
 * lexicographically; kv parity is "keys bit-exact, (key,value) multiset
 * equal".  Partition512 IS restated step by step (same pointer walk, same
 * compress order), so its in-place arrangement matches the reference bit for
 * bit -- that is what pins this file against the reference's own outputs.
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* drand48 (the reference tests' generator: createRandVec, sort512test.cpp:77-83,
 * seeded with srand48(0) at e.g. sort512test.cpp:178).  POSIX LCG:
 * X' = (0x5DEECE66D * X + 0xB) mod 2^48; srand48(s) sets X = (s << 16) | 0x330E. */
typedef struct { uint64_t x; } oracle_rng48;

ORACLE_API void oracle_srand48(oracle_rng48* st, long seed) {
    st->x = (((uint64_t)(uint32_t)seed) << 16) | 0x330EULL;
}

static double rng48_next(oracle_rng48* st) {
    st->x = (0x5DEECE66DULL * st->x + 0xBULL) & ((1ULL << 48) - 1);
    return ldexp((double)st->x, -48);
}

ORACLE_API double oracle_drand48(oracle_rng48* st) { return rng48_next(st); }

/* createRandVec<int>: array[i] = int(drand48()*size) (sort512test.cpp:77-83) */
ORACLE_API void oracle_rand_vec_i32(oracle_rng48* st, int* a, size_t n) {
    for (size_t i = 0; i < n; ++i) a[i] = (int)(rng48_next(st) * (double)n);
}

/* createRandVec<double> */
ORACLE_API void oracle_rand_vec_f64(oracle_rng48* st, double* a, size_t n) {
    for (size_t i = 0; i < n; ++i) a[i] = (double)(rng48_next(st) * (double)n);
}

/* ------------------------------------------------------------------------ */
/* popcount (sort512.hpp:5714-5725) */
ORACLE_API int oracle_popcount(unsigned mask) { return __builtin_popcount(mask); }

/* ------------------------------------------------------------------------ */
/* Type-generic pieces are written once per type with a macro so that the int
 * and double paths are literally the same statements, as in the reference
 * (where they are two hand-written copies). */

#define DEFINE_SCALAR_PARTITION(NAME, T)                                       \
    /* CoreScalarPartition (sort512.hpp:5695-5711) */                          \
    static size_t NAME(T* a, size_t left, size_t right, T pivot) {             \
        for (; left <= right && a[left] <= pivot; ++left) {                    \
        }                                                                      \
        for (size_t idx = left; idx <= right; ++idx) {                         \
            if (a[idx] <= pivot) {                                             \
                T t = a[idx]; a[idx] = a[left]; a[left] = t;                   \
                left += 1;                                                     \
            }                                                                  \
        }                                                                      \
        return left;                                                           \
    }

DEFINE_SCALAR_PARTITION(scalar_partition_i32, int)
DEFINE_SCALAR_PARTITION(scalar_partition_f64, double)

/* One masked compress-store pair of Partition512: lanes with val<=pivot go,
 * in lane order, to a[*left_w...]; the others, in lane order, to the block
 * that ends at *right_w (sort512.hpp:5765-5775).  `lanes` limits the lanes
 * considered (the remainder step, 5777-5791). */
#define DEFINE_COMPRESS(NAME, T, S)                                            \
    static void NAME(T* a, const T* val, unsigned lanes, T pivot,              \
                     size_t* left_w, size_t* right_w) {                        \
        unsigned nb_low = 0, nb_high = 0;                                      \
        for (unsigned l = 0; l < lanes; ++l) {                                 \
            if (val[l] <= pivot) nb_low++; else nb_high++;                     \
        }                                                                      \
        size_t lw = *left_w;                                                   \
        size_t rw = *right_w - nb_high;                                        \
        for (unsigned l = 0; l < lanes; ++l) {                                 \
            if (val[l] <= pivot) a[lw++] = val[l];                             \
        }                                                                      \
        size_t hw = rw;                                                        \
        for (unsigned l = 0; l < lanes; ++l) {                                 \
            if (!(val[l] <= pivot)) a[hw++] = val[l];                          \
        }                                                                      \
        *left_w = lw;                                                          \
        *right_w = rw;                                                         \
    }

DEFINE_COMPRESS(compress_i32, int, 16)
DEFINE_COMPRESS(compress_f64, double, 8)

/* Partition512 (int: sort512.hpp:5729-5819, double: 5821-5912).
 * Inclusive [left,right]; returns the first index whose value is > pivot.
 * The vector width S is 16 ints / 8 doubles; ranges shorter than 2S use the
 * scalar partition (5735-5737). */
#define DEFINE_PARTITION(NAME, T, S, SCALAR, COMPRESS)                         \
    ORACLE_API size_t NAME(T* a, size_t left, size_t right, T pivot) {         \
        if (right - left + 1 < 2 * (size_t)(S)) return SCALAR(a, left, right, pivot); \
        T left_val[S], right_val[S], val[S];                                   \
        memcpy(left_val, &a[left], sizeof(left_val));                          \
        size_t left_w = left;                                                  \
        left += (S);                                                           \
        size_t right_w = right + 1;                                            \
        right -= (S) - 1;                                                      \
        memcpy(right_val, &a[right], sizeof(right_val));                        \
        while (left + (S) <= right) {                                          \
            const size_t free_left = left - left_w;                            \
            const size_t free_right = right_w - right;                         \
            if (free_left <= free_right) {                                     \
                memcpy(val, &a[left], sizeof(val));                            \
                left += (S);                                                   \
            } else {                                                           \
                right -= (S);                                                  \
                memcpy(val, &a[right], sizeof(val));                           \
            }                                                                  \
            COMPRESS(a, val, (S), pivot, &left_w, &right_w);                   \
        }                                                                      \
        {                                                                      \
            const size_t remaining = right - left;                             \
            memcpy(val, &a[left], sizeof(val));                                \
            left = right;                                                      \
            COMPRESS(a, val, (unsigned)remaining, pivot, &left_w, &right_w);   \
        }                                                                      \
        COMPRESS(a, left_val, (S), pivot, &left_w, &right_w);                  \
        COMPRESS(a, right_val, (S), pivot, &left_w, &right_w);                 \
        return left_w;                                                         \
    }

DEFINE_PARTITION(oracle_partition_i32, int, 16, scalar_partition_i32, compress_i32)
DEFINE_PARTITION(oracle_partition_f64, double, 8, scalar_partition_f64, compress_f64)

/* ------------------------------------------------------------------------ */
/* SmallSort16V (double: sort512.hpp:2255-2634, int: 5312-5689).
 * nbVecs = ceil(len/S) vectors; the tail vector is padded with INT_MAX /
 * DBL_MAX; the padded vectors go through the bitonic network and the first
 * `len` lanes are stored back.  The restatement sorts the padded buffer with
 * an insertion sort (same output for ints and non-NaN doubles) and stores the
 * first len.  len == 0 is a no-op here (the reference reads 16 vectors). */
static int cmp_i32(const void* x, const void* y) {
    int a = *(const int*)x, b = *(const int*)y;
    return (a > b) - (a < b);
}
static int cmp_f64(const void* x, const void* y) {
    double a = *(const double*)x, b = *(const double*)y;
    return (a > b) - (a < b);
}

ORACLE_API void oracle_smallsort_i32(int* p, size_t len) {
    if (len == 0) return;
    int buf[256];
    const size_t S = 16;
    size_t nb = (len + S - 1) / S;
    if (nb > 16) nb = 16; /* the reference's default branch is 16 vectors */
    size_t padded = nb * S;
    size_t n = len < padded ? len : padded;
    memcpy(buf, p, n * sizeof(int));
    for (size_t i = n; i < padded; ++i) buf[i] = INT_MAX;
    qsort(buf, padded, sizeof(int), cmp_i32);
    memcpy(p, buf, n * sizeof(int));
}

ORACLE_API void oracle_smallsort_f64(double* p, size_t len) {
    if (len == 0) return;
    double buf[128];
    const size_t S = 8;
    size_t nb = (len + S - 1) / S;
    if (nb > 16) nb = 16;
    size_t padded = nb * S;
    size_t n = len < padded ? len : padded;
    memcpy(buf, p, n * sizeof(double));
    for (size_t i = n; i < padded; ++i) buf[i] = DBL_MAX;
    qsort(buf, padded, sizeof(double), cmp_f64);
    memcpy(p, buf, n * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* Quicksort driver: CoreSortGetPivot (sort512.hpp:5916-5927),
 * CoreSortPivotPartition (5929-5939), CoreSort (5947-5958), Sort (5960-5964).
 * Leaf threshold SortLimite = 16*64/sizeof(T): 256 int, 128 double. */
#define DEFINE_CORESORT(SUF, T, LIMIT)                                         \
    static size_t get_pivot_##SUF(const T* a, size_t left, size_t right) {     \
        const size_t middle = ((right - left) / 2) + left;                     \
        if (a[left] <= a[middle] && a[middle] <= a[right]) return middle;      \
        else if (a[middle] <= a[left] && a[left] <= a[right]) return left;     \
        else return right;                                                     \
    }                                                                          \
    static size_t pivot_partition_##SUF(T* a, size_t left, size_t right) {     \
        if (right - left > 1) {                                                \
            const size_t pivotIdx = get_pivot_##SUF(a, left, right);           \
            T t = a[pivotIdx]; a[pivotIdx] = a[right]; a[right] = t;           \
            const size_t part = oracle_partition_##SUF(a, left, right - 1, a[right]); \
            t = a[part]; a[part] = a[right]; a[right] = t;                     \
            return part;                                                       \
        }                                                                      \
        return left;                                                           \
    }                                                                          \
    static void core_sort_##SUF(T* a, size_t left, size_t right) {             \
        if (right - left < (size_t)(LIMIT)) {                                  \
            oracle_smallsort_##SUF(a + left, right - left + 1);                \
        } else {                                                               \
            const size_t part = pivot_partition_##SUF(a, left, right);         \
            if (part + 1 < right) core_sort_##SUF(a, part + 1, right);         \
            if (part && left < part - 1) core_sort_##SUF(a, left, part - 1);   \
        }                                                                      \
    }                                                                          \
    ORACLE_API void oracle_sort_##SUF(T* a, size_t n) {                        \
        if (n == 0) return; /* the reference's Sort(a,0) is undefined */       \
        core_sort_##SUF(a, 0, n - 1);                                          \
    }

DEFINE_CORESORT(i32, int, 256)
DEFINE_CORESORT(f64, double, 128)

/* ------------------------------------------------------------------------ */
/* Key/value path (sort512kv.hpp).  Values follow keys through every swap.   */

/* CoreScalarPartition kv (sort512kv.hpp:5924-5941) */
static size_t scalar_partition_kv(int* k, int* v, size_t left, size_t right, int pivot) {
    for (; left <= right && k[left] <= pivot; ++left) {
    }
    for (size_t idx = left; idx <= right; ++idx) {
        if (k[idx] <= pivot) {
            int t = k[idx]; k[idx] = k[left]; k[left] = t;
            t = v[idx]; v[idx] = v[left]; v[left] = t;
            left += 1;
        }
    }
    return left;
}

/* One compress pair of kv Partition512: keys and values are compressed with
 * the same mask (sort512kv.hpp:5990-6003). */
static void compress_kv(int* k, int* v, const int* kval, const int* vval, unsigned lanes,
                        int pivot, size_t* left_w, size_t* right_w) {
    unsigned nb_high = 0;
    for (unsigned l = 0; l < lanes; ++l) nb_high += !(kval[l] <= pivot);
    size_t lw = *left_w, rw = *right_w - nb_high, hw = rw;
    for (unsigned l = 0; l < lanes; ++l) {
        if (kval[l] <= pivot) { k[lw] = kval[l]; v[lw] = vval[l]; lw++; }
    }
    for (unsigned l = 0; l < lanes; ++l) {
        if (!(kval[l] <= pivot)) { k[hw] = kval[l]; v[hw] = vval[l]; hw++; }
    }
    *left_w = lw;
    *right_w = rw;
}

/* Partition512 kv (sort512kv.hpp:5959-6082), same walk as the int version. */
ORACLE_API size_t oracle_partition_kv_i32(int* k, int* v, size_t left, size_t right, int pivot) {
    const size_t S = 16;
    if (right - left + 1 < 2 * S) return scalar_partition_kv(k, v, left, right, pivot);
    int lk[16], lv[16], rk[16], rv[16], kv_[16], vv_[16];
    memcpy(lk, &k[left], sizeof(lk));
    memcpy(lv, &v[left], sizeof(lv));
    size_t left_w = left;
    left += S;
    size_t right_w = right + 1;
    right -= S - 1;
    memcpy(rk, &k[right], sizeof(rk));
    memcpy(rv, &v[right], sizeof(rv));
    while (left + S <= right) {
        const size_t free_left = left - left_w;
        const size_t free_right = right_w - right;
        if (free_left <= free_right) {
            memcpy(kv_, &k[left], sizeof(kv_));
            memcpy(vv_, &v[left], sizeof(vv_));
            left += S;
        } else {
            right -= S;
            memcpy(kv_, &k[right], sizeof(kv_));
            memcpy(vv_, &v[right], sizeof(vv_));
        }
        compress_kv(k, v, kv_, vv_, 16, pivot, &left_w, &right_w);
    }
    {
        const size_t remaining = right - left;
        memcpy(kv_, &k[left], sizeof(kv_));
        memcpy(vv_, &v[left], sizeof(vv_));
        left = right;
        compress_kv(k, v, kv_, vv_, (unsigned)remaining, pivot, &left_w, &right_w);
    }
    compress_kv(k, v, lk, lv, 16, pivot, &left_w, &right_w);
    compress_kv(k, v, rk, rv, 16, pivot, &left_w, &right_w);
    return left_w;
}

/* kv leaf (sort512kv.hpp:5235-5916): pairs sorted by (key, value).  The
 * reference's network keeps keys bit-exact but orders equal keys' values
 * arbitrarily (and can lose values on INT_MAX keys); see the file header. */
typedef struct { int k, v; } kvpair;
static int cmp_pair(const void* x, const void* y) {
    const kvpair* a = (const kvpair*)x;
    const kvpair* b = (const kvpair*)y;
    if (a->k != b->k) return (a->k > b->k) - (a->k < b->k);
    return (a->v > b->v) - (a->v < b->v);
}

ORACLE_API void oracle_smallsort_kv_i32(int* k, int* v, size_t len) {
    if (len == 0) return;
    kvpair buf[256];
    size_t n = len > 256 ? 256 : len;
    for (size_t i = 0; i < n; ++i) { buf[i].k = k[i]; buf[i].v = v[i]; }
    qsort(buf, n, sizeof(kvpair), cmp_pair);
    for (size_t i = 0; i < n; ++i) { k[i] = buf[i].k; v[i] = buf[i].v; }
}

/* kv CoreSortGetPivot / CoreSortPivotPartition / CoreSort / Sort
 * (sort512kv.hpp:6086-6136). */
static size_t get_pivot_kv(const int* a, size_t left, size_t right) {
    const size_t middle = ((right - left) / 2) + left;
    if (a[left] <= a[middle] && a[middle] <= a[right]) return middle;
    else if (a[middle] <= a[left] && a[left] <= a[right]) return left;
    else return right;
}

static size_t pivot_partition_kv(int* k, int* v, size_t left, size_t right) {
    if (right - left > 1) {
        const size_t p = get_pivot_kv(k, left, right);
        int t = k[p]; k[p] = k[right]; k[right] = t;
        t = v[p]; v[p] = v[right]; v[right] = t;
        const size_t part = oracle_partition_kv_i32(k, v, left, right - 1, k[right]);
        t = k[part]; k[part] = k[right]; k[right] = t;
        t = v[part]; v[part] = v[right]; v[right] = t;
        return part;
    }
    return left;
}

static void core_sort_kv(int* k, int* v, size_t left, size_t right) {
    if (right - left < 256) {
        oracle_smallsort_kv_i32(k + left, v + left, right - left + 1);
    } else {
        const size_t part = pivot_partition_kv(k, v, left, right);
        if (part + 1 < right) core_sort_kv(k, v, part + 1, right);
        if (part && left < part - 1) core_sort_kv(k, v, left, part - 1);
    }
}

ORACLE_API void oracle_sort_kv_i32(int* k, int* v, size_t n) {
    if (n == 0) return;
    core_sort_kv(k, v, 0, n - 1);
}

/* ------------------------------------------------------------------------ */
/* Merge semantics of the OpenMP drivers.
 * SortOmpMerge / SortOmpMergeDeps (sort512.hpp:6006-6102) sort nbParts
 * chunks of ceil(n/nbParts) with CoreSort, then merge neighbouring runs
 * level by level with std::inplace_merge.  SortOmpParMerge (6104-6174) does
 * the same with ParallelInplace::parallelMergeInPlace (parallelInplace.hpp:
 * 210-306), whose result is the same merged run.  The restatement uses a
 * stable buffered merge (the result std::inplace_merge defines). */
#define DEFINE_MERGE(SUF, T)                                                   \
    ORACLE_API void oracle_merge_##SUF(T* a, size_t n, size_t middle) {        \
        if (middle == 0 || middle >= n) return;                                \
        T* tmp = (T*)malloc(n * sizeof(T));                                    \
        size_t i = 0, j = middle, o = 0;                                       \
        while (i < middle && j < n) tmp[o++] = (a[j] < a[i]) ? a[j++] : a[i++]; \
        while (i < middle) tmp[o++] = a[i++];                                  \
        while (j < n) tmp[o++] = a[j++];                                       \
        memcpy(a, tmp, n * sizeof(T));                                         \
        free(tmp);                                                             \
    }                                                                          \
    ORACLE_API void oracle_sort_chunks_merge_##SUF(T* a, size_t n, int nbParts) { \
        if (n == 0) return;                                                    \
        if (nbParts < 1) nbParts = 1;                                          \
        const size_t chunk = (n + (size_t)nbParts - 1) / (size_t)nbParts;      \
        for (int p = 0; p < nbParts; ++p) {                                    \
            size_t first = chunk * (size_t)p; if (first > n) first = n;        \
            size_t last = chunk * (size_t)(p + 1); if (last > n) last = n;     \
            if (first < last) core_sort_##SUF(a, first, last - 1);             \
        }                                                                      \
        for (int level = 1; (1 << level) <= nbParts; ++level) {                \
            const size_t span = (size_t)1 << level;                           \
            for (size_t part = 0; part < (size_t)nbParts / span; ++part) {     \
                size_t first = part * span * chunk; if (first > n) first = n;  \
                size_t middle = first + (span / 2) * chunk; if (middle > n) middle = n; \
                size_t last = first + span * chunk; if (last > n) last = n;    \
                oracle_merge_##SUF(a + first, last - first, middle - first);   \
            }                                                                  \
        }                                                                      \
    }

DEFINE_MERGE(i32, int)
DEFINE_MERGE(f64, double)

/* ------------------------------------------------------------------------ */
/* Batched sort: the reference's analogue (sort512perf.cpp:612-709 timeSmall)
 * loops SmallSort16V over independent arrays; longer arrays use Sort.
 * offsets has nseg+1 entries. */
ORACLE_API void oracle_segsort_i32(int* a, const size_t* off, size_t nseg) {
    for (size_t s = 0; s < nseg; ++s) oracle_sort_i32(a + off[s], off[s + 1] - off[s]);
}
ORACLE_API void oracle_segsort_f64(double* a, const size_t* off, size_t nseg) {
    for (size_t s = 0; s < nseg; ++s) oracle_sort_f64(a + off[s], off[s + 1] - off[s]);
}
ORACLE_API void oracle_segsort_kv_i32(int* k, int* v, const size_t* off, size_t nseg) {
    for (size_t s = 0; s < nseg; ++s) oracle_sort_kv_i32(k + off[s], v + off[s], off[s + 1] - off[s]);
}
