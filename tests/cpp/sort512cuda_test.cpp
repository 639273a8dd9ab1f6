// sort512cuda_test.cpp -- the reference's unit-test program (sort512test.cpp),
// re-expressed against the drop-in header sort512cuda.hpp.  Same checks, same
// sizes, same drand48 inputs:
//   assertNotSorted        (sort512test.cpp:29-39)
//   assertNotPartitioned   (41-60)
//   Checker: multiset kept (100-119)
//   createRandVec          (77-83)
//   testPopcount (122-146), KAT vectors (169-202, 290-375),
//   testSortNVec for N = 1..16 (165-1333), kv pair tests (*_pair),
//   testSmallVecSort (1551-1567), testSmallVecSort_pair (1569-1600),
//   testQs512 (1368-1408), testQs512_pair (1410-1450),
//   testPartition (1452-1484), testPartition_pair (1486-1549).
// Exit code 0 when every check passes.  Extra cases the reference leaves
// undefined (size 0) are checked as no-ops.
#include "sort512cuda.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

static int g_fail = 0;

template <class T>
static void assert_sorted(const T* a, size_t n, const std::string& what) {
    for (size_t i = 1; i < n; ++i)
        if (a[i - 1] > a[i]) {
            std::printf("not sorted at %zu: %s\n", i, what.c_str());
            g_fail = 1;
            return;
        }
}

template <class T>
static void assert_partitioned(const T* a, size_t n, T pivot, size_t limit, const std::string& what) {
    for (size_t i = 0; i < limit; ++i)
        if (a[i] > pivot) {
            std::printf("not partitioned (low side) at %zu: %s\n", i, what.c_str());
            g_fail = 1;
            return;
        }
    for (size_t i = limit; i < n; ++i)
        if (a[i] <= pivot) {
            std::printf("not partitioned (high side) at %zu: %s\n", i, what.c_str());
            g_fail = 1;
            return;
        }
}

template <class T>
static void assert_equal(const T* a, const T* b, size_t n, const std::string& what) {
    for (size_t i = 0; i < n; ++i)
        if (!(a[i] == b[i])) {
            std::printf("not equal at %zu: %s\n", i, what.c_str());
            g_fail = 1;
            return;
        }
}

template <class T>
static void rand_vec(T* a, size_t n) {
    for (size_t i = 0; i < n; ++i) a[i] = T(drand48() * double(n));
}

// keeps a copy; on destruction checks the multiset was preserved
template <class T>
class Checker {
  public:
    Checker(const T* src, T* dst, size_t n) : dst_(dst), copy_(src, src + n) {}
    ~Checker() {
        std::vector<T> got(dst_, dst_ + copy_.size());
        std::sort(got.begin(), got.end());
        std::sort(copy_.begin(), copy_.end());
        assert_equal(copy_.data(), got.data(), copy_.size(), "Checker");
    }

  private:
    T* dst_;
    std::vector<T> copy_;
};

static void test_popcount() {
    std::printf("popcount\n");
    if (Sort512::popcount(0) != 0 || Sort512::popcount(3) != 2 || Sort512::popcount(0xFFFF) != 16 ||
        Sort512::popcount(0xFF) != 8)
        g_fail = 1;
    for (int i = 0; i < 16; ++i)
        if (Sort512::popcount(1u << i) != 1) g_fail = 1;
}

// N vectors through the CoreSmallSortN pointer forms, with the KAT vectors
template <class T, int S>
static void core_sort_n(T* p, int nvec) {
    switch (nvec) {
        case 1: Sort512::CoreSmallSort(p); break;
        case 2: Sort512::CoreSmallSort2(p, p + S); break;
        case 3: Sort512::CoreSmallSort3(p, p + S, p + 2 * S); break;
        case 4: Sort512::CoreSmallSort4(p, p + S, p + 2 * S, p + 3 * S); break;
        case 5: Sort512::CoreSmallSort5(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S); break;
        case 6: Sort512::CoreSmallSort6(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S); break;
        case 7: Sort512::CoreSmallSort7(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S); break;
        case 8:
            Sort512::CoreSmallSort8(p, p + S, p + 2 * S, p + 3 * S, p + 4 * S, p + 5 * S, p + 6 * S, p + 7 * S);
            break;
        default: {
            // 9..16: the same network over consecutive vectors
            std::vector<T*> v;
            for (int i = 0; i < nvec; ++i) v.push_back(p + i * S);
            if (nvec == 16)
                Sort512::CoreSmallSort16(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11],
                                         v[12], v[13], v[14], v[15]);
            else if (nvec == 12)
                Sort512::CoreSmallSort12(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11]);
            else
                Sort512::SmallSort16V(p, (size_t)nvec * S);
        }
    }
}

template <class T, int S>
static void test_sort_nvec() {
    std::printf("CoreSmallSortN %s\n", sizeof(T) == 4 ? "int" : "double");
    {   // sorted and reverse KAT (sort512test.cpp:169-202)
        T a[S], r[S];
        for (int i = 0; i < S; ++i) a[i] = T(i + 1), r[i] = T(i + 1);
        core_sort_n<T, S>(a, 1);
        assert_equal(a, r, S, "KAT sorted");
        for (int i = 0; i < S; ++i) a[i] = T(S - i);
        core_sort_n<T, S>(a, 1);
        assert_equal(a, r, S, "KAT reversed");
    }
    {   // paired-duplicate KATs in four orders (290-375)
        const int N = 2 * S;
        T res[N];
        for (int i = 0; i < N; ++i) res[i] = T(i / 2 + 1);
        std::vector<std::vector<T>> orders(4, std::vector<T>(N));
        for (int i = 0; i < N; ++i) {
            orders[0][i] = res[i];
            orders[1][i] = res[N - 1 - i];
            orders[2][i] = res[(i + S) % N];
            orders[3][i] = i < S ? res[S - 1 - i] : res[N - 1 - (i - S)];
        }
        for (auto& o : orders) {
            core_sort_n<T, S>(o.data(), 2);
            assert_sorted(o.data(), N, "KAT pairs");
            assert_equal(o.data(), res, N, "KAT pairs");
        }
    }
    srand48(0);
    for (int nvec = 1; nvec <= 16; ++nvec) {
        for (int loop = 0; loop < 1000 / 10; ++loop) {
            std::vector<T> a(nvec * S);
            rand_vec(a.data(), a.size());
            Checker<T> c(a.data(), a.data(), a.size());
            core_sort_n<T, S>(a.data(), nvec);
            assert_sorted(a.data(), a.size(), "CoreSmallSortN");
        }
    }
}

static void test_sort_nvec_pair() {
    std::printf("CoreSmallSortN pairs\n");
    srand48(0);
    for (int nvec = 1; nvec <= 16; ++nvec) {
        for (int loop = 0; loop < 100; ++loop) {
            const int n = nvec * 16;
            std::vector<int> k(n), v(n);
            rand_vec(k.data(), n);
            for (int i = 0; i < n; ++i) v[i] = k[i] * 100 + 1;
            Checker<int> c(k.data(), k.data(), n);
            switch (nvec) {
                case 1: Sort512kv::CoreSmallSort(k.data(), v.data()); break;
                case 2: Sort512kv::CoreSmallSort2(k.data(), v.data()); break;
                case 8: Sort512kv::CoreSmallSort8(k.data(), v.data()); break;
                case 16: Sort512kv::CoreSmallSort16(k.data(), v.data()); break;
                default: Sort512kv::SmallSort16V(k.data(), v.data(), (size_t)n);
            }
            assert_sorted(k.data(), n, "kv CoreSmallSortN");
            for (int i = 0; i < n; ++i)
                if (v[i] != k[i] * 100 + 1) {
                    std::printf("kv pair broken at %d\n", i);
                    g_fail = 1;
                    break;
                }
        }
    }
}

template <class T>
static void test_small_vec_sort() {
    std::printf("SmallSort16V %s\n", sizeof(T) == 4 ? "int" : "double");
    const int max_len = (64 / (int)sizeof(T)) * 16;
    for (int len = 1; len <= max_len; ++len) {
        std::vector<T> a(len);
        for (int t = 0; t < 100; ++t) {
            rand_vec(a.data(), len);
            Checker<T> c(a.data(), a.data(), len);
            Sort512::SmallSort16V(a.data(), (size_t)len);
            assert_sorted(a.data(), len, "SmallSort16V");
        }
    }
}

static void test_small_vec_sort_pair() {
    std::printf("SmallSort16V pairs\n");
    for (int len = 1; len <= 256; ++len) {
        std::vector<int> k(len), v(len);
        for (int t = 0; t < 100; ++t) {
            rand_vec(k.data(), len);
            Checker<int> c(k.data(), k.data(), len);
            for (int i = 0; i < len; ++i) v[i] = k[i] * 100 + 1;
            Sort512kv::SmallSort16V(k.data(), v.data(), (size_t)len);
            assert_sorted(k.data(), len, "kv SmallSort16V");
            for (int i = 0; i < len; ++i)
                if (v[i] != k[i] * 100 + 1) {
                    std::printf("kv SmallSort16V pair broken at len %d\n", len);
                    g_fail = 1;
                    break;
                }
        }
    }
}

template <class T>
static void test_qs512() {
    std::printf("Sort + SortOmp* %s\n", sizeof(T) == 4 ? "int" : "double");
    for (int variant = 0; variant < 5; ++variant) {
        for (size_t n = 1; n <= (1 << 10); n *= 2) {
            std::unique_ptr<T[]> a(new T[n]);
            rand_vec(a.get(), n);
            Checker<T> c(a.get(), a.get(), n);
            switch (variant) {
                case 0: Sort512::Sort<T, size_t>(a.get(), n); break;
                case 1: Sort512::SortOmpPartition<T, size_t>(a.get(), n); break;
                case 2: Sort512::SortOmpMerge<T, size_t>(a.get(), n); break;
                case 3: Sort512::SortOmpMergeDeps<T, size_t>(a.get(), n); break;
                default: Sort512::SortOmpParMerge<T, size_t>(a.get(), n); break;
            }
            assert_sorted(a.get(), n, "Sort variant " + std::to_string(variant));
        }
    }
    // larger than one leaf: runs the partition levels
    for (size_t n : {size_t(20000), size_t(100003), size_t(1) << 20}) {
        std::vector<T> a(n);
        rand_vec(a.data(), n);
        Checker<T> c(a.data(), a.data(), n);
        Sort512::Sort<T, size_t>(a.data(), n);
        assert_sorted(a.data(), n, "Sort large");
    }
    // size 0 is a no-op here (undefined in the reference)
    Sort512::Sort<T, size_t>(nullptr, 0);
}

static void test_qs512_pair() {
    std::printf("kv Sort + SortOmpPartition\n");
    for (int variant = 0; variant < 2; ++variant) {
        for (size_t n = 1; n <= (1 << 10); n *= 2) {
            std::unique_ptr<int[]> k(new int[n]), v(new int[n]);
            rand_vec(k.get(), n);
            Checker<int> c(k.get(), k.get(), n);
            for (size_t i = 0; i < n; ++i) v[i] = k[i] * 100 + 1;
            if (variant == 0) Sort512kv::Sort<int, size_t>(k.get(), v.get(), n);
            else Sort512kv::SortOmpPartition<int, size_t>(k.get(), v.get(), n);
            assert_sorted(k.get(), n, "kv Sort");
            for (size_t i = 0; i < n; ++i)
                if (v[i] != k[i] * 100 + 1) {
                    std::printf("kv Sort pair broken\n");
                    g_fail = 1;
                    break;
                }
        }
    }
}

template <class T>
static void test_partition() {
    std::printf("Partition512 %s\n", sizeof(T) == 4 ? "int" : "double");
    auto one = [](size_t n, bool prefill) {
        std::unique_ptr<T[]> a(new T[n]);
        if (prefill)
            for (size_t i = 0; i < n; ++i) a[i] = T(n);
        rand_vec(a.get(), n);
        Checker<T> c(a.get(), a.get(), n);
        const T pivot = T(n / 2);
        const size_t limit = Sort512::Partition512<size_t>(&a[0], 0, n - 1, pivot);
        assert_partitioned(a.get(), n, pivot, limit, "Partition512");
    };
    for (size_t n = 1; n <= (1 << 10); n *= 2) one(n, false);
    for (size_t n = 1; n <= 1000; ++n) one(n, false);
    for (size_t n = 1; n <= (1 << 10); n *= 2) one(n, true);
}

static void test_partition_pair() {
    std::printf("Partition512 pairs\n");
    auto one = [](size_t n) {
        std::unique_ptr<int[]> k(new int[n]), v(new int[n]);
        rand_vec(k.get(), n);
        Checker<int> c(k.get(), k.get(), n);
        for (size_t i = 0; i < n; ++i) v[i] = k[i] * 100 + 1;
        const int pivot = int(n / 2);
        const size_t limit = Sort512kv::Partition512<size_t>(&k[0], &v[0], 0, n - 1, pivot);
        assert_partitioned(k.get(), n, pivot, limit, "kv Partition512");
        for (size_t i = 0; i < n; ++i)
            if (v[i] != k[i] * 100 + 1) {
                std::printf("kv Partition512 pair broken\n");
                g_fail = 1;
                break;
            }
    };
    for (size_t n = 1; n <= (1 << 10); n *= 2) one(n);
    for (size_t n = 1; n <= 1000; ++n) one(n);
}

// ParallelInplace::parallelMergeInPlace on two sorted halves (parallelInplace.hpp:210)
template <class T>
static void test_parallel_merge() {
    std::printf("parallelMergeInPlace %s\n", sizeof(T) == 4 ? "int" : "double");
    for (size_t n : {size_t(2), size_t(17), size_t(1000), size_t(65537), size_t(1) << 20}) {
        for (size_t center : {size_t(1), n / 3, n / 2, n - 1}) {
            if (center == 0 || center >= n) continue;
            std::vector<T> a(n);
            rand_vec(a.data(), n);
            std::sort(a.begin(), a.begin() + center);
            std::sort(a.begin() + center, a.end());
            std::vector<T> want(a);
            std::inplace_merge(want.begin(), want.begin() + center, want.end());
            ParallelInplace::parallelMergeInPlace(a.data(), (long)n, (long)center);
            assert_equal(a.data(), want.data(), n, "parallelMergeInPlace");
        }
    }
}

// Extensions: 64-bit integer keys and interleaved int[2] pairs.
static void test_wide_words() {
    std::printf("Sort<long long>, Sort512kv::Sort(int[2])\n");
    for (size_t n : {size_t(1), size_t(100), size_t(5000), size_t(300000)}) {
        std::vector<long long> a(n);
        for (size_t i = 0; i < n; ++i)
            a[i] = (long long)((drand48() - 0.5) * 9.0e18);
        std::vector<long long> want(a);
        std::sort(want.begin(), want.end());
        Sort512::Sort<long long, size_t>(a.data(), n);
        assert_equal(a.data(), want.data(), n, "Sort<long long>");

        std::vector<int> p(2 * n);
        for (size_t i = 0; i < n; ++i) {
            p[2 * i] = int(drand48() * double(n / 4 + 1)) - int(n / 8);
            p[2 * i + 1] = int(drand48() * 2.0e9) - 1000000000;
        }
        std::vector<std::pair<int, int>> wp(n);
        for (size_t i = 0; i < n; ++i) wp[i] = {p[2 * i], p[2 * i + 1]};
        std::sort(wp.begin(), wp.end());
        Sort512kv::Sort(reinterpret_cast<int(*)[2]>(p.data()), n);
        for (size_t i = 0; i < n; ++i)
            if (p[2 * i] != wp[i].first || p[2 * i + 1] != wp[i].second) {
                std::printf("pairs differ at %zu (n=%zu)\n", i, n);
                g_fail = 1;
                break;
            }
    }
}

int main() {
    test_popcount();
    test_sort_nvec<int, 16>();
    test_sort_nvec<double, 8>();
    test_sort_nvec_pair();
    test_small_vec_sort<int>();
    test_small_vec_sort<double>();
    test_small_vec_sort_pair();
    test_qs512<double>();
    test_qs512<int>();
    test_qs512_pair();
    test_partition<int>();
    test_partition<double>();
    test_partition_pair();
    test_parallel_merge<int>();
    test_parallel_merge<double>();
    test_wide_words();
    if (g_fail) std::printf("Test failed!\n");
    else std::printf("All tests passed\n");
    return g_fail;
}
