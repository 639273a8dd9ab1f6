"""GPU parity: libsort512cuda (through its C ABI) against the reference's
outputs (golden digests made by the reference compiled in place) and the C
restatement (oracle), on the reference tests' own inputs and sizes, plus edge
cases and larger sizes checked through size-independent properties."""
import numpy as np
import pytest

from helpers import (assert_partitioned, assert_same_multiset, assert_same_pairs, assert_sorted, digest,
                     kv_input, pairs_digest, sort_f64_total_order)

pytestmark = pytest.mark.gpu


# ---- SmallSort16V / CoreSmallSortN (sort512test.cpp:1551-1600, 165-1333) ----
def test_smallsort_every_length_matches_reference(golden, oracle, s512, cuda):
    for case in golden["smallsort"]:
        st = oracle.rng(case["seed"])
        for d in case["digests"]:
            a = oracle.rand_vec(st, case["n"], case["dtype"])
            s512.small_sort(a)
            assert digest(a) == d, (case["dtype"], case["n"])


def test_smallsort_100_trials_vs_oracle(oracle, s512, cuda):
    # testSmallVecSort: every length, 100 trials (here on the device, batched
    # through torch tensors to keep the test short)
    import torch
    st = oracle.rng(0)
    for dt, lim in ((np.int32, 256), (np.float64, 128)):
        for n in range(1, lim + 1):
            for _ in range(10):
                a = oracle.rand_vec(st, n, dt)
                t = torch.from_numpy(a.copy()).to(cuda)
                s512.small_sort(t)
                oracle.smallsort(a)
                assert np.array_equal(t.cpu().numpy(), a), (dt, n)


def test_core_small_sort_matches_reference(golden, oracle, s512, cuda):
    for case in golden["core_small_sort"]:
        lanes = 16 if case["dtype"] == "int32" else 8
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["nvec"] * lanes, case["dtype"])
        s512.core_small_sort(a, case["nvec"])
        assert digest(a) == case["digest"], case


def test_kat_vectors(golden, s512, cuda):
    for case in golden["kat"]:
        a = np.array(case["input"], dtype=case["dtype"])
        s512.core_small_sort(a, 1 if case["kind"] == "core1" else 2)
        assert a.tolist() == case["output"], case


def test_kv_smallsort_matches_reference(golden, oracle, s512, cuda):
    for case in golden["kv_smallsort"]:
        st = oracle.rng(case["seed"])
        k, v = kv_input(oracle, st, case["n"])
        s512.small_sort_kv(k, v)
        assert digest(k) == case["keys"], case["n"]
        assert pairs_digest(k, v) == case["pairs"], case["n"]


def test_kv_core_small_sort_pairs(oracle, s512, cuda):
    # testSortNVec_pair: values follow keys (value = key*100+1)
    st = oracle.rng(0)
    for nvec in range(1, 17):
        for _ in range(20):
            k = oracle.rand_vec(st, nvec * 16, np.int32)
            v = (k * 100 + 1).astype(np.int32)
            k0 = k.copy()
            s512.core_small_sort_kv(k, v, nvec)
            assert_sorted(k)
            assert np.array_equal(v, k * 100 + 1)
            assert_same_multiset(k, k0)


# ---- Sort / SortOmp* (testQs512, sort512test.cpp:1368-1408) ---------------
def test_sort_matches_reference(golden, oracle, s512, cuda):
    for case in golden["sort"]:
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        s512.sort(a)
        assert digest(a) == case["digest"], (case["dtype"], case["n"])


def test_sort_omp_variants_match_reference(golden, oracle, s512, cuda):
    for case in golden["sort_omp"]:
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        s512.sort(a)
        assert digest(a) == case["digest"], case


def test_sort_device_pointer_and_stream(oracle, s512, cuda):
    import torch
    st = oracle.rng(77)
    for dt in (np.int32, np.float64):
        for n in (1, 7, 300, 5000, 20000, 123457, 1 << 20):
            a = oracle.rand_vec(st, n, dt)
            t = torch.from_numpy(a.copy()).to(cuda)
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                s512.sort(t, stream=s)
            s.synchronize()
            oracle.sort(a)
            assert np.array_equal(t.cpu().numpy(), a), (dt, n)


def test_config_c1_exact(golden, s512, cuda):
    # int32 2^20 uniform over the full range, seed 0 -- equal to
    # the reference's Sort output
    import workloads
    a = workloads.uniform_i32_np(1 << 20, 0)
    s512.sort(a)
    assert digest(a) == golden["c1"]["sorted"]


# ---- Partition512 (testPartition, sort512test.cpp:1452-1549) --------------
def test_partition_matches_reference_boundary(golden, oracle, s512, cuda):
    for case in golden["partition"]:
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        a0 = a.copy()
        pivot = np.dtype(case["dtype"]).type(case["pivot"])
        lim = s512.partition(a, 0, case["n"] - 1, pivot)
        assert lim == case["boundary"], case
        assert_partitioned(a, pivot, lim, str(case["n"]))
        assert_same_multiset(a, a0)


def test_partition_subrange_and_prefilled(oracle, s512, cuda):
    st = oracle.rng(5)
    for dt in (np.int32, np.float64):
        for n in (1, 2, 32, 1024, 70000):
            a = np.full(n, dt(n))  # testPartition's third loop pre-fills with n
            a[:] = oracle.rand_vec(st, n, dt)
            left, right = n // 4, n - 1 - n // 5
            if right < left:
                left, right = 0, n - 1
            a0 = a.copy()
            b = a.copy()
            pivot = dt(n // 2)
            lim = s512.partition(a, left, right, pivot)
            lo = oracle.partition(b, left, right, pivot)
            assert lim == lo
            assert np.array_equal(a[:left], a0[:left]) and np.array_equal(a[right + 1:], a0[right + 1:])
            assert_partitioned(a[left:right + 1], pivot, lim - left)
            assert_same_multiset(a[left:right + 1], a0[left:right + 1])


def test_kv_partition_matches_reference_boundary(golden, oracle, s512, cuda):
    for case in golden["kv_partition"][::7]:
        st = oracle.rng(case["seed"])
        k, v = kv_input(oracle, st, case["n"])
        k0, v0 = k.copy(), v.copy()
        lim = s512.partition_kv(k, v, 0, case["n"] - 1, case["pivot"])
        assert lim == case["boundary"]
        assert_partitioned(k, case["pivot"], lim)
        assert_same_pairs(k, v, k0, v0)


# ---- Sort512kv::Sort (testQs512_pair, sort512test.cpp:1410-1450) ----------
def test_kv_sort_matches_reference(golden, oracle, s512, cuda):
    for case in golden["kv_sort"]:
        st = oracle.rng(case["seed"])
        k, v = kv_input(oracle, st, case["n"])
        s512.sort_kv(k, v)
        assert digest(k) == case["keys"], case
        assert pairs_digest(k, v) == case["pairs"], case


def test_kv_sort_int_max_keys_keep_values(s512, cuda):
    # the reference pads values with INT_MAX and can lose values on INT_MAX
    # keys; here every (key, value) pair survives
    rng = np.random.default_rng(1)
    for n in (5, 100, 256, 3000, 50000):
        k = rng.integers(-5, 5, n).astype(np.int32)
        k[rng.random(n) < 0.3] = np.iinfo(np.int32).max
        k[rng.random(n) < 0.1] = np.iinfo(np.int32).min
        v = rng.integers(-2 ** 31, 2 ** 31 - 1, n).astype(np.int32)
        k0, v0 = k.copy(), v.copy()
        s512.sort_kv(k, v)
        assert_sorted(k)
        assert_same_pairs(k, v, k0, v0)
        order = np.lexsort((v0, k0))
        assert np.array_equal(k, k0[order]) and np.array_equal(v, v0[order])


# ---- edge cases -----------------------------------------------------------
def test_empty_and_single(s512, cuda):
    a = np.zeros(0, np.int32)
    s512.sort(a)
    b = np.array([42], np.int32)
    s512.sort(b)
    assert b[0] == 42
    c = np.array([3.5])
    s512.sort(c)
    assert c[0] == 3.5
    assert s512.partition(np.array([5], np.int32), 0, 0, 4) == 0
    assert s512.partition(np.array([5], np.int32), 0, 0, 5) == 1


@pytest.mark.parametrize("n", [300, 17000, 1 << 20])
def test_degenerate_inputs(n, s512, cuda, oracle):
    # inputs on which the reference quicksort is quadratic (all equal, sorted,
    # reversed, few distinct) and the type extremes
    i32 = np.iinfo(np.int32)
    cases = [
        np.zeros(n, np.int32),
        np.arange(n, dtype=np.int32),
        np.arange(n, dtype=np.int32)[::-1].copy(),
        (np.arange(n) % 3).astype(np.int32),
        np.where(np.arange(n) % 2 == 0, i32.min, i32.max).astype(np.int32),
        np.random.default_rng(n).integers(i32.min, i32.max, n, endpoint=True).astype(np.int32),
    ]
    for a in cases:
        b = a.copy()
        s512.sort(b)
        assert np.array_equal(b, np.sort(a))


def test_double_special_values(s512, cuda):
    rng = np.random.default_rng(3)
    n = 40000
    base = rng.standard_normal(n)
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.finfo(np.float64).max, -np.finfo(np.float64).max,
                         np.finfo(np.float64).tiny, 5e-324, -5e-324])
    idx = rng.integers(0, n, 4000)
    base[idx] = specials[rng.integers(0, len(specials), 4000)]
    for m in (n, 200, 5000):
        a = base[:m].copy()
        s512.sort(a)
        expect = sort_f64_total_order(base[:m])
        assert np.array_equal(a.view(np.uint64), expect.view(np.uint64)), m


def test_double_nan_goes_to_the_ends(s512, cuda):
    a = np.array([1.0, np.nan, -2.0, -np.nan, 0.5] * 100)
    s512.sort(a)
    expect = sort_f64_total_order(np.array([1.0, np.nan, -2.0, -np.nan, 0.5] * 100))
    assert np.array_equal(a.view(np.uint64), expect.view(np.uint64))


# ---- larger sizes: properties + the restatement ---------------------------
def _check_sorted_device(t, t0):
    import torch
    assert bool((t[1:] >= t[:-1]).all())
    ref = torch.sort(t0).values
    if t.dtype == torch.float64:
        assert torch.equal(t.view(torch.int64), ref.view(torch.int64)) or torch.equal(t, ref)
    else:
        assert torch.equal(t, ref)


@pytest.mark.parametrize("n", [1 << 22, (1 << 24) + 12345])
def test_large_int32(n, s512, cuda):
    import torch
    import workloads
    t0 = workloads.uniform_i32_torch(n, seed=n)
    t = t0.clone()
    s512.sort(t)
    _check_sorted_device(t, t0)


def test_large_int32_vs_restatement(s512, cuda, oracle):
    import workloads
    a = workloads.uniform_i32_np(1 << 22, 9)
    b = a.copy()
    s512.sort(a)
    oracle.sort(b)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("dist", ["uniform", "normal", "distinct256", "ascending", "descending",
                                  "lognormal", "gauss_mix"])
def test_large_double_distributions(dist, s512, cuda):
    import torch
    import workloads
    n = 1 << 23
    t0 = workloads.double_dist_torch(dist, n, seed=7)
    t = t0.clone()
    s512.sort(t)
    assert bool((t[1:] >= t[:-1]).all())
    assert torch.equal(t, torch.sort(t0).values)


@pytest.mark.parametrize("copies", [8, 40, 300])
def test_leaves_with_repeated_values(copies, s512, cuda):
    # every value repeated ~`copies` times, too rarely to become an equality
    # bucket: a leaf's value slots hold runs of equal keys, which sends the
    # leaf (copies >= 8 or so) from the slot sort to the block sort
    import torch
    n = 1 << 22
    g = torch.Generator(device=cuda).manual_seed(copies)
    distinct = n // copies
    vals = torch.randint(-(1 << 30), 1 << 30, (distinct,), generator=g, device=cuda, dtype=torch.int64)
    pick = torch.randint(0, distinct, (n,), generator=g, device=cuda)
    t0 = vals[pick].to(torch.int32)
    t = t0.clone()
    s512.sort(t)
    assert torch.equal(t, torch.sort(t0).values)
    d0 = vals[pick].to(torch.float64) * 1e-3
    d = d0.clone()
    s512.sort(d)
    assert torch.equal(d, torch.sort(d0).values)


def test_leaves_mixed_even_and_uneven(s512, cuda):
    # half the keys uniform (slot sort), half a few thousand repeated values
    # in another range (block sort), in one array
    import torch
    n = (1 << 23) + 777
    g = torch.Generator(device=cuda).manual_seed(5)
    u = torch.rand(n, generator=g, device=cuda, dtype=torch.float64)
    coarse = torch.floor(u * 4096.0) / 4096.0 + 2.0
    t0 = torch.where(torch.arange(n, device=cuda) % 2 == 0, u, coarse)
    t = t0.clone()
    s512.sort(t)
    assert torch.equal(t, torch.sort(t0).values)


@pytest.mark.parametrize("keys", ["uniform", "zipf"])
def test_large_kv(keys, s512, cuda):
    import torch
    import workloads
    n = 1 << 22
    k0 = workloads.uniform_i32_torch(n, 11) if keys == "uniform" else workloads.zipf_i32_torch(n, seed=11)
    v0 = torch.arange(n, dtype=torch.int32, device=cuda)
    k, v = k0.clone(), v0.clone()
    s512.sort_kv(k, v)
    assert bool((k[1:] >= k[:-1]).all())
    # (key, value) pairs: value = original index, so gathering the keys by the
    # values must give back the sorted keys, and values must be a permutation
    assert torch.equal(k0[v.long()], k)
    assert torch.equal(torch.sort(v).values, v0)
    # ties ordered by value (pairs in (key, value) order)
    same = k[1:] == k[:-1]
    assert bool((v[1:][same] > v[:-1][same]).all())


def test_large_partition(s512, cuda):
    import torch
    import workloads
    n = (1 << 23) + 77
    t0 = workloads.uniform_i32_torch(n, 3)
    t = t0.clone()
    lim = s512.partition(t, 0, n - 1, 12345)
    assert lim == int((t0 <= 12345).sum())
    assert bool((t[:lim] <= 12345).all()) and bool((t[lim:] > 12345).all())
    assert torch.equal(torch.sort(t).values, torch.sort(t0).values)


def test_stats_are_reported(s512, cuda):
    import workloads
    s512.set_config(collect_stats=1)
    try:
        a = workloads.uniform_i32_np(1 << 22, 1)
        s512.sort(a)
        st = s512.stats()
        assert st["levels"] >= 1 and st["partition_ms"][0] > 0 and st["total_ms"] > 0
        assert st["partition_keys"][0] == 1 << 22
        assert st["fallbacks"] == 0
        # sampled quantile splitters on uniform keys: buckets within a few
        # tens of percent of each other (sample counts per bucket ~ 64-128)
        assert 0.0 < st["bucket_cv"][0] < 0.5 and st["max_bucket_over_mean"][0] < 2.0
    finally:
        s512.set_config(collect_stats=0)


def test_unaligned_device_input(s512, cuda, oracle):
    # a sub-array that starts 1 element into an allocation is not 16-byte
    # aligned: the partition pass reads it with plain loads instead of bulk copies
    import torch
    import workloads
    for dt, n in ((torch.int32, 300001), (torch.float64, 200003)):
        base = (workloads.uniform_i32_torch(n + 1, 21) if dt == torch.int32
                else workloads.uniform01_torch(n + 1, 21)).to(cuda)
        t = base[1:]
        assert t.data_ptr() % 16 != 0
        ref = torch.sort(t.clone()).values
        s512.sort(t)
        assert torch.equal(t, ref)
        assert base[0].item() == (workloads.uniform_i32_torch(1, 21) if dt == torch.int32
                                  else workloads.uniform01_torch(1, 21)).item()
    k = workloads.uniform_i32_torch(100001, 22)
    v = torch.arange(100001, dtype=torch.int32, device=cuda)
    kk, vv = k[1:].clone(), v[1:].clone()
    k1, v1 = k[1:], v[1:]
    s512.sort_kv(k1, v1)
    assert torch.equal(k1, torch.sort(kk).values)
    assert torch.equal(kk[(v1 - 1).long()], k1)


# ---- merge path (SortOmpMerge / SortOmpParMerge / parallelMergeInPlace) ----
def test_merge_matches_restated_inplace_merge(s512, cuda, oracle):
    import workloads
    rng = np.random.default_rng(4)
    for dt in (np.int32, np.float64):
        for n, mid in ((2, 1), (10, 3), (4097, 4096), (5000, 17), (100000, 50000), (1 << 20, 123457),
                       (1 << 20, (1 << 20) - 1), (300000, 299000)):
            a = workloads.uniform_i32_np(n, n) if dt == np.int32 else workloads.uniform01_np(n, n)
            if dt == np.int32:
                a = (a % 1000).astype(np.int32)  # many ties: stability is visible
            a[:mid].sort()
            a[mid:].sort()
            b = a.copy()
            s512.merge(a, mid)
            oracle.merge(b, mid)
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (dt, n, mid)


def test_merge_keeps_signed_zero_order(s512, cuda, oracle):
    # -0.0 and +0.0 compare equal: a stable merge keeps the left run's zeros first
    a = np.array([-1.0, -0.0, 0.0, 2.0, -0.5, 0.0, -0.0, 3.0])
    b = a.copy()
    s512.merge(a, 4)
    oracle.merge(b, 4)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_sort_omp_merge_matches_reference(golden, oracle, s512, cuda):
    for case in golden["sort_omp"]:
        if case["fn"] not in ("sort_omp_merge", "sort_omp_merge_deps", "sort_omp_parmerge"):
            continue
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        s512.sort_omp_merge(a, 8)
        assert digest(a) == case["digest"], case


@pytest.mark.parametrize("parts", [1, 2, 3, 7, 8, 64])
def test_sort_omp_merge_any_part_count(parts, s512, cuda):
    import torch
    import workloads
    n = 1_000_003
    t0 = workloads.uniform_i32_torch(n, parts)
    t = t0.clone()
    s512.sort_omp_merge(t, parts)
    assert torch.equal(t, torch.sort(t0).values)
