"""The CPU restatement (oracle/sort512_oracle.c) pinned against the reference's
own outputs: the golden fixture made from the reference compiled in place, and,
where the reference library can run here, direct comparison on fresh inputs."""
import os

import numpy as np
import pytest

from helpers import digest, kv_input, pairs_digest


def test_kat_vectors(golden, oracle):
    # the hand-written vectors of sort512test.cpp:169-202 and 290-375
    for case in golden["kat"]:
        a = np.array(case["input"], dtype=case["dtype"])
        oracle.smallsort(a)  # one or two vectors: the leaf sorts them
        assert a.tolist() == case["output"], case


def test_smallsort_digests(golden, oracle):
    for case in golden["smallsort"]:
        st = oracle.rng(case["seed"])
        for d in case["digests"]:
            a = oracle.rand_vec(st, case["n"], case["dtype"])
            oracle.smallsort(a)
            assert digest(a) == d, (case["dtype"], case["n"])


def test_core_small_sort_digests(golden, oracle):
    for case in golden["core_small_sort"]:
        lanes = 16 if case["dtype"] == "int32" else 8
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["nvec"] * lanes, case["dtype"])
        oracle.smallsort(a)
        assert digest(a) == case["digest"], case


def test_sort_digests(golden, oracle):
    for case in golden["sort"]:
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        oracle.sort(a)
        assert digest(a) == case["digest"], (case["dtype"], case["n"])


def test_sort_omp_variants_digests(golden, oracle):
    # every OpenMP driver returns the sorted array; the chunk-sort + merge tree
    # restatement must agree with each of them
    for case in golden["sort_omp"]:
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        if case["fn"] == "sort_omp_partition":
            oracle.sort(a)
        else:
            oracle.sort_chunks_merge(a, 8)
        assert digest(a) == case["digest"], case


def test_partition_bit_exact(golden, oracle):
    # Partition512 is restated step by step: same arrangement, same boundary
    for case in golden["partition"]:
        st = oracle.rng(case["seed"])
        a = oracle.rand_vec(st, case["n"], case["dtype"])
        pivot = np.dtype(case["dtype"]).type(case["pivot"])
        lim = oracle.partition(a, 0, case["n"] - 1, pivot)
        assert lim == case["boundary"], case
        assert digest(a) == case["digest"], case


def test_kv_partition_bit_exact(golden, oracle):
    for case in golden["kv_partition"]:
        st = oracle.rng(case["seed"])
        k, v = kv_input(oracle, st, case["n"])
        lim = oracle.partition_kv(k, v, 0, case["n"] - 1, case["pivot"])
        assert lim == case["boundary"]
        assert digest(k) == case["keys"] and digest(v) == case["values"], case["n"]


def test_kv_sort_keys_and_pairs(golden, oracle):
    for case in golden["kv_sort"]:
        st = oracle.rng(case["seed"])
        k, v = kv_input(oracle, st, case["n"])
        oracle.sort_kv(k, v)
        assert digest(k) == case["keys"], case
        assert pairs_digest(k, v) == case["pairs"], case
    for case in golden["kv_smallsort"]:
        st = oracle.rng(case["seed"])
        k, v = kv_input(oracle, st, case["n"])
        oracle.smallsort_kv(k, v)
        assert digest(k) == case["keys"] and pairs_digest(k, v) == case["pairs"], case


def test_config_c1(golden, oracle):
    import workloads
    a = workloads.uniform_i32_np(1 << 20, 0)
    assert digest(a) == golden["c1"]["input"]
    oracle.sort(a)
    assert digest(a) == golden["c1"]["sorted"]


def test_popcount(oracle):
    # testPopcount (sort512test.cpp:122-146)
    assert oracle.popcount(0) == 0 and oracle.popcount(3) == 2 and oracle.popcount(0xFFFF) == 16
    assert all(oracle.popcount(1 << i) == 1 for i in range(16))


def test_merge_and_segsort(oracle):
    import workloads
    a = workloads.uniform_i32_np(5000, 3)
    a[:2000].sort()
    a[2000:].sort()
    oracle.merge(a, 2000)
    assert np.array_equal(a, np.sort(a))
    lens = workloads.segment_lengths_np(300, 1, mu=3.0)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    x = workloads.uniform_i32_np(int(off[-1]), 2)
    ref = x.copy()
    oracle.segsort(x, off)
    for s in range(len(lens)):
        assert np.array_equal(x[off[s]:off[s + 1]], np.sort(ref[off[s]:off[s + 1]]))


def _reference_or_skip():
    from oracle import Reference, REF_SO, cpu_has_avx512
    if not os.path.exists(REF_SO) or not cpu_has_avx512():
        pytest.skip("reference library not built or host lacks AVX-512")
    return Reference()


def test_restatement_matches_reference_fuzz(oracle):
    ref = _reference_or_skip()
    st = oracle.rng(12345)
    for dt in (np.int32, np.float64):
        for n in [1, 2, 15, 16, 17, 31, 32, 33, 100, 257, 999, 4096, 30011]:
            a = oracle.rand_vec(st, n, dt)
            b, c = a.copy(), a.copy()
            pv = dt(n // 3)
            assert oracle.partition(b, 0, n - 1, pv) == ref.partition(c, 0, n - 1, pv)
            assert np.array_equal(b, c)
            b, c = a.copy(), a.copy()
            oracle.sort(b)
            ref.call("sort", c)
            assert np.array_equal(b, c)
