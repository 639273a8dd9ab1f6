"""Shared checks for the parity tests."""
from __future__ import annotations

import hashlib

import numpy as np


def digest(*arrays) -> str:
    """sha256(bytes)[:32] -- the digest format of tests/golden/golden.json."""
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


def pairs_digest(k, v) -> str:
    order = np.lexsort((v, k))
    return digest(k[order], v[order])


def kv_input(oracle, st, n):
    """Keys from drand48; value = key*100+1 (sort512test.cpp:241-253) xor the
    index, so that a value moved to the wrong key shows up."""
    k = oracle.rand_vec(st, n, np.int32)
    v = ((k.astype(np.int64) * 100 + 1) ^ np.arange(n)).astype(np.int32)
    return k, v


def assert_sorted(a, what=""):
    a = np.asarray(a)
    if a.size > 1:
        bad = np.nonzero(a[1:] < a[:-1])[0]
        assert bad.size == 0, f"not sorted at {bad[:5] + 1} {what}"


def assert_partitioned(a, pivot, limit, what=""):
    a = np.asarray(a)
    assert np.all(a[:limit] <= pivot), f"low side holds > pivot {what}"
    assert not np.any(a[limit:] <= pivot), f"high side holds <= pivot {what}"


def assert_same_multiset(a, b, what=""):
    assert np.array_equal(np.sort(np.asarray(a), kind="stable"), np.sort(np.asarray(b), kind="stable")), \
        f"multiset changed {what}"


def assert_same_pairs(k1, v1, k2, v2, what=""):
    o1 = np.lexsort((v1, k1))
    o2 = np.lexsort((v2, k2))
    assert np.array_equal(k1[o1], k2[o2]) and np.array_equal(v1[o1], v2[o2]), f"pair multiset changed {what}"


def f64_total_order_key(x: np.ndarray) -> np.ndarray:
    """uint64 keys whose unsigned order is the IEEE total order of doubles."""
    u = np.ascontiguousarray(x, dtype=np.float64).view(np.uint64)
    neg = (u >> np.uint64(63)) == 1
    return np.where(neg, ~u, u | np.uint64(1 << 63))


def sort_f64_total_order(x: np.ndarray) -> np.ndarray:
    return x[np.argsort(f64_total_order_key(x), kind="stable")]
