"""Host arrays larger than the device budget: the streamed external sort
(sorted runs, then output pieces cut at exact ranks and sorted on the
device).  A small s512_config.device_budget makes arrays of a few million
keys take that path; results are compared with numpy's sort."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BUDGET = 32 << 20  # bytes: pieces of ~0.7 M int32 / 0.35 M double keys


@pytest.fixture
def small_budget(s512):
    s512.set_config(device_budget=BUDGET)
    try:
        yield
    finally:
        s512.set_config(device_budget=0)


@pytest.mark.parametrize("n", [(1 << 22) + 3, 3 << 20])
def test_streamed_int32(n, s512, cuda, small_budget):
    import workloads
    a = workloads.uniform_i32_np(n, 12)
    want = np.sort(a)
    s512.sort(a)
    assert np.array_equal(a, want)


def test_streamed_double_with_specials(s512, cuda, small_budget):
    rng = np.random.default_rng(5)
    n = (1 << 21) + 12345
    a = rng.standard_normal(n) * 1e3
    a[rng.integers(0, n, 5000)] = rng.choice([0.0, -0.0, np.inf, -np.inf, 5e-324, -5e-324], 5000)
    key = np.where(np.signbit(a), ~a.view(np.uint64), a.view(np.uint64) | np.uint64(1 << 63))
    want = a[np.argsort(key, kind="stable")]
    s512.sort(a)
    assert np.array_equal(a.view(np.uint64), want.view(np.uint64))


def test_streamed_int64(s512, cuda, small_budget):
    rng = np.random.default_rng(8)
    n = (1 << 21) + 7
    a = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64, endpoint=True)
    want = np.sort(a)
    s512.sort(a)
    assert np.array_equal(a, want)


@pytest.mark.parametrize("values", [1, 3, 1000])
def test_streamed_repeated_keys(values, s512, cuda, small_budget):
    # ties across run boundaries: cut ranks fall inside runs of equal keys
    rng = np.random.default_rng(values)
    a = rng.integers(0, values, 3 << 20).astype(np.int32)
    want = np.sort(a)
    s512.sort(a)
    assert np.array_equal(a, want)


def test_device_arrays_are_not_streamed(s512, cuda, small_budget):
    import torch
    t0 = torch.randint(-(1 << 31), (1 << 31) - 1, (1 << 21,), device=cuda, dtype=torch.int32)
    t = t0.clone()
    s512.sort(t)  # device memory: the budget concerns host arrays only
    assert torch.equal(t, torch.sort(t0).values)


@pytest.mark.parametrize("distinct", [None, 17])
def test_streamed_kv_pairs(distinct, s512, cuda, small_budget):
    # Sort512kv::Sort on two host arrays past the budget: pairs end in
    # (key, value) order, values travel with their keys
    import workloads
    n = (1 << 21) + 333
    if distinct is None:
        k = workloads.uniform_i32_np(n, 21)
    else:  # ties across run boundaries, broken by the values
        k = (workloads.uniform_i32_np(n, 21) % distinct).astype(np.int32)
    v = workloads.uniform_i32_np(n, 22)
    order = np.lexsort((v, k))
    wk, wv = k[order], v[order]
    s512.sort_kv(k, v)
    assert np.array_equal(k, wk) and np.array_equal(v, wv)
