"""The 64-bit words the reference's interface names but does not implement:
int64 keys, and int key/value pairs stored interleaved as int[2] (the
reference's README.md:6; its kv interface takes two arrays,
sort512kv.hpp:6133).  Checked against numpy / torch sorts and against the
two-array kv sort of this library on the same pairs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 255, 300, 16384, 16385, 123457, 1 << 22])
def test_sort_int64(n, s512, cuda):
    rng = np.random.default_rng(n)
    a = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64, endpoint=True)
    if n > 4:
        a[:3] = [np.iinfo(np.int64).min, np.iinfo(np.int64).max, 0]
    want = np.sort(a)
    s512.sort(a)
    assert np.array_equal(a, want)


def test_sort_int64_device_narrow_and_repeated(s512, cuda):
    import torch
    g = torch.Generator(device=cuda).manual_seed(3)
    for lo, hi in ((-(1 << 62), 1 << 62), (-5, 5), (1 << 40, (1 << 40) + 1000)):
        t0 = torch.randint(lo, hi, ((1 << 23) + 77,), generator=g, device=cuda, dtype=torch.int64)
        t = t0.clone()
        s512.sort(t)
        assert torch.equal(t, torch.sort(t0).values)


@pytest.mark.parametrize("n", [1, 3, 256, 257, 5000, 16385, 1 << 20, (1 << 22) + 5])
def test_sort_int_pairs(n, s512, cuda):
    rng = np.random.default_rng(n + 1)
    p = np.empty((n, 2), np.int32)
    p[:, 0] = rng.integers(-(n // 8) - 1, n // 8 + 1, n)  # repeated keys
    p[:, 1] = rng.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, endpoint=True)
    if n > 4:
        p[0] = (np.iinfo(np.int32).max, np.iinfo(np.int32).min)
        p[1] = (np.iinfo(np.int32).min, np.iinfo(np.int32).max)
    order = np.lexsort((p[:, 1], p[:, 0]))
    want = p[order]
    k, v = p[:, 0].copy(), p[:, 1].copy()
    s512.sort_pairs(p)
    assert np.array_equal(p, want)
    # same order as the two-array form of Sort512kv::Sort
    s512.sort_kv(k, v)
    assert np.array_equal(p[:, 0], k) and np.array_equal(p[:, 1], v)


def test_sort_int_pairs_device(s512, cuda):
    import torch
    g = torch.Generator(device=cuda).manual_seed(9)
    n = 1 << 23
    t = torch.randint(-(1 << 31), (1 << 31) - 1, (n, 2), generator=g, device=cuda, dtype=torch.int32)
    keys = t[:, 0].to(torch.int64)
    vals = t[:, 1].to(torch.int64)
    comb = keys * (1 << 32) + (vals + (1 << 31))
    want = torch.sort(comb).values
    s512.sort_pairs(t)
    got = t[:, 0].to(torch.int64) * (1 << 32) + (t[:, 1].to(torch.int64) + (1 << 31))
    assert torch.equal(got, want)
