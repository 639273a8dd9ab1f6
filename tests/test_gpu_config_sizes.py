"""Parity at the workload sizes themselves: every output is compared in full
with an independent sort (torch.sort on the device) of the same input.

* doubles, 2^28 keys (2 GiB), five distributions (uniform [0,1), standard
  normal, 256 distinct values, ascending, descending), sampled splitters;
* key/value pairs, 2^28, keys uniform over int32 or Zipf(1.1) over 2^20 values,
  value = original index: the output must be the pairs in (key, value) order,
  which checks that keys are exact, that values are a permutation that
  travelled with their keys, and that ties are in value order;
* int32 2^29 (Zipf 1.1 over 2^24 values; 8 Gaussians rounded to int) and
  doubles 2^28 (lognormal(0, 2); 8 Gaussians), plain and learned splitters;
* the batched layout of 200,000 segments (lognormal lengths, mu 5, sigma 1.5,
  clipped to 1..65536), int32, double and key/value, every segment checked,
  through the one-call entry point and the captured plan.

These are the sizes at which offsets and level buffers pass 2^31 elements or
bytes.  Doubles are compared by their IEEE total-order keys (the library's
order: -0.0 before +0.0), bit for bit.  The reference sorts the same values
(sort512.hpp:5960 Sort, sort512kv.hpp:6133 Sort512kv::Sort); its own checker
is a multiset comparison after std::sort (sort512test.cpp:100-119).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N28 = 1 << 28
N29 = 1 << 29


def _order_keys(t):
    """int64 keys whose signed order is the library's order of t."""
    import torch
    if t.dtype == torch.float64:
        b = t.view(torch.int64)
        return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFF)
    return t.to(torch.int64)


def _pairs(k, v):
    """(key, value) as one int64 whose signed order is (key, value) order."""
    import torch
    return k.to(torch.int64) * (1 << 32) + (v.to(torch.int64) + (1 << 31))


def _assert_sorted_like(got, x0):
    import torch
    want = torch.sort(_order_keys(x0)).values
    assert torch.equal(_order_keys(got), want)


@pytest.fixture(autouse=True)
def _free_memory(s512, cuda):
    yield
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dist", ["uniform", "normal", "distinct256", "ascending", "descending"])
def test_double_2p28(dist, s512, cuda):
    import workloads
    x0 = workloads.double_dist_torch(dist, N28, seed=41)
    x = x0.clone()
    s512.sort(x, flags=s512.SPLIT_PLAIN)
    _assert_sorted_like(x, x0)


@pytest.mark.parametrize("keys", ["uniform", "zipf"])
def test_kv_2p28(keys, s512, cuda):
    import torch
    import workloads
    k0 = (workloads.uniform_i32_torch(N28, 42) if keys == "uniform"
          else workloads.zipf_i32_torch(N28, s=1.1, ranks=1 << 20, seed=42))
    v0 = torch.arange(N28, dtype=torch.int32, device=cuda)
    k, v = k0.clone(), v0.clone()
    s512.sort_kv(k, v)
    want = torch.sort(_pairs(k0, v0)).values
    assert torch.equal(_pairs(k, v), want)


@pytest.mark.parametrize("mode", ["plain", "learned"])
@pytest.mark.parametrize("case", ["i32_zipf_2p29", "i32_gauss_mix_2p29", "f64_lognormal_2p28",
                                  "f64_gauss_mix_2p28"])
def test_skewed_plain_and_learned(case, mode, s512, cuda):
    import workloads
    if case == "i32_zipf_2p29":
        x0 = workloads.zipf_i32_torch(N29, s=1.1, ranks=1 << 24, seed=43)
    elif case == "i32_gauss_mix_2p29":
        x0 = workloads.gauss_mix_i32_torch(N29, seed=44)
    elif case == "f64_lognormal_2p28":
        x0 = workloads.double_dist_torch("lognormal", N28, seed=45)
    else:
        x0 = workloads.double_dist_torch("gauss_mix", N28, seed=46)
    x = x0.clone()
    s512.sort(x, flags=s512.SPLIT_LEARNED if mode == "learned" else s512.SPLIT_PLAIN)
    _assert_sorted_like(x, x0)


def _segment_layout(cuda):
    import torch
    import workloads
    lens = workloads.segment_lengths_np(200_000, 31)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    d_off = torch.from_numpy(off.view(np.int64)).to(cuda)
    seg = torch.repeat_interleave(torch.arange(lens.size, device=cuda), torch.from_numpy(lens).to(cuda))
    return off, d_off, seg


def _segmented_reference(key, seg):
    """Every segment sorted by `key` (int64), as a permutation of positions:
    a stable sort by key, then a stable sort by segment."""
    import torch
    p1 = torch.sort(key, stable=True).indices
    p2 = torch.sort(seg[p1], stable=True).indices
    return p1[p2]


@pytest.mark.parametrize("dtype", ["i32", "f64", "kv_i32"])
@pytest.mark.parametrize("api", ["call", "plan"])
def test_segmented_200k_every_segment(dtype, api, s512, cuda):
    import torch
    import workloads
    off, d_off, seg = _segment_layout(cuda)
    total = int(off[-1])
    if dtype == "f64":
        k0 = workloads.uniform01_torch(total, 32, cuda)
    else:
        k0 = workloads.uniform_i32_torch(total, 33, cuda)
    v0 = torch.arange(total, dtype=torch.int32, device=cuda) if dtype == "kv_i32" else None
    k = k0.clone()
    v = v0.clone() if v0 is not None else None
    if api == "call":
        if dtype == "kv_i32":
            s512.segsort_kv(k, v, d_off)
        else:
            s512.segsort(k, d_off)
    else:
        dt = {"i32": s512.DTYPE_I32, "f64": s512.DTYPE_F64, "kv_i32": s512.DTYPE_KV_I32}[dtype]
        plan = s512.SegsortPlan(dt, k, d_off, values=v)
        try:
            for _ in range(2):  # replays start from the same input
                k.copy_(k0)
                if v is not None:
                    v.copy_(v0)
                plan.launch()
            torch.cuda.synchronize()
        finally:
            plan.close()
    if dtype == "kv_i32":
        key0 = _pairs(k0, v0)
        got = _pairs(k, v)
    else:
        key0 = _order_keys(k0)
        got = _order_keys(k)
    assert torch.equal(got, key0[_segmented_reference(key0, seg)])
