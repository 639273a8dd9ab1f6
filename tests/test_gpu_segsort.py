"""Batched segmented sort (a persistent launch for short segments, partition
levels for long ones) against the restated per-segment sort of the reference
(the reference sorts a batch by looping SmallSort16V / Sort over the arrays,
sort512perf.cpp:612-709)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _layout(nseg, seed, mu=5.0, sigma=1.5):
    import workloads
    lens = workloads.segment_lengths_np(nseg, seed, mu=mu, sigma=sigma)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)


@pytest.mark.parametrize("dt", [np.int32, np.float64])
def test_segsort_host_matches_restatement(dt, s512, cuda, oracle):
    import workloads
    off = _layout(3000, 1)
    n = int(off[-1])
    a = workloads.uniform_i32_np(n, 5) if dt == np.int32 else workloads.uniform01_np(n, 5)
    b = a.copy()
    s512.segsort(a, off)
    oracle.segsort(b, off)
    assert np.array_equal(a, b)


def test_segsort_edge_layouts(s512, cuda, oracle):
    import workloads
    # empty segments, single keys, exactly 256 / 257, every block class's
    # limit and one past it, long ones
    lens = [0, 1, 2, 0, 255, 256, 257, 1024, 1025, 2048, 2049, 4096, 4097, 8192, 8193, 16384, 16385, 70000, 3, 0]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    a = workloads.uniform_i32_np(int(off[-1]), 7)
    a[1000:1500] = 42  # a run of equal keys
    b = a.copy()
    s512.segsort(a, off)
    oracle.segsort(b, off)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("lens", [[3, 100001, 5], [70001], [1, 0, 40000, 2]])
def test_segsort_one_long_segment(lens, s512, cuda, oracle):
    # exactly one segment above a block's capacity, at an odd offset or alone:
    # it runs the partition levels as a batch of one
    import workloads
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    for dt in (np.int32, np.float64):
        n = int(off[-1])
        a = workloads.uniform_i32_np(n, 8) if dt == np.int32 else workloads.uniform01_np(n, 8)
        b = a.copy()
        s512.segsort(a, off)
        oracle.segsort(b, off)
        assert np.array_equal(a, b), (lens, dt)


def test_segsort_device_and_kv(s512, cuda):
    import torch
    import workloads
    off = _layout(20000, 2)
    n = int(off[-1])
    d_off = torch.from_numpy(off.view(np.int64)).to(cuda)
    k0 = workloads.uniform_i32_torch(n, 9)
    v0 = torch.arange(n, dtype=torch.int32, device=cuda)
    k, v = k0.clone(), v0.clone()
    s512.segsort_kv(k, v, d_off)
    seg_id = torch.repeat_interleave(torch.arange(len(off) - 1, device=cuda),
                                     torch.from_numpy(np.diff(off).astype(np.int64)).to(cuda))
    # values stay with their keys and inside their segment
    assert torch.equal(k0[v.long()], k)
    assert torch.equal(seg_id[v.long()], seg_id)
    # each segment sorted by (key, value)
    same_seg = seg_id[1:] == seg_id[:-1]
    up = (k[1:] > k[:-1]) | ((k[1:] == k[:-1]) & (v[1:] > v[:-1]))
    assert bool(up[same_seg].all())


def test_segsort_plan_graph_and_tuner(s512, cuda):
    import torch
    import workloads
    off = _layout(50000, 3)
    n = int(off[-1])
    d_off = torch.from_numpy(off.view(np.int64)).to(cuda)
    ms, shape = s512.segsort_tune(s512.DTYPE_F64, d_off)
    assert ms > 0 and 0 <= shape < 4
    x0 = workloads.uniform01_torch(n, 4)
    x = x0.clone()
    plan = s512.SegsortPlan(s512.DTYPE_F64, x, d_off)
    for rep in range(3):  # replay on fresh data each time
        x.copy_(workloads.uniform01_torch(n, 10 + rep))
        ref = x.clone().cpu().numpy()
        plan.launch()
        torch.cuda.synchronize()
        got = x.cpu().numpy()
        for s in range(0, len(off) - 1, 997):
            lo, hi = int(off[s]), int(off[s + 1])
            assert np.array_equal(got[lo:hi], np.sort(ref[lo:hi]))
        assert np.array_equal(np.sort(got), np.sort(ref))
    plan.close()
