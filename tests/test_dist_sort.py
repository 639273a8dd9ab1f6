"""The sample sort across ranks (dist_sort.sort_sharded): sample, splitters,
cut points, the all-to-all exchange and the merge of received runs, run with
gloo ranks on the CPU.  The two local steps are the library's kernels on GPU
ranks; here they are stood in for by torch's CPU sort, so that the exchange
logic itself is what is tested."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard(rank, case):
    rng = np.random.default_rng(1000 * case + rank)
    if case == 0:
        return rng.integers(-2 ** 31, 2 ** 31 - 1, 5000 + 1000 * rank).astype(np.int32)
    if case == 1:  # many repeats, one empty shard
        return np.zeros(0, np.int32) if rank == 1 else rng.integers(0, 7, 3000).astype(np.int32)
    if case == 2:
        return rng.standard_normal(4000 - 500 * rank)  # float64
    # float64 with signed zeros, infinities and NaNs of both signs
    x = rng.standard_normal(3000 + 300 * rank)
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan] * (40 + 10 * rank))
    x[rng.choice(x.size, special.size, replace=False)] = special
    return x


def _total_order_key(a):
    """int64 keys whose signed order is the IEEE total order of float64."""
    b = np.ascontiguousarray(a, dtype=np.float64).view(np.int64)
    return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFF)


def _sort_like_library(a):
    if a.dtype != np.float64:
        return np.sort(a)
    return a[np.argsort(_total_order_key(a), kind="stable")]


def _rank_main(rank, world, port, case, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "avx-512-sort_b200"))
    import dist_sort

    # the library's order: IEEE total order for doubles (-0.0 before +0.0,
    # NaNs at the ends by sign)
    def cpu_sort(t):
        if t.dtype == torch.float64:
            t.copy_(t[torch.argsort(dist_sort.order_keys(t), stable=True)])
        else:
            t.copy_(torch.sort(t).values)

    def cpu_merge(t, middle):
        cpu_sort(t)

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        x = torch.from_numpy(_shard(rank, case))
        part = dist_sort.sort_sharded(x, oversample=32, local_sort=cpu_sort, merge=cpu_merge)
        out.put((rank, part.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [(2, 0), (3, 1), (3, 2), (2, 3), (3, 3)])
def test_sharded_sort_is_the_sorted_union(world, case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    union = _sort_like_library(np.concatenate([_shard(r, case) for r in range(world)]))
    joined = np.concatenate([got[r] for r in range(world)])
    # bit-exact (NaN payloads and signed zeros included)
    assert joined.dtype == union.dtype and np.array_equal(joined.view(np.uint8), union.view(np.uint8))
    for r in range(world - 1):  # range partitioned, in the library's order
        if got[r].size and got[r + 1].size:
            if union.dtype == np.float64:
                assert _total_order_key(got[r][-1:])[0] <= _total_order_key(got[r + 1][:1])[0]
            else:
                assert got[r][-1] <= got[r + 1][0]


def test_merge_runs_pairs_neighbours():
    sys.path.insert(0, os.path.join(ROOT, "avx-512-sort_b200"))
    import torch

    import dist_sort
    runs = [np.sort(np.random.default_rng(i).integers(0, 100, n)) for i, n in enumerate([5, 0, 7, 3, 9])]
    t = torch.from_numpy(np.concatenate(runs))
    calls = []

    def merge(seg, middle):
        calls.append((seg.numel(), middle))
        a = seg.numpy().copy()
        seg.copy_(torch.from_numpy(np.concatenate([a[:middle], a[middle:]])))
        seg.copy_(torch.sort(seg).values)

    dist_sort.merge_runs(t, [r.size for r in runs], merge)
    assert np.array_equal(t.numpy(), np.sort(np.concatenate(runs)))
    assert len(calls) == 3  # (5,0) skipped as empty, (7,3), then (5,10), then (15,9)
