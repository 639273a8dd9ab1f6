"""The GPU-side steps of the sample sort across ranks (dist_sort): the merge
of the runs a rank receives, through the library's merge-path kernel, and the
single-rank path of sort_sharded (the collectives themselves are tested with
gloo ranks in test_dist_sort.py)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("dtype", ["int32", "float64"])
def test_merge_runs_with_the_merge_kernel(dtype, s512, cuda):
    import torch
    sys.path.insert(0, os.path.join(ROOT, "avx-512-sort_b200"))
    import dist_sort
    rng = np.random.default_rng(4)
    lens = [100000, 0, 77777, 1, 250000, 31, 99999, 5]
    if dtype == "int32":
        runs = [np.sort(rng.integers(-1000, 1000, n).astype(np.int32)) for n in lens]
    else:
        runs = [np.sort(rng.standard_normal(n)) for n in lens]
    t = torch.from_numpy(np.concatenate(runs)).to(cuda)
    dist_sort.merge_runs(t, lens, lambda seg, mid: s512.merge(seg, mid))
    assert np.array_equal(t.cpu().numpy(), np.sort(np.concatenate(runs), kind="stable"))


def test_sort_sharded_single_rank(s512, cuda):
    import datetime
    import socket

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "avx-512-sort_b200"))
    import dist_sort
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True, timeout=datetime.timedelta(seconds=30))
    pg_was = dist.is_initialized()
    if not pg_was:
        dist.init_process_group("nccl", store=store, rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=30))
    try:
        x0 = torch.randn(1 << 20, dtype=torch.float64, device=cuda)
        out = dist_sort.sort_sharded(x0.clone())
        assert torch.equal(out, torch.sort(x0).values)
    finally:
        if not pg_was:
            dist.destroy_process_group()
