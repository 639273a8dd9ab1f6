"""Sample sort across ranks: every rank holds a shard, the result is the
sorted concatenation of all shards, range-partitioned over the ranks (rank r
ends with keys no larger than any key of rank r+1).

The reference sorts one array in one address space (Sort512::SortOmpPartition,
sort512.hpp:5993-6004, a task quicksort over OpenMP threads).  Across GPUs the
same method becomes one sample-sort level whose exchange step is a single
all-to-all over NVLink / NVSwitch:

  1. each rank sorts its shard (libsort512cuda),
  2. takes `oversample` evenly spaced keys of it as its sample,
  3. the samples are all-gathered and sorted; P-1 splitters are their
     quantiles,
  4. each rank cuts its sorted shard at the splitters (a binary search per
     splitter), exchanges the run lengths and then the runs (all_to_all),
  5. each rank merges the P sorted runs it received (merge-path kernel,
     log2 P rounds of pairwise merges).

torch.distributed carries the collectives (NCCL on GPUs, gloo on CPU); the
local sort and merges are this library's kernels.  The local steps can be
swapped (`local_sort`, `merge`) so that the exchange logic runs on CPU ranks
too.
"""
from __future__ import annotations

from typing import Callable, Optional


def _default_sort(t):
    import sort512cuda
    sort512cuda.sort(t)


def _default_merge(t, middle: int):
    import sort512cuda
    sort512cuda.merge(t, middle)


def order_keys(t):
    """Integers whose order is the library's sort order of `t`: the values
    themselves for integer tensors; for float64 the IEEE total order (-NaN
    first, then -inf .. -0.0, +0.0 .. +inf, +NaN last), as int64 whose signed
    order matches it.  The cut points are searched in these keys, since IEEE
    compares do not order NaNs and tie -0.0 with +0.0."""
    import torch
    if t.dtype != torch.float64:
        return t
    b = t.view(torch.int64)
    return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFF)


def splitters_from_samples(samples, nranks: int):
    """P-1 splitters at the quantiles of the sorted, gathered sample."""
    m = samples.numel()
    if nranks <= 1 or m == 0:
        return samples[:0]
    idx = [(i * m) // nranks for i in range(1, nranks)]
    return samples[idx]


def merge_runs(t, counts, merge: Callable) -> None:
    """Merge the sorted runs laid end to end in t (lengths `counts`) in place,
    pairing neighbours until one run is left."""
    bounds = [0]
    for c in counts:
        bounds.append(bounds[-1] + int(c))
    runs = [(bounds[i], bounds[i + 1]) for i in range(len(counts))]
    while len(runs) > 1:
        nxt = []
        for i in range(0, len(runs), 2):
            if i + 1 == len(runs):
                nxt.append(runs[i])
                continue
            (a0, a1), (b0, b1) = runs[i], runs[i + 1]
            if a1 > a0 and b1 > b0:
                merge(t[a0:b1], a1 - a0)
            nxt.append((a0, b1))
        runs = nxt


def sort_sharded(x, group=None, oversample: int = 256, local_sort: Optional[Callable] = None,
                 merge: Optional[Callable] = None):
    """Sort the union of every rank's 1-D shard `x` across the process group.

    Returns this rank's part of the result (a new tensor, sorted); parts are
    ordered by rank.  `x` itself is sorted in place on the way (step 1).
    Every rank must call it (it runs collectives).  Ties: keys equal to a
    splitter go to the lower rank, so a run of equal keys is not split.
    """
    import torch
    import torch.distributed as dist

    local_sort = local_sort or _default_sort
    merge = merge or _default_merge
    P = dist.get_world_size(group)
    if x.dim() != 1:
        raise ValueError("shard must be 1-D")
    local_sort(x)
    if P == 1:
        return x.clone()

    # 2-3. regular sample of the sorted shard, gathered and sorted
    n = x.numel()
    s = max(1, oversample)
    if n:
        pos = torch.div(torch.arange(s, device=x.device, dtype=torch.int64) * n + n // 2, s,
                        rounding_mode="floor").clamp_(max=n - 1)
        sample = x[pos]
    else:
        sample = x.new_empty(0)
    # shards may be empty: pad every sample to s keys with the shard's own
    # values or, for an empty shard, with a flag marking it unused
    have = torch.tensor([1 if n else 0], device=x.device, dtype=torch.int64)
    pad = sample if n else x.new_zeros(s)
    gathered = [torch.empty_like(pad) for _ in range(P)]
    dist.all_gather(gathered, pad, group=group)
    flags = [torch.empty_like(have) for _ in range(P)]
    dist.all_gather(flags, have, group=group)
    used = [g for g, f in zip(gathered, flags) if int(f.item())]
    allsamp = torch.cat(used) if used else x.new_empty(0)
    local_sort(allsamp)
    spl = splitters_from_samples(allsamp, P)

    # 4. cut points: keys <= splitter r (in the sort's order) go to ranks <= r
    if spl.numel():
        cuts = torch.searchsorted(order_keys(x).contiguous(), order_keys(spl).contiguous(),
                                  right=True).to(torch.int64)
    else:
        cuts = torch.zeros(P - 1, dtype=torch.int64, device=x.device)
    edges = torch.cat([torch.zeros(1, dtype=torch.int64, device=x.device), cuts,
                       torch.tensor([n], dtype=torch.int64, device=x.device)])
    send_counts = (edges[1:] - edges[:-1]).contiguous()
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts, group=group)
    send_sizes = [int(c) for c in send_counts.tolist()]
    recv_sizes = [int(c) for c in recv_counts.tolist()]
    out = x.new_empty(sum(recv_sizes))
    dist.all_to_all_single(out, x, output_split_sizes=recv_sizes, input_split_sizes=send_sizes, group=group)

    # 5. merge the P sorted runs received
    merge_runs(out, recv_sizes, merge)
    return out
