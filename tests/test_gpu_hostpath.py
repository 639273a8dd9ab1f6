"""Host-pointer sorts (the reference sorts host memory in place,
sort512.hpp:5960, sort512kv.hpp:6133): page-locked arrays are copied in by
chunks that the first partition level consumes as they land, and with
S512_ASYNC the call returns before the result is copied back, so calls on two
streams overlap; every stream has its own scratch pool.  Checked against a
sort of the same input on the device."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned_copy(t):
    import torch
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t.cpu())
    return h


def _keys(t):
    import workloads
    return workloads.order_keys_torch(t)


def _pair(k, v):
    import torch
    return k.to(torch.int64) * (1 << 32) + (v.to(torch.int64) + (1 << 31))


@pytest.mark.parametrize("dtype,n", [("f64", (1 << 23) + 4097), ("i32", (1 << 24) + 3), ("i64", 1 << 22)])
def test_pinned_host_sort_chunked(dtype, n, s512, cuda):
    import torch
    import workloads
    if dtype == "f64":
        d0 = workloads.double_dist_torch("normal", n, seed=61, device=cuda)
    elif dtype == "i32":
        d0 = workloads.uniform_i32_torch(n, 62, cuda)
    else:
        d0 = workloads.splitmix64_torch(63, n, cuda)
    h = _pinned_copy(d0)
    s512.sort(h.numpy())
    assert torch.equal(_keys(h.to(cuda)), torch.sort(_keys(d0)).values)


def test_pinned_host_kv_and_pairs_chunked(s512, cuda):
    import torch
    import workloads
    n = (1 << 22) + 77
    k0 = workloads.zipf_i32_torch(n, seed=64, device=cuda)
    v0 = torch.arange(n, dtype=torch.int32, device=cuda)
    hk, hv = _pinned_copy(k0), _pinned_copy(v0)
    s512.sort_kv(hk.numpy(), hv.numpy())
    assert torch.equal(_pair(hk.to(cuda), hv.to(cuda)), torch.sort(_pair(k0, v0)).values)
    p0 = torch.stack([k0, v0], dim=1).contiguous()
    hp = _pinned_copy(p0)
    s512.sort_pairs(hp.numpy())
    got = hp.to(cuda)
    assert torch.equal(_pair(got[:, 0], got[:, 1]), torch.sort(_pair(k0, v0)).values)


def test_async_host_calls_on_two_streams_overlap_correctly(s512, cuda):
    # each call returns once its copy back is queued; the next call, on the
    # other stream and its own pool, copies its input in meanwhile
    import torch
    import workloads
    n = 1 << 23
    inputs = [workloads.uniform01_torch(n, 70 + i, cuda) for i in range(5)]
    hosts = [_pinned_copy(x) for x in inputs]
    streams = [torch.cuda.Stream(device=cuda), torch.cuda.Stream(device=cuda)]
    torch.cuda.synchronize()
    for i, h in enumerate(hosts):
        s512.sort(h.numpy(), flags=s512.ASYNC, stream=streams[i % 2])
    for st in streams:
        st.synchronize()
    for x, h in zip(inputs, hosts):
        assert torch.equal(h.to(cuda), torch.sort(x).values)


def test_pageable_host_memory_is_waited_for(s512, cuda):
    # pageable memory cannot be copied asynchronously: the call waits even
    # with S512_ASYNC
    import workloads
    a = workloads.uniform_i32_np((1 << 20) + 5, 71)
    want = np.sort(a)
    s512.sort(a, flags=s512.ASYNC)
    assert np.array_equal(a, want)


def test_two_threads_two_streams(s512, cuda):
    # calls on different streams use different pools and may run at once
    import torch
    import workloads
    n = 1 << 22
    xs = [workloads.uniform_i32_torch(n, 80 + i, cuda) for i in range(2)]
    wants = [torch.sort(x).values for x in xs]
    outs = [None, None]
    errors = []

    def work(i):
        try:
            torch.cuda.set_device(cuda)
            st = torch.cuda.Stream(device=cuda)
            with torch.cuda.stream(st):
                for _ in range(3):
                    y = xs[i].clone()
                    s512.sort(y, stream=st)
                    outs[i] = y
            st.synchronize()
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    ts = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    for o, w in zip(outs, wants):
        assert torch.equal(o, w)
