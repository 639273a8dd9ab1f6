"""Failure detection, exercised without faulting the GPU: every failure is made
on the host side (a capacity shrunk, a model rejected, an allocation refused,
a status word nobody writes waited for with a short bound) and the library
must report it or recover from it, leaving the device usable."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture()
def faults(s512):
    yield s512
    s512.set_config(fault_inject=0, collect_stats=0)


def test_overflow_falls_back_to_exact_counts(faults, cuda):
    import torch
    import workloads
    s512 = faults
    s512.set_config(fault_inject=s512.FAULT_OVERFLOW)
    for t0 in (workloads.uniform_i32_torch(1 << 22, 1), workloads.uniform01_torch(1 << 21, 2)):
        t = t0.clone()
        s512.sort(t)
        assert torch.equal(t, torch.sort(t0).values)
        assert s512.stats()["fallbacks"] >= 1


def test_rejected_models_fall_back_to_splitters(faults, cuda):
    import torch
    import workloads
    s512 = faults
    s512.set_config(fault_inject=s512.FAULT_REJECT_MODEL)
    t0 = workloads.uniform01_torch(1 << 22, 3)
    t = t0.clone()
    s512.sort(t, flags=s512.SPLIT_LEARNED)
    st = s512.stats()
    assert torch.equal(t, torch.sort(t0).values)
    assert st["learned_levels"] == 0 and st["learned_rejected"] >= 1


def test_allocation_failure_is_reported_then_recovers(faults, cuda):
    import torch
    import workloads
    s512 = faults
    s512.release_scratch()
    s512.set_config(fault_inject=s512.FAULT_ALLOC)
    t0 = workloads.uniform_i32_torch(1 << 20, 4)
    t = t0.clone()
    with pytest.raises(s512.Sort512Error) as e:
        s512.sort(t)
    assert e.value.code == s512.S512_ERR_ALLOC
    assert torch.equal(t, t0)  # untouched
    s512.set_config(fault_inject=0)
    s512.sort(t)
    assert torch.equal(t, torch.sort(t0).values)


def test_lookback_timeout_is_reported_and_device_stays_usable(faults, cuda):
    import torch
    import workloads
    s512 = faults
    s512.set_config(fault_inject=s512.FAULT_TIMEOUT)
    t0 = workloads.uniform_i32_torch(1 << 20, 5)
    t = t0.clone()
    with pytest.raises(s512.Sort512Error) as e:
        s512.sort(t)
    assert e.value.code == s512.S512_ERR_TIMEOUT
    assert b"timed out" in s512.lib().s512_last_error_string()
    s512.set_config(fault_inject=0)
    torch.cuda.synchronize()  # the context is intact
    t = t0.clone()
    s512.sort(t)
    assert torch.equal(t, torch.sort(t0).values)


def test_partition_timeout_leaves_the_data_untouched(faults, cuda):
    # Partition512 writes into scratch and copies back only after the kernel
    # reported no error: after an injected look-back timeout the caller's
    # range (device or host memory, keys and values) is as it was
    import numpy as np
    import torch
    import workloads
    s512 = faults
    n = 1 << 20
    k0 = workloads.uniform_i32_torch(n, 6)
    v0 = torch.arange(n, dtype=torch.int32, device=cuda)
    s512.set_config(fault_inject=s512.FAULT_TIMEOUT)
    try:
        k = k0.clone()
        with pytest.raises(s512.Sort512Error) as e:
            s512.partition(k, 0, n - 1, 0)
        assert e.value.code == s512.S512_ERR_TIMEOUT
        assert torch.equal(k, k0)
        hk = k0.cpu().numpy().copy()
        with pytest.raises(s512.Sort512Error) as e:
            s512.partition(hk, 10, n - 11, 0)
        assert e.value.code == s512.S512_ERR_TIMEOUT
        assert np.array_equal(hk, k0.cpu().numpy())
        k, v = k0.clone(), v0.clone()
        with pytest.raises(s512.Sort512Error) as e:
            s512.partition_kv(k, v, 0, n - 1, 0)
        assert e.value.code == s512.S512_ERR_TIMEOUT
        assert torch.equal(k, k0) and torch.equal(v, v0)
        d = workloads.uniform01_torch(n, 7)
        d0 = d.clone()
        with pytest.raises(s512.Sort512Error) as e:
            s512.partition(d, 0, n - 1, 0.5)
        assert e.value.code == s512.S512_ERR_TIMEOUT
        assert torch.equal(d, d0)
    finally:
        s512.set_config(fault_inject=0)
    torch.cuda.synchronize()  # the context is intact
    k = k0.clone()
    lim = s512.partition(k, 0, n - 1, 0)
    assert lim == int((k0 <= 0).sum())
