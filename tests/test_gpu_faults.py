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
