"""s512_partition_i32_noalloc: Partition512 for callers that cannot allocate
device memory (another allocator owns it all, or the host forbids allocations
after start-up).  Its scratch is a fixed device array inside the library, so it
is checked against the allocating entry point, s512_partition_i32, through the
C ABI on two calls in a row, and shown to need no device memory once its
set-up call has run.  The file is collected last; it passes alone in a fresh
process and after the other tests."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_partition_twice(s512, cuda):
    import torch

    import workloads
    lib = s512.lib()
    for n, seed, pivot in ((1 << 20, 1, 123456789), (300007, 2, -50000000)):
        base = workloads.uniform_i32_torch(n, seed)
        a = base.clone()
        b = base.clone()
        got = ctypes.c_size_t(0)
        rc = lib.s512_partition_i32_noalloc(a.data_ptr(), 0, n - 1, pivot, ctypes.byref(got), None)
        assert rc == s512.S512_OK, lib.s512_last_error_string()
        want = s512.partition(b, 0, n - 1, pivot)  # the allocating entry point
        assert got.value == want
        # same kernel, same tiles: identical arrangement (integers: exact)
        assert torch.equal(a, b)
        assert bool((a[:want] <= pivot).all()) and bool((a[want:] > pivot).all())
        assert torch.equal(torch.sort(a).values, torch.sort(base).values)


def test_noalloc_subrange_and_limit(s512, cuda):
    import torch

    import workloads
    n = 5000
    base = workloads.uniform_i32_torch(n, 3)
    a = base.clone()
    lim = s512.partition_noalloc(a, 100, 4099, 0)
    b = base.clone()
    assert lim == s512.partition(b, 100, 4099, 0)
    assert torch.equal(a, b) and torch.equal(a[:100], base[:100]) and torch.equal(a[4100:], base[4100:])
    # a range beyond the fixed scratch is refused with a message, not run
    big = torch.zeros(s512.NOALLOC_MAX_ELEMS + 1, dtype=torch.int32, device=cuda)
    out = ctypes.c_size_t(0)
    rc = s512.lib().s512_partition_i32_noalloc(big.data_ptr(), 0, big.numel() - 1, 0, ctypes.byref(out), None)
    assert rc == s512.S512_ERR_ARG
    assert b"exceed" in s512.lib().s512_last_error_string()


def test_noalloc_needs_no_device_memory_after_setup(s512, cuda):
    # After the set-up call (an empty range), the entry point must work with
    # the device's memory almost all taken by someone else, allocate nothing
    # (the free memory the driver reports is unchanged), and not touch the
    # library's allocating scratch pool (allocations there are made to fail).
    import torch

    import workloads
    lib = s512.lib()
    out = ctypes.c_size_t(0)
    assert lib.s512_partition_i32_noalloc(None, 5, 4, 0, ctypes.byref(out), None) == s512.S512_OK
    assert out.value == 5
    n = 1 << 20
    base = workloads.uniform_i32_torch(n, 11)
    want = base.clone()
    want_lim = s512.partition(want, 0, n - 1, 7)
    s512.release_scratch()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    a = base.clone()
    hog = None
    s512.set_config(fault_inject=s512.FAULT_ALLOC)
    try:
        free, _ = torch.cuda.mem_get_info()
        # leave 256 MB to the rest of the process (torch's own kernels)
        hog = torch.empty(max(0, free - (256 << 20)), dtype=torch.uint8, device=cuda)
        for _ in range(2):
            a.copy_(base)
            torch.cuda.synchronize()
            before, _ = torch.cuda.mem_get_info()
            rc = lib.s512_partition_i32_noalloc(a.data_ptr(), 0, n - 1, 7, ctypes.byref(out), None)
            after, _ = torch.cuda.mem_get_info()
            assert rc == s512.S512_OK, lib.s512_last_error_string()
            assert after == before
            assert out.value == want_lim and torch.equal(a, want)
    finally:
        s512.set_config(fault_inject=0)
        del hog
        torch.cuda.empty_cache()


def test_noalloc_timeout_leaves_the_data_untouched(s512, cuda):
    import torch

    import workloads
    n = 1 << 20
    base = workloads.uniform_i32_torch(n, 12)
    a = base.clone()
    s512.set_config(fault_inject=s512.FAULT_TIMEOUT)
    try:
        with pytest.raises(s512.Sort512Error) as e:
            s512.partition_noalloc(a, 0, n - 1, 0)
        assert e.value.code == s512.S512_ERR_TIMEOUT
    finally:
        s512.set_config(fault_inject=0)
    assert torch.equal(a, base)
    lim = s512.partition_noalloc(a, 0, n - 1, 0)
    assert lim == int((base <= 0).sum())
