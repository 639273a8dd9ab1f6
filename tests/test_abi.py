"""The C-ABI library loads and exports every symbol include/sort512cuda.h
declares (no device work: these run without a GPU)."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "sort512cuda.h")).read()
    return sorted(set(re.findall(r"S512_API\s+[\w\s\*]*?\b(s512_\w+)\s*\(", hdr)))


def test_header_and_binding_agree(s512):
    assert sorted(s512.EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol(s512):
    lib = ctypes.CDLL(s512.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", s512.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (s512_\w+)", out))
    assert set(declared_symbols()) <= exported


def test_library_is_sm100a_only(s512):
    # the fatbinary holds sm_100a code (cuobjdump is not used: the arch list is
    # read from the ELF note nvcc writes)
    out = subprocess.run(["strings", s512.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out or "compute_100a" in out


def test_config_roundtrip_without_device(s512):
    c = s512.get_config()
    assert c.splitter_mode == s512.SPLIT_PLAIN
    assert c.max_imbalance >= 1.0
    s512.set_config(seed=1234)
    assert s512.get_config().seed == 1234
    s512.set_config(seed=0x5EED)
    bad = s512.Config(99, 0, 3.0, 1, 0)
    assert s512.lib().s512_set_config(ctypes.byref(bad)) == s512.S512_ERR_ARG


def test_popcount_host_only(s512):
    # popcount is a host function (the reference's is a scalar helper)
    assert s512.popcount(0) == 0 and s512.popcount(0xFFFF) == 16 and s512.popcount(0x1FFFF) == 16


def test_cpp_header_compiles():
    src = os.path.join(ROOT, "tests", "cpp", "sort512cuda_test.cpp")
    r = subprocess.run(["/usr/bin/g++", "-std=c++14", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_no_cpu_fallback_in_product():
    # the product sources never reference the CPU oracle
    pkg = os.path.join(ROOT, "avx-512-sort_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".cu", ".cuh", ".py", ".hpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.lower(), f


def test_arguments_checked_before_any_device_work(s512):
    lib = s512.lib()
    assert lib.s512_sort_i32(None, 10, 0, None) == s512.S512_ERR_ARG
    assert lib.s512_sort_f64(None, 10, 0, None) == s512.S512_ERR_ARG
    assert lib.s512_sort_i64(None, 10, 0, None) == s512.S512_ERR_ARG
    assert lib.s512_sort_kv_pairs_i32(None, 10, 0, None) == s512.S512_ERR_ARG
    a = (ctypes.c_int * 4)()
    assert lib.s512_sort_kv_i32(a, None, 4, 0, None) == s512.S512_ERR_ARG
    # an empty array is a no-op (undefined in the reference)
    assert lib.s512_sort_i32(None, 0, 0, None) == 0
    assert lib.s512_sort_f64(None, 0, 0, None) == 0


def test_no_device_fails_loudly(s512):
    # without a B200 the library reports it and leaves the data untouched: no
    # host fallback sorts behind the caller's back
    import torch
    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is present")
    import numpy as np
    a = np.arange(100, dtype=np.int32)[::-1].copy()
    rc = s512.lib().s512_sort_i32(a.ctypes.data, a.size, 0, None)
    assert rc == s512.S512_ERR_UNSUPPORTED
    assert s512.lib().s512_last_error_string()
    assert np.array_equal(a, np.arange(100, dtype=np.int32)[::-1])


def test_partition_ranges_are_checked_before_the_call(s512):
    # an index past the array (or a negative one, which size_t would wrap)
    # is refused in Python and never reaches the library, so no device work
    # starts; an empty range returns `left` without a call
    import numpy as np
    import pytest
    a = np.arange(10, dtype=np.int32)
    for left, right in ((0, 10), (-1, 5), (3, 12), (11, 20)):
        with pytest.raises(ValueError):
            s512.partition(a, left, right, 4)
    with pytest.raises(ValueError):
        s512.partition_kv(a, a[:5].copy(), 0, 7, 4)
    assert s512.partition(a, 5, 4, 0) == 5
    assert s512.partition(a, 0, -1, 0) == 0
