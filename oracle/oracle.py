"""CPU checkers for the sort path -- TEST INFRASTRUCTURE ONLY.

Two libraries, both built by ``oracle/Makefile``:

* ``liboracle.so`` -- the plain-C restatement of the reference's algorithm
  (``sort512_oracle.c``).  Always available (plain C).
* ``_ref/libsort512ref.so`` -- the reference's own headers compiled in place
  behind a C-ABI shim (``ref_shim.cpp``).  Needs an AVX-512 host to run.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module, and only as the checker or as the timed CPU
baseline.  The GPU library never calls into it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsort512ref.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_size_t = ctypes.c_size_t


class Rng48(ctypes.Structure):
    """State of the reference tests' drand48 generator."""

    _fields_ = [("x", ctypes.c_uint64)]


def build(ref: bool = True) -> None:
    """Build liboracle.so (and the reference shim when the sources exist)."""
    targets = ["oracle"] + (["ref-if-present"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
    except OSError:
        return False
    need = ("avx512f", "avx512cd", "avx512vl", "avx512bw", "avx512dq")
    return all(f" {x}" in flags for x in need)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Oracle:
    """ctypes view of liboracle.so (the C restatement)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        self.lib = lib = ctypes.CDLL(path)
        lib.oracle_srand48.argtypes = [ctypes.POINTER(Rng48), ctypes.c_long]
        lib.oracle_drand48.argtypes = [ctypes.POINTER(Rng48)]
        lib.oracle_drand48.restype = ctypes.c_double
        lib.oracle_rand_vec_i32.argtypes = [ctypes.POINTER(Rng48), _c_int_p, _c_size_t]
        lib.oracle_rand_vec_f64.argtypes = [ctypes.POINTER(Rng48), _c_double_p, _c_size_t]
        lib.oracle_popcount.argtypes = [ctypes.c_uint]
        lib.oracle_popcount.restype = ctypes.c_int
        for suf, cp, ct in (("i32", _c_int_p, ctypes.c_int), ("f64", _c_double_p, ctypes.c_double)):
            getattr(lib, f"oracle_sort_{suf}").argtypes = [cp, _c_size_t]
            getattr(lib, f"oracle_smallsort_{suf}").argtypes = [cp, _c_size_t]
            f = getattr(lib, f"oracle_partition_{suf}")
            f.argtypes = [cp, _c_size_t, _c_size_t, ct]
            f.restype = _c_size_t
            getattr(lib, f"oracle_merge_{suf}").argtypes = [cp, _c_size_t, _c_size_t]
            getattr(lib, f"oracle_sort_chunks_merge_{suf}").argtypes = [cp, _c_size_t, ctypes.c_int]
            getattr(lib, f"oracle_segsort_{suf}").argtypes = [cp, ctypes.POINTER(_c_size_t), _c_size_t]
        lib.oracle_sort_kv_i32.argtypes = [_c_int_p, _c_int_p, _c_size_t]
        lib.oracle_smallsort_kv_i32.argtypes = [_c_int_p, _c_int_p, _c_size_t]
        lib.oracle_partition_kv_i32.argtypes = [_c_int_p, _c_int_p, _c_size_t, _c_size_t, ctypes.c_int]
        lib.oracle_partition_kv_i32.restype = _c_size_t
        lib.oracle_segsort_kv_i32.argtypes = [_c_int_p, _c_int_p, ctypes.POINTER(_c_size_t), _c_size_t]

    # -- generators -------------------------------------------------------
    def rng(self, seed: int = 0) -> Rng48:
        st = Rng48()
        self.lib.oracle_srand48(ctypes.byref(st), seed)
        return st

    def rand_vec(self, st: Rng48, n: int, dtype) -> np.ndarray:
        """createRandVec (sort512test.cpp:77-83): T(drand48()*n)."""
        dtype = np.dtype(dtype)
        a = np.empty(n, dtype=dtype)
        if dtype == np.int32:
            self.lib.oracle_rand_vec_i32(ctypes.byref(st), _ptr(a, ctypes.c_int), n)
        else:
            self.lib.oracle_rand_vec_f64(ctypes.byref(st), _ptr(a, ctypes.c_double), n)
        return a

    # -- path ---------------------------------------------------------------
    @staticmethod
    def _suf(a: np.ndarray):
        if a.dtype == np.int32:
            return "i32", ctypes.c_int
        if a.dtype == np.float64:
            return "f64", ctypes.c_double
        raise TypeError(a.dtype)

    def sort(self, a: np.ndarray) -> None:
        suf, ct = self._suf(a)
        getattr(self.lib, f"oracle_sort_{suf}")(_ptr(a, ct), a.size)

    def smallsort(self, a: np.ndarray) -> None:
        suf, ct = self._suf(a)
        getattr(self.lib, f"oracle_smallsort_{suf}")(_ptr(a, ct), a.size)

    def partition(self, a: np.ndarray, left: int, right: int, pivot) -> int:
        suf, ct = self._suf(a)
        return getattr(self.lib, f"oracle_partition_{suf}")(_ptr(a, ct), left, right, pivot)

    def merge(self, a: np.ndarray, middle: int) -> None:
        suf, ct = self._suf(a)
        getattr(self.lib, f"oracle_merge_{suf}")(_ptr(a, ct), a.size, middle)

    def sort_chunks_merge(self, a: np.ndarray, parts: int) -> None:
        suf, ct = self._suf(a)
        getattr(self.lib, f"oracle_sort_chunks_merge_{suf}")(_ptr(a, ct), a.size, parts)

    def segsort(self, a: np.ndarray, offsets: np.ndarray) -> None:
        suf, ct = self._suf(a)
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        getattr(self.lib, f"oracle_segsort_{suf}")(_ptr(a, ct), _ptr(off, _c_size_t), off.size - 1)

    def sort_kv(self, k: np.ndarray, v: np.ndarray) -> None:
        self.lib.oracle_sort_kv_i32(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int), k.size)

    def smallsort_kv(self, k: np.ndarray, v: np.ndarray) -> None:
        self.lib.oracle_smallsort_kv_i32(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int), k.size)

    def partition_kv(self, k, v, left: int, right: int, pivot: int) -> int:
        return self.lib.oracle_partition_kv_i32(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int), left, right, pivot)

    def segsort_kv(self, k, v, offsets) -> None:
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.lib.oracle_segsort_kv_i32(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int),
                                       _ptr(off, _c_size_t), off.size - 1)

    def popcount(self, m: int) -> int:
        return self.lib.oracle_popcount(m)


class Reference:
    """ctypes view of _ref/libsort512ref.so (the reference compiled in place)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        if not cpu_has_avx512():
            raise RuntimeError("host CPU lacks AVX-512 F/CD/VL/BW/DQ; the reference cannot run here")
        self.lib = lib = ctypes.CDLL(path)
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_max_threads.restype = ctypes.c_int
        lib.ref_popcount.argtypes = [ctypes.c_uint]
        lib.ref_popcount.restype = ctypes.c_int
        for suf, cp, ct in (("i32", _c_int_p, ctypes.c_int), ("f64", _c_double_p, ctypes.c_double)):
            for fn in ("sort", "sort_omp_partition", "sort_omp_merge", "sort_omp_merge_deps",
                       "sort_omp_parmerge", "smallsort"):
                getattr(lib, f"ref_{fn}_{suf}").argtypes = [cp, _c_size_t]
            f = getattr(lib, f"ref_partition_{suf}")
            f.argtypes = [cp, _c_size_t, _c_size_t, ct]
            f.restype = _c_size_t
            f = getattr(lib, f"ref_core_small_sort_{suf}")
            f.argtypes = [cp, ctypes.c_int]
            f.restype = ctypes.c_int
        for fn in ("sort", "sort_omp_partition", "smallsort"):
            getattr(lib, f"ref_{fn}_kv_i32").argtypes = [_c_int_p, _c_int_p, _c_size_t]
        lib.ref_partition_kv_i32.argtypes = [_c_int_p, _c_int_p, _c_size_t, _c_size_t, ctypes.c_int]
        lib.ref_partition_kv_i32.restype = _c_size_t
        lib.ref_core_small_sort_kv_i32.argtypes = [_c_int_p, _c_int_p, ctypes.c_int]
        lib.ref_core_small_sort_kv_i32.restype = ctypes.c_int

    def set_threads(self, n: int) -> None:
        self.lib.ref_set_threads(n)

    def max_threads(self) -> int:
        return self.lib.ref_max_threads()

    @staticmethod
    def _suf(a):
        return Oracle._suf(a)

    def call(self, fn: str, a: np.ndarray) -> None:
        """fn in sort, sort_omp_partition, sort_omp_merge, sort_omp_merge_deps,
        sort_omp_parmerge, smallsort."""
        suf, ct = self._suf(a)
        getattr(self.lib, f"ref_{fn}_{suf}")(_ptr(a, ct), a.size)

    def partition(self, a, left, right, pivot) -> int:
        suf, ct = self._suf(a)
        return getattr(self.lib, f"ref_partition_{suf}")(_ptr(a, ct), left, right, pivot)

    def core_small_sort(self, a: np.ndarray, nvec: int) -> None:
        suf, ct = self._suf(a)
        rc = getattr(self.lib, f"ref_core_small_sort_{suf}")(_ptr(a, ct), nvec)
        assert rc == 0

    def call_kv(self, fn: str, k: np.ndarray, v: np.ndarray) -> None:
        getattr(self.lib, f"ref_{fn}_kv_i32")(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int), k.size)

    def partition_kv(self, k, v, left, right, pivot) -> int:
        return self.lib.ref_partition_kv_i32(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int), left, right, pivot)

    def core_small_sort_kv(self, k, v, nvec) -> None:
        rc = self.lib.ref_core_small_sort_kv_i32(_ptr(k, ctypes.c_int), _ptr(v, ctypes.c_int), nvec)
        assert rc == 0

    def popcount(self, m: int) -> int:
        return self.lib.ref_popcount(m)
