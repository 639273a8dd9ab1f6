"""ctypes binding of libsort512cuda (the C ABI in include/sort512cuda.h).

Plumbing for tests, the benchmark and Python callers: arrays are numpy arrays
(host memory) or torch CUDA tensors (device memory); the library decides which
by asking the driver.  The C++ drop-in header (include/sort512cuda.hpp) is the
reference-facing interface; this module mirrors its names.

The module refuses to work without the compiled library: there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsort512cuda.so")

S512_OK = 0
S512_ERR_ARG = 1
S512_ERR_ALLOC = 2
S512_ERR_TIMEOUT = 3
S512_ERR_CUDA = 4
S512_ERR_INTERNAL = 5
S512_ERR_UNSUPPORTED = 6

PTR_AUTO, PTR_HOST, PTR_DEVICE = 0, 1, 2
SPLIT_PLAIN, SPLIT_LEARNED = 4, 8
ASYNC = 16

MAX_LEVELS = 8

# Every exported symbol declared in include/sort512cuda.h (checked by the tests).
EXPORTS = (
    "s512_set_config", "s512_get_config", "s512_get_stats", "s512_last_error_string",
    "s512_release_scratch", "s512_version",
    "s512_sort_i32", "s512_sort_f64", "s512_sort_kv_i32",
    "s512_partition_i32", "s512_partition_f64", "s512_partition_kv_i32",
    "s512_smallsort_i32", "s512_smallsort_f64", "s512_smallsort_kv_i32",
    "s512_core_small_sort_i32", "s512_core_small_sort_f64", "s512_core_small_sort_kv_i32",
    "s512_popcount",
    "s512_partition_i32_noalloc",
    "s512_merge_i32", "s512_merge_f64", "s512_sort_omp_merge_i32", "s512_sort_omp_merge_f64",
    "s512_segsort_i32", "s512_segsort_f64", "s512_segsort_kv_i32", "s512_segsort_tune",
    "s512_segsort_plan_create", "s512_segsort_plan_launch", "s512_segsort_plan_destroy",
    "s512_learned_root_grad", "s512_learned_fit",
    "s512_sort_i64", "s512_sort_kv_pairs_i32",
)

DTYPE_I32, DTYPE_F64, DTYPE_KV_I32 = 0, 1, 2


class Config(ctypes.Structure):
    _fields_ = [("splitter_mode", ctypes.c_int), ("collect_stats", ctypes.c_int),
                ("max_imbalance", ctypes.c_double), ("seed", ctypes.c_uint64), ("fault_inject", ctypes.c_int),
                ("device_budget", ctypes.c_uint64)]


FAULT_OVERFLOW, FAULT_REJECT_MODEL, FAULT_ALLOC, FAULT_TIMEOUT = 1, 2, 4, 8


class Stats(ctypes.Structure):
    _fields_ = [
        ("total_ms", ctypes.c_double),
        ("sample_ms", ctypes.c_double * MAX_LEVELS),
        ("partition_ms", ctypes.c_double * MAX_LEVELS),
        ("leaf_ms", ctypes.c_double * MAX_LEVELS),
        ("partition_keys", ctypes.c_uint64 * MAX_LEVELS),
        ("partition_launches", ctypes.c_uint32 * MAX_LEVELS),
        ("levels", ctypes.c_uint32),
        ("fallbacks", ctypes.c_uint32),
        ("learned_levels", ctypes.c_uint32),
        ("learned_rejected", ctypes.c_uint32),
        ("max_bucket_over_mean", ctypes.c_double * MAX_LEVELS),
        ("kernel_launches", ctypes.c_uint32),
        ("key_bytes", ctypes.c_uint32),
        ("bucket_cv", ctypes.c_double * MAX_LEVELS),
        ("fit_ms", ctypes.c_double * MAX_LEVELS),
        ("learned_segments", ctypes.c_uint32 * MAX_LEVELS),
        ("learned_fitted", ctypes.c_uint32 * MAX_LEVELS),
        ("model_max_over_mean", ctypes.c_double * MAX_LEVELS),
    ]

    def as_dict(self) -> dict:
        lv = max(1, int(self.levels))
        return {
            "total_ms": self.total_ms,
            "levels": int(self.levels),
            "sample_ms": list(self.sample_ms[:lv]),
            "partition_ms": list(self.partition_ms[:lv]),
            "leaf_ms": list(self.leaf_ms[:lv]),
            "partition_keys": [int(x) for x in self.partition_keys[:lv]],
            "partition_launches": [int(x) for x in self.partition_launches[:lv]],
            "fallbacks": int(self.fallbacks),
            "learned_levels": int(self.learned_levels),
            "learned_rejected": int(self.learned_rejected),
            "max_bucket_over_mean": list(self.max_bucket_over_mean[:lv]),
            "kernel_launches": int(self.kernel_launches),
            "key_bytes": int(self.key_bytes),
            "bucket_cv": list(self.bucket_cv[:lv]),
            "fit_ms": list(self.fit_ms[:lv]),
            "learned_segments": [int(x) for x in self.learned_segments[:lv]],
            "learned_fitted": [int(x) for x in self.learned_fitted[:lv]],
            "model_max_over_mean": list(self.model_max_over_mean[:lv]),
        }


class Sort512Error(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def build(verbose: bool = False) -> str:
    """Compile libsort512cuda.so in place (nvcc, sm_100a)."""
    out = subprocess.run(["make", "-s", "-C", HERE], capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("building libsort512cuda failed:\n" + (out.stdout or "") + (out.stderr or ""))
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    """Load libsort512cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run build() (make -C avx-512-sort_b200)")
    L = ctypes.CDLL(LIB_PATH)
    vp, sz, ci = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    szp = ctypes.POINTER(ctypes.c_size_t)
    L.s512_set_config.argtypes = [ctypes.POINTER(Config)]
    L.s512_get_config.argtypes = [ctypes.POINTER(Config)]
    L.s512_get_stats.argtypes = [ctypes.POINTER(Stats)]
    L.s512_last_error_string.restype = ctypes.c_char_p
    for suf in ("i32", "f64"):
        getattr(L, f"s512_sort_{suf}").argtypes = [vp, sz, ci, vp]
        getattr(L, f"s512_smallsort_{suf}").argtypes = [vp, sz, ci, vp]
        getattr(L, f"s512_core_small_sort_{suf}").argtypes = [vp, ci, ci, vp]
    L.s512_partition_i32.argtypes = [vp, sz, sz, ctypes.c_int, szp, ci, vp]
    L.s512_partition_f64.argtypes = [vp, sz, sz, ctypes.c_double, szp, ci, vp]
    L.s512_partition_kv_i32.argtypes = [vp, vp, sz, sz, ctypes.c_int, szp, ci, vp]
    L.s512_sort_kv_i32.argtypes = [vp, vp, sz, ci, vp]
    L.s512_sort_i64.argtypes = [vp, sz, ci, vp]
    L.s512_sort_kv_pairs_i32.argtypes = [vp, sz, ci, vp]
    L.s512_smallsort_kv_i32.argtypes = [vp, vp, sz, ci, vp]
    L.s512_core_small_sort_kv_i32.argtypes = [vp, vp, ci, ci, vp]
    L.s512_popcount.argtypes = [ctypes.c_uint]
    L.s512_partition_i32_noalloc.argtypes = [vp, sz, sz, ctypes.c_int, szp, vp]
    for suf in ("i32", "f64"):
        getattr(L, f"s512_merge_{suf}").argtypes = [vp, sz, sz, ci, vp]
        getattr(L, f"s512_sort_omp_merge_{suf}").argtypes = [vp, sz, ci, ci, vp]
        getattr(L, f"s512_segsort_{suf}").argtypes = [vp, vp, sz, ci, vp]
    L.s512_segsort_kv_i32.argtypes = [vp, vp, vp, sz, ci, vp]
    L.s512_segsort_tune.argtypes = [ci, vp, sz, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ci), vp]
    L.s512_segsort_plan_create.argtypes = [ctypes.POINTER(vp), ci, vp, vp, vp, sz, vp]
    L.s512_segsort_plan_launch.argtypes = [vp, vp]
    L.s512_segsort_plan_destroy.argtypes = [vp]
    L.s512_learned_root_grad.argtypes = [ci, vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), vp]
    L.s512_learned_fit.argtypes = [ci, vp, ctypes.c_uint32, ctypes.c_uint64, vp, vp, vp]
    _lib = L
    return L


def _check(fn: str, rc: int) -> None:
    if rc != S512_OK:
        msg = lib().s512_last_error_string()
        raise Sort512Error(fn, rc, msg.decode() if msg else "")


def _ptr(a):
    """(address, n, dtype name, is_device) of a numpy array or torch tensor."""
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be contiguous")
        return a.ctypes.data, a.size, a.dtype.name, False
    import torch  # noqa: F401  (torch tensors only)
    if not a.is_contiguous():
        raise ValueError("tensor must be contiguous")
    name = {"torch.int32": "int32", "torch.float64": "float64", "torch.int64": "int64"}[str(a.dtype)]
    return a.data_ptr(), a.numel(), name, a.is_cuda


def _flags(is_dev: bool, flags: int) -> int:
    return flags | (PTR_DEVICE if is_dev else PTR_HOST)


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def _suffix(dt: str) -> str:
    if dt == "int32":
        return "i32"
    if dt == "float64":
        return "f64"
    if dt == "int64":
        return "i64"
    raise TypeError(f"unsupported dtype {dt}")


# -- Sort512 ------------------------------------------------------------------
def sort(a, flags: int = 0, stream=None) -> None:
    """Sort512::Sort: in-place ascending sort of int32 / float64 / int64 data."""
    p, n, dt, dev = _ptr(a)
    fn = f"s512_sort_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, n, _flags(dev, flags), _stream(stream)))


def sort_pairs(a, flags: int = 0, stream=None) -> None:
    """Sort512kv::Sort on int[2] pairs (key, value) stored interleaved: an
    int32 array of shape (n, 2), sorted by key, then value."""
    if tuple(a.shape[1:]) != (2,):
        raise ValueError("pairs must have shape (n, 2)")
    p, n, dt, dev = _ptr(a)
    if dt != "int32":
        raise TypeError("pairs must be int32")
    _check("s512_sort_kv_pairs_i32", lib().s512_sort_kv_pairs_i32(p, n // 2, _flags(dev, flags), _stream(stream)))


def small_sort(a, flags: int = 0, stream=None) -> None:
    """Sort512::SmallSort16V."""
    p, n, dt, dev = _ptr(a)
    fn = f"s512_smallsort_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, n, _flags(dev, flags), _stream(stream)))


def core_small_sort(a, nvec: int, flags: int = 0, stream=None) -> None:
    """Sort512::CoreSmallSortN pointer forms: nvec consecutive vectors."""
    p, n, dt, dev = _ptr(a)
    fn = f"s512_core_small_sort_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, nvec, _flags(dev, flags), _stream(stream)))


def _check_range(left: int, right: int, n: int) -> bool:
    """Validate an inclusive range [left, right] of an n-element array before
    it reaches the C ABI (which takes size_t and trusts it).  Returns False
    for an empty range (right < left), which needs no call."""
    left, right = int(left), int(right)
    if right < left:
        if left < 0 or left > n:
            raise ValueError(f"empty range starts at {left}, outside 0..{n}")
        return False
    if left < 0 or right >= n:
        raise ValueError(f"range [{left}, {right}] is outside the array's {n} elements")
    return True


def partition(a, left: int, right: int, pivot, flags: int = 0, stream=None) -> int:
    """Sort512::Partition512: returns the first index whose value is > pivot."""
    p, n, dt, dev = _ptr(a)
    if not _check_range(left, right, n):
        return int(left)
    out = ctypes.c_size_t(0)
    fn = f"s512_partition_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, left, right, pivot, ctypes.byref(out), _flags(dev, flags), _stream(stream)))
    return out.value


def merge(a, middle: int, flags: int = 0, stream=None) -> None:
    """Merge the sorted runs a[:middle] and a[middle:] in place (stable)."""
    p, n, dt, dev = _ptr(a)
    fn = f"s512_merge_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, n, middle, _flags(dev, flags), _stream(stream)))


def sort_omp_merge(a, nparts: int = 8, flags: int = 0, stream=None) -> None:
    """Sort512::SortOmpMerge / SortOmpParMerge: chunk sorts + merge-path tree."""
    p, n, dt, dev = _ptr(a)
    fn = f"s512_sort_omp_merge_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, n, nparts, _flags(dev, flags), _stream(stream)))


# -- batched segmented sort ----------------------------------------------------
def _offsets_ptr(offsets):
    if isinstance(offsets, np.ndarray):
        if offsets.dtype != np.uint64 or not offsets.flags.c_contiguous:
            raise ValueError("offsets must be a contiguous uint64 array")
        return offsets.ctypes.data, offsets.size - 1
    return offsets.data_ptr(), offsets.numel() - 1  # torch int64 tensor on the device


def segsort(a, offsets, flags: int = 0, stream=None) -> None:
    """Sort every segment a[offsets[s]:offsets[s+1]] in place."""
    p, n, dt, dev = _ptr(a)
    po, nseg = _offsets_ptr(offsets)
    fn = f"s512_segsort_{_suffix(dt)}"
    _check(fn, getattr(lib(), fn)(p, po, nseg, _flags(dev, flags), _stream(stream)))


def segsort_kv(keys, values, offsets, flags: int = 0, stream=None) -> None:
    pk, n, _, dev = _ptr(keys)
    pv, _, _, _ = _ptr(values)
    po, nseg = _offsets_ptr(offsets)
    _check("s512_segsort_kv_i32", lib().s512_segsort_kv_i32(pk, pv, po, nseg, _flags(dev, flags), _stream(stream)))


def segsort_tune(dtype: int, d_offsets, stream=None):
    """Time the persistent launch's shapes on this layout; returns (best_ms, shape)."""
    po, nseg = _offsets_ptr(d_offsets)
    ms = ctypes.c_double(0)
    shape = ctypes.c_int(-1)
    _check("s512_segsort_tune", lib().s512_segsort_tune(dtype, po, nseg, ctypes.byref(ms), ctypes.byref(shape),
                                                        _stream(stream)))
    return ms.value, shape.value


class SegsortPlan:
    """A segmented sort captured in a CUDA graph (device buffers only)."""

    def __init__(self, dtype: int, keys, d_offsets, values=None, stream=None):
        self.h = ctypes.c_void_p(0)
        po, nseg = _offsets_ptr(d_offsets)
        pk = keys.data_ptr()
        pv = values.data_ptr() if values is not None else None
        _check("s512_segsort_plan_create", lib().s512_segsort_plan_create(ctypes.byref(self.h), dtype, pk, pv, po,
                                                                          nseg, _stream(stream)))

    def launch(self, stream=None) -> None:
        _check("s512_segsort_plan_launch", lib().s512_segsort_plan_launch(self.h, _stream(stream)))

    def close(self) -> None:
        if self.h:
            lib().s512_segsort_plan_destroy(self.h)
            self.h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


# -- Sort512kv ----------------------------------------------------------------
def sort_kv(keys, values, flags: int = 0, stream=None) -> None:
    """Sort512kv::Sort: keys and values are two int32 arrays of the same length."""
    pk, n, dk, dev = _ptr(keys)
    pv, nv, dv, _ = _ptr(values)
    if n != nv or dk != "int32" or dv != "int32":
        raise ValueError("keys and values must be int32 arrays of equal length")
    _check("s512_sort_kv_i32", lib().s512_sort_kv_i32(pk, pv, n, _flags(dev, flags), _stream(stream)))


def small_sort_kv(keys, values, flags: int = 0, stream=None) -> None:
    pk, n, _, dev = _ptr(keys)
    pv, _, _, _ = _ptr(values)
    _check("s512_smallsort_kv_i32", lib().s512_smallsort_kv_i32(pk, pv, n, _flags(dev, flags), _stream(stream)))


def core_small_sort_kv(keys, values, nvec: int, flags: int = 0, stream=None) -> None:
    pk, _, _, dev = _ptr(keys)
    pv, _, _, _ = _ptr(values)
    _check("s512_core_small_sort_kv_i32",
           lib().s512_core_small_sort_kv_i32(pk, pv, nvec, _flags(dev, flags), _stream(stream)))


def partition_kv(keys, values, left: int, right: int, pivot: int, flags: int = 0, stream=None) -> int:
    pk, n, _, dev = _ptr(keys)
    pv, nv, _, _ = _ptr(values)
    if not _check_range(left, right, min(n, nv)):
        return int(left)
    out = ctypes.c_size_t(0)
    _check("s512_partition_kv_i32", lib().s512_partition_kv_i32(pk, pv, left, right, pivot, ctypes.byref(out),
                                                                _flags(dev, flags), _stream(stream)))
    return out.value


def partition_noalloc(a, left: int, right: int, pivot: int, stream=None) -> int:
    """Partition512 on int32 device data without any allocation (fixed scratch
    of NOALLOC_MAX_ELEMS elements)."""
    p, n, dt, dev = _ptr(a)
    if dt != "int32" or not dev:
        raise ValueError("partition_noalloc takes an int32 CUDA tensor")
    if not _check_range(left, right, n):
        return int(left)
    out = ctypes.c_size_t(0)
    _check("s512_partition_i32_noalloc",
           lib().s512_partition_i32_noalloc(p, left, right, pivot, ctypes.byref(out), _stream(stream)))
    return out.value


NOALLOC_MAX_ELEMS = 1 << 20


def popcount(mask: int) -> int:
    return lib().s512_popcount(mask)


# -- configuration / statistics ----------------------------------------------
def get_config() -> Config:
    c = Config()
    _check("s512_get_config", lib().s512_get_config(ctypes.byref(c)))
    return c


def set_config(**kw) -> Config:
    c = get_config()
    for k, v in kw.items():
        setattr(c, k, v)
    _check("s512_set_config", lib().s512_set_config(ctypes.byref(c)))
    return c


def stats() -> dict:
    s = Stats()
    _check("s512_get_stats", lib().s512_get_stats(ctypes.byref(s)))
    return s.as_dict()


def release_scratch() -> None:
    _check("s512_release_scratch", lib().s512_release_scratch())
