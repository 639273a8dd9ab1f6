"""Generate tests/golden/golden.json from the reference compiled in place.

Run where the reference sources are (oracle/Makefile's REFDIR) on an
AVX-512 CPU:

    make -C oracle all && python tests/golden/make_golden.py

The fixture stores, for each case, how to regenerate the input (generator,
seed, size) and the reference's output as a SHA-256 digest of its bytes, plus
the known-answer vectors of sort512test.cpp (169-202, 290-375) with the
reference's outputs in full.  Tests regenerate the inputs with the C
restatement's drand48 or the splitmix64 generator and compare digests, so the
fixture stays a few KB.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from oracle import Oracle, Reference  # noqa: E402
import workloads  # noqa: E402


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


def pairs_digest(k, v) -> str:
    order = np.lexsort((v, k))
    return digest(k[order], v[order])


def kat_vectors():
    """The hand-written known-answer vectors of sort512test.cpp."""
    out = []
    d8 = np.arange(1, 9, dtype=np.float64)
    i16 = np.arange(1, 17, dtype=np.int32)
    out += [("core1", d8), ("core1", d8[::-1].copy()), ("core1", i16), ("core1", i16[::-1].copy())]
    d16 = np.repeat(np.arange(1, 9, dtype=np.float64), 2)
    i32 = np.repeat(np.arange(1, 17, dtype=np.int32), 2)
    for base, half in ((d16, 8), (i32, 16)):
        asc = base
        desc = base[::-1].copy()
        swapped = np.concatenate([base[half:], base[:half]])
        swapped_desc = np.concatenate([base[:half][::-1], base[half:][::-1]])
        out += [("core2", asc), ("core2", desc), ("core2", swapped), ("core2", swapped_desc)]
    return out


def main():
    o = Oracle()
    r = Reference()
    r.set_threads(min(8, os.cpu_count() or 1))
    g = {"about": "Reference outputs (berenger-eu/avx-512-sort compiled in place) for the "
                  "inputs described per case; digests are sha256(bytes)[:32].",
         "kat": [], "smallsort": [], "sort": [], "sort_omp": [], "partition": [],
         "kv_sort": [], "kv_partition": [], "kv_smallsort": [], "core_small_sort": [], "c1": {}}

    for kind, v in kat_vectors():
        a = v.copy()
        if kind == "core1":
            r.core_small_sort(a, 1)
        else:
            r.core_small_sort(a, 2)
        g["kat"].append({"kind": kind, "dtype": str(v.dtype), "input": v.tolist(), "output": a.tolist()})

    # SmallSort16V: every length 1..16 vectors, 2 trials, drand48 seeded per length
    for dt, lim in ((np.int32, 256), (np.float64, 128)):
        for n in range(1, lim + 1):
            st = o.rng(1000 + n)
            outs = []
            for _t in range(2):
                a = o.rand_vec(st, n, dt)
                r.call("smallsort", a)
                outs.append(digest(a))
            g["smallsort"].append({"dtype": np.dtype(dt).name, "n": n, "seed": 1000 + n, "trials": 2,
                                   "digests": outs})

    # CoreSmallSortN pointer forms: N vectors, drand48 seeded per N
    for dt, lanes in ((np.int32, 16), (np.float64, 8)):
        for nv in range(1, 17):
            st = o.rng(500 + nv)
            a = o.rand_vec(st, nv * lanes, dt)
            r.core_small_sort(a, nv)
            g["core_small_sort"].append({"dtype": np.dtype(dt).name, "nvec": nv, "seed": 500 + nv,
                                         "digest": digest(a)})

    sizes = [1, 2, 3, 4, 8, 16, 31, 64, 100, 128, 255, 256, 257, 512, 1000, 1024, 2048, 4097,
             8192, 10000, 65536, 100003, 1 << 18]
    for dt in (np.int32, np.float64):
        for n in sizes:
            st = o.rng(n)
            a = o.rand_vec(st, n, dt)
            b = a.copy()
            r.call("sort", b)
            g["sort"].append({"dtype": np.dtype(dt).name, "n": n, "seed": n, "gen": "drand48",
                              "digest": digest(b)})
        for n in (1, 2, 4, 16, 128, 1000, 1024, 4096, 100003):
            st = o.rng(n)
            a = o.rand_vec(st, n, dt)
            for fn in ("sort_omp_partition", "sort_omp_merge", "sort_omp_merge_deps", "sort_omp_parmerge"):
                b = a.copy()
                r.call(fn, b)
                g["sort_omp"].append({"fn": fn, "dtype": np.dtype(dt).name, "n": n, "seed": n,
                                      "gen": "drand48", "digest": digest(b)})

    # Partition512: every n in 1..1000 and powers of two to 2^16, pivot = n/2
    pn = list(range(1, 1001)) + [1 << k for k in range(10, 17)]
    for dt in (np.int32, np.float64):
        for n in pn:
            st = o.rng(7 * n + 1)
            a = o.rand_vec(st, n, dt)
            b = a.copy()
            lim = r.partition(b, 0, n - 1, dt(n // 2))
            g["partition"].append({"dtype": np.dtype(dt).name, "n": n, "seed": 7 * n + 1, "pivot": n // 2,
                                   "boundary": int(lim), "digest": digest(b)})

    # key/value: value = key*100+1 (sort512test.cpp:241-253) xor the index, so
    # that value swaps between equal keys would show up in the pair multiset
    def kv_input(st, n):
        k = o.rand_vec(st, n, np.int32)
        v = ((k.astype(np.int64) * 100 + 1) ^ np.arange(n)).astype(np.int32)
        return k, v

    for n in sizes:
        st = o.rng(3 * n + 2)
        k, v = kv_input(st, n)
        for fn in ("sort", "sort_omp_partition"):
            k2, v2 = k.copy(), v.copy()
            r.call_kv(fn, k2, v2)
            g["kv_sort"].append({"fn": fn, "n": n, "seed": 3 * n + 2, "keys": digest(k2),
                                 "pairs": pairs_digest(k2, v2)})
    for n in range(1, 257):
        st = o.rng(3 * n + 2)
        k, v = kv_input(st, n)
        r.call_kv("smallsort", k, v)
        g["kv_smallsort"].append({"n": n, "seed": 3 * n + 2, "keys": digest(k), "pairs": pairs_digest(k, v)})
    for n in pn:
        st = o.rng(11 * n + 5)
        k, v = kv_input(st, n)
        lim = r.partition_kv(k, v, 0, n - 1, n // 2)
        g["kv_partition"].append({"n": n, "seed": 11 * n + 5, "pivot": n // 2, "boundary": int(lim),
                                  "keys": digest(k), "values": digest(v)})

    # Config C1: int32 n=2^20 uniform over the full range, seed 0
    a = workloads.uniform_i32_np(1 << 20, 0)
    b = a.copy()
    r.call("sort", b)
    g["c1"] = {"n": 1 << 20, "gen": "uniform_i32(splitmix64 seed 0)", "input": digest(a), "sorted": digest(b)}

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(g, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
