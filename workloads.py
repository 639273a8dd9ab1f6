"""Seeded synthetic inputs for the sort workloads (CPU numpy and CUDA torch).

The reference publishes no dataset; every workload is synthetic:

* ``uniform_i32``   int32 over the full range: int32(splitmix64(seed, i) >> 32)
* ``uniform01``     double U[0,1): (splitmix64(seed, i) >> 11) * 2^-53
* ``normal``        double N(0,1) by Box-Muller on two uniforms
* ``distinct256``   double, 256 uniform values picked uniformly
* ``ascending`` / ``descending``  sorted doubles
* ``zipf_i32``      Zipf(s) over R ranks (inverse-CDF table), ranks mapped
                    through a seeded permutation of int32 values
* ``gauss_mix``     mixture of 8 Gaussians (means U[lo,hi], sigmas U[slo,shi])
* ``lognormal``     exp(mu + sigma * N(0,1))
* ``drand48``       the reference tests' createRandVec (sort512test.cpp:77-83)

The integer generators are bit-identical between the numpy and torch forms;
the floating ones agree to rounding (they only feed property checks).
"""
from __future__ import annotations

import numpy as np

_M64 = (1 << 64) - 1
_G = 0x9E3779B97F4A7C15
_C1 = 0xBF58476D1CE4E5B9
_C2 = 0x94D049BB133111EB


def splitmix64_np(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """splitmix64 output number i (i = offset .. offset+n-1) for a seed."""
    with np.errstate(over="ignore"):
        i = np.arange(offset, offset + n, dtype=np.uint64)
        z = np.uint64(seed & _M64) + (i + np.uint64(1)) * np.uint64(_G)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(_C1)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(_C2)
        return z ^ (z >> np.uint64(31))


def uniform_i32_np(n: int, seed: int = 0) -> np.ndarray:
    return (splitmix64_np(seed, n) >> np.uint64(32)).astype(np.uint32).view(np.int32)


def uniform01_np(n: int, seed: int = 0) -> np.ndarray:
    return (splitmix64_np(seed, n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def normal_np(n: int, seed: int = 0) -> np.ndarray:
    u1 = uniform01_np(n, seed)
    u2 = uniform01_np(n, seed ^ 0x5BD1E995)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def distinct256_np(n: int, seed: int = 0) -> np.ndarray:
    values = uniform01_np(256, seed ^ 0xD15C)
    idx = (splitmix64_np(seed, n) >> np.uint64(56)).astype(np.int64)
    return values[idx]


def zipf_table(s: float, ranks: int) -> np.ndarray:
    w = 1.0 / np.power(np.arange(1, ranks + 1, dtype=np.float64), s)
    c = np.cumsum(w)
    return c / c[-1]


def zipf_i32_np(n: int, s: float = 1.1, ranks: int = 1 << 20, seed: int = 0) -> np.ndarray:
    cdf = zipf_table(s, ranks)
    u = uniform01_np(n, seed)
    r = np.minimum(np.searchsorted(cdf, u, side="right"), ranks - 1)
    # rank -> a seeded, distinct int32 value (ranks are not ordered by value)
    vals = uniform_i32_np(ranks, seed ^ 0x21F)
    vals = np.unique(vals)
    extra = 0
    while vals.size < ranks:  # practically never: collisions among 2^20 of 2^32
        extra += 1
        vals = np.unique(np.concatenate([vals, uniform_i32_np(ranks, seed ^ (0x21F + extra))]))
    vals = vals[:ranks]
    perm = np.argsort(splitmix64_np(seed ^ 0x9E37, ranks))
    return vals[perm][r].astype(np.int32)


def gauss_mix_np(n: int, seed: int = 0, lo: float = -1e6, hi: float = 1e6,
                 slo: float = 1.0, shi: float = 1e3, k: int = 8) -> np.ndarray:
    p = uniform01_np(3 * k, seed ^ 0xA11CE)
    means = lo + (hi - lo) * p[:k]
    sig = slo + (shi - slo) * p[k:2 * k]
    comp = (splitmix64_np(seed ^ 0xC0, n) % np.uint64(k)).astype(np.int64)
    return means[comp] + sig[comp] * normal_np(n, seed ^ 0x77)


def lognormal_np(n: int, seed: int = 0, mu: float = 0.0, sigma: float = 2.0) -> np.ndarray:
    return np.exp(mu + sigma * normal_np(n, seed))


def segment_lengths_np(nseg: int, seed: int = 0, mu: float = 5.0, sigma: float = 1.5,
                       lo: int = 1, hi: int = 65536) -> np.ndarray:
    z = normal_np(nseg, seed ^ 0x5E6)
    return np.clip(np.round(np.exp(mu + sigma * z)), lo, hi).astype(np.int64)


def double_dist_np(name: str, n: int, seed: int = 0) -> np.ndarray:
    if name == "uniform":
        return uniform01_np(n, seed)
    if name == "normal":
        return normal_np(n, seed)
    if name == "distinct256":
        return distinct256_np(n, seed)
    if name == "ascending":
        return np.sort(uniform01_np(n, seed))
    if name == "descending":
        return np.sort(uniform01_np(n, seed))[::-1].copy()
    if name == "lognormal":
        return lognormal_np(n, seed)
    if name == "gauss_mix":
        return gauss_mix_np(n, seed)
    raise KeyError(name)


DOUBLE_DISTS = ("uniform", "normal", "distinct256", "ascending", "descending")


# ---------------------------------------------------------------------------
# torch (CUDA) forms, for inputs too large to build on the host quickly.

def _torch():
    import torch
    return torch


def _u64(x: int):
    """A Python int in [0, 2^64) as the int64 with the same bits."""
    x &= _M64
    return x - (1 << 64) if x >= (1 << 63) else x


def splitmix64_torch(seed: int, n: int, device="cuda", offset: int = 0):
    torch = _torch()
    i = torch.arange(offset + 1, offset + n + 1, dtype=torch.int64, device=device)
    z = i * _u64(_G) + _u64(seed)

    def lsr(x, s):  # logical shift right on int64 bits
        return (x >> s) & ((1 << (64 - s)) - 1)

    z = (z ^ lsr(z, 30)) * _u64(_C1)
    z = (z ^ lsr(z, 27)) * _u64(_C2)
    return z ^ lsr(z, 31)


def uniform_i32_torch(n: int, seed: int = 0, device="cuda"):
    torch = _torch()
    z = splitmix64_torch(seed, n, device)
    return (z >> 32).to(torch.int32)  # arithmetic shift keeps the high 32 bits


def uniform01_torch(n: int, seed: int = 0, device="cuda"):
    torch = _torch()
    z = splitmix64_torch(seed, n, device)
    return ((z >> 11) & ((1 << 53) - 1)).to(torch.float64) * (2.0 ** -53)


def normal_torch(n: int, seed: int = 0, device="cuda"):
    torch = _torch()
    u1 = uniform01_torch(n, seed, device)
    u2 = uniform01_torch(n, seed ^ 0x5BD1E995, device)
    return torch.sqrt(-2.0 * torch.log1p(-u1)) * torch.cos(2.0 * np.pi * u2)


def double_dist_torch(name: str, n: int, seed: int = 0, device="cuda"):
    torch = _torch()
    if name == "uniform":
        return uniform01_torch(n, seed, device)
    if name == "normal":
        return normal_torch(n, seed, device)
    if name == "distinct256":
        values = torch.from_numpy(uniform01_np(256, seed ^ 0xD15C)).to(device)
        z = splitmix64_torch(seed, n, device)
        return values[(z >> 56) & 0xFF]
    if name == "ascending":
        return torch.sort(uniform01_torch(n, seed, device)).values
    if name == "descending":
        return torch.sort(uniform01_torch(n, seed, device), descending=True).values
    if name == "lognormal":
        return torch.exp(2.0 * normal_torch(n, seed, device))
    if name == "gauss_mix":
        p = uniform01_np(24, seed ^ 0xA11CE)
        means = torch.from_numpy(-1e6 + 2e6 * p[:8]).to(device)
        sig = torch.from_numpy(1.0 + 999.0 * p[8:16]).to(device)
        comp = torch.remainder(splitmix64_torch(seed ^ 0xC0, n, device) & ((1 << 62) - 1), 8)
        return means[comp] + sig[comp] * normal_torch(n, seed ^ 0x77, device)
    raise KeyError(name)


def zipf_i32_torch(n: int, s: float = 1.1, ranks: int = 1 << 20, seed: int = 0, device="cuda"):
    torch = _torch()
    cdf = torch.from_numpy(zipf_table(s, ranks)).to(device)
    u = uniform01_torch(n, seed, device)
    r = torch.clamp(torch.searchsorted(cdf, u, right=True), max=ranks - 1)
    vals = uniform_i32_np(ranks, seed ^ 0x21F)
    vals = np.unique(vals)
    extra = 0
    while vals.size < ranks:
        extra += 1
        vals = np.unique(np.concatenate([vals, uniform_i32_np(ranks, seed ^ (0x21F + extra))]))
    vals = vals[:ranks][np.argsort(splitmix64_np(seed ^ 0x9E37, ranks))]
    return torch.from_numpy(vals.astype(np.int32)).to(device)[r]


def gauss_mix_i32_torch(n: int, seed: int = 0, device="cuda"):
    """Mixture of 8 Gaussians rounded to int32 (means U[-1e6,1e6], sigmas U[1,1e3])."""
    torch = _torch()
    return torch.round(double_dist_torch("gauss_mix", n, seed, device)).to(torch.int32)


# ---------------------------------------------------------------------------
# checks used by the benchmark at full size

def order_keys_torch(t):
    """int64 keys whose signed order is the sort order of t (IEEE total order
    for float64: -0.0 before +0.0, NaNs at the ends by sign)."""
    torch = _torch()
    if t.dtype == torch.float64:
        b = t.view(torch.int64)
        return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFF)
    return t.to(torch.int64)


def multiset_fingerprint_torch(*arrays):
    """An order-independent fingerprint of the multiset of rows (one element
    of each array per row): two wrapping 64-bit sums of differently mixed
    splitmix64 finalisers of the row's bits.  Equal multisets give equal
    fingerprints; a dropped, duplicated or altered element changes them with
    overwhelming probability."""
    torch = _torch()

    def lsr(x, s):
        return (x >> s) & ((1 << (64 - s)) - 1)

    def mix(z):
        z = z + _u64(_G)
        z = (z ^ lsr(z, 30)) * _u64(_C1)
        z = (z ^ lsr(z, 27)) * _u64(_C2)
        return z ^ lsr(z, 31)

    row = None
    for a in arrays:
        b = a.view(torch.int64) if a.element_size() == 8 else a.view(torch.int32).to(torch.int64)
        row = b if row is None else mix(row) ^ b
    h1 = mix(row)
    h2 = mix(h1 ^ 0x5851F42D4C957F2D)
    return int(h1.sum().item()), int(h2.sum().item())


def is_sorted_torch(t) -> bool:
    k = order_keys_torch(t)
    return bool((k[1:] >= k[:-1]).all().item()) if k.numel() > 1 else True
