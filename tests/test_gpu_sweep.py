"""A seeded sweep over sizes (log-uniform up to 3M keys, plus the class and
level boundaries), key types and value distributions, on host and device
pointers, each result checked against numpy's sort: the cases no single
targeted test pins down (bucket classes at their edges, levels of uneven
segments, runs of ties across leaves)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EDGES = [255, 256, 257, 1023, 1024, 1025, 4096, 4097, 6144, 6145, 8192, 8193, 16384, 16385, 65537]


def _keys(rng, n, kind, dist):
    if dist == "uniform":
        if kind == "f64":
            return rng.standard_normal(n) * rng.choice([1e-300, 1.0, 1e300])
        info = np.iinfo(np.int32 if kind != "i64" else np.int64)
        return rng.integers(info.min, info.max, n, endpoint=True).astype(np.int32 if kind != "i64" else np.int64)
    if dist == "few":
        vals = rng.integers(-50, 50, 7)
    elif dist == "narrow":
        vals = np.arange(1000) * 3
    else:  # "sorted" / "reversed" handled below
        vals = None
    if vals is not None:
        a = rng.choice(vals, n)
    else:
        a = np.sort(rng.integers(-10 ** 6, 10 ** 6, n))
        if dist == "reversed":
            a = a[::-1].copy()
    return a.astype(np.float64 if kind == "f64" else (np.int64 if kind == "i64" else np.int32))


def _cases():
    rng = np.random.default_rng(2024)
    sizes = EDGES + [int(x) for x in np.exp(rng.uniform(np.log(2), np.log(3e6), 24))]
    out = []
    for i, n in enumerate(sizes):
        kind = ["i32", "f64", "i64", "kv", "pairs"][i % 5]
        dist = ["uniform", "few", "narrow", "sorted", "reversed"][(i // 5) % 5]
        out.append((n, kind, dist, bool(i % 2)))
    return out


@pytest.mark.parametrize("n,kind,dist,on_device", _cases())
def test_sweep(n, kind, dist, on_device, s512, cuda):
    import torch
    rng = np.random.default_rng(n * 31 + len(kind) + len(dist))
    if kind in ("kv", "pairs"):
        k = _keys(rng, n, "i32", dist)
        v = rng.integers(-2 ** 31, 2 ** 31 - 1, n).astype(np.int32)
        order = np.lexsort((v, k))
        if kind == "kv":
            kk, vv = (torch.from_numpy(k).to(cuda), torch.from_numpy(v).to(cuda)) if on_device else (k.copy(), v.copy())
            s512.sort_kv(kk, vv)
            kk = kk.cpu().numpy() if on_device else kk
            vv = vv.cpu().numpy() if on_device else vv
            assert np.array_equal(kk, k[order]) and np.array_equal(vv, v[order])
        else:
            p = np.stack([k, v], axis=1)
            pp = torch.from_numpy(p).to(cuda) if on_device else p.copy()
            s512.sort_pairs(pp)
            pp = pp.cpu().numpy() if on_device else pp
            assert np.array_equal(pp, p[order])
        return
    a = _keys(rng, n, kind, dist)
    if kind == "f64":
        key = np.where(np.signbit(a), ~a.view(np.uint64), a.view(np.uint64) | np.uint64(1 << 63))
        want = a[np.argsort(key, kind="stable")]
    else:
        want = np.sort(a)
    t = torch.from_numpy(a).to(cuda) if on_device else a.copy()
    s512.sort(t)
    got = t.cpu().numpy() if on_device else t
    assert np.array_equal(got.view(np.uint64) if kind == "f64" else got,
                          want.view(np.uint64) if kind == "f64" else want), (n, kind, dist)


@pytest.mark.parametrize("layout", range(6))
def test_segsort_sweep(layout, s512, cuda):
    rng = np.random.default_rng(700 + layout)
    nseg = [1, 2, 50, 3000, 400, 9][layout]
    # mixtures of empty, tiny, block-sized and long segments
    lens = rng.choice([0, 1, 3, 200, 257, 4000, 9000, 40000, 150000], nseg,
                      p=[0.1, 0.1, 0.2, 0.2, 0.1, 0.1, 0.1, 0.07, 0.03])
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    n = int(off[-1])
    for dt in (np.int32, np.float64):
        a = (rng.integers(-1000, 1000, n).astype(np.int32) if dt == np.int32 and layout % 2
             else rng.integers(-2 ** 31, 2 ** 31 - 1, n).astype(np.int32) if dt == np.int32
             else rng.standard_normal(n))
        b = a.copy()
        for i in range(nseg):
            b[off[i]:off[i + 1]] = np.sort(b[off[i]:off[i + 1]])
        s512.segsort(a, off)
        assert np.array_equal(a, b), (layout, dt)
