"""CPU oracle of the learned splitter model's root -- TEST INFRASTRUCTURE ONLY.

The model is this project's own (the reference has no learned part): a
piecewise-linear CDF of 256 pieces over the key range with slopes w = theta^2
(pieces as root_pieces computes them).  This module recomputes, in float64, the loss the device
trainer minimises and its analytic gradient, so the device's hand-written
forward/backward pass can be checked against it; finite differences check the
analytic gradient itself.
"""
from __future__ import annotations

import numpy as np

R = 256


def encode_i32(x: np.ndarray) -> np.ndarray:
    return (x.astype(np.int32).view(np.uint32) ^ np.uint32(0x80000000)).astype(np.uint32)


def encode_f64(x: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(x, dtype=np.float64).view(np.uint64)
    neg = (u >> np.uint64(63)) == 1
    return np.where(neg, ~u, u | np.uint64(1 << 63))


def root_pieces(keys: np.ndarray):
    """Piece index and fraction of every (sorted, encoded) sample key, in the
    device's float32 arithmetic: zr = float32(key - kmin) * (R / float32(kmax -
    kmin)), piece = min(floor(zr), R - 1), fraction = min(zr - piece, 1)."""
    k = keys.astype(np.uint64)
    kmin = k[0]
    rng = k[-1] - kmin
    zscale = np.float32(R) / np.float32(rng) if rng > 0 else np.float32(0.0)
    zr = ((k - kmin).astype(np.float32) * zscale).astype(np.float32)
    s = np.minimum(np.floor(zr), np.float32(R - 1)).astype(np.float32)
    frac = np.minimum(zr - s, np.float32(1.0))
    return s.astype(np.int64), frac.astype(np.float64)


def root_loss_grad(keys: np.ndarray, theta: np.ndarray):
    """Loss mean((p0 - y)^2) and dL/dtheta, y_i = (i + 0.5) / m."""
    theta = np.asarray(theta, dtype=np.float64)
    s, frac = root_pieces(keys)
    m = len(keys)
    w = theta * theta
    c = np.cumsum(w) - w
    p0 = c[s] + w[s] * frac
    y = (np.arange(m) + 0.5) / m
    r = p0 - y
    loss = float(np.mean(r * r))
    s0 = np.bincount(s, weights=r, minlength=R)
    s1 = np.bincount(s, weights=r * frac, minlength=R)
    later = np.concatenate([np.cumsum(s0[::-1])[::-1][1:], [0.0]])  # sum over pieces > t
    gw = 2.0 / m * (later + s1)
    return loss, gw * 2.0 * theta


def root_init_theta(keys: np.ndarray) -> np.ndarray:
    """The trainer's start: theta = sqrt(fraction of the sample in each piece)."""
    s, _ = root_pieces(keys)
    return np.sqrt(np.bincount(s, minlength=R) / len(keys))


def finite_difference(keys: np.ndarray, theta: np.ndarray, eps: float = 1e-6) -> np.ndarray:
    g = np.zeros(R)
    for t in range(R):
        tp = theta.copy()
        tm = theta.copy()
        tp[t] += eps
        tm[t] -= eps
        g[t] = (root_loss_grad(keys, tp)[0] - root_loss_grad(keys, tm)[0]) / (2 * eps)
    return g
