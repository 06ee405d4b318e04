"""Seeded synthetic test images (the reference's benchmark photograph is replaced by these).

Every generator is a pure function of its seed, built on numpy's Philox4x32 bit generator:
  * gray(w, h, seed): 128 + sum of 8 sinusoids (orientation U[0, pi), wavelength log-U[4, 128] px,
    amplitude U[10, 40], phase U[0, 2 pi)) + N(0, 6^2), rounded half-to-even, clipped to [0, 255].
  * rgb(w, h, seeds=(100, 101, 102, 103)): channel c = 128 + sqrt(.8) S_shared + sqrt(.2) S_c +
    N(0, 6^2) with S_* zero-mean sinusoid sums as above (channel correlation about 0.8).
  * mixed_set(n=256, seed=300): the uneven batch of log-U[64, 2048] sizes described with it.
The sinusoids are evaluated separably, sin(a x + b y + p) = sin(a x + p) cos(b y) +
cos(a x + p) sin(b y), so a 4096^2 image costs a few outer products.
"""
import math

import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.Philox(key=int(seed)))


def sinusoid_field(w, h, rng, n=8):
    theta = rng.uniform(0.0, math.pi, n)
    lam = np.exp(rng.uniform(math.log(4.0), math.log(128.0), n))
    amp = rng.uniform(10.0, 40.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    xs = np.arange(w, dtype=np.float64)
    ys = np.arange(h, dtype=np.float64)
    f = np.zeros((h, w), np.float64)
    for i in range(n):
        kx = 2.0 * math.pi * math.cos(theta[i]) / lam[i]
        ky = 2.0 * math.pi * math.sin(theta[i]) / lam[i]
        sx = amp[i] * np.sin(kx * xs + phi[i])
        cx = amp[i] * np.cos(kx * xs + phi[i])
        f += np.outer(np.cos(ky * ys), sx)
        f += np.outer(np.sin(ky * ys), cx)
    return f


def _to_u8(f):
    return np.clip(np.rint(f), 0, 255).astype(np.uint8)


def gray(w, h, seed=0):
    rng = _rng(seed)
    f = 128.0 + sinusoid_field(w, h, rng) + 6.0 * rng.standard_normal((h, w))
    return _to_u8(f)


def rgb(w, h, seeds=(100, 101, 102, 103)):
    shared = sinusoid_field(w, h, _rng(seeds[0]))
    out = np.empty((h, w, 3), np.uint8)
    a, b = math.sqrt(0.8), math.sqrt(0.2)
    for c in range(3):
        rng = _rng(seeds[1 + c])
        f = 128.0 + a * shared + b * sinusoid_field(w, h, rng) + 6.0 * rng.standard_normal((h, w))
        out[:, :, c] = _to_u8(f)
    return out


def float_batch(n=16, w=1024, h=1024, seed0=200):
    """Batch of single-channel float32 images in [0, 1] (gray images / 255)."""
    return np.stack([gray(w, h, seed0 + i).astype(np.float32) / 255.0 for i in range(n)])


def mixed_set(n=256, seed=300, lo=64, hi=2048):
    """Descriptors of the uneven batch: list of dicts with w, h, ncomp, kernel, levels, cb, seed.

    Sizes are log-uniform integers in [lo, hi] (odd sizes included); images 0..n/2-1 are
    single-channel and n/2..n-1 RGB; even indices use 5/3, odd 9/7; levels =
    clamp(floor(log2(min(w, h))) - 5, 3, 5); code-blocks 32x32 when index % 4 < 2, else 64x64.
    """
    rng = _rng(seed)
    ws = np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), n))).astype(int)
    hs = np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), n))).astype(int)
    out = []
    for i in range(n):
        w, h = int(min(ws[i], hi)), int(min(hs[i], hi))
        lv = int(min(max(int(math.floor(math.log2(min(w, h)))) - 5, 3), 5))
        out.append(dict(index=i, w=w, h=h, ncomp=1 if i < n // 2 else 3,
                        kernel=53 if i % 2 == 0 else 97, levels=lv,
                        cb=32 if i % 4 < 2 else 64, seed=seed + 1 + i))
    return out


def mixed_image(desc):
    if desc["ncomp"] == 1:
        return gray(desc["w"], desc["h"], desc["seed"])
    s = desc["seed"] * 4
    return rgb(desc["w"], desc["h"], seeds=(s, s + 1, s + 2, s + 3))
