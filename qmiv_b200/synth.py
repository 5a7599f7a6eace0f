"""Seeded synthetic frame pairs standing in for the MPEG test sequences (not in this container).

Every workload has the shapes, bit depths, 4:2:0 layout and value distributions of the configuration
it stands in for:

* reference frame: a smooth 2-D gradient plus Gaussian texture, clipped to the bit depth's range;
* distorted frame: the reference with every 16x16 block (8x8 in 4:2:0 chroma) shifted by a seeded
  integer offset, a global per-component offset added, Gaussian noise, rounded and clipped;
  optionally blurred with a seeded Gaussian.

Frames are tuples (Y, Cb, Cr) of numpy arrays, uint8 for bit depth 8, uint16 otherwise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def _gradient_texture(rng, h, w, maxv, tex_sigma):
    yy = np.linspace(0.0, 1.0, h, dtype=np.float32)[:, None]
    xx = np.linspace(0.0, 1.0, w, dtype=np.float32)[None, :]
    a, b = rng.uniform(0.12, 0.28, 2)
    fx, fy, ph = rng.uniform(0.5, 3.0), rng.uniform(0.5, 3.0), rng.uniform(0, 2 * math.pi)
    base = maxv * (0.16 + a * xx + b * yy + 0.06 * np.sin(2 * math.pi * (fx * xx + fy * yy) + ph))
    return base.astype(np.float32) + rng.normal(0.0, tex_sigma, (h, w)).astype(np.float32)


def _block_shift(img, shifts_y, shifts_x, block):
    h, w = img.shape
    by = np.minimum(np.arange(h) // block, shifts_y.shape[0] - 1)
    bx = np.minimum(np.arange(w) // block, shifts_y.shape[1] - 1)
    sy = np.clip(np.arange(h)[:, None] + shifts_y[by][:, bx], 0, h - 1)
    sx = np.clip(np.arange(w)[None, :] + shifts_x[by][:, bx], 0, w - 1)
    return img[sy, sx]


def _blur(img, sigma):
    if not sigma:
        return img
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(img, sigma, mode="nearest")


def make_pair(width, height, bitdepth=8, seed=0, chroma_format=420, shift_range=2, block=16,
              offset=(3, -2, 2), noise_sigma=2.0, texture_sigma=12.0, blur_sigma=None):
    """One (reference, distorted) pair. Offsets and sigmas are given in 8-bit units and scaled."""
    rng = np.random.default_rng(seed)
    maxv = (1 << bitdepth) - 1
    scale = maxv / 255.0
    dtype = np.uint8 if bitdepth <= 8 else np.uint16
    sx = 0 if chroma_format == 444 else 1
    sy = 1 if chroma_format == 420 else 0
    nby, nbx = -(-height // block), -(-width // block)
    shy = rng.integers(-shift_range, shift_range + 1, (nby, nbx))
    shx = rng.integers(-shift_range, shift_range + 1, (nby, nbx))
    ref, dist = [], []
    for c in range(3):
        h = height >> (sy if c else 0)
        w = width >> (sx if c else 0)
        base = _gradient_texture(rng, h, w, maxv, texture_sigma * scale)
        r = np.clip(np.rint(base), 0, maxv)
        if c == 0:
            d = _block_shift(r, shy, shx, block)
        else:
            d = _block_shift(r, shy >> sy if sy else shy, shx >> sx if sx else shx, block >> max(sx, sy))
        d = d + offset[c] * scale + rng.normal(0.0, noise_sigma * scale, (h, w)).astype(np.float32)
        d = _blur(d, blur_sigma)
        ref.append(np.ascontiguousarray(r, dtype=dtype))
        dist.append(np.ascontiguousarray(np.clip(np.rint(d), 0, maxv), dtype=dtype))
    return tuple(ref), tuple(dist)


# ------------------------------------------------------------------------------------------------
# the five workloads
# ------------------------------------------------------------------------------------------------
def config0(seed=0):
    """IV-PSNR plain: one 1920x1080 8-bit 4:2:0 pair, R=2."""
    return [make_pair(1920, 1080, 8, seed)]


def config1(n=8, seed=1, width=4096, height=2048):
    """IV-PSNR + WS-PSNR + IV-SSIM: 4096x2048 10-bit 4:2:0 ERP pairs, noise sigma 8 (10-bit units)."""
    return [make_pair(width, height, 10, seed + i, noise_sigma=2.0, texture_sigma=12.0) for i in range(n)]


def config2(n=16, seed=2, size=2048):
    """MS-SSIM / IV-MS-SSIM: 2048x2048 10-bit pairs with a seeded blur sigma in [0.5, 2]."""
    rng = np.random.default_rng(seed)
    sig = rng.uniform(0.5, 2.0, n)
    return [make_pair(size, size, 10, seed * 1000 + i, blur_sigma=float(sig[i])) for i in range(n)]


CONFIG3_RESOLUTIONS = [(1280, 720), (1920, 1080), (2048, 2048), (4096, 2048)]


def config3_specs(n=64, seed=3):
    """Shapes of the batched uneven set: resolution, bit depth, R drawn uniformly."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w, h = CONFIG3_RESOLUTIONS[rng.integers(0, 4)]
        out.append(dict(width=w, height=h, bitdepth=int(rng.choice([8, 10])), search_range=int(rng.choice([2, 4])),
                        seed=seed * 10000 + i))
    return out


def config3(n=64, seed=3):
    specs = config3_specs(n, seed)
    for s in specs:
        s["frame0"], s["frame1"] = make_pair(s["width"], s["height"], s["bitdepth"], s["seed"])
    return specs


@dataclass
class Request:
    arrival_s: float
    specs: list = field(default_factory=list)
    metrics: int = 0


def config4_requests(duration_s=1.0, rate=200.0, seed=4, max_pairs=32):
    """Poisson arrivals: each request is a sequence of 1..max_pairs pairs of one shape drawn as config 3,
    with a metric set drawn from {IV-PSNR, IV-PSNR+PSNR, IV-PSNR+PSNR+IV-SSIM}."""
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    metric_sets = [4, 4 | 1, 4 | 1 | 32]
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            break
        w, h = CONFIG3_RESOLUTIONS[rng.integers(0, 4)]
        bd = int(rng.choice([8, 10]))
        r = int(rng.choice([2, 4]))
        npairs = int(rng.integers(1, max_pairs + 1))
        specs = [dict(width=w, height=h, bitdepth=bd, search_range=r, seed=int(rng.integers(0, 2**31)))
                 for _ in range(npairs)]
        reqs.append(Request(t, specs, metric_sets[rng.integers(0, 3)]))
    return reqs


def make_mask(width, height, bitdepth=8, seed=0, keep=0.6, block=16):
    """A mask picture's luma for mask mode: blocks of `block` x `block` samples kept (at the maximum
    value) with probability `keep`, the rest masked (0), from a seeded generator."""
    rng = np.random.default_rng(seed)
    maxv = (1 << bitdepth) - 1
    nby, nbx = -(-height // block), -(-width // block)
    keepb = rng.random((nby, nbx)) < keep
    m = np.repeat(np.repeat(keepb, block, axis=0), block, axis=1)[:height, :width]
    return np.where(m, maxv, 0).astype(np.uint8 if bitdepth <= 8 else np.uint16)
