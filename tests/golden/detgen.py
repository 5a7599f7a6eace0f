"""Deterministic integer-only frame generator for the golden fixtures.

Uses only uint32 arithmetic (a counter-based hash, "lowbias32" by C. Wellons, public domain), so
the same (shape, bit depth, seed) gives the same frames with any numpy version; the fixtures store
only expected outputs, never frames.
"""
from __future__ import annotations

import numpy as np


def hash32(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint32).copy()
    x ^= x >> np.uint32(16)
    x *= np.uint32(0x7FEB352D)
    x ^= x >> np.uint32(15)
    x *= np.uint32(0x846CA68B)
    x ^= x >> np.uint32(16)
    return x


def _stream(seed: int, tag: int, n: int) -> np.ndarray:
    base = np.uint32((seed * 0x9E3779B1 + tag * 0x85EBCA77) & 0xFFFFFFFF)
    return hash32(np.arange(n, dtype=np.uint32) ^ base)


def _plane(seed, tag, h, w, maxv, texture):
    y = np.arange(h, dtype=np.int64)[:, None]
    x = np.arange(w, dtype=np.int64)[None, :]
    r = _stream(seed, tag, 4)
    ax, ay = 20 + int(r[0] % 30), 20 + int(r[1] % 30)
    base = (maxv * (ax * x * h + ay * y * w)) // (100 * w * h) + maxv // 8
    noise = (_stream(seed, tag + 1, h * w).astype(np.int64) % (2 * texture + 1)) - texture
    return np.clip(base + noise.reshape(h, w), 0, maxv)


def det_pair(width, height, bitdepth, seed, chroma_format=420, shift=2, block=16, offset=(3, -2, 2), noise=2,
             texture=12):
    """(frame0, frame1): frame1 is frame0 with per-block shifts, a global offset and noise.
    Texture, offset and noise amplitudes are in 8-bit units and scaled to the bit depth."""
    maxv = (1 << bitdepth) - 1
    scale = max(1, maxv // 255)
    dtype = np.uint8 if bitdepth <= 8 else np.uint16
    sx = 0 if chroma_format == 444 else 1
    sy = 1 if chroma_format == 420 else 0
    nby, nbx = -(-height // block), -(-width // block)
    sh = _stream(seed, 7, 2 * nby * nbx).astype(np.int64) % (2 * shift + 1) - shift
    shy, shx = sh[: nby * nbx].reshape(nby, nbx), sh[nby * nbx:].reshape(nby, nbx)
    f0, f1 = [], []
    for c in range(3):
        h = height >> (sy if c else 0)
        w = width >> (sx if c else 0)
        bl = block >> (max(sx, sy) if c else 0)
        ref = _plane(seed, 100 + 10 * c, h, w, maxv, texture * scale)
        by = np.minimum(np.arange(h) // bl, nby - 1)
        bx = np.minimum(np.arange(w) // bl, nbx - 1)
        ys, xs = shy[by][:, bx], shx[by][:, bx]
        if c:
            ys, xs = ys >> sy, xs >> sx
        src_y = np.clip(np.arange(h)[:, None] + ys, 0, h - 1)
        src_x = np.clip(np.arange(w)[None, :] + xs, 0, w - 1)
        nz = (_stream(seed, 200 + c, h * w).astype(np.int64) % (2 * noise * scale + 1)) - noise * scale
        dist = np.clip(ref[src_y, src_x] + offset[c] * scale + nz.reshape(h, w), 0, maxv)
        f0.append(ref.astype(dtype))
        f1.append(dist.astype(dtype))
    return tuple(f0), tuple(f1)


def to444(frame, chroma_format=420):
    """Planar 4:4:4 uint16 (3, H, W) by nearest replication."""
    y = frame[0]
    h, w = y.shape
    sx = 0 if chroma_format == 444 else 1
    sy = 1 if chroma_format == 420 else 0
    out = np.zeros((3, h, w), np.uint16)
    out[0] = y
    for c in (1, 2):
        out[c] = np.repeat(np.repeat(frame[c], 1 << sy, axis=0), 1 << sx, axis=1)[:h, :w]
    return out


def det_mask(width, height, bitdepth, seed, kind="binary"):
    """A mask picture's luma (H, W) for mask mode: 'binary' (0 or the maximum, about 60 % kept),
    'weights' (0..maximum, about 80 % non-zero), 'sparse' (about 5 % non-zero), 'ones' (all maximum),
    'region' (a rectangle kept, the rest masked)."""
    maxv = (1 << bitdepth) - 1
    dtype = np.uint8 if bitdepth <= 8 else np.uint16
    r = _stream(seed, 300, 2 * width * height).astype(np.int64)
    a, b = r[: width * height].reshape(height, width), r[width * height:].reshape(height, width)
    if kind == "binary":
        m = np.where(a % 100 < 60, maxv, 0)
    elif kind == "weights":
        m = np.where(a % 100 < 80, b % (maxv + 1), 0)
    elif kind == "sparse":
        m = np.where(a % 100 < 5, 1 + b % maxv, 0)
    elif kind == "ones":
        m = np.full((height, width), maxv)
    elif kind == "region":
        m = np.zeros((height, width), np.int64)
        m[height // 4: (3 * height) // 4, width // 3: (2 * width) // 3] = maxv
    else:
        raise ValueError(kind)
    return m.astype(dtype)
