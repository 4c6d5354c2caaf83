"""Seeded synthetic inputs for the lattice workloads.

The generator is counter-based (SplitMix64 over (seed, stream, index)), so the same seed
gives the same bytes on every machine and in every process; the CPU checkers and the
GPU path are always fed identical float32 arrays.

Images are planar float32 arrays shaped (channels, height, width) — the channel-major
layout of ImageStack's Image (src/Image.h:34-43) with one frame.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z += np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, stream: int, n: int) -> np.ndarray:
    """n float64 values uniform in [0, 1) from stream `stream` of `seed`."""
    base = _splitmix(np.array([(seed * 0x100000001B3 + stream * 0x9E3779B1) & 0xFFFFFFFFFFFFFFFF],
                              dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        idx = np.arange(n, dtype=np.uint64) * np.uint64(0xD1B54A32D192ED03) + base
    u = _splitmix(idx) >> np.uint64(11)
    return u.astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    """n standard normal float64 values (Box-Muller on two uniform streams)."""
    u1 = uniform(seed, stream, n)
    u2 = uniform(seed, stream + 7919, n)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def image(width: int, height: int, channels: int = 3, rects: int = 16, seed: int = 0,
          noise: float = 0.05) -> np.ndarray:
    """Smooth linear gradients + `rects` constant-colour rectangles + Gaussian noise,
    clamped to [0, 1]; planar float32 (channels, height, width)."""
    out = np.empty((channels, height, width), dtype=np.float64)
    abc = uniform(seed, 1, 3 * channels).reshape(channels, 3) * 0.5
    xs = np.arange(width, dtype=np.float64) / width
    ys = np.arange(height, dtype=np.float64) / height
    for k in range(channels):
        out[k] = abc[k, 0] * xs[None, :] + abc[k, 1] * ys[:, None] + abc[k, 2]
    if rects:
        r = uniform(seed, 2, rects * (4 + channels)).reshape(rects, 4 + channels)
        for i in range(rects):
            x0 = int(r[i, 0] * width)
            y0 = int(r[i, 1] * height)
            w = int(1 + r[i, 2] * max(width / 4 - 1, 0))
            h = int(1 + r[i, 3] * max(height / 4 - 1, 0))
            out[:, y0:y0 + h, x0:x0 + w] = r[i, 4:4 + channels][:, None, None]
    out += noise * normal(seed, 3, out.size).reshape(out.shape)
    np.clip(out, 0.0, 1.0, out=out)
    return out.astype(np.float32)


def luminance(rgb: np.ndarray) -> np.ndarray:
    """Grey guide 0.299 r + 0.587 g + 0.114 b in float32; shape (1, h, w)."""
    r, g, b = rgb[0], rgb[1], rgb[2]
    lum = (np.float32(0.299) * r + np.float32(0.587) * g) + np.float32(0.114) * b
    return lum[None].astype(np.float32)


def gauss_mixture(n: int, d: int = 16, centres: int = 32, spread: float = 10.0,
                  std: float = 0.5, value_channels: int = 4, seed: int = 0):
    """Points of a mixture of isotropic Gaussians and their values.

    Returns (positions (n, d) float32, values (n, value_channels + 1) float32); the last
    value channel is the homogeneous weight 1."""
    c = uniform(seed, 11, centres * d).reshape(centres, d) * spread
    pick = np.minimum((uniform(seed, 12, n) * centres).astype(np.int64), centres - 1)
    pos = c[pick] + std * normal(seed, 13, n * d).reshape(n, d)
    vals = np.empty((n, value_channels + 1), dtype=np.float32)
    vals[:, :value_channels] = (uniform(seed, 14, n * value_channels).reshape(n, value_channels)
                                * 2.0 - 1.0)
    vals[:, value_channels] = 1.0
    return pos.astype(np.float32), vals


def log_uniform_int(seed: int, stream: int, n: int, lo: int, hi: int) -> np.ndarray:
    u = uniform(seed, stream, n)
    return np.floor(np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))).astype(np.int64).clip(lo, hi)


def batch_specs(count: int = 256, lo: int = 128, hi: int = 1024, seed: int = 0):
    """Uneven image batch: per image (width, height, sigma_s, sigma_r, seed)."""
    ws = log_uniform_int(seed, 21, count, lo, hi)
    hs = log_uniform_int(seed, 22, count, lo, hi)
    ss = 4.0 + 28.0 * uniform(seed, 23, count)
    sr = 0.05 + 0.25 * uniform(seed, 24, count)
    return [(int(ws[i]), int(hs[i]), float(ss[i]), float(sr[i]), seed * 100003 + i)
            for i in range(count)]
