"""Seeded synthetic series for the join's workloads.

The reference ships no dataset (its README names only an RTX 3060 Laptop GPU),
so every workload is generated here from a seed:

* ``random_walk``   x_0 = 0, x_t = x_{t-1} + N(0, 1)
* ``ecg_like``      Gaussian pulses (sigma 8 samples, beat period U(180, 220),
                    amplitude U(0.8, 1.2)) plus N(0, 0.05) noise
* ``plant_motifs``  a length-L sum of 3 sines (periods U(50, 300), amplitudes
                    U(0.5, 2)) written into a series at two non-overlapping
                    offsets per pair, each copy with N(0, 0.1) noise and a
                    random +-5 % time warp by linear resampling

``workload(name)`` returns the named configurations used by tests and the
benchmark.  numpy's PCG64 is the generator; outputs are float64.
"""
from __future__ import annotations

import math

import numpy as np


def band(m: int, ratio: float, rounding: str = "ceil") -> int:
    """Sakoe-Chiba band from a ratio: ceil(ratio*m) (or the reference's
    max(round(ratio*m), 1), GPU_version1/src/AAAA.cu:34)."""
    if rounding == "round":
        return max(int(math.floor(ratio * m + 0.5)), 1)
    return max(int(math.ceil(ratio * m - 1e-9)), 1)


def random_walk(n: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    x = np.empty(n, dtype=np.float64)
    x[0] = 0.0
    if n > 1:
        np.cumsum(rng.standard_normal(n - 1), out=x[1:])
    return x


def ecg_like(n: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.normal(0.0, 0.05, n)
    t = float(rng.uniform(0, 200))
    sigma = 8.0
    half = int(6 * sigma)
    while t < n + half:
        amp = rng.uniform(0.8, 1.2)
        c = int(round(t))
        lo, hi = max(c - half, 0), min(c + half + 1, n)
        if lo < hi:
            k = np.arange(lo, hi, dtype=np.float64)
            x[lo:hi] += amp * np.exp(-0.5 * ((k - t) / sigma) ** 2)
        t += rng.uniform(180, 220)
    return x


def _motif(rng: np.random.Generator, length: int) -> np.ndarray:
    k = np.arange(length, dtype=np.float64)
    y = np.zeros(length)
    for _ in range(3):
        period = rng.uniform(50, 300)
        amp = rng.uniform(0.5, 2.0)
        phase = rng.uniform(0, 2 * math.pi)
        y += amp * np.sin(2 * math.pi * k / period + phase)
    return y


def _warped_copy(rng: np.random.Generator, base: np.ndarray, length: int) -> np.ndarray:
    f = rng.uniform(0.95, 1.05)
    pos = np.arange(length, dtype=np.float64) * f
    pos = np.minimum(pos, len(base) - 1)
    return np.interp(pos, np.arange(len(base), dtype=np.float64), base) + rng.normal(0, 0.1, length)


def plant_motifs(x: np.ndarray, pairs: int, length: int, seed: int):
    """Writes `pairs` motif pairs into x (in place, via its increments so the
    series stays continuous).  Returns the list of (offset_a, offset_b)."""
    rng = np.random.Generator(np.random.PCG64(seed + 7919))
    n = len(x)
    inc = np.diff(x, prepend=0.0)
    used: list[tuple[int, int]] = []
    placed = []
    for _ in range(pairs):
        base = _motif(rng, int(length * 1.06) + 2)
        offs = []
        while len(offs) < 2:
            o = int(rng.integers(1, n - length - 1))
            if all(o + length + 8 < a or b + 8 < o for a, b in used):
                used.append((o, o + length))
                offs.append(o)
        for o in offs:
            c = _warped_copy(rng, base, length)
            inc[o + 1:o + length] = np.diff(c)
        placed.append((offs[0], offs[1]))
    x[:] = np.cumsum(inc)
    return placed


def workload(name: str):
    """Named workloads: returns dict(series=..., m=..., w=..., ...)."""
    if name == "rw20k":  # plain method, CPU-runnable
        return dict(series=random_walk(20_000, 0), m=256, w=band(256, 0.01), ratio=0.01)
    if name == "rw65k":  # small case of the at-scale workload
        return dict(series=random_walk(65_536, 3), m=1024, w=band(1024, 0.05), ratio=0.05)
    if name == "rw1m_motif":  # plain GPU at scale
        x = random_walk(1_000_000, 1)
        planted = plant_motifs(x, 1, 1024, 1)
        return dict(series=x, m=1024, w=band(1024, 0.05), ratio=0.05, planted=planted)
    if name in ("rw262k_w52", "rw262k_w103"):
        x = random_walk(262_144, 3)
        r = 0.1 if name.endswith("w52") else 0.2
        return dict(series=x, m=512, w=band(512, r), ratio=r)
    if name in ("ecg16k_w52", "ecg16k_w103"):  # the first 16,384 samples of ecg262k_*
        x = ecg_like(262_144, 3)[:16_384].copy()
        r = 0.1 if name.endswith("w52") else 0.2
        return dict(series=x, m=512, w=band(512, r), ratio=r)
    if name in ("ecg262k_w52", "ecg262k_w103"):
        x = ecg_like(262_144, 3)
        r = 0.1 if name.endswith("w52") else 0.2
        return dict(series=x, m=512, w=band(512, r), ratio=r)
    if name == "rw4m_motif8":
        x = random_walk(4_000_000, 4)
        planted = plant_motifs(x, 8, 256, 4)
        return dict(series=x, m=256, w=band(256, 0.05), ratio=0.05, planted=planted)
    if name == "rw4m_motif8_1m":  # the first 1,000,000 samples of rw4m_motif8
        full = workload("rw4m_motif8")
        n = 1_000_000
        x = full["series"][:n].copy()
        planted = [p for p in full["planted"] if max(p) + 256 <= n]
        return dict(series=x, m=256, w=band(256, 0.05), ratio=0.05, planted=planted)
    raise KeyError(name)


def batch_workload(count: int = 4096, seed: int = 5, lo: int = 2000, hi: int = 65536):
    """Many series of uneven length: lengths log-uniform in [lo, hi], half
    random walks and half ECG-like, m from {64, 128, 256}, ratio 0.05."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        m = int(rng.choice([64, 128, 256]))
        n = max(n, 2 * m + 2)
        s = int(rng.integers(0, 2**31 - 1))
        x = random_walk(n, s) if k % 2 == 0 else ecg_like(n, s)
        out.append(dict(series=x, m=m, w=band(m, 0.05), ratio=0.05))
    return out
