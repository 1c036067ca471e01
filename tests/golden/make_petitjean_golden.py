"""Generates tests/golden/petitjean.json: known answers of the reference's own
LB_Petitjean (lbPetitjean_new, CPU_version1/LB_PETITJEAN.cpp:10) and LB_KK
(CPU_version1/lb_keogh.cpp:9), called through oracle/_ref/libref.so
(ref_lb_petitjean, oracle/ref_shim.cpp) on windows of seeded series.

    python tests/golden/make_petitjean_golden.py

Each record: series kind, n, seed, m, w and a list of (A, B, keogh, terms) —
A and B the 0-based windows, keogh the squared LB_Keogh of A against B's
clipped envelope over all m samples, terms what LB_Petitjean adds to it.
Pairs are drawn at random, plus pairs whose two windows lie close in value
(nearest neighbours by z-normalised distance), where the projection term is
most often non-zero.  Needs the reference sources (only on the machine that
builds the fixtures).
"""
from __future__ import annotations

import ctypes
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "scaling-subsequence-similarity-join-based-on-dynamic-time-warping-cpu-gpu_b200")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")

# (kind, n, seed, m, w, pairs)
CASES = [
    ("rw", 3000, 41, 64, 3, 40),
    ("rw", 4000, 42, 128, 13, 40),
    ("ecg", 5000, 43, 128, 7, 40),
    ("rw", 6000, 44, 256, 26, 30),
    ("ecg", 6000, 45, 200, 52, 30),
    ("rw", 3000, 46, 32, 1, 30),
    ("ecg", 4000, 47, 160, 103, 20),
]


def _synth():
    spec = importlib.util.spec_from_file_location("dtwj_synth", os.path.join(PKG, "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _near_pairs(x, m, count, rng):
    """Pairs (A, B) with B - A >= m whose z-normalised windows are close."""
    s = x.size - m + 1
    win = np.lib.stride_tricks.sliding_window_view(x, m)[::4]
    z = (win - win.mean(1, keepdims=True)) / win.std(1, keepdims=True)
    out = []
    for a in rng.choice(len(z), size=count, replace=False):
        d = ((z - z[a]) ** 2).sum(1)
        idx = np.arange(len(z)) * 4
        d[np.abs(idx - a * 4) < m] = np.inf
        b = int(idx[int(np.argmin(d))])
        out.append((int(a * 4), min(b, s - 1)))
    return out


def main():
    synth = _synth()
    lib = ctypes.CDLL(REF_LIB)
    P = ctypes.POINTER(ctypes.c_double)
    lib.ref_lb_petitjean.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                     ctypes.c_long, P, P]
    recs = []
    for kind, n, seed, m, w, count in CASES:
        x = (synth.random_walk if kind == "rw" else synth.ecg_like)(n, seed)
        x = np.ascontiguousarray(x, dtype=np.float64)
        rng = np.random.default_rng(seed)
        s = n - m + 1
        pairs = [(int(a), int(b)) for a, b in rng.integers(0, s, size=(count, 2))]
        pairs += _near_pairs(x, m, count // 2, rng)
        rows = []
        for a, b in pairs:
            k, t = ctypes.c_double(), ctypes.c_double()
            lib.ref_lb_petitjean(x.ctypes.data_as(P), n, m, w, a, b, ctypes.byref(k),
                                 ctypes.byref(t))
            rows.append([a, b, k.value, t.value])
        recs.append({"kind": kind, "n": n, "seed": seed, "m": m, "w": w, "pairs": rows})
        print("%s n=%d m=%d w=%d: %d pairs, %d with a non-zero projection term"
              % (kind, n, m, w, len(rows), sum(r[3] > 0 for r in rows)))
    with open(os.path.join(HERE, "petitjean.json"), "w") as f:
        json.dump(recs, f, indent=0)


if __name__ == "__main__":
    main()
