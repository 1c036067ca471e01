"""Generates the golden fixtures of this directory by running the reference's
own CPU implementation (CPU_version1, FP64), compiled out of the reference
tree by oracle/build_ref.sh into oracle/_ref/.

    python tests/golden/make_golden.py

Writes
  series_<name>.f64      the seeded input series (raw little-endian float64)
  joins.json             reference top-1 pair per case: 0-based (i, j), the
                         distance it printed (%f) and the same pair's distance
                         recomputed at full FP64 precision with the
                         reference's own mvmean z-normalisation and MON_dtw.
                         When no sweep DTW beats the ED seeds, the reference
                         prints stale indices (those of its last seed,
                         CPU_version1/new_dtw_motifGUI.cpp:76-77); such a
                         case is marked "stale_indices", its pair is taken
                         from the oracle's exhaustive join (LB_Keogh + DTW
                         only) and accepted only if the reference's own
                         MON_dtw on that pair reproduces the printed distance
  kat.json               component known answers from the reference:
                         MON_dtw on random z-normalised pairs, the clipped
                         envelope (lower_upper_lemire), mvmean, mpx_v2, and
                         the global CDF mask (compute_MASK_global)
Needs the reference sources (only on the machine that builds the fixtures).
"""
from __future__ import annotations

import ctypes
import importlib.util
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "scaling-subsequence-similarity-join-based-on-dynamic-time-warping-cpu-gpu_b200")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_join")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")


def _synth():
    spec = importlib.util.spec_from_file_location("dtwj_synth", os.path.join(PKG, "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# name -> (generator, n, seed, m, w)
CASES = [
    ("rw20k", "rw", 20_000, 0, 256, 3),  # the CPU-runnable configuration
    ("rw3k_m64_w3", "rw", 3000, 11, 64, 3),
    ("rw4k_m64_w6", "rw", 4000, 12, 64, 6),
    ("rw6k_m128_w6", "rw", 6000, 13, 128, 6),
    ("rw5k_m128_w13", "rw", 5000, 14, 128, 13),
    ("rw8k_m256_w13", "rw", 8000, 15, 256, 13),
    ("ecg6k_m128_w7", "ecg", 6000, 16, 128, 7),
    ("ecg9k_m200_w20", "ecg", 9000, 17, 200, 20),
    ("rw6k_m100_w52", "rw", 6000, 18, 100, 52),
    ("rw7k_m512_w26", "rw", 7000, 19, 512, 26),
]


# global-mask known answers: (kind, n, seed, m, w)
MASK_CASES = [("rw", 3000, 21, 64, 5), ("rw", 5000, 3, 128, 13), ("ecg", 4000, 7, 100, 10),
              ("rw", 8000, 9, 256, 26)]


def _oracle_brute(x, m, w):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    buf = (ctypes.c_char * 512)()
    rc = lib.orc_join(x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.c_int64(x.size),
                      m, w, 1 | 4, 0, buf)
    assert rc == 0
    i, j = np.frombuffer(bytes(buf)[:16], dtype=np.int64)
    return int(i), int(j)


def _ref_pair_dist(x, m, w, i, j):
    ref = ctypes.CDLL(REF_LIB)
    P = ctypes.POINTER(ctypes.c_double)
    ref.ref_mon_dtw.restype = ctypes.c_double
    s = x.size - m + 1
    mu = np.empty(s)
    sg = np.empty(s)
    ref.ref_mvmean(x.ctypes.data_as(P), ctypes.c_long(x.size), m, mu.ctypes.data_as(P),
                   sg.ctypes.data_as(P))
    q = (x[i:i + m] - mu[i]) / sg[i]
    t = (x[j:j + m] - mu[j]) / sg[j]
    return float(np.sqrt(ref.ref_mon_dtw(q.ctypes.data_as(P), t.ctypes.data_as(P), m, w)))


def run_ref(path, m, w):
    out = subprocess.run([REF_BIN, path, str(m), str(w)], capture_output=True, text=True,
                         check=True).stdout
    line = out.strip().splitlines()[-1]
    return json.loads(line.replace(": -nan", ": NaN").replace(": nan", ": NaN"))


def main():
    synth = _synth()
    if not os.path.exists(REF_BIN):
        sys.exit("build the reference first: oracle/build_ref.sh")
    joins = []
    for name, kind, n, seed, m, w in CASES:
        x = synth.random_walk(n, seed) if kind == "rw" else synth.ecg_like(n, seed)
        path = os.path.join(HERE, "series_%s.f64" % name)
        x.astype("<f8").tofile(path)
        r = run_ref(path, m, w)
        assert r["rc"] == 0, r
        stale = not (r["dist"] == r["dist"]) or abs(r["dist"] - r["dist_printed"]) > 1e-6
        rec = dict(name=name, kind=kind, n=n, seed=seed, m=m, w=w, i=r["i"], j=r["j"],
                   dist=r["dist"], dist_printed=r["dist_printed"], stale_indices=stale)
        if stale:
            i, j = _oracle_brute(x, m, w)
            d = _ref_pair_dist(x, m, w, i, j)
            assert abs(d - r["dist_printed"]) <= 1e-6, (name, d, r)
            rec.update(i=i, j=j, dist=d, ref_printed_i=r["i"], ref_printed_j=r["j"])
        joins.append(rec)
        print(name, rec["i"], rec["j"], rec["dist"], "stale" if stale else "",
              "%.2fs" % r["wall_seconds"])
    with open(os.path.join(HERE, "joins.json"), "w") as f:
        json.dump(joins, f, indent=1)

    ref = ctypes.CDLL(REF_LIB)
    P = ctypes.POINTER(ctypes.c_double)
    ref.ref_mon_dtw.restype = ctypes.c_double
    rng = np.random.Generator(np.random.PCG64(2024))
    dtw = []
    for m, w in [(16, 1), (32, 3), (64, 6), (100, 10), (128, 13), (256, 26), (512, 52), (300, 103)]:
        for _ in range(3):
            q = rng.standard_normal(m)
            t = rng.standard_normal(m)
            q = (q - q.mean()) / q.std()
            t = (t - t.mean()) / t.std()
            d2 = ref.ref_mon_dtw(q.ctypes.data_as(P), t.ctypes.data_as(P), m, w)
            dtw.append(dict(m=m, w=w, q=q.tolist(), t=t.tolist(), d2=d2))
    x = synth.random_walk(3000, 21)
    env = []
    for r in (1, 5, 52):
        lo = np.empty(x.size)
        up = np.empty(x.size)
        ref.ref_lemire(x.ctypes.data_as(P), x.size, r, lo.ctypes.data_as(P), up.ctypes.data_as(P))
        env.append(dict(r=r, lower=lo.tolist(), upper=up.tolist()))
    m = 64
    mu = np.empty(x.size - m + 1)
    sg = np.empty(x.size - m + 1)
    ref.ref_mvmean(x.ctypes.data_as(P), ctypes.c_long(x.size), m, mu.ctypes.data_as(P),
                   sg.ctypes.data_as(P))
    mp = np.empty(x.size - m + 1)
    mpi = np.empty(x.size - m + 1, dtype=np.int32)
    ref.ref_mpx(x.ctypes.data_as(P), ctypes.c_long(x.size), m, mp.ctypes.data_as(P),
                mpi.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    # the global CDF mask (compute_shared_data_global + compute_MASK_global,
    # set up as new_dtw_motifGUI does) on seeded series: the positions where
    # the mask is 1, and the CDF table length
    masks = []
    for kind, n, seed, mm, ww in MASK_CASES:
        xs = synth.random_walk(n, seed) if kind == "rw" else synth.ecg_like(n, seed)
        out = np.empty(n)
        lt = ctypes.c_int()
        rc = ref.ref_mask(xs.ctypes.data_as(P), ctypes.c_long(n), mm, ww, out.ctypes.data_as(P),
                          ctypes.byref(lt))
        assert rc == 0
        masks.append(dict(kind=kind, n=n, seed=seed, m=mm, w=ww, table_len=lt.value,
                          ones=np.flatnonzero(out == 1.0).tolist()))
    kat = dict(dtw=dtw, envelope_series_seed=21, envelope_n=3000, envelope=env,
               mvmean=dict(m=m, mu=mu.tolist(), sig=sg.tolist()),
               mpx=dict(m=m, mp=mp.tolist(), mpi_1based=mpi.tolist()), mask=masks)
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f)
    print("wrote", len(joins), "joins and kat.json")


if __name__ == "__main__":
    main()
