"""LB_Petitjean on the device (csrc/petitjean.cu), through the C ABI.

* dtwj_pair_lb_petitjean with each window's own clipped envelope against the
  reference's own lbPetitjean_new / LB_KK known answers
  (tests/golden/petitjean.json) and the oracle; with the raw-series envelope
  the join reads, against the oracle.  FP64 on both sides: 1e-9 relative.
* Admissibility: endpoint bound + both sums never exceed the squared FP64 DTW
  of the pair, on random pairs and on each window's nearest neighbours.
* Joins with DTWJ_F_PETITJEAN return the plain join's top-1 (indices
  bit-exact, distance within 1e-5 of the oracle), and every pair the stage
  prunes is one DTW fewer, with the sweep as a CUDA graph and launched
  directly."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

REL = 1e-9
JOIN_REL = 1e-5


def _kat_series(synth, rec):
    gen = synth.random_walk if rec["kind"] == "rw" else synth.ecg_like
    return np.ascontiguousarray(gen(rec["n"], rec["seed"]), dtype=np.float64)


def test_device_lb_petitjean_matches_reference_and_oracle(gpu_dtwj, oracle, synth,
                                                          petitjean_kat):
    checked = 0
    for rec in petitjean_kat:
        x = _kat_series(synth, rec)
        m, w = rec["m"], rec["w"]
        pa = np.array([p[0] for p in rec["pairs"]], dtype=np.int64)
        pb = np.array([p[1] for p in rec["pairs"]], dtype=np.int64)
        ref_terms = np.array([p[3] for p in rec["pairs"]])
        km, tt = gpu_dtwj.pair_lb_petitjean(x, m, w, pa, pb, own_env=True)
        np.testing.assert_allclose(tt, ref_terms, rtol=REL, atol=1e-12)
        km0, tt0 = gpu_dtwj.pair_lb_petitjean(x, m, w, pa, pb, own_env=False)
        for k in range(pa.size):
            _, okm, ott = oracle.lb_petitjean(x, m, w, pa[k], pb[k], exact_env=True)
            assert km[k] == pytest.approx(okm, rel=REL, abs=1e-12)
            assert tt[k] == pytest.approx(ott, rel=REL, abs=1e-12)
            _, okm, ott = oracle.lb_petitjean(x, m, w, pa[k], pb[k], exact_env=False)
            assert km0[k] == pytest.approx(okm, rel=REL, abs=1e-12)
            assert tt0[k] == pytest.approx(ott, rel=REL, abs=1e-12)
            checked += 1
    assert checked > 300


@pytest.mark.parametrize("kind,n,m,w,seed", [
    ("rw", 6000, 128, 13, 1), ("ecg", 8000, 200, 20, 2), ("ecg", 6000, 128, 52, 3),
    ("rw", 4000, 64, 70, 4),
])
def test_device_lb_petitjean_is_admissible(gpu_dtwj, oracle, synth, kind, n, m, w, seed):
    x = synth.random_walk(n, seed) if kind == "rw" else synth.ecg_like(n, seed)
    s = n - m + 1
    rng = np.random.default_rng(seed)
    pa = rng.integers(0, s, 300)
    pb = rng.integers(0, s, 300)
    # nearest neighbours by ED: pairs the bound is tight on
    mp, mpi = oracle.mp(x, m)
    near = np.argsort(mp)[:200]
    pa = np.concatenate([pa, near, mpi[near]]).astype(np.int64)
    pb = np.concatenate([pb, mpi[near], near]).astype(np.int64)
    we = min(w, m - 1)
    d2 = gpu_dtwj.pair_dtw(x, m, we, pa, pb, precise=True) ** 2
    mu, sg = oracle.stats(x, m)
    for own in (True, False):
        km, tt = gpu_dtwj.pair_lb_petitjean(x, m, w, pa, pb, own_env=own)
        for k in range(pa.size):
            za = (x[pa[k]:pa[k] + m] - mu[pa[k]]) / sg[pa[k]]
            zb = (x[pb[k]:pb[k] + m] - mu[pb[k]]) / sg[pb[k]]
            lb = oracle.kim2(za, zb) + km[k] + tt[k]
            assert lb <= d2[k] * (1 + 1e-9) + 1e-9, (own, pa[k], pb[k], lb, d2[k])
        assert np.all(tt >= 0) and np.all(km >= 0)


def test_device_lb_petitjean_argument_errors(gpu_dtwj, synth):
    x = synth.random_walk(3000, 5)
    with pytest.raises(gpu_dtwj.DtwjError):
        gpu_dtwj.pair_lb_petitjean(x, 64, 3, [0], [3000 - 64 + 1])  # window past the end
    with pytest.raises(gpu_dtwj.DtwjError):
        gpu_dtwj.pair_lb_petitjean(x, 4, 3, [0], [10])  # m below the minimum


def _check(r, i, j, dist, what=""):
    assert (r.i, r.j) == (i, j), what
    assert abs(r.dist - dist) <= max(JOIN_REL * dist, 1e-9), (what, r.dist, dist)


def _reaching(r):
    """Pairs that reach the stages after LB_Keogh: DTW, the DTW stage's own
    cumulative bound (counted with LB_Keogh) or LB_Petitjean.  The best-so-far
    at the start of each chunk does not depend on the order within it, so this
    count is the same with and without the stage."""
    return r.dtw_calls + r.pruned_keogh + r.pruned_petitjean


def test_join_with_petitjean_matches_golden(gpu_dtwj, golden):
    for c in golden:
        base = gpu_dtwj.join(c["series"], c["m"], c["w"])
        r = gpu_dtwj.join(c["series"], c["m"], c["w"], gpu_dtwj.F_PETITJEAN)
        _check(r, c["i"], c["j"], c["dist"], c["name"])
        assert _reaching(r) == _reaching(base), c["name"]


@pytest.mark.parametrize("n,m,w,seed", [(4000, 64, 13, 21), (6000, 100, 20, 22),
                                        (5000, 128, 52, 23), (3000, 100, 70, 24)])
def test_join_with_petitjean_matches_oracle_on_ecg(gpu_dtwj, oracle, synth, n, m, w, seed):
    """ECG-like series, where most pairs reach DTW: the stage prunes some of
    them and the result stays the oracle's."""
    x = synth.ecg_like(n, seed)
    ref = oracle.join(x, m, w)
    with gpu_dtwj.Context() as ctx:
        base = ctx.join(x, m, w, gpu_dtwj.F_NO_GRAPH)
        for fl in (gpu_dtwj.F_PETITJEAN, gpu_dtwj.F_PETITJEAN,  # capture, then replay
                   gpu_dtwj.F_PETITJEAN | gpu_dtwj.F_NO_GRAPH):
            r = ctx.join(x, m, w, fl)
            _check(r, ref.i, ref.j, ref.dist, (n, m, w, fl))
            assert r.pruned_petitjean > 0
            assert _reaching(r) == _reaching(base)


def _fullsize(name):
    with open(os.path.join(GOLDEN, "fullsize.json")) as f:
        return [r for r in json.load(f) if r["workload"] == name][0]


def test_full_size_ecg_join_with_petitjean(gpu_dtwj, synth):
    rec = _fullsize("ecg16k_w52")
    wl = synth.workload(rec["workload"])
    with gpu_dtwj.Context() as ctx:
        r = ctx.join(wl["series"], wl["m"], wl["w"], gpu_dtwj.F_PETITJEAN)
    assert (r.i, r.j) == (rec["i"], rec["j"])
    assert abs(r.dist - rec["dist"]) <= JOIN_REL * rec["dist"]
    assert r.pruned_petitjean > 0
