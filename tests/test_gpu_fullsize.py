"""Full-size joins against the oracle: the bench workload (n = 1,000,000,
m = 1024, w = 52) and the band/shape sweep at 262,144 samples, checked
against the oracle's top-1 pair on the same seeded series
(tests/golden/fullsize.json, made by tests/golden/make_fullsize.py with the
OpenMP FP64 restatement that tests/test_oracle.py pins to the reference).
Tolerances: indices bit-exact, distance within 1e-5 relative.  Beside the
oracle, properties every full-size join must have: the distance is the FP64
DTW of the reported pair, no planted motif pair beats it, and every flag,
run filter and shard count that must not change the result reproduces it."""
import json
import os

import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

REL = 1e-5


def _records():
    path = os.path.join(GOLDEN, "fullsize.json")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return json.load(f)


@pytest.mark.parametrize("rec", _records(), ids=lambda r: r["workload"])
def test_full_size_join_matches_oracle(gpu_dtwj, synth, rec):
    wl = synth.workload(rec["workload"])
    x, m, w = wl["series"], wl["m"], wl["w"]
    assert (x.size, m, w) == (rec["n"], rec["m"], rec["w"])
    with gpu_dtwj.Context() as ctx:
        r = ctx.join(x, m, w)
        assert (r.i, r.j) == (rec["i"], rec["j"])
        assert abs(r.dist - rec["dist"]) <= REL * rec["dist"], (r.dist, rec["dist"])
        s = x.size - m + 1
        assert r.pairs == (s - m) * (s - m + 1) // 2
        # the distance is the exact FP64 DTW of the pair
        d = gpu_dtwj.pair_dtw(x, m, w, [r.i], [r.j], precise=True)[0]
        assert r.dist == pytest.approx(d, rel=1e-12)
        assert r.dist <= r.seed_bsf * (1 + 1e-6)
        for a, b in wl.get("planted", []):
            dp = gpu_dtwj.pair_dtw(x, m, w, [min(a, b)], [max(a, b)], precise=True)[0]
            assert r.dist <= dp * (1 + 1e-12)
        # the reference's masked cascade, direct launches and two tile shards
        # (F_NO_SEED is for small inputs: with no initial best-so-far the first
        # chunk of a 1M-sample join overflows its queues and is re-swept in
        # one-tile chunks)
        for fl in (gpu_dtwj.F_MASKED_CASCADE, gpu_dtwj.F_NO_GRAPH):
            q = ctx.join(x, m, w, fl)
            assert (q.i, q.j, q.dist) == (r.i, r.j, r.dist), fl
        parts = []
        for k in range(2):
            ctx.set_shard(k, 2)
            parts.append(ctx.join(x, m, w))
        ctx.set_shard(0, 1)
        sh = gpu_dtwj.merge_results(parts)
        assert (sh.i, sh.j, sh.dist) == (r.i, r.j, r.dist) and sh.pairs == r.pairs
