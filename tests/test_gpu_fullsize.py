"""Full-size checks (the 1M-sample bench workload and the 262k random walk)
through properties that need no CPU oracle run (an FP64 oracle join at 1M
samples takes hours): the reported distance is the FP64 DTW of the reported
pair, no smaller DTW exists at the planted motif pair, and every flag, shard
count and order that must not change the result reproduces it exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["rw1m_motif", "rw262k_w52"])
def test_full_size_join_properties(gpu_dtwj, synth, name):
    wl = synth.workload(name)
    x, m, w = wl["series"], wl["m"], wl["w"]
    with gpu_dtwj.Context() as ctx:
        r = ctx.join(x, m, w)
        assert r.j - r.i >= m
        s = x.size - m + 1
        assert r.pairs == (s - m) * (s - m + 1) // 2
        # the distance is the exact FP64 DTW of the pair
        d = gpu_dtwj.pair_dtw(x, m, w, [r.i], [r.j], precise=True)[0]
        assert r.dist == pytest.approx(d, rel=1e-12)
        # the ED seeds bound it from above; a planted motif pair cannot beat it
        assert r.dist <= r.seed_bsf * (1 + 1e-6)
        for a, b in wl.get("planted", []):
            dp = gpu_dtwj.pair_dtw(x, m, w, [min(a, b)], [max(a, b)], precise=True)[0]
            assert r.dist <= dp * (1 + 1e-12)
        # (F_NO_SEED is for small inputs: with no initial best-so-far the first
        # chunk of a 1M-sample join overflows its queues and is re-swept in
        # one-tile chunks)
        for fl in (gpu_dtwj.F_NO_MASKED, gpu_dtwj.F_NO_GRAPH):
            q = ctx.join(x, m, w, fl)
            assert (q.i, q.j, q.dist) == (r.i, r.j, r.dist), fl
        parts = []
        for k in range(2):
            ctx.set_shard(k, 2)
            parts.append(ctx.join(x, m, w))
        ctx.set_shard(0, 1)
        sh = gpu_dtwj.merge_results(parts)
        assert (sh.i, sh.j, sh.dist) == (r.i, r.j, r.dist) and sh.pairs == r.pairs
