"""Learned tile ordering: the device tile features against the FP64 CPU
restatement (features_ref.py), the exact per-tile DTW minima (the training
targets) against brute force, and the ordering's exactness (it only permutes
the tiles, so every join result equals the plain order's)."""
import numpy as np
import pytest

import features_ref

pytestmark = pytest.mark.gpu


def test_tile_features_match_cpu(gpu_dtwj, synth):
    x = synth.random_walk(4500, 17)
    m, w = 32, 2
    with gpu_dtwj.Context() as ctx:
        desc, feat, _ = ctx.tiles(x, m, w)
    assert [tuple(int(v) for v in d[:3]) for d in desc] == features_ref.tiles(x.size, m)
    ref = features_ref.features(x, m, w)
    exact = np.ones(64, dtype=bool)
    exact[32:40] = False
    np.testing.assert_allclose(feat[:, exact], ref[:, exact], rtol=1e-5, atol=1e-6)
    # fractions of rows whose nearest neighbour is in the tile: a near-tie of
    # the profile may move one row's neighbour
    np.testing.assert_allclose(feat[:, 32:40], ref[:, 32:40], rtol=0, atol=0.02)


def test_tile_minima_are_exact(gpu_dtwj, synth):
    x = synth.random_walk(2600, 18)
    m, w = 32, 2
    s = x.size - m + 1
    with gpu_dtwj.Context() as ctx:
        desc, _, md = ctx.tiles(x, m, w, features=False, min_dist=True)
    assert len(desc) >= 3
    for (L0, i0, rows, _lags), got in zip(desc, md):
        ii, ll = np.meshgrid(np.arange(i0, i0 + rows), np.arange(L0, L0 + 896), indexing="ij")
        jj = ii + ll
        ok = jj < s
        d = gpu_dtwj.pair_dtw(x, m, w, ii[ok], jj[ok], precise=True)
        assert got == pytest.approx(d.min(), rel=1e-12, abs=1e-12), (L0, i0)


def test_learned_order_keeps_the_result(gpu_dtwj, golden):
    net = gpu_dtwj.MLP(seed=1)  # whatever the scores, they only permute the tiles
    for c in golden[:5]:
        with gpu_dtwj.Context() as ctx:
            with pytest.raises(gpu_dtwj.DtwjError) as e:
                ctx.join(c["series"], c["m"], c["w"], gpu_dtwj.F_LEARNED)
            assert e.value.code == gpu_dtwj.ERR_NOMODEL
            ctx.set_model(net)
            r = ctx.join(c["series"], c["m"], c["w"], gpu_dtwj.F_LEARNED)
            p = ctx.join(c["series"], c["m"], c["w"])
        assert (r.i, r.j) == (c["i"], c["j"]) == (p.i, p.j), c["name"]
        assert r.dist == pytest.approx(c["dist"], rel=1e-5, abs=1e-9)
        assert r.pairs == p.pairs
