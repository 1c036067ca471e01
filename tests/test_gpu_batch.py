"""Batched join: every series of dtwj_join_batch gets exactly the top-1 pair
that dtwj_join returns for it alone (same indices, same FP64 distance)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(rb, rs, tag):
    assert (rb.i, rb.j) == (rs.i, rs.j), tag
    if np.isfinite(rs.dist):
        assert rb.dist == pytest.approx(rs.dist, rel=1e-12, abs=0.0), tag
    else:
        assert not np.isfinite(rb.dist), tag


def test_batch_matches_single_joins(gpu_dtwj, synth):
    items = synth.batch_workload(count=24, seed=11, lo=2000, hi=12000)
    xs = [it["series"] for it in items]
    ms = [it["m"] for it in items]
    ws = [it["w"] for it in items]
    rb = gpu_dtwj.join_batch(xs, ms, ws)
    for k, (x, m, w) in enumerate(zip(xs, ms, ws)):
        rs = gpu_dtwj.join(x, m, w)
        _same(rb[k], rs, "series %d (n=%d m=%d w=%d)" % (k, len(x), m, w))
        assert rb[k].n == len(x) and rb[k].m == m and rb[k].w == w


def test_batch_with_more_groups_than_workers(gpu_dtwj, synth):
    # seven (m, w) groups: the groups run on up to four contexts at a time,
    # each worker taking the next group when its last one is done
    shapes = [(32, 2), (48, 3), (64, 4), (64, 13), (96, 5), (128, 7), (160, 8)]
    xs, ms, ws = [], [], []
    for k, (m, w) in enumerate(shapes):
        for r in range(3):
            gen = synth.random_walk if (k + r) % 2 == 0 else synth.ecg_like
            xs.append(gen(2500 + 700 * r + 100 * k, 40 + 3 * k + r))
            ms.append(m)
            ws.append(w)
    rb = gpu_dtwj.join_batch(xs, ms, ws)
    for k, (x, m, w) in enumerate(zip(xs, ms, ws)):
        _same(rb[k], gpu_dtwj.join(x, m, w), "series %d (n=%d m=%d w=%d)" % (k, len(x), m, w))


def test_batch_edge_series(gpu_dtwj, synth):
    # a flat series (no valid window), an exact duplicate (tie at distance 0,
    # lowest index wins) and the shortest allowed length, mixed with plain ones
    m = 64
    flat = np.full(3000, 2.5)
    dup = synth.random_walk(4000, 21)
    dup[2500:2500 + m] = dup[300:300 + m]
    short = synth.random_walk(2 * m + 1, 22)
    xs = [synth.random_walk(5000, 23), flat, dup, short, synth.ecg_like(6000, 24)]
    ms = [m] * len(xs)
    ws = [4] * len(xs)
    rb = gpu_dtwj.join_batch(xs, ms, ws)
    for k, x in enumerate(xs):
        _same(rb[k], gpu_dtwj.join(x, m, 4), "edge series %d" % k)
    assert rb[1].i == -1 and rb[1].j == -1
    assert (rb[2].i, rb[2].j) == (300, 2500) and rb[2].dist == pytest.approx(0.0, abs=1e-9)


def test_batch_rejects_a_too_short_series(gpu_dtwj, synth):
    xs = [synth.random_walk(3000, 1), synth.random_walk(100, 2)]
    with pytest.raises(RuntimeError):
        gpu_dtwj.join_batch(xs, [64, 64], [4, 4])
