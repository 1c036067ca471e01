"""Parity of the CUDA path (through the C ABI) with the reference's golden
outputs and with the oracle.  Tolerances: top-1 indices bit-exact; distance
within 1e-5 relative of the FP64 reference / oracle (the device search runs
in FP32 and re-verifies its final candidates in FP64)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR

pytestmark = pytest.mark.gpu

REL = 1e-5
ABS_ZERO = 1e-9  # distances of exact copies are rounding noise around 0


def _check(r, i, j, dist, what=""):
    assert (r.i, r.j) == (i, j), what
    assert abs(r.dist - dist) <= max(REL * dist, ABS_ZERO), (what, r.dist, dist)


def test_golden_reference_joins(gpu_dtwj, golden):
    for c in golden:
        r = gpu_dtwj.join(c["series"], c["m"], c["w"])
        _check(r, c["i"], c["j"], c["dist"], c["name"])
        s = r.n - r.m + 1
        assert r.pairs == (s - r.m) * (s - r.m + 1) // 2  # every pair with j - i >= m


@pytest.mark.parametrize("n,m,w,seed,kind", [
    (2000, 16, 1, 1, "rw"), (2500, 32, 2, 2, "rw"), (3000, 64, 3, 3, "rw"),
    (3000, 64, 13, 4, "ecg"), (4000, 128, 26, 5, "rw"), (3500, 100, 52, 6, "rw"),
    (5000, 256, 103, 7, "rw"), (4000, 300, 103, 8, "ecg"), (3000, 40, 40, 9, "rw"),
    (2600, 24, 70, 10, "rw"),
])
def test_join_matches_oracle(gpu_dtwj, oracle, synth, n, m, w, seed, kind):
    x = synth.random_walk(n, seed) if kind == "rw" else synth.ecg_like(n, seed)
    ref = oracle.join(x, m, min(w, m - 1))
    r = gpu_dtwj.join(x, m, w)
    _check(r, ref.i, ref.j, ref.dist, (n, m, w))


def test_flags_do_not_change_the_result(gpu_dtwj, golden):
    c = [g for g in golden if g["name"] == "rw6k_m128_w6"][0]
    base = gpu_dtwj.join(c["series"], c["m"], c["w"])
    for fl in (gpu_dtwj.F_NO_MASKED, gpu_dtwj.F_NO_SEED, gpu_dtwj.F_NO_DIAG,
               gpu_dtwj.F_NO_SEED | gpu_dtwj.F_NO_MASKED, gpu_dtwj.F_NO_GRAPH):
        r = gpu_dtwj.join(c["series"], c["m"], c["w"], fl)
        assert (r.i, r.j, r.dist) == (base.i, base.j, base.dist), fl
    nd = gpu_dtwj.join(c["series"], c["m"], c["w"], gpu_dtwj.F_NO_DIAG)
    assert nd.pruned_fast == 0 and nd.pairs == base.pairs


def test_masked_cascade_matches_block_mean_filter(gpu_dtwj, golden):
    # the run filter's two forms (the default block-mean LB_Keogh bound, and
    # the reference's masked diagonal bound + endpoint bound) prune different
    # pairs but return the same top-1; the block-mean bound lets fewer pairs
    # reach LB_Keogh
    for c in golden:
        base = gpu_dtwj.join(c["series"], c["m"], c["w"])
        casc = gpu_dtwj.join(c["series"], c["m"], c["w"], gpu_dtwj.F_MASKED_CASCADE)
        kim = gpu_dtwj.join(c["series"], c["m"], c["w"],
                            gpu_dtwj.F_MASKED_CASCADE | gpu_dtwj.F_NO_MASKED)
        for r in (casc, kim):
            assert (r.i, r.j, r.dist) == (base.i, base.j, base.dist), c["name"]
            assert r.pruned_paa == 0 and r.pruned_fast == base.pruned_fast
        assert base.pruned_masked == 0 and kim.pruned_masked == 0
        if c["name"] == "rw20k":
            assert base.pruned_paa > 0 and casc.pruned_masked > 0
            reach_base = base.pruned_keogh + base.dtw_calls
            reach_casc = casc.pruned_keogh + casc.dtw_calls
            assert reach_base < reach_casc, (reach_base, reach_casc)


def test_graph_replay_matches_direct_launches(gpu_dtwj, golden):
    # a context captures the sweep as a CUDA graph on the first join and
    # replays it on the next join of the same shape
    c = [g for g in golden if g["name"] == "rw20k"][0]
    x, m, w = c["series"], c["m"], c["w"]
    with gpu_dtwj.Context() as ctx:
        first = ctx.join(x, m, w, gpu_dtwj.F_PROFILE)
        replay = ctx.join(x, m, w, gpu_dtwj.F_PROFILE)
        direct = ctx.join(x, m, w, gpu_dtwj.F_PROFILE | gpu_dtwj.F_NO_GRAPH)
        again = ctx.join(x, m, w, gpu_dtwj.F_PROFILE)
    for r in (first, replay, direct, again):
        _check(r, c["i"], c["j"], c["dist"], "graph")
        assert r.pairs == first.pairs and r.pruned_fast == first.pruned_fast
    diag = gpu_dtwj.PHASES.index("diag")
    assert replay.phase_launches == first.phase_launches == direct.phase_launches
    assert replay.phase_seconds[diag] > 0


def test_deterministic(gpu_dtwj, golden):
    c = golden[0]
    a = gpu_dtwj.join(c["series"], c["m"], c["w"])
    b = gpu_dtwj.join(c["series"], c["m"], c["w"])
    assert (a.i, a.j, a.dist) == (b.i, b.j, b.dist)


def test_pair_dtw_matches_oracle(gpu_dtwj, oracle, synth):
    x = synth.random_walk(6000, 31)
    rng = np.random.default_rng(5)
    for m, w in [(16, 1), (64, 3), (128, 13), (256, 26), (512, 52), (300, 103), (50, 60)]:
        pi = rng.integers(0, x.size - m + 1, 40)
        pj = rng.integers(0, x.size - m + 1, 40)
        d64 = gpu_dtwj.pair_dtw(x, m, w, pi, pj, precise=True)
        d32 = gpu_dtwj.pair_dtw(x, m, w, pi, pj, precise=False)
        ref = np.array([oracle.pair_dist(x, m, min(w, m - 1), int(a), int(b))
                        for a, b in zip(pi, pj)])
        np.testing.assert_allclose(d64, ref, rtol=1e-10)
        np.testing.assert_allclose(d32, ref, rtol=2e-4)


@pytest.mark.parametrize("n,m,seed,kind", [(5000, 64, 41, "rw"), (8000, 128, 42, "rw"),
                                           (6000, 100, 43, "ecg"), (3000, 16, 44, "rw")])
def test_matrix_profile_matches_oracle(gpu_dtwj, oracle, synth, n, m, seed, kind):
    # every row's nearest-neighbour index equals the oracle's (the device keeps
    # every partner near the row minimum and decides among them at FP64);
    # distances within 1e-6 (the oracle's 1 - correlation form cancels for
    # close neighbours)
    x = synth.random_walk(n, seed) if kind == "rw" else synth.ecg_like(n, seed)
    mp, mpi = gpu_dtwj.matrix_profile(x, m)
    omp, ompi = oracle.mp(x, m)
    np.testing.assert_allclose(mp, omp, rtol=1e-6, atol=1e-6)
    assert np.array_equal(mpi, ompi), np.flatnonzero(mpi != ompi)[:10]


def test_global_mask_matches_reference(gpu_dtwj, oracle, synth, kat):
    # the device's global CDF mask against the reference's own
    # compute_MASK_global (known answers) and the oracle's restatement
    for c in kat["mask"]:
        x = synth.random_walk(c["n"], c["seed"]) if c["kind"] == "rw" else \
            synth.ecg_like(c["n"], c["seed"])
        mask, lt = gpu_dtwj.global_mask(x, c["m"], c["w"])
        assert lt == c["table_len"]
        ones = np.flatnonzero(mask == 1.0)
        ref = np.array(c["ones"])
        assert np.setdiff1d(ones, ref).size + np.setdiff1d(ref, ones).size == 0, c
        omask, _ = oracle.mask(x, c["m"], c["w"])
        assert np.array_equal(mask.astype(np.float64), omask)


def test_nan_input_is_rejected(gpu_dtwj, synth):
    x = synth.random_walk(3000, 1)
    x[77] = np.nan
    with pytest.raises(gpu_dtwj.DtwjError) as e:
        gpu_dtwj.join(x, 64, 3)
    assert e.value.code == gpu_dtwj.ERR_NAN


def test_flat_windows_are_excluded(gpu_dtwj, oracle, synth):
    x = synth.random_walk(3000, 7)
    x[1000:1200] = 5.0
    ref = oracle.join(x, 64, 4)
    # with the bounds off as well: flat windows never reach the DTW stage
    for flags in (0, gpu_dtwj.F_NO_DIAG):
        r = gpu_dtwj.join(x, 64, 4, flags)
        _check(r, ref.i, ref.j, ref.dist)


def test_all_flat_series_has_no_pair(gpu_dtwj):
    # no valid window at all: the best-so-far stays +inf and nothing may reach
    # the DTW stage
    r = gpu_dtwj.join(np.full(4000, -1.25), 64, 4)
    assert (r.i, r.j) == (-1, -1) and not np.isfinite(r.dist)


def test_exact_duplicate_resolves_to_lowest_index(gpu_dtwj, synth):
    x = synth.random_walk(3000, 8)
    seg = x[400:480].copy()
    x[1200:1280] = seg
    x[2200:2280] = seg
    r = gpu_dtwj.join(x, 80, 4)
    assert (r.i, r.j) == (400, 1200) and r.dist == 0.0


def test_context_reuse_and_batch(gpu_dtwj, golden):
    cs = golden[:4]
    with gpu_dtwj.Context() as ctx:
        for c in cs:
            r = ctx.join(c["series"], c["m"], c["w"])
            _check(r, c["i"], c["j"], c["dist"], c["name"])
    rs = gpu_dtwj.join_batch([c["series"] for c in cs], [c["m"] for c in cs],
                             [c["w"] for c in cs])
    for r, c in zip(rs, cs):
        _check(r, c["i"], c["j"], c["dist"], c["name"])


def test_cli_drop_in(tmp_path, golden):
    c = [g for g in golden if g["name"] == "rw20k"][0]
    data = tmp_path / "rw20k.txt"
    np.savetxt(data, c["series"], fmt="%.17g")
    tf = tmp_path / "time.txt"
    tf.write_text("1.5\n")
    cli = os.path.join(PKG_DIR, "bin", "dtwj")
    # ratio 0.01 at m=256 -> w = ceil(2.56) = 3, the fixture's band
    out = subprocess.run([cli, str(data), str(tf), "256", "0.01"], capture_output=True,
                         text=True, check=True).stdout
    assert "first min is %d sec min is %d" % (c["i"] + 1, c["j"] + 1) in out
    assert "final distance :%f" % c["dist"] in out
    lines = tf.read_text().splitlines()
    assert len(lines) == 2 and lines[0] == "1.5" and float(lines[1]) > 0


@pytest.mark.parametrize("where", ["first", "last"])
def test_best_pair_at_the_series_ends(gpu_dtwj, oracle, synth, where):
    # the first window (row 0 of every diagonal) and the last window (last
    # column) must be reachable by the sweep
    x = synth.random_walk(4000, 12)
    m, w = 96, 5
    s = x.size - m + 1
    if where == "first":
        x[2100:2100 + m] = x[0:m] * 1.5 + 7.0   # z-normalised copy of window 0
        expect = (0, 2100)
    else:
        x[s - 1:s - 1 + m] = x[1300:1300 + m] - 2.0  # copy of window 1300 at the end
        expect = (1300, s - 1)
    ref = oracle.join(x, m, w)
    r = gpu_dtwj.join(x, m, w)
    assert (ref.i, ref.j) == expect
    _check(r, ref.i, ref.j, ref.dist)


def test_context_reuse_leaves_no_stale_state(gpu_dtwj, oracle, synth):
    # a larger, survivor-rich join first, then smaller ones on the same
    # context: every result must equal a fresh join and the stage counts must
    # stay consistent (no pair is examined that the diagonal bound dropped)
    big = synth.ecg_like(12000, 5)
    xs = [(synth.random_walk(7000, 21), 128, 7), (synth.random_walk(4500, 22), 64, 3)]
    with gpu_dtwj.Context() as ctx:
        ctx.join(big, 128, 7)
        for x, m, w in xs:
            r = ctx.join(x, m, w)
            ref = oracle.join(x, m, w)
            _check(r, ref.i, ref.j, ref.dist)
            later = r.pruned_masked + r.pruned_kim + r.pruned_keogh + r.dtw_calls
            assert later <= r.pairs - r.pruned_fast + 2 * 100, (later, r.pairs - r.pruned_fast)
            assert 0 <= r.i < r.j < x.size - m + 1


def test_band_mask_cell_of_every_residue(gpu_dtwj, synth, oracle):
    # the join's DTW masks one cell per row step, the one holding diagonal
    # w + 1 at (2w + 1) mod C, with the lanes past the band on the q
    # sentinel: every residue of the one-pair-per-warp layouts with up to 8
    # cells per lane (C = 2 for w < 32, 3 to w = 47, 4 to 63, ... 8 to 127)
    # must reproduce the oracle's join
    ws = [5, 31, 32, 33, 34, 52, 53, 64, 65, 66, 67, 68, 80, 81, 82,
          96, 97, 98, 99, 100, 101, 102, 112, 113, 114, 115]
    x = synth.random_walk(1500, 7)
    e = synth.ecg_like(1500, 7)
    with gpu_dtwj.Context() as ctx:
        for w in ws:
            ref = oracle.join(x, 128, w)
            _check(ctx.join(x, 128, w), ref.i, ref.j, ref.dist, ("rw", w))
        for w in (31, 33, 34, 53):
            ref = oracle.join(e, 128, w)
            _check(ctx.join(e, 128, w), ref.i, ref.j, ref.dist, ("ecg", w))


def test_every_band_layout_gives_the_same_join(gpu_dtwj, golden, synth, oracle):
    # the autotuner may pick any layout: each must reproduce the result
    x = synth.random_walk(3500, 6)
    ref = oracle.join(x, 100, 52)
    cases = [(c["series"], c["m"], c["w"], c["i"], c["j"], c["dist"]) for c in golden[:2]]
    cases.append((x, 100, 52, ref.i, ref.j, ref.dist))
    for xs, m, w, i, j, d in cases:
        shapes = gpu_dtwj.band_shapes(min(w, m - 1))
        assert len(shapes) >= 2
        with gpu_dtwj.Context() as ctx:
            for C, G in shapes:
                ctx.set_band(min(w, m - 1), C, G)
                _check(ctx.join(xs, m, w), i, j, d, (m, w, C, G))


def test_autotune_measures_and_applies(gpu_dtwj, synth, tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "dtwj.autotune", os.path.join(PKG_DIR, "autotune.py"))
    at = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(at)
    path = str(tmp_path / "tune.json")
    with gpu_dtwj.Context() as ctx:
        e = at.apply(ctx, 128, 6, path, pairs=512)
    assert e["cells_per_s"] > 0 and e["C"] * e["G"] >= 13
    assert all(t[2] > 0 for t in e["tried"])
    # timed on joins of a sample series (early abandoning included)
    e2 = at.tune(128, 6, None, timer=at.join_timer(synth.ecg_like(6000, 2)))
    assert e2["cells_per_s"] > 0 and e2["C"] * e2["G"] >= 13
    assert all(t[2] > 0 for t in e2["tried"])


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_join_equals_the_whole(gpu_dtwj, golden, world):
    # the shards of one join (run one after the other on this GPU) merge into
    # the whole join's result; every pair is counted by exactly one shard
    for c in [g for g in golden if g["name"] in ("rw20k", "rw6k_m128_w6")]:
        whole = gpu_dtwj.join(c["series"], c["m"], c["w"])
        parts = []
        with gpu_dtwj.Context() as ctx:
            for r in range(world):
                ctx.set_shard(r, world)
                parts.append(ctx.join(c["series"], c["m"], c["w"]))
        merged = gpu_dtwj.merge_results(parts)
        _check(merged, c["i"], c["j"], c["dist"], (c["name"], world))
        assert merged.pairs == whole.pairs


def test_exchanged_best_so_far_feeds_every_shard(gpu_dtwj, golden):
    # the best-so-far exchange between shards (dtwj_ctx_set_exchange): here the
    # callback lowers each shard's best-so-far to the whole join's distance
    # (squared, rounded up to float: the distance of a real pair), as an
    # all-reduce over shards would once the shard holding that pair found it.
    # The shards still merge into the whole join, and they evaluate no more
    # DTWs than without the exchange.
    import torch

    c = [g for g in golden if g["name"] == "rw20k"][0]
    x, m, w = c["series"], c["m"], c["w"]
    whole = gpu_dtwj.join(x, m, w)
    cap = int(np.float32(whole.dist ** 2 * (1 + 1e-6)).view(np.int32))
    calls = []

    def lower(user, ptr, count, stream):
        words = torch.as_tensor(gpu_dtwj._DeviceWords(ptr, count), device="cuda")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            words.clamp_(max=cap)
        calls.append(count)

    plain, fed = [], []
    with gpu_dtwj.Context() as ctx:
        for r in range(2):
            ctx.set_shard(r, 2)
            plain.append(ctx.join(x, m, w))
        ctx.set_exchange(lower, phases=4)
        for r in range(2):
            ctx.set_shard(r, 2)
            fed.append(ctx.join(x, m, w))
        ctx.set_exchange(None)
    assert calls == [1] * 8
    for parts in (plain, fed):
        merged = gpu_dtwj.merge_results(parts)
        _check(merged, c["i"], c["j"], c["dist"], "exchange")
        assert merged.pairs == whole.pairs
    assert sum(p.dtw_calls for p in fed) <= sum(p.dtw_calls for p in plain)


def test_cli_reads_the_reference_file_formats(tmp_path, golden):
    # the series split into the first column of two files (loadfile_2) and
    # into a 4-column matrix (loadfile_) gives the same join as one column
    c = [g for g in golden if g["name"] == "rw20k"][0]
    x = np.asarray(c["series"])
    half = x.size // 2
    fa, fb, fm = tmp_path / "a.txt", tmp_path / "b.txt", tmp_path / "m.txt"
    np.savetxt(fa, np.stack([x[:half], np.arange(half)], 1), fmt="%.17g")
    np.savetxt(fb, x[half:], fmt="%.17g")
    np.savetxt(fm, x.reshape(-1, 4), fmt="%.17g")
    cli = os.path.join(PKG_DIR, "bin", "dtwj")
    tf = tmp_path / "time.txt"
    for extra, data in ((["--format=first-column", "--data2=%s" % fb], fa), (["--format=rows"], fm)):
        out = subprocess.run([cli, str(data), str(tf), "256", "0.01"] + extra, capture_output=True,
                             text=True, check=True).stdout
        assert "first min is %d sec min is %d" % (c["i"] + 1, c["j"] + 1) in out, extra


def test_queue_overflow_sweeps_only_the_chunks_again(gpu_dtwj, synth):
    # With a small DTW queue (DTWJ_QUEUE_CAP, 2^20 pairs; LB_Keogh queue
    # twice that) most pairs of the ECG-like 16k prefix reach DTW, so chunks
    # overflow; each such chunk is swept again in smaller chunks, its counts
    # taken out first.  The result equals the full-queue join and the oracle
    # record, and every pair is counted once: the stage counters add up to
    # the pair count plus at most the seed DTWs (700 slots).
    import json
    from conftest import GOLDEN
    wl = synth.workload("ecg16k_w52")
    x, m, w = wl["series"], wl["m"], wl["w"]
    rec = {r["workload"]: r for r in json.load(open(os.path.join(GOLDEN, "fullsize.json")))}
    rec = rec["ecg16k_w52"]
    with gpu_dtwj.Context() as ctx:
        full = ctx.join(x, m, w)
    os.environ["DTWJ_QUEUE_CAP"] = str(1 << 20)
    try:
        with gpu_dtwj.Context() as ctx:
            small = ctx.join(x, m, w)
    finally:
        del os.environ["DTWJ_QUEUE_CAP"]
    assert (small.i, small.j, small.dist) == (full.i, full.j, full.dist)
    assert (small.i, small.j) == (rec["i"], rec["j"])
    assert abs(small.dist - rec["dist"]) <= 1e-5 * rec["dist"]
    s = x.size - m + 1
    for r in (full, small):
        assert r.pairs == (s - m) * (s - m + 1) // 2
        total = r.pruned_fast + r.pruned_paa + r.pruned_kim + r.pruned_keogh + r.dtw_calls
        assert 0 <= total - r.pairs <= 700, (total, r.pairs)


def test_tuned_join_equals_the_default(gpu_dtwj, synth, tmp_path):
    # whole-join tuning (band layout, DTW CTA size, sweep chunk) on a sample,
    # applied by a context created with the cache: same result as the default
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "dtwj.autotune", os.path.join(PKG_DIR, "autotune.py"))
    at = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(at)
    x = synth.ecg_like(12000, 5)
    m, w = 128, 7
    path = str(tmp_path / "join_tune.json")
    e = at.tune_join(x[:6000].copy(), m, w, path, warps=(1, 8), chunks=(16, 2048))
    assert e["dtw_warps"] in (1, 8) and e["chunk_tiles"] in (16, 2048)
    assert all(t[4] > 0 for t in e["tried"])
    with gpu_dtwj.Context() as ctx:
        plain = ctx.join(x, m, w)
    with gpu_dtwj.Context(tune_cache=path) as ctx:
        tuned = ctx.join(x, m, w)
        assert (tuned.i, tuned.j, tuned.dist) == (plain.i, plain.j, plain.dist)
        assert tuned.pairs == plain.pairs
        for bad in ((3, 0), (0, 8), (0, 5000)):
            with pytest.raises(gpu_dtwj.DtwjError):
                ctx.set_tuning(*bad)
