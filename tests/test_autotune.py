"""Autotuner cache logic (CPU): candidate layouts, selection of the fastest,
JSON cache round trip."""
import json
import os
import sys

import pytest

from conftest import PKG_DIR, load_package


def _autotune():
    load_package()
    import importlib.util
    spec = importlib.util.spec_from_file_location("dtwj.autotune", os.path.join(PKG_DIR, "autotune.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dtwj.autotune"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_candidate_layouts_cover_the_band():
    dtwj = load_package()
    for w in (0, 1, 3, 13, 26, 52, 103, 255):
        shapes = dtwj.band_shapes(w)
        assert shapes, w
        for C, G in shapes:
            assert C * G >= 2 * w + 1 and G in (4, 8, 16, 32), (w, C, G)
    assert dtwj.band_shapes(256) == []


def test_tune_picks_the_fastest_and_caches(tmp_path):
    at = _autotune()
    path = str(tmp_path / "tune.json")
    calls = []

    def timer(m, w, C, G, pairs):
        calls.append((C, G))
        return 1000.0 / (abs(C * G - 64) + 1)  # fastest: the layout closest to 64 cells

    e = at.tune(256, 13, path, timer=timer)
    assert (e["C"], e["G"]) == min(((C, G) for C, G, _ in e["tried"]), key=lambda t: abs(t[0] * t[1] - 64))
    assert len(calls) == len(e["tried"])
    saved = json.load(open(path))
    assert saved["m=256,w=13"]["C"] == e["C"]
    # second call: from the cache, no measurement
    calls.clear()
    assert at.tune(256, 13, path, timer=timer) == saved["m=256,w=13"]
    assert not calls


def test_tune_join_searches_each_knob_and_caches(tmp_path):
    at = _autotune()
    path = str(tmp_path / "tune.json")
    calls = []

    def measure(C, G, warps, chunk):
        calls.append((C, G, warps, chunk))
        # fastest: the layout with 64 cells, 8 warps, chunks of 256 tiles
        return abs(C * G - 64) + (0 if warps == 8 else 1) + (0 if chunk == 256 else 1)

    shapes = lambda w: [(2, 32), (4, 16), (7, 4)]
    e = at.tune_join(None, 256, 13, path, measure=measure, shapes=shapes)
    assert (e["C"], e["G"], e["dtw_warps"], e["chunk_tiles"]) == (2, 32, 8, 256)
    # three layouts, three CTA sizes, four chunk sizes (the default among them)
    assert len(calls) == 3 + 3 + 4 and len(e["tried"]) == 10
    assert [c[3] for c in calls[-4:]] == [0, 256, 1024, 2048]
    saved = json.load(open(path))
    assert saved[at.join_key(256, 13)]["dtw_warps"] == 8
    calls.clear()
    assert at.tune_join(None, 256, 13, path, measure=measure, shapes=shapes) == saved[at.join_key(256, 13)]
    assert not calls
