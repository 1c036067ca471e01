"""bench.py's algorithmic-bytes model counts the diagonal-sweep tiles the way
the library lays them out (the same enumeration as the CPU restatement in
features_ref.tiles, which the GPU features test ties to the device tiles)."""
import os
import sys

import features_ref

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_bench_tile_count_matches_the_layout():
    for n, m in [(4500, 32), (20000, 256), (100000, 1024), (262144, 512)]:
        tiles = features_ref.tiles(n, m)
        ntiles, rows_sum = bench.sweep_tiles(n, m)
        assert ntiles == len(tiles), (n, m)
        assert sum(r for (_, _, r) in tiles) == rows_sum


def test_launch_traffic_scales_the_capture_by_tiles(tmp_path):
    import json
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles",
                        "ncu_traffic_rw1m_motif.json")
    rec = json.load(open(path))
    tiles = rec["tiles"]
    for k in ("k_lb", "k_paa"):
        b = rec["bytes_per_launch"][k]
        assert bench.launch_traffic(path, k, tiles) == b
        assert abs(bench.launch_traffic(path, k, 1.5 * tiles) - 1.5 * b) < 1e-6 * b
    assert bench.launch_traffic(path, "k_none", tiles) is None
    assert bench.launch_traffic(str(tmp_path / "missing.json"), "k_lb", tiles) is None
    # the bench workload's tiles over its launches: 1M samples, m = 1024
    ntiles, _ = bench.sweep_tiles(1_000_000, 1024)
    assert 1024 * 100 < ntiles < 1776 * 100
