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
