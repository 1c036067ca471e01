"""Autotuner of the DTW band layout, keyed by (m, w), with a JSON cache.

The banded DTW runs G lanes per pair with C band cells per lane; every layout
that covers the band computes the same distances, so the choice is only about
speed.  `tune` times each candidate and keeps the fastest.  The default timer
is band cells per second on exact FP32 DTW of random-walk window pairs
(dtwj_time_band); `join_timer(sample)` times joins of a sample series instead,
which includes early abandoning (groups that share a warp then fall out of
step, which favours one pair per warp).  Results are cached in a JSON file:

    {"m=1024,w=52": {"C": 7, "G": 16, "cells_per_s": ..., "tried": [[C, G, cells_per_s], ...]}}

`apply` sets the cached layout on a context (dtwj_ctx_set_band).

`tune_join` tunes a whole join of one (m, w) on a sample series: the band
layout, the DTW kernel's CTA size in warps and the sweep's tiles per chunk
(dtwj_ctx_set_tuning), by join time.  A Context created with the cache
(tune_cache=, or the DTWJ_TUNE_CACHE environment variable) applies the entry
before its first join of that (m, w).
"""
from __future__ import annotations

import json
import os
import sys

if __package__:
    from . import PHASES, Context, F_PROFILE, band_shapes, time_band
else:  # loaded by path
    _pkg = sys.modules.get("dtwj")
    band_shapes, time_band = _pkg.band_shapes, _pkg.time_band
    Context, F_PROFILE, PHASES = _pkg.Context, _pkg.F_PROFILE, _pkg.PHASES


def join_timer(series, device: int = 0):
    """A timer for `tune` that joins `series` (a representative sample, e.g.
    a prefix of the series to be joined) with each layout and returns the DTW
    stage's band cells per second (`pairs` is ignored)."""
    def timer(m, w, C, G, pairs):
        with Context(device) as ctx:
            ctx.set_band(min(w, m - 1), C, G)
            ctx.join(series, m, w)  # warm-up (kernel loading, graph capture)
            r = ctx.join(series, m, w, F_PROFILE)
        t = r.phase_seconds[PHASES.index("pairs")]
        return r.dtw_cells / t if t > 0 else float("inf")
    return timer


def _key(m: int, w: int) -> str:
    return "m=%d,w=%d" % (m, w)


def load_cache(path: str) -> dict:
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def tune(m: int, w: int, cache_path: str | None = None, pairs: int = 2048, timer=None,
         shapes=None) -> dict:
    """Best layout for (m, w): from the cache if present, else measured (and
    written back to the cache).  `timer(m, w, C, G, pairs)` and `shapes(w)`
    default to the library's measurement and candidate list."""
    cache = load_cache(cache_path)
    k = _key(m, w)
    if k in cache:
        return cache[k]
    timer = timer or (lambda m_, w_, C, G, p: time_band(m_, w_, C, G, p))
    cands = (shapes or band_shapes)(min(w, m - 1))
    tried = [[C, G, float(timer(m, w, C, G, pairs))] for C, G in cands]
    C, G, best = max(tried, key=lambda t: t[2])
    entry = {"C": C, "G": G, "cells_per_s": best, "tried": tried}
    if cache_path:
        cache[k] = entry
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    return entry


def apply(ctx, m: int, w: int, cache_path: str | None = None, **kw) -> dict:
    """Tune (or read the cache for) (m, w) and set the layout on `ctx`."""
    e = tune(m, w, cache_path, **kw)
    ctx.set_band(min(w, m - 1), e["C"], e["G"])
    return e


# ---- whole-join tuning: band layout, DTW CTA size, sweep chunk ----

def join_key(m: int, w: int) -> str:
    return "join:m=%d,w=%d" % (m, w)


def apply_entry(ctx, m: int, w: int, e: dict):
    """Sets a tune_join entry on a context."""
    ctx.set_band(min(w, m - 1), e["C"], e["G"])
    ctx.set_tuning(e["dtw_warps"], e["chunk_tiles"])


def tune_join(series, m: int, w: int, cache_path: str | None = None, device: int = 0,
              warps=(2, 4, 8), chunks=(0, 256, 1024, 2048), measure=None, shapes=None) -> dict:
    """Tunes a join of (m, w) on a sample series (a prefix of the series to be
    joined, or one like it): first the DTW band layout, then the DTW kernel's
    CTA size in warps, then the sweep's tiles per chunk, each by the device
    time of a join of the sample with the others at their best so far (chunk 0
    is the library's default, four tiles per resident CTA of the sweep).  The
    entry is cached under join_key(m, w); a Context created with this cache
    (tune_cache=, or DTWJ_TUNE_CACHE) applies it before its first join of
    (m, w).  measure(C, G, warps, chunk) -> seconds defaults to a warm-up join
    and a timed join on a fresh context."""
    cache = load_cache(cache_path)
    k = join_key(m, w)
    if k in cache:
        return cache[k]

    def default_measure(C, G, wv, ch):
        with Context(device) as ctx:
            ctx.set_band(min(w, m - 1), C, G)
            ctx.set_tuning(wv, ch)
            ctx.join(series, m, w)  # warm-up: kernel loading, graph capture
            return ctx.join(series, m, w).seconds_join

    measure = measure or default_measure
    cands = (shapes or band_shapes)(min(w, m - 1))
    tried = []

    def run(C, G, wv, ch):
        t = float(measure(C, G, wv, ch))
        tried.append([C, G, wv, ch, t])
        return t

    best = min(((run(C, G, 0, 0), C, G) for C, G in cands))
    _, C, G = best
    wbest = min(((run(C, G, wv, 0), wv) for wv in warps))[1]
    t, cbest = min(((run(C, G, wbest, ch), ch) for ch in chunks))
    entry = {"C": C, "G": G, "dtw_warps": wbest, "chunk_tiles": cbest, "join_seconds": t,
             "tried": tried}
    if cache_path:
        cache = load_cache(cache_path)
        cache[k] = entry
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    return entry
