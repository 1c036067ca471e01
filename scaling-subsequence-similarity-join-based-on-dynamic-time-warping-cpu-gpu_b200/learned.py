"""Training and evaluation of the tile-scoring network of the learned order.

    python <package>/learned.py train --out model.bin [--series 4] [--n 262144] ...
    python <package>/learned.py compare --model model.bin --workload rw4m_motif8

Training data are generated by the method itself on held-out seeds: for each
synthetic series (random walk with planted motifs, as in the learned-ordering
workload but with other seeds) the context reports every diagonal-sweep
tile's 64 features and its exact smallest DTW distance (dtwj_ctx_tiles); the
target is that distance / sqrt(2m), the scale of the distance features.  The
network is trained on the GPU by the library's own BF16 forward/backward
kernels with Adam (dtwj_mlp_train).

`compare` runs the same join in the plain tile order and in the learned order
and reports both times; the top-1 pair must be identical.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

if __package__:
    from . import MLP, Context, F_LEARNED, F_PROFILE, PHASES
    from . import synth
else:  # run as a file: load the package directory as "dtwj"
    import importlib.util

    _here = os.path.dirname(os.path.abspath(__file__))
    if "dtwj" not in sys.modules:
        _spec = importlib.util.spec_from_file_location(
            "dtwj", os.path.join(_here, "__init__.py"), submodule_search_locations=[_here])
        _pkg = importlib.util.module_from_spec(_spec)
        sys.modules["dtwj"] = _pkg
        _spec.loader.exec_module(_pkg)
    from dtwj import MLP, Context, F_LEARNED, F_PROFILE, PHASES
    from dtwj import synth


def training_set(seeds, n: int, m: int, w: int, motifs: int = 8, device: int = 0, log=None):
    """(features [T][64], targets [T]) over the tiles of one series per seed."""
    xs, ys = [], []
    with Context(device) as ctx:
        for sd in seeds:
            x = synth.random_walk(n, sd)
            synth.plant_motifs(x, motifs, m, sd)
            t0 = time.time()
            _, feat, md = ctx.tiles(x, m, w, features=True, min_dist=True)
            ok = np.isfinite(md)
            xs.append(feat[ok])
            ys.append((md[ok] / math.sqrt(2.0 * m)).astype(np.float32))
            if log:
                log("seed %d: %d tiles, exact minima in %.1f s" % (sd, ok.sum(), time.time() - t0))
    return np.concatenate(xs), np.concatenate(ys)


def spearman(a, b) -> float:
    ra = np.argsort(np.argsort(a)).astype(np.float64)
    rb = np.argsort(np.argsort(b)).astype(np.float64)
    ra -= ra.mean()
    rb -= rb.mean()
    return float((ra * rb).sum() / math.sqrt((ra * ra).sum() * (rb * rb).sum()))


def train(args) -> int:
    log = lambda s: print(s, file=sys.stderr, flush=True)  # noqa: E731
    seeds = list(range(args.seed0, args.seed0 + args.series))
    X, y = training_set(seeds, args.n, args.m, args.w, args.motifs, log=log)
    Xv, yv = training_set([args.seed0 + 1000], args.n, args.m, args.w, args.motifs, log=log)
    net = MLP(seed=args.seed0)
    p = net.params
    p[-1] = float(np.mean(y))  # output bias starts at the mean target
    net.params = p
    t0 = time.time()
    loss = net.train(X, y, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed0)
    secs = time.time() - t0
    pv = net.predict(Xv)
    rep = dict(samples=int(X.shape[0]), held_out=int(Xv.shape[0]), epochs=args.epochs,
               train_seconds=secs, train_mse=loss,
               held_out_mse=float(np.mean((pv - yv) ** 2)), target_var=float(np.var(yv)),
               held_out_spearman=spearman(pv, yv))
    net.save(args.out)
    print(json.dumps(rep))
    return 0


def compare(args) -> int:
    wl = synth.workload(args.workload)
    x, m, w = wl["series"], wl["m"], wl["w"]
    net = MLP.load_file(args.model)
    out = {}
    with Context() as ctx:
        ctx.set_model(net)
        for name, fl in (("plain", 0), ("learned", F_LEARNED)) * args.reps:
            r = ctx.join(x, m, w, fl | F_PROFILE)
            out.setdefault(name, []).append(dict(
                seconds=r.seconds_join, i=r.i, j=r.j, dist=r.dist, dtw_calls=r.dtw_calls,
                dtw_cells=r.dtw_cells,
                phases={k: round(v, 4) for k, v in zip(PHASES, r.phase_seconds)}))
    same = len({(d["i"], d["j"], d["dist"]) for v in out.values() for d in v}) == 1
    print(json.dumps(dict(workload=args.workload, identical_top1=same, **out)))
    return 0 if same else 1


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    t.add_argument("--series", type=int, default=4)
    t.add_argument("--seed0", type=int, default=100)
    t.add_argument("--n", type=int, default=262144)
    t.add_argument("--m", type=int, default=256)
    t.add_argument("--w", type=int, default=13)
    t.add_argument("--motifs", type=int, default=8)
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--batch", type=int, default=1024)
    t.add_argument("--lr", type=float, default=1e-3)
    c = sub.add_parser("compare")
    c.add_argument("--model", required=True)
    c.add_argument("--workload", default="rw4m_motif8")
    c.add_argument("--reps", type=int, default=2)
    args = ap.parse_args(argv)
    return train(args) if args.cmd == "train" else compare(args)


if __name__ == "__main__":
    sys.exit(main())
