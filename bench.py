#!/usr/bin/env python3
"""Benchmark of the top-1 z-normalised DTW subsequence self-join.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]
    python bench.py --batch 4096     (the batched-join configuration, one line)

Workload (default): one float64 random walk, n = 1,000,000, seed 1, with one
planted motif pair (length-1024 sum of 3 sines, N(0, 0.1) noise, +-5 % time
warp), m = 1024, ratio 0.05 -> w = 52.  A step is one complete join of that
series (ED profile, seeds, diagonal sweep, per-pair bounds, DTW, FP64
verification).  The metric is join throughput in candidate pairs per second
(every pair (i, j) with j - i >= m counts once); join time and DTW cells/s
ride along.

Timing: W untimed warm-up joins, then exactly K joins bracketed by a
synchronize; `value` uses the device time the library measures with CUDA
events on its own stream (inputs resident in HBM).  `e2e` repeats the join
through the public host-pointer API from pinned memory, so the H2D copy of
the series and the D2H read of the result are inside the timed region.  The
series (8 MB) and the per-series arrays (~250 MB) are re-read from HBM on
every join; the sweep's working set far exceeds what one join leaves in L2.

--impl reference times the reference's own CPU implementation (CPU_version1,
built from its sources into oracle/_ref/) on bounded 16,384-sample slices of
the same series, one single-threaded process per physical host core, by the
reference's own join interval; its line names the slices in config.workload
and extrapolates the single-core time of the full series.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "Join time & DTW cells/s, n=1M m=1024 r=0.05: learned-order vs plain GPU, exact"
UNIT = "pairs/s"


def _load_pkg():
    from conftest import load_package, load_synth  # path helpers only
    return load_package(), load_synth()


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured", d.get("sm_max_mhz", 1965.0)
    return 6650.0, "fallback", 1965.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def sweep_tiles(n: int, m: int):
    """(tiles, summed rows of the lag groups) of the diagonal sweep of one
    series: lag groups of 896 lags from m, each split into tiles of at most
    4032 rows, as the library lays them out."""
    s = n - m + 1
    ntiles, rows_sum = 0, 0
    for L0 in range(m, s, 896):
        rows = s - L0
        ntiles += (rows + 4031) // 4032
        rows_sum += rows
    return ntiles, rows_sum


def launch_traffic(tfile: str, kname: str, tiles_per_launch: float):
    """DRAM bytes per launch of a sweep kernel: the ncu capture of one launch
    over a full chunk (profiles/ncu_traffic_rw1m_motif.json, its "tiles"
    field), scaled to this run's average tiles per launch, since each tile
    moves the same bytes.  None without a capture."""
    if not os.path.exists(tfile):
        return None
    with open(tfile) as f:
        rec = json.load(f)
    b = rec.get("bytes_per_launch", {}).get(kname)
    tiles = rec.get("tiles")
    if b is None or not tiles:
        return None
    return b * tiles_per_launch / tiles


def _dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def _max_over_ranks(v: float, dist, local: int) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda:%d" % local)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def host_cpu():
    """(model name, physical cores available to this process)."""
    model, cores_per_socket, sockets = "unknown", None, None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=30).stdout
        for line in out.splitlines():
            k, _, v = line.partition(":")
            k, v = k.strip(), v.strip()
            if k == "Model name":
                model = v
            elif k == "Core(s) per socket":
                cores_per_socket = int(v)
            elif k == "Socket(s)":
                sockets = int(v)
    except (OSError, ValueError, subprocess.TimeoutExpired):
        pass
    avail = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    phys = cores_per_socket * sockets if cores_per_socket and sockets else avail
    return model, max(1, min(avail, phys))


def cpu_sample_reference(x: np.ndarray, m: int, w: int, n_sample: int, procs: int):
    """Runs the reference CPU join (oracle/_ref/ref_join, CPU_version1's
    DTWMotifDiscoveryGUI) on `procs` disjoint n_sample-long slices of x at
    once, one single-threaded process each.  The rate of a process is its
    slice's pairs over the reference's own join interval (the clock() time it
    appends to its time file, CPU_version1/new_dtw_motifGUI.cpp:298,577-584:
    the sweep after mpx_v2 and the O(n m) set-up).  Returns (summed pairs/s
    of the processes, per-process rates, pairs per slice, wall seconds)."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "ref_join")
    if not os.path.exists(ref_bin):
        return None
    files = []
    tmp = tempfile.mkdtemp(prefix="dtwj_ref_")
    nslices = max(1, x.size // n_sample)
    for k in range(procs):
        lo = (k % nslices) * n_sample
        path = os.path.join(tmp, "s%d.f64" % k)
        x[lo:lo + n_sample].astype("<f8").tofile(path)
        files.append(path)
    t0 = time.perf_counter()
    ps = [subprocess.Popen([ref_bin, f, str(m), str(w)], stdout=subprocess.PIPE,
                           stderr=subprocess.DEVNULL, text=True) for f in files]
    outs = [p.communicate()[0] for p in ps]
    wall = time.perf_counter() - t0
    s = n_sample - m + 1
    pairs = (s - m) * (s - m + 1) // 2
    rates = []
    for o in outs:
        try:
            line = o.strip().splitlines()[-1].replace(": -nan", ": null").replace(": nan", ": null")
            r = json.loads(line)
        except (IndexError, json.JSONDecodeError):
            continue
        if r.get("rc") == 0 and r.get("join_seconds", 0) > 0:
            rates.append(pairs / r["join_seconds"])
    for f in files:
        os.unlink(f)
    os.rmdir(tmp)
    if not rates:
        return None
    return sum(rates), rates, pairs, wall


def cpu_sample_port(x: np.ndarray, m: int, w: int, n_sample: int, threads: int):
    """The oracle's C restatement (OpenMP) on one sample; returns pairs/s."""
    from conftest import Oracle, ORACLE_LIB
    if not os.path.exists(ORACLE_LIB):
        return None
    orc = Oracle()
    y = np.ascontiguousarray(x[:n_sample])
    t0 = time.perf_counter()
    r = orc.join(y, m, w, threads=threads)
    wall = time.perf_counter() - t0
    return r.pairs / wall, wall, r.pairs, r.threads


def extrapolate_reference(pairs_total: int, rate_1core: float, n_sample: int):
    """Single-core reference join time of the whole series, extrapolated
    proportionally to the pair count from the measured per-core rate."""
    return {"join_seconds_1core": pairs_total / rate_1core,
            "basis": "pairs of the full series / the reference's per-core join rate "
                     "measured on %d-sample slices" % n_sample,
            "label": "extrapolated"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    _, synth = _load_pkg()
    wl = synth.workload(args.workload)
    x, m, w = wl["series"], wl["m"], wl["w"]
    model, cores = host_cpu()
    n_sample = args.ref_sample
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_join")):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/ref_join not built (needs the reference "
                                         "sources: oracle/build_ref.sh)"}))
        return 0
    for _ in range(args.warmup):
        cpu_sample_reference(x, m, w, n_sample, cores)
    vals, walls, per_core = [], [], []
    for _ in range(args.steps):
        v, rates, pairs, wall = cpu_sample_reference(x, m, w, n_sample, cores)
        vals.append(v)
        walls.append(wall)
        per_core.extend(rates)
    value = statistics.median(vals)
    core_rate = statistics.median(per_core)
    n = x.size
    s = n - m + 1
    pairs_total = (s - m) * (s - m + 1) // 2
    sample = ("%d single-threaded processes (one per physical core), each CPU_version1 "
              "DTWMotifDiscoveryGUI on its own %d-sample slice of the series; pairs/s = the "
              "slices' pairs over the reference's own join interval (clock() t1->t2, "
              "new_dtw_motifGUI.cpp:298,577), summed over the processes; median of %d steps"
              % (cores, n_sample, args.steps))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * statistics.median(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random walk + planted motif)",
        "config": {"workload": "%s[%d-sample slices x %d]" % (args.workload, n_sample, cores),
                   "n": n_sample, "m": m, "w": w,
                   "pairs_per_slice": (n_sample - 2 * m + 1) * (n_sample - 2 * m + 2) // 2,
                   "parallelism": "%d processes" % cores},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "cpu": model, "per_core": core_rate, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_series": dict(extrapolate_reference(pairs_total, core_rate, n_sample),
                            workload=args.workload, n=int(n),
                            join_seconds_all_cores=pairs_total / value),
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    world, rank, local, dist = _dist_init()
    dtwj, synth = _load_pkg()
    wl = synth.workload(args.workload)
    x, m, w = wl["series"], wl["m"], wl["w"]
    n = x.size
    s = n - m + 1
    pairs_total = (s - m) * (s - m + 1) // 2
    try:
        import torch
        have_torch = torch.cuda.is_available()
    except ImportError:
        have_torch = False
    if have_torch:
        torch.cuda.set_device(local)
        xd = torch.from_numpy(x).to("cuda:%d" % local)
        xh = torch.from_numpy(x).pin_memory()
        dptr, hptr = xd.data_ptr(), xh.data_ptr()
    else:
        raise SystemExit("bench.py needs torch with CUDA for device buffers")
    ctx = dtwj.Context(local)
    if world > 1:
        # one join spread over the ranks: rank r sweeps the tiles t % world == r,
        # and after each of 8 sweep phases the ranks lower their best-so-far to
        # the smallest any rank has found (an NCCL all-reduce of one word on the
        # join's stream); every rank runs the same joins, so the same collectives
        ctx.set_shard(rank, world)
        ctx.set_exchange(dtwj.make_exchange(None, local), 8)
    # F_PROFILE records CUDA events around every launch group on the join's
    # stream (no synchronisation), so the timed joins also give the per-phase
    # device times the roofline uses.
    flags = dtwj.F_PROFILE | (dtwj.F_PETITJEAN if args.petitjean else 0)
    for _ in range(args.warmup):
        ctx.join_device(dptr, n, m, w, flags)
    _barrier(dist)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    results = [ctx.join_device(dptr, n, m, w, flags) for _ in range(args.steps)]
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    dev_seconds = sum(r.seconds_join for r in results)
    dev_seconds = _max_over_ranks(dev_seconds, dist, local)
    r0 = results[-1]
    if dist is not None:
        # the shards' results combine into the join's result
        gathered = [None] * world
        dist.all_gather_object(gathered, r0.__dict__)
        r0 = dtwj.merge_results(dtwj.JoinResult(**g) for g in gathered)
    # every pair of the join is swept by exactly one rank: the job processes
    # pairs_total pairs per step, in the slowest rank's device time
    value = pairs_total * args.steps / dev_seconds

    # per-phase device time and launches, averaged over the timed joins
    phases = {p: sum(r.phase_seconds[k] for r in results) / args.steps
              for k, p in enumerate(dtwj.PHASES)}
    launches = {p: sum(r.phase_launches[k] for r in results) / args.steps
                for k, p in enumerate(dtwj.PHASES)}
    dominant = max(phases, key=phases.get)

    # the same join in the learned tile order (the committed network), for
    # the plain-vs-learned comparison the metric names; top-1 must not change
    learned = None
    model_path = os.path.join(os.path.dirname(dtwj.LIB_PATH), "..", "tile_mlp_rw_m256.bin")
    if os.path.exists(model_path) and not args.no_learned and args.learned_reps > 0:
        net = dtwj.MLP.load_file(os.path.abspath(model_path), device=local)
        ctx.set_model(net)
        runs = {"plain": [], "learned": []}
        # warm-up of the learned path (its feature, network and sort kernels load
        # on first use), as the timed joins above had theirs
        for _ in range(max(1, args.warmup // 3)):
            ctx.join_device(dptr, n, m, w, flags | dtwj.F_LEARNED)
        for _ in range(args.learned_reps):  # alternating, so drift hits both alike
            for name, fl in (("plain", flags), ("learned", flags | dtwj.F_LEARNED)):
                runs[name].append(ctx.join_device(dptr, n, m, w, fl))
        ctx.set_model(None)

        def stats(rs):
            t = [r.seconds_join for r in rs]
            return {"mean": statistics.mean(t), "sd": statistics.stdev(t) if len(t) > 1 else 0.0,
                    "dtw_calls": rs[-1].dtw_calls, "dtw_cells": rs[-1].dtw_cells}
        sp, sl = stats(runs["plain"]), stats(runs["learned"])
        learned = {"reps": args.learned_reps, "plain_join_seconds": sp, "learned_join_seconds": sl,
                   "gain": 1.0 - sl["mean"] / sp["mean"],
                   "identical_top1": len({(r.i, r.j, r.dist) for v in runs.values() for r in v}) == 1
                   if world == 1 else None,
                   "model": "tile_mlp_rw_m256.bin (trained on m=256 random walks)"}

    # e2e through the host-pointer API (pinned host buffer)
    fn = dtwj.load().dtwj_ctx_join
    R = dtwj._Result
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(args.steps):
        rr = R()
        rc = fn(ctx._h, ctypes.cast(ctypes.c_void_p(hptr), ctypes.POINTER(ctypes.c_double)),
                n, m, w, flags, ctypes.byref(rr))
        assert rc == 0, dtwj.strerror(rc)
    torch.cuda.synchronize()
    e2e_wall = _max_over_ranks(time.perf_counter() - t1, dist, local)

    hbm_peak, peak_kind, sm_max = _peaks()
    # Algorithmic DRAM bytes of the three sweep kernels over one join (the
    # data each must move at least once; averaged per launch below):
    #   k_lb    reads the six per-index FP64 operands of its rows and columns
    #           ((2 rows + 896 lags) x 48 B per tile) and writes the survivor
    #           bits (896 lags x 126 words x 4 B per tile)
    #   k_paa   reads those bits and the 16-byte block means of the windows a
    #           tile covers (rows + 896 lags + m samples per tile), and writes
    #           one 16-byte LB_Keogh candidate per pair that passes the
    #           block-mean and endpoint bounds (k_runs, the masked cascade's
    #           filter, in its place under F_MASKED_CASCADE)
    #   k_keogh reads the candidates and writes an 8-byte DTW entry per survivor
    ntiles, rows_sum = sweep_tiles(n, m)
    bits_bytes = ntiles * 896 * 126 * 4
    kq_entries = r0.pruned_keogh + r0.dtw_calls  # pairs that reached LB_Keogh (seeds aside)
    alg = {
        "diag": ("k_lb", (2 * rows_sum + ntiles * 896) * 48 + bits_bytes),
        "runs": ("k_paa", bits_bytes + 16 * (rows_sum + ntiles * (896 + m)) + 16 * kq_entries),
        "keogh": ("k_keogh", 16 * kq_entries + 8 * r0.dtw_calls),
    }
    sweep_phases = [p for p in ("runs", "keogh", "diag") if phases.get(p, 0) > 0]
    roof_phase = max(sweep_phases, key=lambda p: phases[p]) if sweep_phases else "diag"
    kname, alg_bytes = alg[roof_phase]
    nl = max(1, launches[roof_phase])
    per_launch_s = phases[roof_phase] / nl
    achieved_gbs = alg_bytes / max(phases[roof_phase], 1e-12) / 1e9
    traffic = None
    if args.workload == "rw1m_motif" and kname in ("k_lb", "k_paa"):
        traffic = launch_traffic(os.path.join(ROOT, "profiles", "ncu_traffic_rw1m_motif.json"),
                                 kname, ntiles / nl)
    fp64_flops = pairs_total * 12.0  # k_lb: 2 recurrences x 2 DFMA + 2 DFMA tests per pair
    fp64_peak = 148 * 64 * 2 * sm_max * 1e6 / 1e12
    cells_per_s = r0.dtw_cells / max(phases.get("pairs", 1e-12) + phases.get("seeds", 0), 1e-12)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        model, _ = host_cpu()
        got = cpu_sample_reference(x, m, w, args.cpu_sample, 1)
        if got is not None:
            v, rates, p, cw = got
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "cpu": model,
                   "sample": "first %d samples of the series, m=%d w=%d, CPU_version1 "
                             "DTWMotifDiscoveryGUI; pairs/s = %d pairs over the reference's own "
                             "join interval (clock() t1->t2, new_dtw_motifGUI.cpp:298,577); "
                             "process wall time %.1f s (with mpx_v2)"
                             % (args.cpu_sample, m, w, p, cw),
                   "full_series": extrapolate_reference(pairs_total, v, args.cpu_sample)}
        else:
            got = cpu_sample_port(x, m, w, args.cpu_sample, 1)
            if got is not None:
                v, cw, p, th = got
                cpu = {"value": v, "unit": UNIT, "cores": th, "kind": "port", "cpu": model,
                       "sample": "first %d samples, oracle C restatement, %.1f s"
                                 % (args.cpu_sample, cw)}
    gpu_launches = int(sum(launches.values()) * args.steps)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * dev_seconds / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic (seeded random walk + planted motif)",
        "config": {"workload": args.workload, "n": n, "m": m, "w": w,
                   "pairs_per_join": pairs_total, "l2": "inputs+working set > L2 per join",
                   "parallelism": "tile shards x%d" % world if world > 1 else "single",
                   "lb_petitjean": bool(args.petitjean)},
        "join_seconds": dev_seconds / args.steps,
        "result": {"i": r0.i, "j": r0.j, "dist": r0.dist},
        "pruned": {"fast": r0.pruned_fast, "paa": r0.pruned_paa, "masked": r0.pruned_masked,
                   "petitjean": r0.pruned_petitjean,
                   "kim": r0.pruned_kim,
                   "keogh": r0.pruned_keogh, "dtw_calls": r0.dtw_calls,
                   "dtw_abandoned": r0.dtw_abandoned},
        "dtw_cells_per_s": cells_per_s,
        # DTW stage against its issue roofline: 5 operations per band cell
        # (subtract, square-add, three-input minimum, band mask) on 148 SMs x
        # 128 lanes at the maximum SM clock
        "dtw_roofline": {"achieved": cells_per_s, "peak": 148 * 128 * sm_max * 1e6 / 5.0,
                         "unit": "cells/s",
                         "frac": cells_per_s / (148 * 128 * sm_max * 1e6 / 5.0)},
        "phase_seconds": phases,
        "roofline": {"bound": "hbm", "kernel": kname, "phase": roof_phase,
                     "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved_gbs / hbm_peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg_bytes / nl,
                     "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                     "per_launch_ms": 1000 * per_launch_s,
                     "note": "issue-bound, not HBM-bound: see profiles/"},
        "issue_roofline": {"pipe": "fp64", "kernel": "k_lb",
                           "achieved": fp64_flops / max(phases["diag"], 1e-12) / 1e12,
                           "peak": fp64_peak, "unit": "TFLOP/s",
                           "frac": fp64_flops / max(phases["diag"], 1e-12) / 1e12 / fp64_peak,
                           "peak_kind": "nominal 148 SM x 64 DFMA/clk x max clock"},
        "dominant_phase": dominant,
        "learned_order": learned,
        "cpu_baseline": cpu,
        "e2e": {"value": pairs_total * args.steps / e2e_wall, "unit": UNIT,
                "h2d_bytes_per_step": int(x.nbytes), "d2h_bytes_per_step": 360},
        "gpu_launches": gpu_launches,
        "clocks": clk,
        "wall_seconds_timed": wall,
    }
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """The batched-join configuration: args.batch series of uneven length
    (log-uniform 2,000-65,536 samples), half random walks and half ECG-like,
    m from {64, 128, 256}, ratio 0.05, each with its own top-1 pair.  Times
    dtwj_join_batch (the series of one (m, w) joined together, one pass each)
    against the same series joined one by one on one context, both from host
    buffers (H2D inside the timed region), and checks that every series gets
    the same pair and distance both ways."""
    dtwj, synth = _load_pkg()
    items = synth.batch_workload(count=args.batch)
    xs = [it["series"] for it in items]
    ms = [it["m"] for it in items]
    ws = [it["w"] for it in items]
    samples = int(sum(x.size for x in xs))
    # warm-up: kernels loaded for every (m, w) group
    warm = []
    for mm in (64, 128, 256):
        warm += [k for k in range(len(items)) if ms[k] == mm][:2]
    dtwj.join_batch([xs[k] for k in warm], [ms[k] for k in warm], [ws[k] for k in warm])
    t0 = time.perf_counter()
    rb = dtwj.join_batch(xs, ms, ws)
    t_batch = time.perf_counter() - t0
    with dtwj.Context() as ctx:
        for k in warm:
            ctx.join(xs[k], ms[k], ws[k])
        t0 = time.perf_counter()
        r1 = [ctx.join(x, m, w) for x, m, w in zip(xs, ms, ws)]
        t_one = time.perf_counter() - t0
    same = all((a.i, a.j, a.dist) == (b.i, b.j, b.dist) for a, b in zip(rb, r1))
    groups = sorted({(m, dtwj.band(m, 0.05)) for m in ms})
    line = {
        "metric": "batched join of %d series (config 4), series/s" % len(items),
        "value": len(items) / t_batch, "unit": "series/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "higher_is_better": True, "dtype": "f64+f32", "data": "synthetic (seeded)",
        "config": {"workload": "batch_workload(count=%d, seed=5)" % len(items),
                   "samples": samples, "groups_m_w": groups},
        "batch_seconds": t_batch, "one_by_one_seconds": t_one,
        "speedup_vs_one_by_one": t_one / t_batch, "identical_per_series": same,
        "timing": "host wall clock around the public API calls (series uploaded inside)",
    }
    print(json.dumps(line))
    return 0 if same else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rw1m_motif")
    ap.add_argument("--cpu-sample", type=int, default=16384)
    ap.add_argument("--ref-sample", type=int, default=16384)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--learned-reps", type=int, default=5)
    ap.add_argument("--petitjean", action="store_true",
                    help="joins with the LB_Petitjean stage (DTWJ_F_PETITJEAN)")
    ap.add_argument("--batch", type=int, default=0,
                    help="time the batched join of this many series (config 4) instead")
    args = ap.parse_args()
    if args.batch > 0:
        return run_batch(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
