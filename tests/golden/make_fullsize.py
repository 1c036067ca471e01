"""Generates tests/golden/fullsize.json: the oracle's top-1 pair on the
full-size named workloads, so the GPU tests can check the join at those
sizes against it (indices exact, distance within 1e-5 relative).

    python tests/golden/make_fullsize.py rw1m_motif rw262k_w52 ...

The oracle (oracle/dtwj_oracle.c, OpenMP FP64) is itself pinned to the
reference's own outputs by tests/test_oracle.py.  Each workload is generated
from its seed by synth.workload(); the record holds the seed-defining name,
the sizes, the pair, the FP64 distance, the oracle's pruning counters, its
wall time and thread count, and the host CPU model.  Records of workloads not
named on the command line are kept.
"""
from __future__ import annotations

import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from conftest import Oracle, load_synth  # noqa: E402

OUT = os.path.join(HERE, "fullsize.json")


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


def main(names):
    synth = load_synth()
    oracle = Oracle()
    recs = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            recs = {r["workload"]: r for r in json.load(f)}
    for name in names:
        wl = synth.workload(name)
        x = wl["series"]
        t = time.time()
        r = oracle.join(x, wl["m"], wl["w"])
        wall = time.time() - t
        rec = dict(workload=name, n=int(x.size), m=wl["m"], w=wl["w"], i=int(r.i), j=int(r.j),
                   dist=float(r.dist), seed_bsf=float(r.seed_bsf), pairs=int(r.pairs),
                   pruned_fast=int(r.pruned_fast), pruned_masked=int(r.pruned_masked),
                   pruned_kim=int(r.pruned_kim), pruned_keogh=int(r.pruned_keogh),
                   dtw_calls=int(r.dtw_calls), wall_seconds=round(wall, 1), threads=int(r.threads),
                   cpu=cpu_model())
        if "planted" in wl:
            rec["planted"] = [list(map(int, p)) for p in wl["planted"]]
        recs[name] = rec
        print(json.dumps(rec), flush=True)
        with open(OUT, "w") as f:
            json.dump(sorted(recs.values(), key=lambda r: r["workload"]), f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
