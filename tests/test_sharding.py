"""Sharding one join over ranks (CPU): the result merge, and the exchange of
the shards' results through torch.distributed with gloo, world size 2."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package


def _res(dtwj, i, j, dist_, **kw):
    base = dict(i=i, j=j, dist=dist_, dist_fp32=dist_, seed_bsf=kw.get("seed", 9.0), pairs=10,
                pruned_fast=5, pruned_kim=1, pruned_masked=1, pruned_keogh=1, dtw_calls=2,
                dtw_abandoned=1, dtw_cells=100, candidates=1, seconds_join=kw.get("t", 1.0),
                seconds_total=2.0, n=1000, m=16, w=2, phase_seconds=[0.1] * 8,
                phase_launches=[1] * 8, pruned_paa=3)
    return dtwj.JoinResult(**base)


def test_merge_is_the_lexicographic_minimum():
    dtwj = load_package()
    a = _res(dtwj, 10, 40, 1.5, t=2.0)
    b = _res(dtwj, 7, 90, 1.5, t=3.0, seed=4.0)   # same distance, lower i wins
    c = _res(dtwj, 3, 30, 1.7)
    none = _res(dtwj, -1, -1, float("inf"))
    r = dtwj.merge_results([a, none, b, c])
    assert (r.i, r.j, r.dist) == (7, 90, 1.5)
    assert r.pairs == 40 and r.dtw_cells == 400 and r.seconds_join == 3.0 and r.seed_bsf == 4.0
    assert dtwj.merge_results([none, none]).i == -1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dtwj = load_package()
        # each rank's shard result: rank 1 holds the best pair
        table = {0: (5, 600, 2.25), 1: (44, 900, 1.125)}

        def fake(r, wsize):
            assert wsize == world
            i, j, d = table[r]
            return _res(dtwj, i, j, d, t=1.0 + r)

        m = dtwj.join_sharded(None, 16, 2, result_fn=fake)
        out[rank] = (m.i, m.j, m.dist, m.pairs, m.seconds_join)
    finally:
        dist.destroy_process_group()


def test_sharded_join_exchange_gloo_two_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == (44, 900, 1.125, 20, 2.0)


def _bsf_worker(rank, world, port, out):
    # the best-so-far exchange between shards: every rank's words become the
    # elementwise minimum of all ranks' words (float bits of squared
    # distances, viewed as int32: non-negative floats order like their bits)
    import struct

    import torch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dtwj = load_package()

        def bits(v):
            return struct.unpack("<i", struct.pack("<f", v))[0]

        mine = {0: [2.0, float("inf"), 0.75, 5.0], 1: [1.5, 3.0, 0.75, float("inf")]}[rank]
        words = torch.tensor([bits(v) for v in mine], dtype=torch.int32)
        for _ in range(3):  # one call per sweep phase; idempotent once equal
            dtwj.bsf_allreduce(words)
        out[rank] = [struct.unpack("<f", struct.pack("<i", int(b)))[0] for b in words.tolist()]
    finally:
        dist.destroy_process_group()


def test_best_so_far_exchange_gloo_two_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_bsf_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == [1.5, 3.0, 0.75, 5.0]


def test_float_bits_order_like_floats():
    # the exchange takes the minimum of the words' integer values: for the
    # non-negative squared distances and +inf this is the minimum distance
    import numpy as np

    v = np.array([0.0, 1e-30, 1.0, 1.5, 2.0, 3.4e38, np.inf], dtype=np.float32)
    b = v.view(np.int32)
    assert np.all(np.diff(b) > 0) and b.max() < 2**31 - 1
