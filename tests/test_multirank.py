"""The N > 1 path of bench.py on CPU: two gloo ranks, each on its own
independently seeded dataset of the same configuration (weak scaling, no
data-path collective), clustering it with the engine's host replay over the
oracle's distances, then reducing the step time to the maximum over ranks."""
from __future__ import annotations

import os
import socket
import sys
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "mnhn-tree-tools_b200"))
    import bench
    import oracle as O
    import swgpu
    from swgpu import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seed = bench.dataset_seed("2", rank)
    seqs, _ = W.config2(seed=seed, n=240)
    t0 = time.perf_counter()
    D = O.all_pairs(seqs)
    clusters = swgpu.dbscan_from_matrix(D, 300.0, 5)
    ms = 1e3 * (time.perf_counter() - t0) + 50.0 * rank  # ranks finish at different times
    ms_max = bench.max_over_ranks(ms, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = {"seed": seed, "ms": ms, "ms_max": ms_max, "ok": clusters == O.dbscan(D, 300.0, 5),
                 "first": seqs[0][:20]}


def test_two_gloo_ranks_independent_datasets_and_max_time():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0]["seed"] != res[1]["seed"] and res[0]["first"] != res[1]["first"]
    assert res[0]["ok"] and res[1]["ok"]
    want = max(res[0]["ms"], res[1]["ms"])
    assert res[0]["ms_max"] == pytest.approx(want) and res[1]["ms_max"] == pytest.approx(want)


def _split_rank_main(rank, world, port, out):
    """One data set split over gloo ranks: tile groups from swgpu.lpt_partition
    (each rank keeps the pairs of its tiles and 0xFF bytes elsewhere, as a
    partitioned score pass leaves them), then split_pass.combine_bytes."""
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "mnhn-tree-tools_b200"))
    import oracle as O
    import swgpu
    from swgpu import split_pass
    from swgpu import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seqs, _ = W.config2(seed=5, n=200)  # the same data set in every rank
    D = O.all_pairs(seqs).astype(np.uint16)
    n, tb = len(seqs), 32
    nb = (n + tb - 1) // tb
    tiles = [(a, b) for a in range(nb) for b in range(a, nb)]
    cost = np.array([(min(n, (a + 1) * tb) - a * tb) * (min(n, (b + 1) * tb) - b * tb) for a, b in tiles], float)
    order = np.argsort(-cost, kind="stable")
    owner = swgpu.lpt_partition(cost[order], world)
    part = np.full_like(D, 0xFFFF)
    for t, o in zip(order, owner):
        if o != rank:
            continue
        a, b = tiles[t]
        rs, cs = slice(a * tb, (a + 1) * tb), slice(b * tb, (b + 1) * tb)
        part[rs, cs] = D[rs, cs]
        part[cs, rs] = D[cs, rs]
    buf = torch.from_numpy(part.view(np.uint8).copy().reshape(-1))
    split_pass.combine_bytes(buf, dist)
    full = buf.numpy().view(np.uint16).reshape(n, n)
    clusters = swgpu.dbscan_from_matrix(full, 300.0, 5)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = {"exact": bool(np.array_equal(full, D)), "ok": clusters == O.dbscan(D, 300.0, 5),
                 "share": float(cost[order][owner == rank].sum() / cost.sum())}


def test_split_pass_exchange_gives_full_matrix_on_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_split_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0]["exact"] and res[1]["exact"] and res[0]["ok"] and res[1]["ok"]
    assert abs(res[0]["share"] - 0.5) < 0.1


def test_lpt_partition_covers_every_tile_once_and_balances():
    import swgpu
    rng = np.random.default_rng(1)
    for nparts in (1, 2, 3, 8):
        cost = np.sort(rng.pareto(1.5, size=500) + 1)[::-1]
        owner = swgpu.lpt_partition(cost, nparts)
        assert owner.min() >= 0 and owner.max() < nparts and len(owner) == len(cost)
        loads = np.array([cost[owner == p].sum() for p in range(nparts)])
        assert loads.max() - loads.min() <= cost.max() + 1e-9  # greedy LPT bound
