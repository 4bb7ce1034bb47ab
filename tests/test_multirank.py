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


class _TileEngine:
    """Stand-in for the engine's exchange calls on the host: a uint16 matrix
    in which this rank holds the pairs of its own tiles (0xFFFF elsewhere),
    tile rectangles (rows ra .. ra+nra-1 x columns b .. b+nb-1, both
    triangles) owned as swgpu.lpt_partition assigns them."""

    def __init__(self, D, rank, world, tb=24):
        import ctypes as C
        import swgpu
        self.C = C
        n = D.shape[0]
        nb = (n + tb - 1) // tb
        rects = [(a * tb, min(n, (a + 1) * tb) - a * tb, b * tb, min(n, (b + 1) * tb) - b * tb)
                 for a in range(nb) for b in range(a + 1)]
        cost = np.array([r[1] * r[3] for r in rects], float)
        order = np.argsort(-cost, kind="stable")
        self.rects = [rects[t] for t in order]
        self.owner = swgpu.lpt_partition(cost[order], world)
        self.rank = rank
        self.M = np.full_like(D, 0xFFFF)
        for (ra, nra, b0, nb_), o in zip(self.rects, self.owner):
            if o == rank:
                self.M[ra:ra + nra, b0:b0 + nb_] = D[ra:ra + nra, b0:b0 + nb_]
                self.M[b0:b0 + nb_, ra:ra + nra] = D[b0:b0 + nb_, ra:ra + nra]

    def _mine(self, part):
        return [r for r, o in zip(self.rects, self.owner) if o == part]

    def partition_bytes(self, part):
        return 2 * sum(r[1] * r[3] for r in self._mine(part))

    def partition_pack(self, ptr):
        blocks = [self.M[ra:ra + nra, b0:b0 + nb].ravel() for ra, nra, b0, nb in self._mine(self.rank)]
        flat = np.concatenate(blocks) if blocks else np.zeros(0, np.uint16)
        self.C.memmove(ptr, flat.ctypes.data, flat.nbytes)

    def partition_unpack(self, part, ptr, offset, nbytes):
        buf = np.frombuffer((self.C.c_char * nbytes).from_address(ptr), dtype=np.uint16)
        e0, e = offset // 2, 0
        pos = 0
        for ra, nra, b0, nb in self._mine(part):
            for k in range(nra * nb):
                if pos + k < e0 or e >= len(buf):
                    continue
                r, c = divmod(k, nb)
                self.M[ra + r, b0 + c] = self.M[b0 + c, ra + r] = buf[e]
                e += 1
            pos += nra * nb


def _tile_exchange_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "mnhn-tree-tools_b200"))
    import oracle as O
    import swgpu
    from swgpu import split_pass
    from swgpu import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seqs, _ = W.config2(seed=5, n=150)  # the same data set in every rank
    D = O.all_pairs(seqs).astype(np.uint16)
    eng = _TileEngine(D, rank, world)
    before = int((eng.M == 0xFFFF).sum())
    rep = split_pass.exchange_tiles(eng, dist, "cpu", chunk_bytes=4000)  # many rounds, chunks cut tiles
    clusters = swgpu.dbscan_from_matrix(eng.M, 300.0, 5)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = {"exact": bool(np.array_equal(eng.M, D)), "ok": clusters == O.dbscan(D, 300.0, 5),
                 "rep": rep, "missing_before": before, "matrix_bytes": int(D.nbytes)}


@pytest.mark.parametrize("world", [2, 3])
def test_split_pass_tile_exchange_on_gloo(world):
    """The exchange sized to the result: each rank sends only its own tiles'
    rectangles (sizes checked first, payloads in chunks that cut through
    tiles); afterwards every rank holds the whole matrix, and the bytes moved
    per rank are a fraction of the matrix."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_tile_exchange_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        assert res[r]["missing_before"] > 0
        assert res[r]["exact"] and res[r]["ok"], r
        assert res[r]["rep"]["rounds"] > 1
        assert res[r]["rep"]["sent"] < 0.7 * res[r]["matrix_bytes"] / world + 4000
