"""Multi-GPU host logic on CPU: shards, max-over-ranks, gathering, with two gloo ranks."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from offline_particles_b200.sharding import shard, shard_bounds


def test_shard_bounds_cover_and_balance():
    for n in (0, 1, 7, 10, 4_194_304, 4_194_305):
        for world in (1, 2, 3, 8):
            parts = [shard_bounds(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out: dict) -> None:
    import torch.distributed as dist

    from offline_particles_b200.sharding import gather_shards, max_over_ranks, sum_over_ranks
    from offline_particles_b200.synth import GridSpec, SyntheticROMS
    from oracle import oracle as O

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=3, seed=9, dtype="float32"))
        z, y, x = g.release(1001)
        zs, ys, xs = shard((z, y, x), rank, world)
        orc = O.OracleROMS(g.time_array, g.oracle_fields(), hc=g.hc, scheme="ab3", dt=np.float64(300.0))
        p = O.new_particles(len(zs), "ab3")
        p["zidx"][:], p["yidx"][:], p["xidx"][:] = zs, ys, xs
        p["status"][:] = O.MULTISTEP_1
        for _ in range(12):
            orc.step(p)
        full = {k: gather_shards(p[k]) for k in ("status", "zidx", "yidx", "xidx")}
        slowest = max_over_ranks(float(rank + 1))
        total = sum_over_ranks(float(len(zs)))
        if rank == 0:
            out.update({k: v for k, v in full.items()}, slowest=slowest, total=total)
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_reassemble_the_single_process_run():
    from offline_particles_b200.synth import GridSpec, SyntheticROMS
    from oracle import oracle as O

    mgr = mp.get_context("spawn").Manager()  # no fork of a process that has threads
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    assert out["slowest"] == 2.0 and out["total"] == 1001.0
    g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=3, seed=9, dtype="float32"))
    z, y, x = g.release(1001)
    orc = O.OracleROMS(g.time_array, g.oracle_fields(), hc=g.hc, scheme="ab3", dt=np.float64(300.0))
    p = O.new_particles(1001, "ab3")
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = z, y, x
    p["status"][:] = O.MULTISTEP_1
    for _ in range(12):
        orc.step(p)
    for k in ("status", "zidx", "yidx", "xidx"):
        assert np.array_equal(out[k], p[k], equal_nan=True), k
