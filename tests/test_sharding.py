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


def _ranks_main(rank: int, world: int, port: int, out: dict, fail_rank: int) -> None:
    """One rank of a product-path job: sharding.Ranks from the launcher's environment, the release shard
    of this rank, the timed region and the gather that bench.py uses."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from offline_particles_b200.sharding import Ranks
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    ranks = Ranks(backend="gloo", timeout_s=5.0)
    try:
        assert (ranks.rank, ranks.world) == (rank, world) and ranks.device.type == "cpu"
        g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=3, seed=9, dtype="float32"))
        z, y, x = shard(g.release(1001), rank, world)
        if rank == fail_rank:
            raise RuntimeError("rank failed before its first collective")
        box = {}
        ms = ranks.timed_ms(lambda: box.update(xz=np.asarray(x) * 2.0 + np.asarray(z)))
        full = ranks.gather(box["xz"])
        count = ranks.sum(len(z))
        slow = ranks.max(float(rank))
        if rank == 0:
            out.update(full=full, count=count, slow=slow, ms=ms)
    except RuntimeError as e:
        out[f"error{rank}"] = str(e)
    finally:
        ranks.close()


def test_ranks_product_path_two_gloo_ranks():
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_ranks_main, args=(2, _free_port(), out, -1), nprocs=2, join=True)
    g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=3, seed=9, dtype="float32"))
    z, y, x = g.release(1001)
    assert np.array_equal(out["full"], x * 2.0 + z)
    assert out["count"] == 1001.0 and out["slow"] == 1.0 and out["ms"] >= 0.0


def test_ranks_failed_rank_ends_the_others_collective_with_an_error():
    """A rank that raises before the first collective leaves the job; the other rank's barrier ends with an
    error within the process group's timeout instead of waiting for ever."""
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_ranks_main, args=(2, _free_port(), out, 1), nprocs=2, join=True)
    assert "error1" in out and "first collective" in out["error1"]
    assert "error0" in out and "full" not in out
