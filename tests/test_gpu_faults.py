"""Failure handling, injected on the host (no device fault, trap or hang).

A snapshot source that raises or stalls, requests cancelled while queued and
while running, and a checkpoint taken mid-run and resumed.
"""

from __future__ import annotations

import time

import numpy as np
import pytest

from helpers import same_bits

pytestmark = pytest.mark.gpu

NAMES = ("status", "zidx", "yidx", "xidx", "z")


@pytest.fixture(scope="module")
def grid():
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=6, seed=71, dtype="float32"))
    return g, g.oracle_fields()


class FaultySource:
    """An array-like snapshot source that raises (or stalls) when asked for one snapshot."""

    def __init__(self, arr: np.ndarray, bad: int, stall: float = 0.0) -> None:
        self.arr, self.bad, self.stall = arr, bad, stall
        self.shape, self.ndim, self.dtype = arr.shape, arr.ndim, arr.dtype

    def __len__(self) -> int:
        return self.shape[0]

    def __getitem__(self, k):
        if k == self.bad:
            if self.stall:
                time.sleep(self.stall)
            else:
                raise OSError(f"read error at snapshot {k}")
        return self.arr[k]


def _fieldset(g, fields, u_source, **field_kw):
    from b200_runner import STAGGERS

    import offline_particles_b200 as opb

    kw = {}
    for n in ("u", "v", "w", "zeta"):
        src = u_source if n == "u" else fields[n]
        kw[n] = opb.TimeDependentField(src, *STAGGERS[n], **field_kw)
    for n in ("h", "dx", "dy", "C"):
        kw[n] = opb.StaticField.from_numpy(fields[n], *STAGGERS[n])
    return opb.Fieldset(fields["u"].shape[0], g.spec.nz, g.spec.ny, g.spec.nx, constants={"hc": g.hc, "NZ": g.spec.nz},
                        **kw)


def _sim(g, fs, scheme="ab3", n=500, time_=None, iteration=0):
    import offline_particles_b200 as opb

    f = opb.roms.rk2_w_advection_timestepper if scheme == "rk2" else opb.roms.ab3_w_advection_timestepper
    kw = {} if time_ is None else {"time": np.float64(time_)}
    ts = f(g.time_array, np.float64(300.0), iteration=iteration, **kw)
    sim = opb.SimulationBuilder(ts, fs).build_simulation(n)
    return sim


def test_a_source_that_raises_surfaces_as_snapshot_load_error(grid):
    from offline_particles_b200.fields import SnapshotLoadError

    g, fields = grid
    fs = _fieldset(g, fields, FaultySource(fields["u"], bad=2))
    sim = _sim(g, fs)
    z, y, x = g.release(500, seed=1)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10)
    sim.run(6)  # snapshots 0, 1 only (30 min)
    with pytest.raises(SnapshotLoadError, match="OSError: read error at snapshot 2") as info:
        sim.run(24)
    assert isinstance(info.value.__cause__, OSError)


def test_a_stalled_source_times_out(grid):
    from offline_particles_b200.fields import SnapshotLoadError

    g, fields = grid
    fs = _fieldset(g, fields, FaultySource(fields["u"], bad=1, stall=3.0), load_timeout=0.5)
    sim = _sim(g, fs, n=200)
    z, y, x = g.release(200, seed=2)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10)
    t0 = time.perf_counter()
    with pytest.raises(SnapshotLoadError, match="delivered nothing"):
        sim.run(6)
    assert time.perf_counter() - t0 < 2.5
    time.sleep(3.0)  # let the stalled read finish before the fixture's arrays go away


@pytest.mark.parametrize("scheme", ["ab3", "rk2"])
def test_checkpoint_and_resume_continue_bit_for_bit(grid, tmp_path, scheme):
    import offline_particles_b200 as opb
    from b200_runner import b200_fieldset

    g, fields = grid
    z, y, x = g.release(800, seed=3)
    sim = _sim(g, b200_fieldset(fields, g.hc, g.spec.nz), scheme, n=800)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10 if scheme == "ab3" else 0)
    sim.run(20)
    sim.save_checkpoint(tmp_path / "ck.npz")
    sim.run(25)
    ref = {k: sim.particles[k] for k in NAMES}
    ck = opb.load_checkpoint(tmp_path / "ck.npz")
    assert ck.iteration == 20 and "_dz1" in ck.particles
    sim2 = _sim(g, b200_fieldset(fields, g.hc, g.spec.nz), scheme, n=800, time_=ck.time, iteration=ck.iteration)
    sim2.restore_particles(ck.particles)
    sim2.run(25)
    for k in NAMES:
        assert same_bits(sim2.particles[k], ref[k]), k


def test_cancelled_requests_leave_the_others_unchanged(grid):
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200.serving import ReleaseRequest, ReleaseServer, RequestCancelled

    g, fields = grid
    t_arr = g.time_array
    per = ReleaseServer.bytes_per_particle(4)
    server = ReleaseServer(b200_fieldset(fields, g.hc, g.spec.nz), t_arr, hbm_budget=2500 * per, max_releases=4)
    reqs = []
    for q, (scheme, hours, n) in enumerate([("ab3", 3, 900), ("rk2", 2, 700), ("ab3", 2, 800), ("rk2", 1, 600)]):
        z, y, x = g.release(n, seed=20 + q)
        reqs.append(ReleaseRequest(z, y, x, scheme, 300.0, hours * 3600.0, id=q))
    for r in reqs:
        server.submit(r)
    server.tick()  # 0, 1 and 2 run; 3 waits for room
    assert server.cancel(reqs[1]) and server.cancel(reqs[3])  # one running, one queued
    server.drain()
    assert isinstance(reqs[1].error, RequestCancelled) and isinstance(reqs[3].error, RequestCancelled)
    assert not server.cancel(reqs[0])  # already finished
    for r in (reqs[0], reqs[2]):
        assert r.error is None
        f = opb.roms.rk2_w_advection_timestepper if r.scheme == "rk2" else opb.roms.ab3_w_advection_timestepper
        sim = opb.SimulationBuilder(f(t_arr, np.float64(300.0), time=np.float64(r.start_time)),
                                    b200_fieldset(fields, g.hc, g.spec.nz)).build_simulation(len(r))
        sim.set_indices(r.zidx, r.yidx, r.xidx)
        sim.set_particle_field("status", 10 if r.scheme == "ab3" else 0)
        sim.run(r.nsteps)
        for k in ("status", "zidx", "yidx", "xidx"):
            assert same_bits(r.result[k], sim.particles[k]), (r.id, k)


def test_a_host_step_table_with_a_bad_slot_is_refused(grid, monkeypatch):
    """A fused launch's host step table is checked entry by entry: a slot outside the fields' slots is an
    argument error, and nothing is launched."""
    import offline_particles_b200 as opb
    from b200_runner import b200_fieldset

    from offline_particles_b200 import timesteppers

    g, fields = grid
    real = timesteppers._fused_fields

    def corrupt(*args, **kw):
        rf, table = real(*args, **kw)
        table[len(table) - 1].next = 7  # no field has 8 slots here
        return rf, table

    monkeypatch.setattr(timesteppers, "_fused_fields", corrupt)
    sim = _sim(g, b200_fieldset(fields, g.hc, g.spec.nz), "ab3", n=300)
    z, y, x = g.release(300, seed=5)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10)
    before = {k: sim.particles[k] for k in NAMES}
    with pytest.raises(ValueError, match="selects slots"):
        sim.run(4)
    for k in NAMES:  # the refused launch changed nothing
        assert same_bits(sim.particles[k], before[k]), k
