"""ReleaseServer on the GPU: every served request's result equals running it alone.

Requests arrive while others run; the HBM budget admits only some at a time,
so later ones wait for earlier ones to finish and free their arena segments.
Each finished request is compared bit for bit with a Simulation that runs the
same release alone from the same start time with the stock ROMS stepper.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import mismatch_report, same_bits

pytestmark = pytest.mark.gpu

NAMES = ("zidx", "yidx", "xidx", "status")


@pytest.fixture(scope="module")
def grid():
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=96, ny=80, nz=12, nt=30, seed=21, dtype="float32"))
    return g, g.oracle_fields()


def _requests(g, specs, seed0):
    from offline_particles_b200.serving import ReleaseRequest

    out = []
    for q, (scheme, dt, hours, n) in enumerate(specs):
        z, y, x = g.release(n, seed=seed0 + q)
        out.append(ReleaseRequest(z, y, x, scheme, dt, hours * 3600.0, id=q))
    return out


def _alone(fs_factory, t_arr, req):
    import offline_particles_b200 as opb

    f = opb.roms.rk2_w_advection_timestepper if req.scheme == "rk2" else opb.roms.ab3_w_advection_timestepper
    ts = f(t_arr, np.float64(req.dt), time=np.float64(req.start_time))
    sim = opb.SimulationBuilder(ts, fs_factory()).build_simulation(len(req))
    sim.set_indices(req.zidx, req.yidx, req.xidx)
    sim.set_particle_field("status", 10 if req.scheme == "ab3" else 0)
    sim.run(req.nsteps)
    P = sim.particles
    return {k: P[k] for k in NAMES}


SPECS = [("ab3", 120.0, 3, 3000), ("rk2", 300.0, 2, 800), ("rk2", 60.0, 1.5, 1), ("ab3", 300.0, 5, 1500),
         ("rk2", 120.0, 2.5, 2500), ("ab3", 60.0, 1, 640), ("rk2", 300.0, 4, 4000), ("ab3", 120.0, 2, 77)]


def test_served_requests_equal_each_request_alone(grid):
    from b200_runner import b200_fieldset

    from offline_particles_b200.serving import ReleaseServer

    g, fields = grid
    t_arr = g.time_array[:fields["u"].shape[0]]
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    per = ReleaseServer.bytes_per_particle(4)
    server = ReleaseServer(fs, t_arr, hbm_budget=6000 * per, max_releases=4, sort_interval=2)
    reqs = _requests(g, SPECS, 500)
    for r in reqs[:5]:
        server.submit(r)
    running_max = 0
    for k in range(60):
        if k == 3:
            for r in reqs[5:]:
                server.submit(r)
        server.tick()
        running_max = max(running_max, len(server.running))
        if not server.busy:
            break
    server.drain()
    assert len(server.done) == len(reqs) and not server.rejected
    assert running_max >= 2  # requests overlapped on the device
    assert len({r.start_time for r in reqs}) >= 3  # and joined at different interval boundaries
    for r in reqs:
        assert r.error is None, r.error
        alone = _alone(lambda: b200_fieldset(fields, g.hc, g.spec.nz), t_arr, r)
        for k in NAMES:
            assert same_bits(r.result[k], alone[k]), f"request {r.id} {k}: " + mismatch_report(r.result[k], alone[k])


def test_oversized_request_is_rejected(grid):
    from b200_runner import b200_fieldset

    from offline_particles_b200.serving import ReleaseRequest, ReleaseServer

    g, fields = grid
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    per = ReleaseServer.bytes_per_particle(2)
    server = ReleaseServer(fs, g.time_array[:fields["u"].shape[0]], hbm_budget=100 * per, max_releases=2)
    z = np.ones(101)
    server.submit(ReleaseRequest(z, z, z, "rk2", 300.0, 3600.0))
    assert len(server.rejected) == 1 and not server.queue


def test_generated_snapshots_serve_like_stored_ones():
    """Snapshots generated on the device on demand (unbounded model time) give the same results in the
    server and alone, and generation is deterministic."""
    import offline_particles_b200 as opb
    from b200_runner import STAGGERS

    from offline_particles_b200.serving import ReleaseServer
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=64, ny=48, nz=8, nt=4, seed=31, dtype="float32"))
    nt = 200  # beyond the grid's own nt: the source generates any snapshot index

    def fieldset():
        src = g.device_source(nt)
        kw = {n: opb.TimeDependentField(src.field(n), *STAGGERS[n], ring_size=4) for n in ("u", "v", "w", "zeta")}
        for n, arr in (("h", g.h), ("dx", g.dx), ("dy", g.dy), ("C", g.C)):
            kw[n] = opb.StaticField.from_numpy(arr, *STAGGERS[n])
        return opb.Fieldset(nt, 8, 48, 64, constants={"hc": g.hc, "NZ": 8}, **kw)

    t_arr = np.arange(nt, dtype=np.float64) * 3600.0
    per = ReleaseServer.bytes_per_particle(4)
    server = ReleaseServer(fieldset(), t_arr, hbm_budget=3000 * per, max_releases=4)
    reqs = _requests(g, [("ab3", 120.0, 6, 1200), ("rk2", 300.0, 4, 900), ("ab3", 300.0, 3, 1500)], 900)
    for r in reqs:
        server.submit(r)
    server.drain()
    assert max(r.start_time for r in reqs) > 0  # the third waited for room
    for r in reqs:
        alone = _alone(fieldset, t_arr, r)
        for k in NAMES:
            assert same_bits(r.result[k], alone[k]), f"request {r.id} {k}: " + mismatch_report(r.result[k], alone[k])
