"""The AB3 isopycnal follower on the GPU against the reference's own run (tests/golden/iso_f32.npz).

ab3_isopycnal_following_timestepper (models/roms/__init__.py:109-141 of the
reference): AB3 with dz/dt = w_max * drho / (rho_scale + |drho|).  Bit for
bit, through the fused multi-step launches, one fused launch per step, and
the stage-by-stage kernels.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import iso_case, iso_fields, load, mismatch_report, same_bits

pytestmark = pytest.mark.gpu


def _run(mode: str, ring_size: int = 4):
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200.kernels import ParticleKernel
    from offline_particles_b200.kernels.validation import domain_bounds_kernel, finite_indices_kernel

    c = iso_case()
    gold = load("iso_f32.npz")
    g, fields = iso_fields()
    t_arr = g.time_array[:fields["u"].shape[0]]
    fs = b200_fieldset(fields, g.hc, g.spec.nz, ring_size, w_max=c["w_max"], rho_scale=c["rho_scale"])
    ts = opb.roms.ab3_isopycnal_following_timestepper(t_arr, np.float64(c["dt"]))
    if mode == "stages":
        ts._pre_step_kernel = ParticleKernel.chain(finite_indices_kernel, domain_bounds_kernel)
        assert not ts.fused()
    else:
        assert ts.fused()
    sb = opb.SimulationBuilder(ts, fs)
    ridx = gold["record_idx"]
    rec = []
    every = c["record_every"]
    if mode == "run_events":
        # the positions read by a deferrable event: recorded inside the fused launches, read after them
        def sample(state):
            P = state.particles
            rec.append(np.stack([P[n][ridx] for n in ("zidx", "yidx", "xidx")]))

        sb.add_event(opb.events.Event("sample", sample, deferrable=True), n=every, first=every)
    sim = sb.build_simulation(c["n"])
    sim.set_indices(gold["z0"], gold["y0"], gold["x0"])
    sim.set_particle_field("status", 10)
    sim.set_particle_field("rho_t", gold["rho_t0"])
    if mode == "run_events":
        sim.run(c["steps"])
    elif mode == "run":
        for _ in range(c["steps"] // every):
            sim.run(every)
            P = sim.particles
            rec.append(np.stack([P[n][ridx] for n in ("zidx", "yidx", "xidx")]))
        sim.run(c["steps"] % every)
    else:
        for k in range(c["steps"]):
            sim.step()
            if (k + 1) % every == 0:
                P = sim.particles
                rec.append(np.stack([P[n][ridx] for n in ("zidx", "yidx", "xidx")]))
    sim.synchronize()
    return gold, np.stack(rec), sim.particles


@pytest.mark.parametrize("mode,ring", [("run", 4), ("step", 4), ("stages", 4), ("run", 2), ("run_events", 4)])
def test_isopycnal_follower_matches_reference(mode, ring):
    gold, rec, P = _run(mode, ring)
    assert same_bits(rec, gold["record"]), mismatch_report(rec, gold["record"])
    for name in ("status", "zidx", "yidx", "xidx", "z", "rho_t", "_dz0", "_dz1", "_dz2", "_dxidx0", "_dxidx1",
                 "_dxidx2", "_dyidx0", "_dyidx1", "_dyidx2"):
        got = P[name]
        assert same_bits(got, gold[name]), f"{name}: {mismatch_report(got, gold[name])}"
