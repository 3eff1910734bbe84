"""Run the B200 implementation through its public API the way make_golden.py runs the reference."""

from __future__ import annotations

import numpy as np

STAGGERS = {
    "u": ("center", "center", "inner"),
    "v": ("center", "inner", "center"),
    "w": ("outer", "center", "center"),
    "zeta": ("invariant", "center", "center"),
    "h": ("invariant", "center", "center"),
    "dx": ("invariant", "center", "center"),
    "dy": ("invariant", "center", "center"),
    "C": ("center", "invariant", "invariant"),
    "rho": ("center", "center", "center"),
}


def b200_fieldset(fields: dict, hc: float, nz: int, ring_size: int = 4, storage: str | None = None,
                  **constants):
    import offline_particles_b200 as opb

    nt, _, ny, nxu = fields["u"].shape
    kw = {}
    for name, arr in fields.items():
        st = STAGGERS[name]
        if name in ("u", "v", "w", "zeta", "rho"):
            kw[name] = opb.TimeDependentField.from_numpy(arr, *st, ring_size=ring_size, storage=storage)
        else:
            kw[name] = opb.StaticField.from_numpy(arr, *st)
    return opb.Fieldset(nt, nz, ny, nxu + 1, constants={"hc": hc, "NZ": nz, **constants}, **kw)


def build_sim(fields, *, hc, nz, scheme, dt, z, y, x, status=None, unfused=False, ring_size=4, time=None,
              sort_interval=None, arithmetic="float64", storage=None, result_ranges=1):
    import offline_particles_b200 as opb
    from offline_particles_b200.kernels import ParticleKernel
    from offline_particles_b200.kernels.validation import domain_bounds_kernel, finite_indices_kernel
    from offline_particles_b200.models.roms import ab3_w_advection_timestepper, rk2_w_advection_timestepper

    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    fs = b200_fieldset(fields, hc, nz, ring_size, storage)
    factory = rk2_w_advection_timestepper if scheme == "rk2" else ab3_w_advection_timestepper
    kw = {} if time is None else {"time": np.float64(time)}
    ts = factory(t_arr, np.float64(dt), **kw)
    if unfused:
        # an equivalent but distinct pre-step kernel object: the stepper then launches stage by stage
        ts._pre_step_kernel = ParticleKernel.chain(finite_indices_kernel, domain_bounds_kernel)
        assert not ts.fused()
    else:
        assert ts.fused()
    kw = {} if sort_interval is None else {"sort_interval": sort_interval}
    sim = opb.SimulationBuilder(ts, fs).build_simulation(len(z), arithmetic=arithmetic, result_ranges=result_ranges,
                                                         **kw)
    sim.set_indices(z, y, x)
    if status is not None:
        sim.set_particle_field("status", status)
    elif scheme == "ab3":
        sim.set_particle_field("status", 10)
    return sim


def run_b200(fields, *, hc, nz, scheme, dt, steps, z, y, x, status=None, mode="step", record_every=0,
             record_idx=None, ring_size=4, sort_interval=None, arithmetic="float64", storage=None):
    """mode: 'step' (one fused launch per step), 'run' (multi-step launches) or 'stages' (stage kernels)."""
    sim = build_sim(fields, hc=hc, nz=nz, scheme=scheme, dt=dt, z=z, y=y, x=x, status=status,
                    unfused=(mode == "stages"), ring_size=ring_size, sort_interval=sort_interval,
                    arithmetic=arithmetic, storage=storage)
    rec = []
    if mode == "run" and record_every:
        for _ in range(steps // record_every):
            sim.run(record_every)
            P = sim.particles
            rec.append(np.stack([P[n][record_idx] for n in ("zidx", "yidx", "xidx")]))
        sim.run(steps % record_every)
    elif mode == "run":
        sim.run(steps)
    else:
        for k in range(steps):
            sim.step()
            if record_every and (k + 1) % record_every == 0:
                P = sim.particles
                rec.append(np.stack([P[n][record_idx] for n in ("zidx", "yidx", "xidx")]))
    sim.synchronize()
    P = sim.particles
    final = {name: np.array(P[name]) for name in P.arrays}
    return final, (np.stack(rec) if rec else None), sim
