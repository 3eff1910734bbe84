"""GPU parity at the benchmarked sizes: the kernel variants the benchmark times, against the CPU oracle.

The small fixtures pin the arithmetic; these cases pin the code paths that
only large grids and many particles take: 32-bit indexing over 39 M-element
fields, snapshot pairs with the 2-D bundles (chosen by the library's own rule
at this particle density), Morton re-sorts inside the run, and a snapshot
boundary crossed inside a fused launch.

The GPU runs the whole release (4,194,304 particles on the 1024 x 768 x 50
grid).  Particles never interact, so the oracle (the reference's algorithm,
bit-pinned to the reference's own outputs) runs a strided subset of 65,536 of
them, and those must match bit for bit.  Snapshots are generated on the
device once and copied to the host, so both sides read the same float32
inputs.  Reference kernels restated: ``kernels/roms/ab3_w_advection.pyx:20-229``,
``kernels/roms/rk2_w_advection.pyx:31-354``.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import mismatch_report, same_bits

pytestmark = pytest.mark.gpu

N_FULL = 4_194_304
SUBSET = 64  # the oracle checks every 64th particle: 65,536 of them


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")


def _host_fields(g, nt):
    import torch

    snaps = g.device_snapshots(nt)
    torch.cuda.synchronize()
    fields = {k: v.cpu().numpy() for k, v in snaps.items()}
    del snaps
    torch.cuda.empty_cache()
    fields.update(h=g.h, dx=g.dx, dy=g.dy, C=g.C)
    return fields


@pytest.fixture(scope="module")
def headline():
    """The benchmark's grid: 1024 x 768 x 50, float32 fields, four hourly snapshots, seed 2."""
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=1024, ny=768, nz=50, nt=4, seed=2, dtype="float32"))
    return g, _host_fields(g, 4)


def _oracle(g, fields, scheme, dt, steps, z, y, x):
    from oracle import oracle as O

    orc = O.OracleROMS(g.time_array[: fields["u"].shape[0]], fields, hc=g.hc, scheme=scheme, dt=np.float64(dt))
    p = O.new_particles(z.size, scheme)
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = z, y, x
    if scheme == "ab3":
        p["status"][:] = O.MULTISTEP_1
    for _ in range(steps):
        orc.step(p)
    return p


@pytest.mark.parametrize("scheme,steps", [("ab3", 70), ("rk2", 40)])
def test_headline_size_matches_oracle(headline, scheme, steps):
    """AB3 (the benchmark's scheme) and RK2 at dt = 120 s across a snapshot boundary (30 steps per
    interval), Morton re-sorts due every 16 steps (made at the interval boundaries), the library's default
    layout decisions."""
    from b200_runner import build_sim

    from offline_particles_b200 import fields as fmod
    from offline_particles_b200 import particles as pmod
    from offline_particles_b200 import timesteppers

    g, fields = headline
    z, y, x = g.release(N_FULL, seed=1000)
    builds, sorts = [], []
    fmod.pair_observers.append(lambda: builds.append(1))
    pmod.sort_observers.append(lambda: sorts.append(1))
    try:
        sim = build_sim(fields, hc=g.hc, nz=g.spec.nz, scheme=scheme, dt=120.0, z=z, y=y, x=x, sort_interval=16)
        assert timesteppers.use_pairs(sim.launcher, timesteppers._time_dependent_fields(sim.launcher), N_FULL)
        assert timesteppers.pair_layout(sim.launcher, timesteppers._time_dependent_fields(sim.launcher)).bundles
        sim.run(steps)
        sim.synchronize()
    finally:
        fmod.pair_observers.clear()
        pmod.sort_observers.clear()
    assert sorts and len(sorts) >= 2, "the run must re-sort particle storage at least once after the first sort"
    assert builds, "the run must build snapshot pairs"
    idx = np.arange(0, N_FULL, SUBSET)
    ref = _oracle(g, fields, scheme, 120.0, steps, z[idx], y[idx], x[idx])
    P = sim.particles
    active = int(((ref["status"] & 0x80) == 0).sum())
    assert active > 0.9 * idx.size  # the comparison covers moving particles, not a frozen set
    for name in ref:
        got = np.asarray(P[name])[idx]
        assert same_bits(got, ref[name]), f"{scheme} {name}: {mismatch_report(got, ref[name])}"
    del sim


# (scheme, release time, steps, particles) on the batched workload's grid at dt = 180 s (20 steps per
# snapshot interval): uneven sizes, release times on and off the snapshot grid
BATCH_SPECS = [
    ("ab3", 0.0, 60, 60_000),
    ("rk2", 1800.0, 45, 20_000),
    ("ab3", 3600.0 * 1.5 + 17.0, 30, 5_000),
    ("rk2", 3600.0 * 2.0, 30, 100_000),
]


def test_batched_grid_releases_match_oracle():
    """Four releases of one ReleaseBatch on the 512 x 512 x 40 grid (snapshot quads with the 2-D bundles,
    Morton buckets, segment re-sorts, graph replays), each against the oracle run of that release alone."""
    from b200_runner import b200_fieldset

    from offline_particles_b200 import timesteppers
    from offline_particles_b200.batching import Release, ReleaseBatch
    from offline_particles_b200.models.roms import ab3_w_advection_timestepper, rk2_w_advection_timestepper
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    assert timesteppers.BATCH_LAYOUT == "quads" and timesteppers.BUNDLE_2D
    nt = 6
    g = SyntheticROMS(GridSpec(nx=512, ny=512, nz=40, nt=nt, seed=4, dtype="float32"))
    fields = _host_fields(g, nt)
    t_arr = g.time_array[:nt]
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    rels, inputs = [], []
    for q, (scheme, t0, nsteps, n) in enumerate(BATCH_SPECS):
        f = rk2_w_advection_timestepper if scheme == "rk2" else ab3_w_advection_timestepper
        zyx = g.release(n, seed=300 + q)
        inputs.append(zyx)
        rels.append(Release(f(t_arr, np.float64(180.0), time=np.float64(t0)), nsteps, *zyx))
    batch = ReleaseBatch(fs, rels, sort_interval=1, buckets=256)
    batch.run()
    batch.synchronize()
    assert batch.graphs and batch.sorts >= 2 and batch.launches >= 3  # re-sorts between graph replays
    from oracle import oracle as O

    for q, (r, (scheme, t0, nsteps, n)) in enumerate(zip(rels, BATCH_SPECS)):
        assert r.error is None and r.done == nsteps
        got = batch.result(r, ("zidx", "yidx", "xidx", "status", "z"))
        orc = O.OracleROMS(t_arr, fields, hc=g.hc, scheme=scheme, dt=np.float64(180.0), time=np.float64(t0))
        p = O.new_particles(n, scheme)
        p["zidx"][:], p["yidx"][:], p["xidx"][:] = inputs[q]
        if scheme == "ab3":
            p["status"][:] = O.MULTISTEP_1
        for _ in range(nsteps):
            orc.step(p)
        for name in got:
            assert same_bits(got[name], p[name]), f"release {q} {name}: {mismatch_report(got[name], p[name])}"


class _CyclicHost:
    """snapshot k of a (nt, ...) series as base[k % len(base)], for the oracle (numpy)."""

    def __init__(self, base: np.ndarray, nt: int) -> None:
        self.base = base
        self.shape = (nt,) + base.shape[1:]

    def __getitem__(self, k):
        return self.base[int(k) % self.base.shape[0]]


def test_streamed_week_matches_oracle():
    """A model week (5040 AB3 steps at dt = 120 s over 170 hourly snapshots) streamed from pinned host
    memory through 4-slot rings, re-sorted every 90 steps, snapshot pairs rebuilt every interval, results
    read back over two id ranges: every 8th particle against the oracle, bit for bit."""
    import torch
    from b200_runner import STAGGERS

    import offline_particles_b200 as opb
    from offline_particles_b200.synth import GridSpec, SyntheticROMS
    from oracle import oracle as O

    nt, dt, steps, n = 170, 120.0, 5040, 20_000
    g = SyntheticROMS(GridSpec(nx=128, ny=96, nz=20, nt=nt, seed=7, dtype="float32"))
    src = g.pinned_cycle(8, nt)
    statics = {"h": g.h, "dx": g.dx, "dy": g.dy, "C": g.C}
    kw = {k: opb.TimeDependentField(v, *STAGGERS[k], ring_size=4) for k, v in src.items()}
    kw.update({k: opb.StaticField.from_numpy(v, *STAGGERS[k]) for k, v in statics.items()})
    fs = opb.Fieldset(nt, g.spec.nz, g.spec.ny, g.spec.nx, constants={"hc": g.hc, "NZ": g.spec.nz}, **kw)
    ts = opb.roms.ab3_w_advection_timestepper(g.time_array[:nt], np.float64(dt))
    sim = opb.SimulationBuilder(ts, fs).build_simulation(n, result_ranges=2)
    z, y, x = g.release(n, seed=77)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10)
    out = {k: torch.empty(n, dtype=sim.device_particles[k].dtype, pin_memory=True)
           for k in ("zidx", "yidx", "xidx", "status", "z")}
    sim.run(steps, results=out)
    sim.synchronize()
    idx = np.arange(0, n, 8)
    fields = {k: _CyclicHost(v.base.numpy(), nt) for k, v in src.items()}
    fields.update(statics)
    orc = O.OracleROMS(g.time_array[:nt], fields, hc=g.hc, scheme="ab3", dt=np.float64(dt))
    p = O.new_particles(idx.size, "ab3")
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = z[idx], y[idx], x[idx]
    p["status"][:] = O.MULTISTEP_1
    for _ in range(steps):
        orc.step(p)
    # most particles leave the 256 x 192 km domain within the week; every one moved, and about a fifth
    # are still moving at the end
    assert int(((p["status"] & 0x80) == 0).sum()) > idx.size // 10
    assert np.mean(p["xidx"] != x[idx]) > 0.99
    for name, got in out.items():
        got = got.numpy()[idx]
        assert same_bits(got, p[name]), f"{name}: {mismatch_report(got, p[name])}"


def test_end_to_end_path_at_size_matches_oracle(headline):
    """The end-to-end configuration the benchmark times: the 4,194,304-particle release from pinned host
    arrays, every snapshot uploaded from pinned host tensors through 8-slot rings, 20 AB3 steps, the results
    read back in original order over two id ranges (the last launch split): every 64th particle against the
    oracle, bit for bit."""
    import torch
    from b200_runner import STAGGERS

    import offline_particles_b200 as opb

    g, fields = headline
    nt = fields["u"].shape[0]
    kw = {k: opb.TimeDependentField(torch.from_numpy(fields[k]).pin_memory(), *STAGGERS[k], ring_size=8)
          for k in ("u", "v", "w", "zeta")}
    kw.update({k: opb.StaticField.from_numpy(fields[k], *STAGGERS[k]) for k in ("h", "dx", "dy", "C")})
    fs = opb.Fieldset(nt, g.spec.nz, g.spec.ny, g.spec.nx, constants={"hc": g.hc, "NZ": g.spec.nz}, **kw)
    ts = opb.roms.ab3_w_advection_timestepper(g.time_array[:nt], np.float64(120.0))
    sim = opb.SimulationBuilder(ts, fs).build_simulation(N_FULL, result_ranges=2)
    z, y, x = g.release(N_FULL, seed=1000)
    hz, hy, hx = (torch.from_numpy(v).pin_memory() for v in (z, y, x))
    names = ("zidx", "yidx", "xidx", "status", "z")
    out = {k: torch.empty(N_FULL, dtype=sim.device_particles[k].dtype, pin_memory=True) for k in names}
    sim.reserve_results(out)
    sim.set_indices(hz, hy, hx)
    sim.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
    sim.run(20, results=out)
    sim.synchronize()
    idx = np.arange(0, N_FULL, SUBSET)
    ref = _oracle(g, fields, "ab3", 120.0, 20, z[idx], y[idx], x[idx])
    for name in names:
        got = out[name].numpy()[idx]
        assert same_bits(got, ref[name]), f"{name}: {mismatch_report(got, ref[name])}"
