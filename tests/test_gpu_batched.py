"""Batched release experiments (ReleaseBatch, opb_batched_steps, opb_sort_segments) on the GPU.

The property: every release's particles end bit-identical to running that
release alone through Simulation with the same stock ROMS stepper, whatever
else shares the launch, and whatever the launch shape, sort schedule or graph
use.  The alone runs are themselves bit-identical to the reference (the
parity tests of the fused steppers).
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import check_bundles, mismatch_report, same_bits

pytestmark = pytest.mark.gpu

NAMES = ("zidx", "yidx", "xidx", "status")


@pytest.fixture(scope="module")
def grid():
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=96, ny=80, nz=12, nt=12, seed=11, dtype="float32"))
    return g, g.oracle_fields()


def _stepper(scheme, t_arr, dt, t0):
    from offline_particles_b200.models.roms import ab3_w_advection_timestepper, rk2_w_advection_timestepper

    f = rk2_w_advection_timestepper if scheme == "rk2" else ab3_w_advection_timestepper
    return f(t_arr, np.float64(dt), time=np.float64(t0))


# (scheme, dt, release time, steps, particles): uneven sizes (one particle, a partial chunk, several
# blocks), release times on and off the snapshot grid, steps that end mid-interval
SPECS = [
    ("ab3", 120.0, 0.0, 200, 5000),
    ("rk2", 300.0, 1800.0, 60, 1),
    ("rk2", 180.0, 3600.0 * 2 + 17.25, 100, 33),
    ("ab3", 60.0, 3600.0 * 3.5, 150, 1000),
    ("rk2", 120.0, 3600.0 * 1, 170, 2500),
    ("ab3", 180.0, 3600.0 * 5 + 0.125, 80, 700),
]


def _releases(g, t_arr, specs):
    from offline_particles_b200.batching import Release

    out = []
    for q, (scheme, dt, t0, nsteps, n) in enumerate(specs):
        z, y, x = g.release(n, seed=100 + q)
        out.append(Release(_stepper(scheme, t_arr, dt, t0), nsteps, z, y, x))
    return out


def _alone(g, fields, spec, seed):
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb

    scheme, dt, t0, nsteps, n = spec
    t_arr = g.time_array[:fields["u"].shape[0]]
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    ts = _stepper(scheme, t_arr, dt, t0)
    sim = opb.SimulationBuilder(ts, fs).build_simulation(n)
    z, y, x = g.release(n, seed=seed)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10 if scheme == "ab3" else 0)
    sim.run(nsteps)
    P = sim.particles
    return {k: P[k] for k in NAMES}


@pytest.fixture(scope="module")
def alone(grid):
    g, fields = grid
    return [_alone(g, fields, spec, 100 + q) for q, spec in enumerate(SPECS)]


def _batch(grid, **kw):
    from b200_runner import b200_fieldset

    from offline_particles_b200.batching import ReleaseBatch

    g, fields = grid
    t_arr = g.time_array[:fields["u"].shape[0]]
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    rels = _releases(g, t_arr, SPECS)
    b = ReleaseBatch(fs, rels, **kw)
    b.run()
    b.synchronize()
    return b


def _check(b, alone):
    for q, r in enumerate(b.releases):
        assert r.error is None and r.done == r.nsteps, (q, r.error)
        got = b.result(r)
        for k in NAMES:
            assert same_bits(got[k], alone[q][k]), f"release {q} {k}: " + mismatch_report(got[k], alone[q][k])


@pytest.mark.parametrize("block,warps,split", [(128, 16, True), (256, 16, True), (256, 24, True), (256, 32, True),
                                               (256, 16, False), (128, 16, False)])
def test_batch_equals_each_release_alone(grid, alone, block, warps, split):
    b = _batch(grid, block=block, warps_per_sm=warps, split_schemes=split)
    assert b.graphs  # ring-streamed fields: intervals replay captured graphs
    _check(b, alone)


@pytest.mark.parametrize("sort_interval,graphs,ctas,buckets", [(0, True, 0, 256), (1, False, 0, 0),
                                                                (3, True, 7, 1), (2, True, 0, 4096)])
def test_batch_independent_of_sorting_graphs_grid_and_order(grid, alone, sort_interval, graphs, ctas, buckets):
    b = _batch(grid, sort_interval=sort_interval, graphs=graphs, ctas=ctas, buckets=buckets)
    _check(b, alone)
    if sort_interval == 1:
        assert b.sorts >= b.launches


def test_release_past_the_last_snapshot_stops_with_an_error(grid):
    from b200_runner import b200_fieldset

    from offline_particles_b200.batching import Release, ReleaseBatch

    g, fields = grid
    nt = fields["u"].shape[0]
    t_arr = g.time_array[:nt]
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    z, y, x = g.release(50, seed=5)
    long = Release(_stepper("ab3", t_arr, 300.0, 3600.0 * (nt - 3)), 1000, z, y, x)
    short = Release(_stepper("rk2", t_arr, 300.0, 0.0), 12, z, y, x)
    b = ReleaseBatch(fs, [long, short])
    b.run()
    b.synchronize()
    assert isinstance(long.error, (IndexError, ValueError)) and 0 < long.done < 1000
    assert short.error is None and short.done == 12


def test_segment_sort_keeps_segments_and_permutes_ids():
    import ctypes

    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.batching import ARENA_FIELDS
    from offline_particles_b200.kernels import _abi
    from offline_particles_b200.particles import Particles

    n = 50_000
    rng = np.random.default_rng(3)
    P = Particles(n, **ARENA_FIELDS)
    for k, hi in (("zidx", 12), ("yidx", 80), ("xidx", 96)):
        P[k].copy_(torch.from_numpy(rng.uniform(0, hi, n)))
    P["z"].copy_(torch.arange(n, dtype=torch.float64))  # a payload that must travel with its particle
    st = np.zeros(n, np.uint8)
    st[rng.integers(0, n, 500)] = 0x82
    P["status"].copy_(torch.from_numpy(st))
    ids = torch.arange(n, dtype=torch.int64, device="cuda")
    starts, counts = [100, 9000, 20000], [5000, 1, 30000]
    lib = _lib.load()
    ws = torch.empty(int(lib.opb_sort_segments_workspace_bytes(sum(counts), 3)), dtype=torch.uint8, device="cuda")
    dims = (ctypes.c_int64 * 3)(12, 80, 96)
    nb = 16
    bounds = torch.full((3, nb + 1), -1, dtype=torch.int64, device="cuda")
    _lib.call("opb_sort_segments", ctypes.byref(_abi.particles_struct(P)), ctypes.byref(dims),
              (ctypes.c_int64 * 3)(*starts), (ctypes.c_int64 * 3)(*counts), 3, ids.data_ptr(), nb,
              bounds.data_ptr(), ws.data_ptr(), ws.numel(), None)
    torch.cuda.synchronize()
    idn = ids.cpu().numpy()
    zn = P["z"].cpu().numpy()
    assert np.array_equal(zn, idn.astype(np.float64))  # payload moved with the ids
    inside = np.zeros(n, bool)
    for s, c in zip(starts, counts):
        seg = idn[s:s + c]
        assert np.array_equal(np.sort(seg), np.arange(s, s + c))  # particles stay in their segment
        inside[s:s + c] = True
        # inactive particles last in each segment
        stn = P["status"].cpu().numpy()[s:s + c]
        act = (stn & 0x80) == 0
        assert not np.any(act[np.argmax(~act):]) if (~act).any() else True
    assert np.array_equal(idn[~inside], np.flatnonzero(~inside))  # outside the segments: untouched
    # bucket bounds: ascending within each segment, first = segment start, last = the first inactive particle
    bn = bounds.cpu().numpy()
    stn = P["status"].cpu().numpy()
    for q, (s, c) in enumerate(zip(starts, counts)):
        row = bn[q]
        assert row[0] == s and np.all(np.diff(row) >= 0)
        assert row[-1] == s + int(((stn[s:s + c] & 0x80) == 0).sum())
    with pytest.raises(ValueError, match="out of order"):
        _lib.call("opb_sort_segments", ctypes.byref(_abi.particles_struct(P)), ctypes.byref(dims),
                  (ctypes.c_int64 * 2)(5000, 100), (ctypes.c_int64 * 2)(10, 10), 2, None, 0, None, ws.data_ptr(),
                  ws.numel(), None)


@pytest.mark.parametrize("scheme,dt", [("rk2", 300.0), ("ab3", 120.0)])
def test_fused_steppers_same_with_and_without_snapshot_pairs(grid, scheme, dt):
    """The fused float64 steppers read streamed fields as plain snapshots, snapshot pairs, quads (static
    x-pairs beside them) or octets (static yx-pairs), with or without the 2-D bundles (zeta with h, dx
    with dy); every layout gives the same bits."""
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200 import timesteppers

    g, fields = grid
    t_arr = g.time_array[:fields["u"].shape[0]]
    z, y, x = g.release(3000, seed=77)
    out = []
    default = timesteppers.SNAPSHOT_LAYOUT
    cases = (("never", "pairs", False), ("always", "pairs", False), ("always", "pairs", True),
             ("always", "quads", False), ("always", "quads", True), ("always", "octets", False))
    for pairs, layout, bundle in cases:
        timesteppers.SNAPSHOT_PAIRS = pairs
        timesteppers.SNAPSHOT_LAYOUT = layout
        timesteppers.BUNDLE_2D = bundle
        try:
            f = opb.roms.rk2_w_advection_timestepper if scheme == "rk2" else opb.roms.ab3_w_advection_timestepper
            sim = opb.SimulationBuilder(f(t_arr, np.float64(dt), time=np.float64(1234.5)),
                                        b200_fieldset(fields, g.hc, g.spec.nz)).build_simulation(len(z))
            sim.set_indices(z, y, x)
            sim.set_particle_field("status", 10 if scheme == "ab3" else 0)
            sim.run(90)
            P = sim.particles
            out.append({k: P[k] for k in NAMES})
        finally:
            timesteppers.SNAPSHOT_PAIRS = "auto"
            timesteppers.SNAPSHOT_LAYOUT = default
            timesteppers.BUNDLE_2D = True
    for k in NAMES:
        for j in range(1, len(cases)):
            assert same_bits(out[0][k], out[j][k]), (k, cases[j])


@pytest.mark.parametrize("layout,bundle", [("pairs", False), ("pairs", True), ("quads", False), ("quads", True),
                                           ("octets", False)])
def test_batch_same_in_every_pair_layout(grid, alone, layout, bundle):
    """The batched launch reads float32 fields as snapshot pairs, quads or octets, with or without the 2-D
    bundles; every release ends with the bits of its run alone."""
    from b200_runner import b200_fieldset

    from offline_particles_b200 import timesteppers
    from offline_particles_b200.batching import ReleaseBatch

    g, fields = grid
    t_arr = g.time_array[:fields["u"].shape[0]]
    default = timesteppers.BATCH_LAYOUT
    timesteppers.BATCH_LAYOUT = layout
    timesteppers.BUNDLE_2D = bundle
    try:
        rels = _releases(g, t_arr, SPECS)
        b = ReleaseBatch(b200_fieldset(fields, g.hc, g.spec.nz), rels, buckets=64)
        b.run()
        b.synchronize()
        got = [b.result(r) for r in rels]
    finally:
        timesteppers.BATCH_LAYOUT = default
        timesteppers.BUNDLE_2D = True
    for q, want in enumerate(alone):
        for k in NAMES:
            assert same_bits(got[q][k], want[k]), (q, k, mismatch_report(got[q][k], want[k]))


@pytest.mark.parametrize("n,offset", [(1_000_003, 0), (4096, 1), (5, 0), (1, 0)])
def test_interleave_quads_and_xpairs_match_torch(n, offset):
    import torch

    from offline_particles_b200 import _lib

    a = torch.randn(n + offset, dtype=torch.float32, device="cuda")[offset:]
    b = torch.randn(n + offset, dtype=torch.float32, device="cuda")[offset:]
    out = torch.full((4 * n,), float("nan"), dtype=torch.float32, device="cuda")
    _lib.call("opb_interleave_quads", a.data_ptr(), b.data_ptr(), out.data_ptr(), n, None)
    nxt = torch.cat((torch.arange(1, n, device="cuda"), torch.tensor([n - 1], device="cuda")))
    want = torch.stack((a, b, a[nxt], b[nxt]), dim=1)
    s = torch.randn(n + offset, dtype=torch.float64, device="cuda")[offset:]
    xp = torch.full((2 * n,), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call("opb_neighbour_pairs", s.data_ptr(), xp.data_ptr(), n, None)
    torch.cuda.synchronize()
    assert torch.equal(out.view(-1, 4), want)
    assert torch.equal(xp.view(-1, 2), torch.stack((s, s[nxt]), dim=1))
    with pytest.raises(ValueError, match="16-byte"):
        _lib.call("opb_interleave_quads", a.data_ptr(), b.data_ptr(), out.data_ptr() + 4, n, None)


@pytest.mark.parametrize("n,row,offset", [(1_000_003, 1021, 0), (4096, 64, 1), (6, 3, 0), (1, 1, 0)])
def test_interleave_octets_and_yxpairs_match_torch(n, row, offset):
    import torch

    from offline_particles_b200 import _lib

    a = torch.randn(n + offset, dtype=torch.float32, device="cuda")[offset:]
    b = torch.randn(n + offset, dtype=torch.float32, device="cuda")[offset:]
    out = torch.full((8 * n,), float("nan"), dtype=torch.float32, device="cuda")
    _lib.call("opb_interleave_octets", a.data_ptr(), b.data_ptr(), out.data_ptr(), n, row, None)
    i = torch.arange(n, device="cuda")
    idx = [torch.clamp(i + d, max=n - 1) for d in (0, 1, row, row + 1)]
    want = torch.stack([t for j in idx for t in (a[j], b[j])], dim=1)
    s = torch.randn(n + offset, dtype=torch.float64, device="cuda")[offset:]
    yx = torch.full((4 * n,), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call("opb_neighbour_quads", s.data_ptr(), yx.data_ptr(), n, row, None)
    torch.cuda.synchronize()
    assert torch.equal(out.view(-1, 8), want)
    assert torch.equal(yx.view(-1, 4), torch.stack([s[j] for j in idx], dim=1))
    with pytest.raises(ValueError, match="32-byte"):
        _lib.call("opb_interleave_octets", a.data_ptr(), b.data_ptr(), out.data_ptr() + 16, n, row, None)


@pytest.mark.parametrize("dtype,n,offset", [("float32", 1_000_003, 0), ("float32", 4096, 1), ("float64", 777_777, 0),
                                            ("float64", 10, 1)])
def test_interleave_pairs_matches_torch(dtype, n, offset):
    import torch

    from offline_particles_b200 import _lib

    td = getattr(torch, dtype)
    a = torch.randn(n + offset, dtype=torch.float64, device="cuda").to(td)[offset:]
    b = torch.randn(n + offset, dtype=torch.float64, device="cuda").to(td)[offset:]
    out = torch.full((2 * n + offset,), float("nan"), dtype=td, device="cuda")[offset:]
    _lib.call("opb_interleave_pairs", a.data_ptr(), b.data_ptr(), out.data_ptr(), n,
              _lib.F32 if dtype == "float32" else _lib.F64, None)
    torch.cuda.synchronize()
    assert torch.equal(out.view(-1, 2), torch.stack((a, b), dim=1))


def test_batch_records_trajectories_like_a_simulation(grid):
    """Rows recorded every 2 snapshot intervals equal a Simulation run alone read at the same model times."""
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200.batching import Release, ReleaseBatch

    g, fields = grid
    t_arr = g.time_array[:fields["u"].shape[0]]
    z, y, x = g.release(1500, seed=44)
    specs = [("ab3", 180.0, 0.0, 150), ("rk2", 300.0, 3600.0, 70)]
    rels = [Release(_stepper(s, t_arr, dt, t0), n, z, y, x) for s, dt, t0, n in specs]
    b = ReleaseBatch(b200_fieldset(fields, g.hc, g.spec.nz), rels, record_every=2)
    b.run()
    b.synchronize()
    for (scheme, dt, t0, nsteps), r in zip(specs, rels):
        tr = r.trajectory()
        assert len(tr["time"]) >= 2
        sim = opb.SimulationBuilder(_stepper(scheme, t_arr, dt, t0),
                                    b200_fieldset(fields, g.hc, g.spec.nz)).build_simulation(len(z))
        sim.set_indices(z, y, x)
        sim.set_particle_field("status", 10 if scheme == "ab3" else 0)
        for q, t in enumerate(tr["time"]):
            steps = int(round((t - t0) / dt)) - sim.iteration
            sim.run(steps)
            assert sim.time == t
            P = sim.particles
            for k in ("zidx", "yidx", "xidx", "status"):
                assert same_bits(tr[k][q], P[k]), (scheme, q, k)


@pytest.mark.parametrize("scheme,dt", [("rk2", 300.0), ("ab3", 120.0)])
def test_host_and_device_step_tables_give_the_same_bits(grid, scheme, dt, monkeypatch):
    """A fused launch takes its step table from host memory (in the launch's parameters) or from device
    memory; both give the same bits."""
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200 import _lib

    g, fields = grid
    t_arr = g.time_array[:fields["u"].shape[0]]
    z, y, x = g.release(2000, seed=78)
    out = []
    for inline in (_lib.INLINE_TABLE, 0):
        monkeypatch.setattr(_lib, "INLINE_TABLE", inline)
        f = opb.roms.rk2_w_advection_timestepper if scheme == "rk2" else opb.roms.ab3_w_advection_timestepper
        sim = opb.SimulationBuilder(f(t_arr, np.float64(dt), time=np.float64(600.0)),
                                    b200_fieldset(fields, g.hc, g.spec.nz)).build_simulation(len(z))
        sim.set_indices(z, y, x)
        sim.set_particle_field("status", 10 if scheme == "ab3" else 0)
        sim.run(70)
        P = sim.particles
        out.append({k: P[k] for k in NAMES})
    for k in NAMES:
        assert same_bits(out[0][k], out[1][k]), k


@pytest.mark.parametrize("n,offset", [(786_433, 0), (4096, 1), (3, 0), (1, 0)])
def test_bundles_match_torch(n, offset):
    import torch

    from offline_particles_b200 import _lib

    a = torch.randn(n + offset, dtype=torch.float32, device="cuda")[offset:]
    b = torch.randn(n + offset, dtype=torch.float32, device="cuda")[offset:]
    h = torch.randn(n + offset, dtype=torch.float64, device="cuda")[offset:]
    dy = torch.randn(n + offset, dtype=torch.float64, device="cuda")[offset:]
    zh = torch.full((4 * n,), -1, dtype=torch.int64, device="cuda")
    dd = torch.full((4 * n,), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call("opb_bundle_zeta_h", a.data_ptr(), b.data_ptr(), h.data_ptr(), zh.data_ptr(), n, None)
    _lib.call("opb_bundle_dx_dy", h.data_ptr(), dy.data_ptr(), dd.data_ptr(), n, None)
    torch.cuda.synchronize()
    check_bundles(zh.cpu().numpy(), dd.cpu().numpy(), a.cpu().numpy(), b.cpu().numpy(), h.cpu().numpy(),
                  dy.cpu().numpy())
