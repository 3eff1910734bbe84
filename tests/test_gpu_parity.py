"""GPU parity: the CUDA path against the reference's golden fixtures and the CPU oracle.

Every comparison is bit-exact (float64 arithmetic in the reference's
operation order, no FMA contraction).
"""

from __future__ import annotations

import ctypes
import json

import numpy as np
import pytest

from b200_runner import build_sim, run_b200
from helpers import (CASES, EDGE_KEYS, GOLDEN, edge_fields, edge_key, edge_particles, fingerprint, load,
                     mismatch_report, same_bits)
from offline_particles_b200.synth import GridSpec, SyntheticROMS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")


@pytest.mark.parametrize("mode", ["step", "run", "stages"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_workload_bit_exact(case, mode):
    c = CASES[case]
    gold = load(f"{case}.npz")
    grid = SyntheticROMS(c["grid"])
    fields = grid.oracle_fields()
    assert fingerprint(fields) == str(gold["fingerprint"])
    z, y, x = grid.release(c["n"])
    final, rec, _ = run_b200(fields, hc=grid.hc, nz=grid.spec.nz, scheme=c["scheme"], dt=c["dt"], steps=c["steps"],
                             z=z, y=y, x=x, mode=mode, record_every=c["record_every"], record_idx=gold["record_idx"])
    assert same_bits(rec, gold["record"]), mismatch_report(rec, gold["record"])
    for name in gold:
        if name in final:
            assert same_bits(final[name], gold[name]), f"{case}/{mode} {name}: {mismatch_report(final[name], gold[name])}"


@pytest.mark.parametrize("mode", ["step", "run", "stages"])
@pytest.mark.parametrize("dtype,scheme,nan_land", EDGE_KEYS)
def test_edge_cases_bit_exact(dtype, scheme, nan_land, mode):
    gold = load("edge_cases.npz")
    key = edge_key(dtype, scheme, nan_land)
    g, f = edge_fields(dtype, nan_land)
    z, y, x, st = edge_particles(g, 512, scheme)
    final, _, _ = run_b200(f, hc=g.hc, nz=g.spec.nz, scheme=scheme, dt=1800.0, steps=5, z=z, y=y, x=x, status=st,
                           mode=mode)
    for name, val in final.items():
        ref = gold[f"{key}__{name}"]
        assert same_bits(val, ref), f"{key} {mode} {name}: {mismatch_report(val, ref)}"


@pytest.mark.parametrize("ring_size", [2, 3, 8])
def test_ring_size_does_not_change_results(ring_size):
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    final, _, _ = run_b200(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"],
                           steps=c["steps"], z=z, y=y, x=x, mode="run", ring_size=ring_size)
    for name in ("status", "zidx", "yidx", "xidx", "z", "_dxidx1", "_dz2"):
        assert same_bits(final[name], gold[name]), f"ring {ring_size} {name}"


def test_lazy_source_streams_like_dense():
    """A lazy snapshot source (generated on the host per snapshot) gives the dense results."""
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    fields = {name: grid.field(name) for name in ("u", "v", "w", "zeta")}
    fields.update(h=grid.h, dx=grid.dx, dy=grid.dy, C=grid.C)
    z, y, x = grid.release(c["n"])
    final, _, _ = run_b200(fields, hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"], steps=c["steps"],
                           z=z, y=y, x=x, mode="run", ring_size=3)
    for name in ("status", "zidx", "yidx", "xidx"):
        assert same_bits(final[name], gold[name])


def test_zero_division_raises():
    expected = json.loads((GOLDEN / "zero_division.json").read_text())
    g = SyntheticROMS(GridSpec(nx=24, ny=20, nz=6, nt=3, seed=31, dtype="float64"))
    f = g.oracle_fields()
    f["dx"] = np.zeros_like(f["dx"])
    z, y, x = g.release(64)
    for scheme in ("rk2", "ab3"):
        assert expected[scheme][0] == "ZeroDivisionError"
        for unfused in (False, True):
            sim = build_sim(f, hc=g.hc, nz=g.spec.nz, scheme=scheme, dt=300.0, z=z, y=y, x=x, unfused=unfused)
            sim.step()
            with pytest.raises(ZeroDivisionError):
                sim.synchronize()


def test_cannot_step_onto_last_snapshot():
    g = SyntheticROMS(GridSpec(nx=16, ny=12, nz=4, nt=2, seed=3, dtype="float32"))
    z, y, x = g.release(8)
    for scheme in ("rk2", "ab3"):
        sim = build_sim(g.oracle_fields(), hc=g.hc, nz=g.spec.nz, scheme=scheme, dt=1800.0, z=z, y=y, x=x)
        sim.step()
        with pytest.raises(IndexError):
            sim.step()
        with pytest.raises((IndexError, ValueError)):
            sim.run(3)


def test_interpolation_known_answers():
    """Output kernels (trilinear / bilinear / linear) vs the reference's, static and time-blended."""
    import torch

    import offline_particles_b200 as opb
    from offline_particles_b200.fields import FieldData
    from offline_particles_b200.kernels.output import (bilinear_interpolation_kernel_function,
                                                       linear_interpolation_kernel_function,
                                                       trilinear_interpolation_kernel_function)
    from offline_particles_b200.particles import Particles

    g = load("interp_kat.npz")
    n = g["z"].size
    P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64, out=np.float64)
    P["zidx"].copy_(torch.from_numpy(g["z"]))
    P["yidx"].copy_(torch.from_numpy(g["y"]))
    P["xidx"].copy_(torch.from_numpy(g["x"]))
    dev = P["zidx"].device
    cases = [("tri", trilinear_interpolation_kernel_function, g["f3"], g["off3"], ()),
             ("bi", bilinear_interpolation_kernel_function, g["f2"], g["off2"], ("yidx", "xidx")),
             ("lin", linear_interpolation_kernel_function, g["f1"], g["off1"], ("zidx",))]
    for kind, fn, arr, off, dims in cases:
        # static
        fd = {"f": FieldData(torch.from_numpy(arr).to(dev), tuple(off))}
        fn(P, {}, fd, *dims, "f", "out")
        out = P["out"].cpu().numpy()
        assert same_bits(out, g[kind]), f"{kind} static: {mismatch_report(out, g[kind])}"
        # time-dependent with ft = 0: prev*1 + next*0 == prev for finite fields
        snaps = np.stack([arr, arr * 3.0])
        st = {3: ("center", "center", "center"), 2: ("invariant", "center", "center"),
              1: ("center", "invariant", "invariant")}[arr.ndim]
        tf = opb.TimeDependentField(snaps, *st)
        fd = {"f": FieldData(tf.get_field_data(0.0).array, tuple(off))}
        P["out"].zero_()
        fn(P, {}, fd, *dims, "f", "out")
        out = P["out"].cpu().numpy()
        assert same_bits(out, g[kind]), f"{kind} blended: {mismatch_report(out, g[kind])}"


def test_vertical_coordinate_known_answers():
    """compute_z and compute_zidx (through compute_z_kernel and ab3_post) vs the reference's."""
    import torch

    from offline_particles_b200.fields import FieldData
    from offline_particles_b200.kernels.roms import ab3_w_advection
    from offline_particles_b200.kernels.roms._roms_core import compute_z_kernel_function
    from offline_particles_b200.particles import Particles

    g = load("vertical_kat.npz")
    n = g["h"].size
    # particle k sits on knot (0, 2k) of a (2, 2n) field whose 2x2 cell around it is constant,
    # which reproduces the reference's per-particle constant 2x2 fields exactly
    h = np.repeat(g["h"], 2)[None, :].repeat(2, axis=0)
    zeta = np.repeat(g["zeta"], 2)[None, :].repeat(2, axis=0)
    P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64, z=np.float64)
    dev = P["z"].device
    P["zidx"].copy_(torch.from_numpy(g["zidx"]))
    P["xidx"].copy_(torch.from_numpy(2.0 * np.arange(n)))
    fd = {"h": FieldData(torch.from_numpy(h).to(dev), (0.0, 0.0)),
          "zeta": FieldData(torch.from_numpy(zeta).to(dev), (0.0, 0.0)),
          "C": FieldData(torch.from_numpy(g["C"]).to(dev), (0.0,))}
    sc = {"hc": float(g["hc"]), "NZ": int(g["nz"])}
    compute_z_kernel_function(P, sc, fd, "z")
    z = P["z"].cpu().numpy()
    assert same_bits(z, g["z_out"]), mismatch_report(z, g["z_out"])
    P["z"].copy_(torch.from_numpy(g["zz"]))
    ab3_w_advection.ab3_post_w_advection(P, sc, fd)
    zi = P["zidx"].cpu().numpy()
    assert same_bits(zi, g["zidx_out"]), mismatch_report(zi, g["zidx_out"])


def test_oracle_agrees_on_a_larger_float32_case():
    """Beyond the fixtures: a 200x160x24 float32 AB3 and RK2 case against the CPU oracle."""
    from oracle import oracle as O

    grid = SyntheticROMS(GridSpec(nx=200, ny=160, nz=24, nt=4, seed=77, dtype="float32"))
    fields = grid.oracle_fields()
    n = 20000
    z, y, x = grid.release(n)
    for scheme in ("ab3", "rk2"):
        orc = O.OracleROMS(grid.time_array, fields, hc=grid.hc, scheme=scheme, dt=np.float64(150.0))
        p = O.new_particles(n, scheme)
        p["zidx"][:], p["yidx"][:], p["xidx"][:] = z, y, x
        if scheme == "ab3":
            p["status"][:] = O.MULTISTEP_1
        for _ in range(60):
            orc.step(p)
        final, _, _ = run_b200(fields, hc=grid.hc, nz=grid.spec.nz, scheme=scheme, dt=150.0, steps=60, z=z, y=y,
                               x=x, mode="run")
        for name in p:
            assert same_bits(final[name], p[name]), f"{scheme} {name}: {mismatch_report(final[name], p[name])}"


def test_pinned_cyclic_source_streams_many_intervals():
    """Snapshots from pinned host tensors (synth.CyclicSnapshots: 3 distinct snapshots over 14), uploaded
    without staging through a 4-slot ring over 12 intervals with re-sorts and results read back range by
    range: bit-identical to the oracle on the same dense series."""
    from offline_particles_b200 import fields as fmod
    from oracle import oracle as O

    import offline_particles_b200 as opb
    from b200_runner import STAGGERS

    nt, dt, steps = 14, 120.0, 12 * 30
    grid = SyntheticROMS(GridSpec(nx=96, ny=80, nz=16, nt=nt, seed=23, dtype="float32"))
    src = grid.pinned_cycle(3, nt)
    assert all(v.base.is_pinned() for v in src.values())
    dense = {k: np.stack([v[i].numpy() for i in range(nt)]) for k, v in src.items()}
    statics = {"h": grid.h, "dx": grid.dx, "dy": grid.dy, "C": grid.C}
    n = 3000
    z, y, x = grid.release(n)
    kw = {k: opb.TimeDependentField(v, *STAGGERS[k], ring_size=4) for k, v in src.items()}
    kw.update({k: opb.StaticField.from_numpy(v, *STAGGERS[k]) for k, v in statics.items()})
    fs = opb.Fieldset(nt, grid.spec.nz, grid.spec.ny, grid.spec.nx, constants={"hc": grid.hc, "NZ": grid.spec.nz},
                      **kw)
    ts = opb.roms.ab3_w_advection_timestepper(grid.time_array[:nt], np.float64(dt))
    sim = opb.SimulationBuilder(ts, fs).build_simulation(n, sort_interval=40, result_ranges=2)
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10)
    out = {k: torch_empty_pinned(n, sim.device_particles[k].dtype) for k in ("zidx", "yidx", "xidx", "status")}
    sim.run(steps, results=out)
    sim.synchronize()
    assert all(isinstance(fs[k]._ring, fmod.SnapshotRing) and not fs[k]._ring.staging for k in src), \
        "pinned snapshots must be uploaded without staging buffers"
    assert sum(fs[k].h2d_bytes for k in src) >= 12 * sum(v.base[0].numel() * 4 for v in src.values())
    orc = O.OracleROMS(grid.time_array[:nt], {**dense, **statics}, hc=grid.hc, scheme="ab3", dt=np.float64(dt))
    p = O.new_particles(n, "ab3")
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = z, y, x
    p["status"][:] = O.MULTISTEP_1
    for _ in range(steps):
        orc.step(p)
    for name, got in out.items():
        assert same_bits(got.numpy(), p[name]), f"{name}: {mismatch_report(got.numpy(), p[name])}"


def torch_empty_pinned(n, dtype):
    import torch

    return torch.empty(n, dtype=dtype, pin_memory=True)


def test_c_abi_rejects_bad_arguments():
    from offline_particles_b200 import _lib

    lib = _lib.load()
    p = _lib.opb_particles()
    p.n = 10
    assert lib.opb_validation(ctypes.byref(p), None, None) == _lib.EINVAL
    assert b"NULL" in lib.opb_last_error()


@pytest.mark.parametrize("table", ["stretched", "plateaus", "nonmonotone", "hc0"])
def test_vertical_search_with_hints_matches_oracle(table):
    """compute_zidx with a level hint (ab3_post) equals the reference's binary search for any hint."""
    import torch

    from offline_particles_b200.fields import FieldData
    from offline_particles_b200.kernels.roms import ab3_w_advection
    from offline_particles_b200.particles import Particles
    from offline_particles_b200.synth import vstretching4
    from oracle import oracle as O

    rng = np.random.default_rng({"stretched": 1, "plateaus": 2, "nonmonotone": 3, "hc0": 4}[table])
    nz, hc = 24, 20.0
    C = vstretching4(nz)
    if table == "plateaus":
        C[5:9] = C[5]
        C[15:18] = C[17]
    elif table == "nonmonotone":
        C[10], C[11] = C[11], C[10]
    elif table == "hc0":
        hc = 0.0
    n = 20000
    h = np.concatenate([rng.uniform(5.0, 1000.0, n - 2000), rng.uniform(0.0, 2.0, 1000), np.full(1000, 50.0)])
    zeta = rng.uniform(-1.0, 1.0, n)
    # z: anywhere in (and a little outside) the column, plus exactly on computed level depths
    z = zeta + (zeta + h) * rng.uniform(-1.05, 0.05, n)
    lev = rng.integers(0, nz, 3000)
    sig = ((lev + 0.5) / nz) - 1.0
    S = (hc * sig + h[:3000] * C[lev]) / (hc + h[:3000])
    z[:3000] = zeta[:3000] + (zeta[:3000] + h[:3000]) * S
    # hints: exact, off by a few, far off, non-finite
    hint = rng.uniform(-2, nz + 2, n)
    hint[::7] = np.nan
    L = O.lib()
    Cf = O.make_field(C, (0.0,))
    ref = np.array([L.oracle_compute_zidx_scalar(zz, hh, ze, hc, nz, ctypes.byref(Cf)) for zz, hh, ze in zip(z, h, zeta)])
    near = ~np.isnan(hint)
    hint[near][: n // 3] = ref[near][: n // 3]
    P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64, z=np.float64)
    dev = P["z"].device
    P["zidx"].copy_(torch.from_numpy(hint))
    P["xidx"].copy_(torch.from_numpy(2.0 * np.arange(n)))
    P["z"].copy_(torch.from_numpy(z))
    hf = np.repeat(h, 2)[None, :].repeat(2, axis=0)
    zf = np.repeat(zeta, 2)[None, :].repeat(2, axis=0)
    fd = {"h": FieldData(torch.from_numpy(hf).to(dev), (0.0, 0.0)),
          "zeta": FieldData(torch.from_numpy(zf).to(dev), (0.0, 0.0)),
          "C": FieldData(torch.from_numpy(C).to(dev), (0.0,))}
    ab3_w_advection.ab3_post_w_advection(P, {"hc": hc, "NZ": nz}, fd)
    got = P["zidx"].cpu().numpy()
    assert same_bits(got, ref), mismatch_report(got, ref)
