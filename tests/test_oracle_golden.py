"""Pin the CPU oracle to the reference: oracle outputs vs the committed golden fixtures.

The fixtures were produced by running the reference's own Cython kernels
(tests/golden/make_golden.py).  Every comparison here is bit-exact.
"""

from __future__ import annotations

import ctypes
import json

import numpy as np
import pytest

from helpers import (CASES, EDGE_KEYS, GOLDEN, POSITION_FIELDS, edge_fields, edge_key, edge_particles, fingerprint,
                     load, mismatch_report, same_bits)
from oracle import oracle as O
from offline_particles_b200.synth import SyntheticROMS


def test_interpolation_known_answers():
    g = load("interp_kat.npz")
    L = O.lib()
    f3 = O.make_field(g["f3"], tuple(g["off3"]))
    f2 = O.make_field(g["f2"], tuple(g["off2"]))
    f1 = O.make_field(g["f1"], tuple(g["off1"]))
    z, y, x = g["z"], g["y"], g["x"]
    off3, off2, off1 = g["off3"], g["off2"], g["off1"]
    tri = np.array([L.oracle_trilinear(ctypes.byref(f3), zi + off3[0], yi + off3[1], xi + off3[2])
                    for zi, yi, xi in zip(z, y, x)])
    bi = np.array([L.oracle_bilinear(ctypes.byref(f2), yi + off2[0], xi + off2[1]) for yi, xi in zip(y, x)])
    lin = np.array([L.oracle_linear(ctypes.byref(f1), zi + off1[0]) for zi in z])
    assert same_bits(tri, g["tri"]), mismatch_report(tri, g["tri"])
    assert same_bits(bi, g["bi"]), mismatch_report(bi, g["bi"])
    assert same_bits(lin, g["lin"]), mismatch_report(lin, g["lin"])


def test_vertical_coordinate_known_answers():
    g = load("vertical_kat.npz")
    L = O.lib()
    C = O.make_field(g["C"], (0.0,))
    nz, hc = int(g["nz"]), float(g["hc"])
    zo = np.array([L.oracle_compute_z_scalar(zi, nz, hc, h, C_lin, ze)
                   for zi, h, ze, C_lin in zip(g["zidx"], g["h"], g["zeta"],
                                               [L.oracle_linear(ctypes.byref(C), v) for v in g["zidx"]])])
    assert same_bits(zo, g["z_out"]), mismatch_report(zo, g["z_out"])
    zi = np.array([L.oracle_compute_zidx_scalar(z, h, ze, hc, nz, ctypes.byref(C))
                   for z, h, ze in zip(g["zz"], g["h"], g["zeta"])])
    assert same_bits(zi, g["zidx_out"]), mismatch_report(zi, g["zidx_out"])


@pytest.mark.parametrize("case", sorted(CASES))
def test_workload_matches_reference(case):
    c = CASES[case]
    gold = load(f"{case}.npz")
    grid = SyntheticROMS(c["grid"])
    fields = grid.oracle_fields()
    assert fingerprint(fields) == str(gold["fingerprint"]), "synthetic inputs drifted from the fixture"
    z, y, x = grid.release(c["n"])
    assert same_bits(z, gold["z0"]) and same_bits(y, gold["y0"]) and same_bits(x, gold["x0"])
    orc = O.OracleROMS(grid.time_array, fields, hc=grid.hc, scheme=c["scheme"], dt=np.float64(c["dt"]))
    p = O.new_particles(c["n"], c["scheme"])
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = z, y, x
    if c["scheme"] == "ab3":
        p["status"][:] = O.MULTISTEP_1
    ridx = gold["record_idx"]
    rec = []
    for k in range(c["steps"]):
        orc.step(p)
        if (k + 1) % c["record_every"] == 0:
            rec.append(np.stack([p[n][ridx] for n in ("zidx", "yidx", "xidx")]))
    assert same_bits(np.stack(rec), gold["record"]), mismatch_report(np.stack(rec), gold["record"])
    for name in gold:
        if name in p:
            assert same_bits(p[name], gold[name]), f"{name}: {mismatch_report(p[name], gold[name])}"
    assert set(POSITION_FIELDS) <= set(gold)


@pytest.mark.parametrize("dtype,scheme,nan_land", EDGE_KEYS)
def test_edge_cases_match_reference(dtype, scheme, nan_land):
    gold = load("edge_cases.npz")
    key = edge_key(dtype, scheme, nan_land)
    g, f = edge_fields(dtype, nan_land)
    assert fingerprint(f) == str(gold[key + "__fingerprint"])
    z, y, x, st = edge_particles(g, 512, scheme)
    orc = O.OracleROMS(g.time_array, f, hc=g.hc, scheme=scheme, dt=np.float64(1800.0))
    p = O.new_particles(512, scheme)
    p["zidx"][:], p["yidx"][:], p["xidx"][:], p["status"][:] = z, y, x, st
    for _ in range(5):
        orc.step(p)
    for name in p:
        ref = gold[f"{key}__{name}"]
        assert same_bits(p[name], ref), f"{key} {name}: {mismatch_report(p[name], ref)}"


def test_zero_division_raises_like_reference():
    expected = json.loads((GOLDEN / "zero_division.json").read_text())
    from offline_particles_b200.synth import GridSpec

    g = SyntheticROMS(GridSpec(nx=24, ny=20, nz=6, nt=3, seed=31, dtype="float64"))
    f = g.oracle_fields()
    f["dx"] = np.zeros_like(f["dx"])
    z, y, x = g.release(64)
    for scheme in ("rk2", "ab3"):
        assert expected[scheme][0] == "ZeroDivisionError"
        orc = O.OracleROMS(g.time_array, f, hc=g.hc, scheme=scheme, dt=np.float64(300.0))
        p = O.new_particles(64, scheme)
        p["zidx"][:], p["yidx"][:], p["xidx"][:] = z, y, x
        with pytest.raises(ZeroDivisionError):
            orc.step(p)


def test_cannot_step_onto_last_snapshot():
    """timesteppers.py:81-83: landing on the final snapshot time raises IndexError."""
    c = CASES["ab3_f32"]
    from dataclasses import replace

    grid = SyntheticROMS(replace(c["grid"], nx=16, ny=12, nz=4, nt=2))
    orc = O.OracleROMS(grid.time_array, grid.oracle_fields(), hc=grid.hc, scheme="ab3", dt=np.float64(1800.0))
    p = O.new_particles(8, "ab3")
    orc.step(p)
    with pytest.raises(IndexError):
        orc.step(p)


def test_isopycnal_follower_matches_reference():
    """ab3_isopycnal_following_timestepper (models/roms/__init__.py:109-141) restated: bit for bit."""
    from helpers import iso_case, iso_fields

    c = iso_case()
    gold = load("iso_f32.npz")
    g, fields = iso_fields()
    assert fingerprint(fields) == str(gold["fingerprint"]), "synthetic inputs drifted from the fixture"
    orc = O.OracleROMS(g.time_array, fields, hc=g.hc, scheme="ab3_iso", dt=np.float64(c["dt"]), w_max=c["w_max"],
                       rho_scale=c["rho_scale"])
    p = O.new_particles(c["n"], "ab3_iso")
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = gold["z0"], gold["y0"], gold["x0"]
    p["rho_t"][:] = gold["rho_t0"]
    p["status"][:] = O.MULTISTEP_1
    ridx = gold["record_idx"]
    rec = []
    for k in range(c["steps"]):
        orc.step(p)
        if (k + 1) % c["record_every"] == 0:
            rec.append(np.stack([p[n][ridx] for n in ("zidx", "yidx", "xidx")]))
    assert same_bits(np.stack(rec), gold["record"]), mismatch_report(np.stack(rec), gold["record"])
    for name in ("status", "zidx", "yidx", "xidx", "z", "_dz0", "_dz1", "_dz2", "_dxidx1", "_dyidx2"):
        assert same_bits(p[name], gold[name]), f"{name}: {mismatch_report(p[name], gold[name])}"
