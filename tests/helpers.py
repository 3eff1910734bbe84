"""Shared helpers for the test suite: fixture loading, workload inputs, bit comparisons."""

from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

from offline_particles_b200.synth import GridSpec, SyntheticROMS

GOLDEN = Path(__file__).resolve().parent / "golden"

# Workloads of the committed fixtures (tests/golden/make_golden.py: CASES).
CASES = {
    "config1_rk2": dict(grid=GridSpec(nx=128, ny=96, nz=20, nt=26, seed=1, dtype="float64"),
                        n=10_000, scheme="rk2", dt=300.0, steps=288, record_every=12),
    "ab3_f32": dict(grid=GridSpec(nx=96, ny=80, nz=16, nt=6, seed=11, dtype="float32"),
                    n=4096, scheme="ab3", dt=120.0, steps=149, record_every=30),
}
POSITION_FIELDS = ("status", "zidx", "yidx", "xidx", "z")


def fingerprint(fields: dict[str, np.ndarray]) -> str:
    h = hashlib.sha256()
    for name in sorted(fields):
        a = np.ascontiguousarray(fields[name])
        h.update(name.encode())
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def load(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    """Bitwise equality, except that any NaN equals any NaN."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype.kind != "f":
        return bool(np.array_equal(a, b))
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return bool(np.array_equal(a[~na].view(np.uint64 if a.dtype.itemsize == 8 else np.uint32),
                               b[~nb].view(np.uint64 if b.dtype.itemsize == 8 else np.uint32)))


def mismatch_report(a: np.ndarray, b: np.ndarray) -> str:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if not bad.any():
        return "ok"
    i = np.flatnonzero(bad)
    d = np.abs(a[i] - b[i])
    return f"{i.size} mismatches; first at {i[:5]}: {a[i[:5]]} vs {b[i[:5]]}; max abs diff {np.nanmax(d) if d.size else 0}"


def edge_fields(dtype: str, nan_land: bool):
    """Inputs of edge_cases.npz (tests/golden/make_golden.py: edge_fields)."""
    g = SyntheticROMS(GridSpec(nx=40, ny=32, nz=10, nt=4, seed=21, dtype=dtype))
    f = g.oracle_fields()
    if nan_land:
        land = g.mask_rho == 0
        for name in ("u", "v", "w"):
            a = f[name].copy()
            if name == "u":
                a[:, :, land[:, :-1] | land[:, 1:]] = np.nan
            elif name == "v":
                a[:, :, land[:-1, :] | land[1:, :]] = np.nan
            else:
                a[:, :, land] = np.nan
            f[name] = a
        f["zeta"] = f["zeta"].copy()
        f["zeta"][2, 5, 5] = np.nan
    return g, f


def edge_particles(g, n: int, scheme: str):
    """Particles of edge_cases.npz (tests/golden/make_golden.py: edge_particles)."""
    z, y, x = g.release(n, seed=77)
    st = np.zeros(n, np.uint8) if scheme == "rk2" else np.full(n, 10, np.uint8)
    ny, nx, nz = g.spec.ny, g.spec.nx, g.spec.nz
    st[0] = 0x80
    st[1] = 0x81
    st[2] = 0x82
    z[3], y[4], x[5] = np.nan, np.inf, -np.inf
    z[6], y[7], x[8] = -0.01, ny - 0.99, nx + 3.0
    z[9], y[9], x[9] = 0.0, 0.0, 0.0
    z[10], y[10], x[10] = nz - 1.0, ny - 1.0, nx - 1.0
    z[11], y[11], x[11] = 3.0, 7.5, 11.5
    y[12], x[12] = 5.0, 5.0
    y[13], x[13] = 5.4, 4.6
    if scheme == "ab3":
        st[14] = 11
        st[15] = 0
    return z, y, x, st


EDGE_KEYS = [(d, s, nl) for d in ("float64", "float32") for s in ("rk2", "ab3") for nl in (False, True)]


def edge_key(dtype: str, scheme: str, nan_land: bool) -> str:
    return f"{dtype}_{scheme}_{'nanland' if nan_land else 'plain'}"


# The isopycnal-follower fixture (tests/golden/make_golden.py: ISO_CASE, iso_inputs).
def iso_case():
    from offline_particles_b200.synth import GridSpec

    return dict(grid=GridSpec(nx=96, ny=80, nz=16, nt=6, seed=13, dtype="float32"), n=4096, dt=120.0, steps=149,
                record_every=30, record_n=256, w_max=2.0e-3, rho_scale=0.05)


def iso_fields():
    """The case's grid and fields: the synthetic ROMS fields with the density field in place of w."""
    from offline_particles_b200.synth import SyntheticROMS

    g = SyntheticROMS(iso_case()["grid"])
    fields = g.oracle_fields()
    del fields["w"]
    fields["rho"] = g.density()
    return g, fields


def check_bundles(zh: np.ndarray, dd: np.ndarray, a: np.ndarray, b: np.ndarray, h: np.ndarray, dy: np.ndarray) -> None:
    """The zeta-with-h bundle ``zh`` (int64 words) of zeta snapshots a, b and h, and the dx-with-dy bundle
    ``dd`` of dx = h and dy: each element with its x-neighbour (the last element's is itself)."""
    n = len(a)
    j = np.minimum(np.arange(n) + 1, n - 1)
    w = zh.reshape(-1, 4)
    assert np.array_equal(np.ascontiguousarray(w[:, 0]).view(np.float64), h)
    assert np.array_equal(np.ascontiguousarray(w[:, 2]).view(np.float64), h[j])
    pair = np.ascontiguousarray(w[:, 1]).view(np.float32).reshape(-1, 2)
    nxt = np.ascontiguousarray(w[:, 3]).view(np.float32).reshape(-1, 2)
    assert np.array_equal(pair[:, 0], a) and np.array_equal(pair[:, 1], b)
    assert np.array_equal(nxt[:, 0], a[j]) and np.array_equal(nxt[:, 1], b[j])
    assert np.array_equal(dd.reshape(-1, 4), np.stack((h, dy, h[j], dy[j]), axis=1))
