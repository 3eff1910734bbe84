"""Generate the golden fixtures in this folder by running the reference itself.

Run in a checkout that has the reference (``offline_particles``) next to it:
``python tests/golden/make_golden.py``.  The reference's Cython kernels are
compiled into ``oracle/_ref`` by ``oracle/build_ref.py`` and imported through
``oracle/ref_import.py``; the reference cannot travel, so its outputs are kept
here as small ``.npz`` files.  Inputs are regenerated by the tests from the
seeded synthetic grid (``offline_particles_b200.synth``) and checked against the
SHA-256 fingerprints stored with each fixture.

Fixtures
--------
interp_kat.npz     reference linear / bilinear / trilinear interpolation
                   (kernels/_interpolation/linear.pxd via the reference's output
                   kernels, kernels/output/linear_interpolation.pyx) at in-range,
                   extrapolated, clamped and non-finite positions.
vertical_kat.npz   reference compute_z / compute_zidx (kernels/roms/
                   _vertical_coordinate.pxd via _roms_core.pyx and
                   ab3_post_w_advection) over deep, shallow, above-surface,
                   below-bottom and non-finite cases.
config1_rk2.npz    the full small workload: 128x96x20 float64 grid, 26 hourly
                   snapshots, 10,000 particles, RK2 dt=300 s, 288 steps.
ab3_f32.npz        AB3 on a 96x80x16 float32 grid, 6 snapshots, 4096 particles,
                   dt=120 s, 149 steps (crosses snapshot boundaries; a 150th
                   step would land on the last snapshot, which the reference
                   rejects with IndexError).
edge_cases.npz     NaN land, inactive / out-of-domain / non-finite particles,
                   steps that land exactly on snapshot times, RK2 and AB3.
zero_division.json the reference's error for a zero grid spacing.
outputs.npz        rows of the reference's output events: linearly_interpolate_fields
                   (h, u, zeta, w) every 1800 s of an RK2 run, time and values.
outputs_mixed.npz  the same run with a second writer (v, zeta) every 7 iterations from
                   iteration 3: both writers' rows.  Output kernels skip inactive
                   particles and every output of one dtype shares a particle field, so
                   an inactive particle's row holds the value the previous output left
                   there; the second writer changes those values in the first's rows.
iso_f32.npz        the AB3 isopycnal follower (ab3_isopycnal_following.pyx) on a
                   96x80x16 float32 grid with a synthetic density field,
                   4096 particles with target densities, dt=120 s, 149 steps.
"""

from __future__ import annotations

import hashlib
import json
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from offline_particles_b200.synth import GridSpec, SyntheticROMS  # noqa: E402
from oracle.ref_import import import_reference  # noqa: E402

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

# the isopycnal follower (models/roms/__init__.py:109-141): AB3 with dz from density
ISO_CASE = dict(grid=GridSpec(nx=96, ny=80, nz=16, nt=6, seed=13, dtype="float32"), n=4096, dt=120.0, steps=149,
                record_every=30, record_n=256, w_max=2.0e-3, rho_scale=0.05)

CASES = {
    "config1_rk2": dict(grid=GridSpec(nx=128, ny=96, nz=20, nt=26, seed=1, dtype="float64"),
                        n=10_000, scheme="rk2", dt=300.0, steps=288, record_every=12, record_n=256,
                        keep=("status", "zidx", "yidx", "xidx", "z")),
    "ab3_f32": dict(grid=GridSpec(nx=96, ny=80, nz=16, nt=6, seed=11, dtype="float32"),
                    n=4096, scheme="ab3", dt=120.0, steps=149, record_every=30, record_n=256),
}


def fingerprint(fields: dict[str, np.ndarray]) -> str:
    h = hashlib.sha256()
    for name in sorted(fields):
        a = np.ascontiguousarray(fields[name])
        h.update(name.encode())
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def ref_fieldset(op, fields: dict[str, np.ndarray], hc: float, nz: int, **constants):
    nt, _, ny, nxu = fields["u"].shape
    kw = {}
    for name, arr in fields.items():
        st = STAGGERS[name]
        if name in ("u", "v", "w", "zeta", "rho"):
            kw[name] = op.TimeDependentField.from_numpy(arr, *st)
        else:
            kw[name] = op.StaticField.from_numpy(arr, *st)
    return op.Fieldset(nt, nz, ny, nxu + 1, constants={"hc": hc, "NZ": nz, **constants}, **kw)


def iso_inputs(c):
    """Fields (rho in place of w), release and target densities of the isopycnal case."""
    g = SyntheticROMS(c["grid"])
    fields = g.oracle_fields()
    del fields["w"]
    fields["rho"] = g.density()
    z, y, x = g.release(c["n"])
    rng = np.random.default_rng(17)
    rho_t = 1026.5 - 1.5 * rng.uniform(0.0, 1.0, c["n"])
    return g, fields, z, y, x, rho_t


def make_isopycnal(op) -> None:
    from offline_particles.models.roms import ab3_isopycnal_following_timestepper

    c = ISO_CASE
    g, fields, z, y, x, rho_t = iso_inputs(c)
    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    fs = ref_fieldset(op, fields, g.hc, g.spec.nz, w_max=c["w_max"], rho_scale=c["rho_scale"])
    ts = ab3_isopycnal_following_timestepper(t_arr, np.float64(c["dt"]))
    sim = op.SimulationBuilder(ts, fs).build_simulation(len(z))
    sim.set_indices(z, y, x)
    sim.set_particle_field("status", 10)
    sim.set_particle_field("rho_t", rho_t)
    ridx = np.sort(np.random.default_rng(5).choice(c["n"], c["record_n"], replace=False))
    rec = []
    for k in range(c["steps"]):
        sim.step()
        if (k + 1) % c["record_every"] == 0:
            P = sim.particles
            rec.append(np.stack([np.asarray(P[n])[ridx] for n in ("zidx", "yidx", "xidx")]))
    P = sim.particles
    final = {name: np.array(P[name]) for name in P.arrays}
    np.savez_compressed(HERE / "iso_f32.npz", fingerprint=fingerprint(fields), z0=z, y0=y, x0=x, rho_t0=rho_t,
                        record_idx=ridx, record=np.stack(rec), **final)
    print("iso_f32 status", np.unique(final["status"], return_counts=True))


def run_reference(op, fields, *, hc, nz, scheme, dt, steps, z, y, x, status=None, record_every=0, record_idx=None,
                  time=None):
    from offline_particles.models.roms import ab3_w_advection_timestepper, rk2_w_advection_timestepper

    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    fs = ref_fieldset(op, fields, hc, nz)
    factory = rk2_w_advection_timestepper if scheme == "rk2" else ab3_w_advection_timestepper
    kw = {} if time is None else {"time": np.float64(time)}
    ts = factory(t_arr, np.float64(dt), **kw)
    sim = op.SimulationBuilder(ts, fs).build_simulation(len(z))
    sim.set_indices(z, y, x)
    if status is not None:
        sim.set_particle_field("status", status)
    elif scheme == "ab3":
        sim.set_particle_field("status", 10)
    rec = []
    for k in range(steps):
        sim.step()
        if record_every and (k + 1) % record_every == 0:
            P = sim.particles
            rec.append(np.stack([np.asarray(P[n])[record_idx] for n in ("zidx", "yidx", "xidx")]))
    P = sim.particles
    final = {name: np.array(P[name]) for name in P.arrays}
    return final, (np.stack(rec) if rec else None)


def make_interp_kat(op) -> None:
    from offline_particles.fields import FieldData
    from offline_particles.kernels.output import linear_interpolation as li

    rng = np.random.default_rng(1234)
    f3 = rng.standard_normal((5, 6, 7))
    f2 = rng.standard_normal((6, 7))
    f1 = rng.standard_normal(9)
    n = 4000
    z = rng.uniform(-2.0, 7.0, n)
    y = rng.uniform(-2.0, 8.0, n)
    x = rng.uniform(-2.0, 9.0, n)
    # exact knots, faces, far out, negative zero and non-finite values
    special = np.array([0.0, -0.0, 1.0, 3.0, 4.0, 4.5, 5.0, 5.999999999999, 6.0, -0.5, -1e-300, 1e300, -1e300,
                        np.inf, -np.inf, np.nan, 2.0**63, -(2.0**63), 9.3e18, 1e-17])
    m = special.size
    z[:m], y[:m], x[:m] = special, special[::-1], np.roll(special, 3)
    off3 = (0.5, 0.0, -0.5)
    off2 = (0.0, -0.5)
    off1 = (0.5,)
    out = {}
    for kind, fn, fd, names in (
        ("tri", li.trilinear_interpolation_kernel_function, FieldData(f3, off3), ()),
        ("bi", li.bilinear_interpolation_kernel_function, FieldData(f2, off2), ("yidx", "xidx")),
        ("lin", li.linear_interpolation_kernel_function, FieldData(f1, off1), ("zidx",)),
    ):
        parts = types.SimpleNamespace(status=np.zeros(n, np.uint8), zidx=z.copy(), yidx=y.copy(), xidx=x.copy(),
                                      out=np.zeros(n))
        parts.__getitem__ = None
        P = _Particles(parts)
        if kind == "tri":
            fn(P, {}, {"f": fd}, "f", "out")
        elif kind == "bi":
            fn(P, {}, {"f": fd}, "yidx", "xidx", "f", "out")
        else:
            fn(P, {}, {"f": fd}, "zidx", "f", "out")
        out[kind] = parts.out.copy()
    np.savez_compressed(HERE / "interp_kat.npz", f3=f3, f2=f2, f1=f1, z=z, y=y, x=x, off3=off3, off2=off2, off1=off1,
                        tri=out["tri"], bi=out["bi"], lin=out["lin"])


class _Particles:
    """Minimal particles mapping for calling reference kernel functions directly."""

    def __init__(self, ns) -> None:
        self._ns = ns

    def __getattr__(self, name):
        return getattr(self._ns, name)

    def __getitem__(self, name):
        return getattr(self._ns, name)


def make_vertical_kat(op) -> None:
    from offline_particles.fields import FieldData
    from offline_particles.kernels.roms import _roms_core, ab3_w_advection

    rng = np.random.default_rng(99)
    nz = 30
    hc = 20.0
    from offline_particles_b200.synth import vstretching4

    C = vstretching4(nz)
    n = 6000
    h = np.concatenate([rng.uniform(5.0, 1000.0, n - 200), np.full(100, 50.0), rng.uniform(0.5, 3.0, 100)])
    zeta = rng.uniform(-1.0, 1.0, n)
    zidx = rng.uniform(-1.0, nz, n)
    zidx[:8] = [0.0, nz - 1.0, -0.5, nz - 0.5, np.nan, np.inf, -3.0, nz + 2.0]
    # z for the inverse: interior, above the surface, below the bottom, non-finite
    zz = zeta + (zeta + h) * rng.uniform(-1.1, 0.1, n)
    zz[:6] = [np.nan, np.inf, -np.inf, 0.0, 5.0, -2000.0]
    # zeta == -h gives a zero divisor in _S_from_z (-> 0.0 in the reference)
    zeta[10] = -h[10]
    res_z = np.empty(n)
    res_zidx = np.empty(n)
    for i0 in range(0, n, 1000):
        sl = slice(i0, i0 + 1000)
        m = sl.stop - sl.start
        # constant-per-particle h/zeta: evaluate one particle per call on 2x2 constant fields
        for j in range(m):
            k = i0 + j
            hf = FieldData(np.full((2, 2), h[k]), (0.0, 0.0))
            zf = FieldData(np.full((2, 2), zeta[k]), (0.0, 0.0))
            cf = FieldData(C, (0.0,))
            ns = types.SimpleNamespace(status=np.zeros(1, np.uint8), zidx=np.array([zidx[k]]), yidx=np.zeros(1),
                                       xidx=np.zeros(1), z=np.zeros(1))
            P = _Particles(ns)
            sc = {"hc": hc, "NZ": nz}
            _roms_core.compute_z_kernel_function(P, sc, {"h": hf, "zeta": zf, "C": cf}, "z")
            res_z[k] = ns.z[0]
            ns.z[0] = zz[k]
            ab3_w_advection.ab3_post_w_advection(P, sc, {"h": hf, "zeta": zf, "C": cf})
            res_zidx[k] = ns.zidx[0]
    np.savez_compressed(HERE / "vertical_kat.npz", C=C, hc=hc, nz=nz, h=h, zeta=zeta, zidx=zidx, zz=zz,
                        z_out=res_z, zidx_out=res_zidx)


def make_workloads(op) -> None:
    for name, c in CASES.items():
        g = SyntheticROMS(c["grid"])
        fields = g.oracle_fields()
        z, y, x = g.release(c["n"])
        rng = np.random.default_rng(5)
        ridx = np.sort(rng.choice(c["n"], c["record_n"], replace=False))
        final, rec = run_reference(op, fields, hc=g.hc, nz=g.spec.nz, scheme=c["scheme"], dt=c["dt"],
                                   steps=c["steps"], z=z, y=y, x=x, record_every=c["record_every"], record_idx=ridx)
        if c.get("keep") is not None:
            final = {k: v for k, v in final.items() if k in c["keep"]}
        np.savez_compressed(HERE / f"{name}.npz", fingerprint=fingerprint(fields), z0=z, y0=y, x0=x,
                            record_idx=ridx, record=rec, **final)
        print(name, "status", np.unique(final["status"], return_counts=True))


def edge_fields(dtype: str, nan_land: bool):
    g = SyntheticROMS(GridSpec(nx=40, ny=32, nz=10, nt=4, seed=21, dtype=dtype))
    f = g.oracle_fields()
    if nan_land:
        land = g.mask_rho == 0
        for name in ("u", "v", "w"):
            a = f[name].copy()
            if name == "u":
                m = land[:, :-1] | land[:, 1:]
                a[:, :, m] = np.nan
            elif name == "v":
                m = land[:-1, :] | land[1:, :]
                a[:, :, m] = np.nan
            else:
                a[:, :, land] = np.nan
            f[name] = a
        # NaN in the *next* snapshot only: exercised at frac = 0 (0 * NaN = NaN)
        f["zeta"] = f["zeta"].copy()
        f["zeta"][2, 5, 5] = np.nan
    return g, f


def edge_particles(g, n: int, scheme: str):
    z, y, x = g.release(n, seed=77)
    st = np.zeros(n, np.uint8) if scheme == "rk2" else np.full(n, 10, np.uint8)
    ny, nx, nz = g.spec.ny, g.spec.nx, g.spec.nz
    # inactive, already-flagged, non-finite, out of bounds, on faces, on bounds
    st[0] = 0x80
    st[1] = 0x81
    st[2] = 0x82
    z[3], y[4], x[5] = np.nan, np.inf, -np.inf
    z[6], y[7], x[8] = -0.01, ny - 0.99, nx + 3.0
    z[9], y[9], x[9] = 0.0, 0.0, 0.0
    z[10], y[10], x[10] = nz - 1.0, ny - 1.0, nx - 1.0
    z[11], y[11], x[11] = 3.0, 7.5, 11.5  # on faces
    y[12], x[12] = 5.0, 5.0  # the NaN zeta cell
    y[13], x[13] = 5.4, 4.6
    if scheme == "ab3":
        st[14] = 11
        st[15] = 0
    return z, y, x, st


def make_edge_cases(op) -> None:
    out = {}
    for dtype in ("float64", "float32"):
        for scheme in ("rk2", "ab3"):
            for nan_land in (False, True):
                g, f = edge_fields(dtype, nan_land)
                z, y, x, st = edge_particles(g, 512, scheme)
                # dt = 1800 s: steps land exactly on snapshot times
                final, _ = run_reference(op, f, hc=g.hc, nz=g.spec.nz, scheme=scheme, dt=1800.0, steps=5, z=z, y=y,
                                         x=x, status=st)
                key = f"{dtype}_{scheme}_{'nanland' if nan_land else 'plain'}"
                out[key + "__fingerprint"] = np.array(fingerprint(f))
                for k, v in final.items():
                    out[f"{key}__{k}"] = v
    np.savez_compressed(HERE / "edge_cases.npz", **out)


def make_zero_division(op) -> None:
    g = SyntheticROMS(GridSpec(nx=24, ny=20, nz=6, nt=3, seed=31, dtype="float64"))
    f = g.oracle_fields()
    f["dx"] = f["dx"].copy()
    f["dx"][:] = 0.0
    z, y, x = g.release(64)
    result = {}
    for scheme in ("rk2", "ab3"):
        try:
            run_reference(op, f, hc=g.hc, nz=g.spec.nz, scheme=scheme, dt=300.0, steps=1, z=z, y=y, x=x)
            result[scheme] = None
        except Exception as e:  # the reference's own error type and message
            result[scheme] = [type(e).__name__, str(e)]
    (HERE / "zero_division.json").write_text(json.dumps(result, indent=1) + "\n")


OUTPUT_CASE = dict(grid=GridSpec(nx=48, ny=40, nz=8, nt=4, seed=41, dtype="float32"), n=512, dt=300.0, steps=24,
                   every=1800.0, variables=("h", "u", "zeta", "w"))


def _memory_writer_classes():
    from offline_particles.output import AbstractOutputWriter, AbstractOutputWriterBuilder

    class MemoryWriter(AbstractOutputWriter):
        def __init__(self, name, outputs):
            self._name = name
            self._outputs = outputs
            self.times, self.rows = [], {k: [] for k in outputs}

        name = property(lambda self: self._name)
        outputs = property(lambda self: self._outputs)

        def write_time(self, state):
            self.times.append(state.time)

        def write_output(self, name, state):
            self.rows[name].append(np.array(state.particles[self._outputs[name].particle_field]))

        def finalise_write_round(self, state):
            pass

    class MemoryBuilder(AbstractOutputWriterBuilder):
        def __init__(self, name):
            self._name = name
            self._outputs = {}
            self.writer = None

        name = property(lambda self: self._name)
        outputs = property(lambda self: self._outputs)

        def add_output(self, *outputs, **kwargs):
            for o in outputs:
                self._outputs[o.name] = o

        def remove_output(self, name):
            del self._outputs[name]

        def build(self, nparticles, time_type=np.dtype(np.float64)):
            self.writer = MemoryWriter(self._name, dict(self._outputs))
            return self.writer

    return MemoryBuilder


def make_outputs_mixed(op) -> None:
    """OUTPUT_CASE with a second writer of (v, zeta) every 7 iterations from iteration 3: the rows of
    both writers when an iteration schedule and a time schedule share one simulation."""
    from offline_particles.models.roms import rk2_w_advection_timestepper
    from offline_particles.output import linearly_interpolate_fields

    MemoryBuilder = _memory_writer_classes()
    c = OUTPUT_CASE
    g = SyntheticROMS(c["grid"])
    fields = g.oracle_fields()
    fs = ref_fieldset(op, fields, g.hc, g.spec.nz)
    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    sb = op.SimulationBuilder(rk2_w_advection_timestepper(t_arr, np.float64(c["dt"])), fs)
    by_time = MemoryBuilder("by_time")
    by_time.add_output(*linearly_interpolate_fields(fs, *c["variables"]))
    sb.add_output_writer(by_time, dt=np.float64(c["every"]))
    by_iter = MemoryBuilder("by_iter")
    by_iter.add_output(*linearly_interpolate_fields(fs, "v", "zeta"))
    sb.add_output_writer(by_iter, n=7, first=3)
    z, y, x = g.release(c["n"], seed=3)
    sim = sb.build_simulation(c["n"])
    sim.set_indices(z, y, x)
    for _ in range(c["steps"]):
        sim.step()
    rows = {f"t_{k}": np.stack(v) for k, v in by_time.writer.rows.items()}
    rows.update({f"i_{k}": np.stack(v) for k, v in by_iter.writer.rows.items()})
    np.savez_compressed(HERE / "outputs_mixed.npz", fingerprint=fingerprint(fields), z0=z, y0=y, x0=x,
                        t_time=np.array(by_time.writer.times), i_time=np.array(by_iter.writer.times), **rows)
    print("outputs_mixed rows", {k: v.shape for k, v in rows.items()})


def make_outputs(op) -> None:
    """Rows the reference's output events produce: linearly_interpolate_fields outputs written every
    `every` seconds by an in-memory writer on the reference's own AbstractOutputWriter interface (the
    reference's zarr writer needs zarr, which is absent)."""
    from offline_particles.models.roms import rk2_w_advection_timestepper
    from offline_particles.output import AbstractOutputWriter, AbstractOutputWriterBuilder, linearly_interpolate_fields

    class MemoryWriter(AbstractOutputWriter):
        def __init__(self, outputs):
            self._outputs = outputs
            self.times, self.rows = [], {k: [] for k in outputs}

        name = "mem"
        outputs = property(lambda self: self._outputs)

        def write_time(self, state):
            self.times.append(state.time)

        def write_output(self, name, state):
            self.rows[name].append(np.array(state.particles[self._outputs[name].particle_field]))

        def finalise_write_round(self, state):
            pass

    class MemoryBuilder(AbstractOutputWriterBuilder):
        name = "mem"

        def __init__(self):
            self._outputs = {}
            self.writer = None

        outputs = property(lambda self: self._outputs)

        def add_output(self, *outputs, **kwargs):
            for o in outputs:
                self._outputs[o.name] = o

        def remove_output(self, name):
            del self._outputs[name]

        def build(self, nparticles, time_type=np.dtype(np.float64)):
            self.writer = MemoryWriter(dict(self._outputs))
            return self.writer

    c = OUTPUT_CASE
    g = SyntheticROMS(c["grid"])
    fields = g.oracle_fields()
    fs = ref_fieldset(op, fields, g.hc, g.spec.nz)
    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    sb = op.SimulationBuilder(rk2_w_advection_timestepper(t_arr, np.float64(c["dt"])), fs)
    mb = MemoryBuilder()
    mb.add_output(*linearly_interpolate_fields(fs, *c["variables"]))
    sb.add_output_writer(mb, dt=np.float64(c["every"]))
    z, y, x = g.release(c["n"], seed=3)
    sim = sb.build_simulation(c["n"])
    sim.set_indices(z, y, x)
    for _ in range(c["steps"]):
        sim.step()
    w = mb.writer
    np.savez_compressed(HERE / "outputs.npz", fingerprint=fingerprint(fields), z0=z, y0=y, x0=x,
                        time=np.array(w.times), **{f"out_{k}": np.stack(v) for k, v in w.rows.items()})
    print("outputs rows", len(w.times), {k: np.stack(v).shape for k, v in w.rows.items()})


def main() -> None:
    op = import_reference()
    if len(sys.argv) > 1:  # only the named fixtures, e.g. outputs_mixed
        for name in sys.argv[1:]:
            globals()[f"make_{name}"](op)
        return
    make_interp_kat(op)
    make_vertical_kat(op)
    make_workloads(op)
    make_edge_cases(op)
    make_zero_division(op)
    make_isopycnal(op)
    make_outputs(op)
    make_outputs_mixed(op)
    for p in sorted(HERE.glob("*.npz")) + sorted(HERE.glob("*.json")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
