"""CPU oracle for the ROMS advection step -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, and only as the checker.  The product package
never imports it.

It restates the reference's algorithm for the hot path:

* the per-particle kernels, in plain C (``oracle/op_oracle.c``), called here
  through ctypes;
* the whole-grid time blend of ``TimeDependentField.get_field_data``
  (``fields.py:394-430``): ``It, ft = divmod(tidx, 1)``; ``ft``/``gt`` cast to
  the storage dtype; ``prev*gt`` and ``next*ft`` in the storage dtype; their sum
  written into float64 (``fields.py:423-428``);
* the stepper bookkeeping of ``Timestepper`` (``timesteppers.py:64-93,157-161``)
  and the launch order of ``RK2Timestepper.timestep_particles``
  (``timesteppers.py:241-257``) and ``ABTimestepper.timestep_particles``
  (``timesteppers.py:296-305``), with the ROMS presets' validation pre-step
  (``models/roms/__init__.py:37-106``).

Parity of this restatement with the reference itself is pinned by
``tests/test_oracle_golden.py`` against fixtures generated by running the
reference (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path
from typing import Mapping

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libop_oracle.so"
SRC = HERE / "op_oracle.c"

# Stagger offsets of the ROMS fields (spatial_arrays.py:29-41): CENTER 0,
# LEFT/OUTER +0.5, RIGHT/INNER -0.5; None = invariant (dimension absent).
STAGGER_OFFSET = {"center": 0.0, "left": 0.5, "outer": 0.5, "right": -0.5, "inner": -0.5, "invariant": None}

# Field conventions used by the ROMS w-advection kernels: (z, y, x) staggers.
ROMS_STAGGERS = {
    "u": ("center", "center", "inner"),
    "v": ("center", "inner", "center"),
    "w": ("outer", "center", "center"),
    "zeta": ("invariant", "center", "center"),
    "h": ("invariant", "center", "center"),
    "dx": ("invariant", "center", "center"),
    "dy": ("invariant", "center", "center"),
    "C": ("center", "invariant", "invariant"),
    "rho": ("center", "center", "center"),  # density at rho points (ab3_isopycnal_following)
}
TIME_DEPENDENT = ("u", "v", "w", "zeta")

INACTIVE, NORMAL, NONFINITE, OUT_OF_DOMAIN, MULTISTEP_1, MULTISTEP_2 = 0x80, 0, 0x81, 0x82, 10, 11


def build(force: bool = False) -> Path:
    """Compile ``op_oracle.c`` (gcc, OpenMP, no FP contraction)."""
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB_PATH
    LIB_PATH.parent.mkdir(parents=True, exist_ok=True)
    gcc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    tmp = LIB_PATH.with_suffix(f".{os.getpid()}.tmp")
    subprocess.run(
        [gcc, "-O3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
         str(SRC), "-o", str(tmp), "-lm"],
        check=True,
    )
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


# ----------------------------------------------------------------- ctypes ABI
class OF1(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("n0", ctypes.c_int64), ("o0", ctypes.c_double)]


class OF2(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("n0", ctypes.c_int64), ("n1", ctypes.c_int64),
                ("o0", ctypes.c_double), ("o1", ctypes.c_double)]


class OF3(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("n0", ctypes.c_int64), ("n1", ctypes.c_int64), ("n2", ctypes.c_int64),
                ("o0", ctypes.c_double), ("o1", ctypes.c_double), ("o2", ctypes.c_double)]


class ORomsFields(ctypes.Structure):
    _fields_ = [("u", OF3), ("v", OF3), ("w", OF3), ("dx", OF2), ("dy", OF2), ("h", OF2), ("zeta", OF2), ("C", OF1)]


_PFIELDS = ("zidx", "yidx", "xidx", "z", "_dxidx0", "_dyidx0", "_dz0", "_dxidx1", "_dyidx1", "_dz1",
            "_dxidx2", "_dyidx2", "_dz2")


class OParticles(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("status", ctypes.c_void_p)] + [
        (name.lstrip("_"), ctypes.c_void_p) for name in _PFIELDS
    ]


class OScalars(ctypes.Structure):
    _fields_ = [("hc", ctypes.c_double), ("NZ", ctypes.c_int32), ("dt", ctypes.c_double),
                ("alpha", ctypes.c_double), ("bounds", ctypes.c_double * 6)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        for name in ("oracle_finite_indices",):
            getattr(_lib, name).argtypes = [ctypes.POINTER(OParticles)]
        _lib.oracle_domain_bounds.argtypes = [ctypes.POINTER(OParticles), ctypes.POINTER(OScalars)]
        for name in ("oracle_rk2_step_1", "oracle_rk2_step_2", "oracle_rk2_update", "oracle_ab3", "oracle_ab3_post"):
            getattr(_lib, name).argtypes = [ctypes.POINTER(OParticles), ctypes.POINTER(OScalars),
                                            ctypes.POINTER(ORomsFields)]
            getattr(_lib, name).restype = ctypes.c_int
        _lib.oracle_ab3_isopycnal.argtypes = [ctypes.POINTER(OParticles), ctypes.POINTER(OScalars),
                                              ctypes.POINTER(ORomsFields), ctypes.c_void_p, ctypes.c_double,
                                              ctypes.c_double]
        _lib.oracle_ab3_isopycnal.restype = ctypes.c_int
        _lib.oracle_compute_z.argtypes = [ctypes.POINTER(OParticles), ctypes.c_void_p, ctypes.POINTER(OScalars),
                                          ctypes.POINTER(ORomsFields)]
        _lib.oracle_trilinear.argtypes = [ctypes.POINTER(OF3), ctypes.c_double, ctypes.c_double, ctypes.c_double]
        _lib.oracle_trilinear.restype = ctypes.c_double
        _lib.oracle_bilinear.argtypes = [ctypes.POINTER(OF2), ctypes.c_double, ctypes.c_double]
        _lib.oracle_bilinear.restype = ctypes.c_double
        _lib.oracle_linear.argtypes = [ctypes.POINTER(OF1), ctypes.c_double]
        _lib.oracle_linear.restype = ctypes.c_double
        _lib.oracle_compute_z_scalar.argtypes = [ctypes.c_double, ctypes.c_int32] + [ctypes.c_double] * 4
        _lib.oracle_compute_z_scalar.restype = ctypes.c_double
        _lib.oracle_compute_zidx_scalar.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int32, ctypes.POINTER(OF1)]
        _lib.oracle_compute_zidx_scalar.restype = ctypes.c_double
    return _lib


def _ptr(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


def make_field(arr: np.ndarray, offsets: tuple[float, ...]):
    """ctypes descriptor of a contiguous float64 field (kernels/_core.pyx:5-24)."""
    a = np.ascontiguousarray(arr, dtype=np.float64)
    if a.ndim == 1:
        f = OF1(_ptr(a), a.shape[0], offsets[0])
    elif a.ndim == 2:
        f = OF2(_ptr(a), *a.shape, *offsets)
    elif a.ndim == 3:
        f = OF3(_ptr(a), *a.shape, *offsets)
    else:
        raise ValueError(a.ndim)
    f._keep = a  # type: ignore[attr-defined]
    return f


def active_offsets(stagger: tuple[str, str, str]) -> tuple[float, ...]:
    return tuple(STAGGER_OFFSET[s] for s in stagger if STAGGER_OFFSET[s] is not None)


# ------------------------------------------------------------ time handling
def time_blend(prev: np.ndarray, nxt: np.ndarray, ft_raw) -> np.ndarray:
    """fields.py:419-428: blend in the storage dtype, result in float64."""
    dtype = prev.dtype
    ft = dtype.type(ft_raw)
    gt = dtype.type(1 - ft)
    a = np.multiply(prev, gt)
    b = np.multiply(nxt, ft)
    out = np.empty(prev.shape, dtype=np.float64)
    np.add(a, b, out=out, casting="unsafe")
    return out


def blend_weights(time_index, dtype) -> tuple[int, object, object]:
    """(It, ft, gt) exactly as fields.py:409-424 computes them."""
    It, ft = divmod(time_index, 1)
    dtype = np.dtype(dtype)
    ft = dtype.type(ft)
    gt = dtype.type(1 - ft)
    return int(It), ft, gt


def get_time_index(time_array: np.ndarray, time) -> np.float64:
    """timesteppers.py:64-85."""
    if time < time_array[0] or time > time_array[-1]:
        raise ValueError("Time is out of bounds of the time array.")
    idx = np.searchsorted(time_array, time, side="right") - 1
    t0 = time_array[idx]
    t1 = time_array[idx + 1]
    fraction = (time - t0) / (t1 - t0)
    return idx + fraction


# --------------------------------------------------------------- the oracle
class OracleROMS:
    """The reference's ROMS RK2/AB3 w-advection simulation, restated on the CPU.

    ``fields`` maps the ROMS field names to numpy arrays: ``u, v, w, zeta`` with
    a leading time axis, ``h, dx, dy`` 2-D and ``C`` 1-D.  ``particles`` maps
    particle-field names to arrays (copied).  Scheme "ab3_iso": the AB3
    isopycnal follower (models/roms/__init__.py:109-141), with ``rho`` in place
    of ``w``, the particle field ``rho_t`` and scalars ``w_max``, ``rho_scale``.
    """

    def __init__(
        self,
        time_array: np.ndarray,
        fields: Mapping[str, np.ndarray],
        *,
        hc: float,
        scheme: str,
        dt: float,
        alpha: float = 2 / 3,
        bounds: tuple[float, float, float, float, float, float] | None = None,
        time=None,
        staggers: Mapping[str, tuple[str, str, str]] = ROMS_STAGGERS,
        w_max: float = 0.0,
        rho_scale: float = 1.0,
    ) -> None:
        if scheme not in ("rk2", "ab3", "ab3_iso"):
            raise ValueError(scheme)
        self.w_max = np.float64(w_max)
        self.rho_scale = np.float64(rho_scale)
        self.scheme = scheme
        self.time_array = np.asarray(time_array)
        self.fields = dict(fields)
        self.staggers = dict(staggers)
        nt, nz, ny, nx = self._shape()
        self.NZ = np.int32(nz)
        self.hc = np.float64(hc)
        if bounds is None:  # fieldset.py:45-54
            bounds = (0, nz - 1, 0, ny - 1, 0, nx - 1)
        self.bounds = tuple(float(np.float64(b)) for b in bounds)
        self._dt = np.float64(dt / np.float64(1.0))  # timesteppers.py:87-93, time_unit 1.0
        self.alpha = alpha
        self.time = self.time_array[0] if time is None else time
        self.tidx = get_time_index(self.time_array, self.time)
        self.iteration = 0
        self._lib = lib()
        self._static = {
            name: make_field(self.fields[name], active_offsets(self.staggers[name])) for name in ("h", "dx", "dy", "C")
        }

    def _shape(self):
        u = self.fields["u"]
        nt, nz, ny = u.shape[0], u.shape[1], u.shape[2]
        nx = u.shape[3] + 1  # u is INNER in x
        return nt, nz, ny, nx

    @property
    def dt(self):
        return self._dt * np.float64(1.0)

    # ---------------------------------------------------------------- fields
    def fielddata(self, time_index, names=TIME_DEPENDENT) -> ORomsFields:
        """Blend the time-dependent ``names`` a launch declares (launcher.py:172)."""
        It, ft = divmod(time_index, 1)
        It = int(It)
        nt = self.fields["u"].shape[0]
        if It < 0 or It > nt - 2:  # fields.py:380-381
            raise IndexError(f"Valid range of time indices is 0,...,{nt - 2}, got {It}.")
        td = {}
        for name in TIME_DEPENDENT:
            if name in names:
                # the isopycnal follower reads rho where the w-advection kernels read w
                data = self.fields["rho" if (name == "w" and self.scheme == "ab3_iso") else name]
                sname = "rho" if (name == "w" and self.scheme == "ab3_iso") else name
                td[name] = make_field(time_blend(data[It], data[It + 1], ft), active_offsets(self.staggers[sname]))
            else:
                td[name] = OF3() if name != "zeta" else OF2()
        f = ORomsFields(td["u"], td["v"], td["w"], self._static["dx"], self._static["dy"], self._static["h"],
                        td["zeta"], self._static["C"])
        f._keep = td  # type: ignore[attr-defined]
        return f

    def _scalars(self) -> OScalars:
        return OScalars(float(self.hc), int(self.NZ), float(self._dt), float(self.alpha),
                        (ctypes.c_double * 6)(*self.bounds))

    @staticmethod
    def _particles(p: Mapping[str, np.ndarray]) -> OParticles:
        n = p["status"].shape[0]
        ptrs = []
        for name in _PFIELDS:
            a = p.get(name)
            ptrs.append(_ptr(a) if a is not None else None)
        return OParticles(n, _ptr(p["status"]), *ptrs)

    def _check(self, rc: int) -> None:
        if rc:
            raise ZeroDivisionError("float division")

    # -------------------------------------------------------------- stepping
    def validate(self, p: Mapping[str, np.ndarray]) -> None:
        op = self._particles(p)
        self._lib.oracle_finite_indices(ctypes.byref(op))
        self._lib.oracle_domain_bounds(ctypes.byref(op), ctypes.byref(self._scalars()))

    def advance_time(self) -> None:  # timesteppers.py:157-161
        self.time += self.dt
        self.tidx = get_time_index(self.time_array, self.time)
        self.iteration += 1

    def step(self, p: Mapping[str, np.ndarray]) -> None:
        op = self._particles(p)
        sc = self._scalars()
        L = self._lib
        self.validate(p)  # pre_step_kernel = validation_kernel
        if self.scheme == "rk2":  # timesteppers.py:241-257
            self._check(L.oracle_rk2_step_1(ctypes.byref(op), ctypes.byref(sc), ctypes.byref(self.fielddata(self.tidx))))
            t_int = self.time + self.alpha * self.dt
            tidx_int = get_time_index(self.time_array, t_int)
            self._check(L.oracle_rk2_step_2(ctypes.byref(op), ctypes.byref(sc), ctypes.byref(self.fielddata(tidx_int))))
            self.advance_time()
            L.oracle_rk2_update(ctypes.byref(op), ctypes.byref(sc), ctypes.byref(self.fielddata(self.tidx, ("zeta",))))
        elif self.scheme == "ab3_iso":  # timesteppers.py:296-305 with the isopycnal kernels
            self._check(L.oracle_ab3_isopycnal(ctypes.byref(op), ctypes.byref(sc),
                                               ctypes.byref(self.fielddata(self.tidx)), _ptr(p["rho_t"]),
                                               float(self.w_max), float(self.rho_scale)))
            self.advance_time()
            L.oracle_ab3_post(ctypes.byref(op), ctypes.byref(sc), ctypes.byref(self.fielddata(self.tidx, ("zeta",))))
        else:  # timesteppers.py:296-305
            self._check(L.oracle_ab3(ctypes.byref(op), ctypes.byref(sc), ctypes.byref(self.fielddata(self.tidx))))
            self.advance_time()
            L.oracle_ab3_post(ctypes.byref(op), ctypes.byref(sc), ctypes.byref(self.fielddata(self.tidx, ("zeta",))))

    def compute_z(self, p: Mapping[str, np.ndarray], out: np.ndarray) -> None:
        """kernels/roms/_roms_core.pyx:17-73 at the current time index."""
        op = self._particles(p)
        self._lib.oracle_compute_z(ctypes.byref(op), _ptr(out), ctypes.byref(self._scalars()),
                                   ctypes.byref(self.fielddata(self.tidx, ("zeta",))))


def particle_fields(scheme: str) -> tuple[str, ...]:
    """Particle fields the preset's kernels declare (merge of their particle_fields)."""
    base = ("status", "zidx", "yidx", "xidx", "z")
    if scheme == "rk2":
        return base + ("_dxidx1", "_dyidx1", "_dz1", "_dxidx2", "_dyidx2", "_dz2")
    ab3 = base + ("_dz0", "_dz1", "_dz2", "_dyidx0", "_dyidx1", "_dyidx2", "_dxidx0", "_dxidx1", "_dxidx2")
    return ab3 + ("rho_t",) if scheme == "ab3_iso" else ab3


def new_particles(n: int, scheme: str) -> dict[str, np.ndarray]:
    """Particles(n, ...) allocates zeros (particles.py:79-89)."""
    return {name: np.zeros(n, dtype=np.uint8 if name == "status" else np.float64) for name in particle_fields(scheme)}
