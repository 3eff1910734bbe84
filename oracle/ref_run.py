"""Time the reference itself on this host's cores -- TEST INFRASTRUCTURE ONLY (the CPU baseline).

Runs the reference's own public API -- ``Fieldset`` of ``TimeDependentField``
/ ``StaticField`` from numpy arrays, the ROMS preset
``ab3_w_advection_timestepper`` (``models/roms/__init__.py:67-106``),
``SimulationBuilder(...).build_simulation(n)`` and ``Simulation.step()``
(``simulation.py:27-229``) -- from the compiled package in ``oracle/_ref``
(``oracle/ref_import.py: import_compiled``): its Cython/OpenMP kernels and its
numpy time blend, unmodified.  Only ``bench.py``'s CPU-baseline leg and tests
call this, as the measured baseline, never the product.
"""

from __future__ import annotations

import ctypes
import os
import time

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
}


def openmp_threads() -> int:
    """Threads an OpenMP parallel region of this process uses (libgomp's omp_get_max_threads)."""
    try:
        return int(ctypes.CDLL("libgomp.so.1").omp_get_max_threads())
    except (OSError, AttributeError):
        return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def physical_cores() -> int | None:
    try:
        import psutil

        return psutil.cpu_count(logical=False)
    except ImportError:
        return None


def time_ab3(time_array, fields: dict, hc: float, nz: int, dt: float, zyx, *, budget_s: float,
             max_steps: int = 30, warmup: int = 1) -> dict:
    """AB3 steps of the reference's ROMS preset on ``fields`` (u, v, w, zeta with a leading time axis;
    h, dx, dy, C) from the release ``zyx``: ``warmup`` untimed steps, then as many timed steps as fit
    ``budget_s`` (at most ``max_steps``, at least 1), estimated from the warm-up's duration."""
    from oracle.ref_import import import_compiled

    op = import_compiled()
    from offline_particles.models.roms import ab3_w_advection_timestepper

    nt, _, ny, nxu = fields["u"].shape
    kw = {}
    for name, arr in fields.items():
        st = STAGGERS[name]
        if name in ("u", "v", "w", "zeta"):
            kw[name] = op.TimeDependentField.from_numpy(arr, *st)
        else:
            kw[name] = op.StaticField.from_numpy(arr, *st)
    fs = op.Fieldset(nt, nz, ny, nxu + 1, constants={"hc": hc, "NZ": nz}, **kw)
    ts = ab3_w_advection_timestepper(np.asarray(time_array[:nt], dtype=np.float64), np.float64(dt))
    z, y, x = zyx
    sim = op.SimulationBuilder(ts, fs).build_simulation(len(z))
    sim.set_indices(zidx=z, yidx=y, xidx=x)
    sim.set_particle_field("status", np.uint8(10))  # MULTISTEP_1: the AB3 bootstrap (status.pxd:1-14)
    t0 = time.perf_counter()
    for _ in range(max(1, warmup)):
        sim.step()
    first = (time.perf_counter() - t0) / max(1, warmup)
    steps = max(1, min(max_steps, int(budget_s / max(first, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step()
    el = time.perf_counter() - t0
    return {"particle_steps_per_s": len(z) * steps / el, "steps": steps, "seconds": el, "warmup": max(1, warmup),
            "threads": openmp_threads(), "physical_cores": physical_cores(), "logical_cpus": os.cpu_count()}
