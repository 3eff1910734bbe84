"""Timesteppers: time bookkeeping and the launch order of one step (timesteppers.py:1-305 of the reference).

The time arithmetic (``get_time_index``, ``advance_time``, ``set_dt``) is the
reference's, in numpy float64, so every launch sees the same time index.

B200 path: when a stepper is built from the stock ROMS kernels (the presets of
``models.roms``), a step runs as ONE fused CUDA launch (validation + all
stages) instead of three or four, and ``timestep_particles_many`` runs many
steps per launch with the particle state held in registers.  Both give results
identical to the stage-by-stage sequence.
"""

from __future__ import annotations

import abc
import bisect
import ctypes
import dataclasses
import math

import numpy as np
import numpy.typing as npt
import torch

from . import _lib
from .fields import StaticField, TimeDependentField
from .kernels import ParticleKernel
from .kernels import _abi
from .launcher import Launcher, ScalarSource

type T = np.float64 | np.datetime64
type D = np.float64 | np.timedelta64

MAX_FUSED_STEPS = 240

# Observers of fused launches: objects with before(nsteps) / after(nsteps),
# called on the host around each fused kernel launch (used for timing).
launch_observers: list = []


def _notify(phase: str, nsteps: int) -> None:
    # an NVTX range around every fused launch (free unless a profiler listens)
    if phase == "before":
        torch.cuda.nvtx.range_push(f"opb fused {nsteps} steps")
    else:
        torch.cuda.nvtx.range_pop()
    for obs in launch_observers:
        getattr(obs, phase)(nsteps)


class Timestepper(abc.ABC):
    """Particle advection time stepping."""

    _dt_scalar = ScalarSource("_dt", lambda self, tidx: self._normalised_dt)
    _time_scalar = ScalarSource("_time", lambda self, tidx: self.time)
    _tidx_scalar = ScalarSource("_tidx", lambda self, tidx: self._tidx)

    def __init__(self, time_array: npt.NDArray, dt: D, *, time_unit: D | None = None, time: T | None = None,
                 iteration: int = 0, index_padding: int = 0) -> None:
        if np.any(time_array[1:] <= time_array[:-1]):
            raise ValueError("time_array must be strictly increasing.")
        self._time_array = time_array
        if time_unit is None:
            if isinstance(dt, np.floating):
                time_unit = np.float64(1.0)
            else:
                raise ValueError("time_unit must be specified for dimensional time.")
        self._time_unit = time_unit
        self.set_dt(dt)
        if time is None:
            time = self._time_array[0]
        self.set_time(time)
        self.set_iteration(iteration)
        self._index_padding = 0
        self.set_index_padding(index_padding)

    # the last time asked for and its index (the planner asks for each step's end time twice: as the end
    # of one step and the start of the next)
    _time_index_memo: tuple | None = None

    def get_time_index(self, time: T) -> np.float64:
        """timesteppers.py:64-85: searchsorted plus the fraction within the interval."""
        memo = self._time_index_memo
        if memo is not None and memo[0] is self._time_array and type(time) is memo[1] and time == memo[2]:
            return memo[3]
        r = self._get_time_index(time)
        if isinstance(time, (float, np.float64)):
            self._time_index_memo = (self._time_array, type(time), time, r)
        return r

    def _get_time_index(self, time: T) -> np.float64:
        fast = self._float_times()
        if fast is not None and isinstance(time, (float, np.float64)):
            # the same arithmetic on Python floats (IEEE doubles, as numpy's float64 scalars): bisect_right
            # is searchsorted(side="right"), and int + float equals numpy's int64 + float64 for these sizes
            if time < fast[0] or time > fast[-1]:
                raise ValueError("Time is out of bounds of the time array.")
            idx = bisect.bisect_right(fast, time) - 1
            t0 = fast[idx]
            t1 = fast[idx + 1]  # IndexError at the last time, as the numpy path raises
            return np.float64(idx + (float(time) - t0) / (t1 - t0))
        time_array = self._time_array
        if time < time_array[0] or time > time_array[-1]:
            raise ValueError("Time is out of bounds of the time array.")
        idx = np.searchsorted(time_array, time, side="right") - 1
        t0 = time_array[idx]
        t1 = time_array[idx + 1]
        fraction = (time - t0) / (t1 - t0)
        return idx + fraction

    def _float_times(self) -> list | None:
        """The time array as Python floats when it is float64 (cached), else None."""
        arr = self._time_array
        cached = self.__dict__.get("_float_times_cache")
        if cached is None or cached[0] is not arr:
            fast = arr.tolist() if isinstance(arr, np.ndarray) and arr.dtype == np.float64 and arr.ndim == 1 else None
            cached = (arr, fast)
            self.__dict__["_float_times_cache"] = cached
        return cached[1]

    def set_dt(self, dt: D) -> None:
        try:
            self._normalised_dt = np.float64(dt / self._time_unit)
        except Exception as e:
            raise TypeError(f"dt must be of the same type as time_unit={self._time_unit!r}") from e

    def set_time(self, time: T) -> None:
        try:
            _ = time + self.dt
        except Exception as e:
            raise TypeError(f"time must be compatible with dt={self.dt!r}") from e
        self._tidx = self.get_time_index(time)
        self._time = time

    def set_iteration(self, iteration: int) -> None:
        if iteration < 0:
            raise ValueError("Iteration must be non-negative.")
        self._iteration = iteration

    def set_index_padding(self, index_padding: int, force: bool = False) -> None:
        if index_padding < 0:
            raise ValueError("Index padding must be non-negative.")
        if force or index_padding > self._index_padding:
            self._index_padding = index_padding

    @property
    def time_unit(self) -> D:
        return self._time_unit

    @property
    def dt(self) -> D:
        return self._normalised_dt * self._time_unit

    @property
    def time(self) -> T:
        return self._time

    @property
    def time_array(self) -> npt.NDArray:
        return self._time_array

    @property
    def iteration(self) -> int:
        return self._iteration

    @property
    def tidx(self) -> np.float64:
        return self._tidx

    @property
    def index_padding(self) -> int:
        return self._index_padding

    def advance_time(self) -> None:
        """timesteppers.py:157-161."""
        self._last_start_tidx = self._tidx
        self._time += self.dt
        self._tidx = self.get_time_index(self._time)
        self._iteration += 1

    # time index at the start of the last step taken (None before the first)
    _last_start_tidx = None

    @property
    def at_interval_start(self) -> bool:
        """True when the next step starts in a later snapshot interval than the last step did (or no step
        has run): the point where a fused launch would start a new snapshot pair anyway."""
        last = self._last_start_tidx
        return last is None or int(divmod(self._tidx, 1)[0]) != int(divmod(last, 1)[0])

    def steps_to_interval_end(self, at_least: int, limit: int = 1 << 16) -> int:
        """The fewest steps n >= max(1, at_least) after which the next step starts in a later snapshot
        interval than step n did: running n steps ends on a snapshot-interval boundary.  Stops early (at
        least 1) where the time array ends."""
        t = self._time
        fast = self._float_times()
        if fast is not None and isinstance(t, (float, np.float64)):
            interval = self._fast_interval(fast)
            t = float(t)
            dt = float(self.dt)  # the same double as self.dt, added as the stepping adds it
        else:
            def interval(x):
                return int(divmod(self.get_time_index(x), 1)[0])

            dt = self.dt
        try:
            cur = interval(t)
        except (ValueError, IndexError):
            return max(1, at_least)
        n = 0
        while n < limit:
            t = t + dt
            n += 1
            try:
                nxt = interval(t)
            except (ValueError, IndexError):
                return max(n, 1, min(at_least, limit))
            if nxt != cur and n >= at_least:
                return n
            cur = nxt
        return max(1, min(at_least, limit))

    @staticmethod
    def _fast_interval(fast: list):
        """int(divmod(get_time_index(x), 1)[0]) for a Python float x: get_time_index's fast path inlined
        (the same operations on the same doubles), without the numpy scalar around the result."""
        lo, hi = fast[0], fast[-1]

        def interval(x: float) -> int:
            if x < lo or x > hi:
                raise ValueError("Time is out of bounds of the time array.")
            idx = bisect.bisect_right(fast, x) - 1
            t0 = fast[idx]
            return int(divmod(idx + (x - t0) / (fast[idx + 1] - t0), 1)[0])

        return interval

    @property
    @abc.abstractmethod
    def kernels(self) -> tuple[ParticleKernel, ...]: ...

    @abc.abstractmethod
    def timestep_particles(self, particles, launcher: Launcher) -> None: ...

    # ------------------------------------------------------------ fused path
    def _stage_times(self, time) -> tuple[list, object]:
        """Time indices of the field lookups of one step starting at ``time``, and the next time."""
        raise NotImplementedError

    def fused(self) -> bool:
        """True when the kernels are the stock ROMS ones and steps can run fused."""
        return False

    @property
    def field_roles(self) -> dict[str, str]:
        """C-ABI field slot -> fieldset name, where the stepper's kernels read another field."""
        return {}

    # last snapshot index worth prefetching (set by Simulation.run for its horizon; None: no limit)
    _prefetch_limit: int | None = None

    def snapshot_horizon(self, nsteps: int) -> int | None:
        """The last snapshot index the next ``nsteps`` steps read (None when past the time array)."""
        t, dt = self._time, self.dt
        if isinstance(t, (float, np.float64)) and isinstance(dt, (float, np.float64)):
            t, dt = float(t), float(dt)  # the same doubles, added without numpy scalars
        for _ in range(nsteps):
            t = t + dt
        try:
            return int(divmod(self.get_time_index(t), 1)[0]) + 1
        except (ValueError, IndexError):
            return None

    def reserve_launch_buffers(self, launcher: Launcher, nparticles: int) -> None:
        """Allocate what the fused launches over ``nparticles`` particles will read besides the snapshots
        (the snapshot-pair buffers; the static bundles or neighbour layouts, built once), so that no
        launch allocates device memory."""
        if not self.fused():
            return
        roles = self.field_roles
        td = _time_dependent_fields(launcher, roles)
        if not use_pairs(launcher, td, nparticles, roles):
            return
        plan = pair_layout(launcher, td, roles)
        for name, field in td.items():
            field.reserve_pairs("zeta_h" if plan.bundles is not None and name == "zeta" else plan.layout)
        if plan.bundles is not None:
            plan.bundles["dx"].bundle(plan.bundles["dy"])
        elif plan.layout in _STATIC_KIND:
            for field in plan.statics.values():
                field.neighbours(_STATIC_KIND[plan.layout])

    def timestep_particles_many(self, particles, launcher: Launcher, nsteps: int,
                                split: "RangeLaunches | None" = None, recorder=None) -> None:
        """Advance ``nsteps`` steps; fused launches where possible, else step by step.  ``split``: run the
        fused launch that takes the last of these steps range by range over particle storage (one launch
        per range, ``split.after(i)`` once range i's launch is queued).  ``recorder``: events that fall
        inside the launches (``recorder.plan`` gives a launch its records, ``after_step`` follows a step
        run on its own)."""
        if not self.fused():
            for _ in range(nsteps):
                self.timestep_particles(particles, launcher)
                if recorder is not None:
                    recorder.after_step(self._iteration)
            return
        done = 0
        while done < nsteps:
            done += self._fused_chunk(particles, launcher, nsteps - done, split, recorder)

    def _fused_chunk(self, particles, launcher: Launcher, max_steps: int,
                     split: "RangeLaunches | None" = None, recorder=None) -> int:
        """Plan and launch as many steps as fit in one fused launch; return the number taken.  ``split``
        applies when the launch takes all ``max_steps``."""
        td = _time_dependent_fields(launcher, self.field_roles)
        # streamed fields: a launch spans at most one snapshot interval (3 snapshots) and a slot stays free,
        # so each launch waits for at most one new upload and the next ones stream in while it runs (a launch
        # spanning n intervals would first wait for all n + 2 uploads)
        capacity = min([_lib.MAX_SLOTS] + [min(3, max(2, f.ring_size - 1)) if f.streamed else f.ring_size
                                           for f in td.values()])
        pairs = use_pairs(launcher, td, len(particles), self.field_roles)
        streamed = any(f.streamed for f in td.values())
        pair_capacity = min([_lib.MAX_SLOTS] + [f.pair_slots for f in td.values()])
        starts: set[int] = set()  # snapshot intervals the launch's stages read (one pair each)
        time = self._time
        steps: list[list] = []
        needed: set[int] = set()
        end_times = []
        last_snapshot = min(f.num_timesteps for f in td.values()) - 1 if td else None
        while len(steps) < min(max_steps, MAX_FUSED_STEPS):
            if recorder is not None and steps and recorder.full(self._iteration, len(steps) + 1):
                break  # the launch's recorded states would pass their memory budget
            try:
                tidxs, nxt = self._stage_times(time)
            except (ValueError, IndexError):
                break
            its = {int(divmod(t, 1)[0]) for t in tidxs}
            more = needed | its | {i + 1 for i in its}
            if len(more) > capacity or (last_snapshot is not None and max(its) + 1 > last_snapshot):
                break
            if pairs and len(starts | its) > pair_capacity:
                break
            # pipelining over streamed snapshots: a launch waits only for the uploads its first step waits
            # for (and for one if that step waits for none), so compute starts as soon as they land and the
            # next snapshots stream in behind it
            if streamed:
                pending = {k for k in more if not all(f.is_ready(k) for f in td.values())}
                if not steps:
                    allowed = max(1, len(pending))
                elif len(pending) > allowed:
                    break
            starts |= its
            needed = more
            steps.append(tidxs)
            end_times.append(nxt)
            time = nxt
        if not steps:
            # the next step raises or cannot be fused: run it the reference way (raises where it raises)
            self._unfused_step(particles, launcher)
            if recorder is not None:
                recorder.after_step(self._iteration)
            return 1
        last = split if split is not None and len(steps) == max_steps else None
        rec = None
        if recorder is not None:
            rec = recorder.plan(self._iteration, end_times, [st[-1] for st in steps])
        self._launch_fused(particles, launcher, steps, sorted(needed), td, last, rec)
        if last is not None:
            last.used = True
        # bookkeeping exactly as advance_time would have left it after each step
        self._last_start_tidx = steps[-1][0]
        self._time = end_times[-1]
        self._tidx = steps[-1][-1]
        self._iteration += len(steps)
        return len(steps)

    def _unfused_step(self, particles, launcher: Launcher) -> None:
        raise NotImplementedError

    def _launch_fused(self, particles, launcher: Launcher, steps: list[list], needed: list[int],
                      td: dict[str, TimeDependentField], split: "RangeLaunches | None" = None, rec=None) -> None:
        raise NotImplementedError


class RangeLaunches:
    """One fused launch issued as one launch per range of particle storage: ``ranges`` are ``(lo, hi)``
    slot ranges covering the particles in order, and ``after(i)`` is called once range i's launch is
    queued (the caller starts reading that range back while the next range computes).  Particles are
    independent, so the split changes no result.  ``used`` is set once a launch was split."""

    def __init__(self, ranges: list[tuple[int, int]], after) -> None:
        self.ranges = list(ranges)
        self.after = after
        self.used = False


def _fused_call(entry: str, particles, split: RangeLaunches | None, args: tuple, stream, rec=None) -> None:
    """Call a fused entry point over all particles, or range by range (``split``); with ``rec`` (a record
    plan: ``struct``, ``at(lo)``) its ``_rec`` form, recording the state after the planned steps."""

    def call(ps, r) -> None:
        if r is None:
            _lib.call(entry, ctypes.byref(ps), *args, stream)
        else:
            _lib.call(entry + "_rec", ctypes.byref(ps), *args, ctypes.byref(r), stream)

    if split is None:
        call(_abi.particles_struct(particles), None if rec is None else rec.struct)
        return
    for i, (lo, hi) in enumerate(split.ranges):
        if hi > lo:
            call(_abi.particles_struct_range(particles, lo, hi), None if rec is None else rec.at(lo))
        split.after(i)


def _require_float64(launcher: Launcher) -> None:
    if launcher.arithmetic != "float64":
        raise ValueError("arithmetic='float32' runs only the fused ROMS steppers; this step needs the "
                         "stage-by-stage float64 path")


def _time_dependent_fields(launcher: Launcher, roles: dict[str, str] | None = None
                           ) -> dict[str, TimeDependentField]:
    """The time-dependent fields by C-ABI slot name; ``roles`` maps a slot to the fieldset name that fills
    it where they differ (the isopycnal follower's rho in the w slot)."""
    fs = launcher.fieldset
    roles = roles or {}
    out = {}
    for n in _abi.ROMS_FIELDS:
        src = roles.get(n, n)
        if src in fs and isinstance(fs[src], TimeDependentField):
            out[n] = fs[src]
    return out


# The float64 fused steppers can read the time-dependent fields as snapshot pairs: one load per stencil
# corner instead of two, about 11 % less kernel time on the 1024x768x50 AB3 workload.  A pair costs one
# pass over two snapshots and a write of both per snapshot interval, so it pays when the particles'
# work per interval outweighs that: measured, and by the cost model, when there is at least one particle
# per 32 grid cells (4.19 M particles on 39.3 M cells: 13.8 -> 15.0 G particle-steps/s; a release of a
# thousand particles would pay more for the pairs than it saves).
# "auto" (default: that rule), "always" or "never".
SNAPSHOT_PAIRS = "auto"
PAIR_CELLS_PER_PARTICLE = 32


def roms_geometry(launcher: Launcher, roles: dict[str, str] | None = None) -> bool:
    """The fields sit on the ROMS Arakawa C grid of the fieldset's nz x ny x nx rho points: u on (nz, ny, nx - 1)
    at x offset -0.5, v on (nz, ny - 1, nx) at y offset -0.5, w on (nz + 1, ny, nx) at z offset +0.5 (the
    isopycnal follower's density in the w slot: on rho points), zeta, h, dx, dy on (ny, nx) and C on nz
    levels, every other offset 0.  The library's compiled-layout kernels (and so the snapshot pairs) need
    exactly this geometry."""
    fs = launcher.fieldset
    roles = roles or {}
    key = (tuple(sorted(roles.items())),
           tuple((n, id(fs[roles.get(n, n)]) if roles.get(n, n) in fs else None) for n in _abi.ROMS_FIELDS))
    cache = launcher.__dict__.setdefault("_roms_geometry_cache", {})
    if key not in cache:
        cache[key] = _roms_geometry(fs, roles)
    return cache[key]


def _roms_geometry(fs, roles: dict[str, str]) -> bool:
    nz, ny, nx = fs.z_size, fs.y_size, fs.x_size
    w_rho = roles.get("w", "w") != "w"
    want = {"u": ((nz, ny, nx - 1), (0.0, 0.0, -0.5)), "v": ((nz, ny - 1, nx), (0.0, -0.5, 0.0)),
            "w": ((nz, ny, nx), (0.0, 0.0, 0.0)) if w_rho else ((nz + 1, ny, nx), (0.5, 0.0, 0.0)),
            "C": ((nz,), (0.0,)), **{n: ((ny, nx), (0.0, 0.0)) for n in ("zeta", "h", "dx", "dy")}}
    for name, (shape, offsets) in want.items():
        src = roles.get(name, name)
        if src not in fs:
            return False
        f = fs[src]
        got = tuple(f.active_offsets)
        if (tuple(f.spatial_shape) != shape or got != offsets
                or any(o == 0.0 and math.copysign(1.0, o) < 0 for o in got)):
            return False
    return True


def use_pairs(launcher: Launcher, td: dict[str, TimeDependentField], nparticles: int,
              roles: dict[str, str] | None = None) -> bool:
    """Snapshot pairs apply to the float64 steppers on the ROMS layout and geometry with float32/float64
    storage (the answer is kept per launcher for the same fields, count and module settings)."""
    key = (SNAPSHOT_PAIRS, PAIR_CELLS_PER_PARTICLE, launcher.arithmetic, nparticles,
           tuple(sorted((roles or {}).items())), tuple((n, id(f)) for n, f in td.items()))
    cache = launcher.__dict__.setdefault("_use_pairs_cache", {})
    hit = cache.get(key)
    if hit is None:
        hit = cache[key] = _use_pairs(launcher, td, nparticles, roles)
    return hit


def _use_pairs(launcher: Launcher, td: dict[str, TimeDependentField], nparticles: int,
               roles: dict[str, str] | None = None) -> bool:
    if SNAPSHOT_PAIRS == "never" or launcher.arithmetic != "float64" or set(td) != {"u", "v", "w", "zeta"}:
        return False
    if not roms_geometry(launcher, roles):
        return False
    if not all(f.storage in ("float32", "float64") for f in td.values()):
        return False
    if SNAPSHOT_PAIRS == "always":
        return True
    fs = launcher.fieldset
    return nparticles * PAIR_CELLS_PER_PARTICLE >= fs.z_size * fs.y_size * fs.x_size


# With float32 storage the pairs can be wider: "quads" (each element's snapshot pair followed by its
# x-neighbour's, static h, dx, dy as x-pairs: a stencil's two x-neighbouring corners in one 16-byte load)
# or "octets" (the pairs of a stencil face's four corners, static h, dx, dy as yx-pairs: one 32-byte load
# per face, one per bilinear stencil); "pairs" keeps the plain pairs.  Measured on B200 (1024x768x50,
# 4.19 M particles, AB3): the fused kernel runs 1.4 % (quads) and 2.9 % (octets) faster per step, but the
# wider build per snapshot interval costs more than that, so the fused steppers keep pairs.  The batched
# launch, whose particles do far more work per interval than one build, gains 9 % with quads (its
# gathers are bound by L1 requests) and 2 % with octets (four times the bytes per element in L1).
SNAPSHOT_LAYOUT = "pairs"  # the fused steppers
BATCH_LAYOUT = "quads"  # ReleaseBatch
NEIGHBOUR_STATICS = ("h", "dx", "dy")
_STATIC_KIND = {"quads": "xpairs", "octets": "yxpairs"}
_PAIR_CODE = {"quads": _lib.F32_QUADS, "octets": _lib.F32_OCTS}
_STATIC_CODE = {"xpairs": _lib.F64_XPAIRS, "yxpairs": _lib.F64_YXPAIRS}


# The 2-D fields h, zeta, dx and dy share one stagger in the ROMS layout: with float32 pairs or quads of
# u, v, w they are read as two bundles, zeta with h and dx with dy, so one 32-byte load fetches two
# stencil corners of both fields of a bundle.
BUNDLE_2D = True


@dataclasses.dataclass
class PairPlan:
    """How a launch that reads pairs reads its fields: ``layout`` of u, v, w (and zeta when not bundled),
    ``statics`` read as neighbour layouts beside quads and octets (h, dx, dy), ``bundles`` the static
    fields of the 2-D bundles (h with zeta, dy with dx) or None."""

    layout: str = "pairs"
    statics: dict | None = None
    bundles: dict | None = None


def pair_layout(launcher: Launcher, td: dict[str, TimeDependentField], roles: dict[str, str] | None = None,
                layout: str | None = None) -> PairPlan:
    """The pair plan of a launch that reads pairs ("pairs", "quads" or "octets"; ``layout``, default
    ``SNAPSHOT_LAYOUT``).  The wider layouts and the bundles need float32 storage and static h, dx, dy;
    otherwise plain pairs."""
    layout = SNAPSHOT_LAYOUT if layout is None else layout
    if layout not in ("pairs", "quads", "octets"):
        raise ValueError(f"unknown pair layout {layout!r}")
    key = (layout, BUNDLE_2D, tuple(sorted((roles or {}).items())), tuple((n, id(f)) for n, f in td.items()))
    cache = launcher.__dict__.setdefault("_pair_layout_cache", {})
    plan = cache.get(key)
    if plan is None:
        plan = cache[key] = _pair_layout(launcher, td, roles, layout)
    return plan


def _pair_layout(launcher: Launcher, td: dict[str, TimeDependentField], roles: dict[str, str] | None,
                 layout: str) -> PairPlan:
    if not td or not all(f.storage == "float32" for f in td.values()):
        return PairPlan()
    fs = launcher.fieldset
    roles = roles or {}
    statics = {n: fs[roles.get(n, n)] for n in NEIGHBOUR_STATICS if roles.get(n, n) in fs}
    if len(statics) != len(NEIGHBOUR_STATICS) or not all(isinstance(f, StaticField) for f in statics.values()):
        return PairPlan()
    plan = PairPlan(layout, statics if layout != "pairs" else None)
    zeta = td.get("zeta")
    if (BUNDLE_2D and layout in ("pairs", "quads") and zeta is not None
            and statics["h"].spatial_shape == zeta.spatial_shape and statics["h"].active_offsets == zeta.active_offsets
            and statics["dx"].spatial_shape == statics["dy"].spatial_shape
            and statics["dx"].active_offsets == statics["dy"].active_offsets):
        plan.statics, plan.bundles = None, statics
    return plan


def pair_fields(rf, its: list[int], td: dict[str, TimeDependentField], plan: PairPlan | None = None
                ) -> dict[int, int]:
    """Point the time-dependent fields of ``rf`` at snapshot pairs ``its`` (slot q holds pair its[q]) as
    ``plan`` (``pair_layout``) says: u, v, w (and zeta) in its layout, h, dx, dy at their neighbour layouts
    beside quads and octets, or zeta with h and dx with dy as bundles; return pair -> slot."""
    plan = plan or PairPlan()
    layout = plan.layout
    keep = set(its)
    bundles = plan.bundles
    h_data = bundles["h"].data.data.contiguous() if bundles else None
    for name, field in td.items():
        f = getattr(rf, name)
        bundled = bundles is not None and name == "zeta"
        if bundled:
            f.dtype = _lib.F32_ZETA_H
        elif layout in _PAIR_CODE:
            f.dtype = _PAIR_CODE[layout]
        else:
            f.dtype = _lib.F32_PAIRS if field.storage == "float32" else _lib.F64_PAIRS
        for q in range(_lib.MAX_SLOTS):
            if q < len(its):
                buf = (field.pair(its[q], keep, layout="zeta_h", static=h_data) if bundled
                       else field.pair(its[q], keep, layout=layout))
                f.data[q] = buf.data_ptr()
            else:
                f.data[q] = None
            f.scale[q] = None
        if len(its) == 1:
            f.data[1] = f.data[0]
        f.nslots = max(2, len(its))
    if bundles is not None:
        rf.h.dtype = _lib.F64_IN_ZETA
        rf.dx.dtype = _lib.F64_DX_DY
        rf.dx.data[0] = bundles["dx"].bundle(bundles["dy"]).data_ptr()
        rf.dy.dtype = _lib.F64_IN_DX
    elif layout in _STATIC_KIND:
        kind = _STATIC_KIND[layout]
        for name, field in plan.statics.items():
            g = getattr(rf, name)
            g.dtype = _STATIC_CODE[kind]
            g.data[0] = field.neighbours(kind).data_ptr()
    return {k: q for q, k in enumerate(its)}


def _fused_fields(launcher: Launcher, steps: list[list], needed: list[int], td: dict[str, TimeDependentField],
                  nparticles: int, roles: dict[str, str] | None = None):
    """opb_roms_fields over the snapshots ``needed`` plus the per-stage opb_time table.  With snapshot
    pairs the launch reads pairs only: the single snapshots are not acquired (a pair build waits for the
    uploads of its own two snapshots, not for those of every field)."""
    pairs = use_pairs(launcher, td, nparticles, roles)
    rf, dtype = window_fields(launcher, needed, td, roles, acquire=not pairs)
    entries = [t for step in steps for t in step]
    if pairs:
        pslot = pair_fields(rf, sorted({int(divmod(t, 1)[0]) for t in entries}), td, pair_layout(launcher, td, roles))
        prev_next = lambda It: (pslot[It], pslot[It])  # noqa: E731
    else:
        slot = {k: j for j, k in enumerate(needed)}
        prev_next = lambda It: (slot[It], slot[It + 1])  # noqa: E731
    table, its = step_table(entries, dtype, prev_next)
    # move the field windows the way the stage launches would have (each distinct index in order)
    seq = [i for j, i in enumerate(its) if j == 0 or i != its[j - 1]]
    for field in td.values():
        for i in seq:
            field.set_time_index(i)
    return rf, table


def step_table(entries, dtype, prev_next):
    """The opb_time table of a fused launch and the snapshot index of each entry.  Per entry (a time index
    tidx): It, ft = divmod(tidx, 1); ft and gt = 1 - ft rounded to the storage ``dtype``
    (fields.py:423-424); (prev, next) = prev_next(It).  The numpy operations of that scalar form, applied
    to the whole table at once."""
    It_f, fr = np.divmod(np.asarray(entries, dtype=np.float64), 1.0)
    ft = fr.astype(dtype)
    gt = dtype.type(1) - ft
    its = It_f.astype(np.int64).tolist()
    rec = np.empty(len(its), dtype=_TIME_DTYPE)
    if its:
        rec["prev"], rec["next"] = zip(*(prev_next(i) for i in its))
    rec["ft"] = ft.astype(np.float64)
    rec["gt"] = gt.astype(np.float64)
    table = (_lib.opb_time * len(its))()
    ctypes.memmove(table, rec.ctypes.data, rec.nbytes)
    return table, its


# opb_time as a numpy record (int32 prev, int32 next, float64 ft, float64 gt: 24 bytes, no padding)
_TIME_DTYPE = np.dtype([("prev", np.int32), ("next", np.int32), ("ft", np.float64), ("gt", np.float64)])
assert _TIME_DTYPE.itemsize == ctypes.sizeof(_lib.opb_time)


def window_fields(launcher: Launcher, needed: list[int], td: dict[str, TimeDependentField],
                  roles: dict[str, str] | None = None, acquire: bool = True):
    """opb_roms_fields whose slot j of every time-dependent field holds snapshot ``needed[j]``, and the
    storage dtype of the time-dependent fields (numpy float64 or float32).  ``acquire=False`` leaves the
    time-dependent slots empty (the caller points them at snapshot pairs)."""
    fs = launcher.fieldset
    roles = roles or {}
    for name in _abi.ROMS_FIELDS:
        if roles.get(name, name) not in fs:
            raise KeyError(f"Field '{roles.get(name, name)}' does not exist in Fieldset.")
    dtypes = {np.dtype(f.dtype) for f in td.values()}
    if len(dtypes) > 1:
        raise ValueError("time-dependent fields of one launch must share one storage dtype")
    dtype = dtypes.pop() if dtypes else np.dtype(np.float64)
    storages = {f.storage for f in td.values()}
    if storages & {"bfloat16", "float16"} and launcher.arithmetic != "float32":
        raise ValueError("bfloat16/float16 field storage needs the float32 steppers "
                         "(build_simulation(..., arithmetic='float32'))")
    slot = {k: j for j, k in enumerate(needed)}
    keep = set(needed)
    rf = _lib.opb_roms_fields()
    for name in _abi.ROMS_FIELDS:
        field = fs[roles.get(name, name)]
        if name in td:
            f = _lib.opb_field.from_buffer_copy(_td_skeleton(field, name))
            for k in needed if acquire else ():
                f.data[slot[k]] = _abi._ptr(field.snapshot(k, keep))
                sc = field.snapshot_scales(k)
                if sc is not None:
                    f.scale[slot[k]] = _abi._ptr(sc)
            f.nslots = len(needed)
        else:
            f = _static_struct(field, name)
        setattr(rf, name, f)
    return rf, dtype


def _td_skeleton(field, name: str):
    """opb_field of a time-dependent field without its snapshot pointers (storage dtype, shape, offsets;
    built once per field and slot name)."""
    cache = field.__dict__.setdefault("_opb_skeletons", {})
    f = cache.get(name)
    if f is None:
        f = _lib.opb_field()
        f.is_static = 0
        f.dtype = _STORAGE_CODE[field.storage]
        shape = field.spatial_shape
        offsets = field.active_offsets
        nd = _abi.ROMS_NDIM[name]
        if len(shape) != nd:
            raise ValueError(f"field '{name}' must have {nd} active dimensions")
        f.ndim = nd
        for d in range(nd):
            f.shape[d] = shape[d]
            f.offset[d] = offsets[d]
        cache[name] = f
    return f


def _static_struct(field, name: str):
    """opb_field of a static field (built once per field and slot name; ctypes copies it into each
    launch's struct)."""
    cache = field.__dict__.setdefault("_opb_structs", {})
    f = cache.get(name)
    if f is None:
        f = cache[name] = _abi.field_struct(field.get_field_data(0.0), _abi.ROMS_NDIM[name], name)
    return f


_STORAGE_CODE = {"float64": _lib.F64, "float32": _lib.F32, "bfloat16": _lib.BF16, "float16": _lib.F16}


def _entry(name: str, launcher: Launcher) -> str:
    """The float64 (bit-exact) or float32 fused entry point."""
    return name + ("_fp32" if launcher.arithmetic == "float32" else "")


def _table_arg(table, device, rf=None):
    """The step-table argument of a fused launch, and what must stay alive until the call returns: the
    host table itself while it fits the launch's parameters (no copy, so the launch does not queue
    behind the snapshot uploads already issued), else a device copy.  The library checks a host table's
    snapshot slots against the fields ``rf``; a device copy it reads unchecked, so its slots are checked
    here before the copy."""
    if len(table) <= _lib.INLINE_TABLE:
        return ctypes.addressof(table), table
    if rf is not None:
        nslots = min(getattr(rf, n).nslots for n in _abi.ROMS_FIELDS if not getattr(rf, n).is_static)
        if any(not (0 <= e.prev < nslots and 0 <= e.next < nslots) for e in table):
            raise ValueError(f"step table selects a snapshot slot outside the fields' {nslots} slots")
    raw = torch.frombuffer(bytearray(bytes(table)), dtype=torch.uint8).pin_memory()
    dev = raw.to(device, non_blocking=True)
    return dev.data_ptr(), dev


def _prefetch_after(td: dict[str, TimeDependentField], needed: list[int], limit: int | None = None) -> None:
    """After a launch: mark its snapshots' slots as read by it, then start uploading the snapshots that
    follow into every slot the next launch does not need (the last two are kept): with a deeper ring the
    host stream never waits for a launch to free a slot."""
    if not needed:
        return
    last = needed[-1]
    for f in td.values():
        f.mark_used(needed)
    streamed = [f for f in td.values() if f.streamed]
    if not streamed:
        return
    keep = {needed[-2], last} if len(needed) > 1 else {last}
    depth = {id(f): max(1, f.ring_size - len(keep)) for f in streamed}
    # snapshot by snapshot, every field of one before any of the next: the copy stream delivers them in
    # that order, so the next launch's snapshots are not queued behind later ones of other fields
    for j in range(1, max(depth.values()) + 1):
        if limit is not None and last + j > limit:
            break  # past the snapshots the current run needs
        keep.add(last + j)
        for f in streamed:
            if j <= depth[id(f)]:
                f.prefetch(last + j, set(keep))


class RK2Timestepper(Timestepper):
    """Two-stage explicit Runge-Kutta (timesteppers.py:164-257).

    Butcher tableau  0 | ; alpha | alpha ; | 1 - 1/(2 alpha), 1/(2 alpha).  The
    ROMS update kernel applies b1 = 1/(2 alpha) to k1 (rk2_w_advection.pyx:
    317-318), the reference's own convention, which is kept.
    """

    _alpha_scalar = ScalarSource("_RK2_alpha", lambda self, tidx: self._alpha)

    def __init__(self, time_array, dt, rk_step_1_kernel: ParticleKernel, rk_step_2_kernel: ParticleKernel,
                 rk_update_kernel: ParticleKernel, *, alpha: float = 2 / 3, time_unit=None, time=None,
                 iteration: int = 0, index_padding: int = 0, pre_step_kernel: ParticleKernel | None = None,
                 post_step_kernel: ParticleKernel | None = None) -> None:
        super().__init__(time_array, dt, time_unit=time_unit, time=time, index_padding=index_padding,
                         iteration=iteration)
        self._rk_step_1_kernel = rk_step_1_kernel
        self._rk_step_2_kernel = rk_step_2_kernel
        self._rk_update_kernel = rk_update_kernel
        self._pre_step_kernel = pre_step_kernel
        self._post_step_kernel = post_step_kernel
        self._alpha = alpha

    @property
    def alpha(self) -> float:
        return self._alpha

    @property
    def kernels(self) -> tuple[ParticleKernel, ...]:
        pre = (self._pre_step_kernel,) if self._pre_step_kernel is not None else ()
        post = (self._post_step_kernel,) if self._post_step_kernel is not None else ()
        return pre + (self._rk_step_1_kernel, self._rk_step_2_kernel, self._rk_update_kernel) + post

    def fused(self) -> bool:
        from .kernels.roms import rk2_w_advection as rk
        from .kernels.validation import validation_kernel

        return (self._rk_step_1_kernel is rk.rk2_w_advection_step_1_kernel
                and self._rk_step_2_kernel is rk.rk2_w_advection_step_2_kernel
                and self._rk_update_kernel is rk.rk2_w_advection_update_kernel
                and self._pre_step_kernel in (None, validation_kernel)
                and self._post_step_kernel is None)

    def _stage_times(self, time):
        tidx1 = self.get_time_index(time)
        tidx2 = self.get_time_index(time + self._alpha * self.dt)
        nxt = time + self.dt
        tidx3 = self.get_time_index(nxt)
        return [tidx1, tidx2, tidx3], nxt

    def timestep_particles(self, particles, launcher: Launcher) -> None:
        """One RK2 step: one fused launch for the ROMS presets, else the reference's sequence."""
        if self.fused():
            self._fused_chunk(particles, launcher, 1)
        else:
            self._unfused_step(particles, launcher)

    def _unfused_step(self, particles, launcher: Launcher) -> None:
        """timesteppers.py:241-257."""
        _require_float64(launcher)
        if self._pre_step_kernel is not None:
            launcher.launch_kernel(self._pre_step_kernel, particles, self._tidx)
        launcher.launch_kernel(self._rk_step_1_kernel, particles, self._tidx)
        intermediate_time = self.time + self._alpha * self.dt
        intermediate_tidx = self.get_time_index(intermediate_time)
        launcher.launch_kernel(self._rk_step_2_kernel, particles, intermediate_tidx)
        self.advance_time()
        launcher.launch_kernel(self._rk_update_kernel, particles, self._tidx)
        if self._post_step_kernel is not None:
            launcher.launch_kernel(self._post_step_kernel, particles, self._tidx)

    def _launch_fused(self, particles, launcher, steps, needed, td, split=None, rec=None) -> None:
        rf, table = _fused_fields(launcher, steps, needed, td, len(particles))
        sc = _abi.scalars_struct({
            "hc": launcher.scalar("hc", self._tidx), "NZ": launcher.scalar("NZ", self._tidx),
            "_dt": self._normalised_dt, "_RK2_alpha": self._alpha,
            **{n: launcher.scalar(n, self._tidx) for n in ("zidx_min", "zidx_max", "yidx_min", "yidx_max",
                                                           "xidx_min", "xidx_max")}})
        table_ptr, _keep = _table_arg(table, particles.device, rf)
        _notify("before", len(steps))
        _fused_call(_entry("opb_rk2_w_advection_steps", launcher), particles, split,
                    (ctypes.byref(sc), ctypes.byref(rf), table_ptr, len(steps), int(self._pre_step_kernel is not None)),
                    _abi.stream(particles), rec)
        _notify("after", len(steps))
        if rec is not None:
            rec.replay(td)
        _prefetch_after(td, needed, self._prefetch_limit)


class ABTimestepper(Timestepper):
    """Adams-Bashforth stepping (timesteppers.py:260-305): pre, ab at t, advance, post at t + dt."""

    def __init__(self, time_array, dt, ab_kernel: ParticleKernel, *, time_unit=None, time=None, iteration: int = 0,
                 index_padding: int = 0, pre_step_kernel: ParticleKernel | None = None,
                 post_step_kernel: ParticleKernel | None = None) -> None:
        super().__init__(time_array, dt, time_unit=time_unit, time=time, index_padding=index_padding,
                         iteration=iteration)
        self._ab_kernel = ab_kernel
        self._pre_step_kernel = pre_step_kernel
        self._post_step_kernel = post_step_kernel

    @property
    def kernels(self) -> tuple[ParticleKernel, ...]:
        pre = (self._pre_step_kernel,) if self._pre_step_kernel is not None else ()
        post = (self._post_step_kernel,) if self._post_step_kernel is not None else ()
        return pre + (self._ab_kernel,) + post

    @property
    def isopycnal(self) -> bool:
        """True for the ROMS isopycnal-following kernels (models/roms/__init__.py:109-141)."""
        from .kernels.roms import ab3_isopycnal_following as iso

        return (self._ab_kernel is iso.ab3_isopycnal_following_kernel
                and self._post_step_kernel is iso.ab3_post_isopycnal_following_kernel)

    @property
    def field_roles(self) -> dict[str, str]:
        return {"w": "rho"} if self.isopycnal else {}

    def fused(self) -> bool:
        from .kernels.roms import ab3_w_advection as ab
        from .kernels.validation import validation_kernel

        stock = (self._ab_kernel is ab.ab3_w_advection_kernel
                 and self._post_step_kernel is ab.ab3_post_w_advection_kernel)
        return (stock or self.isopycnal) and self._pre_step_kernel in (None, validation_kernel)

    def _stage_times(self, time):
        tidx1 = self.get_time_index(time)
        nxt = time + self.dt
        tidx2 = self.get_time_index(nxt)
        return [tidx1, tidx2], nxt

    def timestep_particles(self, particles, launcher: Launcher) -> None:
        if self.fused():
            self._fused_chunk(particles, launcher, 1)
        else:
            self._unfused_step(particles, launcher)

    def _unfused_step(self, particles, launcher: Launcher) -> None:
        """timesteppers.py:296-305."""
        _require_float64(launcher)
        if self._pre_step_kernel is not None:
            launcher.launch_kernel(self._pre_step_kernel, particles, self._tidx)
        launcher.launch_kernel(self._ab_kernel, particles, self._tidx)
        self.advance_time()
        if self._post_step_kernel is not None:
            launcher.launch_kernel(self._post_step_kernel, particles, self._tidx)

    def _launch_fused(self, particles, launcher, steps, needed, td, split=None, rec=None) -> None:
        rf, table = _fused_fields(launcher, steps, needed, td, len(particles), self.field_roles)
        iso = self.isopycnal
        sc = _abi.scalars_struct({
            "hc": launcher.scalar("hc", self._tidx), "NZ": launcher.scalar("NZ", self._tidx),
            "_dt": self._normalised_dt,
            **{n: launcher.scalar(n, self._tidx) for n in ("zidx_min", "zidx_max", "yidx_min", "yidx_max",
                                                           "xidx_min", "xidx_max")},
            **({n: launcher.scalar(n, self._tidx) for n in ("w_max", "rho_scale")} if iso else {})})
        if iso and launcher.arithmetic != "float64":
            raise ValueError("the isopycnal follower has float64 steppers only")
        entry = "opb_ab3_isopycnal_following_steps" if iso else _entry("opb_ab3_w_advection_steps", launcher)
        table_ptr, _keep = _table_arg(table, particles.device, rf)
        _notify("before", len(steps))
        _fused_call(entry, particles, split,
                    (ctypes.byref(sc), ctypes.byref(rf), table_ptr, len(steps), int(self._pre_step_kernel is not None)),
                    _abi.stream(particles), rec)
        _notify("after", len(steps))
        if rec is not None:
            rec.replay(td)
        _prefetch_after(td, needed, self._prefetch_limit)
