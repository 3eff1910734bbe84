"""Batched release experiments: many releases advanced together on one device.

The reference runs one release per ``Simulation`` (simulation.py:27-229); a
study of many releases runs them one after another.  ``ReleaseBatch`` keeps
every release's particles in one device arena, one contiguous segment per
release, and advances all of them one snapshot interval at a time with ONE
persistent launch (``opb_batched_steps``):

* a per-experiment offset table (segment start and count, scheme, dt, alpha,
  step count, offset into a shared stage-time table) is written to pinned host
  memory and copied to the device before the launch;
* the launch (per scheme: work-item planning, work-counter reset, persistent
  kernel) is captured once as a CUDA graph per ring phase and replayed every
  interval (the snapshots of an interval sit in fixed ring slots and the
  tables in fixed device buffers, so only device contents change);
* a release's segment is Morton-sorted when it starts and every
  ``sort_interval`` intervals after that, in place (``opb_sort_segments``).

Each release advances exactly as its own ``Simulation`` with the same stock
ROMS stepper would have: its stage times come from the same float64 time
arithmetic (``Timestepper.get_time_index`` / ``advance_time``,
timesteppers.py:64-85,157-161), and the kernel runs the stage functions of
the fused steppers.  The results are therefore identical to running each
release alone.
"""

from __future__ import annotations

import bisect
import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, timesteppers
from .fields import TimeDependentField
from .fieldset import Fieldset
from .kernels import _abi
from .kernels.status import ParticleStatus
from .launcher import Launcher
from .particles import Particles
from .timesteppers import (ABTimestepper, RK2Timestepper, Timestepper, _time_dependent_fields, pair_fields,
                           pair_layout, window_fields)

TIME_DTYPE = np.dtype([("prev", "<i4"), ("next", "<i4"), ("ft", "<f8"), ("gt", "<f8")])
EXPERIMENT_DTYPE = np.dtype([("start", "<i8"), ("count", "<i8"), ("first_chunk", "<i8"), ("scheme", "<i4"),
                             ("nsteps", "<i4"), ("table_offset", "<i4"), ("validate", "<i4"), ("dt", "<f8"),
                             ("alpha", "<f8"), ("bucket_row", "<i4"), ("_pad", "<i4")])
HEADER_DTYPE = np.dtype([("nexp", "<i4"), ("nbuckets", "<i4"), ("nchunks", "<i8"), ("next_chunk", "<u8")])
assert TIME_DTYPE.itemsize == ctypes.sizeof(_lib.opb_time)
assert EXPERIMENT_DTYPE.itemsize == ctypes.sizeof(_lib.opb_experiment)
assert HEADER_DTYPE.itemsize == ctypes.sizeof(_lib.opb_batch_header)

ARENA_FIELDS = {"status": np.uint8, **{name: np.float64 for name in _lib.PARTICLE_POINTERS}}


def _align(n: int, a: int = 256) -> int:
    return (n + a - 1) // a * a


class TimeIndex:
    """``Timestepper.get_time_index`` (timesteppers.py:64-85) on Python floats.

    numpy float64 scalars and Python floats are both IEEE binary64 with
    round-to-nearest, and ``searchsorted(side="right")`` is ``bisect_right``,
    so the results are bit-identical; this form costs a fraction of a
    microsecond, which matters when thousands of stage times are planned per
    snapshot interval.
    """

    def __init__(self, time_array) -> None:
        self.times = [float(t) for t in np.asarray(time_array, dtype=np.float64)]

    def __call__(self, t: float) -> float:
        T = self.times
        if t < T[0] or t > T[-1]:
            raise ValueError("Time is out of bounds of the time array.")
        idx = bisect.bisect_right(T, t) - 1
        t0 = T[idx]
        t1 = T[idx + 1]  # IndexError at the last time, as numpy indexing raises in the reference
        return idx + (t - t0) / (t1 - t0)


def stage_times(r: "Release", time_index: TimeIndex, t: float) -> tuple[list[float], float]:
    """Stage time indices of one step of ``r`` from time ``t``, and the next time: ``_stage_times`` of
    RK2Timestepper / ABTimestepper (timesteppers.py:241-257, 296-305) in float form."""
    nxt = t + r.dt
    if r.scheme == _lib.SCHEME_RK2:
        return [time_index(t), time_index(t + r.adt), time_index(nxt)], nxt
    return [time_index(t), time_index(nxt)], nxt


class IntervalPlanner:
    """Splits every release's steps into snapshot intervals.

    Interval j holds the steps that START in [T_j, T_j+1); their stages read
    snapshots j, j+1 and j+2 (a step may end past T_j+1).  A release whose
    next step cannot be planned (past the last snapshot, or a dt longer than
    the snapshot spacing) stops before that step with ``error`` set; where the
    reference raises part-way through that step, the batch does not start it.
    """

    def __init__(self, time_array, num_snapshots: int) -> None:
        self.time_index = TimeIndex(time_array)
        self.T = self.time_index.times
        self.num_snapshots = int(num_snapshots)

    def plan(self, releases: list["Release"], j: int):
        """[(release index, release, steps, first table entry)], flat stage time indices; advances the
        releases' time and step count."""
        T = self.T
        Tn = T[j + 1]
        last = min(j + 2, self.num_snapshots - 1)
        ti = self.time_index
        exps = []
        tidx_all: list[float] = []
        for e, r in enumerate(releases):
            if r is None or r.finished or r.time >= Tn:
                continue
            if r.time < T[j]:
                raise RuntimeError(f"release {e} is at time {r.time}, before interval {j}")
            t = r.time
            k = 0
            first = len(tidx_all)
            while r.done + k < r.nsteps and t < Tn:
                try:
                    tidxs, nxt = stage_times(r, ti, t)
                except (ValueError, IndexError) as err:
                    r.error = err
                    break
                if any(int(x) < j or int(x) + 1 > last for x in tidxs):
                    r.error = IndexError(f"step at time {t} needs snapshots outside {j}..{last}: dt longer "
                                         "than the snapshot spacing, or past the last snapshot")
                    break
                tidx_all.extend(tidxs)
                t = nxt
                k += 1
            if k:
                exps.append((e, r, k, first))
                r.time = t
                r.done += k
        return exps, tidx_all


@dataclass
class Release:
    """One release experiment.

    ``timestepper``: a stock ROMS stepper (``models.roms`` presets), whose
    scheme, dt, alpha, validation pre-step and current time (the release time)
    the experiment uses.  ``nsteps``: steps to run.  ``zidx``/``yidx``/``xidx``:
    initial particle indices.  ``status``: initial status (default: MULTISTEP_1
    for AB3, NORMAL for RK2).
    """

    timestepper: Timestepper
    nsteps: int
    zidx: np.ndarray
    yidx: np.ndarray
    xidx: np.ndarray
    status: int | np.ndarray | None = None
    name: str | None = None
    # filled in by the batch
    records: list = field(default_factory=list, init=False, repr=False)  # (model time, Collected) rows
    start: int = field(default=-1, init=False)
    slot: int = field(default=-1, init=False)
    done: int = field(default=0, init=False)
    reported: bool = field(default=False, init=False)  # returned by ReleaseBatch.tick as finished
    error: BaseException | None = field(default=None, init=False)

    def __post_init__(self) -> None:
        ts = self.timestepper
        if not isinstance(ts, (RK2Timestepper, ABTimestepper)) or not ts.fused() or getattr(ts, "isopycnal", False):
            raise TypeError("a Release needs a stock ROMS RK2 or AB3 w-advection timestepper (models.roms presets)")
        if not isinstance(ts.time, (float, np.floating)):
            raise TypeError("batched releases use float64 times")
        if self.nsteps < 0:
            raise ValueError("nsteps must be non-negative")
        self.zidx = np.ascontiguousarray(self.zidx, dtype=np.float64)
        self.yidx = np.ascontiguousarray(self.yidx, dtype=np.float64)
        self.xidx = np.ascontiguousarray(self.xidx, dtype=np.float64)
        if not (self.zidx.shape == self.yidx.shape == self.xidx.shape) or self.zidx.ndim != 1:
            raise ValueError("zidx, yidx and xidx must be 1-D arrays of one length")
        self.scheme = _lib.SCHEME_AB3 if isinstance(ts, ABTimestepper) else _lib.SCHEME_RK2
        self.dt = float(ts._normalised_dt * ts.time_unit)
        self.alpha = float(ts.alpha) if self.scheme == _lib.SCHEME_RK2 else 0.0
        self.adt = float(ts.alpha * ts.dt) if self.scheme == _lib.SCHEME_RK2 else 0.0
        self.validate = int(ts._pre_step_kernel is not None)
        self.time = float(ts.time)
        if self.status is None:
            self.status = ParticleStatus.MULTISTEP_1 if self.scheme == _lib.SCHEME_AB3 else ParticleStatus.NORMAL

    def __len__(self) -> int:
        return self.zidx.shape[0]

    @property
    def finished(self) -> bool:
        return self.done >= self.nsteps or self.error is not None

    @property
    def particle_steps(self) -> int:
        return len(self) * self.nsteps

    def trajectory(self) -> dict[str, np.ndarray]:
        """The recorded rows (``ReleaseBatch(record_every=...)``): ``time`` (rounds,) and each recorded
        field (rounds, particles) in the release's original particle order."""
        if not self.records:
            return {"time": np.zeros(0)}
        rows = [c.result() for _, c in self.records]
        out = {"time": np.array([t for t, _ in self.records])}
        for k in rows[0]:
            out[k] = np.stack([r[k] for r in rows])
        return out


class SegmentAllocator:
    """First-fit allocation of contiguous particle ranges in an arena of ``capacity`` slots."""

    def __init__(self, capacity: int) -> None:
        self.capacity = int(capacity)
        self.free_list: list[tuple[int, int]] = [(0, self.capacity)] if capacity > 0 else []  # (start, length)

    def alloc(self, n: int) -> int | None:
        if n <= 0:
            return None
        for q, (s, ln) in enumerate(self.free_list):
            if ln >= n:
                if ln == n:
                    self.free_list.pop(q)
                else:
                    self.free_list[q] = (s + n, ln - n)
                return s
        return None

    def free(self, start: int, n: int) -> None:
        if n <= 0:
            return
        bisect.insort(self.free_list, (start, n))
        merged: list[tuple[int, int]] = []
        for s, ln in self.free_list:
            if merged and merged[-1][0] + merged[-1][1] == s:
                merged[-1] = (merged[-1][0], merged[-1][1] + ln)
            else:
                merged.append((s, ln))
        self.free_list = merged

    @property
    def free_total(self) -> int:
        return sum(ln for _, ln in self.free_list)

    @property
    def largest_free(self) -> int:
        return max((ln for _, ln in self.free_list), default=0)


class Collected:
    """A release's particle fields on their way to pinned host memory (``ReleaseBatch.collect``)."""

    def __init__(self, release: Release, host: dict[str, torch.Tensor], event: torch.cuda.Event) -> None:
        self.release = release
        self._host = host
        self._event = event

    def ready(self) -> bool:
        return self._event.query()

    def result(self) -> dict[str, np.ndarray]:
        self._event.synchronize()
        return {k: v.numpy() for k, v in self._host.items()}


class ReleaseBatch:
    """Advance many ``Release`` experiments together on one device.

    Static use: ``ReleaseBatch(fieldset, releases).run()``.  Dynamic use (a
    request server): ``ReleaseBatch(fieldset, time_array=..., capacity=N,
    max_releases=R)``, then ``add`` releases at interval boundaries, ``tick``
    one snapshot interval at a time, and ``collect`` / ``retire`` releases that
    have finished.  Every release lives in its own contiguous segment of a
    particle arena of ``capacity`` slots (first-fit); its state stays on the
    device from ``add`` to ``retire``.

    ``fieldset``: the shared fields (u, v, w, zeta time-dependent; h, dx, dy, C
    static).  ``block``, ``warps_per_sm``: the persistent launch's CTA size
    and resident warps per SM (register budget per thread 65536 / 32 /
    warps_per_sm), one of ``_lib.BATCH_SHAPES``.  ``ctas``: CTAs of the launch
    (0: as many as stay resident).  ``split_schemes``: one launch per scheme,
    each kernel compiled for RK2 or AB3 alone (less code, fewer registers),
    instead of one kernel for both.
    ``sort_interval``: snapshot intervals between re-sorts of a release's
    segment (0: never; a release is always sorted when it starts).
    ``graphs``: capture each interval's launches as a CUDA graph (only when
    every time-dependent field streams through a ring, whose slot addresses
    repeat).  ``buckets``: 0 walks one release's segment after another; a
    power of two walks that many Morton buckets of the grid in turn, advancing
    the particles of every release in a bucket together, so that releases
    sharing a region share its field data in L2.  The launches read the
    time-dependent fields as snapshot pairs (two consecutive snapshots
    interleaved element by element), one load per stencil corner.
    ``record_every``: every that many snapshot intervals (at the interval
    boundaries the launches replay on, so output never splits a launch),
    copy ``record_fields`` of every running release to pinned host memory,
    asynchronously; ``Release.trajectory()`` returns the rows.
    """

    def __init__(self, fieldset: Fieldset, releases: list[Release] = (), *, time_array=None,
                 capacity: int | None = None, max_releases: int | None = None, device=None, block: int = 256,
                 warps_per_sm: int = 16, ctas: int = 0, sort_interval: int = 4, graphs: bool = True,
                 buckets: int = 256, split_schemes: bool = True, record_every: int = 0,
                 record_fields=("zidx", "yidx", "xidx", "status")) -> None:
        if record_every < 0:
            raise ValueError("record_every must be non-negative")
        self.record_every = int(record_every)
        self.record_fields = tuple(record_fields)
        if buckets < 0 or (buckets & (buckets - 1)) or buckets > 65536:
            raise ValueError("buckets must be 0 or a power of two up to 65536")
        self.buckets = int(buckets)
        if (block, warps_per_sm) not in _lib.BATCH_SHAPES:
            raise ValueError(f"(block, warps_per_sm) must be one of {_lib.BATCH_SHAPES}")
        if not split_schemes and warps_per_sm != 16:
            raise ValueError("one kernel for both schemes runs at 16 warps per SM only")
        self.warps_per_sm = int(warps_per_sm)
        # one launch per scheme (each kernel compiled for its scheme alone), or one for both
        self.groups = (_lib.SCHEME_RK2, _lib.SCHEME_AB3) if split_schemes else (0,)
        self.fieldset = fieldset
        releases = list(releases)
        self.launcher = Launcher(fieldset)
        self.block = int(block)
        self.ctas = int(ctas)
        self.sort_interval = int(sort_interval)
        self._td = _time_dependent_fields(self.launcher)
        if not self._td:
            raise ValueError("the fieldset has no time-dependent fields")
        nts = {f.num_timesteps for f in self._td.values()}
        if len(nts) != 1:
            raise ValueError("time-dependent fields must have the same number of snapshots")
        self.num_snapshots = nts.pop()
        if time_array is None:
            if not releases:
                raise ValueError("give releases or a time_array")
            time_array = releases[0].timestepper.time_array
        self.time_array = np.asarray(time_array, dtype=np.float64)
        if self.time_array.shape[0] > self.num_snapshots:
            raise ValueError("the time array has more entries than the fields have snapshots")
        self.planner = IntervalPlanner(self.time_array, self.num_snapshots)
        self._T = self.planner.T
        self.graphs = bool(graphs) and all(f.streamed for f in self._td.values())
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.capacity = int(capacity) if capacity is not None else sum(len(r) for r in releases)
        self.max_releases = int(max_releases) if max_releases is not None else max(len(releases), 1)
        self.slots: list[Release | None] = [None] * self.max_releases
        self.allocator = SegmentAllocator(self.capacity)
        self.interval = None  # index j of the next snapshot interval to run
        self.arena = Particles(self.capacity, device=self.device, **ARENA_FIELDS)
        # original arena slot of each storage slot: segments keep their ranges, so a particle's index
        # within its release is order - start
        self.order = torch.arange(self.capacity, dtype=torch.int64, device=self.device)
        min_dt = min((r.dt for r in releases), default=60.0)
        self._init_tables(min_dt)
        self._graphs: dict = {}
        self._sorted_at: dict[int, int] = {}
        self._sort_ws = None
        self.launches = 0
        self.sorts = 0
        self.retired_particle_steps = 0
        # per launched interval: (interval, experiments, particle-steps, most steps of one experiment)
        self.stats: list[tuple[int, int, int, int]] = []
        # objects with before() / after(), called around each interval's launch (timing)
        self.observers: list = []
        for r in releases:
            if not self.add(r):
                raise ValueError("the releases do not fit the arena")

    @property
    def releases(self) -> list[Release]:
        """Releases currently in the batch (slot order)."""
        return [r for r in self.slots if r is not None]

    # ------------------------------------------------------------------ arena
    @staticmethod
    def bytes_per_particle() -> int:
        """Arena bytes per particle slot: status, positions, z, the RK2 stage / AB3 three-step velocity
        history (float64 each), and the original-order index."""
        return 1 + 8 * len(_lib.PARTICLE_POINTERS) + 8

    def add(self, r: Release) -> bool:
        """Place a release in a free slot and segment and upload its initial state; False if it does not fit."""
        if r.slot >= 0:
            raise ValueError("the release is already in a batch")
        ta = np.asarray(r.timestepper.time_array, dtype=np.float64)
        if ta.shape != self.time_array.shape or not np.array_equal(ta, self.time_array):
            raise ValueError("every release must use the batch's time array")
        if self.interval is not None and r.time < self._T[self.interval]:
            raise ValueError(f"release time {r.time} is before the batch's current interval")
        try:
            slot = self.slots.index(None)
        except ValueError:
            return False
        n = len(r)
        start = self.allocator.alloc(n)
        if start is None:
            return False
        r.start, r.slot = start, slot
        self.slots[slot] = r
        self._sorted_at.pop(slot, None)
        A = self.arena.arrays
        sl = slice(start, start + n)
        # pinned sources: a pageable one would make each copy wait for the stream to drain
        for name, arr in (("zidx", r.zidx), ("yidx", r.yidx), ("xidx", r.xidx)):
            A[name][sl].copy_(torch.from_numpy(arr).pin_memory(), non_blocking=True)
        for name in _lib.PARTICLE_POINTERS[3:]:
            A[name][sl].zero_()
        st = r.status
        if isinstance(st, (int, np.integer)):
            A["status"][sl].fill_(int(st))
        else:
            A["status"][sl].copy_(torch.from_numpy(np.ascontiguousarray(st, dtype=np.uint8)).pin_memory(),
                                  non_blocking=True)
        self.order[sl].copy_(torch.arange(start, start + n, dtype=torch.int64, device=self.device))
        return True

    def collect(self, r: Release, names=("zidx", "yidx", "xidx", "status")) -> Collected:
        """Start copying a release's fields, in its original particle order, to pinned host memory."""
        if r.slot < 0 or self.slots[r.slot] is not r:
            raise ValueError("the release is not in this batch")
        sl = slice(r.start, r.start + len(r))
        pos = self.order[sl] - r.start
        host = {}
        for name in names:
            key = name if name in self.arena else "_" + name
            t = self.arena.arrays[key][sl]
            o = torch.empty_like(t)
            o.index_copy_(0, pos, t)
            h = torch.empty(o.shape, dtype=o.dtype, pin_memory=True)
            h.copy_(o, non_blocking=True)
            host[name] = h
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        return Collected(r, host, ev)

    def retire(self, r: Release) -> None:
        """Free a release's slot and segment.  Later uploads into the segment are queued on the same
        stream, so they stay ordered after the work that reads it."""
        if r.slot < 0 or self.slots[r.slot] is not r:
            raise ValueError("the release is not in this batch")
        self.retired_particle_steps += len(r) * r.done
        self.allocator.free(r.start, len(r))
        self.slots[r.slot] = None
        self._sorted_at.pop(r.slot, None)
        r.slot = -1

    def _init_tables(self, min_dt: float) -> None:
        # capacity: at most ceil(interval / dt) + 2 steps per release per interval, 3 entries per RK2 step
        dT = float(np.min(np.diff(self.time_array))) if len(self.time_array) > 1 else 1.0
        self.max_entries = 3 * (int(math.ceil(dT / min_dt)) + 2) * self.max_releases
        self._layout()

    def _layout(self) -> None:
        # one header and one experiment list per launch group, then the shared stage-time table
        ng = len(self.groups)
        self._off_hdr = [g * _align(HEADER_DTYPE.itemsize) for g in range(ng)]
        base = ng * _align(HEADER_DTYPE.itemsize)
        exp_bytes = _align(self.max_releases * EXPERIMENT_DTYPE.itemsize)
        self._off_exps = [base + g * exp_bytes for g in range(ng)]
        self._off_tab = base + ng * exp_bytes
        self._nbytes = self._off_tab + _align(self.max_entries * TIME_DTYPE.itemsize)
        # two pinned staging buffers and two device copies, used alternately
        self._host = [torch.zeros(self._nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        self._dev = [torch.zeros(self._nbytes, dtype=torch.uint8, device=self.device) for _ in range(2)]
        self._host_free: list[torch.cuda.Event | None] = [None, None]
        self._parity = 0
        self._scalars = None
        # per slot: where each Morton bucket starts in its segment (written by every segment sort)
        nb = max(self.buckets, 1)
        self._bounds = torch.zeros((self.max_releases, nb + 1), dtype=torch.int64, device=self.device)
        self._items = torch.zeros((len(self.groups), self.max_releases * nb + 1), dtype=torch.int64,
                                  device=self.device)
        self._graphs = {}

    def _grow_table(self, entries: int) -> None:
        """Stage-time table too small for this interval (a shorter dt than planned for): double it."""
        torch.cuda.current_stream(self.device).synchronize()
        while self.max_entries < entries:
            self.max_entries *= 2
        bounds = self._bounds
        self._layout()
        self._bounds.copy_(bounds)

    # ------------------------------------------------------------- snapshot pairs
    def _pair_fields(self, j: int, window: list[int], rf) -> None:
        """Point the time-dependent fields of ``rf`` at snapshot pairs j and j + 1 (slots 0 and 1;
        ``TimeDependentField.pair``): the kernel fetches both values of a corner's time blend with one
        load (quads or octets with float32 storage: two or four corners per load).  Pair j + 1 exists only when
        snapshot j + 2 is in the window."""
        its = [j, j + 1] if j + 2 <= window[-1] else [j]
        pair_fields(rf, its, self._td, pair_layout(self.launcher, self._td, layout=timesteppers.BATCH_LAYOUT))

    # --------------------------------------------------------------- planning
    def _plan(self, j: int):
        return self.planner.plan(self.slots, j)

    def _write_tables(self, j: int, exps, tidx_all, dtype) -> int:
        """Fill a pinned staging buffer (per launch group: header and experiments; the stage-time table);
        return its parity."""
        if len(tidx_all) > self.max_entries:
            self._grow_table(len(tidx_all))
        b = self._parity
        self._parity ^= 1
        ev = self._host_free[b]
        if ev is not None:
            ev.synchronize()  # the upload that last read this staging buffer has finished
        host = self._host[b].numpy()
        chunk = _lib.BATCH_CHUNK
        for g, scheme in enumerate(self.groups):
            mine = [x for x in exps if scheme == 0 or x[1].scheme == scheme]
            hdr = host[self._off_hdr[g]:self._off_hdr[g] + HEADER_DTYPE.itemsize].view(HEADER_DTYPE)
            off = self._off_exps[g]
            ex = host[off:off + len(mine) * EXPERIMENT_DTYPE.itemsize].view(EXPERIMENT_DTYPE)
            nchunks = 0
            for q, (e, r, k, first) in enumerate(mine):
                ex[q] = (r.start, len(r), nchunks, r.scheme, k, first, r.validate, r.dt, r.alpha, e, 0)
                nchunks += (len(r) + chunk - 1) // chunk
            hdr[0] = (len(mine), self.buckets, nchunks, 0)
        if tidx_all:
            tid = np.asarray(tidx_all, dtype=np.float64)
            It, fr = np.divmod(tid, 1.0)
            It = It.astype(np.int64)
            ft = fr.astype(dtype)
            gt = dtype.type(1) - ft
            # the device reads these tables unchecked: every pair slot must exist (0, and 1 only when
            # snapshot j + 2 is in the window) and every experiment's entries must lie in the table
            npairs = 2 if j + 2 <= min(j + 2, self.num_snapshots - 1) else 1
            if int((It - j).min()) < 0 or int((It - j).max()) >= npairs:
                raise RuntimeError(f"interval {j}: a stage reads a snapshot pair outside the window")
            for e, r, k, first in exps:
                if first < 0 or first + k * (3 if r.scheme == _lib.SCHEME_RK2 else 2) > len(tidx_all):
                    raise RuntimeError(f"interval {j}: release {e}'s stage entries run past the table")
            tab = host[self._off_tab:self._off_tab + len(tidx_all) * TIME_DTYPE.itemsize].view(TIME_DTYPE)
            tab["prev"] = It - j  # pair slot: 0 = snapshots j, j+1; 1 = snapshots j+1, j+2
            tab["next"] = It - j
            tab["ft"] = ft.astype(np.float64)
            tab["gt"] = gt.astype(np.float64)
        return b

    # --------------------------------------------------------------- stepping
    @property
    def finished(self) -> bool:
        return all(r.finished for r in self.releases)

    def _first_interval(self) -> int:
        times = [r.time for r in self.releases if not r.finished]
        t0 = min(times) if times else self._T[0]
        return max(0, bisect.bisect_right(self._T, t0) - 1)

    def _scalars_struct(self):
        if self._scalars is None:
            L = self.launcher
            self._scalars = _abi.scalars_struct({
                "hc": L.scalar("hc", 0.0), "NZ": L.scalar("NZ", 0.0), "_dt": 0.0, "_RK2_alpha": 0.0,
                **{n: L.scalar(n, 0.0) for n in ("zidx_min", "zidx_max", "yidx_min", "yidx_max", "xidx_min",
                                                 "xidx_max")}})
        return self._scalars

    def _sort_due(self, j: int, exps) -> None:
        if not exps:
            return
        due = []
        for e, r, k, first in exps:
            last = self._sorted_at.get(e)
            if last is None or (self.sort_interval > 0 and j - last >= self.sort_interval):
                due.append((e, r))
                self._sorted_at[e] = j
        if not due:
            return
        due.sort(key=lambda er: er[1].start)
        rows = [e for e, _ in due]
        due = [r for _, r in due]
        starts = (ctypes.c_int64 * len(due))(*[r.start for r in due])
        counts = (ctypes.c_int64 * len(due))(*[len(r) for r in due])
        total = sum(len(r) for r in due)
        lib = _lib.load()
        need = int(lib.opb_sort_segments_workspace_bytes(total, len(due)))
        if self._sort_ws is None or self._sort_ws.numel() < need:
            self._sort_ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        fs = self.fieldset
        dims = (ctypes.c_int64 * 3)(fs.z_size, fs.y_size, fs.x_size)
        nb = max(self.buckets, 1)
        out = torch.empty((len(due), nb + 1), dtype=torch.int64, device=self.device)
        _lib.call("opb_sort_segments", ctypes.byref(_abi.particles_struct(self.arena)), ctypes.byref(dims), starts,
                  counts, len(due), self.order.data_ptr(), nb, out.data_ptr(), self._sort_ws.data_ptr(),
                  self._sort_ws.numel(), _abi.stream(self.arena))
        # pinned source: a pageable one would make the copy wait for the stream to drain
        rows_dev = torch.tensor(rows, dtype=torch.int64).pin_memory().to(self.device, non_blocking=True)
        self._bounds.index_copy_(0, rows_dev, out)
        self.sorts += 1

    def _upload(self, b: int, nbytes: int) -> None:
        """Copy the used part of staging buffer b to its device copy (outside any graph: the size varies)."""
        self._dev[b][:nbytes].copy_(self._host[b][:nbytes], non_blocking=True)

    def _launch(self, rf, b: int) -> None:
        base = self._dev[b].data_ptr()
        for g, scheme in enumerate(self.groups):
            _lib.call("opb_batched_steps", ctypes.byref(_abi.particles_struct(self.arena)), base + self._off_hdr[g],
                      base + self._off_exps[g], ctypes.byref(self._scalars_struct()), ctypes.byref(rf),
                      base + self._off_tab, self._bounds.data_ptr(), self._items[g].data_ptr(), scheme, self.block,
                      self.warps_per_sm, self.ctas, _abi.stream(self.arena))

    def _run_launch(self, rf, b: int) -> None:
        if not self.graphs:
            self._launch(rf, b)
            return
        key = (bytes(rf), b)
        g = self._graphs.get(key)
        if g is None:
            if len(self._graphs) >= 32:
                self._graphs.clear()
            # one eager launch first (loads the module, queries occupancy), then capture
            self._launch(rf, b)
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream(device=self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):
                g.capture_begin(capture_error_mode="thread_local")
                self._launch(rf, b)
                g.capture_end()
            torch.cuda.current_stream(self.device).wait_stream(side)
            self._graphs[key] = g
            return  # the eager launch did this interval's work; the capture itself ran nothing
        g.replay()

    def _report(self) -> list[Release]:
        done = [r for r in self.releases if r.finished and not r.reported]
        for r in done:
            r.reported = True
        return done

    def tick(self) -> list[Release]:
        """Run snapshot interval ``interval`` for every release with steps in it, then move to the next
        interval; return the releases that finished (all steps done, or stopped with an error) and were
        not returned before."""
        if self.interval is None:
            self.interval = self._first_interval()
        j = self.interval
        if j + 1 >= len(self._T):
            for r in self.releases:
                if not r.finished:
                    r.error = IndexError("no snapshot interval left")
            return self._report()
        exps, tidx_all = self._plan(j)
        self.interval = j + 1
        if exps:
            torch.cuda.nvtx.range_push(f"opb interval {j}: {len(exps)} releases")
            window = list(range(j, min(j + 3, self.num_snapshots)))
            rf, dtype = window_fields(self.launcher, window, self._td)
            self._pair_fields(j, window, rf)
            b = self._write_tables(j, exps, tidx_all, dtype)
            self._sort_due(j, exps)
            for obs in self.observers:
                obs.before()
            self._upload(b, self._off_tab + len(tidx_all) * TIME_DTYPE.itemsize)
            self._run_launch(rf, b)
            for obs in self.observers:
                obs.after()
            self.stats.append((j, len(exps), sum(len(r) * k for _, r, k, _ in exps), max(k for _, _, k, _ in exps)))
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream(self.device))
            self._host_free[b] = ev
            self.launches += 1
            for f in self._td.values():
                f.mark_used(window)
                f.prefetch(j + 3, set(window[1:]))
            torch.cuda.nvtx.range_pop()
        if self.record_every and (j + 1) % self.record_every == 0:
            for r in self.releases:
                if r.done and (r.done < r.nsteps or not r.reported) and r.error is None:
                    if r.records and r.records[-1][0] == r.time:
                        continue  # already recorded at this model time
                    r.records.append((r.time, self.collect(r, self.record_fields)))
        return self._report()

    def step_interval(self) -> bool:
        """Run one snapshot interval; False once every release is done."""
        if self.finished:
            return False
        self.tick()
        return not self.finished

    def run(self) -> None:
        """Run every release to its end."""
        while self.step_interval():
            pass

    def synchronize(self) -> None:
        torch.cuda.synchronize(self.device)
        self.arena.check_errors()

    # ---------------------------------------------------------------- results
    def result(self, r: Release | int, names=("zidx", "yidx", "xidx", "status")) -> dict[str, np.ndarray]:
        """Host copies of a release's particle fields in its original particle order."""
        if isinstance(r, int):
            r = self.releases[r]
        self.arena.check_errors()
        return self.collect(r, names).result()

    @property
    def particle_steps(self) -> int:
        """Particle-steps planned so far (particles x steps), retired releases included."""
        return self.retired_particle_steps + sum(len(r) * r.done for r in self.releases)
