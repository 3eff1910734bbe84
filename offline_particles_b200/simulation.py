"""Simulation and SimulationBuilder (simulation.py:1-367 of the reference).

Same construction and stepping API.  Particle state lives on the device;
``particles`` returns read-only host copies, ``run(n)`` advances many steps
with fused multi-step launches between events, and ``synchronize()`` waits
for the device and raises any error the kernels recorded (a zero grid
spacing raises ``ZeroDivisionError``, as in the reference).
"""

from __future__ import annotations

import itertools
import types
from typing import Mapping

import numpy as np
import torch

from .events import Event, IterationScheduler, SimulationState, TimeScheduler
from .fieldset import Fieldset
from .kernels import merge_particle_fields
from .launcher import Launcher
from .particles import Particles, ParticlesView
from .timesteppers import Timestepper

# steps between spatial re-sorts of particle storage (particles drift ~0.03 cells per step at
# 0.5 m/s, dx = 2 km, dt = 120 s, so locality decays slowly)
DEFAULT_SORT_INTERVAL = 64


class Simulation:
    """A particle simulation on one CUDA device."""

    def __init__(self, nparticles: int, timestepper: Timestepper, fieldset: Fieldset,
                 iteration_scheduler: IterationScheduler, time_scheduler: TimeScheduler,
                 output_writers: Mapping[str, object] | None = None, *, device=None,
                 sort_interval: int = DEFAULT_SORT_INTERVAL, arithmetic: str = "float64",
                 result_ranges: int = 1) -> None:
        """``sort_interval``: reorder particle storage by cell every that many steps (0: never).
        ``arithmetic``: "float64" (bit-identical to the reference) or "float32" (the reduced-precision
        fused steppers, which also take bfloat16/float16 field storage).  ``result_ranges`` (1 to 4): keep
        particle storage in that many ranges of original ids, each sorted on its own, so that
        ``run(..., results=...)`` copies each range's results to the host while the next range computes
        (``result_bounds``)."""
        if not 1 <= int(result_ranges) <= 4:
            raise ValueError("result_ranges must be between 1 and 4")
        self._timestepper = timestepper
        self._fieldset = fieldset
        self._iteration_scheduler = iteration_scheduler
        self._time_scheduler = time_scheduler
        self._output_writers = output_writers or {}
        self._launcher = Launcher(fieldset, arithmetic=arithmetic)
        self._launcher.maybe_increase_index_padding(timestepper.index_padding)
        self._launcher.register_scalar_data_sources_from_object(self._timestepper)
        for event in itertools.chain(self._iteration_scheduler.events, self._time_scheduler.events):
            self._launcher.register_scalar_data_sources_from_object(event)
        kernels = list(self._timestepper.kernels)
        for event in itertools.chain(self._iteration_scheduler.events, self._time_scheduler.events):
            kernels.extend(event.kernels)
        particle_fields = merge_particle_fields(kernels)
        self._particles = Particles(nparticles, device=device, **particle_fields)
        self._particles_view = ParticlesView(self._particles)
        self._sort_interval = int(sort_interval)
        n = len(self._particles)
        self._id_bounds = result_bounds(n, int(result_ranges))
        self._readback: dict[str, torch.Tensor] = {}  # device buffers of run(results=...), by field
        self._readback_stream: torch.cuda.Stream | None = None
        self._records: dict[str, torch.Tensor] | None = None  # states recorded inside fused launches
        self._steps_since_sort: int | None = None  # None: never sorted
        if self._sort_interval > 0:
            self._particles.reserve_sort()  # the sort's scratch now, not inside the first run
        self._timestepper.reserve_launch_buffers(self._launcher, len(self._particles))
        self._invoke_events()

    @property
    def timestepper(self) -> Timestepper:
        return self._timestepper

    @property
    def fieldset(self) -> Fieldset:
        return self._fieldset

    @property
    def launcher(self) -> Launcher:
        return self._launcher

    @property
    def time(self):
        return self._timestepper.time

    @property
    def iteration(self) -> int:
        return self._timestepper.iteration

    @property
    def dt(self):
        return self._timestepper.dt

    @property
    def tidx(self) -> np.float64:
        return self._timestepper.tidx

    @property
    def particles(self) -> ParticlesView:
        return self._particles_view

    @property
    def device_particles(self) -> Particles:
        """The device particle arrays (mutable; what the kernels write)."""
        return self._particles

    @property
    def iteration_scheduler(self) -> IterationScheduler:
        return self._iteration_scheduler

    @property
    def time_scheduler(self) -> TimeScheduler:
        return self._time_scheduler

    @property
    def state(self) -> SimulationState:
        return SimulationState(time=self.time, dt=self.dt, tidx=self.tidx, iteration=self.iteration,
                               particles=self._particles_view)

    def _invoke_events(self) -> int:
        """Fire the events due now; return how many fired."""
        fired = 0
        for event in itertools.chain(self._iteration_scheduler(self.iteration), self._time_scheduler(self.time)):
            for kernel in event.kernels:
                self._launcher.launch_kernel(kernel, self._particles, self.tidx)
            event(self.state)
            fired += 1
        return fired

    def _prefetch_next_step(self) -> None:
        """Start uploading the snapshots the next step reads (the two around the current time) to every
        streamed field's device ring, snapshot by snapshot across fields, so that they stream in while the
        caller's particle arrays are copied in and sorted."""
        from .timesteppers import _time_dependent_fields

        td = [f for f in _time_dependent_fields(self._launcher, self._timestepper.field_roles).values()
              if f.streamed]
        if not td:
            return
        it = int(divmod(self._timestepper.tidx, 1)[0])
        keep = {it, it + 1}
        for k in (it, it + 1):
            for f in td:
                if k < f.num_timesteps:
                    f.prefetch(k, keep)

    def set_indices(self, zidx=None, yidx=None, xidx=None) -> None:
        """Set the particle indices (broadcast to the particle count; validated before any write).  Then
        the snapshots of the next step start uploading, behind the indices, so that they stream in while
        the particles are sorted."""
        P = self._particles
        vals, direct = {}, {}
        for name, v in (("zidx", zidx), ("yidx", yidx), ("xidx", xidx)):
            if v is None:
                continue
            target = P[name]
            if (isinstance(v, torch.Tensor) and not v.is_cuda and v.is_pinned() and v.dtype == target.dtype
                    and tuple(v.shape) == tuple(target.shape) and v.is_contiguous() and P.order is None):
                direct[name] = v  # pinned, in storage order already: one asynchronous copy into place
            else:
                vals[name] = self._as_device(v, target)
        for name, v in direct.items():
            P[name].copy_(v, non_blocking=True)
        for name, t in vals.items():
            P.assign(name, t)
        self._steps_since_sort = None
        copied = None
        if direct:
            copied = torch.cuda.Event()
            copied.record(torch.cuda.current_stream(P.device))
        self._prefetch_next_step()
        if copied is not None:
            copied.synchronize()  # the caller's host arrays may be reused once this returns

    def set_particle_field(self, field_name: str, values) -> None:
        """Set one particle field to ``values`` (cast to the field's dtype, broadcast)."""
        target = self._particles[field_name]
        self._particles.assign(field_name, self._as_device(values, target))

    @staticmethod
    def _as_device(values, target: torch.Tensor) -> torch.Tensor:
        if isinstance(values, torch.Tensor):
            t = values.to(device=target.device, dtype=target.dtype)
        else:
            from ._device import numpy_dtype

            arr = np.asarray(values, dtype=numpy_dtype(target.dtype))
            if arr.ndim == 0:
                # one value for every particle: filled on the device, no host-to-device copy (which would
                # queue behind snapshot uploads already in flight)
                return torch.full(tuple(target.shape), arr.item(), dtype=target.dtype, device=target.device)
            arr = np.broadcast_to(arr, tuple(target.shape))
            t = torch.from_numpy(np.array(arr, copy=True, order="C")).to(target.device)
        return t.expand(target.shape)

    @property
    def sort_interval(self) -> int:
        return self._sort_interval

    def sort_particles(self) -> None:
        """Reorder particle storage by cell now (results are unchanged; locality improves)."""
        fs = self._fieldset
        self._particles.sort((fs.z_size, fs.y_size, fs.x_size), id_bounds=self._id_bounds)
        self._steps_since_sort = 0

    def _maybe_sort(self) -> int:
        """Sort if due; return how many steps may run before the next sort.  A sort falls due
        ``sort_interval`` steps after the last one and is made at the next snapshot-interval boundary from
        then on, where a fused launch starts a new snapshot pair anyway: sorting never splits a launch, and
        the per-interval work (pair builds, sorts) happens at one point."""
        if self._sort_interval <= 0:
            return 1 << 30
        ts = self._timestepper
        if self._steps_since_sort is None or (self._steps_since_sort >= self._sort_interval
                                              and ts.at_interval_start):
            self.sort_particles()
        return ts.steps_to_interval_end(self._sort_interval - self._steps_since_sort)

    def step(self) -> None:
        """Advance the simulation by one timestep, then run any scheduled events."""
        self._maybe_sort()
        self._timestepper.timestep_particles(self._particles, self._launcher)
        if self._steps_since_sort is not None:
            self._steps_since_sort += 1
        self._invoke_events()

    def steps_to_next_event(self, limit: int) -> int:
        """How many steps can run before an event may fire (at most ``limit``)."""
        n = limit
        nxt = self._iteration_scheduler.next
        if nxt is not None:
            n = min(n, max(1, nxt - self.iteration))
        nt = self._time_scheduler.next_time
        if nt is not None:
            t = self.time
            k = 0
            while k < n:
                t = t + self.dt
                k += 1
                if t >= nt:
                    break
            n = min(n, max(1, k))
        return n

    def run(self, nsteps: int, *, results: Mapping[str, torch.Tensor] | None = None) -> None:
        """Advance ``nsteps`` steps: fused multi-step launches between event firings.  Snapshots are
        prefetched up to the last one these steps read (no uploads past the run's end).

        ``results``: particle field name -> host tensor (CPU, pinned for an asynchronous copy) of the
        particle count and the field's dtype, filled with the field in original particle order as it
        stands after the run.  The copies are queued, not waited for: read the tensors after
        ``synchronize()``.  With ``result_ranges`` > 1 the last fused launch runs range by range and each
        range's copies start as soon as its launch is done, behind the next range's compute."""
        reader = _ResultReader(self, results) if results is not None else None
        ts = self._timestepper
        ts._prefetch_limit = ts.snapshot_horizon(nsteps)
        ok = False
        try:
            self._run(nsteps, reader)
            ok = True
        finally:
            ts._prefetch_limit = None
            if reader is not None:
                reader.finish(read=ok)

    def _record_buffers(self, count: int) -> dict[str, torch.Tensor]:
        """Device buffers for ``count`` recorded states (grown on demand, reused by later launches in stream
        order)."""
        bufs = self._records
        n = len(self._particles)
        if bufs is None or bufs["zidx"].shape[0] < count:
            dev = self._particles.device
            bufs = {name: torch.empty((count, n), dtype=torch.uint8 if name == "status" else torch.float64, device=dev)
                    for name in _RECORDED}
            self._records = bufs
        return bufs

    def reserve_results(self, names) -> None:
        """Allocate what ``run(results=...)`` uses for the fields ``names`` (device buffers in original
        order, a copy stream) now, so that such a run allocates nothing."""
        P = self._particles
        if self._readback_stream is None:
            self._readback_stream = torch.cuda.Stream(device=P.device, priority=-1)
        with torch.cuda.stream(self._readback_stream):
            for name in names:
                t = P[name]
                buf = self._readback.get(name)
                if buf is None or buf.shape != t.shape or buf.dtype != t.dtype:
                    self._readback[name] = torch.empty_like(t)

    def _recordable(self) -> bool:
        """Events may fire after a fused launch on the state it recorded (float64 fused steppers)."""
        return self._timestepper.fused() and self._launcher.arithmetic == "float64"

    def plan_events(self, limit: int) -> tuple[int, set[int]]:
        """How many steps (at most ``limit``) can run before an event that must fire between launches, and
        the iterations before that whose events are all deferrable (recorded inside the launches and fired
        after them, in step order).  The schedulers are looked ahead on copies."""
        if not self._recordable():
            return self.steps_to_next_event(limit), set()
        if self._iteration_scheduler.next is None and self._time_scheduler.next_time is None:
            return limit, set()
        its, tms = self._iteration_scheduler.copy(), self._time_scheduler.copy()
        forward = tms._forward
        it, t, dt = self.iteration, self.time, self.dt
        deferred: set[int] = set()
        nit, nt = its.next, tms.next_time
        for k in range(1, limit + 1):
            t = t + dt
            # the schedulers are asked only where one of them is due (what they would fire is then the same)
            if not ((nit is not None and it + k >= nit) or (nt is not None and (t >= nt if forward else t <= nt))):
                continue
            fired = its(it + k) + tms(t)
            nit, nt = its.next, tms.next_time
            if not fired:
                continue
            if k == limit or not all(e.deferrable for e in fired):
                return k, deferred
            deferred.add(it + k)
        return limit, deferred

    def _run(self, nsteps: int, reader: "_ResultReader | None" = None) -> None:
        done = 0
        while done < nsteps:
            k, deferred = self.plan_events(min(nsteps - done, self._maybe_sort()))
            split = reader.split() if reader is not None and done + k == nsteps else None
            recorder = _EventRecorder(self, deferred) if deferred else None
            self._timestepper.timestep_particles_many(self._particles, self._launcher, k, split, recorder)
            done += k
            if self._steps_since_sort is not None:
                self._steps_since_sort += k
            if self._invoke_events() and split is not None and split.used:
                reader.discard()  # an event ran after the ranges were read: read the final state again

    def synchronize(self) -> None:
        """Wait for queued device work and raise any error it recorded."""
        torch.cuda.synchronize(self._particles.device)
        self._particles.check_errors()

    # ---------------------------------------------------------- checkpoint
    def save_checkpoint(self, path) -> None:
        """Write the particle arrays (every field, the AB3 history included, in original order), the time
        and the iteration to ``path`` (.npz).  Resume with ``load_checkpoint`` and ``restore_particles`` on a
        Simulation built with a timestepper at that time and iteration (the reference's manual restart:
        ``Timestepper(time=..., iteration=...)``, ``set_particle_field``)."""
        self.synchronize()
        arrays = {f"p_{k}": self._particles.original(k).cpu().numpy() for k in self._particles.arrays}
        np.savez(path, time=np.asarray(self.time), iteration=np.int64(self.iteration), **arrays)

    def restore_particles(self, particles: Mapping[str, np.ndarray]) -> None:
        """Set every particle field from ``particles`` (original order), e.g. ``load_checkpoint(...).particles``."""
        missing = set(self._particles.arrays) - set(particles)
        if missing:
            raise KeyError(f"checkpoint lacks particle fields {sorted(missing)}")
        for k, v in particles.items():
            if k in self._particles.arrays:
                self._particles.assign(k, torch.from_numpy(np.ascontiguousarray(v)))
        self._steps_since_sort = None

    @property
    def output_writers(self) -> Mapping[str, object]:
        return self._output_writers

    def close_outputs(self) -> None:
        """Finish every output writer that buffers rows (files complete on disk)."""
        for w in self._output_writers.values():
            close = getattr(w, "close", None)
            if close is not None:
                close()


# bytes of device memory the recorded states of one fused launch may take (status, zidx, yidx, xidx and z:
# 33 bytes per particle and recorded step); at least one step is recorded
RECORD_BUDGET_BYTES = 2 << 30
_RECORDED = ("zidx", "yidx", "xidx", "z", "status")


class _RecordPlan:
    """The records of one fused launch (``opb_records``) and the events they replay."""

    def __init__(self, sim: Simulation, steps: list[tuple[int, object, object, int]]) -> None:
        from . import _lib

        self.sim = sim
        self.steps = steps  # (iteration, time, tidx, step index in the launch)
        P = sim._particles
        n = len(P)
        self.bufs = sim._record_buffers(len(steps))
        st = _lib.opb_records()
        for *_, j in steps:
            st.mask[j >> 6] |= 1 << (j & 63)
        st.stride = n
        for name in _RECORDED:
            setattr(st, name, self.bufs[name].data_ptr())
        self.struct = st

    def at(self, lo: int):
        """The records of a launch over storage slots from ``lo`` on (the same records, offset)."""
        from . import _lib

        st = _lib.opb_records()
        st.mask[:] = self.struct.mask[:]
        st.stride = self.struct.stride
        for name in _RECORDED:
            setattr(st, name, getattr(self.struct, name) + lo * (1 if name == "status" else 8))
        return st

    def replay(self, td) -> None:
        """Fire the recorded steps' events in step order, each on the state recorded at its step (the other
        particle fields, the events' outputs among them, are the simulation's own)."""
        sim = self.sim
        P = sim._particles
        for slot, (it, t, tidx, _) in enumerate(self.steps):
            arrays = dict(P.arrays)
            for name in _RECORDED:
                arrays[name] = self.bufs[name][slot]
            V = Particles.view(arrays, P)
            state = SimulationState(time=t, dt=sim.dt, tidx=tidx, iteration=it, particles=ParticlesView(V))
            for event in itertools.chain(sim._iteration_scheduler(it), sim._time_scheduler(t)):
                if not event.deferrable:
                    raise RuntimeError(f"event {event.name!r} fired inside a fused launch")
                for kernel in event.kernels:
                    sim._launcher.launch_kernel(kernel, V, tidx)
                event(state)


class _EventRecorder:
    """Events inside the fused launches of one stretch of steps (``Simulation.plan_events``): a launch
    records the particle state after the steps whose events are deferred (``opb_records``), and the events
    fire after the launch, in step order, on those states."""

    def __init__(self, sim: Simulation, deferred: set[int]) -> None:
        self.sim = sim
        self.deferred = deferred
        n = max(1, len(sim._particles))
        self.max_records = max(1, min(256, RECORD_BUDGET_BYTES // (33 * n)))

    def full(self, iteration0: int, nsteps: int) -> bool:
        """A launch of ``nsteps`` steps from ``iteration0`` would record more states than the budget."""
        return sum(1 for k in range(iteration0 + 1, iteration0 + nsteps + 1) if k in self.deferred) > self.max_records

    def plan(self, iteration0: int, end_times: list, end_tidxs: list) -> _RecordPlan | None:
        steps = [(iteration0 + j + 1, end_times[j], end_tidxs[j], j) for j in range(len(end_times))
                 if iteration0 + j + 1 in self.deferred]
        return _RecordPlan(self.sim, steps) if steps else None

    def after_step(self, iteration: int) -> None:
        """A step run on its own: its deferred events fire now, on the live state."""
        if iteration in self.deferred:
            self.sim._invoke_events()


def result_bounds(n: int, ranges: int) -> tuple[int, ...] | None:
    """Id bounds of ``ranges`` result ranges of ``n`` particles (None: one range).  The last range holds a
    quarter of the particles: its results are copied back after the last launch, with nothing left to
    hide the copy behind, while each earlier range's copy runs behind the next range's compute.  The
    earlier ranges split the rest evenly.  A range spreads its particles over the whole domain at a
    fraction of the density, which costs the fused kernel locality: four equal ranges took 1.33 times
    the time of one launch over all particles on a 1024 x 768 x 50 grid, two equal ones 1.15 times."""
    ranges = min(int(ranges), n)
    if ranges <= 1:
        return None
    last = -(-n // 4)
    head = n - last
    return tuple(head * j // (ranges - 1) for j in range(ranges)) + (n,)


class _ResultReader:
    """The copies of ``Simulation.run(results=...)``: particle fields in original order into host tensors,
    on a stream of their own (after the launches they read; the current stream waits for them at the
    end), range by range while a split launch computes, or all at once after the run."""

    def __init__(self, sim: Simulation, results: Mapping[str, torch.Tensor]) -> None:
        P = sim._particles
        n = len(P)
        for name, host in results.items():
            if name not in P:
                raise KeyError(f"no particle field {name!r}")
            t = P[name]
            if not isinstance(host, torch.Tensor) or host.is_cuda:
                raise TypeError(f"results[{name!r}] must be a host (CPU) torch tensor")
            if tuple(host.shape) != (n,) or host.dtype != t.dtype or not host.is_contiguous():
                raise ValueError(f"results[{name!r}] must be a contiguous {t.dtype} tensor of shape ({n},)")
        self.sim = sim
        self.results = dict(results)
        self.read: set[int] = set()
        self.ranges: list[tuple[int, int]] = []
        if sim._readback_stream is None:
            sim._readback_stream = torch.cuda.Stream(device=P.device, priority=-1)
        self.stream = sim._readback_stream
        self.began = False

    def split(self):
        """The range split of the run's last launch, or None when storage order keeps no id ranges."""
        from .timesteppers import RangeLaunches

        sim = self.sim
        b, P = sim._id_bounds, sim._particles
        if b is None or P.sort_bounds not in ((), b) or not self.results:
            return None
        self.ranges = list(zip(b[:-1], b[1:]))
        return RangeLaunches(self.ranges, self._read_range)

    def _read_range(self, i: int) -> None:
        self._read(*self.ranges[i])
        self.read.add(i)

    def _read(self, lo: int, hi: int) -> None:
        """Queue the copies of slots [lo, hi), whose original ids are [lo, hi) too (or all slots)."""
        P = self.sim._particles
        cur = torch.cuda.current_stream(P.device)
        side = self.stream
        side.wait_stream(cur)
        self.began = True
        order = P.order
        with torch.cuda.stream(side):
            for name, host in self.results.items():
                t = P.arrays[name]
                if order is None:
                    host[lo:hi].copy_(t[lo:hi], non_blocking=True)
                    continue
                buf = self.sim._readback.get(name)
                if buf is None or buf.shape != t.shape or buf.dtype != t.dtype:
                    buf = self.sim._readback[name] = torch.empty_like(t)
                buf.index_copy_(0, order[lo:hi], t[lo:hi])
                host[lo:hi].copy_(buf[lo:hi], non_blocking=True)

    def discard(self) -> None:
        self.read.clear()

    def finish(self, read: bool = True) -> None:
        """Read what the ranges did not (all of it when the last launch was not split; nothing after a
        failed run), then let the current stream wait for the copies already queued."""
        if read and (not self.ranges or len(self.read) < len(self.ranges)):
            self._read(0, len(self.sim._particles))
        if self.began:
            torch.cuda.current_stream(self.sim._particles.device).wait_stream(self.stream)


class Checkpoint:
    """What ``Simulation.save_checkpoint`` wrote: ``time``, ``iteration`` and ``particles`` (name -> array)."""

    def __init__(self, time, iteration: int, particles: dict[str, np.ndarray]) -> None:
        self.time = time
        self.iteration = iteration
        self.particles = particles


def load_checkpoint(path) -> Checkpoint:
    with np.load(path) as z:
        particles = {k[2:]: z[k] for k in z.files if k.startswith("p_")}
        t = z["time"]
        return Checkpoint(t[()] if t.ndim == 0 else t, int(z["iteration"]), particles)


class SimulationBuilder:
    """Builds a Simulation from a timestepper, a fieldset and events."""

    def __init__(self, timestepper: Timestepper, fieldset: Fieldset) -> None:
        self._timestepper = timestepper
        self._fieldset = fieldset
        self._iteration_scheduler = IterationScheduler()
        self._time_scheduler = TimeScheduler()
        self._output_writers: dict[str, tuple] = {}

    def every_n(self, n: int, event: Event, *, first: int | None = None) -> None:
        if n <= 0:
            raise ValueError("n must be a positive integer.")
        self._iteration_scheduler.register_event(0 if first is None else first, n, event)

    def every_dt(self, dt, event: Event, *, first=None) -> None:
        tt = self._timestepper.time
        if first is None:
            first = tt
        try:
            _ = tt + dt
        except TypeError as e:
            raise TypeError(f"Incompatible dt type {type(dt)} for timestepper time type {type(tt)}") from e
        try:
            _ = first + dt
        except TypeError as e:
            raise TypeError(f"Incompatible first type {type(first)} for timestepper time type {type(tt)}") from e
        self._time_scheduler.register_event(first, dt, event)

    def add_event(self, event: Event, *, n=None, dt=None, first=None) -> None:
        if n is not None and dt is not None:
            raise ValueError("Cannot specify both n and dt.")
        elif n is not None:
            self.every_n(n, event, first=first)
        elif dt is not None:
            self.every_dt(dt, event, first=first)
        else:
            raise ValueError("Either n or dt must be specified.")

    def add_output_writer(self, builder, *, n=None, dt=None, first=None) -> None:
        """Add an output writer (simulation.py:320-342): its events fire every ``n`` iterations or ``dt``."""
        name = builder.name
        if name in self._output_writers:
            raise ValueError(f"Output writer '{name}' already exists.")
        self._output_writers[name] = (builder, {"n": n, "dt": dt, "first": first})

    def build_simulation(self, nparticles: int, *, device=None, sort_interval: int = DEFAULT_SORT_INTERVAL,
                         arithmetic: str = "float64", result_ranges: int = 1) -> Simulation:
        """Build the writers, schedule their events (simulation.py:344-369) and the Simulation."""
        writers = {}
        time_type = np.asarray(self._timestepper.time_array).dtype
        for name, (builder, kwargs) in self._output_writers.items():
            writers[name] = builder.build(nparticles, time_type)
            for event in writers[name].create_events():
                self.add_event(event, **kwargs)
        return Simulation(nparticles=nparticles, timestepper=self._timestepper, fieldset=self._fieldset,
                          iteration_scheduler=self._iteration_scheduler, time_scheduler=self._time_scheduler,
                          output_writers=types.MappingProxyType(writers), device=device, sort_interval=sort_interval,
                          arithmetic=arithmetic, result_ranges=result_ranges)
