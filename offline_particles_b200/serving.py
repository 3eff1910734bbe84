"""Serving release requests with continuous batching on one device.

A request is a release: particle indices, a scheme (RK2 or AB3), a dt and a
duration.  ``ReleaseServer`` keeps one ``ReleaseBatch`` whose model clock
advances one snapshot interval per ``tick``:

* requests wait in a FIFO queue and are admitted at an interval boundary as
  soon as the HBM budget has room for their particle state (positions, z,
  status and the RK2 stage / AB3 three-step velocity history, one arena slot
  per particle, plus its share of the sort scratch) and a release slot is
  free;
* an admitted request starts at the model time of the interval it joins,
  its state stays on the device across intervals, and it advances in the
  same persistent launches as every other running request;
* when it has run its steps, its particles are copied (asynchronously) to
  pinned host memory in their original order and its arena segment is freed
  for the next admission.

Each result equals running that request alone through ``Simulation`` with
the stock ROMS stepper from the same start time (the batched kernel's
guarantee), however many other requests shared its launches.

There is no reference counterpart: the reference runs one release per
``Simulation`` (simulation.py:27-229) and has no request loop.
"""

from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .batching import Collected, Release, ReleaseBatch
from .fieldset import Fieldset
from .models.roms import ab3_w_advection_timestepper, rk2_w_advection_timestepper


class RequestCancelled(Exception):
    """The request was withdrawn (``ReleaseServer.cancel``)."""


@dataclass
class ReleaseRequest:
    """A release to serve: ``zidx``/``yidx``/``xidx`` (float64 index-space positions), ``scheme``
    ("rk2" or "ab3"), ``dt`` and ``duration`` in the time array's units; ``arrival``: wall-clock time
    (``time.perf_counter``) at which it was submitted (0: when ``submit`` is called)."""

    zidx: np.ndarray
    yidx: np.ndarray
    xidx: np.ndarray
    scheme: str
    dt: float
    duration: float
    arrival: float = 0.0
    id: int = -1
    # filled in by the server
    start_time: float | None = field(default=None, init=False)  # model time of its first step
    nsteps: int = field(default=0, init=False)
    admitted: float | None = field(default=None, init=False)  # wall clock
    finished: float | None = field(default=None, init=False)  # wall clock: result on the host
    result: dict | None = field(default=None, init=False)
    error: BaseException | None = field(default=None, init=False)
    release: Release | None = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        if self.scheme not in ("rk2", "ab3"):
            raise ValueError("scheme must be 'rk2' or 'ab3'")
        if self.dt <= 0 or self.duration < 0:
            raise ValueError("dt must be positive and duration non-negative")

    def __len__(self) -> int:
        return len(self.zidx)

    @property
    def latency(self) -> float | None:
        return None if self.finished is None else self.finished - self.arrival


class ReleaseServer:
    """Continuous batching of release requests under an HBM budget.

    ``hbm_budget``: device bytes for particle state and its sort scratch
    (``bytes_per_particle`` each); the fields' snapshot ring and the launch
    tables are outside it.  ``max_releases``: requests that may run at once.
    ``batch_options``: ``ReleaseBatch`` launch options (block, warps_per_sm,
    buckets, sort_interval, ...).
    """

    def __init__(self, fieldset: Fieldset, time_array, *, hbm_budget: int, max_releases: int = 1024,
                 device=None, **batch_options) -> None:
        self.time_array = np.asarray(time_array, dtype=np.float64)
        self.per_particle = self.bytes_per_particle(max_releases)
        capacity = int(hbm_budget // self.per_particle)
        if capacity < 1:
            raise ValueError("the HBM budget holds no particle")
        self.batch = ReleaseBatch(fieldset, time_array=self.time_array, capacity=capacity,
                                  max_releases=max_releases, device=device, **batch_options)
        self.capacity = capacity
        self.device = self.batch.device
        self.queue: collections.deque[ReleaseRequest] = collections.deque()
        self.running: dict[int, ReleaseRequest] = {}  # id(release) -> request
        self.collecting: list[tuple[ReleaseRequest, Collected]] = []
        self.done: list[ReleaseRequest] = []
        self.rejected: list[ReleaseRequest] = []
        self.cancelled: list[ReleaseRequest] = []
        self.ticks = 0
        # the segment sort's scratch for the whole arena, allocated up front so that admission never
        # has to find device memory
        lib = _lib.load()
        ws = int(lib.opb_sort_segments_workspace_bytes(capacity, max_releases))
        self.batch._sort_ws = torch.empty(ws, dtype=torch.uint8, device=self.device)

    @staticmethod
    def bytes_per_particle(max_releases: int = 1024) -> int:
        """Device bytes one admitted particle costs: its arena slot (state + AB3 history + order index)
        and its share of the segment sort's scratch."""
        lib = _lib.load()
        n = 1 << 24
        sort = int(lib.opb_sort_segments_workspace_bytes(n, max_releases)) / n
        return int(np.ceil(ReleaseBatch.bytes_per_particle() + sort))

    # ------------------------------------------------------------------ queue
    def submit(self, req: ReleaseRequest) -> None:
        if req.arrival == 0.0:
            req.arrival = time.perf_counter()
        if len(req) > self.capacity or len(req) == 0:
            req.error = ValueError(f"{len(req)} particles do not fit the budget's {self.capacity}")
            self.rejected.append(req)
            return
        self.queue.append(req)

    def _release_for(self, req: ReleaseRequest, t0: float) -> Release:
        f = rk2_w_advection_timestepper if req.scheme == "rk2" else ab3_w_advection_timestepper
        ts = f(self.time_array, np.float64(req.dt), time=np.float64(t0))
        req.start_time = t0
        req.nsteps = int(round(req.duration / req.dt))
        return Release(ts, req.nsteps, req.zidx, req.yidx, req.xidx)

    def admit(self) -> int:
        """Admit queued requests in arrival order while they fit; return how many were admitted."""
        b = self.batch
        j = b.interval if b.interval is not None else 0
        t0 = float(self.time_array[j])
        n = 0
        while self.queue:
            req = self.queue[0]
            if len(req) > b.allocator.largest_free or None not in b.slots:
                break  # first come, first served: later requests wait behind the head
            r = self._release_for(req, t0)
            if not b.add(r):
                break
            self.queue.popleft()
            req.release = r
            req.admitted = time.perf_counter()
            self.running[id(r)] = req
            n += 1
        if b.interval is None and n:
            b.interval = j
        return n

    def cancel(self, req: ReleaseRequest) -> bool:
        """Withdraw a request: from the queue, or from the device (its particles are dropped and its
        segment freed at once; the launches already queued finish with it).  False when it has already
        finished."""
        queued = [q for q in self.queue if q is req]
        if queued:
            self.queue = collections.deque(q for q in self.queue if q is not req)
        elif req.release is not None and id(req.release) in self.running:
            self.running.pop(id(req.release))
            self.batch.retire(req.release)
        else:
            return False
        req.error = RequestCancelled(f"request {req.id} cancelled")
        req.finished = time.perf_counter()
        self.cancelled.append(req)
        return True

    # ---------------------------------------------------------------- serving
    def _poll(self, wait: bool = False) -> None:
        keep = []
        for req, handle in self.collecting:
            if wait or handle.ready():
                req.result = handle.result()
                req.finished = time.perf_counter()
                self.done.append(req)
            else:
                keep.append((req, handle))
        self.collecting = keep

    @property
    def busy(self) -> bool:
        return bool(self.queue or self.running or self.collecting)

    def tick(self) -> list[ReleaseRequest]:
        """Admit what fits, run one snapshot interval, retire what finished; return requests completed."""
        self.admit()
        before = len(self.done)
        if self.running:
            for r in self.batch.tick():
                req = self.running.pop(id(r))
                req.error = r.error
                handle = self.batch.collect(r)
                self.batch.retire(r)
                self.collecting.append((req, handle))
            self.ticks += 1
        self._poll()
        return self.done[before:]

    def drain(self) -> None:
        """Serve until every submitted request is done."""
        while self.queue or self.running:
            self.tick()
        self._poll(wait=True)
        self.batch.arena.check_errors()

    def latencies(self) -> np.ndarray:
        return np.array([r.latency for r in self.done if r.latency is not None])
