"""Fields on the device: static fields in HBM, time-dependent fields as a snapshot ring.

Mirrors offline_particles' ``fields.py`` (``Field``, ``StaticField``,
``TimeDependentField``, ``FieldData``) with the same constructors, window
semantics and errors.  Two things change, both B200-first:

* The time blend ``prev * (1 - ft) + next * ft`` (fields.py:419-428 of the
  reference) is not materialised over the whole grid at every launch.
  ``get_field_data`` returns a ``FieldData`` whose ``array`` is a
  ``BlendedArray``: the two device snapshots plus the weights, rounded to the
  storage dtype exactly as the reference rounds them.  The kernels blend each
  gathered corner with the same storage-dtype arithmetic, which gives the
  reference's values bit for bit while reading two snapshots instead of
  writing and re-reading a blended float64 grid.
* Snapshots live in a device ring of ``ring_size`` slots.  A background thread
  reads snapshot ``k`` from the host source (a numpy array, a CPU tensor, or
  any object with ``shape``/``ndim``/``dtype``/``__getitem__(k)``), stages it in
  pinned memory and copies it to its slot on a side CUDA stream; the compute
  stream waits on that copy's event.  The next snapshots are prefetched while
  the current interval runs.  A CUDA tensor source is used in place.
"""

from __future__ import annotations

import abc
import collections
import concurrent.futures
import threading

import numpy as np
import torch

from ._device import cuda_device, torch_dtype
from .spatial_arrays import BBox, DeviceArray, SpatialArray, Stagger

# Observers of snapshot pair/quad/octet builds: callables run after each build launch (used for counting
# launches).
pair_observers: list = []
# Observers of snapshot uploads: callables obs(k, copy_stream) run right after a snapshot's copy is queued
# on the copy stream (for timelines; they may record an event on that stream)
upload_observers: list = []
# elements of the storage dtype per grid element in each pair layout
PAIR_WIDTH = {"pairs": 2, "quads": 4, "octets": 8, "zeta_h": 8}

FieldData = collections.namedtuple("FieldData", ["array", "offsets"])

SUPPORTED_DTYPES = (np.dtype(np.float64), np.dtype(np.float32))


class BlendedArray:
    """``prev * gt + next * ft`` of one time-dependent field, left unmaterialised.

    ``ft`` and ``gt`` are numpy scalars of the storage dtype, computed as
    fields.py:409-424 of the reference computes them.
    """

    __slots__ = ("field", "It", "prev", "next", "ft", "gt")

    def __init__(self, field: "TimeDependentField", It: int, prev: torch.Tensor, nxt: torch.Tensor, ft, gt) -> None:
        self.field = field
        self.It = It
        self.prev = prev
        self.next = nxt
        self.ft = ft
        self.gt = gt

    @property
    def dtype(self) -> np.dtype:
        return self.field.dtype

    @property
    def shape(self) -> tuple[int, ...]:
        return tuple(self.prev.shape)

    def materialize(self) -> torch.Tensor:
        """The blended float64 array (both products and the sum in the storage dtype)."""
        td = self.prev.dtype
        a = self.prev * torch.tensor(float(self.gt), dtype=td, device=self.prev.device)
        b = self.next * torch.tensor(float(self.ft), dtype=td, device=self.prev.device)
        return (a + b).to(torch.float64)

    def __array__(self, dtype=None, copy=None):
        out = self.materialize().cpu().numpy()
        return out.astype(dtype) if dtype is not None else out


class Field(abc.ABC):
    """Abstract base class for fields used in particle tracking (fields.py:15-119)."""

    def __init__(self, z_stagger: Stagger, y_stagger: Stagger, x_stagger: Stagger) -> None:
        self._z_stagger = Stagger(z_stagger)
        self._y_stagger = Stagger(y_stagger)
        self._x_stagger = Stagger(x_stagger)
        self._z_offset = self._z_stagger.offset
        self._y_offset = self._y_stagger.offset
        self._x_offset = self._x_stagger.offset

    @property
    def z_stagger(self) -> Stagger:
        return self._z_stagger

    @property
    def y_stagger(self) -> Stagger:
        return self._y_stagger

    @property
    def x_stagger(self) -> Stagger:
        return self._x_stagger

    @property
    def stagger(self) -> tuple[Stagger, Stagger, Stagger]:
        return (self._z_stagger, self._y_stagger, self._x_stagger)

    @property
    def z_offset(self) -> float | None:
        return self._z_offset

    @property
    def y_offset(self) -> float | None:
        return self._y_offset

    @property
    def x_offset(self) -> float | None:
        return self._x_offset

    @property
    def all_offsets(self) -> tuple[float | None, float | None, float | None]:
        return (self._z_offset, self._y_offset, self._x_offset)

    @property
    def active_offsets(self) -> tuple[float, ...]:
        return tuple(o for o in self.all_offsets if o is not None)

    @property
    def dmask(self) -> tuple[bool, bool, bool]:
        return (self._z_stagger.is_active, self._y_stagger.is_active, self._x_stagger.is_active)

    @property
    @abc.abstractmethod
    def dtype(self) -> np.dtype: ...

    @property
    @abc.abstractmethod
    def spatial_shape(self) -> tuple[int, ...]: ...

    @property
    def nspatial_dims(self) -> int:
        return len(self.spatial_shape)

    def _staggered_shape(self, simulation_shape: tuple[int, int, int, int]) -> tuple[int, ...]:
        staggered = (
            self.z_stagger.expected_size(simulation_shape[1]),
            self.y_stagger.expected_size(simulation_shape[2]),
            self.x_stagger.expected_size(simulation_shape[3]),
        )
        return tuple(s for s in staggered if s is not None)

    @abc.abstractmethod
    def validate_shape(self, simulation_shape: tuple[int, int, int, int]) -> None: ...

    @abc.abstractmethod
    def get_field_data(self, time_index: float, bbox: BBox | None = None) -> FieldData: ...


class StaticField(Field):
    """A time-invariant field, held on the device as float64.

    The reference casts every field to contiguous float64 at each launch
    (kernels/_core.pyx:5-24); a static field is cast once, at upload.
    """

    def __init__(self, data: SpatialArray) -> None:
        super().__init__(data.z_stagger, data.y_stagger, data.x_stagger)
        if not isinstance(data, DeviceArray):
            raise TypeError("StaticField expects a DeviceArray / NumpyArray")
        self._source_dtype = data.dtype
        if data.data.dtype != torch.float64:
            data = DeviceArray(data.data, data.z_stagger, data.y_stagger, data.x_stagger, dtype=torch.float64)
        self._data = data
        self._neighbours: dict = {}  # neighbour layouts and bundles: (sources kept alive ..., result)

    @property
    def data(self) -> DeviceArray:
        return self._data

    def __repr__(self) -> str:
        return (f"StaticField(shape={self._data.shape}, z_stagger={self.z_stagger}, "
                f"y_stagger={self.y_stagger}, x_stagger={self.x_stagger})")

    @property
    def dtype(self) -> np.dtype:
        return self._source_dtype

    @property
    def spatial_shape(self) -> tuple[int, ...]:
        return self._data.shape

    def validate_shape(self, simulation_shape: tuple[int, int, int, int]) -> None:
        expected = self._staggered_shape(simulation_shape)
        if self._data.shape != expected:
            raise ValueError(f"Expected shape {expected} but data has shape {self._data.shape}")

    def get_field_data(self, time_index: float, bbox: BBox | None = None) -> FieldData:
        """The float64 device array and its offsets; ``time_index`` is ignored."""
        array, offsets = self._data.get_data_subset(bbox)
        return FieldData(array, offsets)

    def neighbours(self, kind: str = "xpairs") -> torch.Tensor:
        """The field's neighbour layout, the static companion of snapshot quads and octets: "xpairs"
        (shape ``(2 * size,)``, element i holds values i and i + 1; ``opb_neighbour_pairs``) or
        "yxpairs" (shape ``(4 * size,)``, values i, i + 1, i + R, i + R + 1 with R the x size;
        ``opb_neighbour_quads``).  Built once per kind, on the current stream."""
        if kind not in ("xpairs", "yxpairs"):
            raise ValueError(f"unknown neighbour layout {kind!r}")
        if kind not in self._neighbours:
            from . import _lib
            from ._device import stream_handle

            src = self._data.data.contiguous()
            st = stream_handle(src.device)
            if kind == "xpairs":
                out = torch.empty(2 * src.numel(), dtype=torch.float64, device=src.device)
                _lib.call("opb_neighbour_pairs", src.data_ptr(), out.data_ptr(), src.numel(), st)
            else:
                out = torch.empty(4 * src.numel(), dtype=torch.float64, device=src.device)
                _lib.call("opb_neighbour_quads", src.data_ptr(), out.data_ptr(), src.numel(), src.shape[-1], st)
            self._neighbours[kind] = (src, out)  # src kept alive until the build has run
        return self._neighbours[kind][-1]

    def bundle(self, other: "StaticField") -> torch.Tensor:
        """This field bundled with ``other`` of the same shape, each element with its x-neighbour
        (``{self[i], other[i], self[i+1], other[i+1]}``, shape ``(4 * size,)``; ``opb_bundle_dx_dy``): dx
        with dy, one 32-byte load per two stencil corners of both.  Built once per partner."""
        key = ("bundle", other.data.data.data_ptr())  # the partner's buffer, kept alive below
        if key not in self._neighbours:
            from . import _lib
            from ._device import stream_handle

            a = self._data.data.contiguous()
            b = other.data.data.contiguous()
            if a.shape != b.shape:
                raise ValueError("bundled fields must have one shape")
            out = torch.empty(4 * a.numel(), dtype=torch.float64, device=a.device)
            _lib.call("opb_bundle_dx_dy", a.data_ptr(), b.data_ptr(), out.data_ptr(), a.numel(), stream_handle(a.device))
            self._neighbours[key] = (a, b, out)
        return self._neighbours[key][-1]

    @classmethod
    def from_numpy(cls, data, z_stagger: Stagger | str, y_stagger: Stagger | str, x_stagger: Stagger | str,
                   *, device=None) -> "StaticField":
        arr = np.asarray(data)
        spatial = DeviceArray(arr.astype(np.float64, copy=False), Stagger(z_stagger), Stagger(y_stagger),
                              Stagger(x_stagger), dtype=torch.float64, device=device)
        f = cls(spatial)
        f._source_dtype = arr.dtype
        return f

    @classmethod
    def from_tensor(cls, data: torch.Tensor, z_stagger, y_stagger, x_stagger, *, device=None) -> "StaticField":
        spatial = DeviceArray(data, Stagger(z_stagger), Stagger(y_stagger), Stagger(x_stagger), dtype=torch.float64,
                              device=device)
        return cls(spatial)


STORAGE = {None: None, "float32": None, "float64": None, "bfloat16": torch.bfloat16, "float16": torch.float16}


def quantize_levels(src: torch.Tensor, dst: torch.Tensor, scales: torch.Tensor, nlev: int) -> None:
    """dst (bfloat16/float16) = src (float32) / scale, one scale per level (per leading index of src / nlev)."""
    from . import _lib
    from ._device import stream_handle

    if src.dtype != torch.float32 or not src.is_contiguous() or not dst.is_contiguous():
        raise TypeError("quantisation needs a contiguous float32 source")
    code = {torch.bfloat16: _lib.BF16, torch.float16: _lib.F16}[dst.dtype]
    groups = scales.numel()
    per_level = src.numel() // groups
    _lib.call("opb_quantize_levels", src.data_ptr(), 1, groups, per_level, code, dst.data_ptr(), scales.data_ptr(),
              stream_handle(src.device))


class SnapshotLoadError(RuntimeError):
    """A snapshot could not be brought to the device: its source raised, or delivered nothing in time."""


class TicketOrder:
    """Issue in ticket order: ``ticket()`` hands out 0, 1, 2, ...; ``wait_turn(t)`` returns once every
    ticket below ``t`` is released, or after ``limit`` seconds, when it passes the stuck ones over for
    everyone after them; ``release(t)`` marks ticket ``t`` issued (or abandoned).  Host logic only."""

    def __init__(self, limit: float = 2.0) -> None:
        self.limit = limit
        self.cv = threading.Condition()
        self.next_ticket = 0
        self.issued_below = 0  # every ticket below this has been released (or passed over)
        self.done: set[int] = set()

    def ticket(self) -> int:
        with self.cv:
            t = self.next_ticket
            self.next_ticket += 1
            return t

    def wait_turn(self, t: int, limit: float | None = None) -> bool:
        """True if every earlier ticket was released in time, False if they were passed over."""
        with self.cv:
            if self.cv.wait_for(lambda: self.issued_below >= t, timeout=self.limit if limit is None else limit):
                return True
            self.issued_below = t
            self.done = {d for d in self.done if d >= t}
            self.cv.notify_all()
            return False

    def release(self, t: int) -> None:
        with self.cv:
            if t < self.issued_below:
                return  # passed over while it was stuck
            self.done.add(t)
            while self.issued_below in self.done:
                self.done.remove(self.issued_below)
                self.issued_below += 1
            self.cv.notify_all()


class _CopyQueue:
    """The copy stream of one device, shared by every snapshot ring on it, and the order in which the
    rings issue onto it: the order in which their uploads were scheduled (``TicketOrder``).

    A copy engine serves several streams with queued copies one stream at a time rather than in the
    order the copies were queued, so rings with streams of their own deliver every snapshot of one field
    before the first of the next, and a launch that needs snapshot k of every field waits for all the
    later snapshots of the fields served first.  On one stream in scheduling order, snapshot k of every
    field lands before snapshot k + 1 of any.  Host staging still runs in each ring's own thread; only
    the issue of the copy waits for the uploads scheduled before it, at most ``TURN_TIMEOUT`` seconds and
    a quarter of the ring's ``load_timeout`` (a stalled source then gives up the order, never the
    progress of the others, and is the one whose snapshot times out).

    One stream cannot deadlock the rings: a launch waits only for uploads that were issued before it
    was queued (``acquire`` returns once its upload is issued), and an upload waits only for launches
    queued before it (the last reader of its slot)."""

    TURN_TIMEOUT = 2.0
    _by_device: dict = {}
    _registry_lock = threading.Lock()

    @classmethod
    def of(cls, device: torch.device) -> "_CopyQueue":
        index = device.index if device.index is not None else torch.cuda.current_device()
        with cls._registry_lock:
            q = cls._by_device.get(index)
            if q is None:
                q = cls._by_device[index] = cls(torch.device("cuda", index))
            return q

    def __init__(self, device: torch.device) -> None:
        self.stream = torch.cuda.Stream(device=device)
        self.order = TicketOrder(self.TURN_TIMEOUT)


class SnapshotRing:
    """Device slots for the snapshots of one time-dependent field.

    ``acquire(k)`` returns the device tensor of snapshot ``k`` and makes the
    current stream wait for its upload.  Uploads run on the device's copy stream
    (``_CopyQueue``, shared by every ring on the device, in scheduling order)
    from a background thread: host read -> pinned staging buffer -> async H2D
    copy.
    """

    def __init__(self, source, spatial_shape: tuple[int, ...], np_dtype: np.dtype, nslots: int,
                 device: torch.device, storage: torch.dtype | None = None, load_timeout: float | None = 600.0) -> None:
        self.source = source
        self.load_timeout = load_timeout
        self.np_dtype = np.dtype(np_dtype)
        self.device = device
        self.nslots = nslots
        # reduced-precision storage: slots hold bfloat16/float16 values, one scale per level
        self.storage = storage
        slot_dtype = storage if storage is not None else torch_dtype(np_dtype)
        self.slots = torch.empty((nslots,) + tuple(spatial_shape), dtype=slot_dtype, device=device)
        self.nlev = spatial_shape[0] if len(spatial_shape) == 3 else 1
        if storage is not None:
            self.slot_scales = torch.ones((nslots, self.nlev), dtype=torch.float32, device=device)
            self.device_staging = torch.empty(tuple(spatial_shape), dtype=torch.float32, device=device)
        self.slot_of: dict[int, int] = {}
        self.pending: dict[int, concurrent.futures.Future] = {}
        self.ready: dict[int, torch.cuda.Event] = {}
        self.lru: list[int] = []  # snapshots, least recently used first
        # per slot: event recorded after the last launch known to read it (None: unknown -> wait for
        # everything queued so far before overwriting the slot)
        self.last_use: dict[int, torch.cuda.Event | None] = {}
        self.queue = _CopyQueue.of(device)
        self.copy_stream = self.queue.stream
        # pinned host buffers for sources that are neither on the device, generated there, nor already
        # pinned: allocated on the first upload that needs them
        self.spatial_shape = tuple(spatial_shape)
        self.staging: list[torch.Tensor] = []
        self.staging_free = [None, None]  # events: staging buffer's last H2D copy done
        self.staging_next = 0
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=1, thread_name_prefix="opb-snapshots")
        self.lock = threading.Lock()
        self.h2d_bytes = 0
        # start the worker now and bind it to the device, so that the first upload does not pay for a
        # thread start and a first CUDA call
        self.pool.submit(self._bind_worker).result()

    def _bind_worker(self) -> None:
        torch.cuda.set_device(self.device)
        torch.cuda.Event().record(self.copy_stream)

    def _host_snapshot(self, k: int) -> np.ndarray:
        src = self.source
        if isinstance(src, torch.Tensor):
            return src[k].numpy()
        return np.ascontiguousarray(np.asarray(src[k]), dtype=self.np_dtype)

    def _to_slot(self, slot: int, src: torch.Tensor) -> None:
        """Copy (or quantise) one snapshot into its slot; runs on the copy stream."""
        if self.storage is None:
            self.slots[slot].copy_(src, non_blocking=True)
            return
        self.device_staging.copy_(src, non_blocking=True)
        quantize_levels(self.device_staging, self.slots[slot], self.slot_scales[slot], self.nlev)

    def scales(self, k: int) -> torch.Tensor | None:
        return None if self.storage is None else self.slot_scales[self.slot_of[k]]

    def _wait_turn(self, ticket: int) -> None:
        lt = self.load_timeout
        self.queue.order.wait_turn(ticket, None if lt is None else min(_CopyQueue.TURN_TIMEOUT, 0.25 * lt))

    def _upload(self, k: int, slot: int, slot_free: torch.cuda.Event, ticket: int) -> None:
        try:
            self._upload_in_turn(k, slot, slot_free, ticket)
        finally:
            self.queue.order.release(ticket)

    def _upload_in_turn(self, k: int, slot: int, slot_free: torch.cuda.Event, ticket: int) -> None:
        src = self.source
        if hasattr(src, "produce"):
            # generated on the device, on the copy stream
            self._wait_turn(ticket)
            with torch.cuda.device(self.device), torch.cuda.stream(self.copy_stream):
                if slot_free is not None:
                    self.copy_stream.wait_event(slot_free)
                if self.storage is None:
                    src.produce(k, self.slots[slot])
                else:
                    src.produce(k, self.device_staging)
                    quantize_levels(self.device_staging, self.slots[slot], self.slot_scales[slot], self.nlev)
                ev = torch.cuda.Event()
                ev.record(self.copy_stream)
            self.ready[k] = ev
            return
        if isinstance(src, torch.Tensor) and (src.is_pinned() or src.is_cuda):
            self._copy_direct(k, slot, slot_free, ticket, src[k])
            return
        item = None if isinstance(src, torch.Tensor) else src[k]
        if (isinstance(item, torch.Tensor) and (item.is_pinned() or item.is_cuda)
                and item.dtype == torch_dtype(self.np_dtype)):
            # a source whose snapshots are pinned host (or device) tensors: no staging either
            self._copy_direct(k, slot, slot_free, ticket, item)
            return
        if item is None:
            host = self._host_snapshot(k)
        elif isinstance(item, torch.Tensor):
            host = np.ascontiguousarray(item.detach().cpu().numpy(), dtype=self.np_dtype)
        else:
            host = np.ascontiguousarray(np.asarray(item), dtype=self.np_dtype)
        if not self.staging:
            self.staging = [torch.empty(self.spatial_shape, dtype=torch_dtype(self.np_dtype), pin_memory=True)
                            for _ in range(2)]
        with torch.cuda.device(self.device):
            b = self.staging_next
            self.staging_next ^= 1
            if self.staging_free[b] is not None:
                self.staging_free[b].synchronize()
            stage = self.staging[b]
            stage.copy_(torch.from_numpy(host))
            self._wait_turn(ticket)
            with torch.cuda.stream(self.copy_stream):
                if slot_free is not None:
                    self.copy_stream.wait_event(slot_free)
                self._to_slot(slot, stage)
                ev = torch.cuda.Event()
                ev.record(self.copy_stream)
                for obs in upload_observers:
                    obs(k, self.copy_stream)
            self.staging_free[b] = ev
            self.ready[k] = ev
            self.h2d_bytes += stage.numel() * stage.element_size()

    def _copy_direct(self, k: int, slot: int, slot_free, ticket: int, snap: torch.Tensor) -> None:
        """Snapshot ``k`` already in pinned host memory (or on the device): one async copy, no staging."""
        if tuple(snap.shape) != self.spatial_shape:
            raise ValueError(f"snapshot {k} has shape {tuple(snap.shape)}, expected {self.spatial_shape}")
        self._wait_turn(ticket)
        with torch.cuda.device(self.device), torch.cuda.stream(self.copy_stream):
            if slot_free is not None:
                self.copy_stream.wait_event(slot_free)
            self._to_slot(slot, snap)
            ev = torch.cuda.Event()
            ev.record(self.copy_stream)
            for obs in upload_observers:
                obs(k, self.copy_stream)
        self.ready[k] = ev
        if not snap.is_cuda:
            self.h2d_bytes += snap.numel() * snap.element_size()

    def _free_slot(self, keep: set[int]) -> int | None:
        used = set(self.slot_of.values())
        for s in range(self.nslots):
            if s not in used:
                return s
        for k in self.lru:
            if k not in keep:
                slot = self.slot_of.pop(k)
                self.lru.remove(k)
                self.ready.pop(k, None)
                return slot
        return None

    def _schedule(self, k: int, keep: set[int]) -> bool:
        if k in self.slot_of:
            return True
        slot = self._free_slot(keep)
        if slot is None:
            return False
        # the slot's previous contents may still be read by queued launches: wait for the last launch
        # known to read it, or for everything queued so far when that is unknown
        if slot not in self.last_use:
            slot_free = None  # never written or read: nothing to wait for
        else:
            slot_free = self.last_use[slot]
            if slot_free is None:
                slot_free = torch.cuda.Event()
                slot_free.record(torch.cuda.current_stream(self.device))
        self.last_use[slot] = None
        self.slot_of[k] = slot
        self.lru.append(k)
        ticket = self.queue.order.ticket()
        try:
            self.pending[k] = self.pool.submit(self._upload, k, slot, slot_free, ticket)
        except BaseException:
            self.queue.order.release(ticket)
            raise
        return True

    def acquire(self, k: int, keep: set[int] | frozenset = frozenset()) -> torch.Tensor:
        with self.lock:
            if not self._schedule(k, set(keep) | {k}):
                raise RuntimeError(f"snapshot ring of {self.nslots} slots cannot hold snapshots {sorted(keep)}")
            fut = self.pending.pop(k, None)
            self.lru.remove(k)
            self.lru.append(k)
            # a launch that follows may read the slot and nobody may mark it: forget the last-use event
            self.last_use[self.slot_of[k]] = None
        if fut is not None:
            try:
                fut.result(timeout=self.load_timeout)
            except concurrent.futures.TimeoutError:
                with self.lock:
                    self.pending[k] = fut  # still loading: a later acquire waits for it again
                raise SnapshotLoadError(f"snapshot {k}: the source delivered nothing in {self.load_timeout} s") from None
            except Exception as e:
                with self.lock:  # forget the failed snapshot: a later acquire loads it again
                    slot = self.slot_of.pop(k, None)
                    if k in self.lru:
                        self.lru.remove(k)
                    self.ready.pop(k, None)
                    if slot is not None:
                        self.last_use.pop(slot, None)
                raise SnapshotLoadError(f"snapshot {k}: the source raised {type(e).__name__}: {e}") from e
        ev = self.ready.get(k)
        if ev is not None:
            torch.cuda.current_stream(self.device).wait_event(ev)
        return self.slots[self.slot_of[k]]

    def prefetch(self, k: int, keep: set[int]) -> None:
        with self.lock:
            self._schedule(k, set(keep) | {k})

    def mark_used(self, ks) -> None:
        """Record that the launches queued so far are the last to read snapshots ``ks``."""
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        with self.lock:
            for k in ks:
                if k in self.slot_of:
                    self.last_use[self.slot_of[k]] = ev

    def resident(self) -> list[int]:
        return sorted(self.slot_of)

    def is_ready(self, k: int) -> bool:
        """Snapshot k is in its slot and its upload has completed."""
        with self.lock:
            if k not in self.slot_of or (k in self.pending and not self.pending[k].done()):
                return False
            ev = self.ready.get(k)
        return ev is None or ev.query()

    def close(self) -> None:
        self.pool.shutdown(wait=True)


class _PairCache:
    """Device buffers of one pair layout of a field: the pairs by first snapshot (LRU) and free buffers."""

    __slots__ = ("cache", "store", "free", "tag")

    def __init__(self) -> None:
        self.cache: collections.OrderedDict[int, torch.Tensor] = collections.OrderedDict()
        self.store: torch.Tensor | None = None
        self.free: list[torch.Tensor] | None = None
        self.tag = None  # zeta_h: the static field bundled in


class TimeDependentField(Field):
    """A field with a leading time axis, streamed to the device snapshot by snapshot.

    Constructor and window semantics follow fields.py:237-392 of the reference:
    at least 2 spatial+time dimensions, at least 2 snapshots, a window
    ``[It, It + 1]`` moved by ``set_time_index`` / ``increment_time`` /
    ``decrement_time`` with the same errors.
    """

    def __init__(self, data, z_stagger: Stagger | str, y_stagger: Stagger | str, x_stagger: Stagger | str,
                 spatial_array_factory=None, output_dtype=np.float64, *, ring_size: int = 4, prefetch: int = 2,
                 device=None, storage: str | None = None, ring: bool | None = None, pair_slots: int = 4,
                 load_timeout: float | None = 600.0) -> None:
        """``storage``: keep the snapshots on the device as "bfloat16" or "float16" with one scale
        per level (the float32 steppers only); default: the source dtype.  ``ring``: stream the
        snapshots through a ring of ``ring_size`` device slots (default: yes, unless ``data`` is
        already a CUDA tensor, which is then read in place; ring=True copies such a source slot by
        slot, so that every launch reads the same slot addresses).  ``pair_slots``: how many snapshot
        pairs (``pair``) are kept on the device.  ``load_timeout``: seconds a launch waits for a snapshot
        from the source before ``SnapshotLoadError`` (None: no limit)."""
        super().__init__(Stagger(z_stagger), Stagger(y_stagger), Stagger(x_stagger))
        if data.ndim < 2:
            raise ValueError(
                "TimeDependentField requires at least 2 dimensions (time + spatial). For spatially invariant fields,"
                " use ConstantField or TemporalField."
            )
        if data.shape[0] < 2:
            raise ValueError("TimeDependentField requires at least 2 time steps.")
        self._data = data
        self._data_dtype = np.dtype(data.dtype) if not isinstance(data, torch.Tensor) else np.dtype(
            str(data.dtype).replace("torch.", ""))
        if self._data_dtype not in SUPPORTED_DTYPES:
            raise TypeError(f"storage dtype {self._data_dtype} is not supported (float32 or float64)")
        self._output_dtype = output_dtype
        self._num_timesteps = int(data.shape[0])
        self._spatial_shape = tuple(int(s) for s in data.shape[1:])
        self._elements = int(np.prod(self._spatial_shape))
        self._device = cuda_device(device)
        self._prefetch = max(0, int(prefetch))
        if storage not in STORAGE:
            raise ValueError(f"storage must be one of {sorted(k for k in STORAGE if k)}")
        self._storage = STORAGE[storage]
        if self._storage is not None and self._data_dtype != np.float32:
            raise TypeError("bfloat16/float16 storage quantises float32 snapshots")
        self._nlev = self._spatial_shape[0] if len(self._spatial_shape) == 3 else 1
        self._resident_source = isinstance(data, torch.Tensor) and data.is_cuda and not ring
        self._q = self._q_scales = None
        if self._resident_source:
            self._ring = None
            if self._storage is not None:
                self._q = torch.empty(tuple(data.shape), dtype=self._storage, device=data.device)
                self._q_scales = torch.ones((self._num_timesteps, self._nlev), dtype=torch.float32,
                                            device=data.device)
                src = data.contiguous()
                for k in range(self._num_timesteps):
                    quantize_levels(src[k], self._q[k], self._q_scales[k], self._nlev)
        else:
            if ring_size < 2 or ring_size > 8:
                raise ValueError("ring_size must be between 2 and 8")
            self._ring = SnapshotRing(data, self._spatial_shape, self._data_dtype, ring_size, self._device,
                                      storage=self._storage, load_timeout=load_timeout)
        self._It = 0
        if pair_slots < 2:
            raise ValueError("pair_slots must be at least 2")
        self._pair_slots = int(pair_slots)
        self._pair_caches: dict[str, _PairCache] = {}  # by layout: pairs, quads, octets

    # ------------------------------------------------------------ properties
    @property
    def data(self):
        return self._data

    def __repr__(self) -> str:
        return (f"TimeDependentField(shape={tuple(self._data.shape)}, z_stagger={self.z_stagger}, "
                f"y_stagger={self.y_stagger}, x_stagger={self.x_stagger})")

    @property
    def dtype(self) -> np.dtype:
        return self._data_dtype

    @property
    def spatial_shape(self) -> tuple[int, ...]:
        return self._spatial_shape

    @property
    def num_timesteps(self) -> int:
        return self._num_timesteps

    @property
    def ring_size(self) -> int:
        return self._ring.nslots if self._ring is not None else self._num_timesteps

    @property
    def time_index(self) -> int:
        return self._It

    def validate_shape(self, simulation_shape: tuple[int, int, int, int]) -> None:
        expected = (simulation_shape[0],) + self._staggered_shape(simulation_shape)
        if tuple(self._data.shape) != expected:
            raise ValueError(f"Expected shape {expected} but data has shape {tuple(self._data.shape)}")

    # ---------------------------------------------------------------- window
    def increment_time(self) -> None:
        if self._It == self._num_timesteps - 2:
            raise IndexError("Cannot increment past the penultimate timestep.")
        self._It += 1

    def decrement_time(self) -> None:
        if self._It == 0:
            raise IndexError("Cannot decrement past the first timestep.")
        self._It -= 1

    def set_time_index(self, It: int) -> None:
        if It == self._It:
            return
        if It == self._It + 1:
            return self.increment_time()
        if It == self._It - 1:
            return self.decrement_time()
        if It < 0 or It > self._num_timesteps - 2:
            raise IndexError(f"Valid range of time indices is 0,...,{self._num_timesteps - 2}, got {It}.")
        self._It = It

    # -------------------------------------------------------------- snapshots
    def snapshot(self, k: int, keep: set[int] | frozenset = frozenset()) -> torch.Tensor:
        """Device tensor of snapshot ``k`` in the storage dtype (uploaded if needed)."""
        if k < 0 or k >= self._num_timesteps:
            raise IndexError(k)
        if self._ring is None:
            return self._data[k] if self._q is None else self._q[k]
        return self._ring.acquire(k, keep)

    @property
    def pair_slots(self) -> int:
        return self._pair_slots

    def pair(self, k: int, keep: set[int] | frozenset = frozenset(), *, layout: str = "pairs",
             static: torch.Tensor | None = None) -> torch.Tensor:
        """Snapshots k and k + 1 interleaved element by element (shape ``(2 * size,)``; element 2i from
        snapshot k, 2i + 1 from k + 1): the layout in which the float64 fused steppers fetch both values
        of a time blend with one load.  ``layout`` (float32 storage for the last two): "pairs"; "quads",
        each element's pair followed by its x-neighbour's (shape ``(4 * size,)``,
        ``opb_interleave_quads``: one 16-byte load per two stencil corners); "octets", the pairs of
        elements i, i + 1, i + R, i + R + 1 with R the x size (shape ``(8 * size,)``,
        ``opb_interleave_octets``: one 32-byte load per stencil face); "zeta_h", the pair bundled with the
        float64 ``static`` field of the same shape (h beside zeta: 32 bytes per element,
        ``opb_bundle_zeta_h``).  Built on the current stream the
        first time it is asked for; the ``pair_slots`` most recently used pairs of each layout stay on
        the device, and a buffer is reused for a new one in stream order (after the launches queued
        before it that read the old one).  Pairs in ``keep`` are not evicted."""
        width = PAIR_WIDTH.get(layout)
        if width is None:
            raise ValueError(f"unknown pair layout {layout!r}")
        if self._storage is not None:
            raise ValueError("snapshot pairs hold float32/float64 storage only")
        if width > 2 and self._data_dtype != np.float32:
            raise ValueError("snapshot quads and octets hold float32 storage only")
        if k < 0 or k + 1 >= self._num_timesteps:
            raise IndexError(k)
        pc = self._reserve_pair_buffers(layout)
        if layout == "zeta_h":
            if static is None or static.numel() != self._elements:
                raise ValueError("a zeta_h bundle needs the static field of the same shape")
            if pc.tag != static.data_ptr():  # bundled with another static field: rebuild every bundle
                if pc.free is not None:
                    pc.free.extend(pc.cache.values())
                pc.cache.clear()
                pc.tag = static.data_ptr()
        cache = pc.cache
        if k in cache:
            cache.move_to_end(k)
            return cache[k]
        if pc.free:
            buf = pc.free.pop()
        else:
            buf = None
            for old in list(cache):
                if old not in keep:
                    buf = cache.pop(old)
                    break
            if buf is None:
                raise RuntimeError(f"{self._pair_slots} pair slots cannot hold pairs {sorted(keep)}")
        a = self.snapshot(k, {k, k + 1})
        b = self.snapshot(k + 1, {k, k + 1})
        from . import _lib
        from ._device import stream_handle

        st = stream_handle(self._device)
        if layout == "zeta_h":
            _lib.call("opb_bundle_zeta_h", a.data_ptr(), b.data_ptr(), static.data_ptr(), buf.data_ptr(), a.numel(),
                      st)
        elif layout == "octets":
            _lib.call("opb_interleave_octets", a.data_ptr(), b.data_ptr(), buf.data_ptr(), a.numel(),
                      self._spatial_shape[-1], st)
        elif layout == "quads":
            _lib.call("opb_interleave_quads", a.data_ptr(), b.data_ptr(), buf.data_ptr(), a.numel(), st)
        else:
            _lib.call("opb_interleave_pairs", a.data_ptr(), b.data_ptr(), buf.data_ptr(), a.numel(),
                      _lib.F32 if a.dtype == torch.float32 else _lib.F64, st)
        for obs in pair_observers:
            obs()
        cache[k] = buf
        return buf

    def _reserve_pair_buffers(self, layout: str) -> _PairCache:
        """The pair cache of ``layout`` with all ``pair_slots`` buffers allocated: every buffer at once,
        since a large allocation between launches can synchronise the device."""
        pc = self._pair_caches.setdefault(layout, _PairCache())
        if pc.free is None:
            width = PAIR_WIDTH[layout]
            pc.store = torch.empty((self._pair_slots, width * self._elements), dtype=torch_dtype(self._data_dtype),
                                   device=self._device)
            pc.free = list(pc.store.unbind(0))
        return pc

    def reserve_pairs(self, layout: str = "pairs") -> None:
        """Allocate the device buffers of ``pair(..., layout=layout)`` now (``pair_slots`` of them), so
        that the first pair build allocates nothing."""
        if PAIR_WIDTH.get(layout) is None:
            raise ValueError(f"unknown pair layout {layout!r}")
        if self._storage is not None:
            raise ValueError("snapshot pairs hold float32/float64 storage only")
        self._reserve_pair_buffers(layout)

    def snapshot_scales(self, k: int) -> torch.Tensor | None:
        """Per-level scales of resident snapshot ``k`` (None for unscaled storage)."""
        if self._storage is None:
            return None
        if self._ring is None:
            return self._q_scales[k]
        return self._ring.scales(k)

    @property
    def storage(self) -> str:
        """Device storage dtype of the snapshots: "float64", "float32", "bfloat16" or "float16"."""
        name = self.__dict__.get("_storage_name")
        if name is None:
            name = (str(self._data_dtype) if self._storage is None
                    else {torch.bfloat16: "bfloat16", torch.float16: "float16"}[self._storage])
            self.__dict__["_storage_name"] = name
        return name

    @property
    def storage_bytes_per_snapshot(self) -> int:
        n = int(np.prod(self._spatial_shape))
        return n * (2 if self._storage is not None else self._data_dtype.itemsize)

    def prefetch(self, k: int, keep: set[int]) -> None:
        if self._ring is not None and 0 <= k < self._num_timesteps:
            self._ring.prefetch(k, keep)

    def is_ready(self, k: int) -> bool:
        """Snapshot k can be read without waiting for an upload (always, for a device-resident source)."""
        return self._ring is None or self._ring.is_ready(k)

    def mark_used(self, ks) -> None:
        """Tell the ring that the launches queued so far are the last readers of snapshots ``ks``."""
        if self._ring is not None:
            self._ring.mark_used(ks)

    @property
    def streamed(self) -> bool:
        """True when snapshots stream through a device ring (False: the source is resident)."""
        return self._ring is not None

    def blend_weights(self, time_index) -> tuple[int, object, object]:
        """(It, ft, gt) with ft, gt in the storage dtype: fields.py:409-424."""
        It, ft = divmod(time_index, 1)
        ft = self._data_dtype.type(ft)
        gt = self._data_dtype.type(1 - ft)
        return int(It), ft, gt

    def get_field_data(self, time_index: float, bbox: BBox | None = None) -> FieldData:
        """FieldData whose array is the (unmaterialised) blend at ``time_index``."""
        It, ft, gt = self.blend_weights(time_index)
        if self._storage is not None:
            raise ValueError("bfloat16/float16 storage runs only in the fused float32 steppers "
                             "(build_simulation(..., arithmetic='float32'))")
        self.set_time_index(It)
        keep = {It, It + 1}
        prev = self.snapshot(It, keep)
        nxt = self.snapshot(It + 1, keep)
        for j in range(2, 2 + self._prefetch):
            self.prefetch(It + j, keep)
        return FieldData(BlendedArray(self, It, prev, nxt, ft, gt), self.active_offsets)

    @property
    def h2d_bytes(self) -> int:
        return self._ring.h2d_bytes if self._ring is not None else 0

    @classmethod
    def from_numpy(cls, data, z_stagger: Stagger | str, y_stagger: Stagger | str, x_stagger: Stagger | str,
                   **kwargs) -> "TimeDependentField":
        return cls(data, z_stagger, y_stagger, x_stagger, **kwargs)

    @classmethod
    def from_tensor(cls, data: torch.Tensor, z_stagger, y_stagger, x_stagger, **kwargs) -> "TimeDependentField":
        """A CUDA tensor is used in place; a CPU tensor is streamed like a numpy array."""
        return cls(data, z_stagger, y_stagger, x_stagger, **kwargs)
