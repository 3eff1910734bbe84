"""Particles: a structure of arrays in device memory (particles.py:1-122 of the reference).

Each particle field is a 1-D CUDA tensor; the kernels mutate them in place.
The device arrays may be kept in a spatial (Morton) storage order that differs
from the particles' original order: ``sort`` reorders every field together
and remembers each slot's original particle id.  Everything facing the user
-- ``ParticlesView`` items, ``Simulation.set_indices`` / ``set_particle_field``
-- speaks the original order; only the kernels see storage order, and they
are per particle, so the order changes no result.
"""

from __future__ import annotations

import ctypes
import types
from typing import Mapping

import numpy as np
import torch

from ._device import cuda_device, numpy_dtype, stream_handle, torch_dtype


# Observers of storage sorts: callables run after each Particles.sort (used for counting launches).
sort_observers: list = []


class _FrozenArrayMapping:
    """An immutable mapping of equal-length arrays."""

    __slots__ = ("_shape", "_dtypes", "_arrays")

    def __init__(self, **arrays) -> None:
        shapes = {tuple(arr.shape) for arr in arrays.values()}
        if len(shapes) != 1:
            raise ValueError("All arrays must have the same shape. Got shapes: " + ", ".join(str(s) for s in shapes))
        object.__setattr__(self, "_shape", shapes.pop())
        object.__setattr__(self, "_dtypes", types.MappingProxyType(
            {name: numpy_dtype(arr.dtype) if isinstance(arr, torch.Tensor) else arr.dtype
             for name, arr in arrays.items()}))
        object.__setattr__(self, "_arrays", types.MappingProxyType(arrays))

    def __setattr__(self, name, value):
        raise AttributeError(f"{self.__class__.__name__} is immutable")

    def __getattr__(self, name: str):
        try:
            return self[name]
        except KeyError:
            raise AttributeError(f"'{self.__class__.__name__}' object has no attribute '{name}'")

    def __getitem__(self, name: str):
        return object.__getattribute__(self, "_arrays")[name]

    def __contains__(self, name: str) -> bool:
        return name in object.__getattribute__(self, "_arrays")

    @property
    def shape(self) -> tuple[int, ...]:
        return object.__getattribute__(self, "_shape")

    @property
    def arrays(self) -> Mapping:
        return object.__getattribute__(self, "_arrays")

    @property
    def dtypes(self) -> Mapping[str, np.dtype]:
        return object.__getattribute__(self, "_dtypes")

    def __repr__(self) -> str:
        fields = ", ".join(f"{name}:{dtype}" for name, dtype in self.dtypes.items())
        return f"{self.__class__.__name__}(shape={self.shape}, fields={{ {fields} }})"

    def __str__(self) -> str:
        names = list(self.dtypes)
        public = [name for name in names if not name.startswith("_")]
        hidden = sum(1 for name in names if name.startswith("_"))
        hidden_str = f", +{hidden} hidden fields" if hidden > 1 else (", +1 hidden field" if hidden == 1 else "")
        return f"{self.__class__.__name__} (shape={self.shape}, fields=[{', '.join(public)}]{hidden_str})"


class Particles(_FrozenArrayMapping):
    """``nparticles`` particles with the given ``field=dtype`` arrays, zero-initialised on the device."""

    __slots__ = ("_length", "_device", "_err", "_abi_cache", "_order", "_spare", "_perm", "_workspace", "_range")

    def __init__(self, nparticles: int, *, device=None, **fields) -> None:
        dev = cuda_device(device)
        object.__setattr__(self, "_length", int(nparticles))
        object.__setattr__(self, "_device", dev)
        arrays = {f: torch.zeros((int(nparticles),), dtype=torch_dtype(dt), device=dev) for f, dt in fields.items()}
        super().__init__(**arrays)
        # device error word written by the kernels (OPB_ERRF_*)
        object.__setattr__(self, "_err", torch.zeros((1,), dtype=torch.int32, device=dev))
        object.__setattr__(self, "_abi_cache", None)
        object.__setattr__(self, "_order", None)  # original id of each storage slot (None: identity)
        object.__setattr__(self, "_spare", None)
        object.__setattr__(self, "_perm", None)
        object.__setattr__(self, "_workspace", None)
        object.__setattr__(self, "_range", None)  # id bounds kept by the last sort (None: none)

    @classmethod
    def view(cls, arrays: dict[str, torch.Tensor], base: "Particles") -> "Particles":
        """Particles over existing device arrays (no copy), in the storage order of ``base`` and with its
        error word: e.g. a recorded state whose other fields are ``base``'s own."""
        obj = object.__new__(cls)
        _FrozenArrayMapping.__init__(obj, **arrays)
        for slot in ("_length", "_device", "_err", "_order", "_range"):
            object.__setattr__(obj, slot, object.__getattribute__(base, slot))
        for slot in ("_abi_cache", "_spare", "_perm", "_workspace"):
            object.__setattr__(obj, slot, None)
        return obj

    def __len__(self) -> int:
        return object.__getattribute__(self, "_length")

    @property
    def device(self) -> torch.device:
        return object.__getattribute__(self, "_device")

    @property
    def error_word(self) -> torch.Tensor:
        return object.__getattribute__(self, "_err")

    @property
    def order(self) -> torch.Tensor | None:
        """Original particle id of every storage slot, or None while storage order is the original order."""
        return object.__getattribute__(self, "_order")

    def check_errors(self) -> None:
        """Raise what the kernels recorded since the last check (synchronises)."""
        err = object.__getattribute__(self, "_err")
        value = int(err.item())
        if value:
            err.zero_()
            from ._lib import ERRF_ZERO_DIVISION

            if value & ERRF_ZERO_DIVISION:
                raise ZeroDivisionError("float division")
            raise RuntimeError(f"device error word 0x{value:x}")

    # ---------------------------------------------------------- original order
    def original(self, name: str, out: torch.Tensor | None = None) -> torch.Tensor:
        """A device copy of field ``name`` in the particles' original order (into ``out`` when given: a
        device tensor of the field's shape and dtype, so that repeated reads allocate nothing)."""
        t = self.arrays[name]
        if out is None:
            out = torch.empty_like(t)
        elif out.shape != t.shape or out.dtype != t.dtype or out.device != t.device:
            raise ValueError(f"out must be a {t.dtype} tensor of shape {tuple(t.shape)} on {t.device}")
        order = self.order
        if order is None:
            out.copy_(t)
        else:
            out.index_copy_(0, order, t)
        return out

    def assign(self, name: str, values: torch.Tensor) -> None:
        """Set field ``name`` from ``values`` given in the particles' original order."""
        t = self.arrays[name]
        order = self.order
        values = values.to(device=t.device, dtype=t.dtype).expand(t.shape)
        t.copy_(values if order is None else values.index_select(0, order))

    # ------------------------------------------------------------- reordering
    def reserve_sort(self) -> None:
        """Allocate the sort's scratch now (key workspace, permutation, a second copy of every field), so
        that the first ``sort`` allocates nothing."""
        from . import _lib

        n = len(self)
        if n == 0 or object.__getattribute__(self, "_workspace") is not None:
            return
        lib = _lib.load()
        ws = torch.empty(int(lib.opb_sort_workspace_bytes(n)), dtype=torch.uint8, device=self.device)
        object.__setattr__(self, "_workspace", ws)
        object.__setattr__(self, "_perm", torch.empty(n, dtype=torch.int32, device=self.device))
        object.__setattr__(self, "_spare", {k: torch.empty_like(v) for k, v in self.arrays.items()})

    @property
    def sort_bounds(self) -> tuple[int, ...] | None:
        """The id ranges the storage order keeps (``sort(shape, id_bounds=...)``): the particles with
        original ids in ``[b[r], b[r + 1])`` occupy those storage slots.  None after a sort without
        ranges; () while storage order is the original order (any ranges hold)."""
        if self.order is None:
            return ()
        return object.__getattribute__(self, "_range")

    def sort(self, shape: tuple[int, int, int], id_bounds: tuple[int, ...] | None = None) -> None:
        """Reorder storage by the Morton code of each particle's cell on the centred ``(z, y, x)`` grid.
        ``id_bounds``: 0 = b0 < b1 < ... < bR = n, R at most 4: order within the id ranges
        ``[b[r], b[r + 1])`` (``opb_sort_particles_ranges``), each kept in those storage slots, so that
        each range's results can be read back on their own."""
        from . import _lib
        from .kernels import _abi

        n = len(self)
        if n == 0:
            return
        if id_bounds is not None:
            id_bounds = tuple(int(b) for b in id_bounds)
            R = len(id_bounds) - 1
            if not 1 <= R <= 4 or id_bounds[0] != 0 or id_bounds[-1] != n or any(
                    b >= c for b, c in zip(id_bounds, id_bounds[1:])):
                raise ValueError(f"id_bounds must rise from 0 to {n} in 1 to 4 steps, got {id_bounds}")
            if self.sort_bounds not in ((), id_bounds):
                raise ValueError("storage order keeps other id ranges; sort without ranges first")
        self.reserve_sort()
        ws = object.__getattribute__(self, "_workspace")
        perm = object.__getattribute__(self, "_perm")
        spare = object.__getattribute__(self, "_spare")
        src = _abi.particles_struct(self)
        dims = (ctypes.c_int64 * 3)(*[int(s) for s in shape])
        stream = stream_handle(self.device)
        order = self.order
        if id_bounds is None:
            _lib.call("opb_sort_particles", ctypes.byref(src), ctypes.byref(dims), perm.data_ptr(), ws.data_ptr(),
                      ws.numel(), stream)
        else:
            bounds = (ctypes.c_int64 * len(id_bounds))(*id_bounds)
            _lib.call("opb_sort_particles_ranges", ctypes.byref(src), ctypes.byref(dims),
                      None if order is None else order.data_ptr(), bounds, len(id_bounds) - 1, perm.data_ptr(),
                      ws.data_ptr(), ws.numel(), stream)
        if order is None:
            order = torch.arange(n, dtype=torch.int64, device=self.device)
        new_order = torch.empty_like(order)
        dst = _abi.particles_struct_for(spare, n)
        _lib.call("opb_gather_particles", ctypes.byref(src), ctypes.byref(dst), perm.data_ptr(), order.data_ptr(),
                  new_order.data_ptr(), stream)
        # fields the kernels do not know about (e.g. output fields) are gathered by torch
        known = {"status", *_lib.PARTICLE_POINTERS}
        perm64 = None
        for k, t in self.arrays.items():
            if k not in known:
                if perm64 is None:
                    perm64 = perm.to(torch.int64)
                torch.index_select(t, 0, perm64, out=spare[k])
        old = dict(self.arrays)
        object.__setattr__(self, "_arrays", types.MappingProxyType(dict(spare)))
        object.__setattr__(self, "_spare", old)
        object.__setattr__(self, "_order", new_order)
        object.__setattr__(self, "_range", id_bounds)
        object.__setattr__(self, "_abi_cache", None)
        for obs in sort_observers:
            obs()


class ParticlesView:
    """A read-only view of particle arrays; items are host numpy copies in original order."""

    __slots__ = ("_parent",)

    def __init__(self, parent: Particles) -> None:
        object.__setattr__(self, "_parent", parent)

    def __setattr__(self, name, value):
        raise AttributeError("ParticlesView is immutable")

    def __getitem__(self, name: str) -> np.ndarray:
        parent = object.__getattribute__(self, "_parent")
        if name not in parent:
            raise KeyError(name)
        parent.check_errors()
        arr = parent.original(name).cpu().numpy()
        arr.setflags(write=False)
        return arr

    def __getattr__(self, name: str) -> np.ndarray:
        try:
            return self[name]
        except KeyError:
            raise AttributeError(f"'ParticlesView' object has no attribute '{name}'")

    def __contains__(self, name: str) -> bool:
        return name in object.__getattribute__(self, "_parent")

    def tensor(self, name: str) -> torch.Tensor:
        """The device tensor of a particle field in STORAGE order (no copy; do not modify)."""
        return object.__getattribute__(self, "_parent").arrays[name]

    def device_original(self, name: str) -> torch.Tensor:
        """A device copy of a particle field in ORIGINAL order, queued on the current stream (no
        synchronisation, no error check: for asynchronous readers such as output writers)."""
        parent = object.__getattribute__(self, "_parent")
        if name not in parent:
            raise KeyError(name)
        return parent.original(name)

    @property
    def arrays(self) -> Mapping:
        return object.__getattribute__(self, "_parent").arrays

    @property
    def dtypes(self) -> Mapping[str, np.dtype]:
        return object.__getattribute__(self, "_parent").dtypes

    @property
    def shape(self) -> tuple[int, ...]:
        return object.__getattribute__(self, "_parent").shape

    @staticmethod
    def readonly_view(array) -> np.ndarray:
        view = np.asarray(array).view()
        view.setflags(write=False)
        return view

    def __len__(self) -> int:
        return len(object.__getattribute__(self, "_parent"))

    def __repr__(self) -> str:
        fields = ", ".join(f"{name}:{dtype}" for name, dtype in self.dtypes.items())
        return f"ParticlesView(shape={self.shape}, fields={{ {fields} }})"
