"""Particles: a structure of arrays in device memory (particles.py:1-122 of the reference).

Each particle field is a 1-D CUDA tensor; the kernels mutate them in place.
``ParticlesView`` keeps the reference's read-only semantics: indexing it
returns a read-only host numpy copy (which synchronises); ``tensor(name)``
gives the device tensor itself without a copy.
"""

from __future__ import annotations

import types
from typing import Mapping

import numpy as np
import torch

from ._device import cuda_device, numpy_dtype, torch_dtype


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
        arrays = object.__getattribute__(self, "_arrays")
        public = [name for name in arrays if not name.startswith("_")]
        hidden = sum(1 for name in arrays if name.startswith("_"))
        hidden_str = f", +{hidden} hidden fields" if hidden > 1 else (", +1 hidden field" if hidden == 1 else "")
        return f"{self.__class__.__name__} (shape={self.shape}, fields=[{', '.join(public)}]{hidden_str})"


class Particles(_FrozenArrayMapping):
    """``nparticles`` particles with the given ``field=dtype`` arrays, zero-initialised on the device."""

    __slots__ = ("_length", "_device", "_err", "_abi_cache")

    def __init__(self, nparticles: int, *, device=None, **fields) -> None:
        dev = cuda_device(device)
        object.__setattr__(self, "_length", int(nparticles))
        object.__setattr__(self, "_device", dev)
        arrays = {f: torch.zeros((int(nparticles),), dtype=torch_dtype(dt), device=dev) for f, dt in fields.items()}
        super().__init__(**arrays)
        # device error word written by the kernels (OPB_ERRF_*)
        object.__setattr__(self, "_err", torch.zeros((1,), dtype=torch.int32, device=dev))
        object.__setattr__(self, "_abi_cache", None)

    def __len__(self) -> int:
        return object.__getattribute__(self, "_length")

    @property
    def device(self) -> torch.device:
        return object.__getattribute__(self, "_device")

    @property
    def error_word(self) -> torch.Tensor:
        return object.__getattribute__(self, "_err")

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


class ParticlesView(_FrozenArrayMapping):
    """A read-only view of particle arrays; items are host numpy copies."""

    __slots__ = ("_length", "_parent")

    def __init__(self, parent: Particles) -> None:
        object.__setattr__(self, "_length", len(parent))
        object.__setattr__(self, "_parent", parent)
        super().__init__(**dict(parent.arrays))

    def __getitem__(self, name: str) -> np.ndarray:
        parent = object.__getattribute__(self, "_parent")
        t = parent.arrays[name]
        parent.check_errors()
        arr = t.cpu().numpy()
        arr.setflags(write=False)
        return arr

    def tensor(self, name: str) -> torch.Tensor:
        """The device tensor of a particle field (no copy; do not modify)."""
        return object.__getattribute__(self, "_parent").arrays[name]

    @staticmethod
    def readonly_view(array) -> np.ndarray:
        view = np.asarray(array).view()
        view.setflags(write=False)
        return view

    def __len__(self) -> int:
        return object.__getattribute__(self, "_length")
