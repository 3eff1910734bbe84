"""Kernel launcher: resolves a kernel's scalars and fields and calls it (launcher.py:1-194 of the reference)."""

from __future__ import annotations

from typing import Callable, TypeVar

import numpy as np
import torch

from .fields import FieldData
from .fieldset import Fieldset
from .kernels import ParticleKernel
from .spatial_arrays import BBox

T = TypeVar("T", bound=np.number)


class ScalarSource[T]:
    """Descriptor declaring a scalar data source; the getter is ``(self, tidx) -> value``."""

    def __init__(self, name: str, getter: Callable[[object, float], T]) -> None:
        self.name = name
        self._getter = getter

    def __get__(self, obj: object | None, owner: type | None = None):
        if obj is None:
            return self

        def scalar_func(tidx: float) -> T:
            return self._getter(obj, tidx)

        return scalar_func


type ScalarProvider = Callable[[float], np.number]


class Launcher:
    """Launches particle kernels against a fieldset.

    Unlike the reference, ``launch_kernel`` does not build a particle bounding
    box: the fields are whole on the device, so the per-launch O(N) min/max
    (launcher.py:122-148) has no use.  ``construct_bbox`` remains available.
    """

    def __init__(self, fieldset: Fieldset, *, index_padding: int = 0, arithmetic: str = "float64") -> None:
        """``arithmetic``: "float64" (bit-identical to the reference) or "float32" (the reduced-precision
        fused steppers; needed for bfloat16/float16 field storage)."""
        if arithmetic not in ("float64", "float32"):
            raise ValueError("arithmetic must be 'float64' or 'float32'")
        self.arithmetic = arithmetic
        self._scalar_data_sources: dict[str, ScalarProvider] = {}
        self._fieldset = fieldset
        if index_padding < 0:
            raise ValueError("index_padding must be non-negative")
        self._index_padding = index_padding
        for name, value in self._fieldset.constants.items():
            self.register_scalar_data_source(name, self.create_value_scalar_source(value))

    @property
    def fieldset(self) -> Fieldset:
        return self._fieldset

    @staticmethod
    def create_value_scalar_source(value) -> ScalarProvider:
        def value_func(tidx: float):
            return value

        return value_func

    def register_scalar_data_source(self, name: str, source: ScalarProvider) -> None:
        if name in self._scalar_data_sources:
            raise ValueError(
                f"Scalar data source '{name}' is already registered. Deregister it before registering a new one.")
        if name in self._fieldset.fields:
            raise ValueError(f"Scalar data source '{name}' conflicts with a field in the fieldset.")
        self._scalar_data_sources[name] = source

    def deregister_scalar_data_source(self, name: str) -> None:
        if name not in self._scalar_data_sources:
            raise ValueError(f"Scalar data source '{name}' is not registered.")
        del self._scalar_data_sources[name]

    def register_scalar_data_sources_from_object(self, obj: object) -> None:
        for attr_name in dir(type(obj)):
            attr = getattr(type(obj), attr_name)
            if isinstance(attr, ScalarSource):
                self.register_scalar_data_source(attr.name, getattr(obj, attr_name))

    @property
    def index_padding(self) -> int:
        return self._index_padding

    def maybe_increase_index_padding(self, padding: int) -> None:
        if padding > self._index_padding:
            self._index_padding = padding

    def construct_bbox(self, particles) -> BBox:
        """Padded bounding box of the particle indices (one device reduction per dimension)."""
        pad = self._index_padding
        vals = []
        for name in ("zidx", "yidx", "xidx"):
            t = particles[name]
            mm = torch.aminmax(t) if isinstance(t, torch.Tensor) else (np.min(t), np.max(t))
            vals += [float(mm[0]) - pad, float(mm[1]) + pad]
        return BBox(*vals)

    def scalars(self, kernel: ParticleKernel, time_index) -> dict:
        return {name: self._scalar_data_sources[name](time_index) for name in kernel.scalars}

    def scalar(self, name: str, time_index):
        return self._scalar_data_sources[name](time_index)

    def get_field_data(self, name: str, time_index: float, bbox: BBox | None = None) -> FieldData:
        return self._fieldset[name].get_field_data(time_index, bbox)

    def launch_kernel(self, kernel: ParticleKernel, particles, time_index: float) -> None:
        """Resolve the kernel's scalars and fields at ``time_index`` and call it."""
        scalars = self.scalars(kernel, time_index)
        fielddata = {name: self.get_field_data(name, time_index) for name in kernel.simulation_fields}
        kernel(particles, scalars, fielddata)
