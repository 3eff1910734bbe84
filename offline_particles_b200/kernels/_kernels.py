"""ParticleKernel: a named device kernel with its declared requirements.

Same object model as kernels/_kernels.py:1-149 of the reference: a kernel is a
tuple of functions ``fn(particles, scalars, fielddata) -> None`` plus the
particle fields, scalars and simulation fields it needs; ``chain`` merges
kernels.  Here each ``fn`` is a thin host function that marshals its
arguments into the C ABI of include/opb200.h and launches CUDA work on the
current stream.
"""

from __future__ import annotations

import types
from typing import Callable, Iterable, Mapping, Self

import numpy as np
import numpy.typing as npt

type KernelFunction = Callable[..., None]

DEFAULT_PARTICLE_FIELDS: dict[str, np.dtype] = {
    "status": np.dtype(np.uint8),
    "zidx": np.dtype(np.float64),
    "yidx": np.dtype(np.float64),
    "xidx": np.dtype(np.float64),
}


class ParticleKernel:
    """A kernel to be executed on particles."""

    def __init__(
        self,
        fn: KernelFunction | Iterable[KernelFunction],
        particle_fields: Mapping[str, npt.DTypeLike],
        scalars: Mapping[str, npt.DTypeLike],
        simulation_fields: Iterable[str],
    ):
        funcs = (fn,) if callable(fn) else tuple(fn)
        if not all(callable(f) for f in funcs):
            raise TypeError("All kernel functions must be callable")
        self._funcs: tuple[KernelFunction, ...] = funcs
        self._particle_fields = {field: np.dtype(dtype) for field, dtype in particle_fields.items()}
        self._scalars = {scalar: np.dtype(dtype) for scalar, dtype in scalars.items()}
        self._simulation_fields = frozenset(simulation_fields)

    @property
    def particle_fields(self) -> Mapping[str, np.dtype]:
        return types.MappingProxyType(self._particle_fields)

    @property
    def scalars(self) -> Mapping[str, np.dtype]:
        return types.MappingProxyType(self._scalars)

    @property
    def simulation_fields(self) -> frozenset[str]:
        return self._simulation_fields

    @property
    def functions(self) -> tuple[KernelFunction, ...]:
        return self._funcs

    @staticmethod
    def func_name(fn: KernelFunction) -> str:
        return getattr(fn, "__qualname__", getattr(fn, "__name__", repr(fn)))

    def __repr__(self) -> str:
        funcs = ", ".join(self.func_name(fn) for fn in self._funcs)
        return (f"{self.__class__.__name__}(funcs=[{funcs}], particle_fields={list(self._particle_fields)}, "
                f"scalars={list(self._scalars)}, simulation_fields={sorted(self._simulation_fields)})")

    def __str__(self) -> str:
        return "Particle Kernel: " + " → ".join(self.func_name(fn) for fn in self._funcs)

    def __call__(self, particles, scalars, fielddata) -> None:
        for fn in self._funcs:
            fn(particles, scalars, fielddata)

    @classmethod
    def chain(cls, *kernels: Self) -> Self:
        funcs = tuple(fn for kernel in kernels for fn in kernel._funcs)
        return cls(funcs, merge_particle_fields(kernels), merge_scalars(kernels), merge_simulation_fields(kernels))

    def chain_with(self, *others: Self) -> Self:
        return self.__class__.chain(self, *others)


def merge_particle_fields(kernels: Iterable[ParticleKernel]) -> dict[str, np.dtype]:
    merged: dict[str, np.dtype] = DEFAULT_PARTICLE_FIELDS.copy()
    for kernel in kernels:
        for field, dtype in kernel.particle_fields.items():
            if field in merged:
                if merged[field] != dtype:
                    raise TypeError(f"Conflicting dtypes for particle field '{field}': {merged[field]} vs {dtype}")
            else:
                merged[field] = dtype
    return merged


def merge_scalars(kernels: Iterable[ParticleKernel]) -> dict[str, np.dtype]:
    merged: dict[str, np.dtype] = {}
    for kernel in kernels:
        for scalar, dtype in kernel.scalars.items():
            if scalar in merged:
                if merged[scalar] != dtype:
                    raise TypeError(f"Conflicting dtypes for scalar '{scalar}': {merged[scalar]} vs {dtype}")
            else:
                merged[scalar] = dtype
    return merged


def merge_simulation_fields(kernels: Iterable[ParticleKernel]) -> frozenset[str]:
    merged: set[str] = set()
    for kernel in kernels:
        merged.update(kernel.simulation_fields)
    return frozenset(merged)
