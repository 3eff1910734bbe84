"""Linear / bilinear / trilinear sampling of a field at the particles
(kernels/output/linear_interpolation.pyx:1-249 of the reference).

The field may be static or time-dependent; a time-dependent field is blended
per gathered corner in its storage dtype, which gives the values of the
reference's whole-grid blend.
"""

from __future__ import annotations

import ctypes
from functools import partial
from typing import Literal

import numpy as np

from ... import _lib
from ...fields import BlendedArray
from .. import _abi
from .._kernels import ParticleKernel


def _field_and_time(fd, nd: int, name: str):
    f = _abi.field_struct(fd, nd, name)
    t = _lib.opb_time(0, 1, 0.0, 1.0)
    if isinstance(fd.array, BlendedArray):
        t.ft, t.gt = float(fd.array.ft), float(fd.array.gt)
    return f, t


def linear_interpolation_kernel_function(particles, scalars, fielddata, dimension_idx, field_name, particle_name):
    """output = linear interpolation along one dimension (:34-68)."""
    f, t = _field_and_time(fielddata[field_name], 1, field_name)
    _lib.call("opb_linear_interpolation", ctypes.byref(_abi.particles_struct(particles)),
              _abi._ptr(particles[dimension_idx]), ctypes.byref(f), ctypes.byref(t),
              _abi._ptr(particles[particle_name]), _abi.stream(particles))


def bilinear_interpolation_kernel_function(particles, scalars, fielddata, dimension_idx0, dimension_idx1, field_name,
                                           particle_name):
    """output = bilinear interpolation over two dimensions (:70-103)."""
    f, t = _field_and_time(fielddata[field_name], 2, field_name)
    _lib.call("opb_bilinear_interpolation", ctypes.byref(_abi.particles_struct(particles)),
              _abi._ptr(particles[dimension_idx0]), _abi._ptr(particles[dimension_idx1]), ctypes.byref(f),
              ctypes.byref(t), _abi._ptr(particles[particle_name]), _abi.stream(particles))


def trilinear_interpolation_kernel_function(particles, scalars, fielddata, field_name, particle_name):
    """output = trilinear interpolation at (zidx, yidx, xidx) (:105-136)."""
    f, t = _field_and_time(fielddata[field_name], 3, field_name)
    _lib.call("opb_trilinear_interpolation", ctypes.byref(_abi.particles_struct(particles)), ctypes.byref(f),
              ctypes.byref(t), _abi._ptr(particles[particle_name]), _abi.stream(particles))


def linear_interpolation_kernel(field: str, output_name: str | None = None,
                                dimension: Literal["z", "y", "x"] = "z") -> ParticleKernel:
    if dimension not in {"z", "y", "x"}:
        raise ValueError(f"Invalid dimension: {dimension}. Valid options are 'z', 'y', or 'x'.")
    dimension_idx = dimension + "idx"
    output_name = field if output_name is None else output_name
    fn = partial(linear_interpolation_kernel_function, dimension_idx=dimension_idx, field_name=field,
                 particle_name=output_name)
    return ParticleKernel(fn, particle_fields={"status": np.uint8, dimension_idx: np.float64,
                                               output_name: np.float64},
                          scalars={}, simulation_fields=[field])


def bilinear_interpolation_kernel(field: str, output_name: str | None = None,
                                  dimensions: tuple[str, str] = ("y", "x")) -> ParticleKernel:
    valid = {("z", "y"), ("z", "x"), ("y", "x")}
    if dimensions not in valid:
        raise ValueError(f"Invalid dimensions: {dimensions}. Valid options are {valid}.")
    d0, d1 = dimensions[0] + "idx", dimensions[1] + "idx"
    output_name = field if output_name is None else output_name
    fn = partial(bilinear_interpolation_kernel_function, dimension_idx0=d0, dimension_idx1=d1, field_name=field,
                 particle_name=output_name)
    return ParticleKernel(fn, particle_fields={"status": np.uint8, d0: np.float64, d1: np.float64,
                                               output_name: np.float64},
                          scalars={}, simulation_fields=[field])


def trilinear_interpolation_kernel(field: str, output_name: str | None = None) -> ParticleKernel:
    output_name = field if output_name is None else output_name
    fn = partial(trilinear_interpolation_kernel_function, field_name=field, particle_name=output_name)
    return ParticleKernel(fn, particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64,
                                               "xidx": np.float64, output_name: np.float64},
                          scalars={}, simulation_fields=[field])


_SAMPLERS = (linear_interpolation_kernel_function, bilinear_interpolation_kernel_function,
             trilinear_interpolation_kernel_function)


def samples_only(kernel: ParticleKernel, protected) -> bool:
    """True when every function of ``kernel`` samples a field at the particles into a particle field that is
    not in ``protected`` (such a kernel reads only the status and indices and writes only its output)."""
    for fn in kernel.functions:
        if not (isinstance(fn, partial) and fn.func in _SAMPLERS):
            return False
        if fn.keywords.get("particle_name") in protected:
            return False
    return True


def vertical_interpolation_kernel(field: str, output_name: str | None = None) -> ParticleKernel:
    return linear_interpolation_kernel(field, output_name, dimension="z")


def horizontal_interpolation_kernel(field: str, output_name: str | None = None) -> ParticleKernel:
    return bilinear_interpolation_kernel(field, output_name, dimensions=("y", "x"))
