"""compute_z kernel (kernels/roms/_roms_core.pyx:17-112 of the reference)."""

from __future__ import annotations

import functools

import numpy as np

from ... import _lib
from .. import _abi
from .._kernels import ParticleKernel


def compute_z_kernel_function(particles, scalars, fielddata, particle_field: str = "z") -> None:
    """z = zeta + (zeta + h) S(zidx) for active particles, into ``particle_field``."""
    out = particles[particle_field]
    rf, t = _abi.roms_struct(fielddata, names=("h", "zeta", "C"))
    _lib.call("opb_compute_z", _abi.byref(_abi.particles_struct(particles)), _abi._ptr(out),
              _abi.byref(_abi.scalars_struct(scalars)), _abi.byref(rf), _abi.byref(t), _abi.stream(particles))


def compute_z_kernel(particle_field: str = "z") -> ParticleKernel:
    """A kernel that computes the physical vertical coordinate into ``particle_field``."""
    fn = functools.partial(compute_z_kernel_function, particle_field=particle_field)
    fn.__qualname__ = "compute_z_kernel_function"  # type: ignore[attr-defined]
    return ParticleKernel(
        fn,
        particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64,
                         particle_field: np.float64},
        scalars={"hc": np.float64, "NZ": np.int32},
        simulation_fields=["h", "C", "zeta"],
    )
