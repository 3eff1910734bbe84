"""Validation kernels: the non-finite and out-of-domain status flags (kernels/validation.pyx:1-124).

``finite_indices`` sets NONFINITE (0x81) on active particles with a
non-finite index; ``domain_bounds`` sets OUT_OF_DOMAIN (0x82) on active
particles outside ``[*idx_min, *idx_max]``.  The reference has no land mask: a
particle on land keeps moving with whatever velocity the fields hold there
(zero, or NaN, which the next validation turns into NONFINITE).
"""

from __future__ import annotations

import numpy as np

from .. import _lib
from . import _abi
from ._kernels import ParticleKernel

__all__ = ["finite_indices", "domain_bounds", "finite_indices_kernel", "domain_bounds_kernel", "validation_kernel"]


def finite_indices(particles, scalars, fielddata) -> None:
    """validation.pyx:21-43 on the device."""
    _lib.call("opb_finite_indices", _abi.byref(_abi.particles_struct(particles)), _abi.stream(particles))


def domain_bounds(particles, scalars, fielddata) -> None:
    """validation.pyx:45-77 on the device."""
    _lib.call("opb_domain_bounds", _abi.byref(_abi.particles_struct(particles)),
              _abi.byref(_abi.scalars_struct(scalars)), _abi.stream(particles))


finite_indices_kernel = ParticleKernel(
    finite_indices,
    particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64},
    scalars={},
    simulation_fields=[],
)
domain_bounds_kernel = ParticleKernel(
    domain_bounds,
    particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64},
    scalars={"zidx_min": np.float64, "zidx_max": np.float64, "yidx_min": np.float64, "yidx_max": np.float64,
             "xidx_min": np.float64, "xidx_max": np.float64},
    simulation_fields=[],
)
validation_kernel = ParticleKernel.chain(finite_indices_kernel, domain_bounds_kernel)
