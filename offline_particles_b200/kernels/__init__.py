"""Particle kernels (kernels/__init__.py of the reference)."""

from ._kernels import (
    DEFAULT_PARTICLE_FIELDS,
    KernelFunction,
    ParticleKernel,
    merge_particle_fields,
    merge_scalars,
    merge_simulation_fields,
)
from .status import ParticleStatus

__all__ = [
    "DEFAULT_PARTICLE_FIELDS",
    "ParticleKernel",
    "KernelFunction",
    "ParticleStatus",
    "merge_particle_fields",
    "merge_scalars",
    "merge_simulation_fields",
]
