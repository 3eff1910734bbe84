"""AB3 w-advection kernels (kernels/roms/ab3_w_advection.pyx:1-295 of the reference).

Third-order Adams-Bashforth with a forward-Euler / AB2 bootstrap driven by
the MULTISTEP_1 -> MULTISTEP_2 -> NORMAL status sequence.
"""

from __future__ import annotations

import numpy as np

from ... import _lib
from .. import _abi
from .._kernels import ParticleKernel

_VEL = ("u", "v", "w", "dx", "dy", "h", "C", "zeta")
_POS = ("h", "C", "zeta")


def ab3_w_advection(particles, scalars, fielddata) -> None:
    """k0 at the current position; p += dt (23 k0 - 16 k1 + 5 k2) / 12 (ab3_w_advection.pyx:20-178)."""
    rf, t = _abi.roms_struct(fielddata, names=_VEL)
    _lib.call("opb_ab3_w_advection", _abi.byref(_abi.particles_struct(particles)),
              _abi.byref(_abi.scalars_struct(scalars)), _abi.byref(rf), _abi.byref(t), _abi.stream(particles))


def ab3_post_w_advection(particles, scalars, fielddata) -> None:
    """zidx from z with zeta at the new time (ab3_w_advection.pyx:180-229)."""
    rf, t = _abi.roms_struct(fielddata, names=_POS)
    _lib.call("opb_ab3_post_w_advection", _abi.byref(_abi.particles_struct(particles)),
              _abi.byref(_abi.scalars_struct(scalars)), _abi.byref(rf), _abi.byref(t), _abi.stream(particles))


ab3_w_advection_kernel = ParticleKernel(
    ab3_w_advection,
    particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64, "z": np.float64,
                     "_dz0": np.float64, "_dz1": np.float64, "_dz2": np.float64, "_dyidx0": np.float64,
                     "_dyidx1": np.float64, "_dyidx2": np.float64, "_dxidx0": np.float64, "_dxidx1": np.float64,
                     "_dxidx2": np.float64},
    scalars={"_dt": np.float64, "hc": np.float64, "NZ": np.int32},
    simulation_fields=list(_VEL),
)
ab3_post_w_advection_kernel = ParticleKernel(
    ab3_post_w_advection,
    particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64,
                     "z": np.float64},
    scalars={"hc": np.float64, "NZ": np.int32},
    simulation_fields=list(_POS),
)
