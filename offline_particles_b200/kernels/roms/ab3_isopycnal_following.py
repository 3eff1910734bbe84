"""AB3 isopycnal-following kernels (kernels/roms/ab3_isopycnal_following.pyx:1-311 of the reference).

The AB3 step of ab3_w_advection with the vertical velocity of a particle
that seeks its target density: dz/dt = w_max * drho / (rho_scale + |drho|),
drho = rho(x) - rho_t (ab3_isopycnal_following.pyx:5-11,124-132).  The
density field is a time-dependent field named ``rho`` at rho points; it is
passed to the C ABI in the w slot.  The post step is the same computation as
ab3_post_w_advection (:194-241).
"""

from __future__ import annotations

import numpy as np

from ... import _lib
from .. import _abi
from .._kernels import ParticleKernel

_ISO = ("u", "v", "rho", "dx", "dy", "h", "C", "zeta")
_SLOTS = ("u", "v", "w", "dx", "dy", "h", "C", "zeta")
_POS = ("h", "C", "zeta")


def ab3_isopycnal_following(particles, scalars, fielddata) -> None:
    """k0 at the current position (dz0 from the density); p += dt (23 k0 - 16 k1 + 5 k2) / 12
    (ab3_isopycnal_following.pyx:26-192)."""
    rf, t = _abi.roms_struct(fielddata, names=_SLOTS, sources={"w": "rho"})
    _lib.call("opb_ab3_isopycnal_following", _abi.byref(_abi.particles_struct(particles)),
              _abi.byref(_abi.scalars_struct(scalars)), _abi.byref(rf), _abi.byref(t), _abi.stream(particles))


def ab3_post_isopycnal_following(particles, scalars, fielddata) -> None:
    """zidx from z with zeta at the new time (ab3_isopycnal_following.pyx:194-241)."""
    rf, t = _abi.roms_struct(fielddata, names=_POS)
    _lib.call("opb_ab3_post_w_advection", _abi.byref(_abi.particles_struct(particles)),
              _abi.byref(_abi.scalars_struct(scalars)), _abi.byref(rf), _abi.byref(t), _abi.stream(particles))


ab3_isopycnal_following_kernel = ParticleKernel(
    ab3_isopycnal_following,
    particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64, "z": np.float64,
                     "rho_t": np.float64, "_dz0": np.float64, "_dz1": np.float64, "_dz2": np.float64,
                     "_dyidx0": np.float64, "_dyidx1": np.float64, "_dyidx2": np.float64, "_dxidx0": np.float64,
                     "_dxidx1": np.float64, "_dxidx2": np.float64},
    scalars={"_dt": np.float64, "hc": np.float64, "NZ": np.int32, "w_max": np.float64, "rho_scale": np.float64},
    simulation_fields=list(_ISO),
)
ab3_post_isopycnal_following_kernel = ParticleKernel(
    ab3_post_isopycnal_following,
    particle_fields={"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64,
                     "z": np.float64},
    scalars={"hc": np.float64, "NZ": np.int32},
    simulation_fields=list(_POS),
)
