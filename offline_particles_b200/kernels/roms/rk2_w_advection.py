"""RK2 w-advection kernels (kernels/roms/rk2_w_advection.pyx:1-455 of the reference).

Horizontal advection in index space; vertical advection in physical space
with w, converted back to a sigma index through the sigma-grid search.
"""

from __future__ import annotations

import numpy as np

from ... import _lib
from .. import _abi
from .._kernels import ParticleKernel

__all__ = ["rk2_w_advection_step_1", "rk2_w_advection_step_2", "rk2_w_advection_update",
           "rk2_w_advection_step_1_kernel", "rk2_w_advection_step_2_kernel", "rk2_w_advection_update_kernel"]

_VEL = ("u", "v", "w", "dx", "dy", "h", "C", "zeta")
_POS = ("h", "C", "zeta")


def _launch(name: str, particles, scalars, fielddata, names) -> None:
    rf, t = _abi.roms_struct(fielddata, names=names)
    _lib.call(name, _abi.byref(_abi.particles_struct(particles)), _abi.byref(_abi.scalars_struct(scalars)),
              _abi.byref(rf), _abi.byref(t), _abi.stream(particles))


def rk2_w_advection_step_1(particles, scalars, fielddata) -> None:
    """First stage: z from zidx, k1 = (u/dx, v/dy, w) (rk2_w_advection.pyx:31-153)."""
    _launch("opb_rk2_w_advection_step_1", particles, scalars, fielddata, _VEL)


def rk2_w_advection_step_2(particles, scalars, fielddata) -> None:
    """Second stage at p + alpha dt k1 (rk2_w_advection.pyx:155-275)."""
    _launch("opb_rk2_w_advection_step_2", particles, scalars, fielddata, _VEL)


def rk2_w_advection_update(particles, scalars, fielddata) -> None:
    """p += b1 dt k1 + b2 dt k2, b1 = 1/(2 alpha); zidx from z (rk2_w_advection.pyx:278-354)."""
    _launch("opb_rk2_w_advection_update", particles, scalars, fielddata, _POS)


_STAGE_FIELDS = {"status": np.uint8, "zidx": np.float64, "yidx": np.float64, "xidx": np.float64, "z": np.float64,
                 "_dxidx1": np.float64, "_dyidx1": np.float64, "_dz1": np.float64}
_ALL_FIELDS = dict(_STAGE_FIELDS, _dxidx2=np.float64, _dyidx2=np.float64, _dz2=np.float64)

rk2_w_advection_step_1_kernel = ParticleKernel(
    rk2_w_advection_step_1, particle_fields=_STAGE_FIELDS, scalars={"hc": np.float64, "NZ": np.int32},
    simulation_fields=list(_VEL))
rk2_w_advection_step_2_kernel = ParticleKernel(
    rk2_w_advection_step_2, particle_fields=_ALL_FIELDS,
    scalars={"_dt": np.float64, "_RK2_alpha": np.float64, "hc": np.float64, "NZ": np.int32},
    simulation_fields=list(_VEL))
rk2_w_advection_update_kernel = ParticleKernel(
    rk2_w_advection_update, particle_fields=_ALL_FIELDS,
    scalars={"_dt": np.float64, "_RK2_alpha": np.float64, "hc": np.float64, "NZ": np.int32},
    simulation_fields=list(_POS))
