"""ROMS kernels (kernels/roms/__init__.py of the reference)."""

from ._roms_core import compute_z_kernel
from .ab3_isopycnal_following import ab3_isopycnal_following_kernel, ab3_post_isopycnal_following_kernel
from .ab3_w_advection import ab3_post_w_advection_kernel, ab3_w_advection_kernel
from .rk2_w_advection import (
    rk2_w_advection_step_1_kernel,
    rk2_w_advection_step_2_kernel,
    rk2_w_advection_update_kernel,
)

__all__ = [
    "compute_z_kernel",
    "ab3_isopycnal_following_kernel",
    "ab3_post_isopycnal_following_kernel",
    "ab3_w_advection_kernel",
    "ab3_post_w_advection_kernel",
    "rk2_w_advection_step_1_kernel",
    "rk2_w_advection_step_2_kernel",
    "rk2_w_advection_update_kernel",
]
