"""ROMS timestepper presets (models/roms/__init__.py:1-140 of the reference).

Same factories, keywords and defaults (``index_padding=5``, ``alpha=2/3``,
the validation kernel as pre-step).  Steppers built here run each step as one
fused CUDA launch.
"""

from __future__ import annotations

import numpy as np
import numpy.typing as npt

from ...kernels.roms import (
    ab3_isopycnal_following_kernel,
    ab3_post_isopycnal_following_kernel,
    ab3_post_w_advection_kernel,
    ab3_w_advection_kernel,
    compute_z_kernel,
    rk2_w_advection_step_1_kernel,
    rk2_w_advection_step_2_kernel,
    rk2_w_advection_update_kernel,
)
from ...kernels.validation import validation_kernel
from ...timesteppers import ABTimestepper, RK2Timestepper

__all__ = [
    "compute_z_kernel",
    "ab3_isopycnal_following_kernel",
    "ab3_post_isopycnal_following_kernel",
    "ab3_isopycnal_following_timestepper",
    "ab3_w_advection_kernel",
    "ab3_post_w_advection_kernel",
    "ab3_w_advection_timestepper",
    "rk2_w_advection_step_1_kernel",
    "rk2_w_advection_step_2_kernel",
    "rk2_w_advection_update_kernel",
    "rk2_w_advection_timestepper",
]

type D = np.float64 | np.timedelta64
type T = np.float64 | np.datetime64


def rk2_w_advection_timestepper(time_array: npt.NDArray, dt: D, *, time: T | None = None,
                                time_unit: D | None = None, iteration: int = 0, index_padding: int = 5,
                                alpha: float = 2 / 3) -> RK2Timestepper:
    """RK2 timestepper with the ROMS w-advection kernels and the validation pre-step."""
    return RK2Timestepper(
        time_array, dt,
        rk_step_1_kernel=rk2_w_advection_step_1_kernel,
        rk_step_2_kernel=rk2_w_advection_step_2_kernel,
        rk_update_kernel=rk2_w_advection_update_kernel,
        time=time, time_unit=time_unit, iteration=iteration, index_padding=index_padding, alpha=alpha,
        pre_step_kernel=validation_kernel,
    )


def ab3_w_advection_timestepper(time_array: npt.NDArray, dt: D, *, time: T | None = None,
                                time_unit: D | None = None, iteration: int = 0,
                                index_padding: int = 5) -> ABTimestepper:
    """AB3 timestepper with the ROMS w-advection kernels, validation pre-step and zidx post-step."""
    return ABTimestepper(
        time_array, dt,
        ab_kernel=ab3_w_advection_kernel,
        time=time, time_unit=time_unit, iteration=iteration, index_padding=index_padding,
        pre_step_kernel=validation_kernel,
        post_step_kernel=ab3_post_w_advection_kernel,
    )


def ab3_isopycnal_following_timestepper(time_array: npt.NDArray, dt: D, *, time: T | None = None,
                                        time_unit: D | None = None, iteration: int = 0,
                                        index_padding: int = 5) -> ABTimestepper:
    """AB3 timestepper with the ROMS isopycnal-following kernels, validation pre-step and zidx post-step
    (models/roms/__init__.py:109-141 of the reference).  The fieldset needs a time-dependent ``rho`` and
    the constants ``w_max`` and ``rho_scale``; particles carry ``rho_t``."""
    return ABTimestepper(
        time_array, dt,
        ab_kernel=ab3_isopycnal_following_kernel,
        time=time, time_unit=time_unit, iteration=iteration, index_padding=index_padding,
        pre_step_kernel=validation_kernel,
        post_step_kernel=ab3_post_isopycnal_following_kernel,
    )
