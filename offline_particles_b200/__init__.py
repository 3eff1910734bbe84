"""offline_particles_b200: the ROMS offline-particle advection step on NVIDIA B200.

A drop-in for the hot path of offline_particles (RK2 / AB3 w-advection with
trilinear interpolation on the Arakawa-C grid, time interpolation between
snapshots, the sigma-grid vertical search and the validation flags), with the
same Python API over hand-written sm_100a CUDA kernels reached through a C ABI
(include/opb200.h).  There is no CPU fallback.
"""

from . import kernels, output
from .events import Event, SimulationState
from .fields import BlendedArray, FieldData, StaticField, TimeDependentField
from .fieldset import Fieldset
from .models import roms
from .simulation import Checkpoint, Simulation, SimulationBuilder, load_checkpoint
from .spatial_arrays import DeviceArray, NumpyArray, Stagger
from .timesteppers import ABTimestepper, RK2Timestepper, Timestepper

__all__ = [
    "TimeDependentField",
    "StaticField",
    "FieldData",
    "BlendedArray",
    "Fieldset",
    "Simulation",
    "SimulationBuilder",
    "Checkpoint",
    "load_checkpoint",
    "Event",
    "SimulationState",
    "RK2Timestepper",
    "ABTimestepper",
    "Timestepper",
    "Stagger",
    "DeviceArray",
    "NumpyArray",
    "kernels",
    "output",
    "roms",
]


def build() -> None:
    """Compile the CUDA library (sm_100a) if it is missing or stale."""
    from ._build import build_library

    build_library()
