"""Output kernels: sample fields at particle positions (kernels/output/ of the reference)."""

from .linear_interpolation import (
    bilinear_interpolation_kernel,
    bilinear_interpolation_kernel_function,
    horizontal_interpolation_kernel,
    linear_interpolation_kernel,
    linear_interpolation_kernel_function,
    trilinear_interpolation_kernel,
    trilinear_interpolation_kernel_function,
    vertical_interpolation_kernel,
)

__all__ = [
    "linear_interpolation_kernel_function",
    "bilinear_interpolation_kernel_function",
    "trilinear_interpolation_kernel_function",
    "linear_interpolation_kernel",
    "bilinear_interpolation_kernel",
    "trilinear_interpolation_kernel",
    "vertical_interpolation_kernel",
    "horizontal_interpolation_kernel",
]
