"""Marshal ``(particles, scalars, fielddata)`` into the C-ABI structs of include/opb200.h."""

from __future__ import annotations

import ctypes
from typing import Mapping

import numpy as np
import torch

from .. import _lib
from .._device import stream_handle
from ..fields import BlendedArray, FieldData

ROMS_FIELDS = ("u", "v", "w", "dx", "dy", "h", "zeta", "C")
ROMS_NDIM = {"u": 3, "v": 3, "w": 3, "dx": 2, "dy": 2, "h": 2, "zeta": 2, "C": 1}


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("particle and field arrays must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("particle and field arrays must be contiguous")
    return t.data_ptr()


def particles_struct_for(arrays: Mapping[str, torch.Tensor], n: int, err: torch.Tensor | None = None
                         ) -> _lib.opb_particles:
    """opb_particles over a dict of particle-field tensors."""
    kw = {}
    for name in _lib.PARTICLE_POINTERS:
        t = arrays.get(name)
        if t is not None and t.dtype != torch.float64:
            raise TypeError(f"particle field {name} must be float64")
        kw[name.lstrip("_")] = _ptr(t)
    status = arrays["status"]
    if status.dtype != torch.uint8:
        raise TypeError("particle field status must be uint8")
    if status.shape[0] != n:
        raise ValueError("particle arrays do not match the particle count")
    rho_t = arrays.get("rho_t")
    if rho_t is not None and rho_t.dtype != torch.float64:
        raise TypeError("particle field rho_t must be float64")
    return _lib.opb_particles(n=n, status=_ptr(status), err=_ptr(err), rho_t=_ptr(rho_t), **kw)


def particles_struct(particles) -> _lib.opb_particles:
    """opb_particles for a Particles object (cached until its storage is reordered)."""
    cached = hasattr(type(particles), "_abi_cache")
    if cached:
        cache = object.__getattribute__(particles, "_abi_cache")
        if cache is not None:
            return cache
    s = particles_struct_for(particles.arrays, particles.arrays["status"].shape[0],
                             getattr(particles, "error_word", None))
    if cached:
        object.__setattr__(particles, "_abi_cache", s)
    return s


def particles_struct_range(particles, lo: int, hi: int) -> _lib.opb_particles:
    """opb_particles over storage slots ``[lo, hi)`` of a Particles object (the same arrays, offset; the
    error word is shared)."""
    full = particles_struct(particles)
    if not 0 <= lo <= hi <= full.n:
        raise ValueError(f"slots [{lo}, {hi}) outside 0..{full.n}")
    s = _lib.opb_particles(n=hi - lo, err=full.err)
    s.status = None if full.status is None else full.status + lo
    for name in ("rho_t", *(p.lstrip("_") for p in _lib.PARTICLE_POINTERS)):
        ptr = getattr(full, name)
        setattr(s, name, None if ptr is None else ptr + 8 * lo)
    return s


def scalars_struct(scalars: Mapping[str, object]) -> _lib.opb_scalars:
    s = _lib.opb_scalars()
    s.hc = float(scalars.get("hc", 0.0))
    s.NZ = int(scalars.get("NZ", 0))
    s.dt = float(scalars.get("_dt", 0.0))
    s.alpha = float(scalars.get("_RK2_alpha", 0.0))
    for k, name in enumerate(("zidx_min", "zidx_max", "yidx_min", "yidx_max", "xidx_min", "xidx_max")):
        s.bounds[k] = float(scalars.get(name, 0.0))
    s.w_max = float(scalars.get("w_max", 0.0))
    s.rho_scale = float(scalars.get("rho_scale", 0.0))
    return s


def _dtype_code(dt) -> int:
    dt = np.dtype(dt)
    if dt == np.float64:
        return _lib.F64
    if dt == np.float32:
        return _lib.F32
    raise TypeError(f"unsupported storage dtype {dt}")


def field_struct(fd: FieldData, ndim: int, name: str, slots: dict[int, int] | None = None) -> _lib.opb_field:
    """opb_field for one FieldData.  ``slots`` maps snapshot index -> slot (fused launches)."""
    f = _lib.opb_field()
    arr, offsets = fd
    if isinstance(arr, BlendedArray):
        f.is_static = 0
        f.dtype = _dtype_code(arr.dtype)
        f.data[0] = _ptr(arr.prev)
        f.data[1] = _ptr(arr.next)
        f.nslots = 2
        shape = arr.shape
    else:
        if not isinstance(arr, torch.Tensor) or arr.dtype != torch.float64:
            raise TypeError(f"field '{name}': static field data must be a float64 CUDA tensor")
        f.is_static = 1
        f.dtype = _lib.F64
        f.data[0] = _ptr(arr)
        f.nslots = 1
        shape = tuple(arr.shape)
    if len(shape) != ndim or len(offsets) != ndim:
        raise ValueError(f"field '{name}' must have {ndim} active dimensions, got shape {shape}")
    for d in range(ndim):
        f.shape[d] = int(shape[d])
        f.offset[d] = float(offsets[d])
    f.ndim = ndim
    return f


def roms_struct(fielddata: Mapping[str, FieldData], names=ROMS_FIELDS,
                sources: Mapping[str, str] | None = None) -> tuple[_lib.opb_roms_fields, _lib.opb_time]:
    """opb_roms_fields + opb_time for one launch (all time-dependent fields at one time index).  ``names``:
    the slots the kernel reads; ``sources``: slot -> fielddata key where they differ (the isopycnal
    follower's density in the w slot)."""
    rf = _lib.opb_roms_fields()
    t = _lib.opb_time(0, 1, 0.0, 1.0)
    weights = None
    sources = sources or {}
    for name in ROMS_FIELDS:
        if name not in names:
            # unused by this kernel: a placeholder static field
            g = getattr(rf, name)
            g.is_static = 1
            g.ndim = ROMS_NDIM[name]
            continue
        fd = fielddata[sources.get(name, name)]
        setattr(rf, name, field_struct(fd, ROMS_NDIM[name], name))
        if isinstance(fd.array, BlendedArray):
            w = (fd.array.It, float(fd.array.ft), float(fd.array.gt), np.dtype(fd.array.dtype))
            if weights is None:
                weights = w
            elif weights != w:
                raise ValueError("time-dependent fields of one launch must share time index and storage dtype")
    if weights is not None:
        t.ft, t.gt = weights[1], weights[2]
    return rf, t


def stream(particles=None) -> int:
    dev = particles.device if particles is not None and hasattr(particles, "device") else None
    return stream_handle(dev)


def byref(x):
    return ctypes.byref(x)
