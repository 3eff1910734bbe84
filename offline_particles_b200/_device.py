"""CUDA device and stream plumbing (PyTorch is used for device memory and streams only)."""

from __future__ import annotations

import torch


def cuda_device(device=None) -> torch.device:
    """The CUDA device to use; raises if there is none (no CPU fallback)."""
    if not torch.cuda.is_available():
        raise RuntimeError("offline_particles_b200 runs on a CUDA device (B200, sm_100a); none is available")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"offline_particles_b200 keeps its data on a CUDA device, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def stream_handle(device: torch.device | None = None) -> int:
    """cudaStream_t of the current torch stream on ``device`` (the raw-handle query where torch offers
    it: the launch path asks for it several times per launch)."""
    if _raw_stream is not None:
        index = device.index if isinstance(device, torch.device) and device.index is not None else (
            torch.cuda.current_device() if device is None else torch.device(device).index)
        if index is not None:
            return _raw_stream(index)
    return torch.cuda.current_stream(device).cuda_stream


def torch_dtype(np_dtype) -> torch.dtype:
    import numpy as np

    d = np.dtype(np_dtype)
    table = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
             np.dtype(np.float16): torch.float16, np.dtype(np.uint8): torch.uint8,
             np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}
    if d not in table:
        raise TypeError(f"unsupported dtype {d}")
    return table[d]


def numpy_dtype(t: torch.dtype):
    import numpy as np

    table = {torch.float64: np.float64, torch.float32: np.float32, torch.float16: np.float16, torch.uint8: np.uint8,
             torch.int32: np.int32, torch.int64: np.int64}
    return np.dtype(table[t])
