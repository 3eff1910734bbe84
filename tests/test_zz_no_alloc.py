"""opb_sort_particles_noalloc: the sort for callers that cannot allocate device memory.

Such callers (a runtime that reserved all device memory for its own pool, a
latency-critical loop where cudaMalloc / cudaFree would synchronise the device)
get the spatial-order permutation from a static device array inside the
library instead of a workspace they pass in.  This file is collected last so
that a run stopping at the first failure has run every other test before it;
it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _particles(n: int, seed: int):
    import torch

    from offline_particles_b200.particles import Particles

    rng = np.random.default_rng(seed)
    P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64)
    P["zidx"].copy_(torch.from_numpy(rng.uniform(-1, 51, n)))
    P["yidx"].copy_(torch.from_numpy(rng.uniform(-2, 770, n)))
    P["xidx"].copy_(torch.from_numpy(rng.uniform(-2, 1026, n)))
    st = np.zeros(n, np.uint8)
    st[rng.integers(0, n, n // 20)] = 0x81
    P["status"].copy_(torch.from_numpy(st))
    return P


def _reference_perm(lib, P, dims):
    """The permutation of the existing entry point (caller-allocated workspace)."""
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.kernels import _abi

    n = len(P)
    ws = torch.empty(lib.opb_sort_workspace_bytes(n), dtype=torch.uint8, device=P.device)
    perm = torch.empty(n, dtype=torch.int32, device=P.device)
    _lib.call("opb_sort_particles", ctypes.byref(_abi.particles_struct(P)), ctypes.byref(dims), perm.data_ptr(),
              ws.data_ptr(), ws.numel(), None)
    return perm.cpu().numpy()


def test_noalloc_sort_matches_workspace_sort_twice():
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.kernels import _abi

    lib = _lib.load()
    dims = (ctypes.c_int64 * 3)(50, 768, 1024)
    side = torch.cuda.Stream()
    for seed, n in ((1, 300_001), (2, _lib.NOALLOC_MAX_PARTICLES)):
        P = _particles(n, seed)
        ref = _reference_perm(lib, P, dims)
        for call, stream in enumerate((None, side)):  # two calls in a row share (and reuse) the static scratch
            perm = torch.full((n,), -1, dtype=torch.int32, device=P.device)
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            handle = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
            rc = lib.opb_sort_particles_noalloc(ctypes.byref(_abi.particles_struct(P)), ctypes.byref(dims),
                                                perm.data_ptr(), handle)
            assert rc == _lib.OK, lib.opb_last_error()
            torch.cuda.synchronize()
            if call > 0:  # the first call on a device may load the module; later calls allocate nothing
                assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
            got = perm.cpu().numpy()
            assert np.array_equal(got, ref), f"n={n} call {call}: permutation differs from opb_sort_particles"


def test_noalloc_sort_rejects_more_than_its_limit():
    import torch

    from offline_particles_b200 import _lib

    lib = _lib.load()
    n = _lib.NOALLOC_MAX_PARTICLES + 1
    p = _lib.opb_particles()
    p.n = n
    dims = (ctypes.c_int64 * 3)(50, 768, 1024)
    perm = torch.empty(1, dtype=torch.int32, device="cuda")
    rc = lib.opb_sort_particles_noalloc(ctypes.byref(p), ctypes.byref(dims), perm.data_ptr(), None)
    assert rc == _lib.EINVAL
    assert b"static scratch limit" in lib.opb_last_error()
