"""Spatial ordering of particle storage: permutation, gather, and unchanged results."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from b200_runner import run_b200
from helpers import CASES, load, mismatch_report, same_bits
from offline_particles_b200.synth import SyntheticROMS

pytestmark = pytest.mark.gpu


def spread3(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & 0x3FF
    out = np.zeros_like(v)
    for b in range(10):
        out |= ((v >> b) & 1) << (3 * b)
    return out


def host_keys(status, z, y, x, shape):
    """Morton keys as include/opb200.h documents them (x quantised by 4, each dim under 2^10)."""
    def shift(n, extra):
        bits = int(np.ceil(np.log2(n))) if n > 1 else 0
        s = extra
        while bits - s > 10:
            s += 1
        return s

    def cell(idx, n, sh):
        c = np.where((idx >= 0) & (idx < 9e18), np.floor(np.nan_to_num(idx, nan=0.0, posinf=0, neginf=0)), 0)
        c = np.minimum(c.astype(np.int64), n - 1)
        return (c >> sh).astype(np.uint64)

    nz, ny, nx = shape
    key = (spread3(cell(z, nz, shift(nz, 0))) << 2) | (spread3(cell(y, ny, shift(ny, 0))) << 1) | spread3(
        cell(x, nx, shift(nx, 2)))
    return np.where(status & 0x80, np.uint64(0xFFFFFFFF), key)


def test_sort_permutation_and_gather():
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.kernels import _abi
    from offline_particles_b200.particles import Particles

    rng = np.random.default_rng(3)
    n, shape = 100_003, (50, 768, 1024)
    z = rng.uniform(-1, 50, n)
    y = rng.uniform(-3, 770, n)
    x = rng.uniform(-3, 1030, n)
    z[:5] = [np.nan, np.inf, -np.inf, 1e300, -1e300]
    st = np.zeros(n, np.uint8)
    st[rng.integers(0, n, 5000)] = 0x82
    P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64, z=np.float64,
                  _dz0=np.float64, extra=np.float32)
    for name, v in (("zidx", z), ("yidx", y), ("xidx", x), ("status", st)):
        P[name].copy_(torch.from_numpy(v))
    P["z"].copy_(torch.arange(n, dtype=torch.float64))
    P["extra"].copy_(torch.arange(n, dtype=torch.float32))
    lib = _lib.load()
    ws = torch.empty(lib.opb_sort_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    dims = (ctypes.c_int64 * 3)(*shape)
    _lib.call("opb_sort_particles", ctypes.byref(_abi.particles_struct(P)), ctypes.byref(dims), perm.data_ptr(),
              ws.data_ptr(), ws.numel(), None)
    p = perm.cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(p), np.arange(n))
    keys = host_keys(st, z, y, x, shape)
    assert np.all(np.diff(keys[p].astype(np.int64)) >= 0), "not in key order"
    same = np.diff(keys[p].astype(np.int64)) == 0
    assert np.all(np.diff(p)[same] > 0), "ties not in index order (sort must be stable)"
    assert np.all(st[p][-int((st & 0x80).astype(bool).sum()):] & 0x80), "inactive particles must come last"
    # workspace too small is an argument error
    assert lib.opb_sort_particles(ctypes.byref(_abi.particles_struct(P)), ctypes.byref(dims), perm.data_ptr(),
                                  ws.data_ptr(), 16, None) == _lib.EINVAL
    # the Particles-level sort keeps original order at the API
    P.sort(shape)
    assert np.array_equal(P["z"].cpu().numpy(), p.astype(np.float64))  # gathered by the kernel
    assert np.array_equal(P["extra"].cpu().numpy(), p.astype(np.float32))  # gathered by torch
    assert np.array_equal(P.order.cpu().numpy(), p)
    for name, v in (("zidx", z), ("yidx", y), ("xidx", x), ("status", st)):
        assert same_bits(P.original(name).cpu().numpy(), v), name


@pytest.mark.parametrize("sort_interval", [0, 1, 7])
@pytest.mark.parametrize("mode", ["step", "run"])
def test_results_do_not_depend_on_sorting(sort_interval, mode):
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    final, rec, _ = run_b200(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"],
                             steps=c["steps"], z=z, y=y, x=x, mode=mode, record_every=c["record_every"],
                             record_idx=gold["record_idx"], sort_interval=sort_interval)
    assert same_bits(rec, gold["record"]), mismatch_report(rec, gold["record"])
    for name in gold:
        if name in final:
            assert same_bits(final[name], gold[name]), f"{name}: {mismatch_report(final[name], gold[name])}"


def _particles_with_keys(n, shape, seed):
    """Particles spread over the grid, a third of them packed into a few cells (long runs of equal keys), some
    outside it, some inactive; their Morton keys computed on the host."""
    import torch

    from offline_particles_b200.particles import Particles

    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z = rng.uniform(-1, nz + 1, n)
    y = rng.uniform(-2, ny + 2, n)
    x = rng.uniform(-2, nx + 2, n)
    packed = rng.random(n) < 1 / 3
    z[packed], y[packed], x[packed] = 2.5, rng.integers(3, 5, packed.sum()) + 0.5, 7.5
    st = np.zeros(n, np.uint8)
    st[rng.random(n) < 0.05] = 0x82
    P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64)
    for name, v in (("zidx", z), ("yidx", y), ("xidx", x), ("status", st)):
        P[name].copy_(torch.from_numpy(v))
    return P, host_keys(st, z, y, x, shape)


@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 4095, 4096, 4097, 100_003, 4_194_304 + 17])
def test_sort_permutation_is_the_stable_key_order(n):
    """The radix sort's permutation is exactly the stable order of the keys (numpy's stable argsort of the
    host keys), for counts below, at and across the 2048-key tiles of its passes, and with more tiles than
    one chunk of its per-digit scan (1024 tiles)."""
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.kernels import _abi

    shape = (50, 768, 1024)
    P, keys = _particles_with_keys(n, shape, seed=n)
    lib = _lib.load()
    ws = torch.empty(lib.opb_sort_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    _lib.call("opb_sort_particles", ctypes.byref(_abi.particles_struct(P)), ctypes.byref((ctypes.c_int64 * 3)(*shape)),
              perm.data_ptr(), ws.data_ptr(), ws.numel(), None)
    assert np.array_equal(perm.cpu().numpy(), np.argsort(keys, kind="stable"))


def test_ranged_sort_permutation_is_the_stable_key_order():
    """Within id ranges: the stable order of (range index, cell key), the range index in the key's top bits."""
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.kernels import _abi

    n, shape = 250_001, (40, 512, 512)
    P, keys = _particles_with_keys(n, shape, seed=11)
    ids = np.random.default_rng(12).permutation(n).astype(np.int64)
    bounds = (0, 60_000, 61_000, n)
    rng_of = np.searchsorted(np.array(bounds[1:-1]), ids, side="right").astype(np.uint64)
    expect = np.argsort((rng_of << np.uint64(30)) | (keys & np.uint64(0x3FFFFFFF)), kind="stable")
    lib = _lib.load()
    ws = torch.empty(lib.opb_sort_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    dev_ids = torch.from_numpy(ids).cuda()
    _lib.call("opb_sort_particles_ranges", ctypes.byref(_abi.particles_struct(P)),
              ctypes.byref((ctypes.c_int64 * 3)(*shape)), dev_ids.data_ptr(), (ctypes.c_int64 * 4)(*bounds), 3,
              perm.data_ptr(), ws.data_ptr(), ws.numel(), None)
    assert np.array_equal(perm.cpu().numpy(), expect)


def test_segment_sort_is_the_stable_key_order_in_each_segment():
    """The segment sort (64-bit keys: segment above the cell key, five digit passes) leaves in each segment
    exactly the stable key order of its particles."""
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.batching import ARENA_FIELDS
    from offline_particles_b200.kernels import _abi
    from offline_particles_b200.particles import Particles

    n, shape = 400_000, (12, 80, 96)
    Q, keys = _particles_with_keys(n, shape, seed=21)
    P = Particles(n, **ARENA_FIELDS)
    for k in ("status", "zidx", "yidx", "xidx"):
        P[k].copy_(Q[k])
    ids = torch.arange(n, dtype=torch.int64, device="cuda")
    starts, counts = [0, 5000, 5001, 70_000, 399_000], [4000, 1, 60_000, 300_000, 1000]
    lib = _lib.load()
    ws = torch.empty(int(lib.opb_sort_segments_workspace_bytes(sum(counts), len(starts))), dtype=torch.uint8,
                     device="cuda")
    _lib.call("opb_sort_segments", ctypes.byref(_abi.particles_struct(P)), ctypes.byref((ctypes.c_int64 * 3)(*shape)),
              (ctypes.c_int64 * 5)(*starts), (ctypes.c_int64 * 5)(*counts), 5, ids.data_ptr(), 0, None,
              ws.data_ptr(), ws.numel(), None)
    got = ids.cpu().numpy()
    expect = np.arange(n)
    for s, c in zip(starts, counts):
        expect[s:s + c] = s + np.argsort(keys[s:s + c], kind="stable")
    assert np.array_equal(got, expect)
