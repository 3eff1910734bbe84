"""The reduced-precision steppers (float32 arithmetic; float32 / bfloat16 / float16 storage).

They are not bit-identical to the reference; these tests bound their error
against the float64 path (itself bit-identical to the reference), in index
units of the grid (1 unit = 2 km horizontally on these grids):
  float32 storage : max |d index| <= 2e-4 after 149 AB3 steps (0.4 m), statuses identical
  float16 storage : max |d index| <= 0.02 (40 m),  >= 99.5 % of statuses identical
  bfloat16 storage: max |d index| <= 0.2 (400 m),  >= 99 % of statuses identical
"""

from __future__ import annotations

import numpy as np
import pytest

from b200_runner import build_sim, run_b200
from helpers import CASES, load
from offline_particles_b200.synth import GridSpec, SyntheticROMS

pytestmark = pytest.mark.gpu

TOL = {None: (2e-4, 1.0), "float16": (0.02, 0.995), "bfloat16": (0.2, 0.99)}


def _compare(final, gold, storage):
    tol, agree = TOL[storage]
    st, gst = final["status"], gold["status"]
    assert np.mean(st == gst) >= agree, f"{storage}: status agreement {np.mean(st == gst)}"
    both = (st & 0x80) == 0
    both &= (gst & 0x80) == 0
    for name in ("zidx", "yidx", "xidx"):
        d = np.abs(final[name][both] - gold[name][both])
        assert np.all(np.isfinite(d)) and d.max() <= tol, f"{storage} {name}: max |d| = {d.max()}"


@pytest.mark.parametrize("storage", [None, "float16", "bfloat16"])
@pytest.mark.parametrize("mode", ["step", "run"])
def test_ab3_float32_tracks_float64(storage, mode):
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    final, _, _ = run_b200(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"],
                           steps=c["steps"], z=z, y=y, x=x, mode=mode, arithmetic="float32", storage=storage)
    _compare(final, gold, storage)


@pytest.mark.parametrize("storage", [None, "float16"])
def test_rk2_float32_tracks_float64(storage):
    grid = SyntheticROMS(GridSpec(nx=96, ny=80, nz=16, nt=6, seed=13, dtype="float32"))
    fields = grid.oracle_fields()
    z, y, x = grid.release(4096)
    ref, _, _ = run_b200(fields, hc=grid.hc, nz=grid.spec.nz, scheme="rk2", dt=240.0, steps=60, z=z, y=y, x=x,
                         mode="run")
    got, _, _ = run_b200(fields, hc=grid.hc, nz=grid.spec.nz, scheme="rk2", dt=240.0, steps=60, z=z, y=y, x=x,
                         mode="run", arithmetic="float32", storage=storage)
    _compare(got, ref, storage)


def test_quantize_levels_matches_torch():
    import torch

    from offline_particles_b200.fields import quantize_levels

    rng = np.random.default_rng(0)
    src = torch.from_numpy((rng.standard_normal((7, 33, 41)) * np.logspace(-6, 1, 7)[:, None, None]).astype(
        np.float32)).cuda()
    src[3].zero_()
    for dt in (torch.bfloat16, torch.float16):
        q = torch.empty(src.shape, dtype=dt, device="cuda")
        scales = torch.empty(7, dtype=torch.float32, device="cuda")
        quantize_levels(src, q, scales, 7)
        absmax = src.abs().amax(dim=(1, 2))
        ref_scales = torch.where(absmax > 0, absmax / 32768.0, torch.ones_like(absmax))
        assert torch.equal(scales, ref_scales)
        ref_q = (src / ref_scales[:, None, None]).to(dt)
        assert torch.equal(q.view(torch.int16), ref_q.view(torch.int16))


def test_reduced_storage_needs_float32_arithmetic():
    grid = SyntheticROMS(GridSpec(nx=24, ny=20, nz=6, nt=3, seed=31, dtype="float32"))
    z, y, x = grid.release(64)
    sim = build_sim(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=300.0, z=z, y=y, x=x,
                    storage="bfloat16")
    with pytest.raises(ValueError, match="float32"):
        sim.step()
