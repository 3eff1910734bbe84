"""Results read back range by range: ``Simulation(result_ranges=R)`` and ``run(..., results=...)``.

Particle storage is kept in R ranges of original ids (``opb_sort_particles_ranges``), the last fused
launch of a run is issued range by range, and each range's fields are copied to host memory in original
order while the next range computes.  Particles are independent, so every result must equal the
reference's golden fixture bit for bit, whatever the split.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from b200_runner import build_sim
from helpers import CASES, load, mismatch_report, same_bits
from offline_particles_b200.synth import SyntheticROMS
from test_gpu_sort import host_keys

pytestmark = pytest.mark.gpu

NAMES = ("zidx", "yidx", "xidx", "status", "z")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")


def _host_buffers(sim, names=NAMES, pinned=True):
    import torch

    P = sim.device_particles
    return {k: torch.empty(len(P), dtype=P[k].dtype, pin_memory=pinned) for k in names}


def _launch_counter():
    from offline_particles_b200 import timesteppers
    from offline_particles_b200.kernels import _abi

    calls = []
    orig = _abi.particles_struct_range

    def counted(particles, lo, hi):
        calls.append((lo, hi))
        return orig(particles, lo, hi)

    return calls, orig, counted, timesteppers


@pytest.mark.parametrize("case,ranges", [("ab3_f32", 4), ("config1_rk2", 3), ("ab3_f32", 2)])
def test_results_stream_range_by_range(case, ranges):
    """The golden run's final fields, read back through run(results=...) with the last launch split."""
    from offline_particles_b200.kernels import _abi

    c = CASES[case]
    gold = load(f"{case}.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    sim = build_sim(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme=c["scheme"], dt=c["dt"], z=z, y=y,
                    x=x, result_ranges=ranges, sort_interval=16)
    out = _host_buffers(sim)
    calls, orig, counted, _ = _launch_counter()
    _abi.particles_struct_range = counted
    try:
        sim.run(c["steps"], results=out)
    finally:
        _abi.particles_struct_range = orig
    sim.synchronize()
    from offline_particles_b200.simulation import result_bounds

    b = result_bounds(c["n"], ranges)
    assert calls == list(zip(b[:-1], b[1:])), "the last launch must run range by range"
    P = sim.device_particles
    assert P.sort_bounds == b
    order = P.order.cpu().numpy()
    for lo, hi in zip(b[:-1], b[1:]):
        assert np.array_equal(np.sort(order[lo:hi]), np.arange(lo, hi)), "a sort moved a particle out of its range"
    for name in NAMES:
        got = out[name].numpy()
        assert same_bits(got, gold[name]), f"{case} R={ranges} {name}: {mismatch_report(got, gold[name])}"
        assert same_bits(got, np.asarray(sim.particles[name])), name


def test_results_without_ranges_and_unpinned():
    """result_ranges=1 (global sort): the results are read after the run, unpinned buffers too."""
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    sim = build_sim(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"], z=z, y=y, x=x)
    out = _host_buffers(sim, pinned=False)
    sim.run(c["steps"], results=out)
    sim.synchronize()
    for name in NAMES:
        assert same_bits(out[name].numpy(), gold[name]), name


def test_results_stage_path_and_repeated_runs():
    """A stepper that runs stage by stage (no fused launch to split) and runs in pieces, each read back."""
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    fields = grid.oracle_fields()
    for unfused in (False, True):
        sim = build_sim(fields, hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"], z=z, y=y, x=x,
                        unfused=unfused, result_ranges=4)
        out = _host_buffers(sim)
        for part in (40, 40, 69):
            sim.run(part, results=out)
        sim.synchronize()
        for name in NAMES:
            assert same_bits(out[name].numpy(), gold[name]), f"unfused={unfused} {name}"


def test_results_after_an_event_at_the_last_step(tmp_path):
    """An output event fires at the run's last step: the results are the state after it."""
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200.output import NpyOutputBuilder, linearly_interpolate_fields

    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    fields = grid.oracle_fields()
    fs = b200_fieldset(fields, grid.hc, grid.spec.nz)
    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    sb = opb.SimulationBuilder(opb.roms.ab3_w_advection_timestepper(t_arr, np.float64(c["dt"])), fs)
    ob = NpyOutputBuilder("npy", tmp_path / "out")
    ob.add_output(*linearly_interpolate_fields(fs, "h"))
    sb.add_output_writer(ob, dt=np.float64(1800.0))  # every 15 steps: fires after step 135, 150, ...
    sim = sb.build_simulation(c["n"], result_ranges=4)
    sim.set_indices(*grid.release(c["n"]))
    sim.set_particle_field("status", 10)
    out = _host_buffers(sim)
    sim.run(135, results=out)
    sim.synchronize()
    for name in NAMES:
        assert same_bits(out[name].numpy(), np.asarray(sim.particles[name])), f"after the event: {name}"
    sim.run(c["steps"] - 135, results=out)
    sim.synchronize()
    sim.close_outputs()
    for name in NAMES:
        assert same_bits(out[name].numpy(), gold[name]), name


def test_results_argument_errors():
    import torch

    c = CASES["ab3_f32"]
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(256)
    sim = build_sim(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"], z=z, y=y, x=x,
                    result_ranges=4)
    with pytest.raises(KeyError):
        sim.run(1, results={"nope": torch.empty(256, dtype=torch.float64)})
    with pytest.raises(ValueError):
        sim.run(1, results={"zidx": torch.empty(255, dtype=torch.float64)})
    with pytest.raises(ValueError):
        sim.run(1, results={"zidx": torch.empty(256, dtype=torch.float32)})
    with pytest.raises(TypeError):
        sim.run(1, results={"zidx": torch.empty(256, dtype=torch.float64, device="cuda")})
    with pytest.raises(ValueError, match="result_ranges"):
        build_sim(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"], z=z, y=y, x=x,
                  result_ranges=5)


def test_sort_in_id_ranges_is_the_global_order_within_each_range():
    """opb_sort_particles_ranges: range r holds ids [b[r], b[r + 1]), in the global sort's order."""
    import torch

    from offline_particles_b200 import _lib
    from offline_particles_b200.kernels import _abi
    from offline_particles_b200.particles import Particles

    rng = np.random.default_rng(9)
    n, shape = 100_003, (50, 768, 1024)
    z = rng.uniform(-1, 50, n)
    y = rng.uniform(-3, 770, n)
    x = rng.uniform(-3, 1030, n)
    z[:3] = [np.nan, np.inf, -1e300]
    st = np.zeros(n, np.uint8)
    st[rng.integers(0, n, 3000)] = 0x82

    def fresh():
        P = Particles(n, status=np.uint8, zidx=np.float64, yidx=np.float64, xidx=np.float64, z=np.float64)
        for name, v in (("zidx", z), ("yidx", y), ("xidx", x), ("status", st)):
            P[name].copy_(torch.from_numpy(v))
        P["z"].copy_(torch.arange(n, dtype=torch.float64))
        return P

    b = (0, 17, 50_000, 99_000, n)  # uneven ranges, one of 17 particles
    P = fresh()
    P.sort(shape, id_bounds=b)
    order = P.order.cpu().numpy()
    G = fresh()
    G.sort(shape)
    gorder = G.order.cpu().numpy()
    for lo, hi in zip(b[:-1], b[1:]):
        want = gorder[(gorder >= lo) & (gorder < hi)]
        assert np.array_equal(order[lo:hi], want), f"range [{lo}, {hi})"
    assert np.array_equal(P["z"].cpu().numpy(), order.astype(np.float64)), "fields must move with their ids"
    keys = host_keys(st, z, y, x, shape)
    for lo, hi in zip(b[:-1], b[1:]):
        assert np.all(np.diff(keys[order[lo:hi]].astype(np.int64)) >= 0)
    # a second sort with the same bounds keeps every particle in its range (ids from the order array)
    P["zidx"].copy_(torch.from_numpy(rng.uniform(0, 50, n)))
    P.sort(shape, id_bounds=b)
    order2 = P.order.cpu().numpy()
    for lo, hi in zip(b[:-1], b[1:]):
        assert np.array_equal(np.sort(order2[lo:hi]), np.arange(lo, hi))
    # other bounds, five ranges, bounds that do not rise from 0 to n, or ranges after a global sort: errors
    for bad in ((0, 18, 50_000, 99_000, n), (0, 1, 2, 3, 4, n), (0, 5, 5, n), (1, 5, n), (0, 5, n - 1)):
        with pytest.raises(ValueError):
            (P if bad[1] == 18 else fresh()).sort(shape, id_bounds=bad)
    with pytest.raises(ValueError):
        G.sort(shape, id_bounds=b)
    lib = _lib.load()
    ws = torch.empty(lib.opb_sort_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    dims = (ctypes.c_int64 * 3)(*shape)
    Q = fresh()
    for bad in ((0, 5, 5, n), (0, n - 1), (0, 1, 2, 3, 4, n), (1, n)):
        arr = (ctypes.c_int64 * len(bad))(*bad)
        rc = lib.opb_sort_particles_ranges(ctypes.byref(_abi.particles_struct(Q)), ctypes.byref(dims), None, arr,
                                           len(bad) - 1, perm.data_ptr(), ws.data_ptr(), ws.numel(), None)
        assert rc == _lib.EINVAL, bad
    rc = lib.opb_sort_particles_ranges(ctypes.byref(_abi.particles_struct(Q)), ctypes.byref(dims), None, None, 2,
                                       perm.data_ptr(), ws.data_ptr(), ws.numel(), None)
    assert rc == _lib.EINVAL


@pytest.mark.parametrize("n", [1, 3, 5])
def test_results_with_fewer_particles_than_ranges(n):
    """result_ranges=4 with fewer particles than ranges: as many ranges as particles, one launch each."""
    c = CASES["ab3_f32"]
    gold = load("ab3_f32.npz")
    grid = SyntheticROMS(c["grid"])
    z, y, x = grid.release(c["n"])
    sim = build_sim(grid.oracle_fields(), hc=grid.hc, nz=grid.spec.nz, scheme="ab3", dt=c["dt"], z=z[:n], y=y[:n],
                    x=x[:n], result_ranges=4)
    out = _host_buffers(sim)
    sim.run(c["steps"], results=out)
    sim.synchronize()
    for name in NAMES:
        assert same_bits(out[name].numpy(), gold[name][:n]), name


def test_record_budget_shortens_launches_not_results(tmp_path, monkeypatch):
    """Events at every step with a record budget of two states per launch: the launches stop at the budget,
    the rows equal step mode's."""
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200 import simulation as simmod
    from offline_particles_b200.output import NpyOutputBuilder, linearly_interpolate_fields

    c = CASES["ab3_f32"]
    grid = SyntheticROMS(c["grid"])
    fields = grid.oracle_fields()
    z, y, x = grid.release(c["n"])
    rows = {}
    for mode in ("step", "run"):
        if mode == "run":
            monkeypatch.setattr(simmod, "RECORD_BUDGET_BYTES", 33 * c["n"] * 2)
        fs = b200_fieldset(fields, grid.hc, grid.spec.nz)
        t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
        sb = opb.SimulationBuilder(opb.roms.ab3_w_advection_timestepper(t_arr, np.float64(c["dt"])), fs)
        ob = NpyOutputBuilder("o", tmp_path / mode)
        ob.add_output(*linearly_interpolate_fields(fs, "h", "u"))
        sb.add_output_writer(ob, n=1)
        sim = sb.build_simulation(c["n"])
        sim.set_indices(z, y, x)
        sim.set_particle_field("status", 10)
        if mode == "step":
            for _ in range(40):
                sim.step()
        else:
            sim.run(40)
        sim.synchronize()
        sim.close_outputs()
        rows[mode] = {k: np.load(tmp_path / mode / f"{k}.npy") for k in ("time", "h", "u")}
    for k, v in rows["step"].items():
        assert v.shape[0] == 41 and same_bits(rows["run"][k], v), k


def test_results_of_a_run_that_raises():
    """A run that steps onto the last snapshot time raises as the reference does; the copies already queued
    are joined, and the simulation stays usable."""
    from offline_particles_b200.synth import GridSpec

    g = SyntheticROMS(GridSpec(nx=16, ny=12, nz=4, nt=2, seed=3, dtype="float32"))
    z, y, x = g.release(8)
    sim = build_sim(g.oracle_fields(), hc=g.hc, nz=g.spec.nz, scheme="ab3", dt=1800.0, z=z, y=y, x=x,
                    result_ranges=2)
    out = _host_buffers(sim)
    with pytest.raises((IndexError, ValueError)):
        sim.run(3, results=out)
    sim.synchronize()
    assert np.asarray(sim.particles["zidx"]).shape == (8,)
