"""Output writers on the GPU against the reference's own output rows (tests/golden/outputs.npz).

linearly_interpolate_fields (h, u, zeta, w) written every 1800 s of an RK2 run
(output/_linear_interpolation.py, output/_output.py, simulation.py:320-369 of
the reference): the same events, kernels and row format, through
NpyOutputBuilder; rows bit for bit, stepping one step at a time and with
fused multi-step runs, inside which the output events replay on the particle
states the launches recorded at their steps.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import fingerprint, load, mismatch_report, same_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["step", "run"])
def test_output_rows_match_reference(tmp_path, mode):
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200.output import NpyOutputBuilder, linearly_interpolate_fields
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    gold = load("outputs.npz")
    g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=4, seed=41, dtype="float32"))
    fields = g.oracle_fields()
    fs = b200_fieldset(fields, g.hc, g.spec.nz)
    t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
    sb = opb.SimulationBuilder(opb.roms.rk2_w_advection_timestepper(t_arr, np.float64(300.0)), fs)
    ob = NpyOutputBuilder("npy", tmp_path / "out")
    ob.add_output(*linearly_interpolate_fields(fs, "h", "u", "zeta", "w"))
    sb.add_output_writer(ob, dt=np.float64(1800.0))
    sim = sb.build_simulation(512)
    sim.set_indices(gold["z0"], gold["y0"], gold["x0"])
    if mode == "step":
        for _ in range(24):
            sim.step()
    else:
        sim.run(24)
    sim.synchronize()
    sim.close_outputs()
    out = tmp_path / "out"
    assert same_bits(np.load(out / "time.npy"), gold["time"])
    for name in ("h", "u", "zeta", "w"):
        got = np.load(out / f"{name}.npy")
        assert got.shape == gold[f"out_{name}"].shape
        assert same_bits(got, gold[f"out_{name}"]), f"{name}: {mismatch_report(got, gold[f'out_{name}'])}"


def test_output_writer_errors(tmp_path):
    from offline_particles_b200.kernels.validation import validation_kernel
    from offline_particles_b200.output import NpyOutputBuilder, Output

    with pytest.raises(ValueError, match="not found"):
        Output("nope", validation_kernel)
    ob = NpyOutputBuilder("npy", tmp_path)
    o = Output("zidx", validation_kernel)
    ob.add_output(o)
    with pytest.raises(KeyError):
        ob.add_output(o)
    ob.remove_output("zidx")
    with pytest.raises(KeyError):
        ob.remove_output("zidx")


def test_simulation_from_roms_history_files(tmp_path):
    """Fields streamed from NetCDF history files give the same particles as the same fields in memory."""
    from b200_runner import STAGGERS

    import offline_particles_b200 as opb
    from offline_particles_b200.roms_history import RomsHistory, write_history
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=64, ny=48, nz=10, nt=6, seed=61, dtype="float32"))
    f = g.oracle_fields()
    write_history(tmp_path / "a.nc", {**f, **{n: f[n][:4] for n in ("u", "v", "w", "zeta")}}, g.time_array[:4],
                  hc=g.hc, mask_rho=g.mask_rho, fill_land=1e37)
    write_history(tmp_path / "b.nc", {**f, **{n: f[n][4:] for n in ("u", "v", "w", "zeta")}}, g.time_array[4:],
                  hc=g.hc, mask_rho=g.mask_rho, fill_land=1e37)
    h = RomsHistory([tmp_path / "a.nc", tmp_path / "b.nc"])
    z, y, x = g.release(2000, seed=8)
    outs = []
    for source in ("files", "memory"):
        if source == "files":
            fs = h.fieldset()
        else:
            kw = {n: opb.TimeDependentField.from_numpy(np.asarray(h.variable(n)), *STAGGERS[n])
                  for n in ("u", "v", "w", "zeta")}
            for n, arr in h.statics().items():
                kw[n] = opb.StaticField.from_numpy(arr, *STAGGERS[n])
            fs = opb.Fieldset(6, 10, 48, 64, constants={"hc": h.hc, "NZ": 10}, **kw)
        ts = opb.roms.ab3_w_advection_timestepper(h.time_array, np.float64(120.0))
        sim = opb.SimulationBuilder(ts, fs).build_simulation(len(z))
        sim.set_indices(z, y, x)
        sim.set_particle_field("status", 10)
        sim.run(140)
        P = sim.particles
        outs.append({k: P[k] for k in ("status", "zidx", "yidx", "xidx", "z")})
    h.close()
    for k in outs[0]:
        assert same_bits(outs[0][k], outs[1][k]), k


def test_mixed_schedules_run_equals_step_and_reference(tmp_path):
    """An output writer every 1800 s and one every 7 iterations from iteration 3 in one simulation: run()
    records the particle state at both schedules' events inside its fused launches and fires the events
    on those states after each launch (also with the last launch split over two result ranges), and every
    row of both writers equals the
    step-by-step run and the reference's rows (outputs_mixed.npz).  Inactive particles keep what the
    previous output kernel left in the shared particle field, so the second writer changes some of the
    first writer's rows exactly as it does in the reference."""
    import torch
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200 import timesteppers
    from offline_particles_b200.output import NpyOutputBuilder, linearly_interpolate_fields
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    gold = load("outputs_mixed.npz")
    g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=4, seed=41, dtype="float32"))
    fields = g.oracle_fields()
    assert fingerprint(fields) == str(gold["fingerprint"])
    rows = {}
    launches = {}
    for mode in ("step", "run", "run_ranges"):
        fs = b200_fieldset(fields, g.hc, g.spec.nz)
        t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
        sb = opb.SimulationBuilder(opb.roms.rk2_w_advection_timestepper(t_arr, np.float64(300.0)), fs)
        by_time = NpyOutputBuilder("by_time", tmp_path / mode / "t")
        by_time.add_output(*linearly_interpolate_fields(fs, "h", "u", "zeta", "w"))
        sb.add_output_writer(by_time, dt=np.float64(1800.0))
        by_iter = NpyOutputBuilder("by_iter", tmp_path / mode / "i")
        by_iter.add_output(*linearly_interpolate_fields(fs, "v", "zeta"))
        sb.add_output_writer(by_iter, n=7, first=3)
        sim = sb.build_simulation(512, result_ranges=2 if mode == "run_ranges" else 1)
        sim.set_indices(gold["z0"], gold["y0"], gold["x0"])
        counter = _LaunchCounter()
        timesteppers.launch_observers.append(counter)
        try:
            if mode == "step":
                for _ in range(24):
                    sim.step()
            elif mode == "run":
                sim.run(24)
            else:
                res = {k: torch.empty(512, dtype=sim.device_particles[k].dtype) for k in ("zidx", "status")}
                sim.run(24, results=res)
        finally:
            timesteppers.launch_observers.remove(counter)
        launches[mode] = counter.launches
        sim.synchronize()
        if mode == "run_ranges":
            for k, v in res.items():
                assert same_bits(v.numpy(), np.asarray(sim.particles[k])), k
        sim.close_outputs()
        rows[mode] = {f"{d}_{n}": np.load(tmp_path / mode / d / f"{n}.npy")
                      for d, names in (("t", ("time", "h", "u", "zeta", "w")), ("i", ("time", "v", "zeta")))
                      for n in names}
    for key, val in rows["step"].items():
        for mode in ("run", "run_ranges"):
            assert same_bits(rows[mode][key], val), f"{mode} {key}: {mismatch_report(rows[mode][key], val)}"
        assert same_bits(val, gold[key]), f"{key}: {mismatch_report(val, gold[key])}"
    # the output events (iterations 3, 6, 10, 12, 17, 18 inside the run) no longer end fused launches:
    # they replay on the states the launches recorded
    assert launches["step"] == 24
    assert launches["run"] <= 3 and launches["run_ranges"] <= 3, launches


class _LaunchCounter:
    """A launch observer: counts fused launches."""

    def __init__(self) -> None:
        self.launches = 0

    def before(self, nsteps: int) -> None:
        self.launches += 1

    def after(self, nsteps: int) -> None:
        pass


def test_events_that_are_not_deferrable_still_end_launches():
    """A user event (not declared deferrable) sees the live state at its own iteration, so a fused launch
    ends there; a deferrable one reads the state recorded at its step: both see the step-by-step state."""
    from b200_runner import b200_fieldset

    import offline_particles_b200 as opb
    from offline_particles_b200 import timesteppers
    from offline_particles_b200.events import Event
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    g = SyntheticROMS(GridSpec(nx=48, ny=40, nz=8, nt=4, seed=41, dtype="float32"))
    fields = g.oracle_fields()
    z, y, x = g.release(700, seed=3)
    seen = {}
    launches = {}
    for mode in ("step", "run"):
        fs = b200_fieldset(fields, g.hc, g.spec.nz)
        t_arr = np.arange(fields["u"].shape[0], dtype=np.float64) * 3600.0
        sb = opb.SimulationBuilder(opb.roms.ab3_w_advection_timestepper(t_arr, np.float64(300.0)), fs)
        log = seen.setdefault(mode, {"live": [], "deferred": []})

        def live(state, log=log):
            log["live"].append((state.iteration, np.asarray(state.particles["xidx"]).copy()))

        def deferred(state, log=log):
            log["deferred"].append((state.iteration, state.time, np.asarray(state.particles["zidx"]).copy(),
                                    np.asarray(state.particles["status"]).copy()))

        sb.add_event(Event("live", live), n=9, first=5)
        sb.add_event(Event("deferred", deferred, deferrable=True), n=4, first=2)
        sim = sb.build_simulation(len(z))
        sim.set_indices(z, y, x)
        sim.set_particle_field("status", 10)
        counter = _LaunchCounter()
        timesteppers.launch_observers.append(counter)
        try:
            if mode == "step":
                for _ in range(23):
                    sim.step()
            else:
                sim.run(23)
        finally:
            timesteppers.launch_observers.remove(counter)
        sim.synchronize()
        launches[mode] = counter.launches
    for kind in ("live", "deferred"):
        a, b = seen["step"][kind], seen["run"][kind]
        assert [r[0] for r in a] == [r[0] for r in b] and len(a) > 2, kind
        for ra, rb in zip(a, b):
            for va, vb in zip(ra[1:], rb[1:]):
                assert same_bits(np.asarray(va), np.asarray(vb)), (kind, ra[0])
    # launches end at the live event (iterations 5, 14) and at the interval boundary (12), not at the
    # deferrable ones (2, 6, 10, 14, 18, 22)
    assert launches["run"] <= 5, launches
