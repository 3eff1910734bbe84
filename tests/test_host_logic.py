"""Host-side logic of result ranges and event planning (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from offline_particles_b200.events import Event, IterationScheduler, TimeScheduler
from offline_particles_b200.simulation import result_bounds


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 100, 4096, 4_194_304, 10_000_019])
@pytest.mark.parametrize("ranges", [1, 2, 3, 4])
def test_result_bounds_cover_the_particles_in_rising_ranges(n, ranges):
    b = result_bounds(n, ranges)
    if ranges == 1 or n == 1:
        assert b is None
        return
    assert b[0] == 0 and b[-1] == n
    assert len(b) - 1 == min(ranges, n)
    assert all(lo < hi for lo, hi in zip(b, b[1:]))
    # the last range holds a quarter of the particles (its copy is the one left after the last launch)
    assert b[-1] - b[-2] == -(-n // 4) or n < 4 * ranges


def _fire_sequence(sched, points):
    return [[e.name for e in sched(p)] for p in points]


def test_scheduler_copies_fire_like_the_originals_and_leave_them_alone():
    a, b = Event("a", lambda s: None), Event("b", lambda s: None, deferrable=True)
    its = IterationScheduler()
    its.register_event(3, 7, a)
    its.register_event(0, 4, b)
    c = its.copy()
    seq = _fire_sequence(c, range(0, 40))
    assert its.next == 0  # the original did not move
    assert seq == _fire_sequence(its, range(0, 40))
    tms = TimeScheduler()
    tms.register_event(np.float64(0.0), np.float64(1800.0), a)
    tms.register_event(np.float64(600.0), np.float64(900.0), b)
    times = [np.float64(0.0)]
    for _ in range(60):
        times.append(times[-1] + np.float64(120.0))
    c = tms.copy()
    seq = _fire_sequence(c, times)
    assert tms.next_time == 0.0
    assert seq == _fire_sequence(tms, times)
    assert b.deferrable and not a.deferrable


def test_writer_events_are_deferrable_only_with_sampling_kernels(tmp_path):
    from offline_particles_b200.kernels import ParticleKernel
    from offline_particles_b200.kernels.output.linear_interpolation import trilinear_interpolation_kernel
    from offline_particles_b200.output import NpyOutputBuilder, Output

    ob = NpyOutputBuilder("w", tmp_path)
    ob.add_output(Output("u", trilinear_interpolation_kernel("u", "_out"), particle_field="_out"))
    w = ob.build(8)
    assert all(e.deferrable for e in w.create_events())
    # a sampling kernel that writes a field the stepping kernels own is not deferrable
    ob2 = NpyOutputBuilder("w2", tmp_path / "b")
    ob2.add_output(Output("u", trilinear_interpolation_kernel("u", "zidx"), particle_field="zidx"))
    assert not any(e.deferrable for e in ob2.build(8).create_events())
    # nor is any other kernel
    odd = ParticleKernel(lambda p, s, f: None, {"_odd": np.float64}, {}, [])
    ob3 = NpyOutputBuilder("w3", tmp_path / "c")
    ob3.add_output(Output("odd", odd, particle_field="_odd"))
    assert not any(e.deferrable for e in ob3.build(8).create_events())
