"""The batch's interval planner against the stepper's own time arithmetic (CPU only).

Each release in a batch must see exactly the stage time indices its own
Simulation would: Timestepper._stage_times + advance_time
(timesteppers.py:64-85,157-161,241-257,296-305), split into snapshot
intervals.  These tests replay both and compare the floats bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from offline_particles_b200.batching import IntervalPlanner, Release, TimeIndex
from offline_particles_b200.models.roms import ab3_w_advection_timestepper, rk2_w_advection_timestepper


def _release(scheme, t_arr, dt, t0, nsteps, alpha=2 / 3):
    if scheme == "rk2":
        ts = rk2_w_advection_timestepper(t_arr, np.float64(dt), time=np.float64(t0), alpha=alpha)
    else:
        ts = ab3_w_advection_timestepper(t_arr, np.float64(dt), time=np.float64(t0))
    z = np.zeros(3)
    return Release(ts, nsteps, z, z, z), ts


def _reference_sequence(ts, nsteps):
    """Stage time indices of up to nsteps steps as the fused stepper plans them; stops where it raises."""
    out = []
    time = ts.time
    for _ in range(nsteps):
        try:
            tidxs, nxt = ts._stage_times(time)
        except (ValueError, IndexError):
            break
        out.append([float(x) for x in tidxs])
        time = nxt
    return out


def test_time_index_matches_timestepper_bitwise():
    rng = np.random.default_rng(0)
    t_arr = np.cumsum(rng.uniform(1800, 5400, 40)).astype(np.float64)
    ts = ab3_w_advection_timestepper(t_arr, np.float64(60.0), time=t_arr[0])
    ti = TimeIndex(t_arr)
    times = np.concatenate([rng.uniform(t_arr[0], t_arr[-1], 2000), t_arr[:-1], np.nextafter(t_arr[1:], 0)])
    for t in times:
        a = ts.get_time_index(np.float64(t))
        b = ti(float(t))
        assert np.float64(a).tobytes() == np.float64(b).tobytes(), t
    with pytest.raises(ValueError):
        ti(float(t_arr[-1]) + 1.0)
    with pytest.raises(ValueError):
        ti(float(t_arr[0]) - 1.0)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_planner_reproduces_each_release_alone(seed):
    rng = np.random.default_rng(seed)
    nt = 30
    t_arr = np.arange(nt, dtype=np.float64) * 3600.0
    specs = []
    for _ in range(24):
        scheme = ["rk2", "ab3"][int(rng.integers(2))]
        dt = float(rng.choice([60.0, 120.0, 180.0, 300.0, 7.3, 3599.0]))
        t0 = float(rng.uniform(0, 20 * 3600.0)) if rng.random() < 0.7 else float(3600.0 * rng.integers(0, 20))
        nsteps = int(rng.integers(0, 2500))  # some run past the last snapshot
        specs.append((scheme, dt, t0, nsteps))
    rels = []
    refs = []
    for scheme, dt, t0, nsteps in specs:
        r, ts = _release(scheme, t_arr, dt, t0, nsteps)
        rels.append(r)
        refs.append(_reference_sequence(ts, nsteps))
    planner = IntervalPlanner(t_arr, nt)
    got = [[] for _ in rels]
    for j in range(nt - 1):
        exps, tidx = planner.plan(rels, j)
        for e, r, k, first in exps:
            per = 3 if r.scheme == 1 else 2
            seg = tidx[first:first + per * k]
            for s in range(k):
                step = seg[per * s:per * (s + 1)]
                # every stage reads snapshots j .. j + 2
                assert all(j <= int(x) and int(x) + 1 <= j + 2 for x in step)
                got[e].append(step)
    for e, (r, ref) in enumerate(zip(rels, refs)):
        assert r.done == len(got[e])
        n_ok = len(ref)
        if r.error is None:
            assert r.done == r.nsteps == n_ok, e
        else:
            # a step is not planned when the stepper raises for it (or it would need a fourth snapshot)
            assert r.done <= n_ok, e
        for a, b in zip(got[e], ref[:r.done]):
            assert np.array(a).tobytes() == np.array(b).tobytes(), e


def test_dt_longer_than_the_snapshot_spacing_stops_the_release():
    t_arr = np.arange(10, dtype=np.float64) * 3600.0
    r, _ = _release("rk2", t_arr, 3 * 3600.0, 0.0, 2)
    planner = IntervalPlanner(t_arr, 10)
    exps, _ = planner.plan([r], 0)
    assert not exps and r.done == 0 and isinstance(r.error, IndexError)


def test_step_table_equals_the_scalar_form():
    """The vectorised step table of the fused launches equals, bit for bit, the table built entry by entry
    as the stage launches' blend weights are (fields.py:423-424)."""
    import ctypes

    import numpy as np

    from offline_particles_b200 import _lib
    from offline_particles_b200.timesteppers import step_table

    rng = np.random.default_rng(3)
    for dtype in (np.dtype(np.float32), np.dtype(np.float64)):
        entries = [np.float64(v) for v in np.concatenate([rng.uniform(0, 40, 500), np.arange(0, 12, 0.25),
                                                           [3.0 - 2 ** -40, 7.0, 1e-18]])]
        slot = {k: k % 8 for k in range(64)}
        table, its = step_table(entries, dtype, lambda It: (slot[It], slot[It + 1]))
        for j, tidx in enumerate(entries):
            It, ft = divmod(tidx, 1)
            It = int(It)
            ft = dtype.type(ft)
            gt = dtype.type(1 - ft)
            want = _lib.opb_time(slot[It], slot[It + 1], float(ft), float(gt))
            assert its[j] == It
            assert bytes(table[j]) == bytes(want), (j, tidx)
        assert ctypes.sizeof(table) == len(entries) * ctypes.sizeof(_lib.opb_time)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_steps_to_interval_end_fast_path_equals_the_generic_one(seed):
    """steps_to_interval_end on Python floats (get_time_index's fast path inlined) gives the step counts
    of the path through get_time_index, for odd time arrays, dt that do not divide the spacing, and starts
    next to snapshot times."""
    rng = np.random.default_rng(seed)
    for _ in range(20):
        nt = int(rng.integers(3, 30))
        t_arr = np.cumsum(np.concatenate([[rng.uniform(-5e4, 5e4)], rng.choice([3600.0, 1800.0, 977.3], nt - 1)]))
        dt = np.float64(rng.choice([120.0, 300.0, 61.7, 3600.0]))
        start = t_arr[int(rng.integers(0, nt - 1))] + rng.choice([0.0, 1e-9, dt / 3])
        for maker in (ab3_w_advection_timestepper, rk2_w_advection_timestepper):
            ts = maker(t_arr, dt, time=np.float64(start))
            fast = [ts.steps_to_interval_end(k) for k in (0, 1, 5, 64, 200)]
            ts.__dict__["_float_times_cache"] = (ts.time_array, None)  # force the generic path
            slow = [ts.steps_to_interval_end(k) for k in (0, 1, 5, 64, 200)]
            assert fast == slow, (t_arr, dt, start)
