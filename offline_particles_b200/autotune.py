"""Autotuner for the batched release launch.

Picks the work order (Morton buckets walked in turn across releases, or one
release after another), the launch shape (CTA size, resident warps per SM,
which sets the register budget) and the re-sort interval of ``ReleaseBatch`` by timing them
on a sample of the caller's own workload, and keeps the answer in a JSON
cache keyed by the device, the grid and the workload's shape.

The sample: every release keeps its scheme, dt and validation, with
``sample_fraction`` of its particles, and all start together at the first
release's interval, so that one measured interval holds the whole mix.  The
work order and then the launch shape are timed first (``shape_intervals``
intervals each, re-sort interval fixed), then the re-sort interval with the
best of both over
``sort_intervals`` intervals (long enough that locality decays and re-sorts
pay for themselves or not).

Field storage dtype is not a free axis here: the batched kernel computes in
float64 on the fields' own storage (float32 or float64), and bfloat16/float16
storage fails the 1 m p99 separation bound after 7 days (the precision
study), so the tuner reports the storage dtype it was given.
"""

from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .batching import Release, ReleaseBatch

CACHE_PATH = Path(os.environ.get("OPB_AUTOTUNE_CACHE", Path(__file__).resolve().parent / "_lib" / "autotune.json"))
SHAPES = list(_lib.BATCH_SHAPES)
BUCKETS = (0, 64, 256, 1024)
SORT_INTERVALS = (1, 2, 4, 8, 16)


def _signature(batch_fieldset, releases: list[Release], device) -> str:
    fs = batch_fieldset
    n = sum(len(r) for r in releases)
    rk2 = sum(r.scheme == _lib.SCHEME_RK2 for r in releases)
    dts = sorted({r.dt for r in releases})
    dtype = sorted({str(fs[name].storage) for name in ("u", "v", "w", "zeta") if name in fs})
    return json.dumps({"device": torch.cuda.get_device_name(device), "grid": [fs.z_size, fs.y_size, fs.x_size],
                       "storage": dtype, "particles_log2": int(math.log2(max(n, 1))),
                       "releases_log2": int(math.log2(max(len(releases), 1))),
                       "rk2_share": round(rk2 / max(len(releases), 1), 1), "dt": dts}, sort_keys=True)


def _load_cache(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _sample(releases: list[Release], fraction: float, t0: float, nsteps: int) -> list[Release]:
    out = []
    for r in releases:
        m = max(1, int(round(len(r) * fraction)))
        ts = type(r.timestepper)
        st = r.timestepper
        # the same stepper at the common start time
        clone = ts.__new__(ts)
        clone.__dict__.update(st.__dict__)
        clone.set_time(np.float64(t0))
        status = r.status if isinstance(r.status, (int, np.integer)) else np.asarray(r.status)[:m]
        out.append(Release(clone, nsteps, r.zidx[:m], r.yidx[:m], r.xidx[:m], status=status))
    return out


def _time_config(fieldset, releases, t0, warm, measure, **kw) -> float:
    """Particle-steps/s of ``measure`` intervals after ``warm`` untimed ones."""
    steps = 0
    batch = ReleaseBatch(fieldset, releases, **kw)
    for _ in range(warm):
        batch.step_interval()
    torch.cuda.synchronize()
    before = batch.particle_steps
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(measure):
        if not batch.step_interval():
            break
    e.record()
    torch.cuda.synchronize()
    steps = batch.particle_steps - before
    ms = s.elapsed_time(e)
    del batch
    return steps / (ms * 1e-3) if ms > 0 else 0.0


def autotune(fieldset, releases: list[Release], *, device=None, sample_fraction: float = 0.25,
             shape_intervals: int = 4, sort_intervals: int = 24, warm: int = 1, cache: Path | None = CACHE_PATH,
             force: bool = False) -> dict:
    """Best ``{"block", "warps_per_sm", "split_schemes", "sort_interval", "buckets"}`` for this workload
    (cached), plus the timings."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    key = _signature(fieldset, releases, dev)
    store = _load_cache(cache) if cache is not None else {}
    if not force and key in store:
        return dict(store[key], cached=True)
    t_start = time.perf_counter()
    T = [float(t) for t in releases[0].timestepper.time_array]
    t0 = min(float(r.timestepper.time) for r in releases)
    j0 = max(0, int(np.searchsorted(T, t0, side="right")) - 1)
    t0 = T[j0]
    dt_max = max(r.dt for r in releases)
    span = (warm + max(shape_intervals, sort_intervals) + 1) * (T[j0 + 1] - T[j0])
    nsteps = int(span / min(r.dt for r in releases)) + 1
    if j0 + warm + max(shape_intervals, sort_intervals) + 3 >= len(T) or dt_max > T[j0 + 1] - T[j0]:
        raise ValueError("not enough snapshots after the first release to tune on")
    orders = {}
    for nb in BUCKETS:
        sample = _sample(releases, sample_fraction, t0, nsteps)
        orders[str(nb)] = _time_config(fieldset, sample, t0, warm, shape_intervals, device=dev, block=256,
                                       warps_per_sm=16, sort_interval=4, buckets=nb)
    buckets = int(max(orders, key=orders.get))
    shapes = {}
    for block, warps, split in [(b, w, True) for b, w in SHAPES] + [(256, 16, False)]:
        sample = _sample(releases, sample_fraction, t0, nsteps)
        shapes[f"{block}x{warps}x{'split' if split else 'one'}"] = _time_config(
            fieldset, sample, t0, warm, shape_intervals, device=dev, block=block, warps_per_sm=warps,
            sort_interval=4, buckets=buckets, split_schemes=split)
    best_shape = max(shapes, key=shapes.get)
    block, warps, split = best_shape.split("x")
    block, warps, split = int(block), int(warps), split == "split"
    sorts = {}
    for si in SORT_INTERVALS:
        sample = _sample(releases, sample_fraction, t0, nsteps)
        sorts[str(si)] = _time_config(fieldset, sample, t0, warm, sort_intervals, device=dev, block=block,
                                      warps_per_sm=warps, sort_interval=si, buckets=buckets, split_schemes=split)
    best_sort = int(max(sorts, key=sorts.get))
    result = {"block": block, "warps_per_sm": warps, "split_schemes": split, "sort_interval": best_sort,
              "buckets": buckets,
              "order_rates": orders, "shape_rates": shapes, "sort_rates": sorts, "sample_fraction": sample_fraction,
              "field_storage": sorted({str(fieldset[n].storage) for n in ("u", "v", "w", "zeta") if n in fieldset}),
              "tuning_s": time.perf_counter() - t_start}
    if cache is not None:
        store = _load_cache(cache)
        store[key] = result
        cache.parent.mkdir(parents=True, exist_ok=True)
        tmp = cache.with_suffix(f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps(store, indent=1, sort_keys=True))
        os.replace(tmp, cache)
    return dict(result, cached=False)
