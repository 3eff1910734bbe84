#!/usr/bin/env python
"""Benchmark: particle-steps/s of the ROMS advection step on B200.

Workload (the plain GPU drop-in at production size): synthetic ROMS-like
grid 1024 x 768 x 50 (float32 fields, hourly snapshots), 4,194,304 particles
uniform in wet cells, AB3 w-advection at dt = 120 s, as the ROMS preset
``ab3_w_advection_timestepper`` runs it (validation pre-step, AB3, zidx
post-step).  A "step" is one AB3 step of every particle.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  ``value``: fields and particles resident in HBM,
K steps through ``Simulation.run`` (fused multi-step launches), CUDA events
on the launching stream, max over ranks.  ``e2e``: the same K steps through
the public API from host buffers -- particle indices copied in from pinned
memory, every snapshot streamed from pinned host memory through the device
ring, results copied back -- all inside the timed region.  ``--impl
reference`` times the CPU implementation of the path (the oracle restatement
of the reference's Cython/OpenMP kernels and numpy time blend) on the host's
cores.  Multi-GPU runs shard particles (weak scaling, no collective on the
data path).
"""

from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s (1 B200) vs plain GPU path"
UNIT = "particle-steps/s"
STAGGERS = {
    "u": ("center", "center", "inner"),
    "v": ("center", "inner", "center"),
    "w": ("outer", "center", "center"),
    "zeta": ("invariant", "center", "center"),
    "h": ("invariant", "center", "center"),
    "dx": ("invariant", "center", "center"),
    "dy": ("invariant", "center", "center"),
    "C": ("center", "invariant", "invariant"),
}
TD = ("u", "v", "w", "zeta")
# id ranges of the end-to-end simulation (Simulation(result_ranges=...)): its last launch runs range by range
# and each range's results are copied back while the next computes
E2E_RANGES = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--particles", type=int, default=4_194_304)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=768)
    ap.add_argument("--nz", type=int, default=50)
    ap.add_argument("--dt", type=float, default=120.0)
    ap.add_argument("--ring-size", type=int, default=8, help="device snapshot slots of the end-to-end arm")
    ap.add_argument("--e2e-ranges", type=int, default=E2E_RANGES,
                    help="id ranges of the end-to-end simulation (Simulation(result_ranges=...))")
    ap.add_argument("--layout", choices=("auto", "octets", "quads", "pairs", "plain"), default="auto",
                    help="how the kernels read snapshots: auto (the library defaults: pairs in the fused "
                         "steppers where they pay, quads in the batched launch), octets, quads, pairs (every "
                         "launch), or plain snapshots")
    ap.add_argument("--no-bundles", action="store_true",
                    help="read h, zeta, dx, dy as separate fields (no 2-D bundles)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget-s", type=float, default=25.0)
    ap.add_argument("--study", choices=("precision", "batched", "serving", "launch"), default=None,
                    help="precision: float64 vs float32 arithmetic with float32/float16/bfloat16 storage, "
                         "separation in metres after --days; batched: release experiments in one batch vs "
                         "one after another through the plain path")
    ap.add_argument("--days", type=str, default="1,3,7")
    ap.add_argument("--release-box", type=str, default=None,
                    help="--study launch: release in a box of nz,ny,nx cells at the middle of the grid")
    # batched releases (--study batched)
    ap.add_argument("--batch-grid", type=str, default="40,512,512", help="nz,ny,nx of the batched workload")
    ap.add_argument("--experiments", type=int, default=256)
    ap.add_argument("--count-range", type=str, default="1e3,1e6", help="log-uniform particle counts")
    ap.add_argument("--count-scale", type=float, default=1.0, help="multiply every experiment's particle count")
    ap.add_argument("--release-days", type=float, default=10.0)
    ap.add_argument("--duration-days", type=str, default="1,20")
    ap.add_argument("--batch-dt", type=float, default=180.0)
    ap.add_argument("--block", type=int, default=None, help="batched launch shape (default: autotuned)")
    ap.add_argument("--warps-per-sm", type=int, default=None)
    ap.add_argument("--sort-interval", type=int, default=None)
    ap.add_argument("--buckets", type=int, default=None)
    ap.add_argument("--no-plain", action="store_true", help="skip the one-release-at-a-time arm")
    # serving (--study serving)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson request rate (1/s)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="arrival window (s)")
    ap.add_argument("--serve-count", type=str, default="100,2e6", help="log-uniform particles per request")
    ap.add_argument("--serve-count-scale", type=float, default=1.0)
    ap.add_argument("--serve-days", type=str, default="1,30", help="request duration range (days)")
    ap.add_argument("--serve-budget-gb", type=float, default=60.0, help="HBM budget for particle state")
    ap.add_argument("--serve-plain", type=int, default=64, help="requests of the trace the plain arm runs")
    ap.add_argument("--serve-plain-budget-s", type=float, default=30.0, help="seconds of plain-arm service")
    ap.add_argument("--serve-drain", action="store_true",
                    help="serve every request to its end (only a stream the GPU keeps up with drains)")
    ap.add_argument("--no-batched", action="store_true", help="default run: skip the config-4 batched block")
    ap.add_argument("--no-served", action="store_true", help="default run: skip the config-5 served block")
    ap.add_argument("--no-streamed", action="store_true", help="default run: skip the streamed-week block")
    ap.add_argument("--stream-days", type=float, default=7.0, help="model days of the streamed-week block")
    return ap.parse_args()


def workload_config(a, nt: int, pair_bytes: float | None = None) -> dict:
    state = a.particles * (1 + 13 * 8)
    pair = pair_bytes if pair_bytes is not None else 2 * 4 * (a.nz * a.ny * (a.nx - 1) + a.nz * (a.ny - 1) * a.nx
                                                               + (a.nz + 1) * a.ny * a.nx + a.ny * a.nx)
    return {
        "workload": f"AB3 w-advection, {a.nx}x{a.ny}x{a.nz} float32 synthetic ROMS grid, {a.particles:,} particles "
                    f"per GPU, dt={a.dt:g} s",
        "grid": [a.nz, a.ny, a.nx],
        "particles_per_gpu": a.particles,
        "scheme": "ab3",
        "dt_s": a.dt,
        "field_dtype": "float32",
        "state_dtype": "float64",
        "snapshots_resident": nt,
        "l2": f"inputs larger than L2 (snapshot pair {pair / 1e6:.0f} MB, particle state {state / 1e6:.0f} MB "
              f"per GPU; L2 126 MB), no flush",
        "parallelism": f"particle shards x{a.gpus}" if a.gpus > 1 else "single GPU",
    }


# --------------------------------------------------------------- inputs
def make_grid(a, nt: int):
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    return SyntheticROMS(GridSpec(nx=a.nx, ny=a.ny, nz=a.nz, nt=nt, seed=2, dtype="float32"))


def make_inputs(a, rank: int, steps: int | None = None):
    """Host snapshots for ``steps`` steps from t = 0 (default: warm-up + timed steps), and the release."""
    span = (a.warmup + a.steps if steps is None else steps) * a.dt
    nt = int(math.floor(span / 3600.0)) + 3
    grid = make_grid(a, nt)
    snaps = {name: np.stack([grid.snapshot(k)[name] for k in range(nt)]) for name in TD}
    z, y, x = grid.release(a.particles, seed=1000 + rank)
    return grid, snaps, (z, y, x), nt


def field_bytes(grid, snaps) -> dict:
    per_snap = sum(snaps[n][0].nbytes for n in TD)
    static = grid.h.nbytes + grid.dx.nbytes + grid.dy.nbytes + grid.C.nbytes
    return {"snapshot": per_snap, "pair": 2 * per_snap, "static": static}


def build_sim(grid, sources: dict, n: int, a, *, ring_size: int = 4, **sim_kw):
    import offline_particles_b200 as opb

    kw = {}
    for name in TD:
        kw[name] = opb.TimeDependentField.from_tensor(sources[name], *STAGGERS[name], ring_size=ring_size)
    for name, arr in (("h", grid.h), ("dx", grid.dx), ("dy", grid.dy), ("C", grid.C)):
        kw[name] = opb.StaticField.from_numpy(arr, *STAGGERS[name])
    nt = sources["u"].shape[0]
    fs = opb.Fieldset(nt, a.nz, a.ny, a.nx, constants={"hc": grid.hc, "NZ": a.nz}, **kw)
    ts = opb.roms.ab3_w_advection_timestepper(grid.time_array[:nt], np.float64(a.dt))
    return opb.SimulationBuilder(ts, fs).build_simulation(n, **sim_kw), fs


def window_plan(a) -> dict:
    """Where the timed K steps sit in the run.

    The per-interval work (a new snapshot pair for u, v, w and the zeta bundle
    at every snapshot-interval boundary; a Morton re-sort at the first boundary
    at least ``sort_interval`` steps after the last) belongs in the timed
    region.  With P steps per snapshot interval, re-sorts fall every R =
    ceil(sort_interval / P) * P steps.  The K timed steps straddle the first
    re-sort boundary B >= W + ceil(K / 2): steps [B - K // 2, B - K // 2 + K),
    after at least W untimed warm-up steps.  ``amortised`` times the R steps
    [B, B + R) again on a second simulation: whole intervals with their pair
    builds and one re-sort, the steady-state rate.
    """
    from offline_particles_b200.simulation import DEFAULT_SORT_INTERVAL

    P = 3600.0 / a.dt
    if abs(P - round(P)) > 1e-9 or P < 1:
        return {"start": a.warmup, "boundary": None, "resort_every": None, "steps_per_interval": None,
                "last_step": a.warmup + a.steps}
    P = int(round(P))
    R = -(-DEFAULT_SORT_INTERVAL // P) * P
    B = R * max(1, -(-(a.warmup + (a.steps + 1) // 2) // R))
    start = B - a.steps // 2
    return {"start": start, "boundary": B, "resort_every": R, "steps_per_interval": P,
            "last_step": max(start + a.steps, B + R)}


# --------------------------------------------------------------- clocks
class ClockSampler:
    """NVML samples of the SM clock and clock-event reasons every ``period_s`` while running (reads only)."""

    REASONS = (("nvmlClocksEventReasonHwSlowdown", "hw_slowdown"),
               ("nvmlClocksEventReasonHwThermalSlowdown", "hw_thermal_slowdown"),
               ("nvmlClocksEventReasonSwThermalSlowdown", "sw_thermal_slowdown"),
               ("nvmlClocksEventReasonSwPowerCap", "sw_power_cap"),
               ("nvmlClocksEventReasonHwPowerBrakeSlowdown", "hw_power_brake"))

    def __init__(self, index: int, period_s: float = 0.01) -> None:
        self.index = index
        self.period_s = period_s
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self.stop = threading.Event()
        self.nv = None

    def __enter__(self):
        """Start sampling (again: the samples of every ``with`` block add up)."""
        self.stop.clear()
        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception:  # no NVML: the summary says so
            self.nv = None
        return self

    def _run(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
            except Exception:
                pass
            self.stop.wait(self.period_s)

    def __exit__(self, *exc):
        if self.nv is not None:
            self.stop.set()
            self.t.join(timeout=5)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"], "samples": 0}
        reasons = set()
        for _, bits in self.samples:
            for attr, name in self.REASONS:
                mask = getattr(self.nv, attr, 0)
                if mask and bits & mask:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "source": f"NVML, every {self.period_s * 1e3:g} ms"}


# --------------------------------------------------------------- timing helpers
class LaunchTimer:
    """CUDA events around every fused launch, on the stream the kernel runs on."""

    def __init__(self) -> None:
        import torch

        self.torch = torch
        self.pairs = []
        self.steps = []

    def before(self, nsteps: int) -> None:
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.torch.cuda.current_stream())
        self.pairs.append([e, None])
        self.steps.append(nsteps)

    def after(self, nsteps: int) -> None:
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.torch.cuda.current_stream())
        self.pairs[-1][1] = e

    def durations_ms(self) -> list[float]:
        return [a.elapsed_time(b) for a, b in self.pairs]


# --------------------------------------------------------------- CPU path
def cpu_run(grid, snaps, zyx, a, budget_s: float) -> dict:
    """The reference's own code on this host's cores when its compiled form is in oracle/_ref (its Cython/
    OpenMP kernels and numpy time blend, through its public API), else the oracle (the same algorithm
    restated: numpy blend + C/OpenMP loops), on this workload."""
    from oracle import ref_import

    fields = dict(snaps)
    fields.update(h=grid.h, dx=grid.dx, dy=grid.dy, C=grid.C)
    n = zyx[0].size
    if ref_import.compiled_available():
        from oracle import ref_run

        r = ref_run.time_ab3(grid.time_array, fields, grid.hc, a.nz, a.dt, zyx, budget_s=budget_s)
        return {"value": r["particle_steps_per_s"], "unit": UNIT, "cores": r["threads"], "kind": "reference",
                "physical_cores": r["physical_cores"], "logical_cpus": r["logical_cpus"],
                "sample": f"{r['steps']} AB3 steps of all {n:,} particles on the same grid after {r['warmup']} "
                          f"warm-up step ({r['seconds']:.1f} s): the reference's Simulation.step() with its ROMS "
                          f"preset, Cython/OpenMP kernels and numpy time blend, {r['threads']} OpenMP threads on "
                          f"{r['physical_cores']} physical cores"}
    from oracle import oracle as O
    from oracle.ref_run import openmp_threads, physical_cores

    orc = O.OracleROMS(grid.time_array[: snaps["u"].shape[0]], fields, hc=grid.hc, scheme="ab3",
                       dt=np.float64(a.dt))
    p = O.new_particles(n, "ab3")
    p["zidx"][:], p["yidx"][:], p["xidx"][:] = zyx
    p["status"][:] = O.MULTISTEP_1
    t0 = time.perf_counter()
    orc.step(p)  # untimed warm-up step
    first = time.perf_counter() - t0
    steps = max(1, min(30, int(budget_s / max(first, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.step(p)
    el = time.perf_counter() - t0
    threads = openmp_threads()
    return {"value": n * steps / el, "unit": UNIT, "cores": threads, "kind": "port",
            "physical_cores": physical_cores(), "logical_cpus": os.cpu_count(),
            "sample": f"{steps} AB3 steps of all {n:,} particles on the same grid after 1 warm-up step "
                      f"({el:.1f} s): the oracle restatement (numpy time blend + C/OpenMP kernels), {threads} "
                      f"OpenMP threads; the compiled reference was not in oracle/_ref"}


def reference_arm(a) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    grid, snaps, zyx, nt = make_inputs(a, 0, steps=a.warmup + a.steps + 1)
    budget = max(10.0, min(150.0, 3.0 * a.cpu_budget_s))
    cb = cpu_run(grid, snaps, zyx, a, budget)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": a.particles / cb["value"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a, nt), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- B200 path
class Counters:
    """Observers counting the per-interval work inside a region: Morton re-sorts and snapshot-pair builds."""

    def __init__(self) -> None:
        from offline_particles_b200 import fields as fmod
        from offline_particles_b200 import particles as pmod

        self.sorts, self.builds = [], []
        self._mods = (pmod.sort_observers, fmod.pair_observers)

    def __enter__(self):
        self._s = lambda: self.sorts.append(1)
        self._b = lambda: self.builds.append(1)
        self._mods[0].append(self._s)
        self._mods[1].append(self._b)
        return self

    def __exit__(self, *exc):
        self._mods[0].remove(self._s)
        self._mods[1].remove(self._b)


def resident_sim(grid, dsrc, zyx, a, upto: int):
    """A simulation on resident snapshots, advanced untimed to step ``upto``."""
    import offline_particles_b200 as opb

    sim, _ = build_sim(grid, dsrc, a.particles, a)
    sim.set_indices(*zyx)
    sim.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
    if upto:
        sim.run(upto)
    sim.synchronize()
    return sim


def timed_run(ranks, sim, nsteps: int):
    """``sim.run(nsteps)`` between barriers (slowest rank's CUDA-event time), with CUDA events around every
    fused launch and counts of the re-sorts and pair builds it made."""
    import torch

    from offline_particles_b200 import timesteppers

    timer = LaunchTimer()
    timesteppers.launch_observers.append(timer)
    first = {}

    def work():
        first["t0"] = torch.cuda.Event(enable_timing=True)
        first["t0"].record()
        sim.run(nsteps)

    try:
        with Counters() as cnt:
            ms = ranks.timed_ms(work)
    finally:
        timesteppers.launch_observers.remove(timer)
    sim.synchronize()
    # device time before the first launch: host work inside the region (planning, table building, the sort
    # and pair builds it enqueued first)
    lead_ms = first["t0"].elapsed_time(timer.pairs[0][0]) if timer.pairs else None
    return ms, timer, cnt, lead_ms


def kernel_counters() -> dict | None:
    """ncu counters of the headline kernel (profiles/k_ab3_steps_config2_counters.json) when they were taken
    on the current kernel sources: the file records the SHA-256 of the sources it was measured on."""
    import hashlib

    path = ROOT / "profiles" / "k_ab3_steps_config2_counters.json"
    try:
        rec = json.loads(path.read_text())
    except (OSError, ValueError):
        return None
    h = hashlib.sha256()
    for rel in rec.get("sources", []):
        try:
            h.update((ROOT / rel).read_bytes())
        except OSError:
            return None
    if h.hexdigest() != rec.get("sources_sha256"):
        return {"stale": True, "path": str(path.relative_to(ROOT))}
    return rec


def b200_arm(a) -> None:
    import torch

    import offline_particles_b200 as opb
    from offline_particles_b200 import fields as fmod
    from offline_particles_b200 import timesteppers
    from offline_particles_b200.sharding import Ranks

    ranks = Ranks()
    rank, world, local = ranks.rank, ranks.world, ranks.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = a.particles
    plan = window_plan(a)
    nt_dev = int(math.floor(plan["last_step"] * a.dt / 3600.0)) + 3
    grid = make_grid(a, nt_dev)
    zyx = grid.release(n, seed=1000 + rank)

    # ---- device-resident: fused multi-step launches -------------------------------------
    dsrc = grid.device_snapshots(nt_dev)
    torch.cuda.synchronize()
    sim = resident_sim(grid, dsrc, zyx, a, plan["start"])
    # clocks during the three timed regions of the resident arm (the window, the amortised steps and
    # the plain steps): a few ms each, sampled every ms
    clocks = ClockSampler(local, period_s=0.001)
    with clocks:
        run_ms, timer, cnt, lead_ms = timed_run(ranks, sim, a.steps)
    launch_ms = timer.durations_ms()
    launch_steps = timer.steps
    active = int((sim.particles.tensor("status") & 0x80).eq(0).sum().item())
    del sim

    # ---- amortised: whole snapshot intervals with their pair builds and one re-sort ------------
    amort = None
    if plan["boundary"] is not None:
        sim = resident_sim(grid, dsrc, zyx, a, plan["boundary"])
        with clocks:
            am_ms, _, am_cnt, _ = timed_run(ranks, sim, plan["resort_every"])
        amort = {"value": world * n * plan["resort_every"] / (am_ms * 1e-3), "unit": UNIT,
                 "steps": plan["resort_every"], "first_step": plan["boundary"],
                 "ms_per_step": am_ms / plan["resort_every"], "sorts": len(am_cnt.sorts),
                 "pair_builds": len(am_cnt.builds)}
        del sim

    # ---- plain path: Simulation.step(), one fused launch per step, same window --------------
    sim = resident_sim(grid, dsrc, zyx, a, plan["start"])

    def steps_one_by_one():
        for _ in range(a.steps):
            sim.step()

    with clocks:
        step_ms = ranks.timed_ms(steps_one_by_one)
    sim.synchronize()
    del sim, dsrc
    torch.cuda.empty_cache()

    # ---- end to end from host buffers --------------------------------------------------
    nt_host = int(math.floor(a.steps * a.dt / 3600.0)) + 3
    hsrc = grid.device_snapshots(nt_host)
    psrc = {k: v.cpu().pin_memory() for k, v in hsrc.items()}
    del hsrc
    torch.cuda.empty_cache()
    hz, hy, hx = (torch.from_numpy(v).pin_memory() for v in zyx)
    outs = {k: torch.empty(n, dtype=torch.float64, pin_memory=True) for k in ("zidx", "yidx", "xidx")}
    outs["status"] = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    # the box's pinned host -> device bandwidth, for reading e2e (one snapshot of u)
    probe = torch.empty_like(psrc["u"][0], device=dev)
    probe.copy_(psrc["u"][0], non_blocking=True)
    torch.cuda.synchronize()
    hs, he = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hs.record()
    for k in range(3):
        probe.copy_(psrc["u"][k % psrc["u"].shape[0]], non_blocking=True)
    he.record()
    torch.cuda.synchronize()
    h2d_gbs = 3 * probe.numel() * probe.element_size() / (hs.elapsed_time(he) * 1e-3) / 1e9
    del probe
    gsnap = {k: v.numpy() for k, v in psrc.items()}
    fb = field_bytes(grid, gsnap)
    grid_h = grid
    # untimed warm-up of the same path (allocator, ring, copy stream)
    simw, _ = build_sim(grid_h, psrc, n, a, ring_size=a.ring_size, result_ranges=a.e2e_ranges)
    simw.set_indices(hz, hy, hx)
    simw.run(a.warmup, results=outs)
    simw.synchronize()
    del simw
    gc.collect()  # the warm-up simulation's teardown (reference cycles) stays out of the timed region
    # particle storage in 4 id ranges: the results of each range stream back while the next computes
    sim3, fs3 = build_sim(grid_h, psrc, n, a, ring_size=a.ring_size, result_ranges=a.e2e_ranges)
    # device buffers for the results in original order (allocated before the region, as a caller that
    # reads results every run would keep them)
    sim3.reserve_results(outs)
    host = {}
    # timeline of the region on the device: events on the compute stream, around every fused launch and
    # after every snapshot upload (on the copy stream)
    marks, uploads = {}, []
    e2e_timer = LaunchTimer()

    def on_upload(k, stream):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        uploads.append(ev)

    def mark(name):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks[name] = ev

    def e2e():
        mark("start")
        w0 = time.perf_counter()
        sim3.set_indices(hz, hy, hx)
        sim3.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
        mark("indices_in")
        w1 = time.perf_counter()
        sim3.run(a.steps, results=outs)
        mark("results_out")
        w2 = time.perf_counter()
        host.update(set_indices=(w1 - w0) * 1e3, run=(w2 - w1) * 1e3)

    fmod.upload_observers.append(on_upload)
    timesteppers.launch_observers.append(e2e_timer)

    m0 = torch.cuda.memory_stats(dev)
    wall0 = time.perf_counter()
    e2e_dev_ms = ranks.timed_ms(e2e)
    wall_e2e = time.perf_counter() - wall0
    fmod.upload_observers.remove(on_upload)
    timesteppers.launch_observers.remove(e2e_timer)
    t0 = marks["start"]
    timeline = {k: t0.elapsed_time(v) for k, v in marks.items() if k != "start"}
    if uploads:
        timeline["uploads_done"] = max(t0.elapsed_time(u) for u in uploads)
        timeline["uploads"] = len(uploads)
    if e2e_timer.pairs:
        timeline["first_launch_start"] = t0.elapsed_time(e2e_timer.pairs[0][0])
        timeline["last_launch_end"] = t0.elapsed_time(e2e_timer.pairs[-1][1])
        timeline["launches"] = len(e2e_timer.pairs)
    m1 = torch.cuda.memory_stats(dev)
    # device allocations inside the region (cudaMalloc calls, and retries that freed cached blocks first)
    e2e_alloc = {"cuda_mallocs": m1.get("segment.all.allocated", 0) - m0.get("segment.all.allocated", 0),
                 "retries": m1.get("num_alloc_retries", 0) - m0.get("num_alloc_retries", 0)}
    sim3.synchronize()
    e2e_ms = ranks.max(max(e2e_dev_ms, wall_e2e * 1e3))
    h2d = 3 * 8 * n + sum(fs3[k].h2d_bytes for k in TD)
    d2h = sum(t.numel() * t.element_size() for t in outs.values())
    del sim3, fs3

    # ---- CPU baseline (rank 0, one GPU) ------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_run(grid_h, gsnap, zyx, a, a.cpu_budget_s)
    ranks.close()
    if rank != 0:
        return
    del psrc, gsnap
    gc.collect()
    torch.cuda.empty_cache()

    # ---- the batched and served forms (one GPU): config 4 and config 5 ---------------------
    batched = served = None
    if world == 1 and not a.no_batched:
        b = batched_measure(a)
        batched = {"value": b["value"], "unit": UNIT, "vs_plain": b["vs_plain"],
                   "plain_value": b["plain"]["value"] if b["plain"] else None,
                   "identical_to_plain": b["identical_to_plain"], "roofline": b["batched"]["roofline"],
                   "seconds": b["batched"]["seconds"], "launch_time_share": b["batched"]["launch_time_share"],
                   "shape": {k: b["batched"][k] for k in ("block", "warps_per_sm", "sort_interval_intervals",
                                                          "buckets", "split_schemes")},
                   "autotuned": b["batched"]["autotune"] is not None, "errors": b["batched"]["errors"],
                   "workload": b["workload"], "clocks": b["batched"]["clocks"]}
        gc.collect()
        torch.cuda.empty_cache()
    if world == 1 and not a.no_served:
        served = serving_measure(a, a.serve_seconds, a.serve_drain)
        gc.collect()
        torch.cuda.empty_cache()
    streamed = None
    if world == 1 and not a.no_streamed:
        streamed = streamed_measure(a, h2d_gbs)

    # ---- roofline of the fused kernel -------------------------------------------------
    peak = measured_peak_gbs()
    state_bytes = 2 * (1 + 3 * 8 + 6 * 8)  # status + 3 indices + 6 AB3 history values, float64, read + written
    b_step = n * state_bytes + fb["pair"] + fb["static"]
    tot_steps = sum(launch_steps)
    kernel_ms = sum(launch_ms)
    avg_launch_ms = kernel_ms / max(1, len(launch_ms))
    avg_launch_steps = tot_steps / max(1, len(launch_steps))
    achieved = b_step * tot_steps / (kernel_ms * 1e-3) / 1e9
    ctr = kernel_counters()
    fresh = ctr is not None and not ctr.get("stale")
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": ctr["dram_bytes_per_step"] * avg_launch_steps if fresh else None,
            "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum, {ctr['traffic_case']}"
                               if fresh else "no ncu capture of the current kernel sources"),
            "peak_source": peak_source(), "algorithmic_bytes_per_step": b_step,
            "bytes_per_particle_step": b_step / n, "steps_per_launch": avg_launch_steps,
            "launch_ms": avg_launch_ms, "kernel": "k_ab3_steps<float, int, ROMS layout, pairs, 2-D bundles>"}
    if fresh:
        # the bound that applies after sorting: instruction issue (4 schedulers per SM, one warp
        # instruction per cycle each, at the SM clock sampled during the region)
        mhz = clocks.summary().get("sm_mhz") or 1965
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        issue_peak = sms * 4 * mhz * 1e6
        ps_rate = n * tot_steps / (kernel_ms * 1e-3)
        roof["issue"] = {"warp_inst_per_particle_step": ctr["warp_inst_per_particle_step"],
                         "achieved_warp_inst_per_s": ctr["warp_inst_per_particle_step"] * ps_rate,
                         "peak_warp_inst_per_s": issue_peak,
                         "frac": ctr["warp_inst_per_particle_step"] * ps_rate / issue_peak,
                         "ncu_issue_active": ctr.get("issue_active"), "source": ctr["inst_case"]}
    elif ctr is not None:
        roof["counters"] = "stale: recorded on other kernel sources"

    total = world * n * a.steps
    line = {
        "metric": METRIC, "value": total / (run_ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": run_ms / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ROMS-like grid; no ROMS output offline)",
        "config": workload_config(a, nt_dev),
        "window": {"first_step": plan["start"], "untimed_steps_before": plan["start"],
                   "straddles_resort_boundary": plan["boundary"],
                   "note": "the K timed steps straddle a snapshot-interval boundary at which a new snapshot pair "
                           "is built and particles are re-sorted"},
        "amortised": amort,
        "plain_step": {"value": total / (step_ms * 1e-3), "unit": UNIT, "ms_per_step": step_ms / a.steps,
                       "path": "Simulation.step(): one fused launch (validation + AB3 + post) per step"},
        "e2e": {"value": total / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d / a.steps),
                "d2h_bytes_per_step": int(d2h / a.steps),
                "path": "Simulation.set_indices from pinned host + run(K, results=...) streaming every snapshot "
                        "from pinned host memory, zidx/yidx/xidx/status copied back in original order into pinned "
                        f"host memory ({a.e2e_ranges} id range(s), each read back as its launch ends)",
                "h2d_gbs_measured": h2d_gbs, "device_ms": e2e_dev_ms, "wall_ms": wall_e2e * 1e3,
                "host_ms": host, "allocator": e2e_alloc, "timeline_ms": timeline,
                "h2d_bound_value": total / ((h2d + d2h) / (h2d_gbs * 1e9)) if h2d_gbs else None},
        "roofline": roof,
        "gpu_launches": len(launch_ms) + 2 * len(cnt.sorts) + len(cnt.builds),
        "sorts_in_timed_region": len(cnt.sorts),
        "pair_builds_in_timed_region": len(cnt.builds),
        "kernel_ms_in_timed_region": kernel_ms,
        "lead_ms_before_first_launch": lead_ms,
        "snapshot_layout": a.layout, "bundles_2d": not a.no_bundles,
        "active_particles_end": active,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
        "batched": batched,
        "served": served,
        "streamed_week": streamed,
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- precision study
def precision_study(a) -> None:
    """Trajectory separation of the float32 steppers against the float64 (bit-exact) path.

    The config-2 workload for max(--days) simulated days; snapshots are
    generated on the device (all resident), particles released as for the
    headline.  Every arm starts from the same state; separations are taken at
    each requested day over particles active in both arms: horizontal
    hypot(dx*d_xidx, dy*d_yidx) and vertical |d z|, in metres.
    """
    import torch

    import offline_particles_b200 as opb
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    torch.cuda.set_device(0)
    days = [float(d) for d in a.days.split(",")]
    steps_at = [int(round(d * 86400.0 / a.dt)) for d in days]
    nt = int(math.ceil(max(days) * 24.0)) + 2
    grid = SyntheticROMS(GridSpec(nx=a.nx, ny=a.ny, nz=a.nz, nt=nt, seed=2, dtype="float32"))
    t0 = time.perf_counter()
    snaps = grid.device_snapshots(nt)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    z0, y0, x0 = grid.release(a.particles, seed=1000)
    dxm = grid.spec.dx
    arms = (("float64", None), ("float32", None), ("float32", "float16"), ("float32", "bfloat16"))
    results, positions = {}, {}
    for arith, storage in arms:
        name = arith if storage is None else f"{arith}+{storage}"
        kw = {n: opb.TimeDependentField.from_tensor(snaps[n], *STAGGERS[n], storage=storage) for n in TD}
        for n, arr in (("h", grid.h), ("dx", grid.dx), ("dy", grid.dy), ("C", grid.C)):
            kw[n] = opb.StaticField.from_numpy(arr, *STAGGERS[n])
        fs = opb.Fieldset(nt, a.nz, a.ny, a.nx, constants={"hc": grid.hc, "NZ": a.nz}, **kw)
        ts = opb.roms.ab3_w_advection_timestepper(grid.time_array[:nt], np.float64(a.dt))
        sim = opb.SimulationBuilder(ts, fs).build_simulation(a.particles, arithmetic=arith)
        sim.set_indices(z0, y0, x0)
        sim.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
        done, elapsed, pos = 0, 0.0, []
        for target in steps_at:
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record()
            sim.run(target - done)
            e_.record()
            torch.cuda.synchronize()
            elapsed += s_.elapsed_time(e_) * 1e-3
            done = target
            P = sim.particles
            pos.append({k: P[k] for k in ("status", "yidx", "xidx", "z")})
        sim.synchronize()
        field_pair = 2 * sum(fs[n].storage_bytes_per_snapshot for n in TD)
        b_step = a.particles * 2 * (1 + 3 * 8 + 6 * 8) + field_pair + grid.h.nbytes * 3
        results[name] = {"value": a.particles * done / elapsed, "unit": UNIT, "ms_per_step": elapsed / done * 1e3,
                         "field_storage": storage or "float32", "arithmetic": arith,
                         "algorithmic_bytes_per_step": b_step}
        positions[name] = pos
        del sim, fs, kw
        torch.cuda.empty_cache()
    ref = positions["float64"]
    for name, pos in positions.items():
        if name == "float64":
            continue
        sep = {}
        for d, p, r in zip(days, pos, ref):
            both = ((p["status"] & 0x80) == 0) & ((r["status"] & 0x80) == 0)
            hz = np.hypot((p["xidx"][both] - r["xidx"][both]) * dxm, (p["yidx"][both] - r["yidx"][both]) * dxm)
            vt = np.abs(p["z"][both] - r["z"][both])
            sep[f"day{d:g}"] = {"horizontal_mean_m": float(hz.mean()), "horizontal_p99_m": float(np.percentile(hz, 99)),
                                "vertical_mean_m": float(vt.mean()), "vertical_p99_m": float(np.percentile(vt, 99)),
                                "active_in_both": int(both.sum()),
                                "status_agreement": float(np.mean(p["status"] == r["status"]))}
        results[name]["separation_vs_float64"] = sep
    line = {"study": "precision", "metric": "trajectory separation vs the float64 path (m); particle-steps/s",
            "workload": workload_config(a, nt), "days": days, "steps": steps_at, "snapshot_generation_s": gen_s,
            "arms": results, "data": "synthetic, snapshots generated on the device"}
    print(json.dumps(line), flush=True)


FALLBACK_HBM_GBS = 6650.0


def peak_source() -> str:
    """Where the HBM peak comes from: the measured copy bandwidth, or the fallback figure."""
    return ("MEASURED_PEAKS.json hbm_gbs (of measured)" if _measured_peaks().get("hbm_gbs")
            else f"fallback {FALLBACK_HBM_GBS:g} GB/s, an earlier copy measurement on B200 (of fallback; "
                 "MEASURED_PEAKS.json absent)")


def _measured_peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def measured_peak_gbs() -> float:
    """HBM copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json), else the fallback."""
    return float(_measured_peaks().get("hbm_gbs") or FALLBACK_HBM_GBS)


class EventPairs:
    """CUDA events around each launch of a ReleaseBatch (its observer protocol)."""

    def __init__(self) -> None:
        self.pairs = []

    def before(self) -> None:
        import torch

        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.pairs.append([e, None])

    def after(self) -> None:
        import torch

        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.pairs[-1][1] = e

    def durations_ms(self) -> list[float]:
        return [s.elapsed_time(e) for s, e in self.pairs]


def batched_workload(a, grid):
    """The release experiments: log-uniform counts, uniform release times and durations, RK2/AB3 at random."""
    rng = np.random.default_rng(4)
    E = a.experiments
    lo, hi = (float(v) for v in a.count_range.split(","))
    dlo, dhi = (float(v) for v in a.duration_days.split(","))
    counts = np.maximum(1, np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), E)) * a.count_scale)).astype(int)
    t0 = rng.uniform(0.0, a.release_days * 86400.0, E)
    nsteps = np.floor(rng.uniform(dlo, dhi, E) * 86400.0 / a.batch_dt).astype(int)
    schemes = np.where(rng.random(E) < 0.5, "rk2", "ab3")
    return [dict(scheme=str(schemes[e]), t0=float(t0[e]), nsteps=int(nsteps[e]), n=int(counts[e]), seed=5000 + e)
            for e in range(E)]


def batched_measure(a) -> dict:
    """Config-4 batched releases: one ReleaseBatch vs the plain path one release at a time.

    Snapshots are generated on the device and stay resident; the plain arm
    reads them in place, the batched arm streams them device-to-device through
    a 4-slot ring (fixed slot addresses, so intervals replay CUDA graphs).
    Both arms start from the same host arrays; the timed regions include
    building each arm's particle state from them.  Every experiment's final
    state is compared bit for bit between the arms.
    """
    import torch

    import offline_particles_b200 as opb
    from offline_particles_b200.batching import Release, ReleaseBatch
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    torch.cuda.set_device(0)
    nz, ny, nx = (int(v) for v in a.batch_grid.split(","))
    specs = batched_workload(a, None)
    t_end = max(s["t0"] + s["nsteps"] * a.batch_dt for s in specs)
    nt = int(math.ceil(t_end / 3600.0)) + 2
    grid = SyntheticROMS(GridSpec(nx=nx, ny=ny, nz=nz, nt=nt, seed=4, dtype="float32"))
    t_arr = grid.time_array[:nt]
    t0 = time.perf_counter()
    snaps = grid.device_snapshots(nt)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    inputs = [grid.release(s["n"], seed=s["seed"]) for s in specs]
    total_ps = sum(s["n"] * s["nsteps"] for s in specs)
    statics = {n: opb.StaticField.from_numpy(arr, *STAGGERS[n])
               for n, arr in (("h", grid.h), ("dx", grid.dx), ("dy", grid.dy), ("C", grid.C))}

    def fieldset(ring: bool):
        kw = {n: opb.TimeDependentField.from_tensor(snaps[n], *STAGGERS[n], ring=ring, ring_size=4) for n in TD}
        return opb.Fieldset(nt, nz, ny, nx, constants={"hc": grid.hc, "NZ": nz}, **kw, **statics)

    def stepper(s):
        f = opb.roms.rk2_w_advection_timestepper if s["scheme"] == "rk2" else opb.roms.ab3_w_advection_timestepper
        return f(t_arr, np.float64(a.batch_dt), time=np.float64(s["t0"]))

    # ---- batched ---------------------------------------------------------------
    fs_ring = fieldset(True)
    tuned = None
    if a.block is None or a.warps_per_sm is None or a.sort_interval is None or a.buckets is None:
        from offline_particles_b200.autotune import autotune

        probe = [Release(stepper(s), s["nsteps"], *inputs[q]) for q, s in enumerate(specs)]
        tuned = autotune(fs_ring, probe)
        del probe
    block = a.block if a.block is not None else tuned["block"]
    warps = a.warps_per_sm if a.warps_per_sm is not None else tuned["warps_per_sm"]
    sort_interval = a.sort_interval if a.sort_interval is not None else tuned["sort_interval"]
    buckets = a.buckets if a.buckets is not None else tuned["buckets"]
    split = tuned["split_schemes"] if tuned is not None else True
    torch.cuda.empty_cache()
    timer = EventPairs()
    with ClockSampler(0) as clocks:
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record()
        rels = [Release(stepper(s), s["nsteps"], *inputs[q]) for q, s in enumerate(specs)]
        batch = ReleaseBatch(fs_ring, rels, block=block, warps_per_sm=warps, sort_interval=sort_interval,
                             buckets=buckets, split_schemes=split)
        batch.observers.append(timer)
        batch.run()
        e_.record()
        torch.cuda.synchronize()
        batch_wall = time.perf_counter() - w0
    batch_s = s_.elapsed_time(e_) * 1e-3
    launch_ms = timer.durations_ms()
    errors = [q for q, r in enumerate(rels) if r.error is not None]
    batch_res = [batch.result(r, ("zidx", "yidx", "xidx", "status")) for r in rels]
    per_snap = sum(fs_ring[n].storage_bytes_per_snapshot for n in TD)
    f_pair = 2 * per_snap + 3 * grid.h.nbytes + grid.C.nbytes
    state_b = {"rk2": 2 * (1 + 3 * 8), "ab3": 2 * (1 + 3 * 8 + 6 * 8)}
    alg_bytes = sum(s["n"] * s["nsteps"] * state_b[s["scheme"]] for s in specs) + f_pair * sum(
        st[3] for st in batch.stats)
    kernel_s = sum(launch_ms) * 1e-3
    peak = measured_peak_gbs()
    batched = {"value": total_ps / batch_s, "unit": UNIT, "seconds": batch_s, "wall_s": batch_wall,
               "launches": batch.launches, "segment_sorts": batch.sorts, "graphs": batch.graphs,
               "block": block, "warps_per_sm": warps, "sort_interval_intervals": sort_interval, "buckets": buckets,
               "split_schemes": split,
               "autotune": tuned,
               "launch_ms_median": statistics.median(launch_ms) if launch_ms else None,
               "launch_time_share": kernel_s / batch_s,
               "roofline": {"bound": "hbm", "achieved": alg_bytes / kernel_s / 1e9, "peak": peak, "unit": "GB/s",
                            "frac": alg_bytes / kernel_s / 1e9 / peak,
                            "algorithmic_bytes": alg_bytes, "peak_source": peak_source(),
                            "definition": "sum over experiments of particle-steps x state bytes (RK2 50 B, AB3 146 B) "
                                          "+ per interval the snapshot pair and statics x the most steps of one "
                                          "experiment, over the summed launch times"},
               "errors": errors, "clocks": clocks.summary()}
    del batch, fs_ring
    torch.cuda.empty_cache()

    # ---- plain: one release at a time ------------------------------------------
    plain = None
    identical = None
    if not a.no_plain:
        fs_res = fieldset(False)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record()
        plain_res = []
        per = []
        for q, s in enumerate(specs):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record()
            sim = opb.SimulationBuilder(stepper(s), fs_res).build_simulation(s["n"])
            sim.set_indices(*inputs[q])
            sim.set_particle_field("status", 10 if s["scheme"] == "ab3" else 0)
            sim.run(s["nsteps"])
            P = sim.particles
            plain_res.append({k: P[k] for k in ("zidx", "yidx", "xidx", "status")})
            ev1 = torch.cuda.Event(enable_timing=True)
            ev1.record()
            per.append((ev0, ev1))
            del sim
        e_.record()
        torch.cuda.synchronize()
        plain_s = s_.elapsed_time(e_) * 1e-3
        # plain rate by release size: where one-at-a-time leaves the GPU idle
        secs = np.array([a_.elapsed_time(b_) * 1e-3 for a_, b_ in per])
        ns = np.array([s["n"] for s in specs])
        ps = np.array([s["n"] * s["nsteps"] for s in specs], dtype=np.float64)
        bands = {}
        for lo_, hi_ in ((0, 1e4), (1e4, 1e5), (1e5, 1e7)):
            m = (ns >= lo_) & (ns < hi_)
            if m.any():
                bands[f"{lo_:.0e}-{hi_:.0e}"] = {"releases": int(m.sum()), "particle_steps": float(ps[m].sum()),
                                                  "seconds": float(secs[m].sum()),
                                                  "rate": float(ps[m].sum() / secs[m].sum())}
        plain = {"value": total_ps / plain_s, "unit": UNIT, "seconds": plain_s,
                 "wall_s": time.perf_counter() - w0, "by_release_size": bands}
        identical = all(np.array_equal(br[k].view(np.uint8), pr[k].view(np.uint8))
                        for br, pr in zip(batch_res, plain_res) for k in br)
    counts = [s["n"] for s in specs]
    del snaps
    torch.cuda.empty_cache()
    return {"metric": METRIC, "unit": UNIT,
            "value": batched["value"], "vs_plain": (batched["value"] / plain["value"]) if plain else None,
            "batched": batched, "plain": plain, "identical_to_plain": identical,
            "workload": {"grid": [nz, ny, nx], "field_dtype": "float32", "snapshots": nt,
                         "experiments": len(specs), "particles": int(sum(counts)),
                         "particles_min_max": [int(min(counts)), int(max(counts))],
                         "rk2": sum(s["scheme"] == "rk2" for s in specs), "dt_s": a.batch_dt,
                         "particle_steps": int(total_ps), "release_days": a.release_days,
                         "duration_days": a.duration_days, "count_scale": a.count_scale},
            "snapshot_generation_s": gen_s,
            "data": "synthetic; snapshots generated on the device and resident (plain reads them in place, "
                    "batched copies them into a 4-slot ring)"}


def batched_study(a) -> None:
    print(json.dumps({"study": "batched", **batched_measure(a)}), flush=True)


class TracedRequest:
    """One request of the trace before it arrives: its particles are drawn from its own seed when it is
    materialised, so a long trace holds only the arrays of requests in the system."""

    def __init__(self, grid, id: int, offset: float, n: int, scheme: str, dt: float, duration: float) -> None:
        self.grid, self.id, self.offset, self.n = grid, id, offset, n
        self.scheme, self.dt, self.duration = scheme, dt, duration

    def __len__(self) -> int:
        return self.n

    @property
    def nsteps(self) -> int:
        return round(self.duration / self.dt)

    def materialise(self):
        from offline_particles_b200.serving import ReleaseRequest

        z, y, x = self.grid.release_in_box(self.n, np.random.default_rng((5, self.id)))
        r = ReleaseRequest(z, y, x, self.scheme, self.dt, self.duration, id=self.id)
        r.offset = self.offset  # arrival time after the start of the run
        return r


def serving_trace(a, grid):
    """Poisson arrivals; per request: log-uniform count, random wet rectangle and sigma band, duration,
    scheme and dt (config-5 construction, seeded; particles drawn on arrival)."""
    rng = np.random.default_rng(5)
    lo, hi = (float(v) for v in a.serve_count.split(","))
    dlo, dhi = (float(v) for v in a.serve_days.split(","))
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / a.serve_rate)
        if t > a.serve_seconds:
            break
        n = max(1, int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))) * a.serve_count_scale)))
        dt = float(rng.choice([60.0, 120.0, 300.0]))
        days = rng.uniform(dlo, dhi)
        scheme = "rk2" if rng.random() < 0.5 else "ab3"
        reqs.append(TracedRequest(grid, len(reqs), t, n, scheme, dt, round(days * 86400.0 / dt) * dt))
    return reqs


# distinct snapshots the streamed week cycles through (pinned host memory: 8 x 478 MB on the 1024x768x50 grid)
STREAM_DISTINCT = 8


def streamed_measure(a, h2d_gbs: float | None) -> dict:
    """The headline workload over a whole model week: hourly snapshots (``--stream-days`` x 24 + 2 of
    them) streamed from pinned host memory through the fields' device rings while the particles advance,
    from ``set_indices`` to the results in pinned host memory (``run(..., results=...)``), timed on the
    device.  The series repeats ``STREAM_DISTINCT`` distinct snapshots (``synth.CyclicSnapshots``): a week
    of distinct snapshots is 81 GB of pinned memory, more than a host should be asked to pin, and the
    upload of each snapshot costs the same whatever its values.  The same run on the same snapshots
    uploaded from device memory (no PCIe) gives the compute-bound time and must match bit for bit."""
    import torch

    import offline_particles_b200 as opb
    from offline_particles_b200.synth import CyclicSnapshots

    n = a.particles
    steps = int(round(a.stream_days * 86400.0 / a.dt))
    nt = int(math.floor(steps * a.dt / 3600.0)) + 2
    grid = make_grid(a, nt)
    host_src = grid.pinned_cycle(STREAM_DISTINCT, nt)
    z, y, x = grid.release(n, seed=1000)
    hz, hy, hx = (torch.from_numpy(v).pin_memory() for v in (z, y, x))
    names = ("zidx", "yidx", "xidx", "status")

    def outs():
        o = {k: torch.empty(n, dtype=torch.float64, pin_memory=True) for k in names[:3]}
        o["status"] = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        return o

    def build(src):
        kw = {name: opb.TimeDependentField(src[name], *STAGGERS[name], ring_size=a.ring_size) for name in TD}
        for name, arr in (("h", grid.h), ("dx", grid.dx), ("dy", grid.dy), ("C", grid.C)):
            kw[name] = opb.StaticField.from_numpy(arr, *STAGGERS[name])
        fs = opb.Fieldset(nt, a.nz, a.ny, a.nx, constants={"hc": grid.hc, "NZ": a.nz}, **kw)
        ts = opb.roms.ab3_w_advection_timestepper(grid.time_array[:nt], np.float64(a.dt))
        return opb.SimulationBuilder(ts, fs).build_simulation(n, result_ranges=a.e2e_ranges), fs

    def week(src, res):
        w, _ = build(src)  # untimed warm-up of the same path
        w.set_indices(hz, hy, hx)
        w.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
        w.run(a.warmup, results=res)
        w.synchronize()
        del w
        gc.collect()
        sim, fs = build(src)
        sim.reserve_results(res)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        t0.record()
        sim.set_indices(hz, hy, hx)
        sim.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
        sim.run(steps, results=res)
        t1.record()
        torch.cuda.synchronize()
        ms = max(t0.elapsed_time(t1), (time.perf_counter() - w0) * 1e3)
        sim.synchronize()
        h2d = 3 * 8 * n + sum(fs[k].h2d_bytes for k in TD)
        del sim, fs
        gc.collect()
        return ms, h2d

    streamed = outs()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        ms, h2d = week(host_src, streamed)
    dev_src = {k: CyclicSnapshots(v.base.cuda(), nt) for k, v in host_src.items()}
    resident = outs()
    ms_dev, _ = week(dev_src, resident)
    identical = all(torch.equal(streamed[k], resident[k]) for k in names)
    d2h = sum(t.numel() * t.element_size() for t in streamed.values())
    del dev_src, host_src
    gc.collect()
    torch.cuda.empty_cache()
    total = n * steps
    bound_ms = (h2d + d2h) / (h2d_gbs * 1e9) * 1e3 if h2d_gbs else None
    return {"value": total / (ms * 1e-3), "unit": UNIT, "steps": steps, "days": a.stream_days, "snapshots": nt,
            "distinct_snapshots": STREAM_DISTINCT, "ms": ms, "h2d_bytes": h2d, "d2h_bytes": d2h,
            "pcie_bound_value": total / (bound_ms * 1e-3) if bound_ms else None,
            "from_device_value": total / (ms_dev * 1e-3), "from_device_ms": ms_dev,
            "identical_to_from_device": identical,
            "path": "Simulation.set_indices from pinned host + run(steps, results=...): every snapshot uploaded "
                    "from pinned host memory through the rings while the particles advance, results copied "
                    "back in original order",
            "clocks": clocks.summary()}


def serving_measure(a, window_s: float, drain: bool) -> dict:
    """Config-5 serving: a Poisson request stream served with continuous batching (ReleaseServer), and
    the plain path serving a sample of the same trace one request at a time.

    Snapshots of the config-4 grid are generated on the device when a ring
    asks for them (model time runs as long as the service does).  Served arm:
    requests are submitted at their arrival times (wall clock) over
    ``window_s`` seconds and admitted at interval boundaries by the HBM budget;
    latency = arrival to result in host memory.  With ``drain`` the server
    then runs until every request is done; without, it stops at the end of
    the window (a stream that offers more than the GPU serves never drains):
    requests still queued or running are counted, and their age at the end is
    a lower bound of their latency.  Served throughput counts every
    particle-step advanced in the run, finished requests or not.  Plain arm:
    the first --serve-plain finished requests, each alone through Simulation
    from the start time the server gave it (FIFO from the same arrival times;
    its results are compared bit for bit with the served ones), within
    --serve-plain-budget-s seconds.
    """
    import torch

    import offline_particles_b200 as opb
    from offline_particles_b200.serving import ReleaseRequest, ReleaseServer
    from offline_particles_b200.synth import GridSpec, SyntheticROMS

    torch.cuda.set_device(0)
    nz, ny, nx = (int(v) for v in a.batch_grid.split(","))
    grid = SyntheticROMS(GridSpec(nx=nx, ny=ny, nz=nz, nt=4, seed=4, dtype="float32"))
    a_window = a.serve_seconds
    a.serve_seconds = window_s
    try:
        reqs = serving_trace(a, grid)
    finally:
        a.serve_seconds = a_window
    nt = 400_000  # hourly snapshot indices available to the device source (45 model years)
    t_arr = np.arange(nt, dtype=np.float64) * 3600.0
    statics = {n: opb.StaticField.from_numpy(arr, *STAGGERS[n])
               for n, arr in (("h", grid.h), ("dx", grid.dx), ("dy", grid.dy), ("C", grid.C))}

    def fieldset():
        src = grid.device_source(nt)
        kw = {n: opb.TimeDependentField(src.field(n), *STAGGERS[n], ring_size=4) for n in TD}
        return opb.Fieldset(nt, nz, ny, nx, constants={"hc": grid.hc, "NZ": nz}, **kw, **statics)

    budget = int(a.serve_budget_gb * 1e9)
    server = ReleaseServer(fieldset(), t_arr, hbm_budget=budget, max_releases=1024, block=256, warps_per_sm=16,
                           buckets=256, sort_interval=4)
    offered = sum(len(r) * r.nsteps for r in reqs) / window_s
    # warm the kernels (module load, occupancy, graph capture) on a throwaway server
    warm = ReleaseServer(fieldset(), t_arr, hbm_budget=64 * server.per_particle, max_releases=4)
    wz, wy, wx = grid.release(32, seed=1)
    for sch in ("rk2", "ab3"):
        warm.submit(ReleaseRequest(wz, wy, wx, sch, 300.0, 7200.0))
    warm.drain()
    del warm
    torch.cuda.synchronize()

    timeline = []
    live = []  # every submitted request
    kept = 0
    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        i, n = 0, len(reqs)
        max_running = 0
        next_sample = 0.0
        while True:
            now = time.perf_counter() - t0
            if now >= next_sample:
                timeline.append((round(now, 2), len(server.queue), len(server.running), len(server.done)))
                next_sample += 1.0
            while i < n and reqs[i].offset <= now:
                r = reqs[i].materialise()
                r.arrival = t0 + r.offset
                server.submit(r)
                live.append(r)
                i += 1
            if len(server.done) > kept:  # keep the arrays of the requests the plain arm replays
                for r in server.done[kept:]:
                    if r.id >= a.serve_plain:
                        r.zidx = r.yidx = r.xidx = r.release = None
                        r.result = {"kept": False} if r.result is not None else None
                kept = len(server.done)
            if not drain and now >= window_s:
                break
            if not server.queue and not server.running:
                if i >= n:
                    break
                server._poll()
                time.sleep(max(0.0, min(0.002, reqs[i].offset - (time.perf_counter() - t0))))
                continue
            server.tick()
            max_running = max(max_running, len(server.running))
        if drain:
            server.drain()
        else:
            torch.cuda.synchronize()
            server._poll()
        t_end = time.perf_counter()
    span = t_end - t0
    advanced = server.batch.particle_steps
    lat = server.latencies()
    waiting = [r for r in live if r.finished is None and r.error is None]
    ages = np.array([t_end - r.arrival for r in waiting])
    every = np.concatenate([lat, ages]) if ages.size else lat
    served = {"requests_arrived": i, "requests_done": len(server.done), "rejected": len(server.rejected),
              "queued_at_end": len(server.queue), "running_at_end": len(server.running),
              "value": advanced / span, "unit": UNIT, "particle_steps_advanced": int(advanced),
              "makespan_s": span, "ticks": server.ticks, "launches": server.batch.launches,
              "latency_p50_s": float(np.percentile(lat, 50)) if lat.size else None,
              "latency_p99_s": float(np.percentile(lat, 99)) if lat.size else None,
              "latency_mean_s": float(lat.mean()) if lat.size else None,
              "latency_p50_lower_bound_s": float(np.percentile(every, 50)) if every.size else None,
              "latency_p99_lower_bound_s": float(np.percentile(every, 99)) if every.size else None,
              "max_running": max_running, "capacity_particles": server.capacity,
              "bytes_per_particle": server.per_particle,
              "timeline_s_queued_running_done": timeline[:: max(1, len(timeline) // 60)],
              "clocks": clocks.summary()}
    done = sorted(server.done, key=lambda r: r.id)
    del server
    torch.cuda.empty_cache()

    # ---- plain: the same requests one at a time, FIFO ---------------------------
    plain = None
    if a.serve_plain > 0 and done:
        fs = fieldset()
        free_at, lat_p, ps, busy, same, k = 0.0, [], 0, 0.0, 0, 0
        for r in [r for r in done if r.id < a.serve_plain]:
            if busy > a.serve_plain_budget_s:
                break
            f = opb.roms.rk2_w_advection_timestepper if r.scheme == "rk2" else opb.roms.ab3_w_advection_timestepper
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            ts = f(t_arr, np.float64(r.dt), time=np.float64(r.start_time))
            sim = opb.SimulationBuilder(ts, fs).build_simulation(len(r))
            sim.set_indices(r.zidx, r.yidx, r.xidx)
            sim.set_particle_field("status", 10 if r.scheme == "ab3" else 0)
            sim.run(r.nsteps)
            P = sim.particles
            res = {key: P[key] for key in ("zidx", "yidx", "xidx", "status")}
            service = time.perf_counter() - w0
            del sim
            busy += service
            start = max(free_at, r.offset)
            free_at = start + service
            lat_p.append(free_at - r.offset)
            ps += len(r) * r.nsteps
            same += all(np.array_equal(res[key].view(np.uint8), r.result[key].view(np.uint8)) for key in res)
            k += 1
        lat_p = np.array(lat_p)
        plain = {"requests": k, "value": ps / busy, "unit": UNIT, "busy_s": busy,
                 "latency_p50_s": float(np.percentile(lat_p, 50)), "latency_p99_s": float(np.percentile(lat_p, 99)),
                 "identical_to_served": f"{same}/{k}",
                 "note": "service times measured one request at a time (the first finished requests by arrival); "
                         "FIFO latencies from the same arrival times"}
    sizes = [len(r) for r in reqs]
    return {"metric": "served particle-steps/s and request latency p50/p99", "unit": UNIT,
            "value": served["value"], "vs_plain": served["value"] / plain["value"] if plain else None,
            "offered_particle_steps_per_s": offered, "served": served, "plain": plain,
            "workload": {"grid": [nz, ny, nx], "field_dtype": "float32", "rate_per_s": a.serve_rate,
                         "window_s": window_s, "drained": drain, "requests": len(reqs),
                         "particles_per_request": [int(min(sizes)), int(np.median(sizes)), int(max(sizes))],
                         "count_range": a.serve_count, "count_scale": a.serve_count_scale,
                         "duration_days": a.serve_days, "dt_s": [60, 120, 300],
                         "hbm_budget_gb": a.serve_budget_gb},
            "data": "synthetic; snapshots generated on the device on demand"}


def serving_study(a) -> None:
    print(json.dumps({"study": "serving", **serving_measure(a, a.serve_seconds, a.serve_drain)}), flush=True)


def launch_study(a) -> None:
    """One fused AB3 launch of exactly --steps steps after an explicit Morton sort, inside one snapshot
    interval (fields resident, no re-sort or pair build inside): the unit an ncu capture of the headline
    kernel compares between builds.  Runs --warmup steps first (their own launch), then the measured
    launch; prints its CUDA-event time per step.  Capture it with ``-k regex:k_ab3_steps -s 1 -c 1``.
    ``--release-box nz,ny,nx``: release every particle uniformly in a box of that many cells at the middle
    of the grid instead of over all wet cells, so that every gather hits the caches: the kernel's time
    without memory latency."""
    import torch

    import offline_particles_b200 as opb

    torch.cuda.set_device(0)
    steps_per_interval = int(round(3600.0 / a.dt))
    if a.warmup + a.steps > steps_per_interval:
        raise SystemExit(f"--warmup + --steps must fit one snapshot interval ({steps_per_interval} steps)")
    grid = make_grid(a, 3)
    dsrc = grid.device_snapshots(3)
    sim, _ = build_sim(grid, dsrc, a.particles, a, sort_interval=0)
    if a.release_box:
        bz, by, bx = (float(v) for v in a.release_box.split(","))
        rng = np.random.default_rng(5)
        n = a.particles
        zyx = (20.0 + rng.uniform(0, bz, n), a.ny / 2 + rng.uniform(0, by, n), a.nx / 2 + rng.uniform(0, bx, n))
    else:
        zyx = grid.release(a.particles, seed=1000)
    sim.set_indices(*zyx)
    sim.set_particle_field("status", opb.kernels.ParticleStatus.MULTISTEP_1)
    sim.sort_particles()
    sim.run(a.warmup)
    torch.cuda.synchronize()
    s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_.record()
    sim.run(a.steps)
    e_.record()
    torch.cuda.synchronize()
    ms = s_.elapsed_time(e_)
    print(json.dumps({"study": "launch", "steps": a.steps, "particles": a.particles, "grid": [a.nz, a.ny, a.nx],
                      "release_box": a.release_box,
                      "ms": ms, "ms_per_step": ms / a.steps,
                      "particle_steps_per_s": a.particles * a.steps / (ms * 1e-3)}), flush=True)


def set_layout(layout: str) -> None:
    """The snapshot layout of every launch in this process (``--layout``)."""
    from offline_particles_b200 import timesteppers

    if layout in ("octets", "quads", "pairs"):
        timesteppers.SNAPSHOT_PAIRS = "always"
        timesteppers.SNAPSHOT_LAYOUT = timesteppers.BATCH_LAYOUT = layout
    elif layout == "plain":
        timesteppers.SNAPSHOT_PAIRS = "never"


def main() -> None:
    a = parse()
    set_layout(a.layout)
    if a.no_bundles:
        from offline_particles_b200 import timesteppers

        timesteppers.BUNDLE_2D = False
    if a.study == "precision":
        precision_study(a)
    elif a.study == "batched":
        batched_study(a)
    elif a.study == "serving":
        serving_study(a)
    elif a.study == "launch":
        launch_study(a)
    elif a.impl == "reference":
        reference_arm(a)
    else:
        b200_arm(a)


if __name__ == "__main__":
    main()
