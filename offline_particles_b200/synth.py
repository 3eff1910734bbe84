"""Seeded synthetic ROMS-like grids and particle releases.

No ROMS output is available offline, so every workload here runs on a
synthetic grid with the construction below (the same one for every size):

* rho grid ``nx x ny``, ``dx = dy = 2 km`` (constant static fields);
* bathymetry ``h = 50 + 950 G`` with ``G`` a Gaussian-filtered random field
  (sigma ~ 8 cells) normalised to [0, 1], clipped to [50, 1000] m;
* land: one contiguous blob of ~10 % of the cells (a disc around a seeded
  point, its edge perturbed by a smooth field); velocities are zero on masked
  faces, as ROMS writes them;
* ``zeta = 0.5 sin(2 pi t / 12.42 h)``, uniform in space;
* ``C = Cs_r`` from the published ROMS ``Vstretching = 4`` formula with
  ``theta_s = 5``, ``theta_b = 0.4``, ``hc = 20 m`` (``Vtransform = 2`` is what
  the reference's vertical coordinate implements);
* ``u, v`` from a streamfunction of 16 seeded Fourier modes plus a weak
  potential-flow part, with a decaying vertical profile, scaled to 0.5 m/s rms
  and modulated in time;
* ``w`` from continuity on the sigma layers, zero at the bottom (~1e-4 m/s).

Snapshots are produced lazily and deterministically from (seed, snapshot
index), so an object of this module can stand in for a ``(t, z, y, x)`` array:
it exposes ``shape``, ``ndim``, ``dtype`` and ``__getitem__(it)``.
"""

from __future__ import annotations

import dataclasses
import functools

import numpy as np

HOUR = 3600.0
M2_PERIOD = 12.42 * HOUR


def vstretching4(nz: int, theta_s: float = 5.0, theta_b: float = 0.4, *, w_levels: bool = False) -> np.ndarray:
    """ROMS Vstretching = 4 stretching function at rho (or w) levels."""
    if w_levels:
        sc = (np.arange(nz + 1, dtype=np.float64) - nz) / nz
    else:
        sc = (np.arange(nz, dtype=np.float64) + 0.5) / nz - 1.0
    if theta_s > 0:
        csur = (1.0 - np.cosh(theta_s * sc)) / (np.cosh(theta_s) - 1.0)
    else:
        csur = -(sc**2)
    if theta_b > 0:
        return (np.exp(theta_b * csur) - 1.0) / (1.0 - np.exp(-theta_b))
    return csur


def _smooth_field(rng: np.random.Generator, ny: int, nx: int, sigma: float) -> np.ndarray:
    """Gaussian-filtered white noise (periodic FFT filter), normalised to [0, 1]."""
    noise = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    filt = np.exp(-2.0 * (np.pi * sigma) ** 2 * (kx**2 + ky**2))
    g = np.fft.irfft2(np.fft.rfft2(noise) * filt, s=(ny, nx))
    g -= g.min()
    g /= max(g.max(), 1e-300)
    return g


@dataclasses.dataclass(frozen=True)
class GridSpec:
    nx: int
    ny: int
    nz: int
    nt: int
    seed: int
    dtype: str = "float64"
    dx: float = 2000.0
    hc: float = 20.0
    theta_s: float = 5.0
    theta_b: float = 0.4
    land_fraction: float = 0.10
    snapshot_interval: float = HOUR


class _LazyField:
    """(t, ...) array-like over the snapshots of one time-dependent field."""

    def __init__(self, grid: "SyntheticROMS", name: str, spatial_shape: tuple[int, ...]) -> None:
        self._grid = grid
        self._name = name
        self.shape = (grid.spec.nt,) + spatial_shape
        self.ndim = len(self.shape)
        self.dtype = grid.dtype

    def __len__(self) -> int:
        return self.shape[0]

    def __getitem__(self, key):
        if isinstance(key, tuple):
            it, rest = key[0], key[1:]
        else:
            it, rest = key, ()
        if isinstance(it, (int, np.integer)):
            snap = self._grid.snapshot(int(it))[self._name]
            return snap[rest] if rest and rest != (Ellipsis,) else snap
        if isinstance(it, slice):
            idx = range(*it.indices(self.shape[0]))
            out = np.stack([self._grid.snapshot(i)[self._name] for i in idx])
            return out[(slice(None),) + rest] if rest and rest != (Ellipsis,) else out
        raise TypeError(f"unsupported index {key!r}")

    def __array__(self, dtype=None, copy=None):
        out = self[0 : self.shape[0]]
        return out.astype(dtype) if dtype is not None else out


class SyntheticROMS:
    """A seeded synthetic ROMS grid; see the module docstring."""

    def __init__(self, spec: GridSpec) -> None:
        self.spec = spec
        self.dtype = np.dtype(spec.dtype)
        nx, ny, nz = spec.nx, spec.ny, spec.nz
        rng = np.random.default_rng(spec.seed)
        self.time_array = np.arange(spec.nt, dtype=np.float64) * spec.snapshot_interval

        # bathymetry
        g = _smooth_field(rng, ny, nx, sigma=8.0)
        self.h64 = np.clip(50.0 + 950.0 * g, 50.0, 1000.0)

        # land: perturbed disc around a seeded point covering ~land_fraction
        cy, cx = rng.uniform(0.2, 0.8) * ny, rng.uniform(0.2, 0.8) * nx
        yy, xx = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
        d = np.hypot(yy - cy, xx - cx)
        r0 = np.sqrt(spec.land_fraction * nx * ny / np.pi)
        d = d + 0.35 * r0 * (_smooth_field(rng, ny, nx, sigma=12.0) - 0.5)
        thresh = np.quantile(d, spec.land_fraction)
        self.mask_rho = (d > thresh).astype(np.float64)  # 1 = wet

        # vertical
        self.C64 = vstretching4(nz, spec.theta_s, spec.theta_b)
        self.Cw64 = vstretching4(nz, spec.theta_s, spec.theta_b, w_levels=True)
        self.sigma_w = (np.arange(nz + 1, dtype=np.float64) - nz) / nz

        # flow modes: 16 streamfunction modes + 4 weak potential modes
        nm = 16
        L = rng.uniform(25.0, 150.0, nm)  # wavelength in cells
        ang = rng.uniform(0, 2 * np.pi, nm)
        self._k = 2 * np.pi / L * np.cos(ang)
        self._l = 2 * np.pi / L * np.sin(ang)
        self._phi = rng.uniform(0, 2 * np.pi, nm)
        self._omega = 2 * np.pi / (rng.uniform(1.0, 6.0, nm) * 86400.0) * rng.choice([-1.0, 1.0], nm)
        self._amp = rng.uniform(0.5, 1.0, nm) / np.sqrt(nm)
        npm = 4
        Lp = rng.uniform(40.0, 120.0, npm)
        angp = rng.uniform(0, 2 * np.pi, npm)
        self._kp = 2 * np.pi / Lp * np.cos(angp)
        self._lp = 2 * np.pi / Lp * np.sin(angp)
        self._phip = rng.uniform(0, 2 * np.pi, npm)
        self._ampp = rng.uniform(0.5, 1.0, npm) / np.sqrt(npm) * 0.02
        self._prof = 0.4 + 0.6 * np.exp((np.arange(nz) + 0.5 - nz) / (0.4 * nz))  # surface-intensified
        self._scale = None
        self._cache: dict[int, dict[str, np.ndarray]] = {}
        self._cache_order: list[int] = []
        self.max_cached = 3

    # ---------------------------------------------------------------- static
    @functools.cached_property
    def h(self) -> np.ndarray:
        return self.h64.astype(self.dtype)

    @functools.cached_property
    def dx(self) -> np.ndarray:
        return np.full((self.spec.ny, self.spec.nx), self.spec.dx, dtype=self.dtype)

    @functools.cached_property
    def dy(self) -> np.ndarray:
        return np.full((self.spec.ny, self.spec.nx), self.spec.dx, dtype=self.dtype)

    @property
    def C(self) -> np.ndarray:
        return self.C64.copy()

    @property
    def hc(self) -> float:
        return self.spec.hc

    # ------------------------------------------------------------- dynamics
    def zeta_value(self, t: float) -> float:
        return 0.5 * np.sin(2 * np.pi * t / M2_PERIOD)

    @functools.cached_property
    def _taper(self) -> tuple[np.ndarray, np.ndarray]:
        """Smooth [0, 1] coastal taper at rho points and at cell corners (0 on land)."""
        ny, nx = self.spec.ny, self.spec.nx
        m = self.mask_rho
        ky = np.fft.fftfreq(ny)[:, None]
        kx = np.fft.rfftfreq(nx)[None, :]
        filt = np.exp(-2.0 * (np.pi * 4.0) ** 2 * (kx**2 + ky**2))
        blur = np.fft.irfft2(np.fft.rfft2(m) * filt, s=(ny, nx))
        rho = np.clip((blur - 0.5) * 2.0, 0.0, 1.0) ** 2 * m
        pad = np.pad(rho, 1, mode="edge")
        corner = 0.25 * (pad[:-1, :-1] + pad[1:, :-1] + pad[:-1, 1:] + pad[1:, 1:])  # (ny+1, nx+1)
        corner = np.minimum(corner, np.minimum.reduce([pad[:-1, :-1], pad[1:, :-1], pad[:-1, 1:], pad[1:, 1:]]) + 0.0)
        return rho, corner

    def _uv_full(self, t: float) -> tuple[np.ndarray, np.ndarray]:
        """Depth-independent velocity on ALL faces (unscaled): u (ny, nx+1), v (ny+1, nx).

        Face u[:, i] sits at x = i - 0.5 and v[j, :] at y = j - 0.5.  The
        rotational part is the discrete curl of a corner streamfunction tapered
        to zero at the coast, so it is exactly divergence-free on the C grid;
        the weak potential part carries all of the divergence.
        """
        nx, ny = self.spec.nx, self.spec.ny
        yc = np.arange(ny + 1, dtype=np.float64)[:, None] - 0.5
        xc = np.arange(nx + 1, dtype=np.float64)[None, :] - 0.5
        psi = np.zeros((ny + 1, nx + 1))
        for m in range(self._k.size):
            ph = self._phi[m] + self._omega[m] * t
            psi += self._amp[m] * np.cos(self._k[m] * xc + self._l[m] * yc + ph)
        rho_t, corner_t = self._taper
        psi *= corner_t
        u = -(psi[1:, :] - psi[:-1, :])  # (ny, nx+1)
        v = psi[:, 1:] - psi[:, :-1]  # (ny+1, nx)
        # potential part, tapered on faces
        yu = np.arange(ny, dtype=np.float64)[:, None]
        xu = np.arange(nx + 1, dtype=np.float64)[None, :] - 0.5
        yv = np.arange(ny + 1, dtype=np.float64)[:, None] - 0.5
        xv = np.arange(nx, dtype=np.float64)[None, :]
        pad = np.pad(rho_t, ((0, 0), (1, 1)), mode="edge")
        tu = np.minimum(pad[:, :-1], pad[:, 1:])
        pad = np.pad(rho_t, ((1, 1), (0, 0)), mode="edge")
        tv = np.minimum(pad[:-1, :], pad[1:, :])
        for m in range(self._kp.size):
            a = self._ampp[m]
            u += -a * self._kp[m] * np.sin(self._kp[m] * xu + self._lp[m] * yu + self._phip[m]) * tu
            v += -a * self._lp[m] * np.sin(self._kp[m] * xv + self._lp[m] * yv + self._phip[m]) * tv
        mod = 1.0 + 0.2 * np.sin(2 * np.pi * t / 86400.0)
        return u * mod, v * mod

    def _velocity_scale(self) -> float:
        if self._scale is None:
            u, v = self._uv_full(0.0)
            wet = self.mask_rho > 0
            um = u[:, 1:-1][wet[:, :-1] & wet[:, 1:]]
            vm = v[1:-1, :][wet[:-1, :] & wet[1:, :]]
            rms = np.sqrt(0.5 * (np.mean(um**2) + np.mean(vm**2)))
            self._scale = 0.5 / max(rms, 1e-300)
        return self._scale

    def snapshot(self, it: int) -> dict[str, np.ndarray]:
        """u, v, w, zeta of snapshot ``it`` in the storage dtype."""
        if it < 0 or it >= self.spec.nt:
            raise IndexError(it)
        if it in self._cache:
            return self._cache[it]
        t = float(self.time_array[it])
        s = self._velocity_scale()
        uf, vf = self._uv_full(t)
        uf *= s
        vf *= s
        prof = self._prof
        u = (prof[:, None, None] * uf[None, :, 1:-1]).astype(self.dtype)
        v = (prof[:, None, None] * vf[None, 1:-1, :]).astype(self.dtype)

        # continuity: w(k+1) = w(k) - div(k) Hz(k), w(0) = 0 (bottom)
        ny, nx = self.spec.ny, self.spec.nx
        div = ((uf[:, 1:] - uf[:, :-1]) + (vf[1:, :] - vf[:-1, :])) / self.spec.dx
        zeta = self.zeta_value(t)
        hc, h = self.spec.hc, self.h64
        Sw = (hc * self.sigma_w[:, None, None] + h[None] * self.Cw64[:, None, None]) / (hc + h)[None]
        Hz = (zeta + h)[None] * np.diff(Sw, axis=0)  # (nz, ny, nx)
        cum = np.concatenate([np.zeros((1, ny, nx)), np.cumsum(prof[:, None, None] * Hz, axis=0)], axis=0)
        w = (-div[None] * cum * self.mask_rho[None]).astype(self.dtype)
        zeta_arr = np.full((ny, nx), zeta, dtype=self.dtype)
        snap = {"u": u, "v": v, "w": w, "zeta": zeta_arr}
        self._cache[it] = snap
        self._cache_order.append(it)
        while len(self._cache_order) > self.max_cached:
            self._cache.pop(self._cache_order.pop(0), None)
        return snap

    # ------------------------------------------------------- device generation
    def _device_consts(self, dev) -> dict:
        """Time-independent tensors of the device construction (float64 on ``dev``)."""
        import torch

        nx, ny = self.spec.nx, self.spec.ny
        f64 = dict(dtype=torch.float64, device=dev)
        rho_t, corner_t = self._taper
        pad = np.pad(rho_t, ((0, 0), (1, 1)), mode="edge")
        tu = torch.tensor(np.minimum(pad[:, :-1], pad[:, 1:]), **f64)
        pad = np.pad(rho_t, ((1, 1), (0, 0)), mode="edge")
        tv = torch.tensor(np.minimum(pad[:-1, :], pad[1:, :]), **f64)
        h = torch.tensor(self.h64, **f64)
        hc = self.spec.hc
        Sw = (hc * torch.tensor(self.sigma_w, **f64)[:, None, None]
              + h[None] * torch.tensor(self.Cw64, **f64)[:, None, None]) / (hc + h)[None]
        return {
            "corner": torch.tensor(corner_t, **f64), "tu": tu, "tv": tv, "h": h,
            "mask": torch.tensor(self.mask_rho, **f64), "prof": torch.tensor(self._prof, **f64),
            "dSw": Sw[1:] - Sw[:-1],
            "yc": torch.arange(ny + 1, **f64)[:, None] - 0.5, "xc": torch.arange(nx + 1, **f64)[None, :] - 0.5,
            "yu": torch.arange(ny, **f64)[:, None], "xu": torch.arange(nx + 1, **f64)[None, :] - 0.5,
            "yv": torch.arange(ny + 1, **f64)[:, None] - 0.5, "xv": torch.arange(nx, **f64)[None, :],
            "scale": self._velocity_scale(),
        }

    def _snapshot_time(self, it: int) -> float:
        return float(self.time_array[it]) if it < len(self.time_array) else it * self.spec.snapshot_interval

    def _device_snapshot(self, it: int, c: dict, td, out: dict | None = None) -> dict:
        """Snapshot ``it`` of u, v, w, zeta computed on the device in float64, stored in ``td``."""
        import torch

        nx, ny, nz = self.spec.nx, self.spec.ny, self.spec.nz
        dev = c["h"].device
        f64 = dict(dtype=torch.float64, device=dev)
        if out is None:
            out = {"u": torch.empty((nz, ny, nx - 1), dtype=td, device=dev),
                   "v": torch.empty((nz, ny - 1, nx), dtype=td, device=dev),
                   "w": torch.empty((nz + 1, ny, nx), dtype=td, device=dev),
                   "zeta": torch.empty((ny, nx), dtype=td, device=dev)}
        t = self._snapshot_time(it)
        psi = torch.zeros((ny + 1, nx + 1), **f64)
        for m in range(self._k.size):
            ph = self._phi[m] + self._omega[m] * t
            psi += self._amp[m] * torch.cos(self._k[m] * c["xc"] + self._l[m] * c["yc"] + ph)
        psi *= c["corner"]
        uf = -(psi[1:, :] - psi[:-1, :])
        vf = psi[:, 1:] - psi[:, :-1]
        for m in range(self._kp.size):
            a = self._ampp[m]
            uf += -a * self._kp[m] * torch.sin(self._kp[m] * c["xu"] + self._lp[m] * c["yu"] + self._phip[m]) * c["tu"]
            vf += -a * self._lp[m] * torch.sin(self._kp[m] * c["xv"] + self._lp[m] * c["yv"] + self._phip[m]) * c["tv"]
        mod = (1.0 + 0.2 * np.sin(2 * np.pi * t / 86400.0)) * c["scale"]
        uf *= mod
        vf *= mod
        prof = c["prof"]
        out["u"].copy_(prof[:, None, None] * uf[None, :, 1:-1])
        out["v"].copy_(prof[:, None, None] * vf[None, 1:-1, :])
        div = ((uf[:, 1:] - uf[:, :-1]) + (vf[1:, :] - vf[:-1, :])) / self.spec.dx
        zeta = self.zeta_value(t)
        Hz = (zeta + c["h"])[None] * c["dSw"]
        cum = torch.cat([torch.zeros((1, ny, nx), **f64), torch.cumsum(prof[:, None, None] * Hz, dim=0)])
        out["w"].copy_(-div[None] * cum * c["mask"][None])
        out["zeta"].fill_(zeta)
        return out

    def device_snapshots(self, nt: int, device=None, dtype=None) -> dict:
        """Snapshots 0..nt-1 of u, v, w, zeta generated on a CUDA device.

        The same construction as ``snapshot`` evaluated with torch in float64 on
        the device (equal to the host arrays to rounding, not bit for bit), for
        workloads whose snapshots would take minutes to build on the host.
        Returns CUDA tensors of shape ``(nt, ...)`` in ``dtype`` (default: the
        grid's storage dtype).
        """
        import torch

        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        td = _torch_dtype(dtype if dtype is not None else self.dtype)
        nx, ny, nz = self.spec.nx, self.spec.ny, self.spec.nz
        out = {
            "u": torch.empty((nt, nz, ny, nx - 1), dtype=td, device=dev),
            "v": torch.empty((nt, nz, ny - 1, nx), dtype=td, device=dev),
            "w": torch.empty((nt, nz + 1, ny, nx), dtype=td, device=dev),
            "zeta": torch.empty((nt, ny, nx), dtype=td, device=dev),
        }
        c = self._device_consts(dev)
        for it in range(nt):
            self._device_snapshot(it, c, td, {k: v[it] for k, v in out.items()})
        return out

    def pinned_cycle(self, distinct: int, nt: int, device=None) -> dict:
        """u, v, w, zeta as ``CyclicSnapshots`` of ``nt`` snapshots repeating the first ``distinct`` ones,
        generated on the device and held in pinned host memory."""
        import torch

        snaps = self.device_snapshots(distinct, device)
        out = {}
        for name, t in snaps.items():
            host = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
            host.copy_(t)
            out[name] = CyclicSnapshots(host, nt)
        return out

    def device_source(self, nt: int, device=None, dtype=None, cache: int = 6) -> "DeviceSnapshotSource":
        """Snapshots 0..nt-1 generated on the device when a field's ring asks for them (no storage for
        the whole series: serving runs whose model time has no fixed end)."""
        return DeviceSnapshotSource(self, nt, device, dtype, cache)

    # ------------------------------------------------------------ accessors
    def field(self, name: str) -> _LazyField:
        nz, ny, nx = self.spec.nz, self.spec.ny, self.spec.nx
        shapes = {"u": (nz, ny, nx - 1), "v": (nz, ny - 1, nx), "w": (nz + 1, ny, nx), "zeta": (ny, nx)}
        return _LazyField(self, name, shapes[name])

    def dense(self, name: str) -> np.ndarray:
        """All snapshots of a time-dependent field as one array (small grids only)."""
        return np.asarray(self.field(name))

    def release(self, n: int, seed: int | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """``n`` particles uniform in wet cells, at uniform random sigma levels.

        Returns (zidx, yidx, xidx) float64 arrays in centred index space.
        """
        rng = np.random.default_rng(self.spec.seed * 7919 + 17 if seed is None else seed)
        wet = np.flatnonzero(self.mask_rho.ravel() > 0)
        cells = wet[rng.integers(0, wet.size, n)]
        j, i = np.divmod(cells, self.spec.nx)
        y = np.clip(j + rng.uniform(-0.5, 0.5, n), 0.0, self.spec.ny - 1.0)
        x = np.clip(i + rng.uniform(-0.5, 0.5, n), 0.0, self.spec.nx - 1.0)
        z = rng.uniform(0.0, self.spec.nz - 1.0, n)
        return z, y, x

    def density(self, nt: int | None = None) -> np.ndarray:
        """A seeded density field at rho points, ``(nt, nz, ny, nx)`` in the grid's dtype (kg/m^3): a
        stable stratification (denser at depth) with a slowly moving horizontal wave, for the isopycnal
        follower.  Deterministic in the grid's spec."""
        nt = self.spec.nt if nt is None else nt
        nz, ny, nx = self.spec.nz, self.spec.ny, self.spec.nx
        k = np.arange(nz, dtype=np.float64)[:, None, None]
        j = np.arange(ny, dtype=np.float64)[None, :, None]
        i = np.arange(nx, dtype=np.float64)[None, None, :]
        out = np.empty((nt, nz, ny, nx), dtype=self.dtype)
        for it in range(nt):
            t = self._snapshot_time(it) / 86400.0
            out[it] = (1026.5 - 1.5 * k / max(nz - 1, 1)
                       + 0.3 * np.sin(2 * np.pi * j / ny + 0.7 * t) * np.cos(2 * np.pi * i / nx - 0.3 * t))
        return out

    def release_in_box(self, n: int, rng: np.random.Generator, min_frac: float = 0.05,
                       max_frac: float = 0.5) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """``n`` particles uniform in the wet cells of a random rectangle (sides ``min_frac`` to
        ``max_frac`` of the grid's) at uniform random levels of a random sigma band."""
        ny, nx, nz = self.spec.ny, self.spec.nx, self.spec.nz
        while True:
            hy = max(1, int(ny * rng.uniform(min_frac, max_frac)))
            hx = max(1, int(nx * rng.uniform(min_frac, max_frac)))
            y0 = int(rng.integers(0, ny - hy + 1))
            x0 = int(rng.integers(0, nx - hx + 1))
            box = self.mask_rho[y0:y0 + hy, x0:x0 + hx] > 0
            wet = np.flatnonzero(box.ravel())
            if wet.size:
                break
        cells = wet[rng.integers(0, wet.size, n)]
        j, i = np.divmod(cells, hx)
        y = np.clip(y0 + j + rng.uniform(-0.5, 0.5, n), 0.0, ny - 1.0)
        x = np.clip(x0 + i + rng.uniform(-0.5, 0.5, n), 0.0, nx - 1.0)
        za, zb = np.sort(rng.uniform(0.0, nz - 1.0, 2))
        z = rng.uniform(za, zb, n)
        return z, y, x

    def oracle_fields(self) -> dict[str, np.ndarray]:
        """Dense field dict (u, v, w, zeta with a time axis; h, dx, dy, C)."""
        out = {name: self.dense(name) for name in ("u", "v", "w", "zeta")}
        out.update(h=self.h, dx=self.dx, dy=self.dy, C=self.C)
        return out


class CyclicSnapshots:
    """An array-like ``(nt, ...)`` for ``TimeDependentField`` whose snapshot k is ``base[k % len(base)]``:
    a long series (a week of hourly snapshots) from a few distinct snapshots held in pinned host memory,
    which the field's ring uploads with one asynchronous copy each (no staging), as it would uploads from
    a reader that fills pinned buffers."""

    def __init__(self, base, nt: int) -> None:
        import torch

        if not isinstance(base, torch.Tensor) or base.ndim < 2 or base.shape[0] < 1:
            raise ValueError("base must be a tensor of at least one snapshot")
        self.base = base
        self.shape = (int(nt),) + tuple(base.shape[1:])
        self.ndim = len(self.shape)
        self.dtype = np.dtype(str(base.dtype).replace("torch.", ""))

    def __len__(self) -> int:
        return self.shape[0]

    def __getitem__(self, k):
        k = int(k)
        if not 0 <= k < self.shape[0]:
            raise IndexError(k)
        return self.base[k % self.base.shape[0]]


def _torch_dtype(dtype):
    import torch

    return {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}[np.dtype(dtype)]


class _GeneratedField:
    """One field of a DeviceSnapshotSource: an array-like ``(nt, ...)`` whose snapshots are produced on
    the device into a caller's tensor (``produce``), for a TimeDependentField ring."""

    def __init__(self, source: "DeviceSnapshotSource", name: str, spatial_shape: tuple[int, ...]) -> None:
        self._source = source
        self.name = name
        self.shape = (source.nt,) + tuple(spatial_shape)
        self.ndim = len(self.shape)
        self.dtype = source.np_dtype

    def __len__(self) -> int:
        return self.shape[0]

    def produce(self, k: int, out) -> None:
        self._source.produce(k, self.name, out)


class DeviceSnapshotSource:
    """Synthetic snapshots generated on a CUDA device on demand.

    ``field(name)`` gives the array-like for ``TimeDependentField``; when a
    field's ring asks for snapshot k, all four fields of k are generated once
    (on the asking stream) and kept in a small cache, so the other fields'
    rings copy them instead of generating again.  Generation is deterministic:
    snapshot k has the same bits every time it is produced.
    """

    def __init__(self, grid: "SyntheticROMS", nt: int, device=None, dtype=None, cache: int = 6) -> None:
        import threading

        import torch

        self.grid = grid
        self.nt = int(nt)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.np_dtype = np.dtype(dtype if dtype is not None else grid.dtype)
        self.td = _torch_dtype(self.np_dtype)
        self.cache_size = max(2, int(cache))
        self._consts = None
        self._cache: dict[int, tuple[dict, object]] = {}
        self._lock = threading.Lock()
        self.generated = 0

    def field(self, name: str) -> _GeneratedField:
        nz, ny, nx = self.grid.spec.nz, self.grid.spec.ny, self.grid.spec.nx
        shapes = {"u": (nz, ny, nx - 1), "v": (nz, ny - 1, nx), "w": (nz + 1, ny, nx), "zeta": (ny, nx)}
        return _GeneratedField(self, name, shapes[name])

    def produce(self, k: int, name: str, out) -> None:
        """Write field ``name`` of snapshot ``k`` into the device tensor ``out`` on the current stream."""
        import torch

        if not 0 <= k < self.nt:
            raise IndexError(k)
        stream = torch.cuda.current_stream(self.device)
        with self._lock:
            entry = self._cache.pop(k, None)
            if entry is None:
                if self._consts is None:
                    self._consts = self.grid._device_consts(self.device)
                fields = self.grid._device_snapshot(k, self._consts, self.td)
                ev = torch.cuda.Event()
                ev.record(stream)
                entry = (fields, ev)
                self.generated += 1
            self._cache[k] = entry  # most recently used last
            while len(self._cache) > self.cache_size:
                self._cache.pop(next(iter(self._cache)))
        fields, ev = entry
        stream.wait_event(ev)
        out.copy_(fields[name])
        fields[name].record_stream(stream)


# The workloads: grid, snapshots, particles, scheme, dt (seconds).
CONFIGS = {
    "config1": dict(grid=GridSpec(nx=128, ny=96, nz=20, nt=26, seed=1, dtype="float64"),
                    particles=10_000, scheme="rk2", dt=300.0, steps=288),
    "config2": dict(grid=GridSpec(nx=1024, ny=768, nz=50, nt=170, seed=2, dtype="float32"),
                    particles=4_194_304, scheme="ab3", dt=120.0, steps=5040),
}


def make_grid(name: str, **overrides) -> SyntheticROMS:
    spec = CONFIGS[name]["grid"]
    if overrides:
        spec = dataclasses.replace(spec, **overrides)
    return SyntheticROMS(spec)
