"""ROMS history files as a field source.

The reference takes its fields as in-memory or dask arrays (fields.py:237-392,
spatial_arrays.py:228-351); reading ROMS output is left to its users.  Here a
``RomsHistory`` reads ROMS history or average files in NetCDF classic format
(one file or several, concatenated along ``ocean_time``) and hands each
time-dependent variable to a ``TimeDependentField`` as a lazy array: the
field's snapshot ring asks for one snapshot at a time, on its staging thread,
which reads it from the memory-mapped file into pinned host memory and copies
it to its device slot while the kernels run.  Nothing is read twice or held in
host memory beyond the two staging buffers.

Land: ROMS writes a fill value (or garbage) under the land mask of masked
variables.  With ``mask_land`` (default) every snapshot is staged with zeros on
land faces of u (mask_rho of both neighbouring cells), v, w and zeta, the
convention of the synthetic grids and of ROMS itself for velocities.

Static fields: ``h``, ``dx = 1 / pm``, ``dy = 1 / pn`` (float64) and
``C = Cs_r``; constants ``hc`` and ``NZ = len(s_rho)``.
"""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np

# (dimension names, stagger) of the ROMS variables on the Arakawa-C grid
ROMS_VARIABLES = {
    "u": (("s_rho", "eta_u", "xi_u"), ("center", "center", "inner")),
    "v": (("s_rho", "eta_v", "xi_v"), ("center", "inner", "center")),
    "w": (("s_w", "eta_rho", "xi_rho"), ("outer", "center", "center")),
    "zeta": (("eta_rho", "xi_rho"), ("invariant", "center", "center")),
}
STATIC_STAGGERS = {
    "h": ("invariant", "center", "center"),
    "dx": ("invariant", "center", "center"),
    "dy": ("invariant", "center", "center"),
    "C": ("center", "invariant", "invariant"),
}


def _open(path: Path):
    from scipy.io import netcdf_file

    return netcdf_file(str(path), "r", mmap=True, maskandscale=False)


class _HistoryVariable:
    """One time-dependent variable across the files: ``shape`` (nt, ...), ``dtype``, ``[k]`` -> snapshot."""

    def __init__(self, history: "RomsHistory", name: str) -> None:
        self._h = history
        self.name = name
        first = history._files[0].variables[name]
        self.shape = (history.num_snapshots,) + tuple(first.shape[1:])
        self.ndim = len(self.shape)
        self.dtype = np.dtype(first.data.dtype).newbyteorder("=")

    def __len__(self) -> int:
        return self.shape[0]

    def __getitem__(self, k):
        if not isinstance(k, (int, np.integer)):
            raise TypeError("read one snapshot at a time")
        f, j = self._h._locate(int(k))
        out = np.array(self._h._files[f].variables[self.name].data[j], dtype=self.dtype)  # native byte order
        mask = self._h.land_masks.get(self.name)
        if mask is not None:
            out[..., mask] = 0
        return out

    def __array__(self, dtype=None, copy=None):
        a = np.stack([self[k] for k in range(len(self))])
        return a if dtype is None else a.astype(dtype)


class RomsHistory:
    """ROMS history/average files (NetCDF classic) as a field source."""

    def __init__(self, paths, *, time_name: str = "ocean_time", mask_land: bool = True) -> None:
        if isinstance(paths, (str, os.PathLike)):
            paths = [paths]
        self.paths = [Path(p) for p in paths]
        if not self.paths:
            raise ValueError("no files")
        self._files = [_open(p) for p in self.paths]
        missing = [v for v in ("u", "v", "w", "zeta", "h", "pm", "pn", "Cs_r", "hc", time_name)
                   if v not in self._files[0].variables]
        if missing:
            raise KeyError(f"{self.paths[0]} lacks ROMS variables {missing}")
        for name, (dims, _) in ROMS_VARIABLES.items():
            got = self._files[0].variables[name].dimensions
            if tuple(got[1:]) != dims:
                raise ValueError(f"variable {name} has dimensions {got}, expected (time,) + {dims}")
        self._counts = []
        times = []
        for f in self._files:
            t = np.array(f.variables[time_name].data, dtype=np.float64)
            self._counts.append(len(t))
            times.append(t)
        self.time_array = np.concatenate(times)
        if np.any(np.diff(self.time_array) <= 0):
            raise ValueError("ocean_time must increase strictly across the files")
        self._offsets = np.concatenate([[0], np.cumsum(self._counts)])
        v0 = self._files[0].variables
        self.nz = v0["Cs_r"].shape[0]
        self.ny, self.nx = v0["h"].shape
        self.hc = float(np.asarray(v0["hc"].data))
        self.land_masks: dict[str, np.ndarray] = {}
        if mask_land and "mask_rho" in v0:
            m = np.array(v0["mask_rho"].data, dtype=np.float64) > 0
            land_u = ~(m[:, :-1] & m[:, 1:])
            land_v = ~(m[:-1, :] & m[1:, :])
            self.land_masks = {"u": land_u, "v": land_v, "w": ~m, "zeta": ~m}

    @property
    def num_snapshots(self) -> int:
        return int(self._offsets[-1])

    def _locate(self, k: int) -> tuple[int, int]:
        if not 0 <= k < self.num_snapshots:
            raise IndexError(k)
        f = int(np.searchsorted(self._offsets, k, side="right")) - 1
        return f, k - int(self._offsets[f])

    def variable(self, name: str) -> _HistoryVariable:
        if name not in ROMS_VARIABLES:
            raise KeyError(name)
        return _HistoryVariable(self, name)

    def statics(self) -> dict[str, np.ndarray]:
        """h, dx = 1/pm, dy = 1/pn (float64) and C = Cs_r."""
        v = self._files[0].variables
        pm = np.array(v["pm"].data, dtype=np.float64)
        pn = np.array(v["pn"].data, dtype=np.float64)
        return {"h": np.array(v["h"].data, dtype=np.float64), "dx": 1.0 / pm, "dy": 1.0 / pn,
                "C": np.array(v["Cs_r"].data, dtype=np.float64)}

    def fieldset(self, *, ring_size: int = 4, storage: str | None = None, device=None, **constants):
        """A Fieldset over the files: u, v, w, zeta streamed snapshot by snapshot through device rings,
        the statics resident; constants hc, NZ and any ``constants`` given."""
        from .fields import StaticField, TimeDependentField
        from .fieldset import Fieldset

        kw = {}
        for name, (_, stagger) in ROMS_VARIABLES.items():
            kw[name] = TimeDependentField(self.variable(name), *stagger, ring_size=ring_size, storage=storage,
                                          device=device)
        for name, arr in self.statics().items():
            kw[name] = StaticField.from_numpy(arr, *STATIC_STAGGERS[name])
        return Fieldset(self.num_snapshots, self.nz, self.ny, self.nx,
                        constants={"hc": self.hc, "NZ": self.nz, **constants}, **kw)

    def close(self) -> None:
        for f in self._files:
            f.close()
        self._files = []


def write_history(path, grid_fields: dict[str, np.ndarray], time_array: np.ndarray, *, hc: float,
                  mask_rho: np.ndarray | None = None, fill_land: float | None = None) -> None:
    """Write fields in ROMS history layout (NetCDF classic): ``u, v, w, zeta`` with a time axis, ``h``,
    ``dx``/``dy`` (stored as pm = 1/dx, pn = 1/dy), ``C`` (as Cs_r), hc and mask_rho.  ``fill_land``: write
    this value on land faces of the time-dependent variables, as ROMS does for masked output."""
    from scipy.io import netcdf_file

    u, v, w, zeta = (grid_fields[n] for n in ("u", "v", "w", "zeta"))
    nt, nz, ny, nxu = u.shape
    nx = nxu + 1
    with netcdf_file(str(path), "w", version=2) as f:
        f.createDimension("ocean_time", nt)
        for d, n in (("s_rho", nz), ("s_w", nz + 1), ("eta_rho", ny), ("xi_rho", nx), ("eta_u", ny),
                     ("xi_u", nx - 1), ("eta_v", ny - 1), ("xi_v", nx)):
            f.createDimension(d, n)
        tv = f.createVariable("ocean_time", "d", ("ocean_time",))
        tv[:] = np.asarray(time_array, dtype=np.float64)
        hcv = f.createVariable("hc", "d", ())
        hcv.data[...] = hc
        land = {}
        if mask_rho is not None:
            mv = f.createVariable("mask_rho", "d", ("eta_rho", "xi_rho"))
            mv[:] = mask_rho
            m = mask_rho > 0
            land = {"u": ~(m[:, :-1] & m[:, 1:]), "v": ~(m[:-1, :] & m[1:, :]), "w": ~m, "zeta": ~m}
        for name, arr in (("u", u), ("v", v), ("w", w), ("zeta", zeta)):
            dims = ("ocean_time",) + ROMS_VARIABLES[name][0]
            var = f.createVariable(name, "f" if arr.dtype == np.float32 else "d", dims)
            data = np.array(arr)
            if fill_land is not None and name in land:
                data[..., land[name]] = fill_land
            var[:] = data
        for name, arr, dims in (("h", grid_fields["h"], ("eta_rho", "xi_rho")),
                                ("pm", 1.0 / np.asarray(grid_fields["dx"], dtype=np.float64), ("eta_rho", "xi_rho")),
                                ("pn", 1.0 / np.asarray(grid_fields["dy"], dtype=np.float64), ("eta_rho", "xi_rho")),
                                ("Cs_r", grid_fields["C"], ("s_rho",))):
            var = f.createVariable(name, "d", dims)
            var[:] = arr
