"""ROMS history files (NetCDF classic) as a field source: reading, land masking, file concatenation."""

from __future__ import annotations

import numpy as np
import pytest

from offline_particles_b200.roms_history import RomsHistory, write_history
from offline_particles_b200.synth import GridSpec, SyntheticROMS


def _masks(mask_rho):
    m = mask_rho > 0
    return {"u": ~(m[:, :-1] & m[:, 1:]), "v": ~(m[:-1, :] & m[1:, :]), "w": ~m, "zeta": ~m}


@pytest.fixture(scope="module")
def history(tmp_path_factory):
    g = SyntheticROMS(GridSpec(nx=40, ny=32, nz=6, nt=5, seed=51, dtype="float32"))
    f = g.oracle_fields()
    d = tmp_path_factory.mktemp("his")
    # two files, split along time; ROMS' fill value on land faces
    write_history(d / "his_0001.nc", {**f, **{n: f[n][:3] for n in ("u", "v", "w", "zeta")}}, g.time_array[:3],
                  hc=g.hc, mask_rho=g.mask_rho, fill_land=1e37)
    write_history(d / "his_0002.nc", {**f, **{n: f[n][3:] for n in ("u", "v", "w", "zeta")}}, g.time_array[3:],
                  hc=g.hc, mask_rho=g.mask_rho, fill_land=1e37)
    h = RomsHistory([d / "his_0001.nc", d / "his_0002.nc"])
    yield g, f, h
    h.close()


def test_reads_snapshots_across_files_with_land_zeroed(history):
    g, f, h = history
    assert h.num_snapshots == 5 and np.array_equal(h.time_array, g.time_array)
    assert (h.nz, h.ny, h.nx, h.hc) == (6, 32, 40, g.hc)
    land = _masks(g.mask_rho)
    for name in ("u", "v", "w", "zeta"):
        var = h.variable(name)
        assert var.shape == f[name].shape and var.dtype == np.float32
        for k in range(5):
            expect = f[name][k].copy()
            expect[..., land[name]] = 0
            got = var[k]
            assert got.dtype == np.float32 and np.array_equal(got, expect), (name, k)
            assert np.all(got[..., land[name]] == 0)  # the fill value never reaches the device


def test_statics(history):
    g, f, h = history
    s = h.statics()
    assert np.array_equal(s["h"], f["h"]) and np.array_equal(s["C"], f["C"])
    assert np.allclose(s["dx"], f["dx"], rtol=1e-15) and np.allclose(s["dy"], f["dy"], rtol=1e-15)


def test_rejects_missing_variables(tmp_path):
    from scipy.io import netcdf_file

    with netcdf_file(str(tmp_path / "bad.nc"), "w", version=2) as f:
        f.createDimension("ocean_time", 2)
        v = f.createVariable("ocean_time", "d", ("ocean_time",))
        v[:] = [0.0, 1.0]
    with pytest.raises(KeyError, match="lacks ROMS variables"):
        RomsHistory(tmp_path / "bad.nc")
