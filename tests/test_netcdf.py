"""The NetCDF classic writer of the reference's result files (SaveOutput1D/2D/3D,
src/io.cc:696-850, as used by SaveModelResults and SaveResultEntirePeriod,
src/io.cc:854-996), read back with an independent reader (scipy.io's
NetCDF-3 module).  Host code only: no GPU."""
import os

import numpy as np
import pytest

import dhara_b200 as db

netcdf = pytest.importorskip("scipy.io").netcdf_file


def test_snapshot_files_round_trip(tmp_path):
    nx, ny, nz = 7, 5, 3
    rng = np.random.default_rng(1)
    H, h = rng.standard_normal(nx * ny), rng.random(nx * ny)
    psi, th = rng.standard_normal(nx * ny * nz), rng.random(nx * ny * nz)
    f2, f3 = str(tmp_path / "olf_12.nc"), str(tmp_path / "ssf_12.nc")
    db.write_netcdf_state(f2, f3, nx, ny, nz, H, h, psi, th)
    with netcdf(f2, "r", mmap=False) as f:
        assert f.version_byte == 1
        assert f.dimensions == {"x": ny, "y": nx}
        assert f.variables["water_elevation"].dimensions == ("x", "y")
        assert np.array_equal(f.variables["water_elevation"][:], H.reshape(ny, nx))
        assert np.array_equal(f.variables["water_depth"][:], h.reshape(ny, nx))
    with netcdf(f3, "r", mmap=False) as f:
        assert f.dimensions == {"x": nx, "y": ny, "z": nz}
        assert f.variables["pressure_head"].dimensions == ("z", "y", "x")
        assert np.array_equal(f.variables["pressure_head"][:], psi.reshape(nz, ny, nx))
        assert np.array_equal(f.variables["moisture"][:], th.reshape(nz, ny, nx))


def test_statistics_files_round_trip(tmp_path):
    nsteps, nz = 9, 4
    rng = np.random.default_rng(2)
    mb, ps, th = rng.standard_normal(nsteps), rng.standard_normal((nsteps, nz)), rng.random((nsteps, nz))
    f1, fs = str(tmp_path / "ssf1d.nc"), str(tmp_path / "stat.nc")
    db.write_netcdf_statistics(f1, fs, nz, mb, ps, th)
    with netcdf(f1, "r", mmap=False) as f:
        assert f.dimensions == {"time_series": nsteps}
        assert np.array_equal(f.variables["mb_subsurfaceW"][:], mb)
    with netcdf(fs, "r", mmap=False) as f:
        assert f.dimensions == {"x": nsteps, "y": nz}
        assert np.array_equal(f.variables["pressure_mean"][:], ps)
        assert np.array_equal(f.variables["moisture_mean"][:], th)


def test_odd_sizes_pad_names(tmp_path):
    # a 1-character name and odd lengths exercise the 4-byte padding of names and data
    db.write_netcdf_state(str(tmp_path / "a.nc"), None, 3, 1, 1, np.arange(3.0), np.ones(3))
    with netcdf(str(tmp_path / "a.nc"), "r", mmap=False) as f:
        assert np.array_equal(f.variables["water_elevation"][:], np.arange(3.0).reshape(1, 3))


def test_unwritable_path_is_an_error(tmp_path):
    with pytest.raises(db.DharaError) as e:
        db.write_netcdf_state(str(tmp_path / "no" / "such" / "dir.nc"), None, 2, 2, 1, np.zeros(4), np.zeros(4))
    assert e.value.code == 1
