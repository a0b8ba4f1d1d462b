"""Output path: per-step statistics (the reference's CopyLayers layer sums and
mb_subsurfaceW) and asynchronous snapshots."""
import numpy as np
import pytest
import torch

import dhara_b200 as db
from dhara_b200 import inputs

pytestmark = pytest.mark.gpu


def small(**kw):
    args = dict(seed=7, rain_mm_per_h=30.0, nsteps=6, krylov_tol=1e-12, krylov_maxiter=2000)
    args.update(kw)
    return inputs.make_domain(20, 13, 9, **args)


@pytest.mark.parametrize("prec", [db.FP64, db.MIXED])
def test_layer_statistics(gpu, prec):
    d = small(precision=prec)
    p = d.params
    s = db.Solver(p)
    s.load(d)
    s.enable_statistics(10)
    s.prepare()
    ps_ref, th_ref, mb_ref = [], [], []
    for t in range(5):
        s.step(1, graph=(t % 2 == 1))
        psi = s.download("psi").reshape(p.nz, -1)
        th = s.download("theta_new").reshape(p.nz, -1)
        ps_ref.append(psi[:, :-1].sum(axis=1))   # the reference's range leaves out each layer's last cell
        th_ref.append(th[:, :-1].sum(axis=1))
        mb_ref.append(s.diagnostics()["mb_subsurface_last"])
    st = s.statistics()
    s.close()
    assert st["pressure_sum"].shape == (5, p.nz)
    np.testing.assert_allclose(st["pressure_sum"], np.array(ps_ref), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(st["moisture_sum"], np.array(th_ref), rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(st["mb_subsurfaceW"], np.array(mb_ref))


def test_snapshot_overlaps_next_steps(gpu):
    d = small()
    p = d.params
    N, C = p.nx * p.ny * p.nz, p.nx * p.ny
    s = db.Solver(p)
    s.load(d)
    s.prepare()
    s.step(2)
    want = {k: s.download(k) for k in ("psi", "theta", "waterelev", "waterdepth")}
    bufs = [{"pressure_head": torch.empty(N, dtype=torch.float64, pin_memory=True).numpy(),
             "moisture": torch.empty(N, dtype=torch.float64, pin_memory=True).numpy(),
             "water_elevation": torch.empty(C, dtype=torch.float64, pin_memory=True).numpy(),
             "water_depth": torch.empty(C, dtype=torch.float64, pin_memory=True).numpy()} for _ in range(2)]
    s.snapshot(bufs[0])
    s.step(1)
    s.snapshot(bufs[1])
    s.step(2)   # overwrites the state while the copies drain
    s.snapshot_wait()
    np.testing.assert_array_equal(bufs[0]["pressure_head"], want["psi"])
    np.testing.assert_array_equal(bufs[0]["moisture"], want["theta"])
    np.testing.assert_array_equal(bufs[0]["water_elevation"], want["waterelev"])
    np.testing.assert_array_equal(bufs[0]["water_depth"], want["waterdepth"])
    assert not np.array_equal(bufs[1]["pressure_head"], want["psi"])
    s.close()


def test_netcdf_files_from_a_handle(gpu, tmp_path):
    """The reference's result files (SaveModelResults / SaveResultEntirePeriod,
    src/io.cc:854-996) written from a handle, read back with scipy's NetCDF
    reader: the current state and the statistics kept on the device."""
    netcdf = pytest.importorskip("scipy.io").netcdf_file
    d = small()
    p = d.params
    s = db.Solver(p)
    s.load(d)
    s.enable_statistics(8)
    s.prepare()
    s.step(3)
    s.synchronize()
    f2, f3 = str(tmp_path / "olf_3.nc"), str(tmp_path / "ssf_3.nc")
    f1, fs = str(tmp_path / "ssf1d.nc"), str(tmp_path / "stat.nc")
    s.save_netcdf(f2, f3)
    s.save_netcdf_statistics(f1, fs)
    state = {k: s.download(k) for k in ("waterelev", "waterdepth", "psi", "theta")}
    st = s.statistics()
    s.close()
    with netcdf(f2, "r", mmap=False) as f:
        assert np.array_equal(f.variables["water_elevation"][:], state["waterelev"].reshape(p.ny, p.nx))
        assert np.array_equal(f.variables["water_depth"][:], state["waterdepth"].reshape(p.ny, p.nx))
    with netcdf(f3, "r", mmap=False) as f:
        assert np.array_equal(f.variables["pressure_head"][:], state["psi"].reshape(p.nz, p.ny, p.nx))
        assert np.array_equal(f.variables["moisture"][:], state["theta"].reshape(p.nz, p.ny, p.nx))
    with netcdf(f1, "r", mmap=False) as f:
        assert np.array_equal(f.variables["mb_subsurfaceW"][:], st["mb_subsurfaceW"])
    with netcdf(fs, "r", mmap=False) as f:
        assert np.array_equal(f.variables["pressure_mean"][:], st["pressure_sum"])
        assert np.array_equal(f.variables["moisture_mean"][:], st["moisture_sum"])
