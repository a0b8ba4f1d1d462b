"""The drop-in entry points (include/dhara_dropin.h) driven by a C++ host
program written like the reference's host code (tests/dropin/dropin_driver.cc:
reference struct layout, caller-allocated device arrays, one
SubsurfaceFlowModel + OverlandFlowModel call per step), checked against the
FP64 oracle of the reference algorithm on the same inputs, and against the
same steps through the C ABI directly (the drop-in adds no arithmetic)."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs
import oracle

from conftest import rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def build_driver(tmp):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = os.path.join(tmp, "dropin_driver")
    libdir = os.path.join(ROOT, "dhara_b200")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-x", "cu", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "dropin", "dropin_driver.cc"), "-L", libdir, "-ldhara_b200",
                    f"-Xlinker=-rpath,{libdir}", "-o", exe], check=True)
    return exe


def test_dropin_matches_oracle(gpu):
    nsteps = 4
    d = inputs.make_domain(20, 14, 8, seed=31, rain_mm_per_h=30.0, nsteps=nsteps, krylov_tol=1e-12,
                           krylov_maxiter=1000)
    p = d.params
    with tempfile.TemporaryDirectory() as tmp:
        exe = build_driver(tmp)
        with open(os.path.join(tmp, "params.bin"), "wb") as f:
            f.write(bytes(p))
        for k in ("psi", "ksat", "ztopo", "mann"):
            d.fields[k].astype(np.float64).tofile(os.path.join(tmp, f"{k}.bin"))
        d.rain_mm.astype(np.float64).tofile(os.path.join(tmp, "rain.bin"))
        out = subprocess.run([exe, tmp, str(nsteps)], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = {k: np.fromfile(os.path.join(tmp, f"out_{k}.bin")) for k in ("psi", "theta", "ph", "H", "mb")}
        # SaveModelResults / SaveResultEntirePeriod wrote the reference's files
        from scipy.io import netcdf_file
        with netcdf_file(os.path.join(tmp, f"ssf_{nsteps}.nc"), "r", mmap=False) as f:
            assert np.array_equal(f.variables["pressure_head"][:].reshape(-1), got["psi"])
            assert np.array_equal(f.variables["moisture"][:].reshape(-1), got["theta"])
        with netcdf_file(os.path.join(tmp, f"olf_{nsteps}.nc"), "r", mmap=False) as f:
            assert np.array_equal(f.variables["water_elevation"][:].reshape(-1), got["H"])
        with netcdf_file(os.path.join(tmp, "ssf1d.nc"), "r", mmap=False) as f:
            assert np.array_equal(f.variables["mb_subsurfaceW"][:], got["mb"])
    # the reference algorithm (FP64 oracle, converged 3D solves)
    o, od, _ = oracle.run(d, nsteps, solver3d=oracle.SOLVER_CG)
    assert rel_err(got["psi"], o["psi"]) < 1e-7
    assert rel_err(got["theta"], o["theta"]) < 1e-7
    assert rel_err(got["H"], o["waterelev"]) < 1e-7
    assert rel_err(got["ph"], o["ponding"]) < 1e-6
    assert abs(got["mb"].sum() - od["mb_subsurface_cum"]) <= 1e-9 * max(1.0, abs(od["mb_subsurface_cum"]))
    # and the drop-in is the C ABI's computation
    ref, dg, _ = db.run(d, nsteps=nsteps)
    assert rel_err(got["psi"], ref["psi"]) < 1e-12
    assert rel_err(got["theta"], ref["theta"]) < 1e-12
    assert rel_err(got["ph"], ref["ponding"]) < 1e-10
    assert rel_err(got["H"], ref["waterelev"]) < 1e-12
    assert abs(got["mb"].sum() - dg["mb_subsurface_cum"]) <= 1e-12 * max(1.0, abs(dg["mb_subsurface_cum"]))
