"""Dirichlet (type 0) side and bottom faces on the GPU path against the oracle
(which is pinned to the reference's assembly kernel with Dirichlet faces,
tests/test_ref_kernels.py::test_assembly[True]): uniform faces, a corner where
two faces meet, and faces whose type varies along the face."""
import numpy as np
import pytest

import dhara_b200 as db
import oracle
from dhara_b200 import inputs, _abi

pytestmark = pytest.mark.gpu


def domain_with_faces(faces, seed=11, prec=db.FP64, nsteps=3, varying=False):
    nx, ny, nz = 14, 11, 9
    d = inputs.make_domain(nx, ny, nz, seed=seed, krylov_tol=1e-13, krylov_maxiter=6000, nsteps=nsteps,
                           rain_mm_per_h=25.0, picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-10,
                           overland_tol=1e-13, overland_maxiter=5000, precision=prec, water_table=0.25)
    C, WE, SN = nx * ny, nz * ny, nz * nx
    rng = np.random.default_rng(seed)
    spec = {"bottom": (C, "bcb", "bcpsib"), "south": (SN, "bcs", "bcpsis"), "north": (SN, "bcn", "bcpsin"),
            "west": (WE, "bcw", "bcpsiw"), "east": (WE, "bce", "bcpsie")}
    for face, head in faces.items():
        n, tkey, pkey = spec[face]
        t = np.zeros(n, np.int32)
        if varying:
            t[rng.random(n) < 0.5] = 1
        d.int_fields[tkey] = t
        d.fields[pkey] = head + 0.05 * rng.standard_normal(n)
    return d


def compare(d, nsteps, tol):
    so, od, _ = oracle.run(d, nsteps=nsteps, solver3d=oracle.SOLVER_BICGSTAB)
    sg, gd, _ = db.run(d, nsteps=nsteps)
    for k in ("psi", "theta", "ponding"):
        err = np.max(np.abs(sg[k] - so[k])) / max(np.max(np.abs(so[k])), 1e-30)
        assert err < tol, (k, err)
    assert gd["nonfinite"] == 0


@pytest.mark.parametrize("faces", [{"bottom": 0.2}, {"west": -0.3}, {"east": -0.2, "north": -0.1},
                                   {"south": -0.4, "west": -0.3, "bottom": 0.1}])
def test_dirichlet_faces_match_oracle(gpu, faces):
    compare(domain_with_faces(faces), 3, 1e-6)


def test_dirichlet_varying_types(gpu):
    compare(domain_with_faces({"bottom": 0.1, "south": -0.3, "east": -0.2}, varying=True), 3, 1e-6)


def test_dirichlet_mixed_precision(gpu):
    compare(domain_with_faces({"west": -0.3, "bottom": 0.1}, prec=db.MIXED), 3, 1e-6)
