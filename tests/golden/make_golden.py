"""Writes the golden vectors in this directory from the FP64 oracle.

The reference's solver (CUSP 0.5.1 on CUDA Thrust) cannot be built in this
environment and the reference ships no outputs, so the golden vectors are the
oracle's results on small seeded domains.  The oracle's per-kernel functions
are checked against the reference's own kernels compiled from their sources
(tests/test_ref_kernels.py); these vectors pin the composed time stepping
against regressions and are the fixed targets of the GPU parity tests.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from dhara_b200 import _abi, inputs  # noqa: E402

CASES = [
    dict(name="relative_rule_10x7x6", nsteps=4, solver3d=oracle.SOLVER_BICGSTAB, solver2d=oracle.SOLVER_CG,
         rtol=1e-8, atol=1e-11,
         domain=dict(nx=10, ny=7, nz=6, seed=11, rain_mm_per_h=25.0, nsteps=4, krylov_tol=1e-13,
                     krylov_maxiter=4000, overland_maxiter=5000, overland_tol=1e-13,
                     picard_rule=_abi.PICARD_PSI_RELATIVE, picard_tol=1e-8, picard_maxiter=10)),
    dict(name="absolute_rule_conservative_12x9x8", nsteps=5, solver3d=oracle.SOLVER_CG, solver2d=oracle.SOLVER_CG,
         rtol=1e-8, atol=1e-11,
         domain=dict(nx=12, ny=9, nz=8, seed=12, rain_mm_per_h=40.0, nsteps=5, krylov_tol=1e-13,
                     krylov_maxiter=4000, overland_maxiter=5000, overland_tol=1e-13,
                     picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-7, picard_maxiter=20,
                     theta_update=_abi.THETA_CONSERVATIVE)),
    dict(name="heterogeneous_slope_16x5x10", nsteps=3, solver3d=oracle.SOLVER_BICGSTAB, solver2d=oracle.SOLVER_CG,
         rtol=1e-8, atol=1e-11,
         domain=dict(nx=16, ny=5, nz=10, seed=13, rain_mm_per_h=60.0, nsteps=3, ks_sigma_ln=1.5, slope=0.03,
                     topo_sigma=0.08, krylov_tol=1e-13, krylov_maxiter=4000, overland_maxiter=5000,
                     overland_tol=1e-13, picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-7,
                     picard_maxiter=15)),
]


def main():
    manifest = []
    for c in CASES:
        dom = dict(c["domain"])
        nx, ny, nz = dom.pop("nx"), dom.pop("ny"), dom.pop("nz")
        d = inputs.make_domain(nx, ny, nz, **dom)
        st, dg, _ = oracle.run(d, nsteps=c["nsteps"], solver3d=c["solver3d"], solver2d=c["solver2d"])
        fname = c["name"] + ".npz"
        np.savez_compressed(os.path.join(HERE, fname), psi=st["psi"], theta=st["theta"], ponding=st["ponding"],
                            waterelev=st["waterelev"], picard_iters_total=dg["picard_iters_total"],
                            mb_subsurface_cum=dg["mb_subsurface_cum"])
        entry = dict(c, file=fname)
        entry["domain"] = dict(c["domain"])
        manifest.append(entry)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py (FP64 oracle)", "cases": manifest}, f, indent=1)


if __name__ == "__main__":
    main()
