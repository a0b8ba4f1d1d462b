"""The multigrid-preconditioned overland CG (dhara_params.overland_solver 0,
csrc/overland_mg.cu) against the pipelined Jacobi-PCG it replaces as the
default (overland_solver 1): both solve the reference's system
(src/overland.cu:65-189, 410-411) with the same stopping rule, so converged
they agree to the tolerance; the multigrid solve converges in tens of
iterations where ponded cells stall Jacobi; batching uneven domains (down
to a single interior cell, or none) does not change any domain's bits.
"""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

pytestmark = pytest.mark.gpu


def storm(n, solver, tol=1e-12, maxiter=20000, nsteps=8, seed=2):
    """The 512x512x40 storm's physics on an n x n x 20 domain."""
    return inputs.mixed_512x512x40(nx=n, ny=n, nz=20, seed=seed, nsteps=nsteps, precision=db.FP64,
                                   overland_tol=tol, overland_maxiter=maxiter, overland_solver=solver)


def run(doms, nsteps):
    s = db.Solver([d.params for d in doms])
    for i, d in enumerate(doms):
        s.load(d, i)
    s.prepare()
    s.step(nsteps)
    out = [({k: s.download(k, i) for k in ("psi", "ponding", "waterelev")}, s.diagnostics(i))
           for i in range(len(doms))]
    s.close()
    return out


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_multigrid_matches_jacobi_when_both_converge(gpu):
    # the storm's first steps, before ponding makes the Jacobi solve stall
    (mg, dmg), = run([storm(96, 0, nsteps=4)], 4)
    (jc, djc), = run([storm(96, 1, nsteps=4)], 4)
    assert dmg["overland_nonconverged"] == 0 and djc["overland_nonconverged"] == 0
    print("overland iterations: multigrid", dmg["overland_iters_total"], "Jacobi", djc["overland_iters_total"])
    assert dmg["overland_iters_total"] < djc["overland_iters_total"]
    assert rel(mg["waterelev"], jc["waterelev"]) < 1e-9
    assert rel(mg["ponding"], jc["ponding"]) < 1e-6
    assert rel(mg["psi"], jc["psi"]) < 1e-8


def test_multigrid_converges_where_jacobi_stalls(gpu):
    # 24 storm steps on a 192 x 192 surface (pools form after ~10 steps),
    # at most 400 iterations per solve
    (_, dmg), = run([storm(192, 0, maxiter=400, nsteps=24)], 24)
    (_, djc), = run([storm(192, 1, maxiter=400, nsteps=24)], 24)
    print("solves at the cap: multigrid", dmg["overland_nonconverged"], "Jacobi", djc["overland_nonconverged"],
          "iterations", dmg["overland_iters_total"], djc["overland_iters_total"])
    assert dmg["overland_nonconverged"] == 0
    assert djc["overland_nonconverged"] > 0
    assert dmg["overland_iters_total"] / 24 < 200


def test_multigrid_batch_equals_individual(gpu):
    """Uneven domains, including one with a single interior cell and one with
    none (a 2-cell-wide strip), one elongated and one large enough for grid
    levels: each domain's results are the same bits batched or alone."""
    kw = dict(precision=db.FP64, rain_mm_per_h=40.0, nsteps=3, overland_tol=1e-12, overland_maxiter=5000)
    doms = [inputs.make_domain(3, 3, 5, seed=1, **kw), inputs.make_domain(2, 9, 5, seed=2, **kw),
            inputs.make_domain(5, 70, 6, seed=3, **kw), inputs.make_domain(140, 90, 6, seed=4, **kw),
            inputs.make_domain(33, 17, 8, seed=5, **kw)]
    both = run(doms, 3)
    for i, d in enumerate(doms):
        (alone, da), = run([d], 3)
        sb, dbt = both[i]
        for k in alone:
            assert np.array_equal(alone[k], sb[k]), (i, k)
        assert da["overland_iters_total"] == dbt["overland_iters_total"], i
        assert da["overland_nonconverged"] == 0, i


def test_multigrid_rejects_mixed_solvers(gpu):
    a = inputs.make_domain(8, 8, 4, seed=1, overland_solver=0)
    b = inputs.make_domain(8, 8, 4, seed=2, overland_solver=1)
    with pytest.raises(db.DharaError, match="overland solver"):
        db.Solver([a.params, b.params])
