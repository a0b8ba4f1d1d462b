"""GPU parity: the CUDA path through the C ABI against the FP64 CPU oracle.

Tolerances (norm-wise max|gpu-oracle| / max|oracle|):
  FP64 mode, 1 step ........ 1e-8   (measured ~1e-9)
  FP64 mode, 5 steps ....... 1e-7
  mixed mode, 1 step ....... 1e-4   (the mixed-precision target)
Longer horizons are checked through size-independent properties (mass
closure, batch = individual runs, graph replay = eager) because the
reference scheme's discrete switches (Manning K0 / Manning branch, Picard stop
iteration) amplify 1e-12 solver noise ~1e5-fold over tens of steps -- the
oracle run with two different Krylov solvers differs by 3e-7 after 60 steps.
"""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs
import oracle

from conftest import rel_err

pytestmark = pytest.mark.gpu


def small(nx=16, ny=12, nz=10, **kw):
    args = dict(seed=7, krylov_tol=1e-12, krylov_maxiter=2000, nsteps=10, rain_mm_per_h=30.0)
    args.update(kw)
    return inputs.make_domain(nx, ny, nz, **args)


def run_both(d, nsteps, **kw):
    g, gd, _ = db.run(d, nsteps=nsteps, **kw)
    o, od, _ = oracle.run(d, nsteps=nsteps, solver3d=oracle.SOLVER_CG)
    return g, gd, o, od


def test_closure_matches_oracle(gpu):
    d = small()
    s = db.Solver(d.params)
    s.load(d)
    s.prepare()
    C, th, K = oracle.van_genuchten(d.params, d.fields["psi"], d.fields["ksat"])
    assert rel_err(s.download("K"), K) < 1e-13
    assert rel_err(s.download("C"), C) < 1e-13
    assert rel_err(s.download("theta"), th) < 1e-14
    s.close()


def test_psi_from_theta_matches_oracle(gpu):
    d = small()
    theta = np.repeat(0.3 + 0.01 * np.arange(d.params.nz), d.params.nx * d.params.ny)
    s = db.Solver(d.params)
    s.load(d)
    s.upload("theta", theta)
    s.psi_from_theta()
    ref = oracle.van_genuchten_inverse(d.params, theta)
    assert rel_err(s.download("psi"), ref) < 1e-13
    s.close()


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-8), (5, 1e-7)])
def test_fp64_steps(gpu, nsteps, tol):
    d = inputs.plain_fp64_32x32x20(krylov_tol=1e-12, krylov_maxiter=2000)
    g, gd, o, od = run_both(d, nsteps)
    for k in ("psi", "theta", "waterelev"):
        assert rel_err(g[k], o[k]) < tol, k
    # ponded depth is a small difference H - z: its relative error carries the
    # overland solve's tolerance (1e-12 of ||H||); the FP64 target is 1e-6
    assert rel_err(g["ponding"], o["ponding"]) < 1e-6
    assert gd["picard_iters_total"] == od["picard_iters_total"]
    assert gd["nonfinite"] == 0
    assert abs(gd["mb_subsurface_cum"] - od["mb_subsurface_cum"]) < 1e-9 * max(1.0, abs(od["mb_subsurface_cum"]))


@pytest.mark.parametrize("nsteps", [1, 5])
def test_mixed_steps(gpu, nsteps):
    d = inputs.plain_fp64_32x32x20(precision=db.MIXED, krylov_tol=1e-12, krylov_maxiter=2000)
    g, gd, o, od = run_both(d, nsteps)
    for k in ("psi", "theta", "ponding", "waterelev"):
        assert rel_err(g[k], o[k]) < 1e-6, k
    assert gd["refine_iters_total"] >= gd["picard_iters_total"]


def test_mixed_fp32_closure(gpu):
    """FP32 closure: the refinement converges to the FP32-coefficient system,
    which stays within the mixed-precision target of the FP64 oracle for a
    step and keeps the discrete mass balance closed."""
    d = inputs.plain_fp64_32x32x20(precision=db.MIXED, closure_fp32=1, krylov_tol=1e-10,
                                   theta_update=db.THETA_CONSERVATIVE)
    g, gd, o, od = run_both(d, 1)
    assert rel_err(g["theta"], o["theta"]) < 1e-4
    assert gd["nonfinite"] == 0
    err = gd["storage_change_cum"] - (gd["top_inflow_cum"] - gd["bottom_outflow_cum"])
    assert abs(err) <= 1e-8 * gd["rain_cum"]


@pytest.mark.parametrize("prec", [db.FP64, db.MIXED])
def test_conservative_mass_closure(gpu, prec):
    d = inputs.plain_fp64_32x32x20(precision=prec, theta_update=db.THETA_CONSERVATIVE, nsteps=20)
    _, gd, _ = db.run(d, nsteps=20)
    err = gd["storage_change_cum"] - (gd["top_inflow_cum"] - gd["bottom_outflow_cum"])
    assert abs(err) <= 1e-8 * gd["rain_cum"], err
    total = gd["storage_change_cum"] + gd["ponded_volume"] - (
        gd["rain_cum"] - gd["bottom_outflow_cum"] - gd["overland_boundary_out_cum"] + gd["overland_clip_cum"])
    assert abs(total) <= 1e-6 * gd["rain_cum"], total


def test_graph_replay_equals_eager(gpu):
    d = small(precision=db.MIXED, theta_update=db.THETA_CONSERVATIVE)
    a, ad, _ = db.run(d, nsteps=6, graph=False)
    b, bd, _ = db.run(d, nsteps=6, graph=True)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert ad["krylov_iters_total"] == bd["krylov_iters_total"]


@pytest.mark.parametrize("prec", [db.FP64, db.MIXED])
def test_batch_equals_individual(gpu, prec):
    doms = [small(17, 9, 7, seed=1, precision=prec), small(40, 33, 12, seed=2, precision=prec),
            small(5, 70, 4, seed=3, precision=prec)]
    batch = db.run(doms, nsteps=3)
    for d, (st, dg, _) in zip(doms, batch):
        one, od, _ = db.run(d, nsteps=3)
        for k in st:
            assert np.array_equal(st[k], one[k]), k
        assert dg["krylov_iters_total"] == od["krylov_iters_total"]


@pytest.mark.parametrize("shape", [(1, 1, 2), (2, 2, 2), (3, 1, 5), (33, 5, 3), (1, 40, 6)])
def test_ragged_and_tiny_domains(gpu, shape):
    d = small(*shape, seed=11)
    g, gd, o, od = run_both(d, 2)
    for k in ("psi", "theta", "ponding", "waterelev"):
        assert rel_err(g[k], o[k]) < 1e-8, (k, shape)


def test_reference_defaults_unsaturated(gpu):
    """The reference's own configuration style: device-default physics
    (alpha 0.02 /cm, n 1.8, theta_r 0.1, am 0), relative Picard rule, theta
    initial condition 0.3 + 0.01 k converted by vanGenuchtenInverse."""
    nx, ny, nz = 12, 10, 15
    p = db.make_params(nx, ny, nz, dx=1.2, dy=1.2, dz=0.2, dt=1800.0, krylov_tol=1e-12,
                       krylov_maxiter=2000, overland_maxiter=3000, overland_tol=1e-12)
    rng = np.random.default_rng(5)
    C = nx * ny
    theta = np.repeat(0.3 + 0.01 * np.arange(nz), C)
    dom = inputs.Domain(params=p, fields=dict(
        theta=theta, ksat=np.full(nx * ny * nz, 0.0025 / 1800.0),
        ztopo=220.0 + 0.05 * rng.standard_normal(C), mann=np.full(C, 0.025),
        waterdepth=np.zeros(C), ponding=np.zeros(C), ppt=np.full(C, 2.0),
        esoil=np.zeros(C), tr=np.zeros(C)), int_fields={}, rain_mm=np.zeros(0))
    s = db.Solver(p)
    s.load(dom, schedule=False)
    s.psi_from_theta()
    s.prepare()
    o = oracle.Oracle(p, oracle.SOLVER_CG)
    o.load(dom)
    o.psi_from_theta()
    o.prepare()
    for _ in range(3):
        s.step(1)
        o.step()
    s.synchronize()
    for k in ("psi", "theta", "ponding"):
        assert rel_err(s.download(k), o.download(k)) < 1e-8, k
    s.close()
    o.close()


def test_transpiration_roots(gpu):
    d = small(12, 8, 6, seed=4)
    rng = np.random.default_rng(3)
    nproc = 3
    rda = rng.uniform(0, 0.3, size=(nproc, d.params.nz)).reshape(-1)
    procmap = rng.integers(0, nproc, size=d.params.nx * d.params.ny).astype(np.int32)
    tr = rng.uniform(0, 2e-4, size=d.params.nx * d.params.ny)
    s = db.Solver(d.params)
    s.load(d)
    s.set_roots(rda, nproc)
    s.upload("procmap", procmap)
    s.upload("tr", tr)
    s.prepare()
    s.step(2)
    s.synchronize()
    o = oracle.Oracle(d.params, oracle.SOLVER_CG)
    o.load(d)
    lib = oracle.lib()
    import ctypes as ct
    lib.oracle_set_roots(o.h, rda.ctypes.data_as(ct.POINTER(ct.c_double)), nproc)
    o.upload("procmap", procmap)
    o.upload("tr", tr)
    o.prepare()
    for t in range(2):
        o.step(d.rain_mm[t])
    for k in ("psi", "theta", "ponding"):
        assert rel_err(s.download(k), o.download(k)) < 1e-8, k
    assert abs(s.diagnostics()["mb_subsurface_cum"] - o.diagnostics()["mb_subsurface_cum"]) < 1e-9
    s.close()
    o.close()


def test_per_cell_parameters_equal_scalars(gpu):
    d = small(seed=9)
    a, _, _ = db.run(d, nsteps=2)
    d2 = small(seed=9, per_cell_vg=True)
    b, _, _ = db.run(d2, nsteps=2)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_error_paths(gpu):
    d = small()
    s = db.Solver(d.params)
    with pytest.raises(db.DharaError) as e:
        s.step(1)
    assert e.value.code == 7
    with pytest.raises(db.DharaError) as e:
        s.upload("psi", np.zeros(3))
    assert e.value.code == 1
    # Dirichlet faces are accepted, but the adjoint does not cover them
    s.upload("bcw", np.zeros(d.params.nz * d.params.ny, np.int32))
    with pytest.raises(db.DharaError) as e:
        s.adjoint(np.zeros((1, 3, d.params.nx * d.params.ny)), np.zeros(1), 1)
    assert e.value.code == 4
    with pytest.raises(db.DharaError) as e:
        s.upload("ksat", np.full(d.ncells, np.nan))
    assert e.value.code == 5
    s.close()


def _golden():
    import json
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with open(os.path.join(here, "manifest.json")) as f:
        return here, json.load(f)["cases"]


@pytest.mark.parametrize("precision", [db.FP64, db.MIXED])
@pytest.mark.parametrize("case", _golden()[1], ids=lambda c: c["name"])
def test_gpu_against_golden(gpu, case, precision):
    """The CUDA path against the committed golden vectors (FP64 oracle)."""
    import os
    here, _ = _golden()
    data = np.load(os.path.join(here, case["file"]))
    d = inputs.make_domain(**dict(case["domain"], precision=precision))
    st, dg, _ = db.run(d, nsteps=case["nsteps"])
    for k in ("psi", "theta", "waterelev"):
        assert rel_err(st[k], data[k]) < 1e-8, k
    assert rel_err(st["ponding"], data["ponding"]) < 1e-6
    assert dg["picard_iters_total"] == int(data["picard_iters_total"])
