"""CPU tests of the FP64 oracle: known answers, invariants and golden vectors.

The oracle is the checker of the GPU library.  Its per-kernel functions are
pinned against the reference's own kernels on the GPU (test_ref_kernels.py);
these CPU tests pin the rest: closed-form van Genuchten values computed here
independently, the theta -> psi -> theta round trip, the structure of the
assembled matrix, the Krylov solves' convergence, the discrete mass balance,
and regression against committed golden vectors (tests/golden/).
"""
import json
import os

import numpy as np
import pytest

import oracle
from dhara_b200 import _abi, inputs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def vg_closed_form(psi, alpha_m, n, ts, tr, ks):
    """theta, K, C of van Genuchten-Mualem written directly from the formulas
    (alpha in 1/m, psi in m)."""
    m = 1 - 1 / n
    x = alpha_m * np.abs(psi)
    th = np.where(psi < 0, tr + (ts - tr) * (1 + x ** n) ** (-m), ts)
    se = (th - tr) / (ts - tr)
    K = ks * np.sqrt(se) * (1 - (1 - se ** (1 / m)) ** m) ** 2
    C = np.where(psi < 0, alpha_m * (n - 1) * (ts - tr) * x ** (n - 1) * (1 + x ** n) ** (-(2 * n - 1) / n), 0.0)
    return th, K, C


@pytest.fixture(scope="module")
def p():
    return _abi.make_params(8, 6, 5, alpha=3.5, n=1.6, theta_s=0.45, theta_r=0.05, porosity=0.45)


def test_van_genuchten_closed_form(p):
    psi = np.array([-10.0, -2.0, -1.0, -0.5, -0.1, -0.01, -1e-4, 0.0, 0.3])
    ks = np.full(psi.size, 1e-5)
    C, th, K = oracle.van_genuchten(p, psi, ks)
    th_r, K_r, C_r = vg_closed_form(psi, 3.5, 1.6, 0.45, 0.05, 1e-5)
    np.testing.assert_allclose(th, th_r, rtol=1e-13)
    np.testing.assert_allclose(C, C_r, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(K[psi < -1e-3], K_r[psi < -1e-3], rtol=1e-12)
    assert np.all(K[psi >= 0] == 1e-5) and np.all(C[psi >= 0] == 0) and np.all(th[psi >= 0] == 0.45)


def test_capacity_is_dtheta_dpsi(p):
    psi = np.linspace(-3, -0.01, 50)
    h = 1e-6
    C, _, _ = oracle.van_genuchten(p, psi, np.ones(psi.size))
    _, tp, _ = oracle.van_genuchten(p, psi + h, np.ones(psi.size))
    _, tm, _ = oracle.van_genuchten(p, psi - h, np.ones(psi.size))
    np.testing.assert_allclose(C, (tp - tm) / (2 * h), rtol=1e-6)


def test_inverse_round_trip(p):
    theta = np.linspace(0.06, 0.449, 40)
    psi = oracle.van_genuchten_inverse(p, theta)
    _, th2, _ = oracle.van_genuchten(p, psi, np.ones(theta.size))
    np.testing.assert_allclose(th2, theta, rtol=1e-12)
    assert oracle.van_genuchten_inverse(p, np.array([0.45]))[0] == 0.0


def small_domain(**kw):
    args = dict(seed=3, krylov_tol=1e-13, krylov_maxiter=4000, nsteps=8, rain_mm_per_h=25.0)
    args.update(kw)
    return inputs.make_domain(10, 7, 6, **args)


def test_neumann_matrix_symmetric_and_dominant():
    d = small_domain()
    o = oracle.Oracle(d.params)
    o.load(d)
    o.prepare()
    a3d, _ = o.assemble()
    p = d.params
    N = p.nx * p.ny * p.nz
    offs = [-p.nx * p.ny, -p.nx, -1, 0, 1, p.nx, p.nx * p.ny]
    A = np.zeros((N, N))
    for dgi, off in enumerate(offs):
        for row in range(N):
            col = row + off
            if 0 <= col < N:
                A[row, col] += a3d[dgi * N + row]
    np.testing.assert_allclose(A, A.T, rtol=1e-14, atol=0)
    off_sum = np.sum(np.abs(A), axis=1) - np.abs(np.diag(A))
    assert np.all(np.diag(A) > off_sum)
    o.close()


def test_solvers_agree():
    d = small_domain()
    a, _, _ = oracle.run(d, nsteps=3, solver3d=oracle.SOLVER_BICGSTAB)
    b, _, _ = oracle.run(d, nsteps=3, solver3d=oracle.SOLVER_CG)
    for k in ("psi", "theta", "ponding"):
        assert np.max(np.abs(a[k] - b[k])) <= 1e-9 * np.max(np.abs(a[k])), k


def test_conservative_update_closes_balance():
    d = small_domain(theta_update=_abi.THETA_CONSERVATIVE, overland_maxiter=5000, overland_tol=1e-13)
    _, dg, _ = oracle.run(d, nsteps=8, solver3d=oracle.SOLVER_CG)
    sub = dg["storage_change_cum"] - (dg["top_inflow_cum"] - dg["bottom_outflow_cum"])
    assert abs(sub) <= 1e-10 * dg["rain_cum"]
    total = dg["storage_change_cum"] + dg["ponded_volume"] - (
        dg["rain_cum"] - dg["bottom_outflow_cum"] - dg["overland_boundary_out_cum"] + dg["overland_clip_cum"])
    assert abs(total) <= 1e-8 * dg["rain_cum"]


def test_reference_rollover_leaves_picard_defect():
    """The reference's theta^n <- theta(psi^m) rollover does not close the
    discrete balance; the conservative one does (why the benchmark uses it)."""
    d = small_domain(theta_update=_abi.THETA_REFERENCE, picard_maxiter=3)
    _, dg, _ = oracle.run(d, nsteps=8, solver3d=oracle.SOLVER_CG)
    sub = dg["storage_change_cum"] - (dg["top_inflow_cum"] - dg["bottom_outflow_cum"])
    assert abs(sub) > 1e-9 * dg["rain_cum"]


def test_stateless_kernels_drive_the_step():
    """oracle_k_assemble on the oracle's own state equals oracle_assemble."""
    d = small_domain()
    o = oracle.Oracle(d.params)
    o.load(d)
    o.prepare()
    a1, b1 = o.assemble()
    a2, b2 = o.assemble()
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    o.close()


def _golden_cases():
    path = os.path.join(GOLDEN, "manifest.json")
    with open(path) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_oracle_against_golden(case):
    data = np.load(os.path.join(GOLDEN, case["file"]))
    d = inputs.make_domain(**case["domain"])
    st, dg, _ = oracle.run(d, nsteps=case["nsteps"], solver3d=case["solver3d"], solver2d=case["solver2d"])
    for k in ("psi", "theta", "ponding", "waterelev"):
        np.testing.assert_allclose(st[k], data[k], rtol=case["rtol"], atol=case["atol"], err_msg=k)
    assert dg["picard_iters_total"] == int(data["picard_iters_total"])
