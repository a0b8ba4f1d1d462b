"""CPU checks of the FP64 reference gradient (oracle/adjoint_ref.py): its
forward restatement reproduces the oracle's time steps, and its autograd
gradient matches central finite differences of the loss."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
from oracle import adjoint_ref as ar
from dhara_b200 import inputs, _abi


def tiny(picard_tol=1e-9, **kw):
    args = dict(seed=4, krylov_tol=1e-14, krylov_maxiter=5000, nsteps=6, rain_mm_per_h=40.0,
                picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=picard_tol, picard_maxiter=4,
                theta_update=_abi.THETA_CONSERVATIVE, overland_tol=1e-14, overland_maxiter=5000,
                water_table=0.3)
    args.update(kw)
    return inputs.make_domain(7, 6, 8, **args)


def test_forward_matches_oracle():
    d = tiny(picard_maxiter=6)
    st, dg, _ = oracle.run(d, nsteps=6, solver3d=oracle.SOLVER_CG)
    with torch.no_grad():
        out = ar.Model(d).run(6)
    assert np.max(np.abs(out["psi"].reshape(-1).numpy() - st["psi"])) < 1e-10
    assert np.max(np.abs(out["theta"][-1].reshape(-1).numpy() - st["theta"])) < 1e-11
    assert np.max(np.abs(out["ph"].reshape(-1).numpy() - st["ponding"])) < 1e-11
    assert abs(float(sum(out["q"])) - dg["overland_boundary_out_cum"]) < 1e-10


@pytest.mark.parametrize("update", [_abi.THETA_CONSERVATIVE, _abi.THETA_REFERENCE])
def test_gradient_matches_finite_differences(update):
    d = tiny(picard_tol=1e-300, theta_update=update)
    m = ar.Model(d)
    rng = np.random.default_rng(0)
    th_t, q_t = ar.targets_from(d, 6, logks=m.logks0 + 0.3 * torch.tensor(rng.standard_normal(m.logks0.shape)))
    L, g_lk, g_al, g_n, _ = ar.reference_gradient(d, 6, th_t, q_t)

    def loss(**kw):
        with torch.no_grad():
            return float(ar.loss_of(m.run(6, **kw), th_t, q_t))

    h = 1e-4
    for name, base, g in (("logks", m.logks0, g_lk), ("alpha", m.alpha0, g_al), ("n", m.n0, g_n)):
        scale = np.max(np.abs(g))
        for c in rng.choice(m.N, 4, replace=False):
            up, dn = base.clone().reshape(-1), base.clone().reshape(-1)
            up[c] += h
            dn[c] -= h
            kw = {"logks": "logks", "alpha": "alpha", "n": "n"}[name]
            fd = (loss(**{kw: up.reshape(base.shape)}) - loss(**{kw: dn.reshape(base.shape)})) / (2 * h)
            assert abs(g[c] - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale), (name, c, g[c], fd)
