"""The GPU discrete adjoint (dhara_adjoint) against the FP64 reference
gradient (oracle/adjoint_ref.py, autograd through an exact-solve restatement
of the same discrete model) and against central finite differences of the GPU
forward loss."""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs, _abi

torch = pytest.importorskip("torch")
from oracle import adjoint_ref as ar  # noqa: E402

pytestmark = pytest.mark.gpu
NSTEPS = 6


def tiny(**kw):
    args = dict(seed=4, krylov_tol=1e-13, krylov_maxiter=5000, nsteps=NSTEPS, rain_mm_per_h=40.0,
                picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-300, picard_maxiter=4,
                theta_update=_abi.THETA_CONSERVATIVE, overland_tol=1e-14, overland_maxiter=5000,
                water_table=0.3)
    args.update(kw)
    return inputs.make_domain(7, 6, 8, **args)


def targets(d, nsteps, seed=0):
    m = ar.Model(d)
    rng = np.random.default_rng(seed)
    th_t, q_t = ar.targets_from(d, nsteps, logks=m.logks0 + 0.3 * torch.tensor(rng.standard_normal(m.logks0.shape)))
    th = np.stack([t[:3].reshape(3, -1).numpy() for t in th_t])
    q = np.array([float(x) for x in q_t])
    return th_t, q_t, th, q


def gpu_adjoint(d, th, q, nsteps, precision=db.FP64, every=4, gradients=True):
    p = type(d.params).from_buffer_copy(d.params)
    p.precision = precision
    s = db.Solver(p)
    s.load(d)
    s.prepare()
    out = s.adjoint(th, q, nsteps, checkpoint_every=every, gradients=gradients)
    st = {k: s.download(k) for k in ("psi", "theta", "ponding", "waterelev")}
    s.close()
    return out, st


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("update", [_abi.THETA_CONSERVATIVE, _abi.THETA_REFERENCE])
def test_adjoint_matches_reference_gradient(gpu, update):
    d = tiny(theta_update=update)
    th_t, q_t, th, q = targets(d, NSTEPS)
    L_ref, g_lk, g_al, g_n, _ = ar.reference_gradient(d, NSTEPS, th_t, q_t)
    (L, a_lk, a_al, a_n), _ = gpu_adjoint(d, th, q, NSTEPS)
    assert abs(L - L_ref) <= 1e-9 * L_ref
    assert rel(a_lk, g_lk) < 1e-6
    assert rel(a_al, g_al) < 1e-6
    assert rel(a_n, g_n) < 1e-6


def test_checkpoint_interval_and_state(gpu):
    d = tiny()
    _, _, th, q = targets(d, NSTEPS)
    (L1, g1, _, _), st1 = gpu_adjoint(d, th, q, NSTEPS, every=1)
    (L6, g6, _, _), st6 = gpu_adjoint(d, th, q, NSTEPS, every=NSTEPS)
    L0, st0 = gpu_adjoint(d, th, q, NSTEPS, gradients=False)
    assert L1 == L6 == L0
    assert rel(g1, g6) < 1e-10
    # the handle ends in the state of the forward run
    st, _, _ = db.run(d, nsteps=NSTEPS)
    for k in ("psi", "theta", "ponding", "waterelev"):
        assert np.array_equal(st1[k], st[k]) and np.array_equal(st0[k], st[k]), k


def test_mixed_precision_adjoint(gpu):
    d = tiny()
    _, _, th, q = targets(d, NSTEPS)
    (L64, g64, a64, n64), _ = gpu_adjoint(d, th, q, NSTEPS)
    (L32, g32, a32, n32), _ = gpu_adjoint(d, th, q, NSTEPS, precision=db.MIXED)
    assert abs(L32 - L64) <= 1e-6 * L64
    assert rel(g32, g64) < 1e-4 and rel(a32, a64) < 1e-4 and rel(n32, n64) < 1e-4


def test_adjoint_matches_gpu_finite_differences(gpu):
    """Central differences of the GPU FP64 loss at h = 1e-4 and, where that
    step straddles a switch of the forward (the top-flux selection, the depth
    clip, Manning's wet test: the loss is piecewise smooth), h = 1e-5.  Where a
    cell's gradient is significant (|fd| >= 1e-3 of the largest gradient) the
    better of the two agrees to 1e-4 relative; elsewhere the loss differences
    are at its noise floor (~1e-11 in L), so the check is absolute, 1e-6 of
    the largest gradient."""
    nsteps = 8
    d = inputs.make_domain(20, 14, 12, seed=9, krylov_tol=1e-13, krylov_maxiter=5000, nsteps=nsteps,
                           rain_mm_per_h=30.0, picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-300,
                           picard_maxiter=5, theta_update=_abi.THETA_CONSERVATIVE, overland_tol=1e-14,
                           overland_maxiter=5000, water_table=0.4, per_cell_vg=True)
    _, _, th, q = targets(d, nsteps, seed=1)
    (L, g_lk, g_al, g_n), _ = gpu_adjoint(d, th, q, nsteps, every=3)
    rng = np.random.default_rng(5)
    h = 1e-4
    N = d.ncells
    for name, g in (("ksat", g_lk), ("alpha", g_al), ("nvg", g_n)):
        scale = np.max(np.abs(g))
        big = np.flatnonzero(np.abs(g) >= 1e-2 * scale)
        cells = np.concatenate([rng.choice(N, 2, replace=False), rng.choice(big, 2, replace=False)])
        for c in cells:
            def fd_at(hh):
                vals = []
                for sgn in (1, -1):
                    dd = inputs.Domain(params=d.params, fields={k: v.copy() for k, v in d.fields.items()},
                                       int_fields=d.int_fields, rain_mm=d.rain_mm)
                    if name == "ksat":
                        dd.fields["ksat"][c] *= np.exp(sgn * hh)
                    else:
                        dd.fields[name][c] += sgn * hh
                    Lh, _ = gpu_adjoint(dd, th, q, nsteps, gradients=False)
                    vals.append(Lh)
                return (vals[0] - vals[1]) / (2 * hh)
            fd = fd_at(h)
            if abs(fd) >= 1e-3 * scale:
                if abs(g[c] - fd) > 1e-4 * abs(fd):
                    fd = fd_at(h / 10)
                assert abs(g[c] - fd) <= 1e-4 * abs(fd), (name, c, g[c], fd)
            else:
                assert abs(g[c] - fd) <= 1e-6 * scale, (name, c, g[c], fd)
