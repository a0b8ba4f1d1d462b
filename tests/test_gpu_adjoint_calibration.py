"""The discrete adjoint at the size of the calibration configuration
(128x128x30 cells, the 32x32x20 workload's physics, all ten Picard
iterations every step) over a shortened horizon of 10 steps:

* against the FP64 reference gradient of oracle/adjoint_ref.py (autograd
  through a restatement of the same discrete model whose linear systems are
  solved to 1e-14 and differentiated implicitly; each step recomputed in the
  backward pass) -- FP64 mode within 1e-6, mixed mode within 1e-4;
* against central finite differences of the GPU loss on 32 random cells
  (log Ks) and 8 cells each for alpha and n, and along a random direction of
  the cells below the initial water table (a Taylor test).  The loss is only
  piecewise smooth: the forward switches branches (top-flux selection,
  ponding and depth clips, Manning's wet test; src/global.cu:236-251,
  src/subsurface.cu:480, src/overland.cu:279-297,378), so a difference is
  accepted only for a step h whose +h and -h runs took exactly the branches
  of the unperturbed run (dhara_diagnostics' branch_signature over those
  decisions and the Picard counts); accepted differences agree to 1e-4
  relative where the gradient is significant, and elsewhere to 1e-6 of the
  largest gradient plus the loss's noise over 2h.  The difference runs solve
  to 1e-13 (3D) and 1e-12 (overland, up to 50,000 iterations), so the loss
  is known to about 1e-13 of itself and a difference to 1e-13 |L| / h; the
  overland iteration counts are part of the branch pattern (a CG that stops
  at another iteration is another map).

The forward this reverses is src/subsurface.cu:686-847 + src/overland.cu:387-419.
"""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

torch = pytest.importorskip("torch")
from oracle import adjoint_ref as ar  # noqa: E402

pytestmark = pytest.mark.gpu
NSTEPS = 10
EVERY = 5
# every switch of the loss: top flux, ponding clip, Manning test, depth clip, Picard counts,
# overland iteration counts
SWITCHES = 1 | 2 | 4 | 8 | 32 | 64


def calib(precision=db.FP64, **kw):
    args = dict(nsteps=NSTEPS, precision=precision, overland_maxiter=20000, record_branches=SWITCHES)
    args.update(kw)
    return inputs.adjoint_128x128x30(**args)


def targets(d):
    """The calibration target: the same domain with log Ks perturbed by
    0.3 N(0, 1), run on the GPU; theta of every step and the overland flow
    into the ring per step."""
    p = d.params
    C = p.nx * p.ny
    rng = np.random.default_rng(11)
    t = inputs.Domain(params=p, fields={k: v.copy() for k, v in d.fields.items()}, int_fields=d.int_fields,
                      rain_mm=d.rain_mm)
    t.fields["ksat"] = t.fields["ksat"] * np.exp(0.3 * rng.standard_normal(d.ncells))
    s = db.Solver(p)
    s.load(t)
    s.prepare()
    th, q, th_full = np.zeros((NSTEPS, 3, C)), np.zeros(NSTEPS), []
    prev = s.diagnostics()["overland_boundary_out_cum"]
    for k in range(NSTEPS):
        s.step(1)
        full = s.download("theta")
        th[k] = full[:3 * C].reshape(3, C)
        th_full.append(torch.tensor(full.reshape(p.nz, p.ny, p.nx)))
        cur = s.diagnostics()["overland_boundary_out_cum"]
        q[k] = cur - prev
        prev = cur
    s.close()
    return th, q, th_full, [torch.tensor(x, dtype=torch.float64) for x in q]


def run(d, th, q, gradients=True, diag=False):
    s = db.Solver(d.params)
    s.load(d)
    s.prepare()
    out = s.adjoint(th, q, NSTEPS, checkpoint_every=EVERY, gradients=gradients)
    dg = s.diagnostics()
    s.close()
    return (out, dg["branch_signature"], dg) if diag else (out, dg["branch_signature"])


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def reference():
    torch.set_num_threads(max(1, __import__("os").cpu_count() or 1))
    d = calib()
    th, q, th_t, q_t = targets(d)
    L, g_lk, g_al, g_n, _ = ar.reference_gradient(d, NSTEPS, th_t, q_t, sparse=True, checkpoint=True)
    return d, th, q, L, g_lk, g_al, g_n


@pytest.fixture(scope="module")
def tight():
    """The calibration domain with tight solves, and its targets."""
    d = calib(krylov_tol=1e-13, krylov_maxiter=5000, overland_tol=1e-12, overland_maxiter=50000)
    th, q, _, _ = targets(d)
    return d, th, q


@pytest.mark.parametrize("precision,tol", [(db.FP64, 1e-6), (db.MIXED, 1e-4)], ids=["fp64", "mixed"])
def test_calibration_gradient_matches_fp64_reference(gpu, reference, precision, tol):
    d0, th, q, L_ref, r_lk, r_al, r_n = reference
    d = calib(precision)
    (L, g_lk, g_al, g_n), _ = run(d, th, q)
    errs = (abs(L - L_ref) / L_ref, rel(g_lk, r_lk), rel(g_al, r_al), rel(g_n, r_n))
    print("loss / log Ks / alpha / n relative errors", ["%.2e" % e for e in errs])
    assert errs[0] < tol
    assert errs[1] < tol and errs[2] < tol and errs[3] < tol


def perturbed(d, field, cell, delta):
    dd = inputs.Domain(params=d.params, fields={k: v.copy() for k, v in d.fields.items()},
                       int_fields=d.int_fields, rain_mm=d.rain_mm)
    if field == "ksat":
        if cell is None:
            dd.fields["ksat"] = dd.fields["ksat"] * np.exp(delta)
        else:
            dd.fields["ksat"][cell] *= np.exp(delta)
    else:
        base = dd.fields.get(field, np.full(d.ncells, d.params.alpha if field == "alpha" else d.params.n))
        dd.fields[field] = base.copy()
        if cell is None:
            dd.fields[field] += delta
        else:
            dd.fields[field][cell] += delta
    return dd


def central_difference(d, th, q, field, cell, base_sig, steps=(1e-4, 1e-5, 1e-6), direction=None):
    """The first h of `steps` whose +h and -h runs kept every branch of the
    unperturbed run, and its central difference (None, None if none did)."""
    for h in steps:
        vals, sigs = [], []
        for sgn in (1, -1):
            delta = sgn * h * (direction if direction is not None else 1.0)
            (Lh, sig) = run(perturbed(d, field, cell, delta), th, q, gradients=False)
            vals.append(Lh)
            sigs.append(sig)
        if sigs[0] == base_sig and sigs[1] == base_sig:
            return h, (vals[0] - vals[1]) / (2 * h)
    return None, None


def test_calibration_gradient_matches_central_differences(gpu, tight):
    d, th, q = tight
    (L, g_lk, g_al, g_n), base_sig, dg = run(d, th, q, diag=True)
    print("overland solves at their cap:", dg["overland_nonconverged"], "of", NSTEPS,
          "3D:", dg["krylov_nonconverged"])
    assert base_sig != 0
    # differences of a map whose solves stopped short are not derivatives of the exact map
    assert dg["overland_nonconverged"] == 0 and dg["krylov_nonconverged"] == 0
    rng = np.random.default_rng(2024)
    N = d.ncells
    report = {}
    for field, g, ncells in (("ksat", g_lk, 32), ("alpha", g_al, 8), ("nvg", g_n, 8)):
        scale = float(np.max(np.abs(g)))
        noise = 1e-13 * abs(L)  # half the spread of the loss between two runs of one map
        cells = rng.choice(N, ncells, replace=False)
        accepted = worst = 0.0
        for c in cells:
            h, fd = central_difference(d, th, q, field, int(c), base_sig)
            if h is None:
                continue   # every step flipped a branch: this cell is not differentiable at FD scale
            accepted += 1
            if abs(fd) >= 1e-3 * scale:
                err = abs(g[c] - fd) / abs(fd)
                assert err <= 1e-4, (field, int(c), h, g[c], fd)
            else:
                err = abs(g[c] - fd) / scale
                assert abs(g[c] - fd) <= 1e-6 * scale + noise / h, (field, int(c), h, g[c], fd, L)
            worst = max(worst, err)
        report[field] = (int(accepted), len(cells), worst)
        assert accepted >= len(cells) // 2, (field, accepted)
    print("loss", L, "cells accepted / drawn / worst error:", report)


def test_calibration_taylor_direction(gpu, tight):
    """Directional derivative along a random direction v of log Ks over every
    cell: (L(+h v) - L(-h v)) / 2h against g . v, at the first h in
    1e-3..1e-7 that keeps every branch, to 1e-4 relative plus the loss's
    noise over 2h."""
    d, th, q = tight
    (L, g_lk, _, _), base_sig = run(d, th, q)
    v = np.random.default_rng(7).standard_normal(d.ncells)
    h, fd = central_difference(d, th, q, "ksat", None, base_sig, steps=(1e-3, 1e-4, 1e-5, 1e-6, 1e-7),
                               direction=v)
    assert h is not None, "no step kept the branch pattern"
    gv = float(np.dot(g_lk, v))
    print("Taylor: h", h, "fd", fd, "g.v", gv, "loss", L)
    assert abs(gv) > 1e-6 * abs(L)  # the direction moves the loss
    assert abs(fd - gv) <= 1e-4 * abs(gv) + 1e-13 * abs(L) / h
