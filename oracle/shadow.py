"""Step-by-step ("shadowing") comparison of a solver trajectory against the
FP64 oracle -- TEST INFRASTRUCTURE.

Over tens of steps two correct solvers of the reference scheme drift apart
by more than their per-step agreement: the top-boundary switch
(IdentifyTopBoundary, src/global.cu:206-257), the Picard stop test
(src/subsurface.cu:762-789) and the overland depth clip
(src/overland.cu:371-383) are discontinuous, so solver-level differences of
1e-12 are amplified.  Shadowing removes that amplification from the check:
before every step the oracle is given the state the solver under test
starts the step from, it advances one step (SubsurfaceFlowModel +
OverlandFlowModel), and the two end-of-step states are compared.  The
largest one-step error over the whole horizon is then the parity figure.

The state a step starts from (everything the reference's next step reads
that the step itself does not overwrite first):
  psi    psin               src/subsurface.cu:704 (psinp1m <- psin)
  theta  thetan             rhs and top-flux bound, :106-122, global.cu:236-251
  K      knp1m (top layer)  EstimateFluxes' qcapa, src/global.cu:181-186
  ponding ph                EstimateFluxes' hpoten, src/global.cu:181
  waterdepth, waterelev     overland h and the CG warm start, src/overland.cu:394-411
The Krylov warm start psinp1mp1 is the oracle's own previous solution; the
solves run to a relative residual of 1e-12, so the start does not matter.

`solver` is duck-typed: step(n), download(name), synchronize(), diagnostics().
"""
import numpy as np

from . import Oracle, SOLVER_PCG_COLUMN, SOLVER_CG

STATE = ("psi", "theta", "K", "ponding", "waterdepth", "waterelev")
COMPARED = ("psi", "theta", "ponding", "waterelev")


def rel_err(a, b):
    """Norm-wise relative error max|a-b| / max|b| (the absolute error when b is 0)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if b.size else 0.0
    return num / den if den > 0 else num


def shadow(solver, domain, nsteps, oracle_solver3d=SOLVER_PCG_COLUMN, oracle_tol=1e-12,
           oracle_maxiter=20000, rain=None):
    """Advances `solver` nsteps one at a time; before each step the oracle is
    loaded with the solver's state and advanced one step beside it.  Returns
    a dict: per-field arrays of the one-step relative errors, the largest of
    each, and per-step Picard iteration counts of both."""
    p = type(domain.params).from_buffer_copy(domain.params)
    p.precision = 0
    p.krylov_tol = min(p.krylov_tol, oracle_tol)
    p.krylov_maxiter = max(p.krylov_maxiter, oracle_maxiter)
    o = Oracle(p, oracle_solver3d, SOLVER_CG)
    try:
        o.load(domain)
        o.prepare()
        rain = domain.rain_mm if rain is None else rain
        errs = {k: np.zeros(nsteps) for k in COMPARED + ("waterdepth",)}
        pic_s = np.zeros(nsteps, np.int64)
        pic_o = np.zeros(nsteps, np.int64)
        for t in range(nsteps):
            solver.synchronize()
            for k in STATE:
                o.upload(k, solver.download(k))
            o.step(rain[t] if t < len(rain) else 0.0)
            solver.step(1)
            solver.synchronize()
            for k in errs:
                errs[k][t] = rel_err(solver.download(k), o.download(k))
            pic_s[t] = solver.diagnostics()["picard_iters_last"]
            pic_o[t] = o.diagnostics()["picard_iters_last"]
        return {"errors": errs, "max": {k: float(v.max()) for k, v in errs.items()},
                "picard_solver": pic_s, "picard_oracle": pic_o,
                "picard_mismatch_steps": [int(t) for t in np.nonzero(pic_s != pic_o)[0]]}
    finally:
        o.close()


def free_run_drift(domain, nsteps, solver_a, solver_b, tol=1e-12, maxiter=20000, fields=COMPARED):
    """Runs the oracle twice from the same initial state with two different
    Krylov solvers (each a (3D, 2D) pair of oracle solver ids, or a 3D id
    with CG for 2D; the 3D solves to relative residual `tol`) and returns the
    relative differences of the end states: how far the scheme itself
    carries solver-level differences over `nsteps`."""
    out = []
    for sv in (solver_a, solver_b):
        s3, s2 = sv if isinstance(sv, tuple) else (sv, SOLVER_CG)
        p = type(domain.params).from_buffer_copy(domain.params)
        p.precision = 0
        p.krylov_tol = tol
        p.krylov_maxiter = maxiter
        o = Oracle(p, s3, s2)
        try:
            o.load(domain)
            o.prepare()
            for t in range(nsteps):
                o.step(domain.rain_mm[t] if t < len(domain.rain_mm) else 0.0)
            out.append({k: o.download(k) for k in fields})
        finally:
            o.close()
    return {k: rel_err(out[0][k], out[1][k]) for k in fields}
