"""FP64 reference gradient of the coupled flow model -- TEST INFRASTRUCTURE.

A differentiable restatement, in PyTorch float64 on the CPU, of the time step
that oracle/dhara_oracle.cc restates (itself following the reference's
SubsurfaceFlowModel, src/subsurface.cu:686-847, and OverlandFlowModel,
src/overland.cu:387-419), for small domains: the linear systems are built
dense and solved exactly, so autograd through the whole run gives the exact
gradient of the discrete map (with the realised Picard iteration counts and
branch decisions held fixed).  Only tests/ use it, as the checker of the GPU
adjoint.

Scope (the adjoint workloads): top flux boundary (the reference's
IdentifyTopBoundary always yields a flux condition), bottom free drainage
(q = K at the bottom cell, src/subsurface.cu:209), no-flux sides, zero ET and
transpiration, reference or conservative theta rollover.

Loss (per run): sum over steps of sum over the top three layers of
(theta^{n+1} - theta_target)^2, plus w_q * sum over steps of
(Q_out - Q_target)^2, where Q_out is the overland flow into the fixed ring
during the step (the implicit flux of the solved elevation across the ring
faces, in metres summed over cells).
"""
import numpy as np
import torch
import torch.nn.functional as F

from dhara_b200 import _abi

T = torch.float64


# ------------------------------------------------------- sparse exact solves
# For domains too large for dense matrices the linear systems are solved by
# preconditioned CG to a relative residual of 1e-14 and differentiated
# implicitly: x = x* + A^-1 (b - A x*) with x* the (detached) solution, whose
# value is x* and whose derivative is A^-1 (db - dA x*) -- the exact-solve
# derivative, because A is symmetric the backward pass is another solve with A.

def _pcg(apply, precond, b, x0, tol, maxiter):
    """Preconditioned CG (no autograd) to ||b - A x|| <= tol ||b||."""
    x = x0.clone()
    r = b - apply(x)
    bn = float(torch.linalg.vector_norm(b))
    if bn == 0.0:
        return torch.zeros_like(b)
    z = precond(r)
    p = z.clone()
    rz = torch.sum(r * z)
    for _ in range(maxiter):
        if float(torch.linalg.vector_norm(r)) <= tol * bn:
            break
        q = apply(p)
        a = rz / torch.sum(p * q)
        x = x + a * p
        r = r - a * q
        z = precond(r)
        rz_n = torch.sum(r * z)
        p = z + (rz_n / rz) * p
        rz = rz_n
    else:
        raise RuntimeError("reference PCG did not reach its tolerance")
    return x


class _ApplyInverse(torch.autograd.Function):
    """y = A^-1 r for a symmetric positive definite A given as a solver;
    the backward pass applies the same solver to the incoming gradient."""

    @staticmethod
    def forward(ctx, r, solver):
        ctx.solver = solver
        return solver(r)

    @staticmethod
    def backward(ctx, g):
        return ctx.solver(g), None


def implicit_solve(matvec, precond, b, x0, tol=1e-14, maxiter=100000):
    """Solution of A x = b with exact-solve derivatives; matvec(v) = A v is
    differentiable in A's coefficients, precond(r) ~ A^-1 r (no autograd)."""
    with torch.no_grad():
        app = lambda v: matvec(v)
        xs = _pcg(app, precond, b.detach(), x0.detach(), tol, maxiter)
    solver = lambda v: _pcg(lambda u: matvec(u).detach(), precond, v.detach(), torch.zeros_like(v), tol, maxiter)
    return xs + _ApplyInverse.apply(b - matvec(xs), solver)


def matvec3(x, Dg, kz, ky, kx):
    """7-point operator D x + sum_f k_f (x_c - x_f) on a [nz, ny, nx] grid,
    zero flux through the domain faces (k* are face coefficients / h^2)."""
    fz = kz * (x[:-1] - x[1:])
    fy = ky * (x[:, :-1] - x[:, 1:])
    fx = kx * (x[:, :, :-1] - x[:, :, 1:])
    return (Dg * x + F.pad(fz, (0, 0, 0, 0, 0, 1)) - F.pad(fz, (0, 0, 0, 0, 1, 0))
            + F.pad(fy, (0, 0, 0, 1)) - F.pad(fy, (0, 0, 1, 0)) + F.pad(fx, (0, 1)) - F.pad(fx, (1, 0)))


def column_preconditioner(Dg, kz, ky, kx):
    """r -> M^-1 r with M the vertical (k) tridiagonal part of the operator."""
    with torch.no_grad():
        dg = (Dg + F.pad(kz, (0, 0, 0, 0, 0, 1)) + F.pad(kz, (0, 0, 0, 0, 1, 0)) + F.pad(ky, (0, 0, 0, 1))
              + F.pad(ky, (0, 0, 1, 0)) + F.pad(kx, (0, 1)) + F.pad(kx, (1, 0)))
        off = -kz
        nz = dg.shape[0]
        den, cp = [dg[0]], []
        for k in range(1, nz):
            cp.append(off[k - 1] / den[k - 1])
            den.append(dg[k] - off[k - 1] * cp[k - 1])

    def apply(r):
        y = [r[0] / den[0]]
        for k in range(1, nz):
            y.append((r[k] - off[k - 1] * y[k - 1]) / den[k])
        for k in range(nz - 2, -1, -1):
            y[k] = y[k] - cp[k] * y[k + 1]
        return torch.stack(y)
    return apply


def closure(psi, ks, alpha_m, n, ts, tr):
    """vanGenuchten (src/global.cu:66-105) with psi in m and alpha in 1/m;
    returns theta, K, C.  Written with safe branches so the saturated cells
    (psi >= 0: theta = theta_s, K = Ks, C = 0) have finite derivatives."""
    a_cm = alpha_m / 100.0
    m = (n - 1.0) / n
    neg = psi < 0
    x = torch.where(neg, a_cm * (-psi * 100.0), torch.ones_like(psi))   # alpha |psi| in the reference's cm
    xn = x ** n
    th_u = (ts - tr) / (1.0 + xn) ** m + tr
    theta = torch.where(neg, th_u, torch.full_like(psi, ts))
    se_u = (th_u - tr) / (ts - tr)
    inner = 1.0 - (1.0 - se_u ** (1.0 / m)) ** m
    K_u = ks * torch.sqrt(se_u) * inner * inner
    K = torch.where(neg, K_u, ks)
    C_u = 100 * a_cm * n * (1.0 / n - 1.0) * x ** (n - 1) * (tr - ts) * (xn + 1) ** (1.0 / n - 2.0)
    C = torch.where(neg, C_u, torch.zeros_like(psi))
    return theta, K, C


class Model:
    """The coupled model on one domain (reference layouts flattened to
    [nz, ny, nx] and [ny, nx] grids).  sparse=False builds the linear systems
    dense and solves them directly (small domains); sparse=True applies them
    as stencils and solves them by PCG to 1e-14 with implicit derivatives, and
    checkpoint=True recomputes each time step in the backward pass instead of
    keeping its graph (the 128x128x30 calibration domain)."""

    def __init__(self, domain, sparse=False, checkpoint=False):
        self.sparse = sparse
        self.checkpoint = checkpoint
        p = domain.params
        self.p = p
        self.nx, self.ny, self.nz = p.nx, p.ny, p.nz
        f = domain.fields
        sh3 = (p.nz, p.ny, p.nx)
        sh2 = (p.ny, p.nx)
        self.psi0 = torch.tensor(f["psi"], dtype=T).reshape(sh3)
        self.z = torch.tensor(f["ztopo"], dtype=T).reshape(sh2)
        self.mann = torch.tensor(f["mann"], dtype=T).reshape(sh2)
        self.h0 = torch.tensor(f["waterdepth"], dtype=T).reshape(sh2)
        self.rain = [float(r) for r in domain.rain_mm]
        self.logks0 = torch.tensor(np.log(f["ksat"]), dtype=T).reshape(sh3)
        self.alpha0 = torch.tensor(f.get("alpha", np.full(p.nx * p.ny * p.nz, p.alpha)), dtype=T).reshape(sh3)
        self.n0 = torch.tensor(f.get("nvg", np.full(p.nx * p.ny * p.nz, p.n)), dtype=T).reshape(sh3)
        ints = domain.int_fields
        assert np.all(ints["bcw"] != 0) and np.all(ints["bce"] != 0) and np.all(ints["bcs"] != 0) \
            and np.all(ints["bcn"] != 0) and np.all(ints["bcb"] != 0), "adjoint scope: no Dirichlet faces"
        assert not np.any(f["esoil"]) and not np.any(f["tr"]), "adjoint scope: zero ET and transpiration"
        self._index()

    def _index(self):
        nz, ny, nx = self.nz, self.ny, self.nx
        N = nz * ny * nx
        idx = np.arange(N).reshape(nz, ny, nx)
        self.N = N
        pairs = []   # (cell, neighbour, axis) for each interior face, once
        for ax in range(3):
            sl_a = [slice(None)] * 3
            sl_b = [slice(None)] * 3
            sl_a[ax] = slice(0, -1)
            sl_b[ax] = slice(1, None)
            a = idx[tuple(sl_a)].ravel()
            b = idx[tuple(sl_b)].ravel()
            pairs.append((torch.tensor(a), torch.tensor(b)))
        self.pairs = pairs   # axis 0: k (z), 1: j (y), 2: i (x)
        C = ny * nx
        idx2 = np.arange(C).reshape(ny, nx)
        ring = np.zeros((ny, nx), bool)
        ring[0, :] = ring[-1, :] = ring[:, 0] = ring[:, -1] = True
        self.ring = torch.tensor(ring.ravel())
        self.C = C

    # ---------------------------------------------------------- subsurface
    def assemble(self, psi_m, psin, thetan, theta_m, K, Cm, qt):
        """Dense A and rhs of SetUpLinearSystemsSubsurface for the scope."""
        p = self.p
        N, nz = self.N, self.nz
        dxs = (p.dz, p.dy, p.dx)
        Kf = K.reshape(-1)
        A = torch.zeros((N, N), dtype=T)
        diag = (p.Ss / p.dt * theta_m / p.porosity + Cm / p.dt).reshape(-1)
        A = A + torch.diag(diag)
        for ax, (a, b) in enumerate(self.pairs):
            kf = 0.5 * (Kf[a] + Kf[b]) / (dxs[ax] ** 2)
            A = A.index_put((a, a), kf, accumulate=True)
            A = A.index_put((b, b), kf, accumulate=True)
            A = A.index_put((a, b), -kf, accumulate=True)
            A = A.index_put((b, a), -kf, accumulate=True)
        return A, self.rhs3(psi_m, psin, thetan, theta_m, K, Cm, qt).reshape(-1)

    def rhs3(self, psi_m, psin, thetan, theta_m, K, Cm, qt):
        """Right-hand side of SetUpLinearSystemsSubsurface for the scope."""
        p = self.p
        nz = self.nz
        # rhs: storage, C psi^m, gravity, theta change
        rhs = (p.Ss / p.dt * theta_m / p.porosity * psin + Cm / p.dt * psi_m + (thetan - theta_m) / p.dt)
        # gravity -(ku - kd)/dz with ku the face below (k+1) and kd the face above (k-1)
        ku = torch.zeros_like(K)
        kd = torch.zeros_like(K)
        ku[:-1] = 0.5 * (K[:-1] + K[1:])
        kd[1:] = 0.5 * (K[1:] + K[:-1])
        rhs = rhs - (ku - kd) / p.dz
        # top flux and bottom free drainage
        top = torch.zeros_like(K)
        top[0] = qt / p.dz
        bot = torch.zeros_like(K)
        bot[nz - 1] = -K[nz - 1] / p.dz
        return rhs + top + bot

    def coeffs3(self, theta_m, K, Cm):
        """Storage diagonal and face coefficients (arithmetic-mean K / h^2)."""
        p = self.p
        Dg = p.Ss / p.dt * theta_m / p.porosity + Cm / p.dt
        kz = 0.5 * (K[:-1] + K[1:]) / (p.dz ** 2)
        ky = 0.5 * (K[:, :-1] + K[:, 1:]) / (p.dy ** 2)
        kx = 0.5 * (K[:, :, :-1] + K[:, :, 1:]) / (p.dx ** 2)
        return Dg, kz, ky, kx

    def prologue(self, ph, psin_top, K_top, ks_top, thetan_top, rain_mm):
        """EstimateFluxes + IdentifyTopBoundary (src/global.cu:172-257) with
        zero ET: hpoten, and the top flux (always a flux condition)."""
        p = self.p
        dt, dz = p.dt, p.dz
        hpoten = ph + rain_mm / 1000.0
        qcapa = -K_top * ((psin_top - hpoten - 0.5 * dz) / (0.5 * dz))
        qcapa = torch.where(ph / dt > ks_top, torch.maximum(qcapa, ks_top), qcapa)
        q = torch.where(hpoten / dt > qcapa, qcapa, hpoten / dt)
        q = torch.minimum(q, (p.theta_s - thetan_top) * dz / dt)
        q = torch.minimum(q, ks_top)
        qt = torch.where(hpoten > 0.0, q, hpoten / dt)
        return hpoten, qt

    def subsurface_step(self, psin, thetan, Kn, ph, rain_mm, ks, al, nv):
        p = self.p
        hpoten, qt = self.prologue(ph, psin[0], Kn[0], ks[0], thetan[0], rain_mm)
        psi_m = psin
        it = 0
        while True:
            theta_m, K_m, C_m = closure(psi_m, ks, al, nv, p.theta_s, p.theta_r)
            if self.sparse:
                co = self.coeffs3(theta_m, K_m, C_m)
                rhs = self.rhs3(psi_m, psin, thetan, theta_m, K_m, C_m, qt)
                pre = column_preconditioner(*[c.detach() for c in co])
                # bind this iteration's coefficients (the backward solve runs later)
                x = implicit_solve(lambda v, co=co: matvec3(v, *co), pre, rhs, psi_m)
            else:
                A, rhs = self.assemble(psi_m, psin, thetan, theta_m, K_m, C_m, qt)
                x = torch.linalg.solve(A, rhs).reshape(psin.shape)
            it += 1
            if p.picard_rule == _abi.PICARD_PSI_ABSOLUTE:
                err = float(torch.max(torch.abs(x - psi_m)).detach())
            elif p.picard_rule == _abi.PICARD_PSI_RELATIVE:
                err = float(torch.max(torch.abs((x - psi_m) / x)).detach())
            else:
                th1, _, _ = closure(x, ks, al, nv, p.theta_s, p.theta_r)
                err = float(torch.max(torch.abs((th1 - theta_m) / th1)).detach())
            if err < p.picard_tol or it >= p.picard_maxiter:
                break
            psi_m = p.am * psi_m + (1 - p.am) * x
        if p.theta_update == _abi.THETA_CONSERVATIVE:
            theta_next = theta_m + C_m * (x - psi_m)
        elif p.theta_update == _abi.THETA_FINAL:
            theta_next, _, _ = closure(x, ks, al, nv, p.theta_s, p.theta_r)
        else:
            theta_next = theta_m
        _, K_next, _ = closure(x, ks, al, nv, p.theta_s, p.theta_r)
        # SubsurfaceEstimateInfiltrationPonding, flux branch (src/subsurface.cu:465-491)
        ph_out = torch.clamp(hpoten - qt * p.dt, min=0.0)
        return x, theta_next, K_next, ph_out, it

    # ------------------------------------------------------------ overland
    def manning(self, H, h):
        """UpdateKOverland (src/overland.cu:193-368) for the interior rows."""
        p = self.p
        dx, dy = p.dx, p.dy
        ny, nx = self.ny, self.nx
        mann = self.mann
        out = {}

        def sh(a, dj, di):
            return a[1 + dj:ny - 1 + dj, 1 + di:nx - 1 + di]

        Hc, hc, mc = sh(H, 0, 0), sh(h, 0, 0), sh(mann, 0, 0)

        def kface(Hnb, hnb, mnb, S):
            hup = torch.where(Hnb > Hc, hnb, hc)
            hav = (hnb + hc) / 2.0
            ok = (hup > p.hmin) & (hav > p.hmin) & (torch.abs(S) > p.delta)
            hav_s = torch.where(ok, hav, torch.ones_like(hav))
            S_s = torch.where(ok, S, torch.ones_like(S))
            k = hav_s ** (5.0 / 3.0) / (0.5 * (mnb + mc) * torch.sqrt(S_s))
            return torch.where(ok, k, torch.full_like(k, p.K0))

        def slope(a, b):
            s2 = a * a + b * b
            pos = s2 > 0
            return torch.where(pos, torch.sqrt(torch.where(pos, s2, torch.ones_like(s2))), torch.zeros_like(s2))

        Sse = slope((sh(H, 0, 1) - Hc) / dx, (sh(H, 1, 1) + sh(H, 1, 0) - sh(H, -1, 1) - sh(H, -1, 0)) / (4 * dy))
        Ssw = slope((Hc - sh(H, 0, -1)) / dx, (sh(H, 1, 0) + sh(H, 1, -1) - sh(H, -1, 0) - sh(H, -1, -1)) / (4 * dy))
        Ssn = slope((sh(H, 1, 0) - Hc) / dy, (sh(H, 1, 1) + sh(H, 0, 1) - sh(H, 1, -1) - sh(H, 0, -1)) / (4 * dx))
        Sss = slope((Hc - sh(H, -1, 0)) / dy, (sh(H, 0, 1) + sh(H, -1, 1) - sh(H, 0, -1) - sh(H, -1, -1)) / (4 * dx))
        out["ke"] = kface(sh(H, 0, 1), sh(h, 0, 1), sh(mann, 0, 1), Sse)
        out["kw"] = kface(sh(H, 0, -1), sh(h, 0, -1), sh(mann, 0, -1), Ssw)
        out["kn"] = kface(sh(H, 1, 0), sh(h, 1, 0), sh(mann, 1, 0), Ssn)
        out["ks"] = kface(sh(H, -1, 0), sh(h, -1, 0), sh(mann, -1, 0), Sss)
        return out

    def overland_step(self, h):
        """Implicit diffusive wave with the fixed ring (src/overland.cu:387-419);
        returns the new depth and the flow into the ring."""
        p = self.p
        ny, nx = self.ny, self.nx
        H = h + self.z
        k = self.manning(H, h)
        cx, cy = p.dt / p.dx ** 2, p.dt / p.dy ** 2
        mi, mj = nx - 2, ny - 2
        n_int = mi * mj
        lid = torch.arange(n_int).reshape(mj, mi)
        A = None if self.sparse else torch.zeros((n_int, n_int), dtype=T)
        cw, ce, cs, cn = cx * k["kw"], cx * k["ke"], cy * k["ks"], cy * k["kn"]
        if not self.sparse:
            A = A + torch.diag((1.0 + cw + ce + cs + cn).reshape(-1))
        b = H[1:-1, 1:-1].clone()
        # neighbours: interior ones into A, ring ones into b
        for coef, dj, di in ((cw, 0, -1), (ce, 0, 1), (cs, -1, 0), (cn, 1, 0)):
            jj, ii = torch.meshgrid(torch.arange(mj), torch.arange(mi), indexing="ij")
            nj, ni = jj + dj, ii + di
            inner = (nj >= 0) & (nj < mj) & (ni >= 0) & (ni < mi)
            rows = lid[jj[inner], ii[inner]]
            cols = lid[nj[inner], ni[inner]]
            if not self.sparse:
                A = A.index_put((rows, cols), -coef[inner], accumulate=True)
            ringv = H[1:-1, 1:-1].new_zeros((mj, mi))
            Hr = H[1 + dj:ny - 1 + dj, 1 + di:nx - 1 + di]
            b = b + torch.where(~inner, coef * Hr, ringv)
        if self.sparse:
            diag = 1.0 + cw + ce + cs + cn

            def mv(v):
                vp = F.pad(v, (1, 1, 1, 1))
                return diag * v - cw * vp[1:-1, :-2] - ce * vp[1:-1, 2:] - cs * vp[:-2, 1:-1] - cn * vp[2:, 1:-1]
            dd = diag.detach()
            x = implicit_solve(mv, lambda r: r / dd, b, H[1:-1, 1:-1])
        else:
            x = torch.linalg.solve(A, b.reshape(-1)).reshape(mj, mi)
        Hn = H.clone()
        Hn = Hn.index_put((torch.arange(1, ny - 1)[:, None].expand(mj, mi), torch.arange(1, nx - 1)[None, :].expand(mj, mi)), x)
        # flow into the ring: implicit flux across the ring faces
        q = (cw[:, 0] * (x[:, 0] - H[1:-1, 0])).sum() + (ce[:, -1] * (x[:, -1] - H[1:-1, -1])).sum() + \
            (cs[0, :] * (x[0, :] - H[0, 1:-1])).sum() + (cn[-1, :] * (x[-1, :] - H[-1, 1:-1])).sum()
        hn = torch.clamp(Hn - self.z, min=0.0)
        return hn, q

    # ----------------------------------------------------------------- run
    def run(self, nsteps, logks=None, alpha=None, n=None, record=False):
        p = self.p
        ks = torch.exp(self.logks0 if logks is None else logks)
        al = self.alpha0 if alpha is None else alpha
        nv = self.n0 if n is None else n
        psin = self.psi0
        thetan, Kn, _ = closure(psin, ks, al, nv, p.theta_s, p.theta_r)
        ph = self.h0
        thetas, qs, iters = [], [], []
        def step(psin, thetan, Kn, ph, ks, al, nv, rain):
            psin, thetan, Kn, ph, it = self.subsurface_step(psin, thetan, Kn, ph, rain, ks, al, nv)
            ph, q = self.overland_step(ph)
            return psin, thetan, Kn, ph, q, torch.tensor(it)

        for t in range(nsteps):
            rain = self.rain[t] if t < len(self.rain) else 0.0
            if self.checkpoint and torch.is_grad_enabled():
                from torch.utils.checkpoint import checkpoint
                psin, thetan, Kn, ph, q, it = checkpoint(step, psin, thetan, Kn, ph, ks, al, nv, rain,
                                                         use_reentrant=False)
            else:
                psin, thetan, Kn, ph, q, it = step(psin, thetan, Kn, ph, ks, al, nv, rain)
            thetas.append(thetan)
            qs.append(q)
            iters.append(int(it))
        return {"theta": thetas, "q": qs, "psi": psin, "ph": ph, "picard_iters": iters}


def loss_of(out, theta_target, q_target, w_q=1.0):
    L = 0.0
    for t, th in enumerate(out["theta"]):
        L = L + torch.sum((th[:3] - theta_target[t][:3]) ** 2)
    for t, q in enumerate(out["q"]):
        L = L + w_q * (q - q_target[t]) ** 2
    return L


def reference_gradient(domain, nsteps, theta_target, q_target, w_q=1.0, sparse=False, checkpoint=False):
    """Loss and its gradient with respect to per-cell log Ks, alpha (1/m) and
    n, each in the reference 3D layout (k*nx*ny + j*nx + i)."""
    m = Model(domain, sparse=sparse, checkpoint=checkpoint)
    lk = m.logks0.clone().requires_grad_(True)
    al = m.alpha0.clone().requires_grad_(True)
    nv = m.n0.clone().requires_grad_(True)
    out = m.run(nsteps, lk, al, nv)
    L = loss_of(out, theta_target, q_target, w_q)
    L.backward()
    return float(L.detach()), lk.grad.reshape(-1).numpy(), al.grad.reshape(-1).numpy(), nv.grad.reshape(-1).numpy(), out


def targets_from(domain, nsteps, logks=None, alpha=None, n=None, sparse=False):
    """theta and Q_out series of a run (used to make a seeded target)."""
    m = Model(domain, sparse=sparse)
    with torch.no_grad():
        out = m.run(nsteps, logks, alpha, n)
    return [t.clone() for t in out["theta"]], [q.clone() for q in out["q"]]
