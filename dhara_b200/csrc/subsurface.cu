// subsurface.cu -- 3D mixed-form Richards kernels (the reference's
// SubsurfaceFlowModel, src/subsurface.cu:686-847, and the kernels it calls).
//
// Kernel map (reference -> here):
//   EstimateFluxes + IdentifyTopBoundary (src/global.cu:172-257)  -> k_prologue
//   vanGenuchten + SetUpLinearSystemsSubsurface (subsurface.cu:381-429)
//     + ModifiedPicardUpdate (450-461)                             -> k_assemble
//   CUSP BiCGSTAB on the DIA matrix (subsurface.cu:750-751)        -> k_krylov
//   GetIterationDifference + max_element (432-446, 762-789)        -> k_picard_check
//   vanGenuchten + SubsurfaceEstimateInfiltrationPonding (465-491)
//     + WaterFluxEstimate + reductions (494-629, 809-826)
//     + state rollover (833-840)                                   -> k_epilogue
//
// The 7-point matrix is never stored: each kernel recomputes the face
// conductivities 0.5*(K_c + K_nb) (arithmetic mean, zero on domain faces,
// HydraulicConductivityAtInterface, subsurface.cu:26-79) from the cell K
// array and applies  (A p)_c = D_c p_c + sum_f w_f k_f (p_c - p_f),
// w = 1/dx^2, 1/dy^2, 1/dz^2,  D = Ss theta/(phi dt) + C/dt, which is the
// reference's DIA row (subsurface.cu:83-102) rearranged.
#include "device_common.cuh"

#include <cstdio>

#define MAX_CYCLES 30

// The closure of the assembled system: FP64 (the reference's expressions)
// unless the domain asks for the FP32 closure.
__device__ __forceinline__ void closure(const DomainDesc &D, double psi, double a, double n, double ks,
                                        double &th, double &K, double &C) {
    if (D.closure_fp32) {
        float Kf, Cf;
        vg_eval<float>(psi, a, n, D.theta_s, D.theta_r, ks, th, Kf, Cf);
        K = (double)Kf;
        C = (double)Cf;
    } else {
        vg_eval<double>(psi, a, n, D.theta_s, D.theta_r, ks, th, K, C);
    }
}

// ------------------------------------------------------------------ init
__global__ void k_psi_from_theta(DevPtrs P) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const double a = D.has_alpha ? P.alpha[g] : D.alpha;
        const double n = D.has_n ? P.nvg[g] : D.n;
        const double m = (n - 1.0) / n;
        const double th = P.thetan[g];
        // vanGenuchtenInverse (src/global.cu:32-52), SI alpha.
        P.psin[g] = (th < D.theta_s)
                        ? -(1.0 / a) * pow(pow((D.theta_s - D.theta_r) / (th - D.theta_r), 1.0 / m) - 1.0,
                                           1.0 / n)
                        : 0.0;
    }
}

// PreRunningFlowModel (src/global.cu:270-296): theta^n, K at psi^n.  The
// Krylov iterate starts from psi^n.
template <typename T>
__global__ void k_prepare(DevPtrs P) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const double a = D.has_alpha ? P.alpha[g] : D.alpha;
        const double n = D.has_n ? P.nvg[g] : D.n;
        double th, Kv, C;
        closure(D, P.psin[g], a, n, P.ksat[g], th, Kv, C);
        P.thetan[g] = th;
        P.K64[g] = Kv;
        if (!std::is_same<T, double>::value) ((T *)P.K)[g] = (T)Kv;
        P.x[g] = P.psin[g];
        P.psim[g] = P.psin[g];
        if (k == 0) P.ktop[cr.c] = Kv;
    }
}

// -------------------------------------------------------------- prologue
// One thread per column: EstimateFluxes (src/global.cu:172-191) and
// IdentifyTopBoundary (206-257).  The top flux does not change between Picard
// iterations (its inputs hpoten, qcapa, theta^n, Ks are fixed for the step), so
// it is evaluated once per step.  Also resets the per-step control state.
__global__ void k_prologue(DevPtrs P) {
    const int tile = blockIdx.x;
    const ColumnRef cr = column_of(P, tile);
    const DomainDesc &D = P.dom[cr.dom];
    const TileDesc td = P.tiles[tile];
    if (threadIdx.x == 0) {
        if (tile == 0) {
            P.gctrl->n_active = 0;
            P.gctrl->n_inner_active = 0;
            P.gctrl->n_olf_active = 0;
        }
        if (tile == D.tile_begin) {
            PicardCtrl &pc = P.pctrl[td.dom];
            pc.iter = 0;
            pc.done = 0;
            pc.converged = 0;
            pc.err = 0.0;
            P.diag[td.dom].krylov_iters_last = 0;
            for (int q = 0; q < 16; ++q) P.step_acc[td.dom * 16 + q] = 0.0;
        }
    }
    if (!cr.valid) return;
    const long long c = cr.c, g = cr.g0;  // top cell k = 0
    const double dt = D.dt, dz = D.dz;
    const int step = P.pctrl[td.dom].step;
    double ppt;
    if (D.sched_len > 0)
        ppt = (step < D.sched_len) ? P.rain_sched[D.sched_off + step] : 0.0;
    else
        ppt = P.ppt[c];
    P.ppt[c] = ppt;
    const double ph = P.ph[c];
    const double hpoten = ph + ppt / 1000 - P.esoil[c] * D.sec * dt;
    const double ks = P.ksat[g];
    double qcapa = -P.ktop[c] * ((P.psin[g] - hpoten - 0.5 * dz) / (0.5 * dz));
    if (ph / dt > ks) qcapa = fmax(qcapa, ks);
    double q;
    if (hpoten > 0.0) {
        q = (hpoten / dt > qcapa) ? qcapa : hpoten / dt;
        q = fmin(q, (D.theta_s - P.thetan[g]) * dz / dt);
        q = fmin(q, ks);
    } else {
        q = hpoten / dt;
    }
    P.hpoten[c] = hpoten;
    P.qtop[c] = q;
}

// -------------------------------------------------------------- assembly
// One thread per column marching k = 0..nz-1 with K of k-1, k, k+1 in
// registers.  For Picard iteration m it forms psi^m (psi^n at m = 0, else the
// reference's relaxation am*psi^m + (1-am)*psi^{m+1}), evaluates the closure
// in T, and writes K (T), the storage diagonal D (T), the right-hand side b
// (double) and psi^m (double).  The right-hand side is
// SetUpRightHandSideSubsurface (src/subsurface.cu:106-122) plus the Neumann
// terms of SetUpBoundaryConditionsSubsurface (126-353) in the reference's
// order top, bottom, south, north, west, east; the bottom is free drainage
// (q_b = K of the bottom cell, written to bcqb as the reference does).
template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_assemble(DevPtrs P) {
    const int tile = blockIdx.x;
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    const PicardCtrl &pc = P.pctrl[td.dom];
    const int done = pc.done;
    const int iter = pc.iter;
    if (threadIdx.x == 0 && tile == D.tile_begin) {
        KrylovCtrl &kc = P.kctrl[td.dom];
        kc.active = done ? 0 : 1;
        kc.inner_active = 0;
        kc.cycles = 0;
        kc.total_iter = 0;
        kc.parity = 0;
        kc.first_inner = 1;
        if (!done) atomicAdd(&P.gctrl->n_active, 1);
    }
    if (done) return;
    const ColumnRef cr = column_of(P, tile);
    if (!cr.valid) return;
    const int nz = cr.nz;
    const double dt = D.dt, dz = D.dz, dx = D.dx, dy = D.dy;
    const double am = D.am;
    const double ssc = D.Ss / dt / D.porosity;
    const double tr_col = P.tr[cr.c];
    const int proc = P.procmap[cr.c];
    const double *root = P.rda + (size_t)cr.dom * P.rda_stride + (size_t)proc * nz;

    auto psi_m_at = [&](long long g) -> double {
        return (iter == 0) ? P.psin[g] : am * P.psim[g] + (1.0 - am) * P.x[g];
    };
    auto eval = [&](long long g, double psi, double &th, double &Kv, double &Cv) {
        const double a = D.has_alpha ? P.alpha[g] : D.alpha;
        const double n = D.has_n ? P.nvg[g] : D.n;
        closure(D, psi, a, n, P.ksat[g], th, Kv, Cv);
    };

    long long g = cr.g0;
    double psi_c = psi_m_at(g);
    double th_c, K_c, C_c;
    eval(g, psi_c, th_c, K_c, C_c);
    double K_up = 0.0;
    for (int k = 0; k < nz; ++k, g += cr.sxy) {
        double psi_n_nb = 0.0, th_n = 0.0, K_n = 0.0, C_n = 0.0;
        if (k + 1 < nz) {
            psi_n_nb = psi_m_at(g + cr.sxy);
            eval(g + cr.sxy, psi_n_nb, th_n, K_n, C_n);
        }
        const double kd = (k == 0) ? 0.0 : 0.5 * (K_c + K_up);
        const double ku = (k == nz - 1) ? 0.0 : 0.5 * (K_c + K_n);
        const double thm = th_c, Cm = C_c;
        double trodz = 0.0;
        if (tr_col > 0) trodz = -tr_col * root[k] * D.sec / dz;
        double rhs = ssc * thm * P.psin[g] + Cm / dt * psi_c - (ku - kd) / dz +
                     (P.thetan[g] - thm) / dt + trodz / dt;
        const double dz2inv = -1.0 / (dz * dz), dy2inv = -1.0 / (dy * dy), dx2inv = -1.0 / (dx * dx);
        if (k == 0) rhs += (-P.qtop[cr.c] * dz) * dz2inv;
        if (k == nz - 1) {
            const double qb = K_c;
            P.bcqb[cr.c] = qb;
            rhs += (qb * dz) * dz2inv;
        }
        const long long bi = D.offWE + (long long)k * cr.ny + cr.j;
        const long long bj = D.offSN + (long long)k * cr.nx + cr.i;
        if (cr.j == 0) rhs += (-P.bcqs[bj] * dy) * dy2inv;
        if (cr.j == cr.ny - 1) rhs += (P.bcqn[bj] * dy) * dy2inv;
        if (cr.i == 0) rhs += (-P.bcqw[bi] * dx) * dx2inv;
        if (cr.i == cr.nx - 1) rhs += (P.bcqe[bi] * dx) * dx2inv;

        const double Dv = ssc * thm + Cm / dt;
        P.psim[g] = psi_c;
        P.K64[g] = K_c;
        P.D64[g] = Dv;
        if (!std::is_same<T, double>::value) {
            ((T *)P.K)[g] = (T)K_c;
            ((T *)P.D)[g] = (T)Dv;
        }
        P.b[g] = rhs;

        K_up = K_c;
        psi_c = psi_n_nb;
        th_c = th_n;
        K_c = K_n;
        C_c = C_n;
    }
}

// ------------------------------------------------------------ Krylov solve
// Persistent cooperative kernel: for every active domain it solves
// A x = b to ||b - A x|| <= tol ||b|| (the CUSP monitor's rule,
// CUSP/detail/monitor.inl:108-111,181-201) by iterative refinement:
//   R: r = b - A x in FP64 arithmetic, r_T = (T) r, z = M^-1 r_T
//   inner PCG in T on A d = r_T, M = the z-line (column) tridiagonal part of A
//   U: x += d
// In FP64 mode T = double and one cycle normally converges (the inner target
// is the outer tolerance).  In mixed mode T = float, the inner solve reduces
// the residual by inner_tol and cycles repeat until the FP64 residual meets
// the tolerance.  The reference runs unpreconditioned BiCGSTAB; any solver
// converged to the same tolerance yields the same head field.
struct KrylovPhaseArgs {
    int nz, i, j, nx, ny;
    long long g0, sxy;
};

template <typename T>
struct StencilW {
    T cx, cy, cz;
};

// Forward Thomas step for the column tridiagonal preconditioner.
template <typename T>
__device__ __forceinline__ void thomas_fwd(T rk, T a, T c, T bd, T &cprev, T &dprev, T *s_c, int k,
                                           T *zg) {
    const T inv = T(1) / (bd - a * cprev);
    const T cp = c * inv;
    const T dp = (rk - a * dprev) * inv;
    s_c[k * TILE_THREADS + threadIdx.x] = cp;
    *zg = dp;
    cprev = cp;
    dprev = dp;
}

template <typename T>
__device__ __forceinline__ double thomas_bwd(const ColumnRef &cr, const T *s_c, T *z, const T *r) {
    T zn = T(0);
    double rz = 0.0;
    long long g = cr.g0 + (long long)(cr.nz - 1) * cr.sxy;
    for (int k = cr.nz - 1; k >= 0; --k, g -= cr.sxy) {
        const T zk = z[g] - s_c[k * TILE_THREADS + threadIdx.x] * zn;
        z[g] = zk;
        zn = zk;
        rz += (double)r[g] * (double)zk;
    }
    return rz;
}

// Lateral face conductivities and neighbour values of vector v at cell g.
template <typename T, typename V, typename Get>
__device__ __forceinline__ void lateral(const ColumnRef &cr, const T *__restrict__ K, long long g,
                                        T Kc, Get get, T &kw, T &ke, T &ks, T &kn, V &vw, V &ve,
                                        V &vs, V &vn) {
    kw = ke = ks = kn = T(0);
    vw = ve = vs = vn = V(0);
    if (cr.i > 0) { kw = T(0.5) * (Kc + __ldg(K + g - 1)); vw = get(g - 1); }
    if (cr.i < cr.nx - 1) { ke = T(0.5) * (Kc + __ldg(K + g + 1)); ve = get(g + 1); }
    if (cr.j > 0) { ks = T(0.5) * (Kc + __ldg(K + g - cr.nx)); vs = get(g - cr.nx); }
    if (cr.j < cr.ny - 1) { kn = T(0.5) * (Kc + __ldg(K + g + cr.nx)); vn = get(g + cr.nx); }
}

// Phase R: FP64 residual with the FP64 coefficients, its cast to T, the
// column solve with the T coefficients of the inner operator (the same
// rounding as the stored K, D), and partial sums v = {||r||^2, ||b||^2, r.z}.
template <typename T>
__device__ void phase_R(const DevPtrs &P, const ColumnRef &cr, const StencilW<T> &w, T *s_c,
                        double (&v)[3]) {
    const double *__restrict__ K = P.K64;
    const double *__restrict__ Dg = P.D64;
    T *r = (T *)P.r, *z = (T *)P.z;
    const double *x = P.x;
    const int nz = cr.nz;
    long long g = cr.g0;
    double x_up = 0.0, x_c = x[g], x_dn = 0.0;
    double K_up = 0.0, K_c = __ldg(K + g), K_dn = 0.0;
    T cprev = T(0), dprev = T(0);
    const double cx = (double)w.cx, cy = (double)w.cy, cz = (double)w.cz;
    for (int k = 0; k < nz; ++k, g += cr.sxy) {
        if (k + 1 < nz) { x_dn = x[g + cr.sxy]; K_dn = __ldg(K + g + cr.sxy); }
        else { x_dn = 0.0; K_dn = 0.0; }
        const double kd = (k > 0) ? 0.5 * (K_c + K_up) : 0.0;
        const double ku = (k < nz - 1) ? 0.5 * (K_c + K_dn) : 0.0;
        double kw, ke, ks, kn, xw, xe, xs, xn;
        lateral<double, double>(cr, K, g, K_c, [&](long long q) { return x[q]; }, kw, ke, ks, kn, xw, xe,
                                xs, xn);
        const double Dk = __ldg(Dg + g);
        const double Ax = Dk * x_c + cx * (kw * (x_c - xw) + ke * (x_c - xe)) +
                          cy * (ks * (x_c - xs) + kn * (x_c - xn)) +
                          cz * (kd * (x_c - x_up) + ku * (x_c - x_dn));
        const double bk = __ldg(P.b + g);
        const double rk = bk - Ax;
        v[0] += rk * rk;
        v[1] += bk * bk;
        const T rT = (T)rk;
        r[g] = rT;
        // inner-operator coefficients: T-rounded cell values, T arithmetic
        const T Kt = (T)K_c;
        const T kdT = (k > 0) ? T(0.5) * (Kt + (T)K_up) : T(0);
        const T kuT = (k < nz - 1) ? T(0.5) * (Kt + (T)K_dn) : T(0);
        const T kwT = cr.i > 0 ? T(0.5) * (Kt + (T)__ldg(K + g - 1)) : T(0);
        const T keT = cr.i < cr.nx - 1 ? T(0.5) * (Kt + (T)__ldg(K + g + 1)) : T(0);
        const T ksT = cr.j > 0 ? T(0.5) * (Kt + (T)__ldg(K + g - cr.nx)) : T(0);
        const T knT = cr.j < cr.ny - 1 ? T(0.5) * (Kt + (T)__ldg(K + g + cr.nx)) : T(0);
        const T bd = (T)Dk + w.cx * (kwT + keT) + w.cy * (ksT + knT) + w.cz * (kdT + kuT);
        thomas_fwd<T>(rT, -w.cz * kdT, -w.cz * kuT, bd, cprev, dprev, s_c, k, z + g);
        x_up = x_c; x_c = x_dn; K_up = K_c; K_c = K_dn;
    }
    v[2] += thomas_bwd<T>(cr, s_c, z, r);
}

// Phase A: p_new = z + beta p_old (recomputed at the halo, double-buffered p),
// partial p.Ap.
template <typename T>
__device__ void phase_A(const DevPtrs &P, const ColumnRef &cr, const StencilW<T> &w, T beta,
                        bool first, const T *pold, T *pnew, double (&v)[1]) {
    const T *__restrict__ K = (const T *)P.K;
    const T *__restrict__ Dg = (const T *)P.D;
    const T *z = (const T *)P.z;
    const int nz = cr.nz;
    auto pv = [&](long long q) -> T { return first ? z[q] : z[q] + beta * pold[q]; };
    long long g = cr.g0;
    T p_up = T(0), p_c = pv(g), p_dn = T(0);
    T K_up = T(0), K_c = __ldg(K + g), K_dn = T(0);
    for (int k = 0; k < nz; ++k, g += cr.sxy) {
        if (k + 1 < nz) { p_dn = pv(g + cr.sxy); K_dn = __ldg(K + g + cr.sxy); }
        else { p_dn = T(0); K_dn = T(0); }
        const T kd = (k > 0) ? T(0.5) * (K_c + K_up) : T(0);
        const T ku = (k < nz - 1) ? T(0.5) * (K_c + K_dn) : T(0);
        T kw, ke, ks, kn, pw, pe, ps, pn;
        lateral<T, T>(cr, K, g, K_c, pv, kw, ke, ks, kn, pw, pe, ps, pn);
        const T Ap = __ldg(Dg + g) * p_c + w.cx * (kw * (p_c - pw) + ke * (p_c - pe)) +
                     w.cy * (ks * (p_c - ps) + kn * (p_c - pn)) +
                     w.cz * (kd * (p_c - p_up) + ku * (p_c - p_dn));
        v[0] += (double)p_c * (double)Ap;
        pnew[g] = p_c;
        p_up = p_c; p_c = p_dn; K_up = K_c; K_c = K_dn;
    }
}

// Phase B: d += alpha p, r -= alpha A p (A p recomputed), z = M^-1 r,
// partials {||r||^2, r.z}.
template <typename T>
__device__ void phase_B(const DevPtrs &P, const ColumnRef &cr, const StencilW<T> &w, T alpha,
                        bool first, const T *p, T *s_c, double (&v)[2]) {
    const T *__restrict__ K = (const T *)P.K;
    const T *__restrict__ Dg = (const T *)P.D;
    T *r = (T *)P.r, *z = (T *)P.z, *d = (T *)P.d;
    const int nz = cr.nz;
    long long g = cr.g0;
    T p_up = T(0), p_c = p[g], p_dn = T(0);
    T K_up = T(0), K_c = __ldg(K + g), K_dn = T(0);
    T cprev = T(0), dprev = T(0);
    for (int k = 0; k < nz; ++k, g += cr.sxy) {
        if (k + 1 < nz) { p_dn = p[g + cr.sxy]; K_dn = __ldg(K + g + cr.sxy); }
        else { p_dn = T(0); K_dn = T(0); }
        const T kd = (k > 0) ? T(0.5) * (K_c + K_up) : T(0);
        const T ku = (k < nz - 1) ? T(0.5) * (K_c + K_dn) : T(0);
        T kw, ke, ks, kn, pw, pe, ps, pn;
        lateral<T, T>(cr, K, g, K_c, [&](long long q) { return p[q]; }, kw, ke, ks, kn, pw, pe, ps, pn);
        const T Dk = __ldg(Dg + g);
        const T Ap = Dk * p_c + w.cx * (kw * (p_c - pw) + ke * (p_c - pe)) +
                     w.cy * (ks * (p_c - ps) + kn * (p_c - pn)) +
                     w.cz * (kd * (p_c - p_up) + ku * (p_c - p_dn));
        d[g] = first ? alpha * p_c : d[g] + alpha * p_c;
        const T rk = r[g] - alpha * Ap;
        r[g] = rk;
        v[0] += (double)rk * (double)rk;
        const T bd = Dk + w.cx * (kw + ke) + w.cy * (ks + kn) + w.cz * (kd + ku);
        thomas_fwd<T>(rk, -w.cz * kd, -w.cz * ku, bd, cprev, dprev, s_c, k, z + g);
        p_up = p_c; p_c = p_dn; K_up = K_c; K_c = K_dn;
    }
    v[1] += thomas_bwd<T>(cr, s_c, z, r);
}

__device__ __forceinline__ void finalize_R(const DevPtrs &P, int dom, const double (&v)[3]) {
    KrylovCtrl &c = P.kctrl[dom];
    const DomainDesc &D = P.dom[dom];
    const double rr64 = v[0], bb = v[1];
    c.bb = bb;
    c.rr64 = rr64;
    c.cycles += 1;
    const double tol2 = D.krylov_tol * D.krylov_tol;
    const bool conv = rr64 <= tol2 * bb;
    const bool bad = !(rr64 == rr64) || !(bb == bb) || isinf(rr64);
    if (conv || bad || c.total_iter >= D.krylov_maxiter || c.cycles > MAX_CYCLES) {
        c.active = 0;
        atomicSub(&P.gctrl->n_active, 1);
        DevDiag &dg = P.diag[dom];
        if (!conv) dg.krylov_nonconverged += 1;
        if (bad) dg.nonfinite = 1;
        dg.krylov_relres_last = bb > 0 ? sqrt(rr64 / bb) : sqrt(rr64);
    } else {
        c.inner_active = 1;
        atomicAdd(&P.gctrl->n_inner_active, 1);
        c.inner_iter = 0;
        c.first_inner = 1;
        c.rz = v[2];
        c.beta = 0.0;
        c.inner_target2 = fmax(D.inner_tol * D.inner_tol * rr64, 0.25 * tol2 * bb);
    }
}

__device__ __forceinline__ void stop_inner(const DevPtrs &P, KrylovCtrl &c) {
    c.inner_active = 0;
    atomicSub(&P.gctrl->n_inner_active, 1);
}

template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_krylov(DevPtrs P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s_c = reinterpret_cast<T *>(smem_raw);
    for (;;) {
        // ---- R: outer residual
        for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
            const int dom = P.tiles[t].dom;
            if (!ldcg(&P.kctrl[dom].active)) continue;
            const ColumnRef cr = column_of(P, t);
            const DomainDesc &D = P.dom[dom];
            const StencilW<T> w = {(T)(1.0 / (D.dx * D.dx)), (T)(1.0 / (D.dy * D.dy)),
                                   (T)(1.0 / (D.dz * D.dz))};
            double v[3] = {0.0, 0.0, 0.0};
            if (cr.valid) phase_R<T>(P, cr, w, s_c, v);
            if (domain_reduce<3>(P, t, dom, 0, v) && threadIdx.x == 0) finalize_R(P, dom, v);
        }
        if (!grid_sync(P.barrier)) return;
        if (ldcg(&P.gctrl->n_active) == 0) break;
        // ---- inner PCG
        while (ldcg(&P.gctrl->n_inner_active) > 0) {
            for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
                const int dom = P.tiles[t].dom;
                const KrylovCtrl *kc = &P.kctrl[dom];
                if (!ldcg(&kc->inner_active)) continue;
                const ColumnRef cr = column_of(P, t);
                const DomainDesc &D = P.dom[dom];
                const StencilW<T> w = {(T)(1.0 / (D.dx * D.dx)), (T)(1.0 / (D.dy * D.dy)),
                                       (T)(1.0 / (D.dz * D.dz))};
                const int parity = ldcg(&kc->parity);
                const bool first = ldcg(&kc->first_inner) != 0;
                const T beta = (T)ldcg(&kc->beta);
                const T *pold = (const T *)(parity ? P.p1 : P.p0);
                T *pnew = (T *)(parity ? P.p0 : P.p1);
                double v[1] = {0.0};
                if (cr.valid) phase_A<T>(P, cr, w, beta, first, pold, pnew, v);
                if (domain_reduce<1>(P, t, dom, 0, v) && threadIdx.x == 0) {
                    KrylovCtrl &c = P.kctrl[dom];
                    c.pAp = v[0];
                    c.alpha = c.rz / v[0];
                    c.parity ^= 1;
                    if (!(v[0] > 0.0) || isinf(v[0])) stop_inner(P, c);
                }
            }
            if (!grid_sync(P.barrier)) return;
            for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
                const int dom = P.tiles[t].dom;
                const KrylovCtrl *kc = &P.kctrl[dom];
                if (!ldcg(&kc->inner_active)) continue;
                const ColumnRef cr = column_of(P, t);
                const DomainDesc &D = P.dom[dom];
                const StencilW<T> w = {(T)(1.0 / (D.dx * D.dx)), (T)(1.0 / (D.dy * D.dy)),
                                       (T)(1.0 / (D.dz * D.dz))};
                const int parity = ldcg(&kc->parity);
                const bool first = ldcg(&kc->first_inner) != 0;
                const T alpha = (T)ldcg(&kc->alpha);
                const T *p = (const T *)(parity ? P.p1 : P.p0);
                double v[2] = {0.0, 0.0};
                if (cr.valid) phase_B<T>(P, cr, w, alpha, first, p, s_c, v);
                if (domain_reduce<2>(P, t, dom, 0, v) && threadIdx.x == 0) {
                    KrylovCtrl &c = P.kctrl[dom];
                    c.rr = v[0];
                    c.beta = v[1] / c.rz;
                    c.rz = v[1];
                    c.first_inner = 0;
                    c.inner_iter += 1;
                    c.total_iter += 1;
                    if (v[0] <= c.inner_target2 || c.inner_iter >= D.inner_maxiter ||
                        c.total_iter >= D.krylov_maxiter || !(v[0] == v[0]) || !(v[1] == v[1]))
                        stop_inner(P, c);
                }
            }
            if (!grid_sync(P.barrier)) return;
        }
        // ---- U: x += d
        for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
            const int dom = P.tiles[t].dom;
            const KrylovCtrl *kc = &P.kctrl[dom];
            if (!ldcg(&kc->active) || ldcg(&kc->first_inner)) continue;
            const ColumnRef cr = column_of(P, t);
            if (!cr.valid) continue;
            const T *d = (const T *)P.d;
            long long g = cr.g0;
            for (int k = 0; k < cr.nz; ++k, g += cr.sxy) P.x[g] += (double)d[g];
        }
        if (!grid_sync(P.barrier)) return;
    }
}

// ---------------------------------------------------------- Picard check
// Max of |(psi^{m+1}-psi^m)/psi^{m+1}| (or the theta / absolute variants) per
// domain, then the convergence decision and iteration bookkeeping.
__global__ void __launch_bounds__(TILE_THREADS) k_picard_check(DevPtrs P) {
    const int tile = blockIdx.x;
    const TileDesc td = P.tiles[tile];
    if (tile == 0 && threadIdx.x == 0) {
        P.gctrl->n_active = 0;
        P.gctrl->n_inner_active = 0;
    }
    const PicardCtrl &pc = P.pctrl[td.dom];
    if (pc.done) return;
    const DomainDesc &D = P.dom[td.dom];
    const ColumnRef cr = column_of(P, tile);
    double mx = 0.0;
    int nonfinite = 0;
    if (cr.valid) {
        long long g = cr.g0;
        for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
            const double xn = P.x[g], xm = P.psim[g];
            double d;
            if (D.picard_rule == DHARA_PICARD_THETA_RELATIVE) {
                const double a = D.has_alpha ? P.alpha[g] : D.alpha;
                const double n = D.has_n ? P.nvg[g] : D.n;
                const double t1 = vg_theta(xn, a, n, D.theta_s, D.theta_r);
                const double t0 = vg_theta(xm, a, n, D.theta_s, D.theta_r);
                d = fabs((t1 - t0) / t1);
            } else if (D.picard_rule == DHARA_PICARD_PSI_ABSOLUTE) {
                d = fabs(xn - xm);
            } else {
                d = fabs((xn - xm) / xn);
            }
            if (!(d == d)) { nonfinite = 1; d = INFINITY; }
            mx = fmax(mx, d);
        }
    }
    if (nonfinite) atomicOr(&P.diag[td.dom].nonfinite, 1);
    double v[1] = {mx};
    if (domain_reduce<1, true>(P, tile, td.dom, 1, v) && threadIdx.x == 0) {
        PicardCtrl &c = P.pctrl[td.dom];
        DevDiag &dg = P.diag[td.dom];
        const KrylovCtrl &kc = P.kctrl[td.dom];
        c.err = v[0];
        c.iter += 1;
        c.converged = v[0] < D.picard_tol;
        c.done = c.converged || c.iter >= D.picard_maxiter;
        dg.krylov_iters_total += kc.total_iter;
        dg.refine_iters_total += kc.cycles;
        dg.krylov_iters_last += kc.total_iter;
        dg.picard_err_last = v[0];
    }
}

// -------------------------------------------------------------- epilogue
// Per column after the Picard loop: closure at psi^{m+1} (the reference's
// second vanGenuchten call) and at psi^m (theta^m, C^m of the last assembly,
// recomputed bitwise-identically), infiltration and ponding
// (SubsurfaceEstimateInfiltrationPonding, src/subsurface.cu:465-491), the
// water balance of WaterFluxEstimate + the nine reductions (494-629,
// 809-826) and the rollover (833-840).  Interior face fluxes of the
// reference's balance cancel pairwise (q_e of cell i equals q_w of cell i+1
// bit for bit), so only boundary faces are summed.
template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_epilogue(DevPtrs P) {
    const int tile = blockIdx.x;
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    const ColumnRef cr = column_of(P, tile);
    // v: 0 sum dtheta*dz, 1 dt*sum ssflux, 2 sum transp, 3 dt*boundary flux,
    //    4 storage (telescoping), 5 dt*q_top, 6 dt*q_bottom, 7 rain, 8 nonfinite
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (cr.valid) {
        const double dt = D.dt, dz = D.dz;
        const double ssc = D.Ss / dt / D.porosity;
        const double tr_col = P.tr[cr.c];
        const int proc = P.procmap[cr.c];
        const double *root = P.rda + (size_t)cr.dom * P.rda_stride + (size_t)proc * cr.nz;
        const int upd = D.theta_update;
        long long g = cr.g0;
        for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
            const double a = D.has_alpha ? P.alpha[g] : D.alpha;
            const double n = D.has_n ? P.nvg[g] : D.n;
            const double ks = P.ksat[g];
            const double xn = P.x[g], xm = P.psim[g], psin = P.psin[g], thn = P.thetan[g];
            double th1, th0, K1, C1, K0, C0;
            closure(D, xn, a, n, ks, th1, K1, C1);
            closure(D, xm, a, n, ks, th0, K0, C0);
            const double thp1 = th1, thm = th0, Cm = C0;
            v[0] += (thp1 - thn) * dz;
            v[1] += (xn - psin) * (D.Ss / dt * thp1 / D.porosity) * dz * dt;
            if (tr_col > 0) v[2] += -tr_col * D.sec * root[k];
            double th_next;
            if (upd == DHARA_THETA_FINAL) th_next = thp1;
            else if (upd == DHARA_THETA_CONSERVATIVE) th_next = thm + Cm * (xn - xm);
            else th_next = thm;
            v[4] += dz * (th_next - thn) + dz * ssc * dt * thm * (xn - psin);
            if (!(xn == xn)) v[8] = 1.0;
            // boundary faces (Neumann values; bottom/top below)
            double fb = 0.0;
            if (cr.i == cr.nx - 1) fb += P.bcqe[D.offWE + (long long)k * cr.ny + cr.j];
            if (cr.i == 0) fb -= P.bcqw[D.offWE + (long long)k * cr.ny + cr.j];
            if (cr.j == cr.ny - 1) fb += P.bcqn[D.offSN + (long long)k * cr.nx + cr.i];
            if (cr.j == 0) fb -= P.bcqs[D.offSN + (long long)k * cr.nx + cr.i];
            v[3] += fb * dt;
            P.psin[g] = xn;
            P.thetan[g] = th_next;
            P.K64[g] = K1;
            if (k == 0) P.ktop[cr.c] = K1;
        }
        const double qt = P.qtop[cr.c], qb = P.bcqb[cr.c];
        v[3] += (qb - qt) * dt;
        v[5] += qt * dt;
        v[6] += qb * dt;
        v[7] += P.ppt[cr.c] / 1000.0;
        // infiltration / ponding, then waterdepth <- ph
        const double ph = fmax(P.hpoten[cr.c] - qt * dt, 0.0);
        P.ph[cr.c] = ph;
        P.h[cr.c] = ph;
    }
    if (domain_reduce<9>(P, tile, td.dom, 2, v) && threadIdx.x == 0) {
        DevDiag &dg = P.diag[td.dom];
        PicardCtrl &pc = P.pctrl[td.dom];
        const double mb = v[0] + v[3] - v[2] + v[1];
        dg.mb_last = mb;
        dg.mb_cum += mb;
        dg.storage_cum += v[4];
        dg.top_cum += v[5];
        dg.bottom_cum += v[6];
        dg.rain_cum += v[7];
        if (v[8] != 0.0) dg.nonfinite = 1;
        dg.picard_iters_total += pc.iter;
        dg.picard_iters_last = pc.iter;
        if (!pc.converged) dg.picard_nonconverged += 1;
        pc.step += 1;
    }
}

// Evaluates the closure at psi^n into out: which = 0 theta, 1 K, 2 C.
__global__ void k_eval_fields(DevPtrs P, int which, double *out) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const double a = D.has_alpha ? P.alpha[g] : D.alpha;
        const double n = D.has_n ? P.nvg[g] : D.n;
        double th, Kv, C;
        vg_eval<double>(P.psin[g], a, n, D.theta_s, D.theta_r, P.ksat[g], th, Kv, C);
        out[g] = which == 0 ? th : (which == 1 ? Kv : C);
    }
}

// ------------------------------------------------------------- launchers
cudaError_t launch_psi_from_theta(const DevPtrs &P, cudaStream_t s) {
    k_psi_from_theta<<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_prologue(const DevPtrs &P, cudaStream_t s) {
    k_prologue<<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_picard_check(const DevPtrs &P, cudaStream_t s) {
    k_picard_check<<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_eval_fields(const DevPtrs &P, int which, double *out, cudaStream_t s) {
    k_eval_fields<<<P.ntiles, TILE_THREADS, 0, s>>>(P, which, out);
    return cudaGetLastError();
}

// The following depend on the inner precision.
cudaError_t launch_prepare(const DevPtrs &P, int mixed, cudaStream_t s) {
    if (mixed) k_prepare<float><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    else k_prepare<double><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_assemble(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s) {
    if (L.mixed) k_assemble<float><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    else k_assemble<double><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_epilogue(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s) {
    if (L.mixed) k_epilogue<float><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    else k_epilogue<double><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_krylov(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s) {
    DevPtrs args = P;
    void *kargs[] = {&args};
    const int grid = L.coop_blocks_3d < P.ntiles ? L.coop_blocks_3d : P.ntiles;
    if (L.mixed)
        return cudaLaunchCooperativeKernel((const void *)k_krylov<float>, dim3(grid), dim3(TILE_THREADS),
                                           kargs, (size_t)L.smem_3d, s);
    return cudaLaunchCooperativeKernel((const void *)k_krylov<double>, dim3(grid), dim3(TILE_THREADS),
                                       kargs, (size_t)L.smem_3d, s);
}

cudaError_t configure_3d(LaunchCfg &L, int device, int ntiles) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    const size_t elt = L.mixed ? sizeof(float) : sizeof(double);
    L.smem_3d = (int)(elt * (size_t)L.nz_max * TILE_THREADS);
    const void *fn = L.mixed ? (const void *)k_krylov<float> : (const void *)k_krylov<double>;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, L.smem_3d);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, TILE_THREADS, L.smem_3d);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    L.coop_blocks_3d = per_sm * prop.multiProcessorCount;
    (void)ntiles;
    return cudaSuccess;
}
