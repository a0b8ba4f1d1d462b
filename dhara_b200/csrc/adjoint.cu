// adjoint.cu -- discrete adjoint (reverse mode) of the coupled time step.
//
// The forward map of one step is the reference's sequence (src/subsurface.cu:
// 686-847 then src/overland.cu:387-419):
//   prologue   hpoten, top flux qt from ph, psi^n_top, K(psi^n)_top, Ks, theta^n
//   Picard m   closure at psi^m -> A_m(theta^m, C^m, K^m), b_m; x^m = A_m^-1 b_m;
//              psi^{m+1} = am psi^m + (1 - am) x^m
//   epilogue   psi^{n+1} = x^{M-1}, theta^{n+1} (reference / final / conservative
//              rollover), K(psi^{n+1})_top, ph = max(hpoten - qt dt, 0)
//   overland   H = ph + z, Manning K(H, ph), (I + dt L_K) H' = H with the fixed
//              ring, h' = max(H' - z, 0), Q = flow into the ring
// Its adjoint runs these in reverse.  Each linear solve is reversed by one solve
// with the same matrix (both are symmetric), done by the forward solvers
// themselves (k_krylov, k_olf_pcg) on the adjoint right-hand side; everything
// else is pointwise or a stencil and lives here.  Picard iteration counts and
// every branch of the forward (top-flux selection, depth clip, Manning's wet
// test) are those of the recorded forward run.
//
// Closure derivatives are written from the van Genuchten-Mualem expressions
// with x = alpha |psi|, u = 1 + x^n, m = 1 - 1/n, Se = u^-m:
//   theta = tr + (ts - tr) Se,  C = dtheta/dpsi = (ts - tr)(n - 1) alpha x^(n-1) u^(-m-1)
//   K = Ks Se^(1/2) (1 - w)^2 with w = (1 - 1/u)^m = x^(n-1) Se.
#include "device_common.cuh"

struct VGD {
    double th, K, C;
    double C_psi, K_psi;   // dC/dpsi, dK/dpsi (dtheta/dpsi = C)
    double th_a, C_a, K_a; // d/dalpha (alpha in 1/m)
    double th_n, C_n, K_n; // d/dn
};

__device__ __forceinline__ VGD vg_derivs(double psi, double a, double n, double ts, double tr, double ks) {
    VGD r;
    double th, K, C;
    vg_eval<double>(psi, a, n, ts, tr, ks, th, K, C);
    r.th = th;
    r.K = K;
    r.C = C;
    r.C_psi = r.K_psi = r.th_a = r.C_a = r.K_a = r.th_n = r.C_n = r.K_n = 0.0;
    if (!(psi < 0.0)) return r;  // saturated: theta_s, Ks, 0
    const double x = a * (-psi);
    const double m = 1.0 - 1.0 / n;
    const double dth = ts - tr;
    const double lx = log(x);
    const double xn1 = exp((n - 1.0) * lx);
    const double xn = xn1 * x;
    const double xn2 = xn1 / x;
    const double u = 1.0 + xn;
    const double lu = log1p(xn);
    const double Se = exp(-m * lu);
    const double um1 = Se / u;
    const double um2 = um1 / u;
    const double dSe_dx = -(n - 1.0) * xn1 * um1;
    const double c0 = dth * (n - 1.0) * xn1 * um1;  // C / alpha
    const double dc0_dx = dth * (n - 1.0) * ((n - 1.0) * xn2 * um1 - (m + 1.0) * n * xn1 * xn1 * um2);
    r.C_psi = -a * a * dc0_dx;
    r.th_a = dth * dSe_dx * (x / a);
    r.C_a = c0 + dc0_dx * x;
    const double w = xn1 * Se;
    const double dw_dx = (n - 1.0) * xn2 * Se + xn1 * dSe_dx;
    const double sSe = sqrt(Se);
    const double omw = 1.0 - w;
    const double dK_dx = ks * (0.5 / sSe * dSe_dx * omw * omw - 2.0 * sSe * omw * dw_dx);
    r.K_psi = -a * dK_dx;
    r.K_a = dK_dx * (x / a);
    const double dm_dn = 1.0 / (n * n);
    const double du_dn = xn * lx;
    const double dlnSe_dn = -dm_dn * lu - m * du_dn / u;
    const double dSe_dn = Se * dlnSe_dn;
    r.th_n = dth * dSe_dn;
    r.C_n = C * (1.0 / (n - 1.0) + lx - dm_dn * lu - (m + 1.0) * du_dn / u);
    const double dw_dn = w * (lx + dlnSe_dn);
    r.K_n = ks * (0.5 / sSe * dSe_dn * omw * omw - 2.0 * sSe * omw * dw_dn);
    return r;
}

__device__ __forceinline__ double cell_alpha(const DevPtrs &P, const DomainDesc &D, long long g) {
    return D.has_alpha ? P.alpha[g] : D.alpha;
}
__device__ __forceinline__ double cell_n(const DevPtrs &P, const DomainDesc &D, long long g) {
    return D.has_n ? P.nvg[g] : D.n;
}

__device__ __forceinline__ bool on_ring(int i, int j, int nx, int ny) {
    return i == 0 || j == 0 || i == nx - 1 || j == ny - 1;
}

__device__ __forceinline__ double adj_qbar(const AdjPtrs &A, int t) {
    return 2.0 * A.w_q * (A.qhist[t] - A.q_target[t]);
}

// ------------------------------------------------------------------ loss
// After forward step t: the theta misfit of the top three layers and the
// discharge misfit (seed_slot < 0), or the theta seeds 2 (theta - target) of
// the tape slot (seed_slot >= 0).
__global__ void __launch_bounds__(TILE_THREADS) k_adj_loss(DevPtrs P, AdjPtrs A, int t, int seed_slot) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    const DomainDesc &D = P.dom[cr.dom];
    double v[1] = {0.0};
    if (cr.valid) {
        const long long cl = cr.c - D.off2;
        const long long C = (long long)D.nx * D.ny;
        const int nk = cr.nz < 3 ? cr.nz : 3;
        for (int k = 0; k < nk; ++k) {
            const double th = P.thetan[cr.g0 + k * cr.sxy];
            const double d = th - A.theta_target[((long long)t * 3 + k) * C + cl];
            if (seed_slot >= 0)
                A.t_thseed[((long long)seed_slot * 3 + k) * A.nc + cr.c] = 2.0 * d;
            else
                v[0] += d * d;
        }
    }
    if (seed_slot >= 0) return;
    block_sum<1>(v);
    if (threadIdx.x == 0) {
        double add = v[0];
        if (blockIdx.x == 0) {
            const double out = P.diag[0].olf_out_cum;
            const double q = out - A.q_prev[0];
            A.q_prev[0] = out;
            A.qhist[t] = q;
            const double dq = q - A.q_target[t];
            add += A.w_q * dq * dq;
        }
        atomicAdd(A.loss, add);
    }
}

// --------------------------------------------------------------- overland
// Right-hand side of the adjoint overland solve: dL/dH' on the interior rows
// (the clipped depth passes its adjoint where H' > z; Q adds its ring-face
// coefficients).  The solve starts from zero with a zero ring.
__global__ void __launch_bounds__(TILE_THREADS) k_adj_olf_rhs(DevPtrs P, AdjPtrs A, int t, long long ctot) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    const long long c = cr.c;
    A.olf_Hbar[c] = 0.0;
    A.olf_hbar[c] = 0.0;
    P.H[c] = 0.0;
    if (on_ring(cr.i, cr.j, cr.nx, cr.ny)) {
        P.olf_b[c] = 0.0;
        return;
    }
    const double qbar = adj_qbar(A, t);
    const double cx = D.dt / (D.dx * D.dx), cy = D.dt / (D.dy * D.dy);
    const double x = A.t_hsol[(long long)A.step_in_seg * A.nc + c];
    double g = (x - P.ztopo[c] > 0.0) ? A.phbar[c] : 0.0;
    if (cr.i == 1) g += qbar * cx * P.olf_k[0 * ctot + c];
    if (cr.i == cr.nx - 2) g += qbar * cx * P.olf_k[1 * ctot + c];
    if (cr.j == 1) g += qbar * cy * P.olf_k[2 * ctot + c];
    if (cr.j == cr.ny - 2) g += qbar * cy * P.olf_k[3 * ctot + c];
    P.olf_b[c] = g;
}

// Adjoint of the interior rows' coefficients (row-owned kw, ke, ks, kn) and of
// the pre-solve elevation, chained through UpdateKOverland's Manning
// conductance (src/overland.cu:193-368) into dL/dH and dL/dh (atomics: each
// face's conductance depends on up to six elevations and two depths).
__global__ void __launch_bounds__(TILE_THREADS) k_adj_olf_coef(DevPtrs P, AdjPtrs A, int t, long long ctot) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid || on_ring(cr.i, cr.j, cr.nx, cr.ny)) return;
    const DomainDesc &D = P.dom[cr.dom];
    const int N = cr.nx;
    const long long I = cr.c;
    const double qbar = adj_qbar(A, t);
    const double cx = D.dt / (D.dx * D.dx), cy = D.dt / (D.dy * D.dy);
    const double *hsol = A.t_hsol + (long long)A.step_in_seg * A.nc;
    const double mu = P.H[I];
    const double xa = hsol[I];
    auto Hs = [&](long long q) { return P.h[q] + P.ztopo[q]; };
    atomicAdd(&A.olf_Hbar[I], mu);  // b_a = H_a
    const double dx = D.dx, dy = D.dy;
    // faces: 0 W, 1 E, 2 S, 3 N
    const long long nbs[4] = {I - 1, I + 1, I - N, I + N};
    const int nbi[4] = {cr.i - 1, cr.i + 1, cr.i, cr.i};
    const int nbj[4] = {cr.j, cr.j, cr.j - 1, cr.j + 1};
    const double Hc = Hs(I), hc = P.h[I], mc = P.mann[I];
    for (int f = 0; f < 4; ++f) {
        const long long nb = nbs[f];
        const double sc = (f < 2) ? cx : cy;
        const double kf = P.olf_k[(long long)f * ctot + I];
        const double coef = sc * kf;
        const bool ring_nb = on_ring(nbi[f], nbj[f], cr.nx, cr.ny);
        const double Hnb = Hs(nb);
        const double Xnb = ring_nb ? Hnb : hsol[nb];
        double cbar = mu * (Xnb - xa);
        if (ring_nb) {
            cbar += qbar * (xa - Hnb);
            atomicAdd(&A.olf_Hbar[nb], mu * coef - qbar * coef);
        }
        const double kbar = cbar * sc;
        // Manning conductance of this face (the forward's expression)
        const double hnb = P.h[nb], mnb = P.mann[nb];
        double Ac, Bc;
        long long hA0, hA1, hB[4];
        double sA, sB;
        if (f == 0) {        // W: (Hc - H_{i-1})/dx, (H_{j+1} + H_{i-1,j+1} - H_{j-1} - H_{i-1,j-1})/(4dy)
            Ac = (Hc - Hs(I - 1)) / dx;
            Bc = (Hs(I + N) + Hs(I + N - 1) - Hs(I - N) - Hs(I - N - 1)) / (4 * dy);
            hA0 = I; hA1 = I - 1; sA = 1.0 / dx;
            hB[0] = I + N; hB[1] = I + N - 1; hB[2] = I - N; hB[3] = I - N - 1; sB = 1.0 / (4 * dy);
        } else if (f == 1) { // E: (H_{i+1} - Hc)/dx, (H_{i+1,j+1} + H_{j+1} - H_{i+1,j-1} - H_{j-1})/(4dy)
            Ac = (Hs(I + 1) - Hc) / dx;
            Bc = (Hs(I + N + 1) + Hs(I + N) - Hs(I - N + 1) - Hs(I - N)) / (4 * dy);
            hA0 = I + 1; hA1 = I; sA = 1.0 / dx;
            hB[0] = I + N + 1; hB[1] = I + N; hB[2] = I - N + 1; hB[3] = I - N; sB = 1.0 / (4 * dy);
        } else if (f == 2) { // S: (Hc - H_{j-1})/dy, (H_{i+1} + H_{i+1,j-1} - H_{i-1} - H_{i-1,j-1})/(4dx)
            Ac = (Hc - Hs(I - N)) / dy;
            Bc = (Hs(I + 1) + Hs(I - N + 1) - Hs(I - 1) - Hs(I - N - 1)) / (4 * dx);
            hA0 = I; hA1 = I - N; sA = 1.0 / dy;
            hB[0] = I + 1; hB[1] = I - N + 1; hB[2] = I - 1; hB[3] = I - N - 1; sB = 1.0 / (4 * dx);
        } else {             // N: (H_{j+1} - Hc)/dy, (H_{i+1,j+1} + H_{i+1} - H_{i-1,j+1} - H_{i-1})/(4dx)
            Ac = (Hs(I + N) - Hc) / dy;
            Bc = (Hs(I + N + 1) + Hs(I + 1) - Hs(I + N - 1) - Hs(I - 1)) / (4 * dx);
            hA0 = I + N; hA1 = I; sA = 1.0 / dy;
            hB[0] = I + N + 1; hB[1] = I + 1; hB[2] = I + N - 1; hB[3] = I - 1; sB = 1.0 / (4 * dx);
        }
        const double S = sqrt(pow(Ac, 2.) + pow(Bc, 2.));
        const double hup = (Hnb > Hc) ? hnb : hc;
        const double hav = (hnb + hc) / 2.;
        if (!(hup > D.hmin && hav > D.hmin && fabs(S) > D.delta)) continue;  // K0: constant
        const double k = pow(hav, 5. / 3.) / (0.5 * (mnb + mc) * sqrt(S));
        const double hb = kbar * (5.0 / 3.0) * k / hav * 0.5;
        atomicAdd(&A.olf_hbar[I], hb);
        atomicAdd(&A.olf_hbar[nb], hb);
        const double Sbar = kbar * (-0.5 * k / S);
        const double Abar = Sbar * Ac / S, Bbar = Sbar * Bc / S;
        atomicAdd(&A.olf_Hbar[hA0], Abar * sA);
        atomicAdd(&A.olf_Hbar[hA1], -Abar * sA);
        atomicAdd(&A.olf_Hbar[hB[0]], Bbar * sB);
        atomicAdd(&A.olf_Hbar[hB[1]], Bbar * sB);
        atomicAdd(&A.olf_Hbar[hB[2]], -Bbar * sB);
        atomicAdd(&A.olf_Hbar[hB[3]], -Bbar * sB);
    }
}

// dL/d(ph after the subsurface step): H = ph + z and the Manning depths; the
// fixed ring keeps its depth.
__global__ void __launch_bounds__(TILE_THREADS) k_adj_olf_finish(DevPtrs P, AdjPtrs A) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const long long c = cr.c;
    double v = A.olf_Hbar[c] + A.olf_hbar[c];
    if (on_ring(cr.i, cr.j, cr.nx, cr.ny)) v += A.phbar[c];
    A.phsub_bar[c] = v;
}

// -------------------------------------------------------------- epilogue
// Reverse of the rollover and the infiltration/ponding update; seeds the last
// Picard iteration's adjoints and clears this step's input accumulators.
__global__ void __launch_bounds__(TILE_THREADS) k_adj_epilogue(DevPtrs P, AdjPtrs A, int iters) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    const long long c = cr.c;
    const double dt = D.dt;
    const int s = A.step_in_seg;
    {
        const double a = P.hpoten[c] - P.qtop[c] * dt;
        const double phb = A.phsub_bar[c];
        A.hpbar[c] = (a > 0.0) ? phb : 0.0;
        A.qtbar[c] = (a > 0.0) ? -dt * phb : 0.0;
    }
    const long long last = ((long long)s * A.maxiter + (iters - 1)) * A.np;
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const double x = A.t_xm[last + g], pm = A.t_psim[last + g];
        double thb = A.thbar_next[g];
        if (k < 3) thb += A.t_thseed[((long long)s * 3 + k) * A.nc + c];
        double xb = A.psibar_next[g];
        double thmb = 0.0, cmb = 0.0, pmb = 0.0;
        const double a = cell_alpha(P, D, g), n = cell_n(P, D, g), ks = P.ksat[g];
        double gl = 0.0, ga = 0.0, gn = 0.0;
        if (D.theta_update == DHARA_THETA_CONSERVATIVE) {
            const VGD v = vg_derivs(pm, a, n, D.theta_s, D.theta_r, ks);
            thmb = thb;
            cmb = thb * (x - pm);
            xb += thb * v.C;
            pmb = -thb * v.C;
        } else if (D.theta_update == DHARA_THETA_FINAL) {
            const VGD v = vg_derivs(x, a, n, D.theta_s, D.theta_r, ks);
            xb += thb * v.C;
            ga += thb * v.th_a;
            gn += thb * v.th_n;
        } else {
            thmb = thb;
        }
        if (k == 0) {
            const double kb = A.ktopbar_next[c];
            const VGD v = vg_derivs(x, a, n, D.theta_s, D.theta_r, ks);
            xb += kb * v.K_psi;
            gl += kb * v.K;
            ga += kb * v.K_a;
            gn += kb * v.K_n;
        }
        A.xbar[g] = xb;
        A.psimbar[g] = pmb;
        A.thmbar[g] = thmb;
        A.cmbar[g] = cmb;
        A.psinbar[g] = 0.0;
        A.thnbar[g] = 0.0;
        A.g_lk[g] += gl;
        A.g_al[g] += ga;
        A.g_n[g] += gn;
    }
}

// ----------------------------------------------------------- Picard step
// The matrix of Picard iteration m (the forward assembly's K and storage
// diagonal at the recorded psi^m), the adjoint right-hand side dL/dx^m and a
// initial guess (zero for the first reversed iteration of a step, else the
// previous iteration's lambda, which the next solve starts from), for the
// forward Krylov solver.
template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_adj_matrix(DevPtrs P, AdjPtrs A, int m, int zero_guess) {
    const int tile = blockIdx.x;
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    if (threadIdx.x == 0 && tile == D.tile_begin) {
        KrylovCtrl &kc = P.kctrl[td.dom];
        kc.active = 1;
        kc.inner_active = 0;
        kc.cycles = 0;
        kc.total_iter = 0;
        kc.parity = 0;
        kc.first_inner = 1;
        kc.keep_p = 0;
        kc.rho_last = 0.0;
        atomicAdd(&P.gctrl->n_active, 1);
    }
    const ColumnRef cr = column_of(P, tile);
    if (!cr.valid) return;
    const double ssc = D.Ss / D.dt / D.porosity;
    const long long base = ((long long)A.step_in_seg * A.maxiter + m) * A.np;
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const double psi = A.t_psim[base + g];
        double th, Kv, Cv;
        const double a = cell_alpha(P, D, g), n = cell_n(P, D, g);
        if (D.closure_fp32) {
            float Kf, Cf;
            vg_eval<float>(psi, a, n, D.theta_s, D.theta_r, P.ksat[g], th, Kf, Cf);
            Kv = Kf;
            Cv = Cf;
        } else if (D.closure_fast) {
            vg_eval_fast(psi, a, n, D.theta_s, D.theta_r, P.ksat[g], th, Kv, Cv);
        } else {
            vg_eval<double>(psi, a, n, D.theta_s, D.theta_r, P.ksat[g], th, Kv, Cv);
        }
        const double Dv = ssc * th + Cv / D.dt;
        P.K64[g] = Kv;
        P.D64[g] = Dv;
        if (!std::is_same<T, double>::value) {
            ((T *)P.K)[g] = (T)Kv;
            ((T *)P.D)[g] = (T)Dv;
        }
        P.b[g] = A.xbar[g];
        if (zero_guess) P.x[g] = 0.0;
    }
}

// lambda = A_m^-1 dL/dx^m is in P.x.  With R = b - A x at the recorded x^m,
// every input y of iteration m gets lambda^T dR/dy: theta^m, C^m and K^m
// (faces, gravity, free drainage), psi^m directly (C/dt psi^m), psi^n, theta^n
// and the top flux; then the closure at psi^m chains theta, C, K into psi^m and
// the parameters, and the relaxation passes psi^m's adjoint to iteration m-1.
__global__ void __launch_bounds__(TILE_THREADS) k_adj_picard(DevPtrs P, AdjPtrs A, int m) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    const double dt = D.dt, dz = D.dz;
    const double idx2 = 1.0 / (D.dx * D.dx), idy2 = 1.0 / (D.dy * D.dy), idz2 = 1.0 / (dz * dz);
    const long long base = ((long long)A.step_in_seg * A.maxiter + m) * A.np;
    const double *xm = A.t_xm + base;
    const double *pmv = A.t_psim + base;
    const double *psin = A.t_psin + (long long)A.step_in_seg * A.np;
    const double *lam = P.x;
    const double *K = P.K64;
    const long long sx = 1, sy = cr.nxp, sz = cr.sxy;
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += sz) {
        const double l = lam[g], x = xm[g], Kc = K[g];
        (void)Kc;
        double Kb = 0.0;
        auto face = [&](long long nb, double w) { Kb += -0.5 * (l - lam[nb]) * (x - xm[nb]) * w; };
        if (cr.i > 0) face(g - sx, idx2);
        if (cr.i < cr.nx - 1) face(g + sx, idx2);
        if (cr.j > 0) face(g - sy, idy2);
        if (cr.j < cr.ny - 1) face(g + sy, idy2);
        if (k > 0) {
            face(g - sz, idz2);
            Kb += 0.5 * (l - lam[g - sz]) / dz;
        }
        if (k < cr.nz - 1) {
            face(g + sz, idz2);
            Kb += 0.5 * (lam[g + sz] - l) / dz;
        } else {
            Kb += -l / dz;  // free drainage q_b = K of the bottom cell
        }
        const double pm = pmv[g];
        const double a = cell_alpha(P, D, g), n = cell_n(P, D, g), ks = P.ksat[g];
        const VGD v = vg_derivs(pm, a, n, D.theta_s, D.theta_r, ks);
        const double thb = A.thmbar[g] + l * (D.Ss / (dt * D.porosity) * (psin[g] - x) - 1.0 / dt);
        const double cb = A.cmbar[g] + l * (pm - x) / dt;
        const double pb = A.psimbar[g] + l * v.C / dt + thb * v.C + cb * v.C_psi + Kb * v.K_psi;
        A.g_lk[g] += Kb * v.K;
        A.g_al[g] += thb * v.th_a + cb * v.C_a + Kb * v.K_a;
        A.g_n[g] += thb * v.th_n + cb * v.C_n + Kb * v.K_n;
        A.psinbar[g] += l * D.Ss * v.th / (D.porosity * dt);
        A.thnbar[g] += l / dt;
        if (k == 0) A.qtbar[cr.c] += l / dz;
        if (m > 0) {
            A.psimbar[g] = D.am * pb;
            A.xbar[g] = (1.0 - D.am) * pb;
            A.thmbar[g] = 0.0;
            A.cmbar[g] = 0.0;
        } else {
            A.psinbar[g] += pb;
        }
    }
}

// -------------------------------------------------------------- prologue
// Reverse of EstimateFluxes + IdentifyTopBoundary (src/global.cu:172-257)
// along the branch the forward took.
__global__ void __launch_bounds__(TILE_THREADS) k_adj_prologue(DevPtrs P, AdjPtrs A) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    const long long c = cr.c, g0 = cr.g0;
    const int s = A.step_in_seg;
    const double dt = D.dt, dz = D.dz;
    const double psit = A.t_psin[(long long)s * A.np + g0];
    const double thetat = A.t_thetan[(long long)s * A.np + g0];
    const double ktop = A.t_ktop[(long long)s * A.nc + c];
    const double ph = A.t_ph[(long long)s * A.nc + c];
    const double ks = P.ksat[g0];
    const double hpoten = P.hpoten[c];
    const double qraw = -ktop * ((psit - hpoten - 0.5 * dz) / (0.5 * dz));
    const bool cond_ks = ph / dt > ks;
    const double qcapa = cond_ks ? fmax(qraw, ks) : qraw;
    const double qtb = A.qtbar[c];
    double hpb = A.hpbar[c], ksb = 0.0, qcb = 0.0, ktb = 0.0, psb = 0.0, thb = 0.0;
    if (hpoten > 0.0) {
        const bool cap = hpoten / dt > qcapa;
        const double q1 = cap ? qcapa : hpoten / dt;
        const double qsat = (D.theta_s - thetat) * dz / dt;
        const bool sat_sel = qsat < q1;
        const double q2 = sat_sel ? qsat : q1;
        if (ks < q2) ksb += qtb;
        else if (sat_sel) thb -= qtb * dz / dt;
        else if (cap) qcb += qtb;
        else hpb += qtb / dt;
    } else {
        hpb += qtb / dt;
    }
    if (qcb != 0.0) {
        if (cond_ks && qraw < ks) {
            ksb += qcb;
        } else {
            ktb += qcb * (-(psit - hpoten - 0.5 * dz) / (0.5 * dz));
            psb += qcb * (-ktop / (0.5 * dz));
            hpb += qcb * (ktop / (0.5 * dz));
        }
    }
    A.phbar[c] = hpb;
    A.ktopbar_next[c] = ktb;
    A.psinbar[g0] += psb;
    A.thnbar[g0] += thb;
    A.g_lk[g0] += ksb * ks;
}

// theta^0 and K^0_top come from the closure at the initial head.
__global__ void __launch_bounds__(TILE_THREADS) k_adj_initial(DevPtrs P, AdjPtrs A) {
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    const DomainDesc &D = P.dom[cr.dom];
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const double psi0 = A.t_psin[g];
        const VGD v = vg_derivs(psi0, cell_alpha(P, D, g), cell_n(P, D, g), D.theta_s, D.theta_r, P.ksat[g]);
        const double thb = A.thbar_next[g];
        double gl = 0.0, ga = thb * v.th_a, gn = thb * v.th_n;
        if (k == 0) {
            const double kb = A.ktopbar_next[cr.c];
            gl += kb * v.K;
            ga += kb * v.K_a;
            gn += kb * v.K_n;
        }
        A.g_lk[g] += gl;
        A.g_al[g] += ga;
        A.g_n[g] += gn;
    }
}

// ------------------------------------------------------------- launchers
cudaError_t launch_adj_loss(const DevPtrs &P, const AdjPtrs &A, int t, int seed_slot, cudaStream_t s) {
    k_adj_loss<<<P.ntiles, TILE_THREADS, 0, s>>>(P, A, t, seed_slot);
    return cudaGetLastError();
}
cudaError_t launch_adj_olf_rhs(const DevPtrs &P, const AdjPtrs &A, int t, cudaStream_t s) {
    long long ctot = A.nc;
    k_adj_olf_rhs<<<P.ntiles, TILE_THREADS, 0, s>>>(P, A, t, ctot);
    return cudaGetLastError();
}
cudaError_t launch_adj_olf_coef(const DevPtrs &P, const AdjPtrs &A, int t, long long ctot, cudaStream_t s) {
    k_adj_olf_coef<<<P.ntiles, TILE_THREADS, 0, s>>>(P, A, t, ctot);
    return cudaGetLastError();
}
cudaError_t launch_adj_olf_finish(const DevPtrs &P, const AdjPtrs &A, cudaStream_t s) {
    k_adj_olf_finish<<<P.ntiles, TILE_THREADS, 0, s>>>(P, A);
    return cudaGetLastError();
}
cudaError_t launch_adj_epilogue(const DevPtrs &P, const AdjPtrs &A, int slot, int iters, cudaStream_t s) {
    AdjPtrs a = A;
    a.step_in_seg = slot;
    k_adj_epilogue<<<P.ntiles, TILE_THREADS, 0, s>>>(P, a, iters);
    return cudaGetLastError();
}
cudaError_t launch_adj_matrix(const DevPtrs &P, const AdjPtrs &A, int slot, int m, int zero_guess, int mixed,
                              cudaStream_t s) {
    AdjPtrs a = A;
    a.step_in_seg = slot;
    if (mixed) k_adj_matrix<float><<<P.ntiles, TILE_THREADS, 0, s>>>(P, a, m, zero_guess);
    else k_adj_matrix<double><<<P.ntiles, TILE_THREADS, 0, s>>>(P, a, m, zero_guess);
    return cudaGetLastError();
}
cudaError_t launch_adj_picard(const DevPtrs &P, const AdjPtrs &A, int slot, int m, cudaStream_t s) {
    AdjPtrs a = A;
    a.step_in_seg = slot;
    k_adj_picard<<<P.ntiles, TILE_THREADS, 0, s>>>(P, a, m);
    return cudaGetLastError();
}
cudaError_t launch_adj_prologue(const DevPtrs &P, const AdjPtrs &A, int slot, cudaStream_t s) {
    AdjPtrs a = A;
    a.step_in_seg = slot;
    k_adj_prologue<<<P.ntiles, TILE_THREADS, 0, s>>>(P, a);
    return cudaGetLastError();
}
cudaError_t launch_adj_initial(const DevPtrs &P, const AdjPtrs &A, cudaStream_t s) {
    AdjPtrs a = A;
    a.step_in_seg = 0;
    k_adj_initial<<<P.ntiles, TILE_THREADS, 0, s>>>(P, a);
    return cudaGetLastError();
}
