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
#include "staging.cuh"

#include <cstdio>

#define MAX_CYCLES 30

// The closure of the assembled system: the reference's FP64 expressions in
// FP64 mode, the reformulated FP64 closure in mixed mode, or the FP32 closure
// when the domain asks for it.
__device__ __forceinline__ void closure(const DomainDesc &D, double psi, double a, double n, double ks,
                                        double &th, double &K, double &C) {
    if (D.closure_fp32) {
        float Kf, Cf;
        vg_eval<float>(psi, a, n, D.theta_s, D.theta_r, ks, th, Kf, Cf);
        K = (double)Kf;
        C = (double)Cf;
    } else if (D.closure_fast) {
        vg_eval_fast(psi, a, n, D.theta_s, D.theta_r, ks, th, K, C);
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
__device__ __forceinline__ void prologue_tile(const DevPtrs &P, int tile) {
    const ColumnRef cr = column_of(P, tile);
    const DomainDesc &D = P.dom[cr.dom];
    const TileDesc td = P.tiles[tile];
    if (threadIdx.x == 0) {
        if (tile == 0) {
            P.gctrl->n_active = 0;
            P.gctrl->n_inner_active = 0;
            P.gctrl->n_olf_active = 0;
            P.gctrl->n_picard = P.ndom - P.n_frozen;
        }
        if (tile == D.tile_begin) {
            PicardCtrl &pc = P.pctrl[td.dom];
            pc.iter = 0;
            pc.done = D.frozen;
            pc.converged = 0;
            pc.err = 0.0;
            P.diag[td.dom].krylov_iters_last = 0;
            for (int q = 0; q < 16; ++q) P.step_acc[td.dom * 16 + q] = 0.0;
        }
    }
    unsigned long long bsig = 0;
    if (cr.valid) {
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
        // the step's rain (mm) spread over its sub-steps (sub_frac 1 without halving)
        const double hpoten = ph + ppt * D.sub_frac / 1000 - P.esoil[c] * D.sec * dt;
        const double ks = P.ksat[g];
        double qcapa = -P.ktop[c] * ((P.psin[g] - hpoten - 0.5 * dz) / (0.5 * dz));
        // which branches the selection took, each comparison in three states (band3)
        unsigned code = band3(ph / dt, ks, rel_band(ph / dt, ks, 1e-30));
        if (ph / dt > ks) qcapa = fmax(qcapa, ks);
        double q;
        code = code * 3u + band3(hpoten, 0.0, 1e-15);
        if (hpoten > 0.0) {
            code = code * 3u + band3(hpoten / dt, qcapa, rel_band(hpoten / dt, qcapa, 1e-30));
            q = (hpoten / dt > qcapa) ? qcapa : hpoten / dt;
            const double room = (D.theta_s - P.thetan[g]) * dz / dt;
            code = code * 3u + band3(q, room, rel_band(q, room, 1e-30));
            q = fmin(q, room);
            code = code * 3u + band3(q, ks, rel_band(q, ks, 1e-30));
            q = fmin(q, ks);
        } else {
            q = hpoten / dt;
        }
        P.hpoten[c] = hpoten;
        P.qtop[c] = q;
        if (records(D, BR_TOPFLUX)) bsig = branch_mix(step, BR_TOPFLUX, c, code);
    }
    if (D.record_branches) branch_commit(&P.diag[td.dom].branch_sig, bsig);
}

__global__ void k_prologue(DevPtrs P) {
    prologue_tile(P, blockIdx.x);
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
// Eight blocks per SM (64 registers): the FP64 closure's latency chains need the
// warps more than the registers (measured 18 % faster than the uncapped 96).
template <typename T>
__device__ __forceinline__ void assemble_tile(const DevPtrs &P, int tile) {
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
        kc.keep_p = 0;
        kc.rho_last = 0.0;
        if (!done) atomicAdd(&P.gctrl->n_active, 1);
    }
    if (done) return;
    const ColumnRef cr = column_of(P, tile);
    if (records(D, BR_SATURATION)) {
        // saturation (psi >= 0 switches the closure's branch) of every cell at psi^m
        unsigned long long bsig = 0;
        if (cr.valid) {
            long long g = cr.g0;
            for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
                const double psi = (iter == 0) ? P.psin[g] : D.am * P.psim[g] + (1.0 - D.am) * P.x[g];
                bsig += branch_mix(pc.step * 64 + (iter & 63), BR_SATURATION, g, band3(psi, 0.0, 1e-9));
            }
        }
        branch_commit(&P.diag[td.dom].branch_sig, bsig);
    }
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
        const long long bi = D.offWE + (long long)k * cr.ny + cr.j;
        const long long bj = D.offSN + (long long)k * cr.nx + cr.i;
        // Neumann terms only on non-Dirichlet faces (a Dirichlet face's rows are
        // set by k_dir_fixed / k_dir_rows after this kernel)
        const bool dd = D.has_dirichlet != 0;
        if (k == nz - 1 && !(dd && P.dir_b[cr.c])) {
            const double qb = K_c;
            P.bcqb[cr.c] = qb;
            rhs += (qb * dz) * dz2inv;
        }
        if (cr.j == 0 && !(dd && P.dir_s[bj])) rhs += (-P.bcqs[bj] * dy) * dy2inv;
        if (cr.j == cr.ny - 1 && !(dd && P.dir_n[bj])) rhs += (P.bcqn[bj] * dy) * dy2inv;
        if (cr.i == 0 && !(dd && P.dir_w[bi])) rhs += (-P.bcqw[bi] * dx) * dx2inv;
        if (cr.i == cr.nx - 1 && !(dd && P.dir_e[bi])) rhs += (P.bcqe[bi] * dx) * dx2inv;

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

template <typename T>
__global__ void __launch_bounds__(TILE_THREADS, 8) k_assemble(DevPtrs P) {
    assemble_tile<T>(P, blockIdx.x);
}

// ---------------------------------------------------------- Dirichlet faces
// The reference turns each Dirichlet (type 0) face into identity rows for the
// boundary cells and eliminates their coupling from the next row in, walking
// the faces in the order top, bottom, south, north, west, east
// (SetUpBoundaryConditionsSubsurface, src/subsurface.cu:126-353).  Two of its
// details are kept: the rows next to a west/east/south/north face move the
// fixed head to the right-hand side with the conductance of the face on the
// other side of the row (ke for a west face, kw for east, kn for south, ks for
// north), and a row already set to the identity by an earlier face still takes
// the right-hand-side terms of later faces.  Here the identity rows are cells
// whose storage diagonal is set to -1 (the Krylov phases skip them) and whose
// iterate holds the row's right-hand side; the matrix-free stencil of the next
// row in couples to that value, so its right-hand side is corrected to the
// reference's elimination.
struct DirFaces {
    bool b, s, n, w, e;
    double pb, ps, pn, pw, pe;
};

__device__ __forceinline__ DirFaces dir_faces(const DevPtrs &P, const DomainDesc &D, const ColumnRef &cr, int k) {
    const long long bi = D.offWE + (long long)k * cr.ny + cr.j;
    const long long bj = D.offSN + (long long)k * cr.nx + cr.i;
    DirFaces f;
    f.b = P.dir_b[cr.c] != 0;
    f.s = P.dir_s[bj] != 0;
    f.n = P.dir_n[bj] != 0;
    f.w = P.dir_w[bi] != 0;
    f.e = P.dir_e[bi] != 0;
    f.pb = f.b ? P.psi_b[cr.c] : 0.0;
    f.ps = f.s ? P.psi_s[bj] : 0.0;
    f.pn = f.n ? P.psi_n[bj] : 0.0;
    f.pw = f.w ? P.psi_w[bi] : 0.0;
    f.pe = f.e ? P.psi_e[bi] : 0.0;
    return f;
}

// Face conductances of a cell from K^m (K64), zero on domain faces.
struct FaceK {
    double kw, ke, ks, kn, kd, ku;
};
__device__ __forceinline__ FaceK face_k(const DevPtrs &P, const ColumnRef &cr, long long g, int k) {
    const double *K = P.K64;
    const double Kc = K[g];
    FaceK f;
    f.kw = cr.i > 0 ? 0.5 * (Kc + K[g - 1]) : 0.0;
    f.ke = cr.i < cr.nx - 1 ? 0.5 * (Kc + K[g + 1]) : 0.0;
    f.ks = cr.j > 0 ? 0.5 * (Kc + K[g - cr.nxp]) : 0.0;
    f.kn = cr.j < cr.ny - 1 ? 0.5 * (Kc + K[g + cr.nxp]) : 0.0;
    f.kd = k > 0 ? 0.5 * (Kc + K[g - cr.sxy]) : 0.0;
    f.ku = k < cr.nz - 1 ? 0.5 * (Kc + K[g + cr.sxy]) : 0.0;
    return f;
}

// The reference's right-hand side of a cell after the face rules, starting
// from the assembled value v; returns whether an identity row was set.
__device__ __forceinline__ bool dir_rules(const ColumnRef &cr, int k, const DirFaces &f, const FaceK &fk,
                                          const DomainDesc &D, double &v) {
    const double ix2 = 1.0 / (D.dx * D.dx), iy2 = 1.0 / (D.dy * D.dy), iz2 = 1.0 / (D.dz * D.dz);
    bool fixed = false;
    if (f.b) {
        if (k == cr.nz - 2) v += iz2 * fk.ku * f.pb;
        if (k == cr.nz - 1) { v = f.pb; fixed = true; }
    }
    if (f.s) {
        if (cr.j == 1) v += iy2 * fk.kn * f.ps;
        if (cr.j == 0) { v = f.ps; fixed = true; }
    }
    if (f.n) {
        if (cr.j == cr.ny - 2) v += iy2 * fk.ks * f.pn;
        if (cr.j == cr.ny - 1) { v = f.pn; fixed = true; }
    }
    if (f.w) {
        if (cr.i == 1) v += ix2 * fk.ke * f.pw;
        if (cr.i == 0) { v = f.pw; fixed = true; }
    }
    if (f.e) {
        if (cr.i == cr.nx - 2) v += ix2 * fk.kw * f.pe;
        if (cr.i == cr.nx - 1) { v = f.pe; fixed = true; }
    }
    return fixed;
}

// Pass 1: identity rows (D = -1, x = b = the row's right-hand side).
template <typename T>
__device__ __forceinline__ void dir_fixed_tile(const DevPtrs &P, int tile) {
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    if (!D.has_dirichlet || P.pctrl[td.dom].done) return;
    const ColumnRef cr = column_of(P, tile);
    if (!cr.valid) return;
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        const DirFaces f = dir_faces(P, D, cr, k);
        if (!(f.b || f.s || f.n || f.w || f.e)) continue;
        double v = P.b[g];
        if (!dir_rules(cr, k, f, face_k(P, cr, g, k), D, v)) continue;
        P.b[g] = v;
        P.x[g] = v;
        P.D64[g] = -1.0;
        if (!std::is_same<T, double>::value) ((T *)P.D)[g] = T(-1);
    }
}

template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_dir_fixed(DevPtrs P) {
    dir_fixed_tile<T>(P, blockIdx.x);
}

// Pass 2: the rows next to identity rows get the reference's elimination
// terms, less the coupling the matrix-free stencil applies to the fixed value.
template <typename T>
__device__ __forceinline__ void dir_rows_tile(const DevPtrs &P, int tile) {
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    if (!D.has_dirichlet || P.pctrl[td.dom].done) return;
    const ColumnRef cr = column_of(P, tile);
    if (!cr.valid) return;
    const double ix2 = 1.0 / (D.dx * D.dx), iy2 = 1.0 / (D.dy * D.dy), iz2 = 1.0 / (D.dz * D.dz);
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        if (P.D64[g] < 0.0) continue;  // identity row
        const DirFaces f = dir_faces(P, D, cr, k);
        if (!(f.b || f.s || f.n || f.w || f.e)) continue;
        const FaceK fk = face_k(P, cr, g, k);
        double v = P.b[g];
        dir_rules(cr, k, f, fk, D, v);
        if (f.b && k == cr.nz - 2) v -= iz2 * fk.ku * P.x[g + cr.sxy];
        if (f.s && cr.j == 1) v -= iy2 * fk.ks * P.x[g - cr.nxp];
        if (f.n && cr.j == cr.ny - 2) v -= iy2 * fk.kn * P.x[g + cr.nxp];
        if (f.w && cr.i == 1) v -= ix2 * fk.kw * P.x[g - 1];
        if (f.e && cr.i == cr.nx - 2) v -= ix2 * fk.ke * P.x[g + 1];
        P.b[g] = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_dir_rows(DevPtrs P) {
    dir_rows_tile<T>(P, blockIdx.x);
}

// ------------------------------------------------------------ Krylov solve
// Persistent cooperative kernel: for every active domain it solves
// A x = b to ||b - A x|| <= tol ||b|| (the CUSP monitor's rule,
// CUSP/detail/monitor.inl:108-111,181-201) by iterative refinement:
//   R: r = b - A x in FP64 arithmetic, z = M^-1 (T) r
//   inner PCG in T on A d = (T) r, M = the z-line (column) tridiagonal part of A
//   U: x += d
// In FP64 mode T = double and one cycle normally converges (the inner target
// is the outer tolerance).  In mixed mode T = float, the inner solve reduces
// the residual by inner_tol and cycles repeat until the FP64 residual meets
// the tolerance.  The reference runs unpreconditioned BiCGSTAB; any solver
// converged to the same tolerance yields the same head field.
//
// One inner PCG iteration is ONE sweep and one grid barrier.  The residual r
// and A p are never stored: the sweep carries the preconditioned residual z
// and t = M^-1 A p, whose recurrence z_{i+1} = z_i - alpha_i t_i is the
// residual's r_{i+1} = r_i - alpha_i A p_i mapped through M^-1.  Sweep i
// (alpha_{i-1}, beta_i known from the previous reduction):
//   z_i = z_{i-1} - alpha_{i-1} t_{i-1},  p_i = z_i + beta_i p_{i-1}
//       (formed at the tile's own and halo columns from the staged previous
//       z, t, p, so no neighbour has to publish them first)
//   q = A p_i,  t_i = M^-1 q (column solve),  d += alpha_{i-1} p_{i-1}
//   partial sums sigma = p_i.q, mu = z_i.q, nu = q.t_i, rho_i = z_i.M z_i
// and after the barrier alpha_i = rho_i / sigma and
//   rho_{i+1} = rho_i - 2 alpha_i mu + alpha_i^2 nu    (r_i.t_i = z_i.q by
//   symmetry of M), beta_{i+1} = rho_{i+1} / rho_i.
// rho_i is evaluated directly from z_i rather than carried by the update
// formula, which would accumulate cancellation; the formula is only ever
// applied to a freshly computed rho.  With M = L D L^T from the stored
// factors, z.M z = sum_k (z_k + c'_k z_{k+1})^2 / inv_k per column: a sum of
// positive terms (forming M z from the operator's coefficients instead
// cancels, and costs the FP32 solve 3 % more inner iterations on the
// 512x512x40 storm).  x's last update (alpha of the final iteration times its
// p) is applied in U.
// Per inner iteration each cell reads z, t, p, K (at the halo), D, 1/den, c',
// d and writes z, t, p, d: 12 words (the two factors FP32 in FP64 mode),
// against 15 and two grid barriers for the textbook two-phase iteration.

template <typename T>
struct StencilW {
    T cx, cy, cz;
};

// Planes per staged chunk of the inner phases and of the FP64 outer residual.
template <typename T>
struct Chunk {
    static constexpr int inner = sizeof(T) == 4 ? CHUNK_F32 : CHUNK_F64;
};

// Storage type of the column preconditioner's factors 1/den and c': bf16 in
// mixed mode with FACTOR_NARROW_F32, FP32 in FP64 mode with FACTOR_NARROW_F64.  Any rounding of
// the stored pair still defines a symmetric positive definite M = L D L^T
// (D = 1/inv > 0, L from c'), and every use of M -- phase R's z = M^-1 r,
// the sweep's forward and back substitutions and its z.M z -- goes through
// the stored values, so the inner CG sees one fixed preconditioner.
template <typename T>
struct Fac {
    using type = T;
};
#if FACTOR_NARROW_F32
template <>
struct Fac<float> {
    using type = __nv_bfloat16;
};
#endif
#if FACTOR_NARROW_F64
template <>
struct Fac<double> {
    using type = float;
};
#endif
template <typename T, typename F>
__device__ __forceinline__ T fac_get(F v) {
    if constexpr (std::is_same<F, __nv_bfloat16>::value) return (T)__bfloat162float(v);
    else return (T)v;
}
template <typename F, typename T>
__device__ __forceinline__ F fac_put(T v) {
    if constexpr (std::is_same<F, __nv_bfloat16>::value) return __float2bfloat16_rn((float)v);
    else return (F)v;
}

// Bytes of one staging buffer of each phase (the kernel reserves STAGES buffers
// of the largest).
template <typename T>
struct StageSize {
    static constexpr int C = Chunk<T>::inner;
    using F = typename Fac<T>::type;
    // inner sweep: z, t, p of the previous iteration and K (halo); D, 1/den, c', d (own)
    static constexpr size_t I =
        4 * (size_t)halo_slot<T, C>() + 2 * (size_t)own_bytes<T, C>() + 2 * (size_t)own_bytes<F, C>();
    // phase R: x, K64 (halo); D64, b (own), all FP64
    static constexpr size_t R = 2 * (size_t)halo_slot<double, CH_R>() + 2 * (size_t)own_bytes<double, CH_R>();
    static constexpr size_t buffer() { return I > R ? I : R; }
    static constexpr size_t bytes() { return STAGES * buffer(); }
};

// Chunked march over a tile's planes: thread 0 arms and issues chunk st into
// buffer st % STAGES (issue(st, b)), so STAGES - 1 chunks are in flight while
// one is computed; every thread waits for the chunk and computes its planes
// (plane(b, pl, k)).  With NEXT, the last plane of a chunk also reads the first
// plane of the next chunk (the z-neighbour of a stencil), which is awaited
// first.  A buffer is refilled with chunk st + STAGES once all threads are done
// with it; when the tile is done, issue_next() starts the block's next tile so
// its first chunks stream in during this tile's epilogue.
// pf(st) starts the L2 prefetch of chunk st (PF_DIST chunks beyond the last
// one issued into shared memory), so that more DRAM reads are in flight than
// the staging buffers hold.
template <int CHN, bool NEXT, typename Issue, typename PlaneFn, typename NextFn, typename Prefetch>
__device__ __forceinline__ void march(int nz, StageBars &sb, bool prefetched, Issue issue, PlaneFn plane,
                                      NextFn issue_next, Prefetch pf) {
    const int nst = (nz + CHN - 1) / CHN;
    if (threadIdx.x == 0 && !prefetched)
        for (int q = 0; q < STAGES && q < nst; ++q) issue(q, q);
    if constexpr (PF_DIST > 0)
        if (threadIdx.x == 0)
            for (int q = STAGES; q < STAGES + PF_DIST && q < nst; ++q) pf(q);
    bool next_ready = false;
    for (int st = 0; st < nst; ++st) {
        const int b = st % STAGES;
        if (!next_ready) sb.wait(b);
        next_ready = false;
        for (int pl = 0; pl < CHN; ++pl) {
            const int k = st * CHN + pl;
            if (k >= nz) break;
            if (NEXT && pl == CHN - 1 && k + 1 < nz) {
                sb.wait((b + 1) % STAGES);
                next_ready = true;
            }
            plane(b, pl, k);
        }
        __syncthreads();
        if (threadIdx.x == 0 && st + STAGES < nst) {
            issue(st + STAGES, b);
            if constexpr (PF_DIST > 0)
                if (st + STAGES + PF_DIST < nst) pf(st + STAGES + PF_DIST);
        }
    }
    if (threadIdx.x == 0) issue_next();
}

// The column preconditioner M is the z-coupled (tridiagonal) part of A:
// b_k = D_k + sum_f w_f k_f, a_k = -w_z kd_k, c_k = -w_z ku_k.  The column is
// symmetric (a_{k+1} = c_k: both are -w_z (K_k + K_{k+1}) / 2 from the same
// rounded operands), so M = L D L^T with D = diag(den) and the unit lower
// bidiagonal L of l_{k+1} = c_k / den_k = c'_k.  It is factored once per outer
// cycle (phase R),
//   den_k = b_k - a_k c'_{k-1},  c'_k = c_k / den_k,
// and only 1/den and c' are stored per cell.  Applying M^-1 in the inner
// iterations is three short recurrences:
//   forward  y_k = r_k - c'_{k-1} y_{k-1},  d'_k = y_k / den_k,
//   backward z_k = d'_k - c'_k z_{k+1},
// and r^T M^-1 r = sum_k y_k d'_k is accumulated in the forward sweep.  Any
// rounding of the stored factors still gives a symmetric M (the same c' feeds
// both sweeps), so the inner CG sees a fixed SPD preconditioner.  d' lives in
// shared memory when T is float (DSMEM), else in the z array itself.
template <typename T, bool DSMEM>
__device__ __forceinline__ void put_dprime(T dp, T *s_d, int k, T *__restrict__ zg) {
    if (DSMEM) s_d[k * TILE_THREADS + threadIdx.x] = dp;
    else *zg = dp;
}

// The back substitution loads BACK_BATCH planes of c' and d' before using
// them, so that several loads are in flight per thread (4 measured fastest:
// 0.1667 ms per FP32 inner iteration on the 512x512x40 storm against 0.1713
// for 8 and 0.1989 for 16, where the larger batches cost registers).
#ifndef BACK_BATCH
#define BACK_BATCH 4
#endif
template <typename T, bool DSMEM, typename F>
__device__ __forceinline__ void back_sweep(const ColumnRef &cr, const T *s_d, const F *__restrict__ fc,
                                           T *__restrict__ z) {
    T zn = T(0);
    const unsigned g0 = (unsigned)cr.g0, sxy = (unsigned)cr.sxy;
    for (int k0 = cr.nz - 1; k0 >= 0; k0 -= BACK_BATCH) {
        T cl[BACK_BATCH], dl[BACK_BATCH];
#pragma unroll
        for (int q = 0; q < BACK_BATCH; ++q) {
            const int k = k0 - q;
            if (k >= 0) {
                const unsigned g = g0 + (unsigned)k * sxy;
                cl[q] = fac_get<T>(fc[g]);
                dl[q] = DSMEM ? s_d[k * TILE_THREADS + threadIdx.x] : z[g];
            }
        }
#pragma unroll
        for (int q = 0; q < BACK_BATCH; ++q) {
            const int k = k0 - q;
            if (k >= 0) {
                const T zk = dl[q] - cl[q] * zn;
                z[g0 + (unsigned)k * sxy] = zk;
                zn = zk;
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ T recip(T x);
template <>
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
template <>
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }

// a / b where the quotient only feeds a sum of positive terms (z.M z): the
// hardware reciprocal's approximation (about 2 ulp) in FP32
template <typename T>
__device__ __forceinline__ T quot(T a, T b);
template <>
__device__ __forceinline__ float quot(float a, float b) { return __fdividef(a, b); }
template <>
__device__ __forceinline__ double quot(double a, double b) { return a / b; }

// Face masks of a column: 1 where the face is interior, 0 on a domain face.
struct Masks {
    double w, e, s, n;
};
__device__ __forceinline__ Masks masks_of(const ColumnRef &cr) {
    Masks m;
    m.w = cr.i > 0 ? 1.0 : 0.0;
    m.e = cr.i < cr.nx - 1 ? 1.0 : 0.0;
    m.s = cr.j > 0 ? 1.0 : 0.0;
    m.n = cr.j < cr.ny - 1 ? 1.0 : 0.0;
    return m;
}

// Face weights of a column for the T operator: the stencil weight times the
// 1/2 of the face average, zero on a domain face, so that a face coefficient
// is one add and one multiply, f = h (K_c + K_nb).  The vertical coefficient
// of the face between planes k and k+1 is the same number seen from either
// cell (IEEE addition commutes), so it is computed once and carried.
template <typename T>
struct FaceW {
    T w, e, s, n, z;
};
template <typename T>
__device__ __forceinline__ FaceW<T> face_weights(const ColumnRef &cr, const StencilW<T> &w) {
    FaceW<T> f;
    f.w = cr.i > 0 ? T(0.5) * w.cx : T(0);
    f.e = cr.i < cr.nx - 1 ? T(0.5) * w.cx : T(0);
    f.s = cr.j > 0 ? T(0.5) * w.cy : T(0);
    f.n = cr.j < cr.ny - 1 ? T(0.5) * w.cy : T(0);
    f.z = T(0.5) * w.cz;
    return f;
}

// Diagonal of the column block of M without its vertical couplings (the same
// expression in the factorisation and in the inner sweep's M z).
template <typename T>
__device__ __forceinline__ T lateral_diag(T Dk, T fw, T fe, T fs, T fn) {
    return (Dk + (fw + fe)) + (fs + fn);
}

// Chunk issue of each phase for tile `tile` (thread 0 only): arms buffer b's
// mbarrier with the chunk's bytes and starts one TMA box load per array.
template <typename T>
__device__ __forceinline__ void issue_R(const DevPtrs &P, int tile, int st, int b, unsigned char *stage,
                                        StageBars &sb) {
    constexpr int CHN = CH_R;
    constexpr unsigned HS = halo_slot<double, CHN>();
    constexpr unsigned OB = own_bytes<double, CHN>();
    static_assert(HS % 128 == 0 && OB % 128 == 0, "TMA destinations must be 128-byte aligned");
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    const unsigned HB = halo_bytes<double, CHN>(D.tx, D.ty);
    const CUtensorMap *maps = P.tmaps + (size_t)td.dom * NMAP;
    unsigned char *B = stage + b * StageSize<T>::buffer();
    const int k0 = st * CHN;
    sb.issued(b);
    mbar_expect_tx(sb.bar + b, 2 * HB + 2 * OB);
    tma_halo<double, CHN>((double *)B, maps + MAP_X64_H, td.x0, td.y0, k0, sb.bar + b);
    tma_halo<double, CHN>((double *)(B + HS), maps + MAP_K64_H, td.x0, td.y0, k0, sb.bar + b);
    tma_own<double, CHN>((double *)(B + 2 * HS), maps + MAP_D64_O, td.x0, td.y0, k0, sb.bar + b);
    tma_own<double, CHN>((double *)(B + 2 * HS + OB), maps + MAP_B_O, td.x0, td.y0, k0, sb.bar + b);
}

// The inner sweep's chunk: the previous iteration's z, t, p (buffers `prev`)
// and K at the halo, D, 1/den, c' and d at the own columns.  The first sweep of
// a cycle has no previous t or d (alpha = 0, d starts at zero), and no p
// either unless it continues the previous cycle's direction (keep_p).
template <typename T>
__device__ __forceinline__ void issue_C(const DevPtrs &P, int tile, int st, int b, unsigned char *stage,
                                        StageBars &sb, bool first, bool keep_p, int prev) {
    constexpr int CHN = Chunk<T>::inner;
    using F = typename Fac<T>::type;
    constexpr unsigned HS = halo_slot<T, CHN>(), OB = own_bytes<T, CHN>(), OF = own_bytes<F, CHN>();
    static_assert(HS % 128 == 0 && OB % 128 == 0 && OF % 128 == 0, "TMA destinations must be 128-byte aligned");
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    const unsigned HB = halo_bytes<T, CHN>(D.tx, D.ty);
    const CUtensorMap *maps = P.tmaps + (size_t)td.dom * NMAP;
    unsigned char *B = stage + b * StageSize<T>::buffer();
    const int k0 = st * CHN;
    const bool with_p = !first || keep_p;
    sb.issued(b);
    mbar_expect_tx(sb.bar + b, (first ? 2 : 3) * HB + (with_p ? HB : 0) + (first ? 1 : 2) * OB + 2 * OF);
    tma_halo<T, CHN>((T *)B, maps + (prev ? MAP_Z1_H : MAP_Z0_H), td.x0, td.y0, k0, sb.bar + b);
    if (!first) tma_halo<T, CHN>((T *)(B + HS), maps + (prev ? MAP_T1_H : MAP_T0_H), td.x0, td.y0, k0, sb.bar + b);
    if (with_p) tma_halo<T, CHN>((T *)(B + 2 * HS), maps + (prev ? MAP_P1_H : MAP_P0_H), td.x0, td.y0, k0, sb.bar + b);
    tma_halo<T, CHN>((T *)(B + 3 * HS), maps + MAP_K_H, td.x0, td.y0, k0, sb.bar + b);
    tma_own<T, CHN>((T *)(B + 4 * HS), maps + MAP_D_O, td.x0, td.y0, k0, sb.bar + b);
    tma_own<F, CHN>((F *)(B + 4 * HS + OB), maps + MAP_INV_O, td.x0, td.y0, k0, sb.bar + b);
    tma_own<F, CHN>((F *)(B + 4 * HS + OB + OF), maps + MAP_C_O, td.x0, td.y0, k0, sb.bar + b);
    if (!first) tma_own<T, CHN>((T *)(B + 4 * HS + OB + 2 * OF), maps + MAP_DD_O, td.x0, td.y0, k0, sb.bar + b);
}

// The L2 prefetch of the inner sweep's chunk st (the arrays issue_C loads).
template <typename T>
__device__ __forceinline__ void prefetch_C(const DevPtrs &P, int tile, int st, bool first, bool keep_p, int prev) {
    constexpr int CHN = Chunk<T>::inner;
    const TileDesc td = P.tiles[tile];
    const CUtensorMap *maps = P.tmaps + (size_t)td.dom * NMAP;
    const int k0 = st * CHN;
    tma_halo_prefetch<T>(maps + (prev ? MAP_Z1_H : MAP_Z0_H), td.x0, td.y0, k0);
    if (!first) tma_halo_prefetch<T>(maps + (prev ? MAP_T1_H : MAP_T0_H), td.x0, td.y0, k0);
    if (!first || keep_p) tma_halo_prefetch<T>(maps + (prev ? MAP_P1_H : MAP_P0_H), td.x0, td.y0, k0);
    tma_halo_prefetch<T>(maps + MAP_K_H, td.x0, td.y0, k0);
    tma_own_prefetch(maps + MAP_D_O, td.x0, td.y0, k0);
    tma_own_prefetch(maps + MAP_INV_O, td.x0, td.y0, k0);
    tma_own_prefetch(maps + MAP_C_O, td.x0, td.y0, k0);
    if (!first) tma_own_prefetch(maps + MAP_DD_O, td.x0, td.y0, k0);
}

// Issues chunks 0 and 1 of a tile (the prefetch of the block's next tile).
template <int CHN, typename Issue>
__device__ __forceinline__ void issue_head(int nz, Issue issue) {
    for (int q = 0; q < STAGES && q * CHN < nz; ++q) issue(q, q);
}

// ---- phase R: outer FP64 residual and the preconditioner factors -------------
// r = b - A x with the FP64 coefficients, r_T = (T) r; the column factors of M
// (1/den and c') from the inner operator's T coefficients (the same rounding as
// the stored K, D) are stored; z = M^-1 r_T into the z buffer of the domain's
// current parity (where the next sweep reads it, beside the last p);
// v = {||r||^2, ||b||^2, r.z}.
// Staged: x, K64 (halo), D64, b (own).
template <typename T, bool DSMEM, int TXC>
__device__ __forceinline__ void phase_R(const DevPtrs &P, int tile, int tile_next, bool prefetched, const ColumnRef &cr,
                        const StencilW<T> &w, T *s_d, unsigned char *stage, StageBars &sb, double (&v)[3]) {
    constexpr int CHN = CH_R;
    // the tile shape is a compile-time constant of each instantiation
    const Halo<double> H(TXC, TXC == 32 ? 5 : 4, TILE_THREADS / TXC);
    constexpr unsigned HB = halo_slot<double, CHN>(), OB = own_bytes<double, CHN>();
    // z goes into the buffer that holds the last iteration's p (the next
    // sweep reads both from there)
    T *__restrict__ z = (T *)(ldcg(&P.kctrl[P.tiles[tile].dom].parity) ? P.z1 : P.z0);
    using F = typename Fac<T>::type;
    F *__restrict__ finv = (F *)P.finv;
    F *__restrict__ fc = (F *)P.fc;
    const size_t BUF = StageSize<T>::buffer();
    auto buf = [&](int b) { return stage + b * BUF; };
    auto issue = [&](int st, int b) { issue_R<T>(P, tile, st, b, stage, sb); };
    auto issue_next = [&]() {
        if (tile_next < P.ntiles)
            issue_head<CHN>(P.dom[P.tiles[tile_next].dom].nz,
                            [&](int st, int b) { issue_R<T>(P, tile_next, st, b, stage, sb); });
    };
    const int nz = cr.nz, hc = H.hc, oc = threadIdx.x;
    const Masks M = masks_of(cr);
    const FaceW<T> f = face_weights(cr, w);
    const double cx = (double)w.cx, cy = (double)w.cy, cz = (double)w.cz;
    double x_up = 0.0, K_up = 0.0;
    T cprev = T(0), yprev = T(0), fd = T(0);
    T a2 = T(0);  // r.M^-1 r of the column, summed in T
    auto plane = [&](int b, int pl, int k) {
        if (!cr.valid) return;
        const double *sx = (const double *)buf(b) + pl * H.plane;
        const double *sK = (const double *)(buf(b) + HB) + pl * H.plane;
        const double *sD = (const double *)(buf(b) + 2 * HB) + pl * OWN_PLANE;
        const double *sb_ = (const double *)(buf(b) + 2 * HB + OB) + pl * OWN_PLANE;
        const double xc = sx[hc], Kc = sK[hc];
        double x_dn = 0.0, K_dn = 0.0;
        if (k + 1 < nz) {
            if (pl + 1 < CHN) { x_dn = sx[H.plane + hc]; K_dn = sK[H.plane + hc]; }
            else { x_dn = ((const double *)buf((b + 1) % STAGES))[hc]; K_dn = ((const double *)(buf((b + 1) % STAGES) + HB))[hc]; }
        }
        const double mu = k > 0 ? 1.0 : 0.0, md = k < nz - 1 ? 1.0 : 0.0;
        const double Kw = sK[hc - 1], Ke = sK[hc + 1], Ks = sK[hc - H.bw], Kn = sK[hc + H.bw];
        const double kd = mu * 0.5 * (Kc + K_up), ku = md * 0.5 * (Kc + K_dn);
        const double kw = M.w * 0.5 * (Kc + Kw), ke = M.e * 0.5 * (Kc + Ke);
        const double ks = M.s * 0.5 * (Kc + Ks), kn = M.n * 0.5 * (Kc + Kn);
        const double Dk = sD[oc], bk = sb_[oc];
        // D < 0 marks a Dirichlet (fixed) cell: identity row, x already holds its
        // value, so its residual is zero and the preconditioner leaves it alone
        const bool fixed = Dk < 0.0;
        const double Ax = Dk * xc + cx * (kw * (xc - sx[hc - 1]) + ke * (xc - sx[hc + 1])) +
                          cy * (ks * (xc - sx[hc - H.bw]) + kn * (xc - sx[hc + H.bw])) +
                          cz * (kd * (xc - x_up) + ku * (xc - x_dn));
        const double rk = fixed ? 0.0 : bk - Ax;
        v[0] += rk * rk;
        v[1] += bk * bk;
        const T rT = (T)rk;
        const long long g = cr.g0 + (long long)k * cr.sxy;
        // the column block of M from the T coefficients: diagonal bl + fd + fu,
        // sub-diagonal -fd, super-diagonal -fu
        const T Kt = (T)Kc;
        const T fw = f.w * (Kt + (T)Kw), fe = f.e * (Kt + (T)Ke);
        const T fs = f.s * (Kt + (T)Ks), fn = f.n * (Kt + (T)Kn);
        const T fu = k + 1 < nz ? f.z * (Kt + (T)K_dn) : T(0);
        const T bd = (lateral_diag((T)Dk, fw, fe, fs, fn) + fd) + fu;
        const T den = bd + fd * cprev;  // b_k - a_k c'_{k-1} with a_k = -fd
        // the stored (rounded) factors are the ones applied, here as in the sweeps
        const F inv_s = fac_put<F>(fixed ? T(0) : recip(den));
        const T inv = fac_get<T>(inv_s);
        const F cp_s = fac_put<F>(-fu * inv);
        const T cp = fac_get<T>(cp_s);
        const T y = rT - cprev * yprev;
        const T dp = y * inv;
        finv[g] = inv_s;
        fc[g] = cp_s;
        put_dprime<T, DSMEM>(dp, s_d, k, z + g);
        a2 += y * dp;
        cprev = cp;
        yprev = y;
        fd = fu;
        x_up = xc;
        K_up = Kc;
    };
    march<CHN, true>(nz, sb, prefetched, issue, plane, issue_next, [](int) {});
    v[2] = (double)a2;
    if (cr.valid) back_sweep<T, DSMEM>(cr, s_d, fc, z);
}

// ---- inner sweep C: one PCG iteration --------------------------------------
// With ap = alpha_{i-1} and bt = beta_i (ap zero in a cycle's first sweep, bt
// too unless the sweep continues the previous cycle's direction):
// z = z_prev - ap t_prev and p = z + bt p_prev at the own column and its four
// lateral neighbours (from the staged halo boxes) and at k+1; q = A p;
// t = M^-1 q by the stored factors (forward sweep in the march, back sweep
// after it); d += ap p_prev.  Writes z, p, t into the buffers other than
// `prev`, and v = {p.q, z.q, q.t, z.M z} (each column's sums taken in T).
// The values at k+1 (z, p, K and the vertical face coefficient) are carried
// to the next plane as its own.  The three forms of a sweep (a cycle's first
// without or with the previous direction, and the general one) are compiled
// separately: MODE 0 p = z, 1 p = z + bt p_prev, 2 z and p from t and p_prev.
template <int M_>
struct SweepMode {
    static constexpr int value = M_;
};

template <typename T, bool DSMEM, int TXC>
__device__ __forceinline__ void phase_C(const DevPtrs &P, int tile, int tile_next, bool prefetched, bool first_next,
                        bool keep_next, int prev_next, const ColumnRef &cr, const StencilW<T> &w, T ap, T bt,
                        bool first, bool keep_p, int prev, T *s_d, unsigned char *stage, StageBars &sb,
                        double (&v)[4]) {
    constexpr int CHN = Chunk<T>::inner;
    // the tile shape is a compile-time constant of each instantiation
    const Halo<T> H(TXC, TXC == 32 ? 5 : 4, TILE_THREADS / TXC);
    constexpr unsigned HB = halo_slot<T, CHN>();
    T *__restrict__ z_out = (T *)(prev ? P.z0 : P.z1);
    T *__restrict__ p_out = (T *)(prev ? P.p0 : P.p1);
    T *__restrict__ t_out = (T *)(prev ? P.t0 : P.t1);
    T *__restrict__ d = (T *)P.d;
    using F = typename Fac<T>::type;
    constexpr unsigned OB = own_bytes<T, CHN>(), OF = own_bytes<F, CHN>();
    const F *__restrict__ fc = (const F *)P.fc;
    const size_t BUF = StageSize<T>::buffer();
    auto buf = [&](int b) { return stage + b * BUF; };
    auto issue = [&](int st, int b) { issue_C<T>(P, tile, st, b, stage, sb, first, keep_p, prev); };
    auto issue_next = [&]() {
        if (tile_next < P.ntiles)
            issue_head<CHN>(P.dom[P.tiles[tile_next].dom].nz, [&](int st, int b) {
                issue_C<T>(P, tile_next, st, b, stage, sb, first_next, keep_next, prev_next);
            });
    };
    const int nz = cr.nz, hc = H.hc, oc = threadIdx.x;
    const FaceW<T> f = face_weights(cr, w);
    // carried down the column: this plane's z, p, K and upper face coefficient,
    // the plane above's p, the forward sweep's c'_{k-1} and y_{k-1}
    T zc = T(0), pc = T(0), Kc = T(0), fd = T(0), p_up = T(0), cprev = T(0), yprev = T(0);
    T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
    // 32-bit cell offsets (a handle holds fewer than 2^31 cells): fewer live
    // registers in the sweep than 64-bit indices
    unsigned g = (unsigned)cr.g0;
    const unsigned sxy = (unsigned)cr.sxy;
    auto sweep = [&](auto mode) {
        constexpr int MODE = decltype(mode)::value;
        auto zv = [&](const T *zz, const T *tt, int o) {
            if constexpr (MODE == 2) return zz[o] - ap * tt[o];
            else return zz[o];
        };
        auto pz = [&](T z, const T *pp, int o) {  // p from this iteration's z
            if constexpr (MODE == 0) return z;
            else return z + bt * pp[o];
        };
        auto plane = [&](int b, int pl, int k) {
            if (!cr.valid) return;
            const T *sz = (const T *)buf(b) + pl * H.plane;
            const T *st = (const T *)(buf(b) + HB) + pl * H.plane;
            const T *sp = (const T *)(buf(b) + 2 * HB) + pl * H.plane;
            const T *sK = (const T *)(buf(b) + 3 * HB) + pl * H.plane;
            const unsigned char *ob = buf(b) + 4 * HB;
            const T *ownD = (const T *)ob + pl * OWN_PLANE + oc;
            const F *ownI = (const F *)(ob + OB) + pl * OWN_PLANE + oc;
            const F *ownC = (const F *)(ob + OB + OF) + pl * OWN_PLANE + oc;
            const T *ownd = (const T *)(ob + OB + 2 * OF) + pl * OWN_PLANE + oc;
            if (k == 0) {
                zc = zv(sz, st, hc);
                pc = pz(zc, sp, hc);
                Kc = sK[hc];
            }
            const T Dk = ownD[0], inv = fac_get<T>(ownI[0]), cp = fac_get<T>(ownC[0]);
            T z_dn = T(0), p_dn = T(0), K_dn = T(0), fu = T(0);
            if (k + 1 < nz) {
                const T *nzz = sz + H.plane, *ntt = st + H.plane, *npp = sp + H.plane, *nK = sK + H.plane;
                if (pl + 1 == CHN) {
                    const unsigned char *nb = buf((b + 1) % STAGES);
                    nzz = (const T *)nb;
                    ntt = (const T *)(nb + HB);
                    npp = (const T *)(nb + 2 * HB);
                    nK = (const T *)(nb + 3 * HB);
                }
                z_dn = zv(nzz, ntt, hc);
                p_dn = pz(z_dn, npp, hc);
                K_dn = nK[hc];
                fu = f.z * (Kc + K_dn);
            }
            const T fw = f.w * (Kc + sK[hc - 1]), fe = f.e * (Kc + sK[hc + 1]);
            const T fs = f.s * (Kc + sK[hc - H.bw]), fn = f.n * (Kc + sK[hc + H.bw]);
            const T pw = pz(zv(sz, st, hc - 1), sp, hc - 1), pe = pz(zv(sz, st, hc + 1), sp, hc + 1);
            const T ps = pz(zv(sz, st, hc - H.bw), sp, hc - H.bw), pn = pz(zv(sz, st, hc + H.bw), sp, hc + H.bw);
            const bool fixed = Dk < T(0);  // Dirichlet cell: identity row, z = p = 0 there
            T q = Dk * pc + (fw * (pc - pw) + fe * (pc - pe)) + (fs * (pc - ps) + fn * (pc - pn)) +
                  (fd * (pc - p_up) + fu * (pc - p_dn));
            // z.M z with M = L D L^T from the stored factors: the column's sum of
            // (z_k + c'_k z_{k+1})^2 / inv_k (0 on a fixed cell, where inv = 0)
            const T u = zc + cp * z_dn;
            const T zMz = fixed ? T(0) : quot(u * u, inv);
            if (fixed) q = T(0);
            a0 += pc * q;
            a1 += zc * q;
            a3 += zMz;
            const T y = q - cprev * yprev;
            const T dp = y * inv;
            a2 += y * dp;
            z_out[g] = zc;
            p_out[g] = pc;
            if constexpr (MODE == 2) d[g] = ownd[0] + ap * sp[hc];
            else d[g] = T(0);
            put_dprime<T, DSMEM>(dp, s_d, k, t_out + g);
            cprev = cp;
            yprev = y;
            p_up = pc;
            zc = z_dn;
            pc = p_dn;
            Kc = K_dn;
            fd = fu;
            g += sxy;
        };
        march<CHN, true>(nz, sb, prefetched, issue, plane, issue_next,
                         [&](int st) { prefetch_C<T>(P, tile, st, first, keep_p, prev); });
    };
    if (!first) sweep(SweepMode<2>{});
    else if (keep_p) sweep(SweepMode<1>{});
    else sweep(SweepMode<0>{});
    v[0] = (double)a0;
    v[1] = (double)a1;
    v[2] = (double)a2;
    v[3] = (double)a3;
    if (cr.valid) back_sweep<T, DSMEM>(cr, s_d, fc, t_out);
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
        c.alpha = 0.0;
        // A later cycle continues the direction of the previous one: the true
        // residual replaces the recursive one (z = M^-1 r from phase R) and
        // p = z + beta p with beta = rho_true / rho_last ("reliable update"),
        // so refinement does not discard the Krylov space built so far.
        c.keep_p = (c.total_iter > 0 && c.rho_last > 0.0) ? 1 : 0;
        c.beta = c.keep_p ? v[2] / c.rho_last : 0.0;
        // the inner solve reduces r.M^-1 r by inner_tol^2 (mixed mode), or far
        // enough that ||r|| should meet the outer tolerance (half of it, with
        // the M^-1-norm standing in for the 2-norm); R checks the true residual
        c.inner_target2 = v[2] * fmax(D.inner_tol * D.inner_tol, 0.25 * tol2 * bb / rr64);
    }
}

__device__ __forceinline__ void stop_inner(const DevPtrs &P, KrylovCtrl &c) {
    c.inner_active = 0;
    atomicSub(&P.gctrl->n_inner_active, 1);
}

// Shared memory of the persistent 3D solve: [d' of the column solves (float
// only)][STAGES staging buffers], the staging buffers 128-byte aligned for the
// TMA, and the stage mbarriers (initialised here, once per launch).
template <typename T>
struct SolveSmem {
    T *s_d;
    unsigned char *stage;
};

template <typename T, bool DSMEM>
__device__ __forceinline__ SolveSmem<T> solve_smem(const DevPtrs &P, unsigned char *smem_raw, uint64_t *s_bar) {
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    const size_t dprime_bytes = DSMEM ? (size_t)P.smem_nz * TILE_THREADS * sizeof(T) : 0;
    if (threadIdx.x == 0) {
        for (int q = 0; q < STAGES; ++q) mbar_init(&s_bar[q], 1);
        mbar_fence_init();
    }
    __syncthreads();
    return SolveSmem<T>{reinterpret_cast<T *>(base), base + ((dprime_bytes + 127) & ~(size_t)127)};
}

// The whole linear solve of one Picard iteration for every active domain (the
// body of k_krylov, also run by k_step).  Returns false when a grid barrier
// gave up (the handle's error flag is set); the block must then return.
// TXC: the tile width when every domain of the handle has the same tile shape
// (the sweeps are then compiled for it), 0 when shapes differ by domain (each
// tile is dispatched to the sweep of its shape).
template <typename T, bool DSMEM, int TXC>
__device__ __forceinline__ bool krylov_solve(const DevPtrs &P, const SolveSmem<T> &sm, StageBars &sb) {
    T *s_d = sm.s_d;
    unsigned char *stage_raw = sm.stage;
    // every error exit first lets this block's in-flight stage copies land
    auto fail = [&]() {
        if (threadIdx.x == 0) sb.drain();
        return false;
    };
    // next tile of this block with an active domain (stride gridDim.x)
    auto next_outer = [&](int t) {
        while (t < P.ntiles && !ldcg(&P.kctrl[P.tiles[t].dom].active)) t += gridDim.x;
        return t;
    };
    auto next_inner = [&](int t) {
        while (t < P.ntiles && !ldcg(&P.kctrl[P.tiles[t].dom].inner_active)) t += gridDim.x;
        return t;
    };
    auto weights = [&](int dom) {
        const DomainDesc &D = P.dom[dom];
        return StencilW<T>{(T)(1.0 / (D.dx * D.dx)), (T)(1.0 / (D.dy * D.dy)), (T)(1.0 / (D.dz * D.dz))};
    };
    for (;;) {
        // ---- R: outer residual
        {
            bool pre = false;
            for (int t = next_outer(blockIdx.x); t < P.ntiles;) {
                const int tn = next_outer(t + gridDim.x);
                const int dom = P.tiles[t].dom;
                const ColumnRef cr = column_of(P, t);
                double v[3] = {0.0, 0.0, 0.0};
                if constexpr (TXC != 0)
                    phase_R<T, DSMEM, TXC>(P, t, tn, pre, cr, weights(dom), s_d, stage_raw, sb, v);
                else if (cr.tx == TILE_X)
                    phase_R<T, DSMEM, TILE_X>(P, t, tn, pre, cr, weights(dom), s_d, stage_raw, sb, v);
                else
                    phase_R<T, DSMEM, 16>(P, t, tn, pre, cr, weights(dom), s_d, stage_raw, sb, v);
                pre = tn < P.ntiles;
                if (domain_reduce<3>(P, t, dom, 0, v) && threadIdx.x == 0) finalize_R(P, dom, v);
                t = tn;
            }
        }
        if (!grid_sync(P.barrier)) return fail();
        if (ldcg(&P.gctrl->n_active) == 0) break;
        // ---- inner PCG: one sweep and one grid barrier per iteration
        // A domain's control record (inner_active, parity, first_inner, alpha,
        // beta) changes only when its last tile of a sweep finishes, after
        // every tile of it in that sweep has been scheduled, so within a sweep
        // a block reads it once per domain rather than once per tile.
        struct Ctl {
            int dom, active, parity;
            bool first, keep_p;
            double alpha, beta;
        };
        auto ctl_load = [&](Ctl &c, int dom) {
            if (c.dom == dom) return;
            const KrylovCtrl *k = &P.kctrl[dom];
            c.dom = dom;
            c.active = ldcg(&k->inner_active);
            c.parity = ldcg(&k->parity);
            c.first = ldcg(&k->first_inner) != 0;
            c.keep_p = ldcg(&k->keep_p) != 0;
            c.alpha = ldcg(&k->alpha);
            c.beta = ldcg(&k->beta);
        };
        // next tile of this block (stride gridDim.x) whose domain iterates
        auto next_live = [&](Ctl &c, int t) {
            for (; t < P.ntiles; t += gridDim.x) {
                const int dom = P.tiles[t].dom;
                if (dom != c.dom) ctl_load(c, dom);
                if (c.active) break;
            }
            return t;
        };
        while (ldcg(&P.gctrl->n_inner_active) > 0) {
            bool pre = false;
            Ctl cc{-1, 0, 0, false, false, 0.0, 0.0}, cn{-1, 0, 0, false, false, 0.0, 0.0};
            for (int t = next_live(cc, blockIdx.x); t < P.ntiles;) {
                const int tn = next_live(cn, t + gridDim.x);
                const int dom = P.tiles[t].dom;
                ctl_load(cc, dom);
                const ColumnRef cr = column_of(P, t);
                const DomainDesc &D = P.dom[dom];
                const bool first_n = tn < P.ntiles ? cn.first : false;
                const bool keep_n = tn < P.ntiles ? cn.keep_p : false;
                const int prev_n = tn < P.ntiles ? cn.parity : 0;
                double v[4] = {0.0, 0.0, 0.0, 0.0};
                if constexpr (TXC != 0)
                    phase_C<T, DSMEM, TXC>(P, t, tn, pre, first_n, keep_n, prev_n, cr, weights(dom), (T)cc.alpha,
                                           (T)cc.beta, cc.first, cc.keep_p, cc.parity, s_d, stage_raw, sb, v);
                else if (cr.tx == TILE_X)
                    phase_C<T, DSMEM, TILE_X>(P, t, tn, pre, first_n, keep_n, prev_n, cr, weights(dom),
                                              (T)cc.alpha, (T)cc.beta, cc.first, cc.keep_p, cc.parity, s_d,
                                              stage_raw, sb, v);
                else
                    phase_C<T, DSMEM, 16>(P, t, tn, pre, first_n, keep_n, prev_n, cr, weights(dom), (T)cc.alpha,
                                          (T)cc.beta, cc.first, cc.keep_p, cc.parity, s_d, stage_raw, sb, v);
                pre = tn < P.ntiles;
                if (domain_reduce<4>(P, t, dom, 0, v) && threadIdx.x == 0) {
                    KrylovCtrl &c = P.kctrl[dom];
                    const double sigma = v[0], mu = v[1], nu = v[2], rho = v[3];
                    const double alpha = rho / sigma;
                    const double rho_next = rho - 2.0 * alpha * mu + alpha * alpha * nu;
                    const bool bad = !(sigma > 0.0) || isinf(sigma) || !(rho > 0.0) || !(rho_next == rho_next);
                    c.alpha = bad ? 0.0 : alpha;  // a broken iteration leaves x alone
                    c.beta = bad ? 0.0 : rho_next / rho;
                    c.rz = rho_next;
                    c.rho_last = bad ? 0.0 : rho;
                    c.parity ^= 1;
                    c.first_inner = 0;
                    c.inner_iter += 1;
                    c.total_iter += 1;
                    if (bad || rho_next <= c.inner_target2 || c.inner_iter >= D.inner_maxiter ||
                        c.total_iter >= D.krylov_maxiter)
                        stop_inner(P, c);
                }
                t = tn;
            }
            if (!grid_sync(P.barrier)) return fail();
        }
        // ---- U: x += d + alpha p (the last iteration's pending update)
        for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
            const int dom = P.tiles[t].dom;
            const KrylovCtrl *kc = &P.kctrl[dom];
            if (!ldcg(&kc->active) || ldcg(&kc->first_inner)) continue;
            const ColumnRef cr = column_of(P, t);
            if (!cr.valid) continue;
            const T *__restrict__ d = (const T *)P.d;
            const T *__restrict__ p = (const T *)(ldcg(&kc->parity) ? P.p1 : P.p0);
            const double a = ldcg(&kc->alpha);
            double *__restrict__ x = P.x;
#pragma unroll 8
            for (int k = 0; k < cr.nz; ++k) {
                const long long g = cr.g0 + (long long)k * cr.sxy;
                x[g] += (double)d[g] + a * (double)p[g];
            }
        }
        if (!grid_sync(P.barrier)) return fail();
    }
    return true;
}

template <typename T, int TXC>
__global__ void __launch_bounds__(TILE_THREADS, sizeof(T) == 4 ? KRYLOV_BLOCKS_F32 : KRYLOV_BLOCKS_F64)
    k_krylov(DevPtrs P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[STAGES];
    constexpr bool DSMEM = sizeof(T) == 4 && KRYLOV_DSMEM_F32;
    const SolveSmem<T> sm = solve_smem<T, DSMEM>(P, smem_raw, s_bar);
    StageBars sb{s_bar, 0u, P.barrier, 0u};
    krylov_solve<T, DSMEM, TXC>(P, sm, sb);
}


// ---------------------------------------------------------- Picard check
// Max of |(psi^{m+1}-psi^m)/psi^{m+1}| (or the theta / absolute variants) per
// domain, then the convergence decision and iteration bookkeeping.
__device__ __forceinline__ void picard_check_tile(const DevPtrs &P, int tile) {
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
        if (c.done) atomicSub(&P.gctrl->n_picard, 1);  // k_step's loop ends at zero
        dg.krylov_iters_total += kc.total_iter;
        dg.refine_iters_total += kc.cycles;
        dg.krylov_iters_last += kc.total_iter;
        dg.picard_err_last = v[0];
    }
}

__global__ void __launch_bounds__(TILE_THREADS) k_picard_check(DevPtrs P) {
    picard_check_tile(P, blockIdx.x);
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
__device__ __forceinline__ void epilogue_tile(const DevPtrs &P, int tile) {
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    const ColumnRef cr = column_of(P, tile);
    // v: 0 sum dtheta*dz, 1 dt*sum ssflux, 2 sum transp, 3 dt*boundary flux,
    //    4 storage (telescoping), 5 dt*q_top, 6 dt*q_bottom, 7 rain, 8 nonfinite
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    unsigned long long bsig = 0;
    const int step_now = P.pctrl[td.dom].step;
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
            if (records(D, BR_SATURATION)) bsig += branch_mix(step_now * 64 + 63, BR_SATURATION, g, band3(xn, 0.0, 1e-9));
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
        // a Dirichlet bottom has no prescribed flux (the reference keeps q_b out
        // of its balance there too)
        const double qt = P.qtop[cr.c];
        const double qb = (D.has_dirichlet && P.dir_b[cr.c]) ? 0.0 : P.bcqb[cr.c];
        v[3] += (qb - qt) * dt;
        v[5] += qt * dt;
        v[6] += qb * dt;
        v[7] += P.ppt[cr.c] * D.sub_frac / 1000.0;
        // infiltration / ponding, then waterdepth <- ph
        const double ph = fmax(P.hpoten[cr.c] - qt * dt, 0.0);
        P.ph[cr.c] = ph;
        P.h[cr.c] = ph;
        if (records(D, BR_PONDCLIP))
            bsig += branch_mix(step_now, BR_PONDCLIP, cr.c,
                               band3(P.hpoten[cr.c], qt * dt, rel_band(P.hpoten[cr.c], qt * dt, 1e-15)));
    }
    if (D.record_branches) branch_commit(&P.diag[td.dom].branch_sig, bsig);
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
        if (records(D, BR_PICARD))
            atomicAdd(&dg.branch_sig, branch_mix(pc.step, BR_PICARD, td.dom, (unsigned)pc.iter));
        pc.step += D.step_advance;
    }
}

template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) k_epilogue(DevPtrs P) {
    epilogue_tile<T>(P, blockIdx.x);
}

// One whole subsurface step (SubsurfaceFlowModel, src/subsurface.cu:686-847)
// in one persistent launch: the prologue, up to maxiter Picard iterations of
// assembly (+ the Dirichlet passes), linear solve and convergence check, and
// the epilogue, as phases separated by grid barriers.  Each phase runs the same
// per-tile code as the separate kernels (prologue_tile ... epilogue_tile,
// krylov_solve) in the same order, so the results are those of the
// launch-per-kernel sequence bit for bit; the loop ends as soon as every
// domain's Picard iteration is done.
// The phases other than the solve are called, not inlined, so that each gets
// its own register allocation under the kernel's limit and the solve loop
// keeps the registers it has in k_krylov.
enum StepPhase { PH_PROLOGUE, PH_ASSEMBLE, PH_DIR_FIXED, PH_DIR_ROWS, PH_CHECK, PH_EPILOGUE };

template <typename T, int PH>
__device__ __noinline__ void step_phase(const DevPtrs &P) {
    for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
        if constexpr (PH == PH_PROLOGUE) prologue_tile(P, t);
        else if constexpr (PH == PH_ASSEMBLE) assemble_tile<T>(P, t);
        else if constexpr (PH == PH_DIR_FIXED) dir_fixed_tile<T>(P, t);
        else if constexpr (PH == PH_DIR_ROWS) dir_rows_tile<T>(P, t);
        else if constexpr (PH == PH_CHECK) picard_check_tile(P, t);
        else epilogue_tile<T>(P, t);
    }
}

template <typename T, int TXC>
__global__ void __launch_bounds__(TILE_THREADS, sizeof(T) == 4 ? KRYLOV_BLOCKS_F32 : KRYLOV_BLOCKS_F64)
    k_step(const __grid_constant__ DevPtrs P, int maxiter, int dirichlet) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[STAGES];
    constexpr bool DSMEM = sizeof(T) == 4 && KRYLOV_DSMEM_F32;
    const SolveSmem<T> sm = solve_smem<T, DSMEM>(P, smem_raw, s_bar);
    StageBars sb{s_bar, 0u, P.barrier, 0u};
    step_phase<T, PH_PROLOGUE>(P);
    if (!grid_sync(P.barrier)) return;
    for (int m = 0; m < maxiter; ++m) {
        step_phase<T, PH_ASSEMBLE>(P);
        if (!grid_sync(P.barrier)) return;
        if (dirichlet) {
            step_phase<T, PH_DIR_FIXED>(P);
            if (!grid_sync(P.barrier)) return;
            step_phase<T, PH_DIR_ROWS>(P);
            if (!grid_sync(P.barrier)) return;
        }
        if (!krylov_solve<T, DSMEM, TXC>(P, sm, sb)) return;
        step_phase<T, PH_CHECK>(P);
        if (!grid_sync(P.barrier)) return;
        if (ldcg(&P.gctrl->n_picard) == 0) break;
    }
    step_phase<T, PH_EPILOGUE>(P);
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
        closure(D, P.psin[g], a, n, P.ksat[g], th, Kv, C);
        out[g] = which == 0 ? th : (which == 1 ? Kv : C);
    }
}

// Step state save / restore for time-step halving, one block per tile.
__global__ void __launch_bounds__(TILE_THREADS) k_step_state(DevPtrs P, StepState S) {
    const TileDesc td = P.tiles[blockIdx.x];
    const int act = S.action[td.dom];
    if (act == 0) return;
    const bool save = act == 1;
    const DomainDesc &D = P.dom[td.dom];
    if (blockIdx.x == D.tile_begin && threadIdx.x == 0) {
        if (save) S.diag[td.dom] = P.diag[td.dom];
        else P.diag[td.dom] = S.diag[td.dom];
    }
    const ColumnRef cr = column_of(P, blockIdx.x);
    if (!cr.valid) return;
    auto mv = [&](double *handle, double *copy, long long i) {
        if (save) copy[i] = handle[i];
        else handle[i] = copy[i];
    };
    mv(P.ktop, S.ktop, cr.c);
    mv(P.ph, S.ph, cr.c);
    mv(P.h, S.h, cr.c);
    mv(P.H, S.H, cr.c);
    long long g = cr.g0;
    for (int k = 0; k < cr.nz; ++k, g += cr.sxy) {
        mv(P.psin, S.psin, g);
        mv(P.thetan, S.thetan, g);
        if (!save) {
            P.psim[g] = S.psin[g];
            P.x[g] = S.psin[g];
        }
    }
}

__global__ void k_advance_step(DevPtrs P) {
    for (int d = threadIdx.x; d < P.ndom; d += blockDim.x) P.pctrl[d].step += 1;
}

// ------------------------------------------------------------- launchers
cudaError_t launch_step_state(const DevPtrs &P, const StepState &S, cudaStream_t s) {
    k_step_state<<<P.ntiles, TILE_THREADS, 0, s>>>(P, S);
    return cudaGetLastError();
}

cudaError_t launch_advance_step(const DevPtrs &P, cudaStream_t s) {
    k_advance_step<<<1, 256, 0, s>>>(P);
    return cudaGetLastError();
}

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

cudaError_t launch_dirichlet(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s) {
    if (L.mixed) {
        k_dir_fixed<float><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
        k_dir_rows<float><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    } else {
        k_dir_fixed<double><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
        k_dir_rows<double><<<P.ntiles, TILE_THREADS, 0, s>>>(P);
    }
    return cudaGetLastError();
}

// The instantiation for the handle's tile shapes: one shape for every domain
// (L.uniform_tx 32 or 16) or a mix (0).
template <int TXC>
const void *krylov_fn(int mixed) {
    return mixed ? (const void *)k_krylov<float, TXC> : (const void *)k_krylov<double, TXC>;
}
template <int TXC>
const void *step_fn(int mixed) {
    return mixed ? (const void *)k_step<float, TXC> : (const void *)k_step<double, TXC>;
}
const void *krylov_kernel(const LaunchCfg &L, int uniform_tx) {
    return uniform_tx == TILE_X ? krylov_fn<TILE_X>(L.mixed) : uniform_tx == 16 ? krylov_fn<16>(L.mixed)
                                                                                : krylov_fn<0>(L.mixed);
}
const void *step_kernel(const LaunchCfg &L, int uniform_tx) {
    return uniform_tx == TILE_X ? step_fn<TILE_X>(L.mixed) : uniform_tx == 16 ? step_fn<16>(L.mixed)
                                                                              : step_fn<0>(L.mixed);
}

cudaError_t launch_krylov(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s) {
    DevPtrs args = P;
    void *kargs[] = {&args};
    const int blocks = L.krylov_per_sm * L.sms;
    const int grid = blocks < P.ntiles ? blocks : P.ntiles;
    return cudaLaunchCooperativeKernel(krylov_kernel(L, L.uniform_tx), dim3(grid), dim3(TILE_THREADS), kargs,
                                       (size_t)L.smem_3d, s);
}

cudaError_t launch_step(const DevPtrs &P, const LaunchCfg &L, int maxiter, int dirichlet, cudaStream_t s) {
    DevPtrs args = P;
    void *kargs[] = {&args, &maxiter, &dirichlet};
    const int blocks = (L.krylov_per_sm < L.step_per_sm ? L.krylov_per_sm : L.step_per_sm) * L.sms;
    const int grid = blocks < P.ntiles ? blocks : P.ntiles;
    return cudaLaunchCooperativeKernel(step_kernel(L, L.uniform_tx), dim3(grid), dim3(TILE_THREADS), kargs,
                                       (size_t)L.smem_3d, s);
}

cudaError_t configure_3d(LaunchCfg &L, int device, int ntiles) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    const size_t elt = L.mixed ? sizeof(float) : sizeof(double);
    const size_t dprime = (L.mixed && KRYLOV_DSMEM_F32) ? elt * (size_t)L.nz_max * TILE_THREADS : 0;
    const size_t stage = L.mixed ? StageSize<float>::bytes() : StageSize<double>::bytes();
    L.smem_3d = (int)(128 + ((dprime + 127) & ~(size_t)127) + stage);
    // every instantiation (tile shapes 32, 16 and mixed) takes the same shared
    // memory; the co-resident block counts are the smallest over them
    int per_sm = 1 << 30, step_sm = 1 << 30;
    for (int u : {TILE_X, 16, 0}) {
        for (int fused = 0; fused < 2; ++fused) {
            const void *fn = fused ? step_kernel(L, u) : krylov_kernel(L, u);
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, L.smem_3d);
            if (e != cudaSuccess) return e;
            int n = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, TILE_THREADS, L.smem_3d);
            if (e != cudaSuccess) return e;
            int &acc = fused ? step_sm : per_sm;
            acc = n < acc ? n : acc;
        }
    }
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    L.coop_blocks_3d = per_sm * prop.multiProcessorCount;
    L.sms = prop.multiProcessorCount;
    L.krylov_per_sm_max = per_sm;
    L.krylov_per_sm = per_sm;
    L.step_per_sm = step_sm < per_sm ? step_sm : per_sm;
    if (L.step_per_sm < 1) return cudaErrorInvalidConfiguration;
    // one launch per subsurface step by default, where the fused kernel keeps
    // the Krylov kernel's occupancy
    L.fused_step = L.step_per_sm >= L.krylov_per_sm ? 1 : 0;
    (void)ntiles;
    return cudaSuccess;
}
