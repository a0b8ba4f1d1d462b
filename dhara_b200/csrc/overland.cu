// overland.cu -- 2D diffusive-wave overland kernels (the reference's
// OverlandFlowModel, src/overland.cu:387-419).
//
//   WaterElevationOverland (33-45) + UpdateKOverland (193-368)
//     + SetUpLinearSystemsOverland (65-189)                  -> k_olf_setup
//   CUSP CG on the 5-diagonal matrix (410-411)               -> k_olf_solve
//   WaterDepthOverland (371-383) + ph <- waterdepth (417)     -> k_olf_finish
//
// The boundary ring is a fixed-elevation (identity) row in the reference.  Its
// value is known (H_old), so it is eliminated symmetrically: ring residuals and
// directions are zero and only interior rows iterate.  That system has the
// same solution as the reference's, and its interior block is symmetric, so
// Jacobi-preconditioned CG applies.  Interior rows use the reference's
// row-owned conductances kw, ke, ks, kn exactly.
#include "device_common.cuh"

__device__ __forceinline__ bool is_ring(int i, int j, int nx, int ny) {
    return i == 0 || j == 0 || i == nx - 1 || j == ny - 1;
}

// Manning conductance of one face (src/overland.cu:279-297 and the three
// analogous blocks): the depth test is upwinded on the water elevation.
__device__ __forceinline__ double manning_k(double Hnb, double hnb, double mnb, double Hc, double hc,
                                            double mc, double S, const DomainDesc &D) {
    const double hup = (Hnb > Hc) ? hnb : hc;
    if (hup > D.hmin && (hnb + hc) / 2. > D.hmin && fabs(S) > D.delta)
        return pow((hnb + hc) / 2., 5. / 3.) / (0.5 * (mnb + mc) * sqrt(S));
    return D.K0;
}

__global__ void __launch_bounds__(TILE_THREADS) k_olf_setup(DevPtrs P, long long ctot) {
    const int tile = blockIdx.x;
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    if (threadIdx.x == 0 && tile == D.tile_begin) {
        OverlandCtrl &oc = P.octrl[td.dom];
        oc.active = 1;
        oc.iter = 0;
        oc.parity = 0;
        oc.pad = 1;  // first inner iteration
        atomicAdd(&P.gctrl->n_olf_active, 1);
    }
    const ColumnRef cr = column_of(P, tile);
    if (!cr.valid) return;
    const int N = cr.nx, M = cr.ny, i = cr.i, j = cr.j;
    const long long I = cr.c;
    const double *h = P.h, *z = P.ztopo, *mann = P.mann;
    auto Hs = [&](long long q) { return h[q] + z[q]; };
    const double h_ = h[I], Hs_ = Hs(I), mann_ = mann[I];
    P.H[I] = Hs_;
    P.olf_b[I] = Hs_;
    double kw = 0, ke = 0, ks = 0, kn = 0;
    if (!is_ring(i, j, N, M)) {
        const double h_p1 = h[I + 1], Hs_p1 = Hs(I + 1), mann_p1 = mann[I + 1];
        const double h_m1 = h[I - 1], Hs_m1 = Hs(I - 1), mann_m1 = mann[I - 1];
        const double h_pN = h[I + N], Hs_pN = Hs(I + N), mann_pN = mann[I + N];
        const double h_mN = h[I - N], Hs_mN = Hs(I - N), mann_mN = mann[I - N];
        const double Hs_pNp1 = Hs(I + N + 1), Hs_pNm1 = Hs(I + N - 1);
        const double Hs_mNp1 = Hs(I - N + 1), Hs_mNm1 = Hs(I - N - 1);
        const double dx = D.dx, dy = D.dy;
        const double Sse = sqrt(pow((Hs_p1 - Hs_) / dx, 2.) +
                                pow((Hs_pNp1 + Hs_pN - Hs_mNp1 - Hs_mN) / (4 * dy), 2.));
        ke = manning_k(Hs_p1, h_p1, mann_p1, Hs_, h_, mann_, Sse, D);
        const double Ssw = sqrt(pow((Hs_ - Hs_m1) / dx, 2.) +
                                pow((Hs_pN + Hs_pNm1 - Hs_mN - Hs_mNm1) / (4 * dy), 2.));
        kw = manning_k(Hs_m1, h_m1, mann_m1, Hs_, h_, mann_, Ssw, D);
        const double Ssn = sqrt(pow((Hs_pN - Hs_) / dy, 2.) +
                                pow((Hs_pNp1 + Hs_p1 - Hs_pNm1 - Hs_m1) / (4 * dx), 2.));
        kn = manning_k(Hs_pN, h_pN, mann_pN, Hs_, h_, mann_, Ssn, D);
        const double Sss = sqrt(pow((Hs_ - Hs_mN) / dy, 2.) +
                                pow((Hs_p1 + Hs_mNp1 - Hs_m1 - Hs_mNm1) / (4 * dx), 2.));
        ks = manning_k(Hs_mN, h_mN, mann_mN, Hs_, h_, mann_, Sss, D);
    }
    P.olf_k[0 * ctot + I] = kw;
    P.olf_k[1 * ctot + I] = ke;
    P.olf_k[2 * ctot + I] = ks;
    P.olf_k[3 * ctot + I] = kn;
}

struct OlfRow {
    double kw, ke, ks, kn, diag, cx, cy;
    bool ring;
};

__device__ __forceinline__ OlfRow olf_row(const DevPtrs &P, const ColumnRef &cr, const DomainDesc &D,
                                          long long ctot) {
    OlfRow r;
    r.ring = is_ring(cr.i, cr.j, cr.nx, cr.ny);
    r.cx = D.dt / (D.dx * D.dx);
    r.cy = D.dt / (D.dy * D.dy);
    r.kw = P.olf_k[0 * ctot + cr.c];
    r.ke = P.olf_k[1 * ctot + cr.c];
    r.ks = P.olf_k[2 * ctot + cr.c];
    r.kn = P.olf_k[3 * ctot + cr.c];
    r.diag = 1.0 + r.cx * (r.ke + r.kw) + r.cy * (r.kn + r.ks);
    return r;
}

template <typename Get>
__device__ __forceinline__ double olf_apply(const OlfRow &w, const ColumnRef &cr, Get v) {
    const long long I = cr.c;
    const double c = v(I);
    return c + w.cx * (w.ke * (c - v(I + 1)) + w.kw * (c - v(I - 1))) +
           w.cy * (w.kn * (c - v(I + cr.nx)) + w.ks * (c - v(I - cr.nx)));
}

// Persistent cooperative Jacobi-PCG over all domains' interior cells.
__global__ void __launch_bounds__(TILE_THREADS) k_olf_solve(DevPtrs P, long long ctot) {
    double *x = P.H, *r = P.olf_r, *z = P.olf_z;
    // R: r = b - A x, z = r / diag
    for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
        const int dom = P.tiles[t].dom;
        if (!ldcg(&P.octrl[dom].active)) continue;
        const ColumnRef cr = column_of(P, t);
        const DomainDesc &D = P.dom[dom];
        double v[3] = {0, 0, 0};  // rr, bb, rz
        if (cr.valid) {
            const double bI = P.olf_b[cr.c];
            v[1] = bI * bI;
            const OlfRow w = olf_row(P, cr, D, ctot);
            double rI = 0.0, zI = 0.0;
            if (!w.ring) {
                rI = bI - olf_apply(w, cr, [&](long long q) { return x[q]; });
                zI = rI / w.diag;
            }
            r[cr.c] = rI;
            z[cr.c] = zI;
            v[0] = rI * rI;
            v[2] = rI * zI;
        }
        if (domain_reduce<3>(P, t, dom, 3, v) && threadIdx.x == 0) {
            OverlandCtrl &c = P.octrl[dom];
            c.bb = v[1];
            c.rr = v[0];
            c.rz = v[2];
            const double tol2 = D.overland_tol * D.overland_tol;
            if (v[0] <= tol2 * v[1] || c.iter >= D.overland_maxiter || !(v[0] == v[0])) {
                c.active = 0;
                atomicSub(&P.gctrl->n_olf_active, 1);
            }
        }
    }
    if (!grid_sync(P.barrier)) return;
    while (ldcg(&P.gctrl->n_olf_active) > 0) {
        // A: p = z + beta p_old, partial p.Ap
        for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
            const int dom = P.tiles[t].dom;
            const OverlandCtrl *oc = &P.octrl[dom];
            if (!ldcg(&oc->active)) continue;
            const ColumnRef cr = column_of(P, t);
            const DomainDesc &D = P.dom[dom];
            const int parity = ldcg(&oc->parity);
            const bool first = ldcg(&oc->pad) != 0;
            const double beta = ldcg(&oc->beta);
            const double *pold = parity ? P.olf_p1 : P.olf_p0;
            double *pnew = parity ? P.olf_p0 : P.olf_p1;
            double v[1] = {0};
            if (cr.valid) {
                const OlfRow w = olf_row(P, cr, D, ctot);
                auto pv = [&](long long q) { return first ? z[q] : z[q] + beta * pold[q]; };
                const double pI = w.ring ? 0.0 : pv(cr.c);
                if (!w.ring) v[0] = pI * olf_apply(w, cr, pv);
                pnew[cr.c] = pI;
            }
            if (domain_reduce<1>(P, t, dom, 3, v) && threadIdx.x == 0) {
                OverlandCtrl &c = P.octrl[dom];
                c.pAp = v[0];
                c.alpha = c.rz / v[0];
                c.parity ^= 1;
                if (!(v[0] > 0.0)) {
                    c.active = 0;
                    atomicSub(&P.gctrl->n_olf_active, 1);
                }
            }
        }
        if (!grid_sync(P.barrier)) return;
        // B: x += alpha p, r -= alpha A p, z = r / diag
        for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
            const int dom = P.tiles[t].dom;
            const OverlandCtrl *oc = &P.octrl[dom];
            if (!ldcg(&oc->active)) continue;
            const ColumnRef cr = column_of(P, t);
            const DomainDesc &D = P.dom[dom];
            const int parity = ldcg(&oc->parity);
            const double alpha = ldcg(&oc->alpha);
            const double *p = parity ? P.olf_p1 : P.olf_p0;
            double v[2] = {0, 0};
            if (cr.valid) {
                const OlfRow w = olf_row(P, cr, D, ctot);
                if (!w.ring) {
                    const double Ap = olf_apply(w, cr, [&](long long q) { return p[q]; });
                    x[cr.c] += alpha * p[cr.c];
                    const double rI = r[cr.c] - alpha * Ap;
                    const double zI = rI / w.diag;
                    r[cr.c] = rI;
                    z[cr.c] = zI;
                    v[0] = rI * rI;
                    v[1] = rI * zI;
                }
            }
            if (domain_reduce<2>(P, t, dom, 3, v) && threadIdx.x == 0) {
                OverlandCtrl &c = P.octrl[dom];
                c.rr = v[0];
                c.beta = v[1] / c.rz;
                c.rz = v[1];
                c.pad = 0;
                c.iter += 1;
                const double tol2 = D.overland_tol * D.overland_tol;
                if (v[0] <= tol2 * c.bb || c.iter >= D.overland_maxiter || !(v[0] == v[0])) {
                    c.active = 0;
                    atomicSub(&P.gctrl->n_olf_active, 1);
                }
            }
        }
        if (!grid_sync(P.barrier)) return;
    }
}

// h = max(H - z, 0), ph <- h, plus the exact accounting of what the scheme
// does to the water budget: water that flowed into the fixed ring, and water
// created by the clip where the implicit solve left H below the ground.
__global__ void __launch_bounds__(TILE_THREADS) k_olf_finish(DevPtrs P, long long ctot) {
    const int tile = blockIdx.x;
    const TileDesc td = P.tiles[tile];
    const DomainDesc &D = P.dom[td.dom];
    if (tile == 0 && threadIdx.x == 0) P.gctrl->n_olf_active = 0;
    const ColumnRef cr = column_of(P, tile);
    double v[3] = {0, 0, 0};  // boundary out, clip, ponded
    if (cr.valid) {
        const long long I = cr.c;
        const double H = P.H[I];
        const double d = H - P.ztopo[I];
        const double hn = fmax(d, 0.0);
        P.h[I] = hn;
        P.ph[I] = hn;
        if (d < 0) v[1] = -d;
        v[2] = hn;
        if (!is_ring(cr.i, cr.j, cr.nx, cr.ny)) {
            const OlfRow w = olf_row(P, cr, D, ctot);
            if (cr.i == 1) v[0] += w.cx * w.kw * (H - P.H[I - 1]);
            if (cr.i == cr.nx - 2) v[0] += w.cx * w.ke * (H - P.H[I + 1]);
            if (cr.j == 1) v[0] += w.cy * w.ks * (H - P.H[I - cr.nx]);
            if (cr.j == cr.ny - 2) v[0] += w.cy * w.kn * (H - P.H[I + cr.nx]);
        }
    }
    if (domain_reduce<3>(P, tile, td.dom, 3, v) && threadIdx.x == 0) {
        DevDiag &dg = P.diag[td.dom];
        const OverlandCtrl &oc = P.octrl[td.dom];
        dg.olf_out_cum += v[0];
        dg.olf_clip_cum += v[1];
        dg.ponded = v[2];
        dg.overland_iters_total += oc.iter;
        const double tol2 = D.overland_tol * D.overland_tol;
        if (!(oc.rr <= tol2 * oc.bb)) dg.overland_nonconverged += 1;
    }
}

cudaError_t launch_overland_setup(const DevPtrs &P, long long ctot, cudaStream_t s) {
    k_olf_setup<<<P.ntiles, TILE_THREADS, 0, s>>>(P, ctot);
    return cudaGetLastError();
}

cudaError_t launch_overland_solve(const DevPtrs &P, const LaunchCfg &L, long long ctot, cudaStream_t s) {
    DevPtrs args = P;
    long long c = ctot;
    void *kargs[] = {&args, &c};
    const int grid = L.coop_blocks_2d < P.ntiles ? L.coop_blocks_2d : P.ntiles;
    return cudaLaunchCooperativeKernel((const void *)k_olf_solve, dim3(grid), dim3(TILE_THREADS), kargs, 0,
                                       s);
}

cudaError_t launch_overland_finish(const DevPtrs &P, long long ctot, cudaStream_t s) {
    k_olf_finish<<<P.ntiles, TILE_THREADS, 0, s>>>(P, ctot);
    return cudaGetLastError();
}

cudaError_t configure_2d(LaunchCfg &L, int device) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_olf_solve, TILE_THREADS, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    L.coop_blocks_2d = per_sm * prop.multiProcessorCount;
    return cudaSuccess;
}
