// overland.cu -- 2D diffusive-wave overland kernels (the reference's
// OverlandFlowModel, src/overland.cu:387-419).
//
//   WaterElevationOverland (33-45) + UpdateKOverland (193-368)
//     + SetUpLinearSystemsOverland (65-189)                  -> k_olf_setup
//   CUSP CG on the 5-diagonal matrix (410-411)               -> k_olf_pcg_res / k_olf_pcg
//   WaterDepthOverland (371-383) + ph <- waterdepth (417)     -> k_olf_finish
//
// The boundary ring is a fixed-elevation (identity) row in the reference.  Its
// value is known (H_old), so it is eliminated symmetrically: ring residuals and
// directions are zero and only interior rows iterate.  That system has the
// same solution as the reference's, and its interior block is symmetric, so
// Jacobi-preconditioned CG applies.  Interior rows use the reference's
// row-owned conductances kw, ke, ks, kn exactly.
#include "overland_common.cuh"

// Manning conductance of one face (src/overland.cu:279-297 and the three
// analogous blocks): the depth test is upwinded on the water elevation.
// `code` receives the test's three comparisons in three states each (band3;
// depths and slopes are compared to 1e-9 m and 1e-9, the overland solve's
// rounding level), for the branch signature.
__device__ __forceinline__ double manning_k(double Hnb, double hnb, double mnb, double Hc, double hc,
                                            double mc, double S, const DomainDesc &D, unsigned &code) {
    const double hup = (Hnb > Hc) ? hnb : hc;
    code = (band3(hup, D.hmin, 1e-9) * 3u + band3((hnb + hc) / 2., D.hmin, 1e-9)) * 3u + band3(fabs(S), D.delta, 1e-9);
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
        oc.iter = 0;
        oc.rr = 0.0;
        oc.bb = 0.0;
    }
    if (threadIdx.x == 0 && tile == 0) {
        P.gctrl->olf_live[0] = 0;
        P.gctrl->olf_live[1] = 0;
        P.gctrl->olf_live[2] = 0;
        P.gctrl->olf_bar = 0;
    }
    const ColumnRef cr = column_of(P, tile);
    unsigned long long bsig = 0;
    if (cr.valid) {
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
            unsigned we, ww, wn, ws;
            const double Sse = sqrt(pow((Hs_p1 - Hs_) / dx, 2.) +
                                    pow((Hs_pNp1 + Hs_pN - Hs_mNp1 - Hs_mN) / (4 * dy), 2.));
            ke = manning_k(Hs_p1, h_p1, mann_p1, Hs_, h_, mann_, Sse, D, we);
            const double Ssw = sqrt(pow((Hs_ - Hs_m1) / dx, 2.) +
                                    pow((Hs_pN + Hs_pNm1 - Hs_mN - Hs_mNm1) / (4 * dy), 2.));
            kw = manning_k(Hs_m1, h_m1, mann_m1, Hs_, h_, mann_, Ssw, D, ww);
            const double Ssn = sqrt(pow((Hs_pN - Hs_) / dy, 2.) +
                                    pow((Hs_pNp1 + Hs_p1 - Hs_pNm1 - Hs_m1) / (4 * dx), 2.));
            kn = manning_k(Hs_pN, h_pN, mann_pN, Hs_, h_, mann_, Ssn, D, wn);
            const double Sss = sqrt(pow((Hs_ - Hs_mN) / dy, 2.) +
                                    pow((Hs_p1 + Hs_mNp1 - Hs_m1 - Hs_mNm1) / (4 * dx), 2.));
            ks = manning_k(Hs_mN, h_mN, mann_mN, Hs_, h_, mann_, Sss, D, ws);
            if (records(D, BR_MANNING))
                bsig = branch_mix(P.pctrl[td.dom].step, BR_MANNING, I, ((we * 27u + ww) * 27u + wn) * 27u + ws);
        }
        P.olf_k[0 * ctot + I] = kw;
        P.olf_k[1 * ctot + I] = ke;
        P.olf_k[2 * ctot + I] = ks;
        P.olf_k[3 * ctot + I] = kn;
    }
    if (D.record_branches) branch_commit(&P.diag[td.dom].branch_sig, bsig);
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

// ------------------------------------------------------------------ solve
// Pipelined Jacobi-preconditioned CG (Ghysels & Vanroose 2014, Alg. 4) over
// the interior cells of every domain, in one persistent cooperative launch.
// The recurrence needs one inner-product pair (gamma = r.u, delta = w.u) per
// iteration, and its partial sums are written in the same phase as the
// preconditioned vector m = w/diag that the next matrix product reads, so one
// grid barrier per iteration makes both visible.  After the barrier every
// block sums its domains' per-segment partials itself, in the same order in
// every block, so all blocks see bitwise identical scalars without a second
// barrier.  The fixed ring is eliminated (its values stay H_old).
//
// Vectors: x (= H), r, w = A u, z = A q, s = A p, p, with u = r/diag and
// q = s/diag formed on the fly; m alternates between two buffers.  Two
// variants: k_olf_pcg_res (one resident block per segment) and k_olf_pcg
// (blocks loop over segments); both do the same arithmetic in the same order,
// so their results agree bit for bit.

struct OlfCell {
    long long c;
    int nx;
    bool live, ring;
};

__device__ __forceinline__ OlfCell olf_cell(const OlfSeg &sg, const DomainDesc &D, int t) {
    OlfCell q;
    q.live = t < sg.count;
    const int l = sg.l0 + t;
    const int j = l / D.nx, i = l - j * D.nx;
    q.c = sg.begin + t;
    q.nx = D.nx;
    q.ring = is_ring(i, j, D.nx, D.ny);
    return q;
}

// Vectors of one interior row carried by the pipelined recurrence.
struct OlfVec {
    double x, r, w, z, s, p;
};

// One iteration's vector updates at a row (Ghysels & Vanroose, Alg. 4): n is
// (A m)_c, the previous z, s, p are in e unless first.  Adds this row's
// gamma = r.u, delta = w.u and r.r terms to v and returns m = w/diag.
__device__ __forceinline__ double olf_update(OlfVec &e, double dg, double n, double alpha, double beta,
                                             bool first, double (&v)[3]) {
    const double u = e.r / dg;
    if (first) {
        e.z = n;
        e.s = e.w;
        e.p = u;
    } else {
        e.z = n + beta * e.z;
        e.s = e.w + beta * e.s;
        e.p = u + beta * e.p;
    }
    e.x += alpha * e.p;
    e.r -= alpha * e.s;
    e.w -= alpha * e.z;
    const double un = e.r / dg;
    v[0] += e.r * un;
    v[1] += e.w * un;
    v[2] += e.r * e.r;
    return e.w / dg;
}

// Stop test and step lengths of iteration it from the domain sums dsum =
// (gamma, delta, r.r): returns 1 to iterate, with alpha and beta.
__device__ __forceinline__ int olf_step_lengths(const DomainDesc &D, int it, const double (&dsum)[3], double bb,
                                                double gamma_prev, double alpha_prev, double &alpha, double &beta) {
    const double gam = dsum[0], del = dsum[1], rr = dsum[2];
    const double tol2 = D.overland_tol * D.overland_tol;
    bool stop = rr <= tol2 * bb;
    stop = stop || it >= D.overland_maxiter || !(rr == rr) || !(gam == gam);
    alpha = 0.0;
    beta = 0.0;
    if (!stop) {
        if (it == 0) {
            alpha = gam / del;
        } else {
            beta = gam / gamma_prev;
            alpha = gam / (del - beta * gam / alpha_prev);
        }
        if (!(alpha > 0.0) || !(alpha < 1e300)) stop = true;  // breakdown
    }
    return stop ? 0 : 1;
}

// The domain-level effects of that decision, by one thread of the domain's
// first segment: count the domain as live for the next iteration, or record
// its iteration count and residual when it stops.
__device__ __forceinline__ void olf_record(const DevPtrs &P, int s, const OlfSeg &sg, int it, int go,
                                           const double (&dsum)[3], double bb) {
    if (s != sg.first) return;
    if (go) {
        atomicAdd(&P.gctrl->olf_live[(it + 1) % 3], 1);
    } else {
        OverlandCtrl &oc = P.octrl[sg.dom];
        oc.iter = it;
        oc.rr = dsum[2];
        oc.bb = bb;
    }
}

// Both, for one thread that carries the segment's gamma_prev, alpha_prev.
__device__ __forceinline__ int olf_decide(const DevPtrs &P, int s, const OlfSeg &sg, const DomainDesc &D, int it,
                                          const double (&dsum)[3], double bb, double &gamma_prev,
                                          double &alpha_prev, double &alpha, double &beta) {
    const int go = olf_step_lengths(D, it, dsum, bb, gamma_prev, alpha_prev, alpha, beta);
    if (go) {
        gamma_prev = dsum[0];
        alpha_prev = alpha;
    }
    olf_record(P, s, sg, it, go, dsum, bb);
    return go;
}

// Warp sums of NV per-thread values into s_w[i][warp]; after a __syncthreads,
// olf_sum_warps adds the warp sums in warp order -- the order olf_block_sum
// uses, so both give the same bits.
template <int NV>
__device__ __forceinline__ void olf_warp_partials(const double (&v)[NV], double (*s_w)[OLF_THREADS / 32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double a = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) s_w[i][warp] = a;
    }
}

template <int NV>
__device__ __forceinline__ void olf_sum_warps(const double (*s_w)[OLF_THREADS / 32], double (&out)[NV]) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double a = 0.0;
#pragma unroll
        for (int w = 0; w < OLF_THREADS / 32; ++w) a += s_w[i][w];
        out[i] = a;
    }
}

// Streaming variant: blocks loop over segments (more segments than resident
// blocks); the vectors live in global memory and the segment scalars in
// P.osst.
__global__ void __launch_bounds__(OLF_THREADS) k_olf_pcg(DevPtrs P, long long ctot) {
    __shared__ double s_ab[2];
    __shared__ int s_go;
    const int S = P.nseg;
    const int tid = threadIdx.x;
    const int s_lo = (int)(((long long)blockIdx.x * S) / gridDim.x);
    const int s_hi = (int)(((long long)(blockIdx.x + 1) * S) / gridDim.x);
    double *const mbuf0 = P.olf_p0, *const mbuf1 = P.olf_p1;
    double *part = P.olf_part;
    double *bbp = P.olf_part + (size_t)6 * S;

    // ---- r = b - A x, u = r/diag (into m buffer 0), ||b||^2 partials
    for (int s = s_lo; s < s_hi; ++s) {
        const OlfSeg sg = P.oseg[s];
        const DomainDesc &D = P.dom[sg.dom];
        double v[1] = {0.0};
#pragma unroll
        for (int k = 0; k < OLF_CPT; ++k) {
            const int t = tid + k * OLF_THREADS;
            const OlfCell q = olf_cell(sg, D, t);
            if (!q.live) continue;
            const double bI = P.olf_b[q.c];
            v[0] += bI * bI;
            double r = 0.0, u = 0.0;
            if (!q.ring) {
                const OlfCoef cf = olf_coef(P, D, q.c, ctot);
                r = bI - olf_av<false>(cf, P.H, q.c, q.nx, P.H[q.c]);
                u = r / cf.dg;
            }
            mbuf0[q.c] = u;
            P.olf_r[q.c] = r;
        }
        olf_block_sum<1>(v);
        if (tid == 0) {
            __stcg(&bbp[s], v[0]);
            OlfSegState st;
            st.gamma_prev = 0.0; st.alpha_prev = 0.0; st.bb = 0.0; st.iter = 0; st.active = 1;
            P.osst[s] = st;
        }
    }
    if (!grid_sync(P.barrier)) return;

    // ---- w = A u, m_0 = w/diag (into m buffer 1), sums of iteration 0
    for (int s = s_lo; s < s_hi; ++s) {
        const OlfSeg sg = P.oseg[s];
        const DomainDesc &D = P.dom[sg.dom];
        double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < OLF_CPT; ++k) {
            const int t = tid + k * OLF_THREADS;
            const OlfCell q = olf_cell(sg, D, t);
            if (!q.live) continue;
            double w = 0.0, m = 0.0;
            if (!q.ring) {
                const OlfCoef cf = olf_coef(P, D, q.c, ctot);
                const double u = __ldcg(mbuf0 + q.c);
                const double r = P.olf_r[q.c];
                w = olf_av<true>(cf, mbuf0, q.c, q.nx, u);
                m = w / cf.dg;
                v[0] += r * u;
                v[1] += w * u;
                v[2] += r * r;
            }
            mbuf1[q.c] = m;
            P.olf_w[q.c] = w;
        }
        olf_block_sum<3>(v);
        if (tid == 0) {
#pragma unroll
            for (int i = 0; i < 3; ++i) __stcg(&part[(size_t)i * S + s], v[i]);
        }
    }
    if (tid == 0 && blockIdx.x == 0) P.gctrl->olf_live[2] = 0;
    if (!grid_sync(P.barrier)) return;

    // ---- iterations
    for (int it = 0;; ++it) {
        const double *pin = part + (size_t)(it & 1) * 3 * S;
        double *pout = part + (size_t)((it + 1) & 1) * 3 * S;
        const double *mcur = (it & 1) ? mbuf0 : mbuf1;
        double *mnext = (it & 1) ? mbuf1 : mbuf0;
        int prev_dom = -1;
        double dsum[3] = {0.0, 0.0, 0.0};
        for (int s = s_lo; s < s_hi; ++s) {
            const OlfSeg sg = P.oseg[s];
            const DomainDesc &D = P.dom[sg.dom];
            if (sg.dom != prev_dom) {
                olf_domain_sum<3>(pin, S, sg.first, sg.nseg, dsum);
                prev_dom = sg.dom;
            }
            double bbd[1] = {0.0};
            if (it == 0) olf_domain_sum<1>(bbp, S, sg.first, sg.nseg, bbd);
            if (tid == 0) {
                OlfSegState st = P.osst[s];
                if (it == 0) st.bb = bbd[0];
                int go = 0;
                if (st.active) {
                    double alpha, beta;
                    go = olf_decide(P, s, sg, D, it, dsum, st.bb, st.gamma_prev, st.alpha_prev, alpha, beta);
                    if (go) {
                        st.iter = it + 1;
                        s_ab[0] = alpha;
                        s_ab[1] = beta;
                    } else {
                        st.active = 0;
                    }
                    P.osst[s] = st;
                }
                s_go = go;
            }
            __syncthreads();
            const int go = s_go;
            const double alpha = s_ab[0], beta = s_ab[1];
            __syncthreads();
            if (!go) continue;
            double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < OLF_CPT; ++k) {
                const int t = tid + k * OLF_THREADS;
                const OlfCell q = olf_cell(sg, D, t);
                if (!q.live || q.ring) continue;
                const long long c = q.c;
                const OlfCoef cf = olf_coef(P, D, c, ctot);
                const double n = olf_av<true>(cf, mcur, c, q.nx, __ldcg(mcur + c));
                OlfVec e{P.H[c], P.olf_r[c], P.olf_w[c], 0.0, 0.0, 0.0};
                if (it > 0) { e.z = P.olf_z[c]; e.s = P.olf_s[c]; e.p = P.olf_p[c]; }
                const double mn = olf_update(e, cf.dg, n, alpha, beta, it == 0, v);
                mnext[c] = mn;
                P.olf_z[c] = e.z; P.olf_s[c] = e.s; P.olf_p[c] = e.p;
                P.H[c] = e.x; P.olf_r[c] = e.r; P.olf_w[c] = e.w;
            }
            olf_block_sum<3>(v);
            if (tid == 0) {
#pragma unroll
                for (int i = 0; i < 3; ++i) __stcg(&pout[(size_t)i * S + s], v[i]);
            }
        }
        if (tid == 0 && blockIdx.x == 0) P.gctrl->olf_live[(it + 2) % 3] = 0;
        if (!grid_sync(P.barrier)) return;
        if (__ldcg(&P.gctrl->olf_live[(it + 1) % 3]) == 0) break;
    }
}

// Resident variant: one block per segment for the whole solve.  The segment's
// x, r, w, z, s, p, m and row coefficients stay in shared memory and its CG
// scalars in thread 0's registers; only m goes through global memory (for the
// neighbours), and x is written back when the domain stops.  Each iteration
// is latency-bound, so its global reads -- the domain's partial sums, the
// neighbour values of m and the liveness count -- are all issued together
// right after the barrier, and the barrier is a single counter that the
// blocks add to and poll (counter_sync, zeroed by k_olf_setup), with no reset
// step between iterations.
__global__ void __launch_bounds__(OLF_THREADS) k_olf_pcg_res(DevPtrs P, long long ctot) {
    extern __shared__ double s_res[];  // [OV_N][OLF_SEG]
    __shared__ double s_wp[3][OLF_THREADS / 32], s_wv[3][OLF_THREADS / 32];
    const int S = P.nseg;
    const int tid = threadIdx.x;
    const int s = blockIdx.x;
    const OlfSeg sg = P.oseg[s];
    const DomainDesc &D = P.dom[sg.dom];
    double *const mbuf0 = P.olf_p0, *const mbuf1 = P.olf_p1;
    double *part = P.olf_part;
    double *bbp = P.olf_part + (size_t)6 * S;
    unsigned int *const bar = &P.gctrl->olf_bar;
    unsigned int epoch = 0;
    auto sv = [&](int v, int t) -> double & { return s_res[v * OLF_SEG + t]; };
    auto coef = [&](int t) { return OlfCoef{sv(OV_CW, t), sv(OV_CE, t), sv(OV_CS, t), sv(OV_CN, t), sv(OV_DG, t)}; };
    OlfCell cell[OLF_CPT];
#pragma unroll
    for (int k = 0; k < OLF_CPT; ++k) cell[k] = olf_cell(sg, D, tid + k * OLF_THREADS);

    // ---- r = b - A x, u = r/diag (into m buffer 0), ||b||^2 partials
    {
        double v[1] = {0.0};
#pragma unroll
        for (int k = 0; k < OLF_CPT; ++k) {
            const int t = tid + k * OLF_THREADS;
            const OlfCell &q = cell[k];
            if (!q.live) continue;
            const double bI = P.olf_b[q.c];
            v[0] += bI * bI;
            double r = 0.0, u = 0.0;
            const double xc = P.H[q.c];
            OlfCoef cf{0, 0, 0, 0, 1.0};
            if (!q.ring) {
                cf = olf_coef(P, D, q.c, ctot);
                r = bI - olf_av<false>(cf, P.H, q.c, q.nx, xc);
                u = r / cf.dg;
            }
            mbuf0[q.c] = u;
            sv(OV_X, t) = xc; sv(OV_R, t) = r;
            sv(OV_CW, t) = cf.cw; sv(OV_CE, t) = cf.ce; sv(OV_CS, t) = cf.cs; sv(OV_CN, t) = cf.cn;
            sv(OV_DG, t) = cf.dg;
        }
        olf_block_sum<1>(v);
        if (tid == 0) __stcg(&bbp[s], v[0]);
    }
    if (!counter_sync(bar, (++epoch) * gridDim.x, P.barrier)) return;

    // ---- w = A u, m_0 = w/diag (into m buffer 1), sums of iteration 0
    double bb = 0.0;  // the domain's ||b||^2
    {
        double bbd[1];
        olf_domain_sum<1>(bbp, S, sg.first, sg.nseg, bbd);
        bb = bbd[0];
        double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < OLF_CPT; ++k) {
            const int t = tid + k * OLF_THREADS;
            const OlfCell &q = cell[k];
            if (!q.live) continue;
            double w = 0.0, m = 0.0;
            if (!q.ring) {
                const OlfCoef cf = coef(t);
                const double u = __ldcg(mbuf0 + q.c);
                const double r = sv(OV_R, t);
                w = olf_av<true>(cf, mbuf0, q.c, q.nx, u);
                m = w / cf.dg;
                v[0] += r * u;
                v[1] += w * u;
                v[2] += r * r;
            }
            mbuf1[q.c] = m;
            sv(OV_W, t) = w;
            sv(OV_M, t) = m;
        }
        olf_block_sum<3>(v);
        if (tid == 0) {
#pragma unroll
            for (int i = 0; i < 3; ++i) __stcg(&part[(size_t)i * S + s], v[i]);
        }
    }
    if (tid == 0 && blockIdx.x == 0) P.gctrl->olf_live[2] = 0;
    if (!counter_sync(bar, (++epoch) * gridDim.x, P.barrier)) return;

    // ---- iterations
    bool active = true;                        // this segment's domain still iterates
    double gamma_prev = 0.0, alpha_prev = 0.0;
    for (int it = 0;; ++it) {
        const double *pin = part + (size_t)(it & 1) * 3 * S;
        double *pout = part + (size_t)((it + 1) & 1) * 3 * S;
        const double *mcur = (it & 1) ? mbuf0 : mbuf1;
        double *mnext = (it & 1) ? mbuf1 : mbuf0;
        // every global read of the iteration, issued together
        const int live = it > 0 ? __ldcg(&P.gctrl->olf_live[it % 3]) : 1;
        double dpart[3] = {0.0, 0.0, 0.0};
        for (int k = tid; k < sg.nseg; k += OLF_THREADS) {
#pragma unroll
            for (int i = 0; i < 3; ++i) dpart[i] += __ldcg(&pin[(size_t)i * S + sg.first + k]);
        }
        double nb[OLF_CPT][4];
#pragma unroll
        for (int k = 0; k < OLF_CPT; ++k) {
            const OlfCell &q = cell[k];
            if (active && q.live && !q.ring) {
                nb[k][0] = __ldcg(mcur + q.c - 1);
                nb[k][1] = __ldcg(mcur + q.c + 1);
                nb[k][2] = __ldcg(mcur + q.c - q.nx);
                nb[k][3] = __ldcg(mcur + q.c + q.nx);
            }
        }
        if (live == 0) break;  // no domain did work in the previous iteration
        if (!active) {
            if (!counter_sync(bar, (++epoch) * gridDim.x, P.barrier, [&] {
                    if (blockIdx.x == 0) P.gctrl->olf_live[(it + 2) % 3] = 0;
                }))
                return;
            continue;
        }
        // the domain sums, then every thread takes the same decision from them
        olf_warp_partials<3>(dpart, s_wp);
        __syncthreads();
        double dsum[3];
        olf_sum_warps<3>(s_wp, dsum);
        double alpha, beta;
        const int go = olf_step_lengths(D, it, dsum, bb, gamma_prev, alpha_prev, alpha, beta);
        if (go) {
            gamma_prev = dsum[0];
            alpha_prev = alpha;
        }
        if (tid == 0) olf_record(P, s, sg, it, go, dsum, bb);
        if (!go) {
            active = false;
#pragma unroll
            for (int k = 0; k < OLF_CPT; ++k) {
                const int t = tid + k * OLF_THREADS;
                if (t < sg.count) P.H[sg.begin + t] = sv(OV_X, t);
            }
        } else {
            double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < OLF_CPT; ++k) {
                const int t = tid + k * OLF_THREADS;
                const OlfCell &q = cell[k];
                if (!q.live || q.ring) continue;
                const OlfCoef cf = coef(t);
                const double n = olf_av4(cf, sv(OV_M, t), nb[k][0], nb[k][1], nb[k][2], nb[k][3]);
                OlfVec e{sv(OV_X, t), sv(OV_R, t), sv(OV_W, t), 0.0, 0.0, 0.0};
                if (it > 0) { e.z = sv(OV_Z, t); e.s = sv(OV_S, t); e.p = sv(OV_P, t); }
                const double mn = olf_update(e, cf.dg, n, alpha, beta, it == 0, v);
                mnext[q.c] = mn;
                sv(OV_Z, t) = e.z; sv(OV_S, t) = e.s; sv(OV_P, t) = e.p;
                sv(OV_X, t) = e.x; sv(OV_R, t) = e.r; sv(OV_W, t) = e.w; sv(OV_M, t) = mn;
            }
            olf_warp_partials<3>(v, s_wv);
        }
        // thread 0 publishes the segment's partial sums as it arrives
        if (!counter_sync(bar, (++epoch) * gridDim.x, P.barrier, [&] {
                if (go) {
                    double ps[3];
                    olf_sum_warps<3>(s_wv, ps);
#pragma unroll
                    for (int i = 0; i < 3; ++i) __stcg(&pout[(size_t)i * S + s], ps[i]);
                }
                if (blockIdx.x == 0) P.gctrl->olf_live[(it + 2) % 3] = 0;
            }))
            return;
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
    unsigned long long bsig = 0;
    if (cr.valid) {
        const long long I = cr.c;
        const double H = P.H[I];
        const double d = H - P.ztopo[I];
        const double hn = fmax(d, 0.0);
        P.h[I] = hn;
        P.ph[I] = hn;
        if (d < 0) v[1] = -d;
        if (records(D, BR_DEPTHCLIP)) bsig = branch_mix(P.pctrl[td.dom].step, BR_DEPTHCLIP, I, band3(d, 0.0, 1e-9));
        v[2] = hn;
        if (!is_ring(cr.i, cr.j, cr.nx, cr.ny)) {
            const OlfRow w = olf_row(P, cr, D, ctot);
            if (cr.i == 1) v[0] += w.cx * w.kw * (H - P.H[I - 1]);
            if (cr.i == cr.nx - 2) v[0] += w.cx * w.ke * (H - P.H[I + 1]);
            if (cr.j == 1) v[0] += w.cy * w.ks * (H - P.H[I - cr.nx]);
            if (cr.j == cr.ny - 2) v[0] += w.cy * w.kn * (H - P.H[I + cr.nx]);
        }
    }
    if (D.record_branches) branch_commit(&P.diag[td.dom].branch_sig, bsig);
    if (domain_reduce<3>(P, tile, td.dom, 3, v) && threadIdx.x == 0) {
        DevDiag &dg = P.diag[td.dom];
        const OverlandCtrl &oc = P.octrl[td.dom];
        dg.olf_out_cum += v[0];
        dg.olf_clip_cum += v[1];
        dg.ponded = v[2];
        dg.overland_iters_total += oc.iter;
        if (records(D, BR_OLFITER))
            atomicAdd(&dg.branch_sig, branch_mix(P.pctrl[td.dom].step, BR_OLFITER, td.dom, (unsigned)oc.iter));
        const double tol2 = D.overland_tol * D.overland_tol;
        if (!(oc.rr <= tol2 * oc.bb)) dg.overland_nonconverged += 1;
    }
}

cudaError_t launch_overland_setup(const DevPtrs &P, long long ctot, cudaStream_t s) {
    k_olf_setup<<<P.ntiles, TILE_THREADS, 0, s>>>(P, ctot);
    return cudaGetLastError();
}

#define OLF_RES_SMEM (OV_N * OLF_SEG * (int)sizeof(double))

cudaError_t launch_overland_solve(const DevPtrs &P, const LaunchCfg &L, long long ctot, cudaStream_t s) {
    DevPtrs args = P;
    long long c = ctot;
    void *kargs[] = {&args, &c};
    if (L.olf_mg) return launch_overland_mg(P, L, ctot, s);
    if (L.olf_allow_resident && P.nseg <= L.olf_res_blocks)
        return cudaLaunchCooperativeKernel((const void *)k_olf_pcg_res, dim3(P.nseg), dim3(OLF_THREADS), kargs,
                                           OLF_RES_SMEM, s);
    const int blocks = L.olf_stream_per_sm * L.sms;
    const int grid = blocks < P.nseg ? blocks : P.nseg;
    return cudaLaunchCooperativeKernel((const void *)k_olf_pcg, dim3(grid), dim3(OLF_THREADS), kargs, 0, s);
}

cudaError_t launch_overland_finish(const DevPtrs &P, long long ctot, cudaStream_t s) {
    k_olf_finish<<<P.ntiles, TILE_THREADS, 0, s>>>(P, ctot);
    return cudaGetLastError();
}

cudaError_t configure_2d(LaunchCfg &L, int device) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void *)k_olf_pcg_res, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             OLF_RES_SMEM);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_olf_pcg_res, OLF_THREADS,
                                                      OLF_RES_SMEM);
    if (e != cudaSuccess) return e;
    L.olf_res_blocks = per_sm * prop.multiProcessorCount;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_olf_pcg, OLF_THREADS, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    L.olf_stream_blocks = per_sm * prop.multiProcessorCount;
    L.coop_blocks_2d = L.olf_stream_blocks;
    L.olf_stream_per_sm_max = per_sm;
    L.olf_stream_per_sm = per_sm;
    L.olf_allow_resident = 1;
    return cudaSuccess;
}
