// overland_mg.cu -- the overland solve (the reference's CUSP CG on the
// 5-point system, src/overland.cu:410-411) as conjugate gradients
// preconditioned by one geometric multigrid V-cycle per iteration.
//
// Why: over ponded, flat ground Manning's conductance h^(5/3) / (n sqrt S)
// makes the system I + dt L_K nearly singular (dt K / dx^2 reaches 1e4-1e5
// over a pool), and point-Jacobi-preconditioned CG needs thousands of
// iterations for a 1e-12 relative residual (1,400-2,100 on 256 x 256 storm
// surfaces, growing with the grid); the reference's 100-iteration cap stops
// far from the solution.  A V-cycle removes the smooth error that point
// smoothing cannot.
//
// Hierarchy (per domain, planned on the host by mg_plan): level 0 is the
// interior of the surface grid (the fixed ring is eliminated, as in the
// Jacobi solver); level l+1 halves every dimension of level l that has at
// least 3 points, vertex-centred (coarse point I sits on fine point 2I+1),
// until a level has at most MG_DENSE_PTS points; that coarsest level is
// solved exactly by its inverse, formed once per solve.
//
// Interpolation is operator-dependent (the "black box" multigrid rule of
// Dendy, J. Comput. Phys. 48 (1982) 366-386), because the conductance jumps
// by orders of magnitude between ponded and dry cells and bilinear
// interpolation across such a jump is poor: a fine point between two coarse
// points along x takes weights -sum(column W) / sum(column C) and
// -sum(column E) / sum(column C) of its row's 3 x 3 stencil (the row collapsed
// onto the line through the coarse points; along y likewise with the stencil's
// rows), and a point between four coarse points takes the weights its row
// gives once its four edge neighbours are replaced by their own
// interpolation.  The stencils are first made M-matrix rows (positive
// off-diagonal entries moved onto the diagonal) and every weight is clamped
// to [0, 1]; weights are stored in FP32 and used, converted, in FP64.  The
// coarse operators are the Galerkin products A_{l+1} = P^T A_l P with these
// weights, recomputed for every solve.  They are 9-point; each row stores C,
// E, N, NE and NW, and a row's W, S, SW and SE are its neighbours' E, N, NE
// and NW, so every stored operator is symmetric bit for bit.  The smoother is
// Jacobi with per-row weights w_i = max(a_ii / 0.8, 0.55 sum_j |a_ij|)
// (weighted Jacobi at 0.8 wherever that is safe): 2W - A is then diagonally
// dominant, every sweep is convergent, and the V(1,1) cycle -- pre-smoothing
// from zero, coarse correction, post-smoothing, and the exact solve on the
// coarsest level (its inverse symmetrised) -- is a fixed symmetric positive
// definite operator, as CG needs.  On 128 x 128 storm surfaces this takes
// 39-47 CG iterations where bilinear interpolation took 63-81.
//
// Schedule: one persistent cooperative launch per solve for all domains.  A
// domain's coarsest levels, as many as fit MG_SMEM_PTS points together, run
// in one block out of shared memory with block barriers, their operators set
// up there and kept for the whole solve when the block owns one domain; the
// finer ones run as grid phases, level 0 in chunks of MG_CHUNK0 points (four
// per thread) and the others one point per thread.  The pre-smoothing and
// the residual are folded into a stored 5 x 5 restriction stencil per coarse
// point (P^T (I - A W^-1), formed at set-up), and the prolongation is fused
// into the post-smoothing (each point recomputes the few neighbour values it
// needs), so a grid level costs one barrier on the way down and one on the
// way up; with q = A z + beta q
// the CG forms p and q in one phase.  An iteration with L grid levels is
// 2 L + 3 barriers (eleven on a 512 x 512 surface).  Every reduction runs over
// chunks in a fixed order, so results do not depend on the block count.
#include <algorithm>
#include <cstring>

#include "overland_common.cuh"

namespace {

// chunk partial slots: p.q, r.r, r.z (iteration parity 0 / 1), b.b
enum { MP_PQ = 0, MP_RR = 1, MP_RZ = 2, MP_BB = 4 };

// ---------------------------------------------------------------- geometry
// Level l of one domain: its points, where its arrays start, how rows index.
struct Lvl {
    int m, n;
    int nx;          // level 0: the surface row length
    bool fine;       // level 0: vectors live in the surface arrays
    long long base;  // level 0: the domain's surface offset; else the first coarse point
    __device__ __forceinline__ long long at(int i, int j) const {
        return fine ? base + (long long)(j + 1) * nx + (i + 1) : base + (long long)j * m + i;
    }
};

__device__ __forceinline__ Lvl level(const MgDom &g, int l) {
    return Lvl{g.m[l], g.n[l], g.nx, l == 0, g.off[l]};
}

// Vectors of a level: right-hand side, pre-smoothed and post-smoothed
// (final) solution.  Level 0 uses the CG's residual, z and w arrays.
struct LvlVec {
    const double *b;
    double *x, *t;
};

__device__ __forceinline__ LvlVec vectors(const DevPtrs &P, int l) {
    if (l == 0) return LvlVec{P.olf_r, P.olf_z, P.olf_w};
    return LvlVec{P.mg_b, P.mg_x, P.mg_t};
}

// Interpolation weights of level l's point (i, j) to its parents, in the slot
// order (p0x, p0y), (p1x, p0y), (p0x, p1y), (p1x, p1y) of parents2.
__device__ __forceinline__ float4 *pw_ptr(const DevPtrs &P, const MgDom &g, int l, int i, int j) {
    return P.mg_pw + g.pwo[l] + (long long)j * g.m[l] + i;
}
__device__ __forceinline__ float4 pw_at(const DevPtrs &P, const MgDom &g, int l, int i, int j) {
    return __ldcg(pw_ptr(P, g, l, i, j));
}
__device__ __forceinline__ double slot(const float4 &w, int s) {
    return (double)(s == 0 ? w.x : s == 1 ? w.y : s == 2 ? w.z : w.w);
}

// Row (i, j) of level l's operator as a 3 x 3 stencil a[dj+1][di+1]; zero
// where the neighbour is outside the level.  Level 0 is the reference's
// 5-point interior row (row-owned conductances, ring couplings eliminated).
struct Row9 {
    double a[3][3];
};

__device__ __forceinline__ Row9 row_of(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g,
                                       int l, const Lvl &v, int i, int j) {
    Row9 r;
#pragma unroll
    for (int y = 0; y < 3; ++y)
#pragma unroll
        for (int x = 0; x < 3; ++x) r.a[y][x] = 0.0;
    if (l == 0) {
        const OlfCoef cf = olf_coef(P, D, v.at(i, j), ctot);
        r.a[1][1] = cf.dg;
        if (i > 0) r.a[1][0] = -cf.cw;
        if (i < v.m - 1) r.a[1][2] = -cf.ce;
        if (j > 0) r.a[0][1] = -cf.cs;
        if (j < v.n - 1) r.a[2][1] = -cf.cn;
        return r;
    }
    const long long nc = P.mg_nc;
    const double *A = P.mg_a;
    auto e = [&](int k, int ii, int jj) { return __ldcg(A + (size_t)k * nc + v.at(ii, jj)); };
    const bool w = i > 0, ea = i < v.m - 1, s = j > 0, no = j < v.n - 1;
    r.a[1][1] = e(0, i, j);
    if (ea) r.a[1][2] = e(1, i, j);
    if (w) r.a[1][0] = e(1, i - 1, j);
    if (no) r.a[2][1] = e(2, i, j);
    if (s) r.a[0][1] = e(2, i, j - 1);
    if (ea && no) r.a[2][2] = e(3, i, j);
    if (w && s) r.a[0][0] = e(3, i - 1, j - 1);
    if (w && no) r.a[2][0] = e(4, i, j);          // NW couples (i, j) to (i-1, j+1)
    if (ea && s) r.a[0][2] = e(4, i + 1, j - 1);  // SE is (i+1, j-1)'s NW
    return r;
}

// The grid phases' form of row_of: every load is unconditional, at
// an address clamped into the level (level 0's ring cells exist in memory),
// and the entries outside the level are selected to zero after the loads, so
// no load waits on a branch and all of a point's loads can be in flight.
// FINE: level 0 (5-point rows from the conductances).
template <bool FINE>
__device__ __forceinline__ Row9 row_nb(const DevPtrs &P, const DomainDesc &D, long long ctot, const Lvl &v, int i,
                                       int j) {
    Row9 r;
    const bool w = i > 0, ea = i < v.m - 1, s = j > 0, no = j < v.n - 1;
    if constexpr (FINE) {
        const OlfCoef cf = olf_coef(P, D, v.at(i, j), ctot);
        r.a[1][1] = cf.dg;
        r.a[1][0] = w ? -cf.cw : 0.0;
        r.a[1][2] = ea ? -cf.ce : 0.0;
        r.a[0][1] = s ? -cf.cs : 0.0;
        r.a[2][1] = no ? -cf.cn : 0.0;
        r.a[0][0] = r.a[0][2] = r.a[2][0] = r.a[2][2] = 0.0;
    } else {
        const int im = w ? i - 1 : i, ip = ea ? i + 1 : i, jm = s ? j - 1 : j;
        const long long nc = P.mg_nc;
        const double *A = P.mg_a;
        auto e = [&](int k, int ii, int jj) { return __ldcg(A + (size_t)k * nc + v.at(ii, jj)); };
        const double c = e(0, i, j), eE = e(1, i, j), eW = e(1, im, j), nN = e(2, i, j), nS = e(2, i, jm);
        const double neNE = e(3, i, j), neSW = e(3, im, jm), nwNW = e(4, i, j), nwSE = e(4, ip, jm);
        r.a[1][1] = c;
        r.a[1][2] = ea ? eE : 0.0;
        r.a[1][0] = w ? eW : 0.0;
        r.a[2][1] = no ? nN : 0.0;
        r.a[0][1] = s ? nS : 0.0;
        r.a[2][2] = (ea && no) ? neNE : 0.0;
        r.a[0][0] = (w && s) ? neSW : 0.0;
        r.a[2][0] = (w && no) ? nwNW : 0.0;
        r.a[0][2] = (ea && s) ? nwSE : 0.0;
    }
    return r;
}

__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

template <bool FINE>
__device__ __forceinline__ double apply_nb(const Row9 &r, const double *x, const Lvl &v, int i, int j) {
    double s = 0.0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            if (FINE && dx != 0 && dy != 0) continue;  // compile-time: no corners at level 0
            const int ii = FINE ? i + dx : clampi(i + dx, v.m), jj = FINE ? j + dy : clampi(j + dy, v.n);
            s += r.a[dy + 1][dx + 1] * __ldcg(x + v.at(ii, jj));
        }
    return s;
}

// 1 / smoother weight of row (i, j).
__device__ __forceinline__ double smoother_inv(const Row9 &r) {
    double l1 = 0.0;
#pragma unroll
    for (int y = 0; y < 3; ++y)
#pragma unroll
        for (int x = 0; x < 3; ++x) l1 += fabs(r.a[y][x]);
    return 1.0 / fmax(r.a[1][1] / 0.8, 0.55 * l1);
}

// ---------------------------------------------------- transfer operators
// Child a (0, 1, 2 = 2I, 2I+1, 2I+2) of coarse index I along a halved
// dimension, or I itself (a = 1) along one that is not; w = 0 for none.
__device__ __forceinline__ void child(int I, int a, bool halves, int mf, int &f, double &w) {
    if (halves) {
        f = 2 * I + a;
        w = f < mf ? 1.0 : 0.0;
    } else {
        f = I;
        w = a == 1 ? 1.0 : 0.0;
    }
}

// The weight slot of child a's parent I along one dimension: the child 2I
// has I as its second parent, 2I+1 and 2I+2 as their first.
__device__ __forceinline__ int child_slot(int a, bool halves) { return (halves && a == 0) ? 1 : 0; }

// Parents p0, p1 of fine index i along one dimension with u0, u1 nonzero
// where the parent exists: the coarse point on i, or the two beside it.
__device__ __forceinline__ void parents2(int i, bool halves, int mc, int &p0, double &u0, int &p1, double &u1) {
    if (!halves) {
        p0 = p1 = i;
        u0 = 1.0;
        u1 = 0.0;
    } else if (i & 1) {
        p0 = p1 = (i - 1) >> 1;
        u0 = 1.0;
        u1 = 0.0;
    } else {
        p0 = (i >> 1) - 1;
        u0 = p0 >= 0 ? 0.5 : 0.0;
        p1 = i >> 1;
        u1 = p1 < mc ? 0.5 : 0.0;
        p0 = p0 < 0 ? 0 : p0;  // a parent that does not exist points at a valid slot
        p1 = p1 < mc ? p1 : mc - 1;
    }
}

__device__ __forceinline__ double clamp01(double v) { return v > 0.0 ? (v < 1.0 ? v : 1.0) : 0.0; }

// The row with its positive off-diagonal entries moved onto the diagonal.
__device__ __forceinline__ Row9 lumped(Row9 r) {
    double add = 0.0;
#pragma unroll
    for (int y = 0; y < 3; ++y)
#pragma unroll
        for (int x = 0; x < 3; ++x)
            if ((y != 1 || x != 1) && r.a[y][x] > 0.0) {
                add += r.a[y][x];
                r.a[y][x] = 0.0;
            }
    r.a[1][1] += add;
    return r;
}

struct W4 {
    double w[4];
};

// Weights of a point between two coarse points: along x (ex) the stencil's
// columns are summed, along y its rows.
__device__ __forceinline__ W4 edge_weights(const Row9 &s, bool ex) {
    W4 o = {{0.0, 0.0, 0.0, 0.0}};
    if (ex) {
        const double cC = (s.a[0][1] + s.a[1][1]) + s.a[2][1];
        if (cC > 0.0) {
            o.w[0] = clamp01(-((s.a[0][0] + s.a[1][0]) + s.a[2][0]) / cC);
            o.w[1] = clamp01(-((s.a[0][2] + s.a[1][2]) + s.a[2][2]) / cC);
        }
    } else {
        const double cC = (s.a[1][0] + s.a[1][1]) + s.a[1][2];
        if (cC > 0.0) {
            o.w[0] = clamp01(-((s.a[0][0] + s.a[0][1]) + s.a[0][2]) / cC);
            o.w[2] = clamp01(-((s.a[2][0] + s.a[2][1]) + s.a[2][2]) / cC);
        }
    }
    return o;
}

// Interpolation weights of point (i, j) of an m x n level (rowf(i, j): the
// level's rows, only called inside the level).
template <typename RowF>
__device__ __forceinline__ float4 interp_weights(RowF rowf, int i, int j, int m, int n, bool hx, bool hy) {
    const bool ex = hx && !(i & 1), ey = hy && !(j & 1);
    if (!ex && !ey) return make_float4(1.f, 0.f, 0.f, 0.f);
    const Row9 s = lumped(rowf(i, j));
    W4 o = {{0.0, 0.0, 0.0, 0.0}};
    if (!(ex && ey)) {
        o = edge_weights(s, ex);
    } else if (s.a[1][1] > 0.0) {
        double acc[4] = {s.a[0][0], s.a[0][2], s.a[2][0], s.a[2][2]};
        if (i > 0) {
            const W4 e = edge_weights(lumped(rowf(i - 1, j)), false);
            acc[0] += s.a[1][0] * e.w[0];
            acc[2] += s.a[1][0] * e.w[2];
        }
        if (i < m - 1) {
            const W4 e = edge_weights(lumped(rowf(i + 1, j)), false);
            acc[1] += s.a[1][2] * e.w[0];
            acc[3] += s.a[1][2] * e.w[2];
        }
        if (j > 0) {
            const W4 e = edge_weights(lumped(rowf(i, j - 1)), true);
            acc[0] += s.a[0][1] * e.w[0];
            acc[1] += s.a[0][1] * e.w[1];
        }
        if (j < n - 1) {
            const W4 e = edge_weights(lumped(rowf(i, j + 1)), true);
            acc[2] += s.a[2][1] * e.w[0];
            acc[3] += s.a[2][1] * e.w[1];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) o.w[k] = clamp01(-acc[k] / s.a[1][1]);
    }
    return make_float4((float)o.w[0], (float)o.w[1], (float)o.w[2], (float)o.w[3]);
}

// Galerkin row (I, J) of the coarse level: C, E, N, NE and NW of P^T A P, from
// the fine level's rows rowf and weights wf (fm x fn fine points, cm x cn
// coarse).
template <typename RowF, typename WF>
__device__ __forceinline__ void galerkin_row(RowF rowf, WF wf, int fm, int fn, bool hx, bool hy, int cm, int cn,
                                             int I, int J, double (&acc)[5]) {
#pragma unroll
    for (int k = 0; k < 5; ++k) acc[k] = 0.0;
    for (int b = 0; b < 3; ++b) {
        int fy;
        double vy;
        child(J, b, hy, fn, fy, vy);
        if (vy == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
            int fx;
            double vx;
            child(I, a, hx, fm, fx, vx);
            if (vx == 0.0) continue;
            const double pf = slot(wf(fx, fy), child_slot(a, hx) + 2 * child_slot(b, hy));
            if (pf == 0.0) continue;
            const Row9 r = rowf(fx, fy);
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const double av = r.a[dy + 1][dx + 1];
                    if (av == 0.0) continue;
                    const int gx = fx + dx, gy = fy + dy;
                    const float4 wg = wf(gx, gy);
                    int px0, px1, py0, py1;
                    double ux0, ux1, uy0, uy1;
                    parents2(gx, hx, cm, px0, ux0, px1, ux1);
                    parents2(gy, hy, cn, py0, uy0, py1, uy1);
                    for (int s = 0; s < 4; ++s) {
                        const double w = slot(wg, s);
                        const double u = ((s & 1) ? ux1 : ux0) * ((s & 2) ? uy1 : uy0);
                        if (w == 0.0 || u == 0.0) continue;
                        const int di = ((s & 1) ? px1 : px0) - I, dj = ((s & 2) ? py1 : py0) - J;
                        const int k = (di == 0 && dj == 0) ? 0 : (di == 1 && dj == 0) ? 1
                                    : (di == 0 && dj == 1)   ? 2 : (di == 1 && dj == 1) ? 3
                                    : (di == -1 && dj == 1)  ? 4 : -1;
                        if (k >= 0) acc[k] += (pf * av) * w;
                    }
                }
        }
    }
}

// ------------------------------------------------- grid-phase point kernels
// The restriction with the pre-smoothing folded in: V(1,1) starts from x = 0,
// so level l's pre-smoothed x_l = W_l^-1 b_l and the coarse right-hand side
// b_{l+1} = P^T (b_l - A_l x_l) = P^T (I - A_l W_l^-1) b_l, a fixed 5 x 5
// stencil on b_l per coarse point (I, J), stored component-major in mg_r.
// Its fine block starts at (2I - 1, 2J - 1) along a halved dimension and at
// (I - 2, J - 2) along one that is not; entries outside the level are 0.
__device__ __forceinline__ int rblock0(int I, bool halves) { return halves ? 2 * I - 1 : I - 2; }

// Set-up of coarse point (I, J) of level l+1 from level l in global memory:
// its Galerkin row (C, E, N, NE, NW of P^T A_l P) and its restriction
// stencil.  Every loop is unrolled and every load is at a position clamped
// into the level, the terms outside it multiplied by zero, so the loads of a
// child's row, its neighbours' weights and smoother weights are all in
// flight together.  FINE: level 0 (5-point rows, smoother weights from
// mg_w0).
template <bool FINE>
__device__ __noinline__ void setup_point(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g, int l, int I,
                            int J) {
    const Lvl f = level(g, l), c = level(g, l + 1);
    const bool hx = g.hx[l], hy = g.hy[l];
    const double *wsm = FINE ? P.mg_w0 : P.mg_w;
    double R[25], acc[5];
#pragma unroll
    for (int k = 0; k < 25; ++k) R[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) acc[k] = 0.0;
#pragma unroll 1
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int fx, fy;
            double vx, vy;
            child(I, a, hx, f.m, fx, vx);
            child(J, b, hy, f.n, fy, vy);
            fx = clampi(fx, f.m);
            fy = clampi(fy, f.n);
            const Row9 r = row_nb<FINE>(P, D, ctot, f, fx, fy);
            const double pf =
                (vx != 0.0 && vy != 0.0) ? slot(pw_at(P, g, l, fx, fy), child_slot(a, hx) + 2 * child_slot(b, hy)) : 0.0;
            R[(b + 1) * 5 + (a + 1)] += pf;
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    if (FINE && dx != 0 && dy != 0) continue;  // compile-time: no corners at level 0
                    const int gx = clampi(fx + dx, f.m), gy = clampi(fy + dy, f.n);
                    const double av = pf * r.a[dy + 1][dx + 1];  // 0 outside the level or the child set
                    R[(b + 1 + dy) * 5 + (a + 1 + dx)] -= av * __ldcg(wsm + f.at(gx, gy));
                    const float4 wq = pw_at(P, g, l, gx, gy);
                    int px0, px1, py0, py1;
                    double ux0, ux1, uy0, uy1;
                    parents2(gx, hx, c.m, px0, ux0, px1, ux1);
                    parents2(gy, hy, c.n, py0, uy0, py1, uy1);
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const double u = ((s & 1) ? ux1 : ux0) * ((s & 2) ? uy1 : uy0);
                        const double v = u != 0.0 ? av * slot(wq, s) : 0.0;
                        const int di = ((s & 1) ? px1 : px0) - I, dj = ((s & 2) ? py1 : py0) - J;
                        acc[0] += (di == 0 && dj == 0) ? v : 0.0;
                        acc[1] += (di == 1 && dj == 0) ? v : 0.0;
                        acc[2] += (di == 0 && dj == 1) ? v : 0.0;
                        acc[3] += (di == 1 && dj == 1) ? v : 0.0;
                        acc[4] += (di == -1 && dj == 1) ? v : 0.0;
                    }
                }
        }
    const long long at = c.at(I, J);
#pragma unroll
    for (int k = 0; k < 5; ++k) P.mg_a[(size_t)k * P.mg_nc + at] = acc[k];
#pragma unroll
    for (int k = 0; k < 25; ++k) P.mg_r[(size_t)k * P.mg_nc + at] = R[k];
}

// Smoother weight (levels >= 1) and interpolation weights of level l's point.
__device__ __forceinline__ void weight_point(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g,
                                             int l, int i, int j) {
    const Lvl v = level(g, l);
    auto rowf = [&](int ii, int jj) { return row_of(P, D, ctot, g, l, v, ii, jj); };
    if (l > 0) P.mg_w[v.at(i, j)] = smoother_inv(rowf(i, j));
    *pw_ptr(P, g, l, i, j) = interp_weights(rowf, i, j, v.m, v.n, g.hx[l], g.hy[l]);
}

// (P t)(i, j): level l+1's t interpolated to level l's point (i, j) with the
// point's weights w.
__device__ __forceinline__ double prolong_at(const MgDom &g, int l, const Lvl &c, const double *tc, const float4 &w,
                                             int i, int j) {
    int px0, px1, py0, py1;
    double ux0, ux1, uy0, uy1;
    parents2(i, g.hx[l], c.m, px0, ux0, px1, ux1);
    parents2(j, g.hy[l], c.n, py0, uy0, py1, uy1);
    // every parent slot is valid (a weight that does not apply is selected
    // to 0), so the four loads are unconditional
    const double w00 = (ux0 != 0.0 && uy0 != 0.0) ? (double)w.x : 0.0;
    const double w10 = (ux1 != 0.0 && uy0 != 0.0) ? (double)w.y : 0.0;
    const double w01 = (ux0 != 0.0 && uy1 != 0.0) ? (double)w.z : 0.0;
    const double w11 = (ux1 != 0.0 && uy1 != 0.0) ? (double)w.w : 0.0;
    return (w00 * __ldcg(tc + c.at(px0, py0)) + w10 * __ldcg(tc + c.at(px1, py0))) +
           (w01 * __ldcg(tc + c.at(px0, py1)) + w11 * __ldcg(tc + c.at(px1, py1)));
}

// Grid levels (one barrier per level each way): level l+1 point (I, J) gets
// b = P^T (I - A_l W_l^-1) b_l from its stored 5 x 5 stencil, and x = W^-1 b.
// Positions outside the level (coefficient 0) are read clamped, so the 25
// loads of b do not wait on branches.
template <bool FINE>
__device__ void restrict_point(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g, int l, int I,
                               int J) {
    const Lvl f = level(g, l), c = level(g, l + 1);
    const LvlVec vf = vectors(P, l);
    const int ox = rblock0(I, g.hx[l]), oy = rblock0(J, g.hy[l]);
    const long long at = c.at(I, J);
    const double *R = P.mg_r + at;
    const size_t nc = (size_t)P.mg_nc;
    double acc = 0.0;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const int fy = clampi(oy + v, f.n);
#pragma unroll
        for (int u = 0; u < 5; ++u)
            acc += __ldcg(R + (size_t)(v * 5 + u) * nc) * __ldcg(vf.b + f.at(clampi(ox + u, f.m), fy));
    }
    P.mg_b[at] = acc;
    P.mg_x[at] = __ldcg(P.mg_w + at) * acc;
}

// ... and on the way up level l point (i, j) gets t = x' + W^-1 (b - A x')
// with x' = x_l + P t_{l+1} formed at the point and its neighbours (clamped
// positions where a neighbour is outside the level, whose coefficient is 0).
template <bool FINE>
__device__ __forceinline__ double smooth_up_value(const DevPtrs &P, const DomainDesc &D, long long ctot,
                                                  const MgDom &g, int l, int i, int j) {
    const Lvl f = level(g, l), c = level(g, l + 1);
    const LvlVec vf = vectors(P, l);
    const Row9 r = row_nb<FINE>(P, D, ctot, f, i, j);
    double ax = 0.0, xc = 0.0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            if (FINE && dx != 0 && dy != 0) continue;  // compile-time: no corners at level 0
            const int ni = clampi(i + dx, f.m), nj = clampi(j + dy, f.n);
            const double xp =
                __ldcg(vf.x + f.at(ni, nj)) + prolong_at(g, l, c, P.mg_t, pw_at(P, g, l, ni, nj), ni, nj);
            ax += r.a[dy + 1][dx + 1] * xp;
            if (dx == 0 && dy == 0) xc = xp;
        }
    const long long at = f.at(i, j);
    const double winv = FINE ? 0.8 / r.a[1][1] : __ldcg(P.mg_w + at);
    return xc + winv * (__ldcg(vf.b + at) - ax);
}

template <bool FINE>
__device__ void smooth_up_point(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g, int l, int i,
                                int j) {
    vectors(P, l).t[level(g, l).at(i, j)] = smooth_up_value<FINE>(P, D, ctot, g, l, i, j);
}

// ----------------------------------------------------------- block levels
// A domain's block levels live in shared memory: each level's operator (C, E,
// N, NE, NW; level 0 as the same five from its 5-point rows), smoother
// weights, vectors b, x, t and interpolation weights, levels packed one after
// another (the host picks lc so that levels lc .. nlev-1 fit MG_SMEM_PTS), and
// the coarsest level's inverse.  The block sets them up once per solve and
// keeps them while it owns one domain; a block that owns several reloads a
// domain's from global memory before its V-cycle.
struct SmemMG {
    double *a[5], *w, *b, *x, *t, *dinv;
    float4 *pw;
};

__device__ __forceinline__ SmemMG smem_mg(double *base) {
    SmemMG S;
#pragma unroll
    for (int k = 0; k < 5; ++k) S.a[k] = base + (size_t)k * MG_SMEM_PTS;
    S.w = base + 5 * (size_t)MG_SMEM_PTS;
    S.b = base + 6 * (size_t)MG_SMEM_PTS;
    S.x = base + 7 * (size_t)MG_SMEM_PTS;
    S.t = base + 8 * (size_t)MG_SMEM_PTS;
    S.pw = (float4 *)(base + 9 * (size_t)MG_SMEM_PTS);
    S.dinv = base + 11 * (size_t)MG_SMEM_PTS;
    return S;
}

struct SL {
    int m, n, o;  // points and first slot of the level
    __device__ __forceinline__ int at(int i, int j) const { return o + j * m + i; }
};

__device__ __forceinline__ Row9 s_row(const SmemMG &S, const SL &v, int i, int j) {
    Row9 r;
    const bool w = i > 0, ea = i < v.m - 1, s = j > 0, no = j < v.n - 1;
    r.a[1][1] = S.a[0][v.at(i, j)];
    r.a[1][2] = ea ? S.a[1][v.at(i, j)] : 0.0;
    r.a[1][0] = w ? S.a[1][v.at(i - 1, j)] : 0.0;
    r.a[2][1] = no ? S.a[2][v.at(i, j)] : 0.0;
    r.a[0][1] = s ? S.a[2][v.at(i, j - 1)] : 0.0;
    r.a[2][2] = (ea && no) ? S.a[3][v.at(i, j)] : 0.0;
    r.a[0][0] = (w && s) ? S.a[3][v.at(i - 1, j - 1)] : 0.0;
    r.a[2][0] = (w && no) ? S.a[4][v.at(i, j)] : 0.0;
    r.a[0][2] = (ea && s) ? S.a[4][v.at(i + 1, j - 1)] : 0.0;
    return r;
}

__device__ __forceinline__ double s_apply(const Row9 &r, const double *x, const SL &v, int i, int j) {
    double s = 0.0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const bool in = i + dx >= 0 && i + dx < v.m && j + dy >= 0 && j + dy < v.n;
            if (in) s += r.a[dy + 1][dx + 1] * x[v.at(i + dx, j + dy)];
        }
    return s;
}

template <typename Fn>
__device__ __forceinline__ void s_points(const SL &v, Fn fn) {
    const int tot = v.m * v.n;
    for (int p = threadIdx.x; p < tot; p += blockDim.x) fn(p % v.m, p / v.m);
}

// Levels lc .. nlev-1 packed in shared memory.
__device__ __forceinline__ void s_levels(const MgDom &g, SL (&lv)[MG_MAXLEV]) {
    int o = 0;
    for (int l = g.lc; l < g.nlev; ++l) {
        lv[l] = SL{g.m[l], g.n[l], o};
        o += g.m[l] * g.n[l];
    }
}

// Level lc's operator into shared memory (level 0: from the conductances)
// with, when `all`, the coarser operators, the smoother and interpolation
// weights and the coarsest inverse that the set-up left in global memory.
__device__ void block_load(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g, const SmemMG &S,
                           const SL (&lv)[MG_MAXLEV], bool all) {
    const int last = all ? g.nlev - 1 : g.lc;
    for (int l = g.lc; l <= last; ++l) {
        const SL v = lv[l];
        const Lvl gl = level(g, l);
        s_points(v, [&](int i, int j) {
            const int q = v.at(i, j);
            const long long at = gl.at(i, j);
            if (l == 0) {
                const OlfCoef cf = olf_coef(P, D, at, ctot);
                S.a[0][q] = cf.dg;
                S.a[1][q] = -cf.ce;
                S.a[2][q] = -cf.cn;
                S.a[3][q] = 0.0;
                S.a[4][q] = 0.0;
            } else {
#pragma unroll
                for (int k = 0; k < 5; ++k) S.a[k][q] = __ldcg(P.mg_a + (size_t)k * P.mg_nc + at);
            }
            if (all && l + 1 < g.nlev) {
                S.w[q] = l == 0 ? 0.8 / S.a[0][q] : __ldcg(P.mg_w + at);
                S.pw[q] = pw_at(P, g, l, i, j);
            }
        });
    }
    if (all) {
        const int nd = g.m[g.nlev - 1] * g.n[g.nlev - 1];
        for (int k = threadIdx.x; k < nd * nd; k += blockDim.x) S.dinv[k] = __ldcg(P.mg_dinv + g.dio + k);
    }
}

// Inverse of the coarsest level's operator (at most MG_DENSE_PTS points) by
// Gauss-Jordan elimination on [A | I] in the scratch M, one warp, lane c
// owning column c; the result is symmetrised and written to S.dinv and dst.
// No pivoting: the operator is symmetric positive definite.
__device__ void dense_inverse(const SmemMG &S, const SL &v, double *M, double *dst) {
    constexpr int W = 2 * MG_DENSE_PTS;
    const int n = v.m * v.n, lane = threadIdx.x;
    if (lane < 2 * n)
        for (int r = 0; r < n; ++r) {
            double val = 0.0;
            if (lane < n) {
                const int ri = r % v.m, rj = r / v.m, ci = lane % v.m, cj = lane / v.m;
                const int dx = ci - ri, dy = cj - rj;
                if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1) val = s_row(S, v, ri, rj).a[dy + 1][dx + 1];
            } else {
                val = lane - n == r ? 1.0 : 0.0;
            }
            M[r * W + lane] = val;
        }
    __syncwarp();
    for (int k = 0; k < n; ++k) {
        // column k is only read in this step, and its owner writes nothing
        const double piv = M[k * W + k];
        if (lane < 2 * n && lane != k) {
            const double rk = M[k * W + lane] / piv;
            M[k * W + lane] = rk;
            for (int r = 0; r < n; ++r)
                if (r != k) M[r * W + lane] -= M[r * W + k] * rk;
        }
        __syncwarp();
    }
    for (int e = lane; e < n * n; e += 32) {
        const int r = e / n, c = e % n;
        const double s = 0.5 * (M[r * W + n + c] + M[c * W + n + r]);
        S.dinv[e] = s;
        dst[e] = s;
    }
}

// The domain's block levels of the set-up: for l = lc .. nlev-2 the smoother
// and interpolation weights of level l and the Galerkin operator of level
// l+1, then the coarsest level's inverse; in shared memory, and copied to
// global memory for a block that must reload them.
__device__ void block_setup(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g, double *smem) {
    const SmemMG S = smem_mg(smem);
    SL lv[MG_MAXLEV];
    s_levels(g, lv);
    block_load(P, D, ctot, g, S, lv, false);
    for (int l = g.lc; l + 1 < g.nlev; ++l) {
        const SL f = lv[l], c = lv[l + 1];
        const Lvl gf = level(g, l), gc = level(g, l + 1);
        const bool hx = g.hx[l], hy = g.hy[l];
        __syncthreads();
        s_points(f, [&](int i, int j) {
            const int q = f.at(i, j);
            const double w = l == 0 ? 0.8 / S.a[0][q] : smoother_inv(s_row(S, f, i, j));
            S.w[q] = w;
            if (l > 0) P.mg_w[gf.at(i, j)] = w;
            const float4 pw = interp_weights([&](int ii, int jj) { return s_row(S, f, ii, jj); }, i, j, f.m, f.n, hx, hy);
            S.pw[q] = pw;
            *pw_ptr(P, g, l, i, j) = pw;
        });
        __syncthreads();
        s_points(c, [&](int I, int J) {
            double acc[5];
            galerkin_row([&](int i, int j) { return s_row(S, f, i, j); }, [&](int i, int j) { return S.pw[f.at(i, j)]; },
                         f.m, f.n, hx, hy, c.m, c.n, I, J, acc);
            const int q = c.at(I, J);
            const long long at = gc.at(I, J);
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                S.a[k][q] = acc[k];
                P.mg_a[(size_t)k * P.mg_nc + at] = acc[k];
            }
        });
    }
    __syncthreads();
    // the vectors' space is free during the set-up: the elimination's scratch
    if (threadIdx.x < 32) dense_inverse(S, lv[g.nlev - 1], S.x, P.mg_dinv + g.dio);
    __syncthreads();
}

// One V-cycle over the block levels: from x_lc = W^-1 b_lc (already formed)
// down to the coarsest level, its exact solve, and back up; level lc's result
// goes back to its t vector in global memory.  `resident` is the domain whose
// set-up is in shared memory.
__device__ void block_vcycle(const DevPtrs &P, const DomainDesc &D, long long ctot, const MgDom &g, int dom,
                             double *smem, int &resident) {
    const SmemMG S = smem_mg(smem);
    SL lv[MG_MAXLEV];
    s_levels(g, lv);
    const bool reload = resident != dom;
    __syncthreads();  // every thread has read `resident`
    if (reload) {
        block_load(P, D, ctot, g, S, lv, true);
        if (threadIdx.x == 0) resident = dom;
    }
    {
        const SL v = lv[g.lc];
        const Lvl gl = level(g, g.lc);
        const LvlVec gv = vectors(P, g.lc);
        s_points(v, [&](int i, int j) {
            S.b[v.at(i, j)] = __ldcg(gv.b + gl.at(i, j));
            S.x[v.at(i, j)] = __ldcg(gv.x + gl.at(i, j));
        });
    }
    const int L = g.nlev - 1;
    // ---- down
    for (int l = g.lc; l < L; ++l) {
        const SL f = lv[l], c = lv[l + 1];
        const bool hx = g.hx[l], hy = g.hy[l];
        __syncthreads();
        s_points(f, [&](int i, int j) { S.t[f.at(i, j)] = S.b[f.at(i, j)] - s_apply(s_row(S, f, i, j), S.x, f, i, j); });
        __syncthreads();
        s_points(c, [&](int I, int J) {
            double acc = 0.0;
#pragma unroll
            for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                for (int aa = 0; aa < 3; ++aa) {
                    int fx, fy;
                    double vx, vy;
                    child(I, aa, hx, f.m, fx, vx);
                    child(J, bb, hy, f.n, fy, vy);
                    if (vx != 0.0 && vy != 0.0)
                        acc += slot(S.pw[f.at(fx, fy)], child_slot(aa, hx) + 2 * child_slot(bb, hy)) * S.t[f.at(fx, fy)];
                }
            const int q = c.at(I, J);
            S.b[q] = acc;
            if (l + 1 < L) S.x[q] = S.w[q] * acc;
        });
    }
    // ---- coarsest level: t = A^-1 b
    {
        __syncthreads();
        const SL v = lv[L];
        const int nd = v.m * v.n;
        for (int r = threadIdx.x; r < nd; r += blockDim.x) {
            double s = 0.0;
            for (int k = 0; k < nd; ++k) s += S.dinv[r * nd + k] * S.b[v.o + k];
            S.t[v.o + r] = s;
        }
    }
    // ---- up: x_l += P t_{l+1}, then t_l = x_l + W^-1 (b_l - A_l x_l)
    for (int l = L - 1; l >= g.lc; --l) {
        const SL f = lv[l], c = lv[l + 1];
        const bool hx = g.hx[l], hy = g.hy[l];
        __syncthreads();
        s_points(f, [&](int i, int j) {
            int px0, px1, py0, py1;
            double ux0, ux1, uy0, uy1;
            parents2(i, hx, c.m, px0, ux0, px1, ux1);
            parents2(j, hy, c.n, py0, uy0, py1, uy1);
            const float4 w = S.pw[f.at(i, j)];
            double sum = 0.0;
            if (ux0 != 0.0 && uy0 != 0.0) sum += (double)w.x * S.t[c.at(px0, py0)];
            if (ux1 != 0.0 && uy0 != 0.0) sum += (double)w.y * S.t[c.at(px1, py0)];
            if (ux0 != 0.0 && uy1 != 0.0) sum += (double)w.z * S.t[c.at(px0, py1)];
            if (ux1 != 0.0 && uy1 != 0.0) sum += (double)w.w * S.t[c.at(px1, py1)];
            S.x[f.at(i, j)] += sum;
        });
        __syncthreads();
        s_points(f, [&](int i, int j) {
            const int q = f.at(i, j);
            S.t[q] = S.x[q] + S.w[q] * (S.b[q] - s_apply(s_row(S, f, i, j), S.x, f, i, j));
        });
    }
    __syncthreads();
    // ---- level lc's result
    {
        const SL v = lv[g.lc];
        const Lvl gl = level(g, g.lc);
        double *tg = vectors(P, g.lc).t;
        s_points(v, [&](int i, int j) { tg[gl.at(i, j)] = S.t[v.at(i, j)]; });
    }
    __syncthreads();
}

// ------------------------------------------------------------ domain sums
// Sums of the given chunk-partial slots over the domain's level-0 chunks,
// taken by each warp on its own (lane k sums chunks k, k+32, ..., then a
// butterfly), so every warp of every block gets the same bits with no block
// barrier.
template <int NV>
__device__ __forceinline__ void chunk_sums(const DevPtrs &P, const MgDom &g, const int (&slot)[NV], double (&v)[NV]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = 0.0;
#pragma unroll 8
    for (int k = lane; k < g.c0_count; k += 32) {
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] += __ldcg(&P.mg_part[(size_t)slot[i] * P.mg_nchunk0 + g.c0_first + k]);
    }
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
}

// The CG's stop decision of a domain after `it` updates of x: converged
// (||r|| <= tol ||b||), iteration cap, non-finite residual, or a breakdown of
// the last step (p.q or r.z not positive).
__device__ __forceinline__ bool mg_stop(const DomainDesc &D, int it, double rr, double bb, double pq, double rz) {
    const double tol2 = D.overland_tol * D.overland_tol;
    bool stop = rr <= tol2 * bb || it >= D.overland_maxiter || !(rr == rr);
    if (it > 0) stop = stop || !(pq > 0.0) || !(rz > 0.0) || !(pq < 1e300);
    return stop;
}

struct DomSums {
    double rr, bb, pq, rz;
};

__device__ __forceinline__ DomSums decision_sums(const DevPtrs &P, const MgDom &g, int it) {
    const int slots[4] = {MP_RR, MP_BB, MP_PQ, MP_RZ + ((it + 1) & 1)};  // r.z of iteration it-1
    double v[4];
    chunk_sums<4>(P, g, slots, v);
    return DomSums{v[0], v[1], v[2], v[3]};
}

}  // namespace

// --------------------------------------------------------------- the solve
__global__ void __launch_bounds__(OLF_THREADS, 2) k_olf_mgcg(DevPtrs P, long long ctot) {
    extern __shared__ double s_mg[];  // a domain's block levels (block_vcycle)
    __shared__ int s_resident;        // the domain whose block levels are set up in s_mg
    const int tid = threadIdx.x;
    if (tid == 0) s_resident = -1;
    // barrier: one counter that every block adds to once per phase (zeroed by
    // k_olf_setup before every solve)
    unsigned int epoch = 0;
    auto sync = [&]() { return counter_sync(&P.gctrl->olf_bar, (++epoch) * gridDim.x, P.barrier); };
    const int Lg = P.mg_lg;
    const int nchunk0 = P.mg_nchunk0;
    double *part = P.mg_part;
    auto pslot = [&](int slot, int chunk) -> double & { return part[(size_t)slot * nchunk0 + chunk]; };
    // chunks of level l, block-strided; fn(chunk, MgDom, DomainDesc)
    auto chunks = [&](int l, auto fn) {
        for (int k = P.mg_lchunk[l] + blockIdx.x; k < P.mg_lchunk[l + 1]; k += gridDim.x) {
            const MgChunk ch = P.mgc[k];
            fn(k, ch, P.mgd[ch.dom], P.dom[ch.dom]);
        }
    };
    auto point_of = [&](const MgChunk &ch, const MgDom &g, int &i, int &j) {
        const int p = ch.first + tid;
        if (tid >= ch.count) return false;
        i = p % g.m[ch.lev];
        j = p / g.m[ch.lev];
        return true;
    };
    // the points of a level-0 chunk (MG_CHUNK0 = 4 per thread)
    auto points0 = [&](const MgChunk &ch, const MgDom &g, auto fn) {
#pragma unroll
        for (int q = 0; q < MG_CHUNK0 / OLF_THREADS; ++q) {
            const int o = tid + q * OLF_THREADS;
            if (o < ch.count) {
                const int p = ch.first + o;
                fn(p % g.m[0], p / g.m[0]);
            }
        }
    };
    auto active = [&](int d) { return __ldcg(&P.mgctl[d].active) != 0; };

    // ---- S0: r = b - A x, b.b and r.r partials, z = W^-1 r; level 0's
    // interpolation weights where level 0 is a grid level
    if (blockIdx.x == 0)
        for (int d = tid; d < P.ndom; d += blockDim.x) {
            P.mgctl[d].active = (P.mgd[d].nlev > 0 && !P.dom[d].frozen) ? 1 : 0;
            if (!P.mgctl[d].active) {
                P.octrl[d].iter = 0;
                P.octrl[d].rr = 0.0;
                P.octrl[d].bb = 0.0;
            }
        }
    chunks(0, [&](int k, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
        double v[2] = {0.0, 0.0};
        points0(ch, g, [&](int i, int j) {
            const Lvl f = level(g, 0);
            const long long c = f.at(i, j);
            const OlfCoef cf = olf_coef(P, D, c, ctot);
            const double b = P.olf_b[c];
            const double r = b - olf_av<false>(cf, P.H, c, f.nx, P.H[c]);
            const double w0 = 0.8 / cf.dg;
            P.mg_w0[c] = w0;
            P.olf_r[c] = r;
            P.olf_z[c] = w0 * r;
            v[0] += r * r;
            v[1] += b * b;
            if (g.lc >= 1) weight_point(P, D, ctot, g, 0, i, j);
        });
        olf_block_sum<2>(v);
        if (tid == 0) {
            pslot(MP_RR, k) = v[0];
            pslot(MP_BB, k) = v[1];
        }
    });
    if (!sync()) return;
    // ---- set-up of the grid levels: A_l and the restriction into level l,
    // then level l's smoother and interpolation weights where level l is a
    // grid level
    for (int l = 1; l <= Lg; ++l) {
        chunks(l, [&](int, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
            int I, J;
            if (point_of(ch, g, I, J)) {
                if (l == 1) setup_point<true>(P, D, ctot, g, 0, I, J);
                else setup_point<false>(P, D, ctot, g, l - 1, I, J);
            }
        });
        if (!sync()) return;
        if (l < Lg) {
            chunks(l, [&](int, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
                int i, j;
                if (l < g.lc && point_of(ch, g, i, j)) weight_point(P, D, ctot, g, l, i, j);
            });
            if (!sync()) return;
        }
    }
    // ---- set-up of every domain's block levels
    for (int d = blockIdx.x; d < P.ndom; d += gridDim.x) {
        const MgDom &g = P.mgd[d];
        if (g.nlev > 0) {
            block_setup(P, P.dom[d], ctot, g, s_mg);
            if (tid == 0) s_resident = d;
        }
    }
    if (!sync()) return;

    // The stop decision after `it` updates of x, taken in the first phase of a
    // V-cycle: each domain's by block d mod gridDim, which records a stop and
    // counts the domain live (slot it % 3 of olf_live, read after the
    // barrier; the slot of it + 2 is cleared here for later), and again by
    // every block for the domains of its chunks.
    auto decide_own = [&](int it) {
        if (blockIdx.x == 0 && tid == 0) P.gctrl->olf_live[(it + 2) % 3] = 0;
        for (int d = blockIdx.x; d < P.ndom; d += gridDim.x) {
            if (!active(d)) continue;  // only this block writes the flag of d
            const DomSums sm = decision_sums(P, P.mgd[d], it);
            if (tid == 0) {
                if (mg_stop(P.dom[d], it, sm.rr, sm.bb, sm.pq, sm.rz)) {
                    P.mgctl[d].active = 0;
                    P.octrl[d].iter = it;
                    P.octrl[d].rr = sm.rr;
                    P.octrl[d].bb = sm.bb;
                } else {
                    atomicAdd(&P.gctrl->olf_live[it % 3], 1);
                }
            }
        }
    };
    // The same decision for a domain this block works on (the owner may clear
    // the flag during this phase: either value leads to the same outcome).
    auto live_after = [&](int d, int it, int &cache_dom, bool &cache_live) {
        if (d != cache_dom) {
            cache_dom = d;
            cache_live = active(d);
            if (cache_live) {
                const DomSums sm = decision_sums(P, P.mgd[d], it);
                cache_live = !mg_stop(P.dom[d], it, sm.rr, sm.bb, sm.pq, sm.rz);
            }
        }
        return cache_live;
    };

    for (int it = 0;; ++it) {
        // ---- down: restriction with the residual fused, grid levels
        for (int l = 0; l < Lg; ++l) {
            if (l == 0) decide_own(it);
            int cd = -1;
            bool cl = false;
            chunks(l + 1, [&](int, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
                const bool go = l == 0 ? live_after(ch.dom, it, cd, cl) : active(ch.dom);
                int I, J;
                if (go && point_of(ch, g, I, J)) {
                    if (l == 0) restrict_point<true>(P, D, ctot, g, l, I, J);
                    else restrict_point<false>(P, D, ctot, g, l, I, J);
                }
            });
            if (!sync()) return;
            if (l == 0 && __ldcg(&P.gctrl->olf_live[it % 3]) == 0) return;
        }
        // ---- the domains' block levels
        if (Lg == 0) decide_own(it);
        {
            int cd = -1;
            bool cl = false;
            for (int d = blockIdx.x; d < P.ndom; d += gridDim.x) {
                const MgDom &g = P.mgd[d];
                const bool go = Lg == 0 ? live_after(d, it, cd, cl) : active(d);
                if (go && g.nlev > 0) block_vcycle(P, P.dom[d], ctot, g, d, s_mg, s_resident);
            }
        }
        if (!sync()) return;
        if (Lg == 0 && __ldcg(&P.gctrl->olf_live[it % 3]) == 0) return;
        // ---- up: prolongation with the post-smoothing fused, grid levels
        for (int l = Lg - 1; l >= 1; --l) {
            chunks(l, [&](int, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
                int i, j;
                if (ch.lev < g.lc && active(ch.dom) && point_of(ch, g, i, j))
                    smooth_up_point<false>(P, D, ctot, g, l, i, j);
            });
            if (!sync()) return;
        }
        // ---- level 0: z (the preconditioned residual, in olf_w) and r.z
        chunks(0, [&](int k, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
            if (!active(ch.dom)) return;
            // every point's value first, then the stores (as in X and Y)
            constexpr int NQ = MG_CHUNK0 / OLF_THREADS;
            const Lvl f = level(g, 0);
            long long cq[NQ];
            double tq[NQ], rq[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const int o = tid + q * OLF_THREADS;
                const int pt = ch.first + (o < ch.count ? o : 0);
                const int i = pt % f.m, j = pt / f.m;
                cq[q] = f.at(i, j);
                tq[q] = g.lc > 0 ? smooth_up_value<true>(P, D, ctot, g, 0, i, j) : __ldcg(P.olf_w + cq[q]);
                rq[q] = __ldcg(P.olf_r + cq[q]);
            }
            double v[1] = {0.0};
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                if (tid + q * OLF_THREADS >= ch.count) continue;
                if (g.lc > 0) P.olf_w[cq[q]] = tq[q];
                v[0] += rq[q] * tq[q];
            }
            olf_block_sum<1>(v);
            if (tid == 0) pslot(MP_RZ + (it & 1), k) = v[0];
        });
        if (!sync()) return;
        // ---- X: p = z + beta p, q = A z + beta q, p.q
        {
            int cd = -1;
            double beta = 0.0;
            chunks(0, [&](int k, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
                if (!active(ch.dom)) return;
                if (ch.dom != cd) {
                    cd = ch.dom;
                    const int slots[2] = {MP_RZ + (it & 1), MP_RZ + ((it + 1) & 1)};
                    double v[2];
                    chunk_sums<2>(P, g, slots, v);
                    beta = it == 0 ? 0.0 : v[0] / v[1];
                }
                // every point's loads first, then the stores (the compiler may
                // not move a point's loads across an earlier point's stores)
                constexpr int NQ = MG_CHUNK0 / OLF_THREADS;
                const Lvl f = level(g, 0);
                long long cq[NQ];
                double zq[NQ], azq[NQ], pq0[NQ], sq0[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int o = tid + q * OLF_THREADS;
                    const int pt = ch.first + (o < ch.count ? o : 0);
                    cq[q] = f.at(pt % f.m, pt / f.m);
                    const OlfCoef cf = olf_coef(P, D, cq[q], ctot);
                    zq[q] = __ldcg(P.olf_w + cq[q]);
                    azq[q] = olf_av<true>(cf, P.olf_w, cq[q], f.nx, zq[q]);
                    pq0[q] = it == 0 ? 0.0 : __ldcg(P.olf_p + cq[q]);
                    sq0[q] = it == 0 ? 0.0 : __ldcg(P.olf_s + cq[q]);
                }
                double pq[1] = {0.0};
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    if (tid + q * OLF_THREADS >= ch.count) continue;
                    const double p = it == 0 ? zq[q] : zq[q] + beta * pq0[q];
                    const double qv = it == 0 ? azq[q] : azq[q] + beta * sq0[q];
                    P.olf_p[cq[q]] = p;
                    P.olf_s[cq[q]] = qv;
                    pq[0] += p * qv;
                }
                olf_block_sum<1>(pq);
                if (tid == 0) pslot(MP_PQ, k) = pq[0];
            });
        }
        if (!sync()) return;
        // ---- Y: x += alpha p, r -= alpha q, r.r, z = W^-1 r
        {
            int cd = -1;
            double alpha = 0.0;
            chunks(0, [&](int k, const MgChunk &ch, const MgDom &g, const DomainDesc &D) {
                if (!active(ch.dom)) return;
                if (ch.dom != cd) {
                    cd = ch.dom;
                    const int slots[2] = {MP_RZ + (it & 1), MP_PQ};
                    double v[2];
                    chunk_sums<2>(P, g, slots, v);
                    alpha = (v[1] > 0.0 && v[0] > 0.0 && v[1] < 1e300) ? v[0] / v[1] : 0.0;
                }
                constexpr int NQ = MG_CHUNK0 / OLF_THREADS;
                const Lvl f = level(g, 0);
                long long cq[NQ];
                double hq[NQ], pq[NQ], rq[NQ], sq[NQ], wq[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int o = tid + q * OLF_THREADS;
                    const int pt = ch.first + (o < ch.count ? o : 0);
                    cq[q] = f.at(pt % f.m, pt / f.m);
                    hq[q] = __ldcg(P.H + cq[q]);
                    pq[q] = __ldcg(P.olf_p + cq[q]);
                    rq[q] = __ldcg(P.olf_r + cq[q]);
                    sq[q] = __ldcg(P.olf_s + cq[q]);
                    wq[q] = __ldcg(P.mg_w0 + cq[q]);
                }
                double rr[1] = {0.0};
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    if (tid + q * OLF_THREADS >= ch.count) continue;
                    P.H[cq[q]] = hq[q] + alpha * pq[q];
                    const double r = rq[q] - alpha * sq[q];
                    P.olf_r[cq[q]] = r;
                    P.olf_z[cq[q]] = wq[q] * r;
                    rr[0] += r * r;
                }
                olf_block_sum<1>(rr);
                if (tid == 0) pslot(MP_RR, k) = rr[0];
            });
        }
        if (!sync()) return;
    }
}

// ------------------------------------------------------------------- host
bool mg_plan(const std::vector<DomainDesc> &doms, std::vector<MgDom> &mgd, std::vector<MgChunk> &chunks,
             int (&lchunk)[MG_MAXLEV + 2], int &lg, long long &nc, long long &npw, long long &ndinv) {
    const int nd = (int)doms.size();
    mgd.assign(nd, MgDom{});
    nc = npw = ndinv = 0;
    lg = 0;
    for (int d = 0; d < nd; ++d) {
        const DomainDesc &D = doms[d];
        MgDom &g = mgd[d];
        std::memset(&g, 0, sizeof(g));
        g.nx = D.nx;
        g.off[0] = D.off2;
        int m = D.nx - 2, n = D.ny - 2;
        if (m < 1 || n < 1) continue;  // no interior cell: nothing to solve
        int L = 0;
        g.m[0] = m;
        g.n[0] = n;
        while ((m >= 3 || n >= 3) && (long long)m * n > MG_DENSE_PTS) {
            if (L + 1 >= MG_MAXLEV) return false;
            g.pwo[L] = npw;
            npw += (long long)m * n;
            g.hx[L] = m >= 3;
            g.hy[L] = n >= 3;
            m = g.hx[L] ? m / 2 : m;
            n = g.hy[L] ? n / 2 : n;
            ++L;
            g.m[L] = m;
            g.n[L] = n;
            g.off[L] = nc;
            nc += (long long)m * n;
        }
        g.nlev = L + 1;
        g.dio = ndinv;
        ndinv += (long long)(m * n) * (m * n);
        // the block levels: the coarsest ones that fit MG_SMEM_PTS together
        long long tail = 0;
        g.lc = g.nlev;
        while (g.lc > 0 && tail + (long long)g.m[g.lc - 1] * g.n[g.lc - 1] <= MG_SMEM_PTS) {
            --g.lc;
            tail += (long long)g.m[g.lc] * g.n[g.lc];
        }
        lg = std::max(lg, g.lc);
    }
    // chunk lists: level 0 for every domain with an interior (the CG's
    // vectors), level l >= 1 for the domains whose grid phases write it
    chunks.clear();
    for (int l = 0; l <= MG_MAXLEV; ++l) {
        lchunk[l] = (int)chunks.size();
        if (l > lg) continue;
        for (int d = 0; d < nd; ++d) {
            MgDom &g = mgd[d];
            if (g.nlev == 0 || (l > 0 && l > g.lc)) continue;
            const int tot = g.m[l] * g.n[l];
            if (l == 0) g.c0_first = (int)chunks.size();
            const int csize = l == 0 ? MG_CHUNK0 : OLF_THREADS;
            for (int f = 0; f < tot; f += csize) chunks.push_back(MgChunk{d, l, f, std::min(csize, tot - f)});
            if (l == 0) g.c0_count = (int)chunks.size() - g.c0_first;
        }
    }
    lchunk[MG_MAXLEV + 1] = (int)chunks.size();
    return true;
}

cudaError_t configure_mg(LaunchCfg &L, int device) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void *)k_olf_mgcg, cudaFuncAttributeMaxDynamicSharedMemorySize, MG_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_olf_mgcg, OLF_THREADS, MG_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    L.mg_blocks = per_sm * prop.multiProcessorCount;
    return cudaSuccess;
}

cudaError_t launch_overland_mg(const DevPtrs &P, const LaunchCfg &L, long long ctot, cudaStream_t s) {
    DevPtrs args = P;
    long long c = ctot;
    void *kargs[] = {&args, &c};
    int need = P.ndom;
    for (int l = 0; l <= P.mg_lg; ++l) need = std::max(need, P.mg_lchunk[l + 1] - P.mg_lchunk[l]);
    const int grid = std::max(1, std::min(L.mg_blocks, need));
    return cudaLaunchCooperativeKernel((const void *)k_olf_mgcg, dim3(grid), dim3(OLF_THREADS), kargs, MG_SMEM_BYTES,
                                       s);
}
