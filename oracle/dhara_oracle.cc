// dhara_oracle.cc -- FP64 CPU restatement of Dhara's integrated flow hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the GPU library and the timed CPU
// baseline.  Nothing in the product links or calls this file.
//
// The code follows the reference line by line (citations per function) with
// the __constant__ physics of include/devconst.h replaced by runtime
// parameters, which is what the reference's own (disabled)
// CopyConstantToDevice (src/device.cu:174-206) intended.  Units: the
// reference evaluates van Genuchten with psi in cm and alpha in 1/cm
// (src/global.cu:79-97); the restatement does the same conversion from the SI
// values it is given.  Loops are OpenMP-parallel so the same code serves as
// the multi-core CPU baseline.
#include "dhara_oracle.h"
#include "kernel_io.h"

#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::vector<double> vec;

struct dhara_oracle {
    dhara_params p;
    int nx, ny, nz;
    long nxy, N;
    // 2D overland (include/class.h:99-129)
    vec ztopo, mann, waterdepth, waterelev, ph, hpoten, qcapa, ppt, esoil, tr;
    vec kw2, ke2, ks2, kn2, a2d, rhs2d;
    std::vector<int> procmap;
    vec rda;
    int nproc;
    // boundary conditions (include/class.h:138-160)
    std::vector<int> bcw, bce, bcs, bcn, bct, bcb;
    vec bcpsiw, bcpsie, bcpsis, bcpsin, bcpsit, bcpsib;
    vec bcqw, bcqe, bcqs, bcqn, bcqt, bcqb;
    // 3D subsurface (include/class.h:162-196)
    vec ksat, alpha_c, nvg_c;
    bool has_alpha, has_n;
    vec psin, psinp1m, psinp1mp1, thetan, thetanp1m, thetanp1mp1, knp1m, cnp1m, cm_saved, psim_last;
    vec a3d, rhs3d, deltam, qss;
    vec quflux, qdflux, qwflux, qeflux, qsflux, qnflux, dtheta, transp, ssflux;
    int solver3d, solver2d;
    dhara_diagnostics diag;
    bool prepared;
};

// ---------------------------------------------------------------- helpers
static inline double mincomp(double a, double b) { return (a > b) ? b : a; }  // src/global.cu:16-18
static inline double maxcomp(double a, double b) { return (a < b) ? b : a; }  // src/global.cu:20-22

static double dot(const vec &a, const vec &b) {
    const long n = (long)a.size();
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}
static double nrm2(const vec &a) { return std::sqrt(dot(a, a)); }

// CUSP DIA SpMV: y = A x with column-major values (pitch = num_rows) and
// out-of-range columns skipped (CUSP/system/cuda/detail/multiply/dia_spmv.h:59-110).
static void dia_spmv(const vec &values, const long *offsets, int ndiag, long n, const vec &x,
                     vec &y) {
#pragma omp parallel for schedule(static)
    for (long row = 0; row < n; ++row) {
        double sum = 0.0;
        for (int d = 0; d < ndiag; ++d) {
            const long col = row + offsets[d];
            if (col >= 0 && col < n) sum += values[(size_t)d * n + row] * x[col];
        }
        y[row] = sum;
    }
}

// cusp::monitor (CUSP/detail/monitor.inl:30,60-63,108-111,181-201): finished
// when ||r|| <= rel_tol*||b|| (absolute tolerance 0) or the count hits the limit.
struct Monitor {
    double b_norm, tol;
    long limit, count;
    double r_norm;
    Monitor(const vec &b, long lim, double rel) : b_norm(nrm2(b)), tol(rel), limit(lim), count(0),
                                                  r_norm(0) {}
    bool finished(const vec &r) {
        r_norm = nrm2(r);
        if (r_norm <= tol * b_norm) return true;
        return count >= limit;
    }
    bool converged() const { return r_norm <= tol * b_norm; }
};

// cusp::krylov::bicgstab with the identity preconditioner
// (CUSP/krylov/detail/bicgstab.inl:64-146).
static void bicgstab(const vec &A, const long *off, int nd, vec &x, const vec &b, Monitor &mon) {
    const long n = (long)b.size();
    vec p(n), r(n), r_star(n), s(n), AMp(n), AMs(n);
    dia_spmv(A, off, nd, n, x, r);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) r[i] = b[i] - r[i];
    p = r;
    r_star = r;
    double r_r_star_old = dot(r_star, r);
    while (!mon.finished(r)) {
        dia_spmv(A, off, nd, n, p, AMp);  // M = I: Mp = p
        const double alpha = r_r_star_old / dot(r_star, AMp);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) s[i] = r[i] - alpha * AMp[i];
        if (mon.finished(s)) {
#pragma omp parallel for schedule(static)
            for (long i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
            break;
        }
        dia_spmv(A, off, nd, n, s, AMs);
        const double omega = dot(AMs, s) / dot(AMs, AMs);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
            x[i] = x[i] + alpha * p[i] + omega * s[i];
            r[i] = s[i] - omega * AMs[i];
        }
        const double r_r_star_new = dot(r_star, r);
        const double beta = (r_r_star_new / r_r_star_old) * (alpha / omega);
        r_r_star_old = r_r_star_new;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) p[i] = r[i] + beta * p[i] - beta * omega * AMp[i];
        ++mon.count;
    }
}

// cusp::krylov::cg with the identity preconditioner (CUSP/krylov/detail/cg.inl:64-128).
static void cg(const vec &A, const long *off, int nd, vec &x, const vec &b, Monitor &mon) {
    const long n = (long)b.size();
    vec y(n), r(n), p(n);
    dia_spmv(A, off, nd, n, x, y);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) r[i] = b[i] - y[i];
    p = r;  // z = M r = r
    double rz = dot(r, r);
    while (!mon.finished(r)) {
        dia_spmv(A, off, nd, n, p, y);
        const double alpha = rz / dot(y, p);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * y[i];
        }
        const double rz_old = rz;
        rz = dot(r, r);
        const double beta = rz / rz_old;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        ++mon.count;
    }
}

// Not a reference solver: CG preconditioned by the vertical (k) tridiagonal
// block of the 7-point DIA matrix, i.e. diagonals 0 (offset -nx*ny), 3 (main)
// and 6 (+nx*ny) of the CUSP poisson7pt ordering.  It solves the same FP64
// system to the same Monitor rule as cg() and bicgstab(), in ~30 instead of
// ~1000 iterations on dz << dx grids, so long-horizon comparisons finish in a
// test's time.  Each column is factored once per solve (Thomas algorithm:
// c'_k = c_k / den_k, den_k = b_k - a_k c'_{k-1}).
static void pcg_column(const vec &A, const long *off, int nd, vec &x, const vec &b, Monitor &mon) {
    const long n = (long)b.size();
    const long sxy = -off[0];  // offsets start at -nx*ny
    const long ncol = sxy, nz = n / sxy;
    vec y(n), r(n), p(n), z(n), cp(n), dinv(n);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < ncol; ++c) {
        double cprev = 0.0;
        for (long k = 0; k < nz; ++k) {
            const long g = k * sxy + c;
            const double a = k > 0 ? A[0 * (size_t)n + g] : 0.0;
            const double cc = k + 1 < nz ? A[6 * (size_t)n + g] : 0.0;
            const double den = A[3 * (size_t)n + g] - a * cprev;
            dinv[g] = 1.0 / den;
            cp[g] = cc / den;
            cprev = cp[g];
        }
    }
    auto apply = [&](const vec &rr, vec &zz) {
#pragma omp parallel for schedule(static)
        for (long c = 0; c < ncol; ++c) {
            double prev = 0.0;
            for (long k = 0; k < nz; ++k) {
                const long g = k * sxy + c;
                const double a = k > 0 ? A[0 * (size_t)n + g] : 0.0;
                prev = (rr[g] - a * prev) * dinv[g];
                zz[g] = prev;
            }
            for (long k = nz - 2; k >= 0; --k) {
                const long g = k * sxy + c;
                zz[g] -= cp[g] * zz[g + sxy];
            }
        }
    };
    (void)nd;
    dia_spmv(A, off, nd, n, x, y);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) r[i] = b[i] - y[i];
    apply(r, z);
    p = z;
    double rz = dot(r, z);
    while (!mon.finished(r)) {
        dia_spmv(A, off, nd, n, p, y);
        const double alpha = rz / dot(y, p);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * y[i];
        }
        apply(r, z);
        const double rz_old = rz;
        rz = dot(r, z);
        const double beta = rz / rz_old;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        ++mon.count;
    }
}

static void solve(int which, const vec &A, const long *off, int nd, vec &x, const vec &b,
                  Monitor &mon) {
    if (which == ORACLE_SOLVER_CG)
        cg(A, off, nd, x, b, mon);
    else if (which == ORACLE_SOLVER_PCG_COLUMN && nd == 7)
        pcg_column(A, off, nd, x, b, mon);
    else if (which == ORACLE_SOLVER_PCG_COLUMN)
        cg(A, off, nd, x, b, mon);
    else
        bicgstab(A, off, nd, x, b, mon);
}

// ------------------------------------------------------- constitutive laws
static inline double alpha_cm_of(const dhara_oracle *o, long i) {
    return (o->has_alpha ? o->alpha_c[i] : o->p.alpha) / 100.0;
}
static inline double n_of(const dhara_oracle *o, long i) { return o->has_n ? o->nvg_c[i] : o->p.n; }

// vanGenuchten (src/global.cu:66-105); alpha in 1/cm, psi converted to cm.
static inline void vg_cell(double alpha, double n, double theta_S, double theta_R, double Ksat,
                           double psi, double *C, double *theta, double *K) {
    const double lambda = n - 1.0;
    const double m = lambda / n;
    const double _psi = psi * 100;
    double _theta;
    if (_psi < 0)
        _theta = (theta_S - theta_R) / std::pow(1.0 + std::pow((alpha * (-_psi)), n), m) + theta_R;
    else
        _theta = theta_S;
    *theta = _theta;
    const double Se = (_theta - theta_R) / (theta_S - theta_R);
    *K = Ksat * std::sqrt(Se) * (1.0 - std::pow(1.0 - std::pow(Se, 1.0 / m), m)) *
         (1.0 - std::pow(1.0 - std::pow(Se, 1.0 / m), m));
    if (_psi < 0)
        *C = 100 * alpha * n * (1.0 / n - 1.0) * std::pow(alpha * std::fabs(_psi), n - 1) *
             (theta_R - theta_S) * std::pow(std::pow(alpha * std::fabs(_psi), n) + 1, 1.0 / n - 2.0);
    else
        *C = 0.0;
}

static void vg_field(dhara_oracle *o, const vec &psi, vec &C, vec &theta, vec &K) {
    const double ts = o->p.theta_s, tr = o->p.theta_r;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < o->N; ++i)
        vg_cell(alpha_cm_of(o, i), n_of(o, i), ts, tr, o->ksat[i], psi[i], &C[i], &theta[i], &K[i]);
}

extern "C" void oracle_van_genuchten(const dhara_params *p, const double *psi, const double *ksat,
                                     const double *alpha_m, const double *nvg, long long N,
                                     double *C, double *theta, double *K) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
        const double a = (alpha_m ? alpha_m[i] : p->alpha) / 100.0;
        const double n = nvg ? nvg[i] : p->n;
        vg_cell(a, n, p->theta_s, p->theta_r, ksat[i], psi[i], &C[i], &theta[i], &K[i]);
    }
}

// vanGenuchtenInverse (src/global.cu:32-52).
extern "C" void oracle_van_genuchten_inverse(const dhara_params *p, const double *theta,
                                             const double *alpha_m, const double *nvg,
                                             long long N, double *psi) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
        const double alpha = (alpha_m ? alpha_m[i] : p->alpha) / 100.0;
        const double n = nvg ? nvg[i] : p->n;
        const double lambda = n - 1.0;
        const double m = lambda / n;
        if (theta[i] < p->theta_s)
            psi[i] = -(1 / alpha) *
                     std::pow(std::pow((p->theta_s - p->theta_r) / (theta[i] - p->theta_r), 1 / m) - 1.0,
                              1 / n) *
                     0.01;
        else
            psi[i] = 0;
    }
}

// ------------------------------------------------------------- lifetime
extern "C" dhara_oracle *oracle_create(const dhara_params *p) {
    if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1) return nullptr;
    dhara_oracle *o = new dhara_oracle();
    o->p = *p;
    o->nx = p->nx;
    o->ny = p->ny;
    o->nz = p->nz;
    o->nxy = (long)p->nx * p->ny;
    o->N = o->nxy * p->nz;
    const long C = o->nxy, N = o->N, FWE = (long)p->nz * p->ny, FSN = (long)p->nz * p->nx;
    for (vec *v : {&o->ztopo, &o->mann, &o->waterdepth, &o->waterelev, &o->ph, &o->hpoten,
                   &o->qcapa, &o->ppt, &o->esoil, &o->tr, &o->kw2, &o->ke2, &o->ks2, &o->kn2,
                   &o->rhs2d, &o->bcpsit, &o->bcpsib, &o->bcqt, &o->bcqb, &o->qss})
        v->assign(C, 0.0);
    o->a2d.assign(5 * C, 0.0);
    o->procmap.assign(C, 0);
    o->bct.assign(C, 1);
    o->bcb.assign(C, 1);
    o->bcw.assign(FWE, 1);
    o->bce.assign(FWE, 1);
    o->bcs.assign(FSN, 1);
    o->bcn.assign(FSN, 1);
    for (vec *v : {&o->bcpsiw, &o->bcpsie, &o->bcqw, &o->bcqe}) v->assign(FWE, 0.0);
    for (vec *v : {&o->bcpsis, &o->bcpsin, &o->bcqs, &o->bcqn}) v->assign(FSN, 0.0);
    for (vec *v : {&o->ksat, &o->psin, &o->psinp1m, &o->psinp1mp1, &o->thetan, &o->thetanp1m,
                   &o->thetanp1mp1, &o->knp1m, &o->cnp1m, &o->cm_saved, &o->rhs3d, &o->deltam,
                   &o->quflux, &o->qdflux, &o->qwflux, &o->qeflux, &o->qsflux, &o->qnflux,
                   &o->dtheta, &o->transp, &o->ssflux})
        v->assign(N, 0.0);
    o->a3d.assign(7 * N, 0.0);
    o->has_alpha = o->has_n = false;
    o->nproc = 1;
    o->rda.assign(p->nz, 0.0);
    o->solver3d = ORACLE_SOLVER_BICGSTAB;
    o->solver2d = ORACLE_SOLVER_CG;
    std::memset(&o->diag, 0, sizeof(o->diag));
    o->prepared = false;
    return o;
}

extern "C" void oracle_destroy(dhara_oracle *o) { delete o; }
extern "C" void oracle_set_solvers(dhara_oracle *o, int s3, int s2) {
    o->solver3d = s3;
    o->solver2d = s2;
}
extern "C" void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
extern "C" int oracle_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static vec *field_ptr(dhara_oracle *o, int f, long *count) {
    const long N = o->N, C = o->nxy, FWE = (long)o->nz * o->ny, FSN = (long)o->nz * o->nx;
    switch (f) {
        case DHARA_F_PSI: *count = N; return &o->psin;
        case DHARA_F_THETA: *count = N; return &o->thetan;
        case DHARA_F_KSAT: *count = N; return &o->ksat;
        case DHARA_F_ALPHA: *count = N; return &o->alpha_c;
        case DHARA_F_NVG: *count = N; return &o->nvg_c;
        case DHARA_F_K: *count = N; return &o->knp1m;
        case DHARA_F_C: *count = N; return &o->cnp1m;
        case DHARA_F_THETA_NEW: *count = N; return &o->thetanp1mp1;
        case DHARA_F_ZTOPO: *count = C; return &o->ztopo;
        case DHARA_F_MANN: *count = C; return &o->mann;
        case DHARA_F_WATERDEPTH: *count = C; return &o->waterdepth;
        case DHARA_F_WATERELEV: *count = C; return &o->waterelev;
        case DHARA_F_PONDING: *count = C; return &o->ph;
        case DHARA_F_PPT: *count = C; return &o->ppt;
        case DHARA_F_ESOIL: *count = C; return &o->esoil;
        case DHARA_F_TR: *count = C; return &o->tr;
        case DHARA_F_HPOTEN: *count = C; return &o->hpoten;
        case DHARA_F_QTOP: *count = C; return &o->bcqt;
        case DHARA_F_BCQW: *count = FWE; return &o->bcqw;
        case DHARA_F_BCQE: *count = FWE; return &o->bcqe;
        case DHARA_F_BCQS: *count = FSN; return &o->bcqs;
        case DHARA_F_BCQN: *count = FSN; return &o->bcqn;
        case DHARA_F_BCQB: *count = C; return &o->bcqb;
        case DHARA_F_BCPSIW: *count = FWE; return &o->bcpsiw;
        case DHARA_F_BCPSIE: *count = FWE; return &o->bcpsie;
        case DHARA_F_BCPSIS: *count = FSN; return &o->bcpsis;
        case DHARA_F_BCPSIN: *count = FSN; return &o->bcpsin;
        case DHARA_F_BCPSIB: *count = C; return &o->bcpsib;
        default: return nullptr;
    }
}

extern "C" int oracle_upload(dhara_oracle *o, int f, const double *src, long long count) {
    long n = 0;
    vec *v = field_ptr(o, f, &n);
    if (!v || count != n) return DHARA_ERR_INVALID;
    v->assign(src, src + n);
    if (f == DHARA_F_ALPHA) o->has_alpha = true;
    if (f == DHARA_F_NVG) o->has_n = true;
    return DHARA_OK;
}

extern "C" int oracle_upload_int(dhara_oracle *o, int f, const int *src, long long count) {
    std::vector<int> *v = nullptr;
    long n = 0;
    const long C = o->nxy, FWE = (long)o->nz * o->ny, FSN = (long)o->nz * o->nx;
    switch (f) {
        case DHARA_FI_BCW: v = &o->bcw; n = FWE; break;
        case DHARA_FI_BCE: v = &o->bce; n = FWE; break;
        case DHARA_FI_BCS: v = &o->bcs; n = FSN; break;
        case DHARA_FI_BCN: v = &o->bcn; n = FSN; break;
        case DHARA_FI_BCB: v = &o->bcb; n = C; break;
        case DHARA_FI_BCT: v = &o->bct; n = C; break;
        case DHARA_FI_PROCMAP: v = &o->procmap; n = C; break;
        default: return DHARA_ERR_INVALID;
    }
    if (count != n) return DHARA_ERR_INVALID;
    v->assign(src, src + n);
    return DHARA_OK;
}

extern "C" int oracle_download(dhara_oracle *o, int f, double *dst, long long count) {
    long n = 0;
    vec *v = field_ptr(o, f, &n);
    if (!v || count != n || (long)v->size() != n) return DHARA_ERR_INVALID;
    std::copy(v->begin(), v->end(), dst);
    return DHARA_OK;
}

extern "C" int oracle_set_roots(dhara_oracle *o, const double *rda, int nproc) {
    if (nproc < 1) return DHARA_ERR_INVALID;
    o->nproc = nproc;
    o->rda.assign(rda, rda + (long)nproc * o->nz);
    return DHARA_OK;
}

extern "C" int oracle_get_diagnostics(dhara_oracle *o, dhara_diagnostics *out) {
    *out = o->diag;
    return DHARA_OK;
}

// CopyDataToDevice's conversion theta -> psi (src/device.cu:321-330).
extern "C" int oracle_psi_from_theta(dhara_oracle *o) {
    oracle_van_genuchten_inverse(&o->p, o->thetan.data(), o->has_alpha ? o->alpha_c.data() : nullptr,
                                 o->has_n ? o->nvg_c.data() : nullptr, o->N, o->psin.data());
    o->psinp1m = o->psin;
    return DHARA_OK;
}

// PreRunningFlowModel (src/global.cu:270-296): theta, K, C at psin.  The
// Krylov iterate psinp1mp1 starts at zero, as ResizeCuspMemory leaves it
// (src/device.cu:51).
extern "C" int oracle_prepare(dhara_oracle *o) {
    vg_field(o, o->psin, o->cnp1m, o->thetan, o->knp1m);
    o->psinp1m = o->psin;
    std::fill(o->psinp1mp1.begin(), o->psinp1mp1.end(), 0.0);
    // WaterElevation initial: H = z + h as SetInitialConditionsHost (src/host.cc:45-47)
    for (long c = 0; c < o->nxy; ++c) o->waterelev[c] = o->ztopo[c] + o->waterdepth[c];
    o->prepared = true;
    return DHARA_OK;
}

// ------------------------------------------------------------- subsurface
// HydraulicConductivityAtInterface (src/subsurface.cu:26-79): arithmetic mean,
// zero on domain faces.
static inline void face_k(const double *K, long g, int i, int j, int k, int nx, int ny, int nz,
                          double *ke, double *kw, double *kn, double *ks, double *ku, double *kd) {
    const long sxy = (long)nx * ny;
    *kd = (k == 0) ? 0 : 0.5 * (K[g] + K[g - sxy]);
    *ku = (k == nz - 1) ? 0 : 0.5 * (K[g] + K[g + sxy]);
    *ks = (j == 0) ? 0 : 0.5 * (K[g] + K[g - nx]);
    *kn = (j == ny - 1) ? 0 : 0.5 * (K[g] + K[g + nx]);
    *kw = (i == 0) ? 0 : 0.5 * (K[g] + K[g - 1]);
    *ke = (i == nx - 1) ? 0 : 0.5 * (K[g] + K[g + 1]);
}

// SetUpLinearSystemsSubsurface (src/subsurface.cu:381-429) with
// SetUpBlockMatrixSubsurface (83-102), SetUpRightHandSideSubsurface (106-122)
// and SetUpBoundaryConditionsSubsurface (126-353) inlined in reference order.
extern "C" void oracle_k_assemble(const dhara_params *pp, const oracle_asm_io *io) {
    const dhara_params &P = *pp;
    const int nx = io->nx, ny = io->ny, nz = io->nz;
    const long sxy = (long)nx * ny, N = sxy * nz;
    const double dx = P.dx, dy = P.dy, dz = P.dz, dt = P.dt;
    const double Ss = P.Ss, poros = P.porosity, sec = P.sec_p_mm2dt_p_m;
    double *a3d = io->a3d, *rhs = io->rhs;
#pragma omp parallel for schedule(static)
    for (long tid = 0; tid < N; ++tid) {
        const int k = (int)(tid / sxy);
        const int j = (int)((tid % sxy) / nx);
        const int i = (int)((tid % sxy) % nx);
        const double dx2inv = -1.0 / (dx * dx), dy2inv = -1.0 / (dy * dy), dz2inv = -1.0 / (dz * dz);
        const long g = tid;
        double ke, kw, kn, ks, ku, kd;
        face_k(io->knp1m, g, i, j, k, nx, ny, nz, &ke, &kw, &kn, &ks, &ku, &kd);
        // block matrix
        a3d[0 * N + tid] = dz2inv * kd;
        a3d[1 * N + tid] = dy2inv * ks;
        a3d[2 * N + tid] = dx2inv * kw;
        a3d[3 * N + tid] = Ss / dt * io->thetanp1m[g] / poros + io->cnp1m[g] / dt - (ke + kw) * dx2inv -
                           (kn + ks) * dy2inv - (ku + kd) * dz2inv;
        a3d[4 * N + tid] = dx2inv * ke;
        a3d[5 * N + tid] = dy2inv * kn;
        a3d[6 * N + tid] = dz2inv * ku;
        // right-hand side
        const long id2d = (long)j * nx + i;
        const int proc = io->procmap[id2d];
        double trodz;
        if (io->tr[id2d] > 0)
            trodz = -io->tr[id2d] * io->root[(long)proc * nz + k] * sec / dz;
        else
            trodz = 0;
        rhs[tid] = Ss / dt * io->thetanp1m[g] / poros * io->psin[g] + io->cnp1m[g] / dt * io->psinp1m[g] -
                   (ku - kd) / dz + (io->thetan[g] - io->thetanp1m[g]) / dt + trodz / dt;
        // boundary conditions
        const long bi = (long)k * ny + j, bj = (long)k * nx + i, bk = (long)j * nx + i;
        auto identity_row = [&](double v) {
            for (int r = 0; r < 7; ++r) a3d[r * N + tid] = (r == 3) ? 1.0 : 0.0;
            rhs[tid] = v;
        };
        if (io->tbc[bk] == 0) {
            if (k == 1) { a3d[0 * N + tid] = 0.0; rhs[tid] -= dz2inv * kd * io->psi_t[bk]; }
            if (k == 0) identity_row(io->psi_t[bk]);
        } else if (k == 0) {
            rhs[tid] += (-io->qt[bk] * dz) * dz2inv;
        }
        if (io->bbc[bk] == 0) {
            if (k == nz - 2) { a3d[6 * N + tid] = 0.0; rhs[tid] -= dz2inv * ku * io->psi_b[bk]; }
            if (k == nz - 1) identity_row(io->psi_b[bk]);
        } else if (k == nz - 1) {
            io->qb[bk] = io->knp1m[tid];
            rhs[tid] += (io->qb[bk] * dz) * dz2inv;
        }
        if (io->sbc[bj] == 0) {
            if (j == 1) { a3d[1 * N + tid] = 0.0; rhs[tid] -= dy2inv * kn * io->psi_s[bj]; }
            if (j == 0) identity_row(io->psi_s[bj]);
        } else if (j == 0) {
            rhs[tid] += (-io->qs[bj] * dy) * dy2inv;
        }
        if (io->nbc[bj] == 0) {
            if (j == ny - 2) { a3d[5 * N + tid] = 0.0; rhs[tid] -= dy2inv * ks * io->psi_n[bj]; }
            if (j == ny - 1) identity_row(io->psi_n[bj]);
        } else if (j == ny - 1) {
            rhs[tid] += (io->qn[bj] * dy) * dy2inv;
        }
        if (io->wbc[bi] == 0) {
            if (i == 1) { a3d[2 * N + tid] = 0.0; rhs[tid] -= dx2inv * ke * io->psi_w[bi]; }
            if (i == 0) identity_row(io->psi_w[bi]);
        } else if (i == 0) {
            rhs[tid] += (-io->qw[bi] * dx) * dx2inv;
        }
        if (io->ebc[bi] == 0) {
            if (i == nx - 2) { a3d[4 * N + tid] = 0.0; rhs[tid] -= dx2inv * kw * io->psi_e[bi]; }
            if (i == nx - 1) identity_row(io->psi_e[bi]);
        } else if (i == nx - 1) {
            rhs[tid] += (io->qe[bi] * dx) * dx2inv;
        }
    }
}

static void assemble(dhara_oracle *o) {
    oracle_asm_io io;
    io.nx = o->nx; io.ny = o->ny; io.nz = o->nz; io.nproc = o->nproc;
    io.psinp1m = o->psinp1m.data(); io.psin = o->psin.data(); io.thetanp1m = o->thetanp1m.data();
    io.thetan = o->thetan.data(); io.knp1m = o->knp1m.data(); io.cnp1m = o->cnp1m.data();
    io.wbc = o->bcw.data(); io.ebc = o->bce.data(); io.sbc = o->bcs.data(); io.nbc = o->bcn.data();
    io.tbc = o->bct.data(); io.bbc = o->bcb.data();
    io.psi_w = o->bcpsiw.data(); io.psi_e = o->bcpsie.data(); io.psi_s = o->bcpsis.data();
    io.psi_n = o->bcpsin.data(); io.psi_t = o->bcpsit.data(); io.psi_b = o->bcpsib.data();
    io.qw = o->bcqw.data(); io.qe = o->bcqe.data(); io.qs = o->bcqs.data(); io.qn = o->bcqn.data();
    io.qt = o->bcqt.data(); io.qb = o->bcqb.data();
    io.tr = o->tr.data(); io.procmap = o->procmap.data(); io.root = o->rda.data();
    io.a3d = o->a3d.data(); io.rhs = o->rhs3d.data();
    oracle_k_assemble(&o->p, &io);
}

extern "C" int oracle_assemble(dhara_oracle *o, double *a3d, double *rhs) {
    assemble(o);
    std::copy(o->a3d.begin(), o->a3d.end(), a3d);
    std::copy(o->rhs3d.begin(), o->rhs3d.end(), rhs);
    return DHARA_OK;
}

// EstimateFluxes (src/global.cu:172-191) on the top layer.
extern "C" void oracle_k_estimate_fluxes(const dhara_params *p, const oracle_top_io *io) {
    const long C = (long)io->nx * io->ny;
    const double dt = p->dt, dz = p->dz;
    for (long tid = 0; tid < C; ++tid) {
        io->hpoten[tid] = io->ph_in[tid] + io->ppt[tid] / 1000 - io->et[tid] * p->sec_p_mm2dt_p_m * dt;
        io->qcapa[tid] = -io->knp1m[tid] * ((io->psinp1m[tid] - io->hpoten[tid] - 0.5 * dz) / (0.5 * dz));
        if (io->ph_in[tid] / dt > io->ksat[tid]) io->qcapa[tid] = maxcomp(io->qcapa[tid], io->ksat[tid]);
    }
}

// IdentifyTopBoundary (src/global.cu:206-257).
extern "C" void oracle_k_identify_top(const dhara_params *p, const oracle_top_io *io) {
    const long C = (long)io->nx * io->ny;
    const double dt = p->dt, dz = p->dz;
    for (long tid = 0; tid < C; ++tid) {
        io->topbc[tid] = 1;
        if (io->hpoten[tid] > 0.0) {
            if (io->hpoten[tid] / dt > io->qcapa[tid])
                io->topqflux[tid] = io->qcapa[tid];
            else
                io->topqflux[tid] = io->hpoten[tid] / dt;
            io->topqflux[tid] = mincomp(io->topqflux[tid], (p->theta_s - io->thetan[tid]) * dz / dt);
            io->topqflux[tid] = mincomp(io->topqflux[tid], io->ksat[tid]);
        } else {
            io->topqflux[tid] = io->hpoten[tid] / dt;
        }
    }
}

// SubsurfaceEstimateInfiltrationPonding (src/subsurface.cu:465-491).
extern "C" void oracle_k_infiltration(const dhara_params *p, const oracle_top_io *io) {
    const long C = (long)io->nx * io->ny;
    const double dt = p->dt, dz = p->dz;
    for (long tid = 0; tid < C; ++tid) {
        if (io->topbc[tid] == 1) {
            io->qss[tid] = io->topqflux[tid];
            io->ph_out[tid] = maxcomp(io->hpoten[tid] - io->qss[tid] * dt, 0.0);
        } else {
            io->qss[tid] = -io->knp1m[tid] * (io->psinp1mp1[tid] - io->psi_top[tid] - dz) / dz;
            io->ph_out[tid] = maxcomp(io->psi_top[tid] - io->qss[tid] * dt, 0.0);
        }
    }
}

// WaterFluxEstimate (src/subsurface.cu:494-629).
extern "C" void oracle_k_water_flux(const dhara_params *pp, const oracle_flux_io *io) {
    const dhara_params &P = *pp;
    const int N = io->nx, M = io->ny, Pz = io->nz;
    const long sxy = (long)N * M, NN = sxy * Pz;
    const double dx = P.dx, dy = P.dy, dz = P.dz, dt = P.dt;
    const double *K = io->knp1m, *psi = io->psinp1mp1;
    // Dirichlet faces make a cell write its neighbour's flux; run serially in
    // that case to keep the reference's last-writer order.
    bool any_dirichlet = false;
    for (long q = 0; q < sxy; ++q) any_dirichlet |= (io->bbc[q] == 0);
    for (long q = 0; q < (long)Pz * M; ++q) any_dirichlet |= (io->wbc[q] == 0) | (io->ebc[q] == 0);
    for (long q = 0; q < (long)Pz * N; ++q) any_dirichlet |= (io->sbc[q] == 0) | (io->nbc[q] == 0);
#pragma omp parallel for schedule(static) if (!any_dirichlet)
    for (long tid = 0; tid < NN; ++tid) {
        const int k = (int)(tid / sxy);
        const int j = (int)((tid % sxy) / N);
        const int i = (int)((tid % sxy) % N);
        const long g = tid, id2d = (long)j * N + i;
        const int proc = io->procmap[id2d];
        const long bi = (long)k * M + j, bj = (long)k * N + i, bk = (long)j * N + i;
        double ke, kw, kn, ks, ku, kd;
        face_k(K, g, i, j, k, N, M, Pz, &ke, &kw, &kn, &ks, &ku, &kd);
        io->qdflux[g] = 0; io->quflux[g] = 0; io->qwflux[g] = 0;
        io->qeflux[g] = 0; io->qsflux[g] = 0; io->qnflux[g] = 0;
        if (k != 0) io->qdflux[g] = kd * ((psi[g - sxy] - psi[g]) / dz + 1);
        if (k != Pz - 1) {
            io->quflux[g] = ku * ((psi[g] - psi[g + sxy]) / dz + 1);
            if (io->bbc[bk] == 0) io->quflux[g + sxy] = ku * ((psi[g] - psi[g + sxy]) / dz + 1);
        }
        if (i != 0) {
            io->qwflux[g] = kw * (psi[g - 1] - psi[g]) / dx;
            if (io->wbc[bi] == 0) io->qwflux[g - 1] = kw * (psi[g - 1] - psi[g]) / dx;
        }
        if (i != N - 1) {
            io->qeflux[g] = ke * (psi[g] - psi[g + 1]) / dx;
            if (io->ebc[bi] == 0) io->qeflux[g + 1] = ke * (psi[g] - psi[g + 1]) / dx;
        }
        if (j != 0) {
            io->qsflux[g] = ks * (psi[g - N] - psi[g]) / dy;
            if (io->sbc[bj] == 0) io->qsflux[g - N] = ks * (psi[g - N] - psi[g]) / dy;
        }
        if (j != M - 1) {
            io->qnflux[g] = kn * (psi[g] - psi[g + N]) / dy;
            if (io->nbc[bj] == 0) io->qnflux[g + N] = kn * (psi[g] - psi[g + N]) / dy;
        }
        if (k == 0) io->qdflux[g] = io->bcqt[bk];
        if (k == Pz - 1 && io->bbc[bk] != 0) io->quflux[g] = io->bcqb[bk];
        if (i == N - 1 && io->ebc[bi] != 0) io->qeflux[g] = io->bcqe[bi];
        if (i == 0 && io->wbc[bi] != 0) io->qwflux[g] = io->bcqw[bi];
        if (j == M - 1 && io->nbc[bj] != 0) io->qnflux[g] = io->bcqn[bj];
        if (j == 0 && io->sbc[bj] != 0) io->qsflux[g] = io->bcqs[bj];
        io->dtheta[g] = io->thetanp1mp1[g] - io->thetan[g];
        if (io->TR[id2d] > 0)
            io->transp[g] = -io->TR[id2d] * P.sec_p_mm2dt_p_m * io->root[(long)proc * Pz + k];
        else
            io->transp[g] = 0;
        io->ssflux[g] = (psi[g] - io->psin[g]) * (P.Ss / dt * io->thetanp1mp1[g] / P.porosity) * dz;
    }
}

// The nine reductions and the water balance of src/subsurface.cu:809-826.
static double water_balance(dhara_oracle *o) {
    oracle_flux_io io;
    io.nx = o->nx; io.ny = o->ny; io.nz = o->nz; io.nproc = o->nproc;
    io.knp1m = o->knp1m.data(); io.psinp1mp1 = o->psinp1mp1.data(); io.psin = o->psin.data();
    io.thetanp1mp1 = o->thetanp1mp1.data(); io.thetan = o->thetan.data();
    io.E_soil = o->esoil.data(); io.TR = o->tr.data(); io.qss = o->qss.data();
    io.bcqw = o->bcqw.data(); io.bcqe = o->bcqe.data(); io.bcqs = o->bcqs.data(); io.bcqn = o->bcqn.data();
    io.bcqt = o->bcqt.data(); io.bcqb = o->bcqb.data();
    io.wbc = o->bcw.data(); io.ebc = o->bce.data(); io.sbc = o->bcs.data(); io.nbc = o->bcn.data();
    io.tbc = o->bct.data(); io.bbc = o->bcb.data();
    io.procmap = o->procmap.data(); io.root = o->rda.data();
    io.quflux = o->quflux.data(); io.qdflux = o->qdflux.data(); io.qwflux = o->qwflux.data();
    io.qeflux = o->qeflux.data(); io.qsflux = o->qsflux.data(); io.qnflux = o->qnflux.data();
    io.dtheta = o->dtheta.data(); io.transp = o->transp.data(); io.evapo = nullptr; io.ssflux = o->ssflux.data();
    oracle_k_water_flux(&o->p, &io);
    const long NN = o->N;
    const double dz = o->p.dz, dt = o->p.dt;
    double s_qu = 0, s_qd = 0, s_qw = 0, s_qe = 0, s_qs = 0, s_qn = 0, s_ss = 0, s_tr = 0, s_dt = 0;
#pragma omp parallel for schedule(static) reduction(+ : s_qu, s_qd, s_qw, s_qe, s_qs, s_qn, s_ss, s_tr, s_dt)
    for (long g = 0; g < NN; ++g) {
        s_qu += o->quflux[g]; s_qd += o->qdflux[g]; s_qw += o->qwflux[g];
        s_qe += o->qeflux[g]; s_qs += o->qsflux[g]; s_qn += o->qnflux[g];
        s_ss += o->ssflux[g]; s_tr += o->transp[g]; s_dt += o->dtheta[g];
    }
    return s_dt * dz + ((s_qe - s_qw) + (s_qn - s_qs) + (s_qu - s_qd)) * dt - s_tr + s_ss * dt;
}

static oracle_top_io top_io(dhara_oracle *o) {
    oracle_top_io io;
    io.nx = o->nx; io.ny = o->ny;
    io.ph_in = o->ph.data(); io.psinp1m = o->psinp1m.data(); io.knp1m = o->knp1m.data();
    io.ppt = o->ppt.data(); io.et = o->esoil.data(); io.ksat = o->ksat.data(); io.thetan = o->thetan.data();
    io.psinp1mp1 = o->psinp1mp1.data(); io.psi_top = o->bcpsit.data();
    io.hpoten = o->hpoten.data(); io.qcapa = o->qcapa.data(); io.topqflux = o->bcqt.data();
    io.qss = o->qss.data(); io.ph_out = o->ph.data(); io.topbc = o->bct.data();
    return io;
}

// SubsurfaceFlowModel (src/subsurface.cu:686-847).  rain_mm, when given,
// replaces ppt_ground by a uniform depth per step.
extern "C" int oracle_subsurface_step(dhara_oracle *o, const double *rain_mm) {
    if (!o->prepared) return DHARA_ERR_STATE;
    const dhara_params &P = o->p;
    const long C = o->nxy, N = o->N;
    const double dt = P.dt, dz = P.dz;
    if (rain_mm)
        for (long c = 0; c < C; ++c) o->ppt[c] = *rain_mm;
    // psinp1m <- psin (:704)
    o->psinp1m = o->psin;
    const oracle_top_io tio = top_io(o);
    oracle_k_estimate_fluxes(&P, &tio);
    const long lnoff[7] = {-C, -(long)o->nx, -1, 0, 1, (long)o->nx, C};
    int runflag = 0, niter = 0;
    const int maxiter = P.picard_maxiter;
    double maxError = 0;
    long kry_iters = 0;
    while (runflag == 0 && niter < maxiter) {
        vg_field(o, o->psinp1m, o->cnp1m, o->thetanp1m, o->knp1m);
        oracle_k_identify_top(&P, &tio);
        assemble(o);
        if (P.theta_update == DHARA_THETA_CONSERVATIVE) {
            o->cm_saved = o->cnp1m;
            o->psim_last = o->psinp1m;
        }
        Monitor mon(o->rhs3d, P.krylov_maxiter, P.krylov_tol);
        solve(o->solver3d, o->a3d, lnoff, 7, o->psinp1mp1, o->rhs3d, mon);
        kry_iters += mon.count;
        if (!mon.converged()) o->diag.krylov_nonconverged++;
        o->diag.krylov_relres_last = mon.b_norm > 0 ? mon.r_norm / mon.b_norm : mon.r_norm;
        vg_field(o, o->psinp1mp1, o->cnp1m, o->thetanp1mp1, o->knp1m);
        niter += 1;
        // GetIterationDifference + max_element (src/subsurface.cu:432-446,762-780)
        double mx = -INFINITY;
        const int rule = P.picard_rule;
#pragma omp parallel for schedule(static) reduction(max : mx)
        for (long t = 0; t < N; ++t) {
            double d;
            if (rule == DHARA_PICARD_THETA_RELATIVE)
                d = std::fabs((o->thetanp1mp1[t] - o->thetanp1m[t]) / o->thetanp1mp1[t]);
            else if (rule == DHARA_PICARD_PSI_ABSOLUTE)
                d = std::fabs(o->psinp1mp1[t] - o->psinp1m[t]);
            else
                d = std::fabs((o->psinp1mp1[t] - o->psinp1m[t]) / o->psinp1mp1[t]);
            o->deltam[t] = d;
            mx = (d > mx) ? d : mx;
        }
        maxError = mx;
        if (maxError < P.picard_tol) {
            runflag = 1;
        } else {
            // ModifiedPicardUpdate (src/subsurface.cu:450-461)
#pragma omp parallel for schedule(static)
            for (long t = 0; t < N; ++t)
                o->psinp1m[t] = P.am * o->psinp1m[t] + (1 - P.am) * o->psinp1mp1[t];
        }
    }
    oracle_k_infiltration(&P, &tio);
    const double mb = water_balance(o);
    o->diag.mb_subsurface_last = mb;
    o->diag.mb_subsurface_cum += mb;

    // Balance terms that telescope across steps (not computed by the
    // reference): storage uses the theta that becomes the next theta^n and the
    // specific-storage term of the assembled matrix (theta^m).
    const int upd = P.theta_update;
    double s_store = 0, s_top = 0, s_bot = 0;
#pragma omp parallel for schedule(static) reduction(+ : s_store)
    for (long t = 0; t < N; ++t) {
        double th_next;
        if (upd == DHARA_THETA_FINAL)
            th_next = o->thetanp1mp1[t];
        else if (upd == DHARA_THETA_CONSERVATIVE)
            th_next = o->thetanp1m[t] + o->cm_saved[t] * (o->psinp1mp1[t] - o->psim_last[t]);
        else
            th_next = o->thetanp1m[t];
        s_store += dz * (th_next - o->thetan[t]) +
                   dz * P.Ss * o->thetanp1m[t] / P.porosity * (o->psinp1mp1[t] - o->psin[t]);
        o->dtheta[t] = th_next;  // reuse as scratch for the rollover below
    }
    double s_rain = 0;
    for (long c = 0; c < C; ++c) {
        s_top += o->bcqt[c] * dt;
        if (o->bcb[c] != 0) s_bot += o->bcqb[c] * dt;
        s_rain += o->ppt[c] / 1000.0;
    }
    o->diag.storage_change_cum += s_store;
    o->diag.top_inflow_cum += s_top;
    o->diag.bottom_outflow_cum += s_bot;
    o->diag.rain_cum += s_rain;
    o->diag.picard_iters_last = niter;
    o->diag.picard_iters_total += niter;
    o->diag.krylov_iters_last = (int)kry_iters;
    o->diag.krylov_iters_total += kry_iters;
    o->diag.picard_err_last = maxError;
    if (!runflag) o->diag.picard_nonconverged++;
    o->diag.steps++;

    // Rollover (src/subsurface.cu:833-840): waterdepth <- ph, psin <- psi^{m+1},
    // thetan <- thetanp1m (or the chosen alternative).
    o->waterdepth = o->ph;
    o->psin = o->psinp1mp1;
#pragma omp parallel for schedule(static)
    for (long t = 0; t < N; ++t) o->thetan[t] = o->dtheta[t];
    return DHARA_OK;
}

// ---------------------------------------------------------------- overland
// UpdateKOverland (src/overland.cu:193-368): Manning conductances with the
// upwinded depth test and the 9-point slope, K0 where dry or flat.
extern "C" void oracle_update_k_overland(const dhara_params *p, const double *Hs, const double *h,
                                         const double *mann, double *kw, double *ke, double *ks,
                                         double *kn) {
    const int N = p->nx, M = p->ny;
    const double dx = p->dx, dy = p->dy, hmin = p->hmin, delta = p->delta, K0 = p->K0;
#pragma omp parallel for schedule(static)
    for (long I = 0; I < (long)N * M; ++I) {
        const int i = (int)(I % N), j = (int)(I / N);
        const double h_ = h[I], Hs_ = Hs[I], mann_ = mann[I];
        double h_p1, Hs_p1, mann_p1, h_m1, Hs_m1, mann_m1, h_pN, Hs_pN, mann_pN, h_mN, Hs_mN, mann_mN;
        if (i == N - 1) { h_p1 = h_; Hs_p1 = Hs_; mann_p1 = mann_; }
        else { h_p1 = h[I + 1]; Hs_p1 = Hs[I + 1]; mann_p1 = mann[I + 1]; }
        if (i == 0) { h_m1 = h_; Hs_m1 = Hs_; mann_m1 = mann_; }
        else { h_m1 = h[I - 1]; Hs_m1 = Hs[I - 1]; mann_m1 = mann[I - 1]; }
        if (j == M - 1) { h_pN = h_; Hs_pN = Hs_; mann_pN = mann_; }
        else { h_pN = h[I + N]; Hs_pN = Hs[I + N]; mann_pN = mann[I + N]; }
        if (j == 0) { h_mN = h_; Hs_mN = Hs_; mann_mN = mann_; }
        else { h_mN = h[I - N]; Hs_mN = Hs[I - N]; mann_mN = mann[I - N]; }
        double Hs_pNp1 = Hs[I], Hs_pNm1 = Hs[I], Hs_mNp1 = Hs[I], Hs_mNm1 = Hs[I];
        if (i > 0 && i < N - 1 && j > 0 && j < M - 1) {
            Hs_pNp1 = Hs[I + N + 1]; Hs_pNm1 = Hs[I + N - 1];
            Hs_mNp1 = Hs[I - N + 1]; Hs_mNm1 = Hs[I - N - 1];
        }
        auto kface = [&](double Hnb, double hnb, double mnb, double S) {
            const bool up = (Hnb > Hs_);
            const double hup = up ? hnb : h_;
            if (hup > hmin && (hnb + h_) / 2. > hmin && std::fabs(S) > delta)
                return std::pow((hnb + h_) / 2., 5. / 3.) / (0.5 * (mnb + mann_) * std::sqrt(S));
            return K0;
        };
        const double Sse = std::sqrt(std::pow((Hs_p1 - Hs_) / dx, 2.) +
                                     std::pow((Hs_pNp1 + Hs_pN - Hs_mNp1 - Hs_mN) / (4 * dy), 2.));
        ke[I] = kface(Hs_p1, h_p1, mann_p1, Sse);
        const double Ssw = std::sqrt(std::pow((Hs_ - Hs_m1) / dx, 2.) +
                                     std::pow((Hs_pN + Hs_pNm1 - Hs_mN - Hs_mNm1) / (4 * dy), 2.));
        kw[I] = kface(Hs_m1, h_m1, mann_m1, Ssw);
        const double Ssn = std::sqrt(std::pow((Hs_pN - Hs_) / dy, 2.) +
                                     std::pow((Hs_pNp1 + Hs_p1 - Hs_pNm1 - Hs_m1) / (4 * dx), 2.));
        kn[I] = kface(Hs_pN, h_pN, mann_pN, Ssn);
        const double Sss = std::sqrt(std::pow((Hs_ - Hs_mN) / dy, 2.) +
                                     std::pow((Hs_p1 + Hs_mNp1 - Hs_m1 - Hs_mNm1) / (4 * dx), 2.));
        ks[I] = kface(Hs_mN, h_mN, mann_mN, Sss);
    }
}

// WaterElevationOverland (src/overland.cu:33-45), UpdateKOverland (193-368) and
// SetUpLinearSystemsOverland (65-189) with ppt = et = infil = 0 as called at
// src/overland.cu:403-406.
extern "C" void oracle_k_overland_setup(const dhara_params *p, const oracle_olf_io *io) {
    const int nx = io->nx, ny = io->ny;
    const long C = (long)nx * ny;
    const double dt = p->dt, dx = p->dx, dy = p->dy;
    for (long c = 0; c < C; ++c) io->waterelev[c] = io->waterdepth[c] + io->ztopo[c];
    oracle_update_k_overland(p, io->waterelev, io->waterdepth, io->mann, io->kw, io->ke, io->ks, io->kn);
    double *a2d = io->a2d;
    for (long tid = 0; tid < C; ++tid) {
        const int i = (int)(tid % nx), j = (int)(tid / nx);
        const double dtodx2 = -dt / (dx * dx), dtody2 = -dt / (dy * dy);
        const double waterdepth = 0.0;
        io->rhs2d[tid] = io->waterelev[tid] + 0. + 0. + 0.;
        if (i == nx - 1) io->ke[tid] = 0;
        if (i == 0) io->kw[tid] = 0;
        if (j == ny - 1) io->kn[tid] = 0;
        if (j == 0) io->ks[tid] = 0;
        a2d[0 * C + tid] = dtody2 * io->ks[tid];
        a2d[1 * C + tid] = dtodx2 * io->kw[tid];
        a2d[2 * C + tid] = 1.0 - dtodx2 * (io->ke[tid] + io->kw[tid]) - dtody2 * (io->kn[tid] + io->ks[tid]);
        a2d[3 * C + tid] = dtodx2 * io->ke[tid];
        a2d[4 * C + tid] = dtody2 * io->kn[tid];
        if (j == 0 || j == ny - 1 || i == 0 || i == nx - 1) {
            for (int k = 0; k < 5; ++k) a2d[k * C + tid] = 0.0;
            a2d[2 * C + tid] = 1.0;
            io->rhs2d[tid] = io->waterelev[tid] + waterdepth;
        }
    }
}

// WaterDepthOverland (src/overland.cu:371-383).
extern "C" void oracle_k_water_depth(const dhara_params *p, const oracle_olf_io *io) {
    const long C = (long)io->nx * io->ny;
    (void)p;
    for (long c = 0; c < C; ++c) io->waterdepth_out[c] = maxcomp(io->waterelev[c] - io->ztopo[c], 0.0);
}

// OverlandFlowModel (src/overland.cu:387-419).
extern "C" int oracle_overland_step(dhara_oracle *o) {
    if (!o->prepared) return DHARA_ERR_STATE;
    const dhara_params &P = o->p;
    const int nx = o->nx, ny = o->ny;
    const long C = o->nxy;
    const double dt = P.dt, dx = P.dx, dy = P.dy;
    vec &H = o->waterelev, &h = o->waterdepth;
    oracle_olf_io io;
    io.nx = nx; io.ny = ny;
    io.waterdepth = h.data(); io.ztopo = o->ztopo.data(); io.mann = o->mann.data();
    io.waterelev = H.data(); io.kw = o->kw2.data(); io.ke = o->ke2.data(); io.ks = o->ks2.data();
    io.kn = o->kn2.data(); io.a2d = o->a2d.data(); io.rhs2d = o->rhs2d.data(); io.waterdepth_out = h.data();
    oracle_k_overland_setup(&P, &io);
    const long off[5] = {-(long)nx, -1, 0, 1, (long)nx};
    Monitor mon(o->rhs2d, P.overland_maxiter, P.overland_tol);
    solve(o->solver2d, o->a2d, off, 5, H, o->rhs2d, mon);
    o->diag.overland_iters_total += mon.count;
    if (!mon.converged()) o->diag.overland_nonconverged++;
    // boundary outflow: implicit flux from interior rows into the fixed ring
    double out = 0, clip = 0, vol = 0;
    for (long tid = 0; tid < C; ++tid) {
        const int i = (int)(tid % nx), j = (int)(tid / nx);
        if (i == 0 || j == 0 || i == nx - 1 || j == ny - 1) continue;
        const double cx = dt / (dx * dx), cy = dt / (dy * dy);
        if (i == 1) out += cx * o->kw2[tid] * (H[tid] - H[tid - 1]);
        if (i == nx - 2) out += cx * o->ke2[tid] * (H[tid] - H[tid + 1]);
        if (j == 1) out += cy * o->ks2[tid] * (H[tid] - H[tid - nx]);
        if (j == ny - 2) out += cy * o->kn2[tid] * (H[tid] - H[tid + nx]);
    }
    for (long c = 0; c < C; ++c) {
        const double d = H[c] - o->ztopo[c];
        if (d < 0) clip += -d;
    }
    oracle_k_water_depth(&P, &io);
    for (long c = 0; c < C; ++c) vol += h[c];
    o->ph = h;
    o->diag.overland_boundary_out_cum += out;
    o->diag.overland_clip_cum += clip;
    o->diag.ponded_volume = vol;
    return DHARA_OK;
}
