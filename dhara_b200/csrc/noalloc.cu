// noalloc.cu -- an overland step that allocates nothing.
//
// Some callers cannot allocate device memory when they need a step: a host
// application that hands the library only the arrays it owns (a plugin inside
// a model that manages all GPU memory itself and has no spare memory to give),
// or a real-time loop that forbids allocation after start-up.  For
// them dhara_overland_step_noalloc performs one overland step -- the same
// computation as dhara_overland_step for one domain -- on the caller's device
// arrays, and keeps all of its scratch (the four Manning conductances and the
// Krylov vectors) in one file-scope device array of fixed size.
//
// Properties a caller must know:
//  * The scratch array is sized for DHARA_NOALLOC_MAX_COLUMNS columns (nx*ny);
//    larger domains are rejected with DHARA_ERR_UNSUPPORTED.  Every GPU that
//    loads the library holds it (about 1.2 MB) until the process exits.
//  * All calls on a device share that one array, and it keeps the last call's
//    contents.  Calls whose GPU work overlaps (different streams, or
//    different host threads, without ordering between them) race on it and
//    produce wrong results: order them on one stream.
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, that device current) and caches
//    it for the life of the process.  Make that first call before any stream
//    capture begins, and do not call the entry point again on a device after
//    cudaDeviceReset (the cached address then belongs to the old context).
//  * The four arrays must not overlap, except ztopo with mann (both read).
//  * Convergence is not reported: the solve stops at overland_tol or after
//    overland_maxiter iterations, whichever comes first, and returns
//    DHARA_OK either way (the handle-based path counts unconverged solves).
//  * The solve runs in a single thread block, so it suits small domains; the
//    handle-based path is the fast one for large grids.
#include <cstdio>
#include <mutex>

#include "../../include/dhara_gpu.h"

#define NOALLOC_THREADS 1024
#define NOALLOC_ARRAYS 9  // kw, ke, ks, kn, b, r, p, z, q

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_ARRAYS * DHARA_NOALLOC_MAX_COLUMNS];

namespace {

std::mutex g_setup_mutex;
void *g_scratch_ptr[64] = {};

// The same Manning face conductance as the overland set-up kernel (the
// reference's UpdateKOverland, src/overland.cu:279-297).
__device__ __forceinline__ double na_manning(double Hnb, double hnb, double mnb, double Hc, double hc,
                                             double mc, double S, double hmin, double delta, double K0) {
    const double hup = (Hnb > Hc) ? hnb : hc;
    if (hup > hmin && (hnb + hc) / 2. > hmin && fabs(S) > delta)
        return pow((hnb + hc) / 2., 5. / 3.) / (0.5 * (mnb + mc) * sqrt(S));
    return K0;
}

struct NaArgs {
    int nx, ny, maxiter;
    double dx, dy, dt, hmin, delta, K0, tol;
    double *h;           // in: waterdepth before the step; out: after
    const double *z, *mann;
    double *H;           // out: water elevation after the solve
    double *scratch;     // the static array's device address
};

__device__ __forceinline__ double block_sum_na(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < NOALLOC_THREADS / 32; ++w) a += red[w];
        red[32] = a;
    }
    __syncthreads();
    return red[32];
}

// One block: set-up (H = h + z, conductances, right-hand side), Jacobi-PCG on
// the interior with the fixed-elevation ring eliminated, and the depth clip.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_overland_noalloc(NaArgs a) {
    __shared__ double red[33];
    const int N = a.nx, M = a.ny, C = N * M;
    double *kw = a.scratch, *ke = kw + DHARA_NOALLOC_MAX_COLUMNS, *ks = ke + DHARA_NOALLOC_MAX_COLUMNS;
    double *kn = ks + DHARA_NOALLOC_MAX_COLUMNS, *b = kn + DHARA_NOALLOC_MAX_COLUMNS;
    double *r = b + DHARA_NOALLOC_MAX_COLUMNS, *p = r + DHARA_NOALLOC_MAX_COLUMNS;
    double *z = p + DHARA_NOALLOC_MAX_COLUMNS, *q = z + DHARA_NOALLOC_MAX_COLUMNS;
    const double cx = a.dt / (a.dx * a.dx), cy = a.dt / (a.dy * a.dy);
    auto ring = [&](int I) {
        const int i = I % N, j = I / N;
        return i == 0 || j == 0 || i == N - 1 || j == M - 1;
    };
    auto Hs = [&](int I) { return a.h[I] + a.z[I]; };
    // set-up: every value the solve reads is written here, so nothing left in
    // the shared scratch by an earlier call is used
    for (int I = threadIdx.x; I < C; I += blockDim.x) {
        const double h_ = a.h[I], H_ = Hs(I), m_ = a.mann[I];
        a.H[I] = H_;
        b[I] = H_;
        double w_ = 0, e_ = 0, s_ = 0, n_ = 0;
        if (!ring(I)) {
            const double Hp1 = Hs(I + 1), Hm1 = Hs(I - 1), HpN = Hs(I + N), HmN = Hs(I - N);
            const double HpNp1 = Hs(I + N + 1), HpNm1 = Hs(I + N - 1), HmNp1 = Hs(I - N + 1), HmNm1 = Hs(I - N - 1);
            const double Sse = sqrt(pow((Hp1 - H_) / a.dx, 2.) + pow((HpNp1 + HpN - HmNp1 - HmN) / (4 * a.dy), 2.));
            e_ = na_manning(Hp1, a.h[I + 1], a.mann[I + 1], H_, h_, m_, Sse, a.hmin, a.delta, a.K0);
            const double Ssw = sqrt(pow((H_ - Hm1) / a.dx, 2.) + pow((HpN + HpNm1 - HmN - HmNm1) / (4 * a.dy), 2.));
            w_ = na_manning(Hm1, a.h[I - 1], a.mann[I - 1], H_, h_, m_, Ssw, a.hmin, a.delta, a.K0);
            const double Ssn = sqrt(pow((HpN - H_) / a.dy, 2.) + pow((HpNp1 + Hp1 - HpNm1 - Hm1) / (4 * a.dx), 2.));
            n_ = na_manning(HpN, a.h[I + N], a.mann[I + N], H_, h_, m_, Ssn, a.hmin, a.delta, a.K0);
            const double Sss = sqrt(pow((H_ - HmN) / a.dy, 2.) + pow((Hp1 + HmNp1 - Hm1 - HmNm1) / (4 * a.dx), 2.));
            s_ = na_manning(HmN, a.h[I - N], a.mann[I - N], H_, h_, m_, Sss, a.hmin, a.delta, a.K0);
        }
        kw[I] = w_;
        ke[I] = e_;
        ks[I] = s_;
        kn[I] = n_;
    }
    __syncthreads();
    auto diag = [&](int I) { return 1.0 + cx * (ke[I] + kw[I]) + cy * (kn[I] + ks[I]); };
    auto apply = [&](const double *v, int I) {
        const double c = v[I];
        return c + cx * (ke[I] * (c - v[I + 1]) + kw[I] * (c - v[I - 1])) +
               cy * (kn[I] * (c - v[I + N]) + ks[I] * (c - v[I - N]));
    };
    double rr = 0, bb = 0, rz = 0;
    for (int I = threadIdx.x; I < C; I += blockDim.x) {
        bb += b[I] * b[I];
        double rI = 0, zI = 0;
        if (!ring(I)) {
            rI = b[I] - apply(a.H, I);
            zI = rI / diag(I);
        }
        r[I] = rI;
        z[I] = zI;
        p[I] = zI;
        rr += rI * rI;
        rz += rI * zI;
    }
    bb = block_sum_na(bb, red);
    rr = block_sum_na(rr, red);
    rz = block_sum_na(rz, red);
    const double tol2 = a.tol * a.tol * bb;
    for (int it = 0; it < a.maxiter && rr > tol2 && rr == rr; ++it) {
        double pq = 0;
        for (int I = threadIdx.x; I < C; I += blockDim.x) {
            const double qI = ring(I) ? 0.0 : apply(p, I);
            q[I] = qI;
            pq += p[I] * qI;
        }
        pq = block_sum_na(pq, red);
        if (!(pq > 0)) break;
        const double alpha = rz / pq;
        double rr_n = 0, rz_n = 0;
        for (int I = threadIdx.x; I < C; I += blockDim.x) {
            if (ring(I)) continue;
            a.H[I] += alpha * p[I];
            const double rI = r[I] - alpha * q[I];
            const double zI = rI / diag(I);
            r[I] = rI;
            z[I] = zI;
            rr_n += rI * rI;
            rz_n += rI * zI;
        }
        rr_n = block_sum_na(rr_n, red);
        rz_n = block_sum_na(rz_n, red);
        const double beta = rz_n / rz;
        rz = rz_n;
        rr = rr_n;
        for (int I = threadIdx.x; I < C; I += blockDim.x) p[I] = ring(I) ? 0.0 : z[I] + beta * p[I];
        __syncthreads();
    }
    for (int I = threadIdx.x; I < C; I += blockDim.x) a.h[I] = fmax(a.H[I] - a.z[I], 0.0);
}

}  // namespace

int dhara_internal_fail(int code, const char *msg);  // api.cu: sets dhara_last_error

namespace {

int na_fail(int code, const char *msg) { return dhara_internal_fail(code, msg); }

// Device address of the scratch array on the current device, looked up once
// per device with that device current.
int scratch_address(void **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return na_fail(DHARA_ERR_CUDA, "dhara_overland_step_noalloc: no current CUDA device");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            return na_fail(DHARA_ERR_CUDA, "dhara_overland_step_noalloc: cudaGetSymbolAddress failed");
        }
        g_scratch_ptr[dev] = ptr;
    }
    *out = g_scratch_ptr[dev];
    return DHARA_OK;
}

}  // namespace

extern "C" int dhara_overland_step_noalloc(const dhara_params *p, double *waterdepth, const double *ztopo,
                                           const double *mann, double *waterelev, void *stream) {
    if (!p || !waterdepth || !ztopo || !mann || !waterelev)
        return na_fail(DHARA_ERR_INVALID, "dhara_overland_step_noalloc: NULL argument");
    if (p->struct_size != (int)sizeof(dhara_params))
        return na_fail(DHARA_ERR_INVALID, "dhara_overland_step_noalloc: struct_size mismatch");
    if (p->nx < 1 || p->ny < 1 || !(p->dx > 0) || !(p->dy > 0) || !(p->dt > 0) || p->overland_maxiter < 0 ||
        !(p->overland_tol > 0))
        return na_fail(DHARA_ERR_INVALID, "dhara_overland_step_noalloc: invalid grid, time step or tolerance");
    if ((long long)p->nx * p->ny > DHARA_NOALLOC_MAX_COLUMNS) {
        char buf[160];
        snprintf(buf, sizeof(buf),
                 "dhara_overland_step_noalloc: %d x %d = %lld columns exceeds the fixed scratch of %d columns",
                 p->nx, p->ny, (long long)p->nx * p->ny, DHARA_NOALLOC_MAX_COLUMNS);
        return na_fail(DHARA_ERR_UNSUPPORTED, buf);
    }
    // The two written arrays must not overlap each other or the inputs: the
    // set-up writes H while neighbouring threads still read h, z and n.
    {
        const size_t bytes = (size_t)p->nx * p->ny * sizeof(double);
        auto overlap = [bytes](const void *x, const void *y) {
            const char *a0 = (const char *)x, *b0 = (const char *)y;
            return a0 < b0 + bytes && b0 < a0 + bytes;
        };
        if (overlap(waterelev, waterdepth) || overlap(waterelev, ztopo) || overlap(waterelev, mann) ||
            overlap(waterdepth, ztopo) || overlap(waterdepth, mann))
            return na_fail(DHARA_ERR_INVALID,
                           "dhara_overland_step_noalloc: waterdepth and waterelev must not overlap each other, "
                           "ztopo or mann");
    }
    void *scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc) return rc;
    NaArgs a;
    a.nx = p->nx;
    a.ny = p->ny;
    a.maxiter = p->overland_maxiter;
    a.dx = p->dx;
    a.dy = p->dy;
    a.dt = p->dt;
    a.hmin = p->hmin;
    a.delta = p->delta;
    a.K0 = p->K0;
    a.tol = p->overland_tol;
    a.h = waterdepth;
    a.z = ztopo;
    a.mann = mann;
    a.H = waterelev;
    a.scratch = (double *)scratch;
    k_overland_noalloc<<<1, NOALLOC_THREADS, 0, (cudaStream_t)stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(DHARA_ERR_CUDA, cudaGetErrorString(e));
    return DHARA_OK;
}
