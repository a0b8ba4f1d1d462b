// device_common.cuh -- device helpers shared by the 3D and 2D kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include <cuda_bf16.h>

#include "internal.h"

// ---------------------------------------------------------------- loads
// Data written by other blocks of a persistent kernel is read through L2
// (ld.global.cg) so no stale L1 line can be returned after a grid barrier.
template <typename T>
__device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

// ------------------------------------------------------- bounded barrier
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// A wait longer than this means a co-residency or logic failure; the kernel
// then records DHARA_ERR_TIMEOUT and returns instead of spinning forever.
#define BARRIER_TIMEOUT_NS 4000000000ull

// Sense-free generation barrier over all blocks of a cooperative launch.
// Returns false (in every thread of the block) when the barrier gave up or
// another block reported an error; the caller must then return.
__device__ __forceinline__ bool grid_sync(GridBarrier *gb) {
    __shared__ int s_ok;
    // global writes of this phase are read by TMA (async proxy) in the next
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned int *vgen = &gb->gen;
        volatile int *verr = &gb->error;
        const unsigned int g = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&gb->count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned int spins = 0;
            while (*vgen == g) {
                if (*verr) { ok = 0; break; }
                if ((++spins & 63u) == 0 && global_ns() - t0 > BARRIER_TIMEOUT_NS) {
                    atomicExch(&gb->error, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*verr) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Grid barrier over a counter: every block adds one (a release reduction)
// and polls with acquire loads until the count reaches target = epoch x
// blocks, so no block resets anything between barriers; the count must be
// zero when the launch starts (the caller zeroes it).  Unlike grid_sync it
// does not order the phase's writes for TMA reads.  Bounded like grid_sync: a
// wait beyond BARRIER_TIMEOUT_NS, or an error raised by another block, sets or
// reads GridBarrier::error and returns false in every thread.
// before_arrive() runs in thread 0 after the block's threads have met and
// before the arrival is released, so what it writes is published with it.
template <typename BeforeArrive>
__device__ __forceinline__ bool counter_sync(unsigned int *count, unsigned int target, GridBarrier *gb,
                                             BeforeArrive before_arrive,
                                             unsigned long long limit_ns = BARRIER_TIMEOUT_NS) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        before_arrive();
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
        const unsigned long long t0 = global_ns();
        unsigned int spins = 0;
        for (;;) {
            unsigned int v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if ((int)(v - target) >= 0) break;
            if ((++spins & 63u) == 0) {
                if (*(volatile int *)&gb->error) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > limit_ns) {
                    atomicExch(&gb->error, 1);
                    ok = 0;
                    break;
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ bool counter_sync(unsigned int *count, unsigned int target, GridBarrier *gb) {
    return counter_sync(count, target, gb, [] {});
}

// --------------------------------------------------------- reductions
// Deterministic block sum of NV doubles (fixed warp/shuffle order); the
// result is returned in every thread.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
    __shared__ double s_w[NV][TILE_THREADS / 32];
    __shared__ double s_out[NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double a = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) s_w[i][warp] = a;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double a = 0.0;
#pragma unroll
        for (int w = 0; w < TILE_THREADS / 32; ++w) a += s_w[threadIdx.x][w];
        s_out[threadIdx.x] = a;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = s_out[i];
    __syncthreads();
}

__device__ __forceinline__ double block_max(double v) {
    __shared__ double s_w[TILE_THREADS / 32];
    __shared__ double s_out;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) s_w[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = s_w[0];
        for (int w = 1; w < TILE_THREADS / 32; ++w) a = fmax(a, s_w[w]);
        s_out = a;
    }
    __syncthreads();
    v = s_out;
    __syncthreads();
    return v;
}

// Per-domain reduction across the tiles of a domain.  Every tile of the
// domain calls it once (all threads, v already block-summed or not: it sums
// the block itself).  The last tile to arrive sums the tiles' partials in
// tile order -- the same order whichever tile is last, so the result is
// bitwise reproducible -- and gets true with the domain totals in v.
template <int NV, bool IS_MAX = false>
__device__ __forceinline__ bool domain_reduce(const DevPtrs &P, int tile, int dom, int slot,
                                              double (&v)[NV]) {
    __shared__ int s_last;
    if (IS_MAX) {
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] = block_max(v[i]);
    } else {
        block_sum<NV>(v);
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) __stcg(&P.partials[(size_t)i * P.ntiles + tile], v[i]);
        __threadfence();
        const DomainDesc &D = P.dom[dom];
        const unsigned int prev = atomicAdd(&P.arrive[dom * 4 + slot], 1u);
        s_last = (prev == (unsigned int)(D.tile_end - D.tile_begin - 1));
    }
    __syncthreads();
    const bool last = s_last != 0;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    const DomainDesc &D = P.dom[dom];
    double acc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = IS_MAX ? -INFINITY : 0.0;
    // SoA partials: consecutive threads read consecutive tiles (coalesced) and
    // the loop carries no dependence, so several loads are in flight.
#pragma unroll 4
    for (int t = D.tile_begin + threadIdx.x; t < D.tile_end; t += blockDim.x) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const double w = __ldcg(&P.partials[(size_t)i * P.ntiles + t]);
            acc[i] = IS_MAX ? fmax(acc[i], w) : acc[i] + w;
        }
    }
    if (IS_MAX) {
#pragma unroll
        for (int i = 0; i < NV; ++i) acc[i] = block_max(acc[i]);
    } else {
        block_sum<NV>(acc);
    }
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = acc[i];
    if (threadIdx.x == 0) P.arrive[dom * 4 + slot] = 0u;
    return true;
}

// ---------------------------------------------------- branch signature
// An order-independent record of discrete decisions: each decision of kind
// `kind` at `step`, entity `index` with outcome `code` contributes
// mix(step, kind, index, code) to a 64-bit sum (mod 2^64), so two runs that
// took the same decisions everywhere have equal sums and any differing
// decision changes the sum (barring a 2^-64 coincidence).  mix is the
// splitmix64 finaliser (Steele, Lea & Flood 2014).
enum { BR_TOPFLUX = 1, BR_PONDCLIP = 2, BR_MANNING = 3, BR_DEPTHCLIP = 4, BR_SATURATION = 5, BR_PICARD = 6,
       BR_OLFITER = 7 };

// whether decisions of `kind` are recorded (DomainDesc::record_branches is a
// bit mask, bit kind - 1)
__device__ __forceinline__ bool records(const DomainDesc &D, int kind) {
    return (D.record_branches >> (kind - 1)) & 1;
}

__device__ __forceinline__ unsigned long long branch_mix(int step, int kind, long long index, unsigned code) {
    unsigned long long x = ((unsigned long long)(unsigned)step << 40) ^ ((unsigned long long)kind << 36) ^
                           (unsigned long long)index ^ ((unsigned long long)code * 0x9e3779b97f4a7c15ull);
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Outcome of the comparison a > b as 0 (below), 1 (within `band` of the
// boundary) or 2 (above).  Decisions are recorded in these three states so
// that a comparison that sits on its boundary up to rounding (a ponding
// clip of exactly the infiltrated depth, a dry cell's H - z) records the same
// state in two runs whatever its rounding; only a move across a band edge
// changes the record.
__device__ __forceinline__ unsigned band3(double a, double b, double band) {
    const double d = a - b;
    return d > band ? 2u : (d < -band ? 0u : 1u);
}
// band for comparing two values of magnitude ~|a|, |b|: relative 1e-9, plus an absolute floor
__device__ __forceinline__ double rel_band(double a, double b, double floor_abs) {
    return 1e-9 * (fabs(a) + fabs(b)) + floor_abs;
}

// Adds every thread's v to *sig: warp sums, one atomic per warp.  All threads
// of the warp must call it (v = 0 where a thread has nothing to add).
__device__ __forceinline__ void branch_commit(unsigned long long *sig, unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sig, v);
}

// ------------------------------------------------------- math wrappers
template <typename T> __device__ __forceinline__ T m_log(T x);
template <> __device__ __forceinline__ double m_log(double x) { return log(x); }
template <> __device__ __forceinline__ float m_log(float x) { return logf(x); }
template <typename T> __device__ __forceinline__ T m_exp(T x);
template <> __device__ __forceinline__ double m_exp(double x) { return exp(x); }
template <> __device__ __forceinline__ float m_exp(float x) { return expf(x); }
template <typename T> __device__ __forceinline__ T m_log1p(T x);
template <> __device__ __forceinline__ double m_log1p(double x) { return log1p(x); }
template <> __device__ __forceinline__ float m_log1p(float x) { return log1pf(x); }
template <typename T> __device__ __forceinline__ T m_expm1(T x);
template <> __device__ __forceinline__ double m_expm1(double x) { return expm1(x); }
template <> __device__ __forceinline__ float m_expm1(float x) { return expm1f(x); }
template <typename T> __device__ __forceinline__ T m_sqrt(T x);
template <> __device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }

// van Genuchten-Mualem closure (the reference's vanGenuchten,
// src/global.cu:66-105).  theta is always returned in double; K and C in T.
//
// T = double: the reference's own expressions and operation order (psi in cm,
// alpha in 1/cm), so the FP64 solver reproduces the reference's arithmetic.
//
// T = float: the same law through the substitution
// s = 1/(1 + (alpha|psi|)^n), Se = s^m, m = 1 - 1/n:
//   K = Ks sqrt(Se) (1 - (1-s)^m)^2 with 1 - (1-s)^m = -expm1(m log1p(-s)),
//   C = alpha (n-1) (theta_s - theta_r) (alpha|psi|)^(n-1) s Se,
// which avoids the cancellation of 1 - pow(Se, 1/m) near saturation that would
// destroy FP32 accuracy.  theta = theta_r + (theta_s - theta_r) Se is formed in
// double so a saturated cell carries theta_s exactly: a rounded theta_s would
// act as a spurious source (theta^n - theta^m)/dt that the tiny specific
// storage of saturated cells turns into a large head error.
template <typename T>
__device__ __forceinline__ void vg_eval(double psi, double alpha, double n, double ts, double tr,
                                        double ks, double &theta, T &K, T &C);

template <>
__device__ __forceinline__ void vg_eval<double>(double psi, double alpha_m, double n, double theta_S,
                                                double theta_R, double Ksat, double &theta, double &K,
                                                double &C) {
    const double alpha = alpha_m / 100.0;
    const double lambda = n - 1.0;
    const double m = lambda / n;
    const double _psi = psi * 100;
    double _theta;
    if (_psi < 0)
        _theta = (theta_S - theta_R) / pow(1.0 + pow((alpha * (-_psi)), n), m) + theta_R;
    else
        _theta = theta_S;
    theta = _theta;
    const double Se = (_theta - theta_R) / (theta_S - theta_R);
    K = Ksat * sqrt(Se) * (1.0 - pow(1.0 - pow(Se, 1.0 / m), m)) * (1.0 - pow(1.0 - pow(Se, 1.0 / m), m));
    if (_psi < 0)
        C = 100 * alpha * n * (1.0 / n - 1.0) * pow(alpha * fabs(_psi), n - 1) * (theta_R - theta_S) *
            pow(pow(alpha * fabs(_psi), n) + 1, 1.0 / n - 2.0);
    else
        C = 0.0;
}

// The same closure in FP64 arithmetic from fewer transcendental calls: with
// x = alpha |psi|, u = 1 + x^n and m = 1 - 1/n,
//   Se = u^-m,  theta = tr + (ts - tr) Se,
//   (1 - Se^(1/m))^m = (x^n / u)^m,  K = Ks Se^(1/2) (1 - (x^n/u)^m)^2,
//   C = alpha (n - 1) (ts - tr) x^(n-1) Se / u,
// from one log, one log1p and three exponentials (expm1 for 1 - (x^n/u)^m).
// It is more accurate than the reference's expressions where Se is close to
// 1 (their 1 - Se^(1/m) cancels, leaving ~1e-8 relative noise in K), so it
// differs from them at that level; the mixed-precision path uses it.
__device__ __forceinline__ void vg_eval_fast(double psi, double alpha_m, double n, double theta_S,
                                             double theta_R, double Ksat, double &theta, double &K, double &C) {
    if (psi < 0.0) {
        const double x = alpha_m * (-psi);
        const double lx = log(x);
        const double xn1 = exp((n - 1.0) * lx);
        const double xn = xn1 * x;
        const double m = (n - 1.0) / n;
        const double lu = log1p(xn);
        const double Se = exp(-m * lu);
        theta = theta_R + (theta_S - theta_R) * Se;
        const double lq = (xn > 1.0) ? -log1p(1.0 / xn) : n * lx - lu;  // log(x^n / u)
        const double f = -expm1(m * lq);
        K = Ksat * sqrt(Se) * f * f;
        C = alpha_m * (n - 1.0) * (theta_S - theta_R) * xn1 * Se / (1.0 + xn);
    } else {
        theta = theta_S;
        K = Ksat;
        C = 0.0;
    }
}

template <>
__device__ __forceinline__ void vg_eval<float>(double psi_d, double alpha_d, double n_d, double ts,
                                               double tr, double ks, double &theta, float &K, float &C) {
    const float psi = (float)psi_d;
    if (psi < 0.f) {
        const float alpha = (float)alpha_d, n = (float)n_d;
        const float x = alpha * (-psi);
        const float lx = logf(x);
        const float xn1 = expf((n - 1.f) * lx);
        const float xn = xn1 * x;
        const float s = 1.f / (1.f + xn);
        const float m = (n - 1.f) / n;
        const float Se = expf(m * logf(s));
        theta = tr + (ts - tr) * (double)Se;
        const float f = -expm1f(m * log1pf(-s));
        K = (float)ks * sqrtf(Se) * f * f;
        C = alpha * (n - 1.f) * (float)(ts - tr) * xn1 * s * Se;
    } else {
        theta = ts;
        K = (float)ks;
        C = 0.f;
    }
}

// theta(psi) alone, in double (the theta Picard rule; src/global.cu:110-114).
__device__ __forceinline__ double vg_theta(double psi, double alpha_m, double n, double theta_S,
                                           double theta_R) {
    const double alpha = alpha_m / 100.0, m = (n - 1.0) / n, _psi = psi * 100;
    if (_psi < 0) return (theta_S - theta_R) / pow(1.0 + pow((alpha * (-_psi)), n), m) + theta_R;
    return theta_S;
}

// Column geometry of a thread inside its tile.
struct ColumnRef {
    int dom, i, j, nx, ny, nz, nxp;
    int tx, ty, tx_log2;  // the tile's shape
    long long g0, sxy;   // cell (i,j,0) index and plane stride
    long long c;         // column index in 2D arrays
    bool valid;
};

__device__ __forceinline__ ColumnRef column_of(const DevPtrs &P, int tile) {
    const TileDesc t = P.tiles[tile];
    const DomainDesc &D = P.dom[t.dom];
    ColumnRef r;
    r.dom = t.dom;
    r.tx = D.tx;
    r.ty = D.ty;
    r.tx_log2 = D.tx_log2;
    r.i = t.x0 + ((int)threadIdx.x & (D.tx - 1));
    r.j = t.y0 + ((int)threadIdx.x >> D.tx_log2);
    r.nx = D.nx;
    r.ny = D.ny;
    r.nz = D.nz;
    r.nxp = D.nxp;
    r.valid = (r.i < D.nx) && (r.j < D.ny);
    r.sxy = (long long)D.nxp * D.ny;
    r.g0 = D.off3 + (long long)r.j * D.nxp + r.i;
    r.c = D.off2 + (long long)r.j * D.nx + r.i;
    return r;
}
