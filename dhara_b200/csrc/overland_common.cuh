// overland_common.cuh -- helpers shared by the overland solvers (the
// pipelined Jacobi-PCG of overland.cu and the multigrid-preconditioned CG of
// overland_mg.cu): the fixed boundary ring, the 5-point interior row of the
// reference's SetUpLinearSystemsOverland (src/overland.cu:65-189) and the
// deterministic block and domain sums.
#pragma once
#include "device_common.cuh"

__device__ __forceinline__ bool is_ring(int i, int j, int nx, int ny) {
    return i == 0 || j == 0 || i == nx - 1 || j == ny - 1;
}

template <int NV>
__device__ __forceinline__ void olf_block_sum(double (&v)[NV]) {
    __shared__ double s_w[NV][OLF_THREADS / 32];
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
        for (int w = 0; w < OLF_THREADS / 32; ++w) a += s_w[threadIdx.x][w];
        s_out[threadIdx.x] = a;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = s_out[i];
    __syncthreads();
}

// Domain totals of per-segment partials (component-major: part[i*nseg + s]).
template <int NV>
__device__ __forceinline__ void olf_domain_sum(const double *part, int nseg_tot, int first, int nseg,
                                               double (&v)[NV]) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = 0.0;
    for (int k = threadIdx.x; k < nseg; k += OLF_THREADS) {
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] += __ldcg(&part[(size_t)i * nseg_tot + first + k]);
    }
    olf_block_sum<NV>(v);
}

// 5-point product of the interior row at c: diag*v_c - sum of the scaled
// conductances times the neighbours (row-owned kw, ke, ks, kn as the
// reference's SetUpLinearSystemsOverland builds them).
struct OlfCoef {
    double cw, ce, cs, cn, dg;
};

__device__ __forceinline__ OlfCoef olf_coef(const DevPtrs &P, const DomainDesc &D, long long c, long long ctot) {
    const double cx = D.dt / (D.dx * D.dx), cy = D.dt / (D.dy * D.dy);
    OlfCoef k;
    k.cw = cx * P.olf_k[0 * ctot + c];
    k.ce = cx * P.olf_k[1 * ctot + c];
    k.cs = cy * P.olf_k[2 * ctot + c];
    k.cn = cy * P.olf_k[3 * ctot + c];
    k.dg = 1.0 + (k.ce + k.cw) + (k.cn + k.cs);
    return k;
}

__device__ __forceinline__ double olf_av4(const OlfCoef &k, double vc, double vw, double ve, double vs, double vn) {
    return k.dg * vc - ((k.ce * ve + k.cw * vw) + (k.cn * vn + k.cs * vs));
}

template <bool CG>
__device__ __forceinline__ double olf_av(const OlfCoef &k, const double *v, long long c, int nx, double vc) {
    const double vw = CG ? __ldcg(v + c - 1) : v[c - 1];
    const double ve = CG ? __ldcg(v + c + 1) : v[c + 1];
    const double vs = CG ? __ldcg(v + c - nx) : v[c - nx];
    const double vn = CG ? __ldcg(v + c + nx) : v[c + nx];
    return olf_av4(k, vc, vw, ve, vs, vn);
}

