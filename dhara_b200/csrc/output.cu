// output.cu -- per-step statistics the reference's time loop collects.
//
// After each step the reference sums, layer by layer, the new head psi^{m+1}
// and theta(psi^{m+1}) (CopyLayers, src/device.cu:135-147, called at
// src/device.cu:464) and keeps the step's water balance mb_subsurfaceW
// (src/subsurface.cu:809-826); SaveResultEntirePeriod (src/io.cc:962-996)
// writes them as pressure_mean, moisture_mean and mb_subsurfaceW.  CopyLayers
// reduces over [k*nx*ny, (k+1)*nx*ny - 1): the last cell of every layer
// (i = nx-1, j = ny-1) is left out, and so it is here.
#include "device_common.cuh"

// Per tile and layer: partial sums of psi and theta over the tile's columns.
__global__ void __launch_bounds__(TILE_THREADS) k_layer_partials(DevPtrs P, double *part, int nz_max) {
    const int tile = blockIdx.x;
    const ColumnRef cr = column_of(P, tile);
    const DomainDesc &D = P.dom[cr.dom];
    __shared__ double s_psi[TILE_THREADS / 32][NZ_MAX], s_th[TILE_THREADS / 32][NZ_MAX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool use = cr.valid && !(cr.i == cr.nx - 1 && cr.j == cr.ny - 1);
    long long g = cr.g0;
    for (int k = 0; k < D.nz; ++k, g += cr.sxy) {
        double ps = 0.0, th = 0.0;
        if (use) {
            const double a = D.has_alpha ? P.alpha[g] : D.alpha;
            const double n = D.has_n ? P.nvg[g] : D.n;
            double t, K, C;
            if (D.closure_fp32) {
                float Kf, Cf;
                vg_eval<float>(P.psin[g], a, n, D.theta_s, D.theta_r, P.ksat[g], t, Kf, Cf);
            } else if (D.closure_fast) {
                vg_eval_fast(P.psin[g], a, n, D.theta_s, D.theta_r, P.ksat[g], t, K, C);
            } else {
                vg_eval<double>(P.psin[g], a, n, D.theta_s, D.theta_r, P.ksat[g], t, K, C);
            }
            ps = P.psin[g];
            th = t;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ps += __shfl_down_sync(0xffffffffu, ps, o);
            th += __shfl_down_sync(0xffffffffu, th, o);
        }
        if (lane == 0) {
            s_psi[warp][k] = ps;
            s_th[warp][k] = th;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < D.nz; k += blockDim.x) {
        double ps = 0.0, th = 0.0;
        for (int w = 0; w < TILE_THREADS / 32; ++w) {
            ps += s_psi[w][k];
            th += s_th[w][k];
        }
        part[((size_t)tile * nz_max + k) * 2 + 0] = ps;
        part[((size_t)tile * nz_max + k) * 2 + 1] = th;
    }
}

// One block per domain: layer sums over the domain's tiles in tile order, and
// the step's water balance, into the domain's history row for the step.
__global__ void k_layer_totals(DevPtrs P, const double *part, int nz_max, double *hist, int max_steps) {
    const int d = blockIdx.x;
    const DomainDesc &D = P.dom[d];
    const int step = P.pctrl[d].step - 1;  // the step just completed
    if (step < 0 || step >= max_steps) return;
    double *row = hist + ((size_t)d * max_steps + step) * (1 + 2 * nz_max);
    if (threadIdx.x == 0) row[0] = P.diag[d].mb_last;
    for (int k = threadIdx.x; k < D.nz; k += blockDim.x) {
        double ps = 0.0, th = 0.0;
        for (int t = D.tile_begin; t < D.tile_end; ++t) {
            ps += part[((size_t)t * nz_max + k) * 2 + 0];
            th += part[((size_t)t * nz_max + k) * 2 + 1];
        }
        row[1 + k] = ps;
        row[1 + nz_max + k] = th;
    }
}

cudaError_t launch_layer_stats(const DevPtrs &P, double *part, int nz_max, double *hist, int max_steps,
                               cudaStream_t s) {
    k_layer_partials<<<P.ntiles, TILE_THREADS, 0, s>>>(P, part, nz_max);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_layer_totals<<<P.ndom, 64, 0, s>>>(P, part, nz_max, hist, max_steps);
    return cudaGetLastError();
}
