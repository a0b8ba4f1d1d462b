// Launchers of the reference's own global.cu kernels, compiled from its source
// (src/global.cu, found through -I on the reference root) -- TEST
// INFRASTRUCTURE for pinning the oracle's restatement.
#include "src/global.cu"

#include "../../include/dhara_gpu.h"
#include "../kernel_io.h"
#include "launch_util.h"

extern "C" int ref_k_van_genuchten(const dhara_params *p, long long N, const double *psi, const double *ksat,
                                   double *C, double *theta, double *K) {
    REF_SET_CONSTANTS(p);
    RefBuf b1, b2, b3, b4, b5;
    double *dC = ref_up<double>(b1, nullptr, N), *dth = ref_up<double>(b2, nullptr, N);
    double *dKs = ref_up(b3, ksat, N), *dK = ref_up<double>(b4, nullptr, N), *dpsi = ref_up(b5, psi, N);
    vanGenuchten<<<(unsigned)((N + 255) / 256), 256>>>(dC, dth, dKs, dK, dpsi, make_int3((int)N, 1, 1));
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    ref_down(C, b1, N);
    ref_down(theta, b2, N);
    ref_down(K, b4, N);
    return 0;
}

extern "C" int ref_k_vg_inverse(const dhara_params *p, long long N, const double *theta, double *psi) {
    REF_SET_CONSTANTS(p);
    RefBuf b1, b2;
    double *dth = ref_up(b1, theta, N), *dpsi = ref_up<double>(b2, nullptr, N);
    vanGenuchtenInverse<<<(unsigned)((N + 255) / 256), 256>>>(dth, dpsi, (int)N);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    ref_down(psi, b2, N);
    return 0;
}

// EstimateFluxes then IdentifyTopBoundary on the top layer (no __syncthreads).
extern "C" int ref_k_top(const dhara_params *p, const oracle_top_io *io) {
    REF_SET_CONSTANTS(p);
    const size_t Cc = (size_t)io->nx * io->ny;
    RefBuf b[12];
    double *ph = ref_up(b[0], io->ph_in, Cc), *hp = ref_up<double>(b[1], nullptr, Cc);
    double *qc = ref_up<double>(b[2], nullptr, Cc), *ps = ref_up(b[3], io->psinp1m, Cc);
    double *kk = ref_up(b[4], io->knp1m, Cc), *pp = ref_up(b[5], io->ppt, Cc), *et = ref_up(b[6], io->et, Cc);
    double *ks = ref_up(b[7], io->ksat, Cc), *th = ref_up(b[8], io->thetan, Cc);
    int *tb = ref_up<int>(b[9], nullptr, Cc);
    double *tq = ref_up<double>(b[10], nullptr, Cc), *pt = ref_up(b[11], io->psi_top, Cc);
    const int3 gs = make_int3(io->nx, io->ny, 1);
    EstimateFluxes<<<(unsigned)((Cc + 127) / 128), 128>>>(ph, hp, qc, ps, kk, pp, et, ks, gs);
    IdentifyTopBoundary<<<(unsigned)((Cc + 127) / 128), 128>>>(hp, qc, tb, tq, ps, pt, th, ks, gs);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    ref_down(io->hpoten, b[1], Cc);
    ref_down(io->qcapa, b[2], Cc);
    ref_down(io->topbc, b[9], Cc);
    ref_down(io->topqflux, b[10], Cc);
    return 0;
}

// The reference's error hook (src/device.cu:162-171) is referenced by its
// host drivers, which these tests never call; a no-op stands in for it.
extern "C" void CheckCudaCall(cudaError_t command, const char *, const char *, int) { (void)command; }
