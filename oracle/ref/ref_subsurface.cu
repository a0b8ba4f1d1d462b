// Launchers of the reference's own subsurface.cu kernels, compiled from its
// source (src/subsurface.cu) -- TEST INFRASTRUCTURE for pinning the oracle.
#include "src/subsurface.cu"

#include "../../include/dhara_gpu.h"
#include "../kernel_io.h"
#include "launch_util.h"

// SetUpLinearSystemsSubsurface calls __syncthreads() inside its grid-stride
// loop; it is launched with exactly one thread per cell in 64-thread blocks,
// so every thread of every block runs the loop once and the barrier is uniform.
extern "C" int ref_k_assemble(const dhara_params *p, const oracle_asm_io *io) {
    REF_SET_CONSTANTS(p);
    const size_t N = (size_t)io->nx * io->ny * io->nz, Cc = (size_t)io->nx * io->ny;
    const size_t WE = (size_t)io->nz * io->ny, SN = (size_t)io->nz * io->nx;
    if (N % 64 != 0) return 2;
    RefBuf b[32];
    int i = 0;
    double *a3d = ref_up<double>(b[i++], nullptr, 7 * N), *rhs = ref_up<double>(b[i++], nullptr, N);
    double *pm = ref_up(b[i++], io->psinp1m, N), *pn = ref_up(b[i++], io->psin, N);
    double *tm = ref_up(b[i++], io->thetanp1m, N), *tn = ref_up(b[i++], io->thetan, N);
    double *km = ref_up(b[i++], io->knp1m, N), *cm = ref_up(b[i++], io->cnp1m, N);
    int *wbc = ref_up(b[i++], io->wbc, WE), *ebc = ref_up(b[i++], io->ebc, WE);
    int *sbc = ref_up(b[i++], io->sbc, SN), *nbc = ref_up(b[i++], io->nbc, SN);
    int *tbc = ref_up(b[i++], io->tbc, Cc), *bbc = ref_up(b[i++], io->bbc, Cc);
    double *pw = ref_up(b[i++], io->psi_w, WE), *pe = ref_up(b[i++], io->psi_e, WE);
    double *pss = ref_up(b[i++], io->psi_s, SN), *pnn = ref_up(b[i++], io->psi_n, SN);
    double *pt = ref_up(b[i++], io->psi_t, Cc), *pb = ref_up(b[i++], io->psi_b, Cc);
    double *qw = ref_up(b[i++], io->qw, WE), *qe = ref_up(b[i++], io->qe, WE);
    double *qs = ref_up(b[i++], io->qs, SN), *qn = ref_up(b[i++], io->qn, SN);
    double *qt = ref_up(b[i++], io->qt, Cc), *qb = ref_up<double>(b[i++], io->qb, Cc);
    double *tr = ref_up(b[i++], io->tr, Cc);
    int *pm2 = ref_up(b[i++], io->procmap, Cc);
    double *root = ref_up(b[i++], io->root, (size_t)io->nproc * io->nz);
    SetUpLinearSystemsSubsurface<<<(unsigned)(N / 64), 64>>>(
        a3d, rhs, pm, pn, tm, tn, km, cm, wbc, ebc, sbc, nbc, tbc, bbc, pw, pe, pss, pnn, pt, pb, qw, qe, qs, qn,
        qt, qb, tr, pm2, root, make_int3(io->nx, io->ny, io->nz));
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    int rc = ref_down_ptr(io->a3d, a3d, 7 * N);
    rc |= ref_down_ptr(io->rhs, rhs, N);
    rc |= ref_down_ptr(io->qb, qb, Cc);
    return rc;
}

extern "C" int ref_k_infiltration(const dhara_params *p, const oracle_top_io *io) {
    REF_SET_CONSTANTS(p);
    const size_t Cc = (size_t)io->nx * io->ny;
    RefBuf b[8];
    double *pm = ref_up(b[0], io->psinp1mp1, Cc), *km = ref_up(b[1], io->knp1m, Cc);
    double *qt = ref_up(b[2], (const double *)io->topqflux, Cc), *qss = ref_up<double>(b[3], nullptr, Cc);
    double *pt = ref_up(b[4], io->psi_top, Cc), *ph = ref_up<double>(b[5], nullptr, Cc);
    int *tb = ref_up(b[6], (const int *)io->topbc, Cc);
    double *hp = ref_up(b[7], (const double *)io->hpoten, Cc);
    SubsurfaceEstimateInfiltrationPonding<<<(unsigned)((Cc + 127) / 128), 128>>>(
        pm, km, qt, qss, pt, ph, tb, hp, make_int3(io->nx, io->ny, 1));
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    ref_down(io->qss, b[3], Cc);
    ref_down(io->ph_out, b[5], Cc);
    return 0;
}

extern "C" int ref_k_water_flux(const dhara_params *p, const oracle_flux_io *io) {
    REF_SET_CONSTANTS(p);
    const size_t N = (size_t)io->nx * io->ny * io->nz, Cc = (size_t)io->nx * io->ny;
    const size_t WE = (size_t)io->nz * io->ny, SN = (size_t)io->nz * io->nx;
    RefBuf b[40];
    int i = 0;
    double *km = ref_up(b[i++], io->knp1m, N), *pp = ref_up(b[i++], io->psinp1mp1, N);
    double *pn = ref_up(b[i++], io->psin, N), *tp = ref_up(b[i++], io->thetanp1mp1, N);
    double *tn = ref_up(b[i++], io->thetan, N);
    double *es = ref_up(b[i++], io->E_soil, Cc), *TR = ref_up(b[i++], io->TR, Cc), *qss = ref_up(b[i++], io->qss, Cc);
    double *qw = ref_up(b[i++], io->bcqw, WE), *qe = ref_up(b[i++], io->bcqe, WE);
    double *qs = ref_up(b[i++], io->bcqs, SN), *qn = ref_up(b[i++], io->bcqn, SN);
    double *qt = ref_up(b[i++], io->bcqt, Cc), *qb = ref_up(b[i++], io->bcqb, Cc);
    const int o0 = i;
    double *out[10];
    for (int q = 0; q < 10; ++q) out[q] = ref_up<double>(b[i++], nullptr, N);
    int *wbc = ref_up(b[i++], io->wbc, WE), *ebc = ref_up(b[i++], io->ebc, WE);
    int *sbc = ref_up(b[i++], io->sbc, SN), *nbc = ref_up(b[i++], io->nbc, SN);
    int *tbc = ref_up(b[i++], io->tbc, Cc), *bbc = ref_up(b[i++], io->bbc, Cc);
    int *pm = ref_up(b[i++], io->procmap, Cc);
    double *root = ref_up(b[i++], io->root, (size_t)io->nproc * io->nz);
    WaterFluxEstimate<<<(unsigned)((N + 127) / 128), 128>>>(
        km, pp, pn, tp, tn, es, TR, qss, qw, qe, qs, qn, qt, qb, out[0], out[1], out[2], out[3], out[4], out[5],
        out[6], out[7], out[8], out[9], wbc, ebc, sbc, nbc, tbc, bbc, pm, root, make_int3(io->nx, io->ny, io->nz));
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    double *dst[10] = {io->quflux, io->qdflux, io->qwflux, io->qeflux, io->qsflux,
                       io->qnflux, io->dtheta, io->transp, io->evapo,  io->ssflux};
    for (int q = 0; q < 10; ++q) ref_down(dst[q], b[o0 + q], N);
    return 0;
}
