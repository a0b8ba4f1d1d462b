// Launchers of the reference's own overland.cu kernels, compiled from its
// source (src/overland.cu) -- TEST INFRASTRUCTURE for pinning the oracle.
#include "src/overland.cu"

#include "../../include/dhara_gpu.h"
#include "../kernel_io.h"
#include "launch_util.h"

// UpdateKOverland and SetUpLinearSystemsOverland call __syncthreads() inside
// their loops.  UpdateKOverland runs as one block of nx threads, so every
// thread walks all ny rows; SetUpLinearSystemsOverland runs one thread per
// column in 32-thread blocks.  Either way every thread of a block executes the
// barrier the same number of times.
extern "C" int ref_k_overland_setup(const dhara_params *p, const oracle_olf_io *io) {
    REF_SET_CONSTANTS(p);
    const size_t Cc = (size_t)io->nx * io->ny;
    if (io->nx > 1024 || Cc % 32 != 0) return 2;
    RefBuf b[10];
    double *h = ref_up(b[0], io->waterdepth, Cc), *z = ref_up(b[1], io->ztopo, Cc), *m = ref_up(b[2], io->mann, Cc);
    double *H = ref_up<double>(b[3], nullptr, Cc);
    double *kw = ref_up<double>(b[4], nullptr, Cc), *ke = ref_up<double>(b[5], nullptr, Cc);
    double *ks = ref_up<double>(b[6], nullptr, Cc), *kn = ref_up<double>(b[7], nullptr, Cc);
    double *a2d = ref_up<double>(b[8], nullptr, 5 * Cc), *rhs = ref_up<double>(b[9], nullptr, Cc);
    const int3 gs = make_int3(io->nx, io->ny, 1);
    WaterElevationOverland<<<(unsigned)((Cc + 127) / 128), 128>>>(H, h, z, (int)Cc);
    UpdateKOverland<<<1, io->nx>>>(H, h, m, kw, ke, ks, kn, gs);
    SetUpLinearSystemsOverland<<<(unsigned)(Cc / 32), 32>>>(a2d, rhs, H, z, kw, ke, ks, kn, 0., 0., 0., gs);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    ref_down(io->waterelev, b[3], Cc);
    ref_down(io->kw, b[4], Cc);
    ref_down(io->ke, b[5], Cc);
    ref_down(io->ks, b[6], Cc);
    ref_down(io->kn, b[7], Cc);
    ref_down(io->a2d, b[8], 5 * Cc);
    ref_down(io->rhs2d, b[9], Cc);
    return 0;
}

extern "C" int ref_k_water_depth(const dhara_params *p, const oracle_olf_io *io) {
    REF_SET_CONSTANTS(p);
    const size_t Cc = (size_t)io->nx * io->ny;
    RefBuf b[3];
    double *H = ref_up(b[0], (const double *)io->waterelev, Cc), *hd = ref_up<double>(b[1], nullptr, Cc);
    double *z = ref_up(b[2], io->ztopo, Cc);
    WaterDepthOverland<<<(unsigned)((Cc + 127) / 128), 128>>>(H, hd, z, (int)Cc);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    ref_down(io->waterdepth_out, b[1], Cc);
    return 0;
}
