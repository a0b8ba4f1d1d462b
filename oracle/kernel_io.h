/*
 * kernel_io.h -- argument records of the reference's per-cell kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  Each record carries the host arrays one kernel
 * of the reference reads and writes, named as in the kernel's signature.  The
 * oracle's stateless restatement of a kernel (oracle_k_*) and the launcher of
 * the reference's own kernel compiled from its sources (ref_k_*, oracle/ref/)
 * take the same record, so a test can run both on identical inputs.
 */
#ifndef DHARA_KERNEL_IO_H
#define DHARA_KERNEL_IO_H

#ifdef __cplusplus
extern "C" {
#endif

/* SetUpLinearSystemsSubsurface (src/subsurface.cu:381-386) */
typedef struct {
    int nx, ny, nz, nproc;
    const double *psinp1m, *psin, *thetanp1m, *thetan, *knp1m, *cnp1m;   /* N */
    const int *wbc, *ebc, *sbc, *nbc, *tbc, *bbc;                        /* faces */
    const double *psi_w, *psi_e, *psi_s, *psi_n, *psi_t, *psi_b;
    const double *qw, *qe, *qs, *qn, *qt;
    double *qb;                                                          /* written */
    const double *tr;                                                    /* C */
    const int *procmap;                                                  /* C */
    const double *root;                                                  /* nproc*nz */
    double *a3d, *rhs;                                                   /* 7N, N */
} oracle_asm_io;

/* WaterFluxEstimate (src/subsurface.cu:494-499) */
typedef struct {
    int nx, ny, nz, nproc;
    const double *knp1m, *psinp1mp1, *psin, *thetanp1mp1, *thetan;       /* N */
    const double *E_soil, *TR, *qss;                                     /* C */
    const double *bcqw, *bcqe, *bcqs, *bcqn, *bcqt, *bcqb;
    const int *wbc, *ebc, *sbc, *nbc, *tbc, *bbc;
    const int *procmap;
    const double *root;
    double *quflux, *qdflux, *qwflux, *qeflux, *qsflux, *qnflux;        /* N, written */
    double *dtheta, *transp, *evapo, *ssflux;                            /* N, written */
} oracle_flux_io;

/* EstimateFluxes + IdentifyTopBoundary + SubsurfaceEstimateInfiltrationPonding
 * (src/global.cu:203-288, src/subsurface.cu:465-491), all on the top layer */
typedef struct {
    int nx, ny;
    const double *ph_in, *psinp1m, *knp1m, *ppt, *et, *ksat, *thetan;   /* C (top layer) */
    const double *psinp1mp1, *psi_top;                                   /* C */
    double *hpoten, *qcapa, *topqflux, *qss, *ph_out;                    /* C, written */
    int *topbc;                                                          /* C, written */
} oracle_top_io;

/* WaterElevationOverland, UpdateKOverland, SetUpLinearSystemsOverland,
 * WaterDepthOverland (src/overland.cu:33-383) */
typedef struct {
    int nx, ny;
    const double *waterdepth, *ztopo, *mann;                             /* C */
    double *waterelev, *kw, *ke, *ks, *kn, *a2d, *rhs2d;                 /* C (a2d 5C), written */
    double *waterdepth_out;                                              /* C, from waterelev */
} oracle_olf_io;

#ifdef __cplusplus
}
#endif
#endif
