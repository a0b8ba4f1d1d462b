/*
 * dhara_oracle.h -- FP64 CPU restatement of Dhara's integrated flow hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU library is compared
 * against, and the timed CPU baseline; the product never links or calls it.
 *
 * Parity status: the reference's GPU path cannot be built here (its vendored
 * CUSP 0.5.1 does not compile against CUDA 12.9's Thrust, and the reference
 * ships no tests, fixtures or golden outputs), so this restatement is pinned
 * by (1) the reference's own kernels compiled from their sources and run on
 * the GPU (oracle/_ref, see oracle/Makefile and tests/test_ref_kernels.py) for
 * every per-cell kernel, and (2) known-answer checks (closed-form van
 * Genuchten values, theta->psi->theta round trips, converged Krylov residuals).
 * The Krylov iterations themselves (CUSP BiCGSTAB / CG) are restated from the
 * vendored CUSP sources and are unpinned by execution.
 *
 * Every function cites the reference file:line it follows.
 */
#ifndef DHARA_ORACLE_H
#define DHARA_ORACLE_H

#include "../include/dhara_gpu.h"
#include "kernel_io.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dhara_oracle dhara_oracle;

/* Linear solver used for the 3D system.  The reference runs unpreconditioned
 * CUSP BiCGSTAB (src/subsurface.cu:750-751); CG is offered for speed on the
 * symmetric all-Neumann matrix, and CG preconditioned by each column's
 * vertical tridiagonal block for long horizons (same system, same stopping
 * rule; the 2D overland system falls back to CG with it). */
enum { ORACLE_SOLVER_BICGSTAB = 0, ORACLE_SOLVER_CG = 1, ORACLE_SOLVER_PCG_COLUMN = 2 };

dhara_oracle *oracle_create(const dhara_params *p);
void oracle_destroy(dhara_oracle *o);
/* 3D and 2D solver choice (ORACLE_SOLVER_*). */
void oracle_set_solvers(dhara_oracle *o, int solver3d, int solver2d);
/* OpenMP threads used by this process (0 = leave the runtime default). */
void oracle_set_threads(int nthreads);
int oracle_get_threads(void);

int oracle_upload(dhara_oracle *o, int field, const double *src, long long count);
int oracle_upload_int(dhara_oracle *o, int field, const int *src, long long count);
int oracle_download(dhara_oracle *o, int field, double *dst, long long count);
int oracle_set_roots(dhara_oracle *o, const double *rda, int nproc);

int oracle_psi_from_theta(dhara_oracle *o);
int oracle_prepare(dhara_oracle *o);
int oracle_subsurface_step(dhara_oracle *o, const double *rain_mm_or_null);
int oracle_overland_step(dhara_oracle *o);
int oracle_get_diagnostics(dhara_oracle *o, dhara_diagnostics *out);

/* Per-cell kernels, exposed for unit parity (same argument meaning as the
 * reference kernels).  alpha_m / nvg may be NULL (scalar params used). */
void oracle_van_genuchten(const dhara_params *p, const double *psi, const double *ksat,
                          const double *alpha_m, const double *nvg, long long N,
                          double *C, double *theta, double *K);
void oracle_van_genuchten_inverse(const dhara_params *p, const double *theta,
                                  const double *alpha_m, const double *nvg, long long N,
                                  double *psi);
/* The assembled reference DIA system of the current Picard state:
 * a3d[7*N] (column-major, pitch N) and rhs[N] (src/subsurface.cu:381-429). */
int oracle_assemble(dhara_oracle *o, double *a3d, double *rhs);
/* Overland conductances ke, kw, kn, ks [C] each from H, h, mann
 * (src/overland.cu:193-368). */
void oracle_update_k_overland(const dhara_params *p, const double *H, const double *h,
                              const double *mann, double *kw, double *ke, double *ks,
                              double *kn);

/* Stateless restatements of the reference kernels, one per kernel, on the
 * records of kernel_io.h.  The oracle's time stepping runs through these. */
void oracle_k_assemble(const dhara_params *p, const oracle_asm_io *io);
void oracle_k_estimate_fluxes(const dhara_params *p, const oracle_top_io *io);
void oracle_k_identify_top(const dhara_params *p, const oracle_top_io *io);
void oracle_k_infiltration(const dhara_params *p, const oracle_top_io *io);
void oracle_k_water_flux(const dhara_params *p, const oracle_flux_io *io);
void oracle_k_overland_setup(const dhara_params *p, const oracle_olf_io *io);
void oracle_k_water_depth(const dhara_params *p, const oracle_olf_io *io);

#ifdef __cplusplus
}
#endif
#endif
