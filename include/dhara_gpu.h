/*
 * dhara_gpu.h -- C ABI of the B200 integrated surface-subsurface flow solver.
 *
 * The library advances one or more independent domains of Dhara's coupled
 * model: the 3D mixed-form Richards equation (modified Picard, van
 * Genuchten-Mualem closure, implicit 7-point finite volumes) followed by the
 * 2D diffusive-wave overland model (Manning conductances, implicit 5-point
 * system with a fixed-elevation boundary ring), coupled through ponding and
 * infiltration at the top boundary, exactly as one call of the reference's
 *
 *     SubsurfaceFlowModel(...)   src/subsurface.cu:686-847
 *     OverlandFlowModel(...)     src/overland.cu:387-419
 *
 * does per time step inside RunCoupledFlowModel (src/device.cu:374-475).
 *
 * Array layouts are the reference's (include/class.h:99-217,
 * src/numerical.cc:38-192):
 *   3D cell   (i,j,k) -> k*nx*ny + j*nx + i, k = 0 is the TOP soil layer
 *   2D column (i,j)   -> j*nx + i
 *   W/E faces [nz*ny] at k*ny + j, S/N faces [nz*nx] at k*nx + i,
 *   top/bottom faces [ny*nx] at j*nx + i            (src/subsurface.cu:139-142)
 * Units are SI: metres, seconds, alpha in 1/m (the reference works in cm
 * internally and converts, src/global.cu:79-97).
 *
 * Every entry point returns a dhara_status; nothing calls exit() or abort().
 * A handle is used by one host thread at a time; all device work of a handle
 * runs on the handle's own CUDA stream.
 */
#ifndef DHARA_GPU_H
#define DHARA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DHARA_ABI_VERSION 1

typedef enum {
    DHARA_OK = 0,
    DHARA_ERR_INVALID = 1,      /* bad argument, size or field */
    DHARA_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    DHARA_ERR_NOMEM = 3,        /* device or host allocation failed */
    DHARA_ERR_UNSUPPORTED = 4,  /* valid input this build does not handle */
    DHARA_ERR_NONFINITE = 5,    /* NaN/Inf detected in the state */
    DHARA_ERR_TIMEOUT = 6,      /* a bounded device-side wait ran out */
    DHARA_ERR_STATE = 7         /* call out of order (e.g. step before upload) */
} dhara_status;

typedef enum { DHARA_FP64 = 0, DHARA_MIXED = 1 } dhara_precision;

/* Picard stopping rule.  The reference's rule is relative
 * max|(psi^{m+1}-psi^m)/psi^{m+1}| (PICARD_METHOD=0) or the same on theta
 * (PICARD_METHOD=1), src/subsurface.cu:432-446,762-789. */
typedef enum {
    DHARA_PICARD_PSI_RELATIVE = 0,
    DHARA_PICARD_THETA_RELATIVE = 1,
    DHARA_PICARD_PSI_ABSOLUTE = 2
} dhara_picard_rule;

/* What becomes theta^n for the next step.  The reference copies thetanp1m,
 * i.e. theta evaluated at the input of the last Picard iteration
 * (src/subsurface.cu:839-840). */
typedef enum {
    DHARA_THETA_REFERENCE = 0,   /* theta(psi^m), as the reference */
    DHARA_THETA_FINAL = 1,       /* theta(psi^{m+1}) */
    DHARA_THETA_CONSERVATIVE = 2 /* theta^m + C^m (psi^{m+1} - psi^m): closes the discrete balance */
} dhara_theta_update;

/* Per-domain parameters.  Field names follow the reference's config keys
 * (src/io.cc:236-274) and __constant__ set (include/devconst.h:6-31). */
typedef struct {
    int32_t struct_size;        /* = sizeof(dhara_params) */
    int32_t nx, ny, nz;
    double dx, dy, dz, dt;      /* m, m, m, s */
    /* van Genuchten-Mualem, scalars (per-cell alpha/n may be uploaded) */
    double alpha;               /* 1/m */
    double n;                   /* pore-size distribution (PORE_SIZE_DISTRIBUTION) */
    double theta_s, theta_r, porosity, Ss;
    double airdry, psimin;      /* carried for completeness (unused by the path) */
    double am;                  /* Picard relaxation psi^m <- am psi^m + (1-am) psi^{m+1}, 0 <= am < 1 */
    /* overland (DELTA, WATERDEPTH_MINIMUM, WATERDEPTH_CRITICAL, KZERO) */
    double delta, hmin, hcri, K0;
    /* converts E_soil / TR rates into metres per step (sec_p_mm2dt_p_m) */
    double sec_p_mm2dt_p_m;
    /* Picard */
    int32_t picard_maxiter;
    int32_t picard_rule;        /* dhara_picard_rule */
    double picard_tol;
    /* 3D linear solve: stop when ||b - A x||_2 <= tol * ||b||_2 or maxiter */
    int32_t krylov_maxiter;
    int32_t theta_update;       /* dhara_theta_update */
    double krylov_tol;
    /* 2D overland linear solve */
    int32_t overland_maxiter;
    int32_t precision;          /* dhara_precision */
    double overland_tol;
    /* mixed precision: inner FP32 solve reduces the FP64 residual by this factor */
    double inner_tol;
    int32_t inner_maxiter;
    /* mixed precision: 0 evaluates the van Genuchten closure in FP64 and the
     * FP64 refinement residual uses FP64 coefficients (the converged head is
     * the FP64 system's); 1 evaluates the closure in FP32 (faster; the
     * refinement then converges to the FP32-coefficient system). */
    int32_t closure_fp32;
    /* Decisions to fold into dhara_diagnostics.branch_signature, a bit mask:
     * 1 top-flux selection, 2 ponding clip, 4 Manning's wet/slope test,
     * 8 overland depth clip, 16 saturation (psi >= 0) of every cell at every
     * closure evaluation, 32 Picard iteration count, 64 overland CG iteration
     * count (a solve that stops at a different iteration is a different
     * map); 0 (the default) records nothing.  Each recorded decision costs a hash and a warp-aggregated
     * atomic.  Saturation is not a switch of the loss (theta and K are
     * continuous there) but of the closure's formula. */
    int32_t record_branches;
    /* Overland linear solver (the same system and stopping rule either way):
     * 0 (the default) conjugate gradients preconditioned by a geometric
     * multigrid V-cycle (Galerkin coarse operators, weighted-Jacobi
     * smoothing), which converges in tens of iterations where ponded cells
     * make the system stiff; 1 pipelined point-Jacobi-preconditioned CG (one
     * grid barrier per iteration, thousands of iterations on stiff systems).
     * Every domain of a handle uses the same solver. */
    int32_t overland_solver;
    /* Time-step halving when the Picard iteration fails to converge (not the
     * reference's scheme, which accepts a non-converged step; 0, the default,
     * keeps it).  With k > 0 a step whose Picard iteration ends at its cap is
     * undone and retried as two steps of dt/2, each of which may halve again,
     * down to dt/2^k, whose last attempt is accepted whatever its Picard
     * outcome.  Rain of a step is spread over its sub-steps in proportion to
     * their length.  Decided per domain: in a batch only the domains that fail
     * take sub-steps (the others are left at the end of their step).  Steps
     * run eagerly (no CUDA graph), with one host synchronisation per round of
     * attempts; layer statistics are not available in this mode. */
    int32_t dt_halvings;
    int32_t reserved_i[3];
    double reserved_d[8];
} dhara_params;

/* Fills p with the reference's device defaults (include/devconst.h) converted
 * to SI with the given grid; dt in seconds. */
void dhara_default_params(dhara_params *p, int nx, int ny, int nz,
                          double dx, double dy, double dz, double dt);

/* Data fields for upload/download.  Sizes: N = nx*ny*nz cells, C = nx*ny
 * columns, FWE = nz*ny, FSN = nz*nx. */
typedef enum {
    /* 3D, double, N */
    DHARA_F_PSI = 0,        /* psin: pressure head of the current state, m */
    DHARA_F_THETA = 1,      /* thetan: moisture of the current state */
    DHARA_F_KSAT = 2,       /* ksat, m/s */
    DHARA_F_ALPHA = 3,      /* optional per-cell alpha, 1/m */
    DHARA_F_NVG = 4,        /* optional per-cell n */
    DHARA_F_K = 5,          /* knp1m: K at the last evaluation (download) */
    DHARA_F_C = 6,          /* cnp1m (download) */
    DHARA_F_THETA_NEW = 7,  /* thetanp1mp1: theta(psi^{m+1}) of the last step (download) */
    /* 2D, double, C */
    DHARA_F_ZTOPO = 16,
    DHARA_F_MANN = 17,
    DHARA_F_WATERDEPTH = 18,/* overland h */
    DHARA_F_WATERELEV = 19, /* overland H = h + z */
    DHARA_F_PONDING = 20,   /* ph */
    DHARA_F_PPT = 21,       /* ppt_ground, mm per step */
    DHARA_F_ESOIL = 22,     /* E_soil */
    DHARA_F_TR = 23,        /* TR */
    DHARA_F_HPOTEN = 24,    /* (download) */
    DHARA_F_QTOP = 25,      /* bcqt: top flux of the last step (download) */
    /* boundary values, double */
    DHARA_F_BCQW = 32, DHARA_F_BCQE = 33,   /* FWE */
    DHARA_F_BCQS = 34, DHARA_F_BCQN = 35,   /* FSN */
    DHARA_F_BCQB = 36,                       /* C (overwritten by free drainage) */
    DHARA_F_BCPSIW = 40, DHARA_F_BCPSIE = 41, DHARA_F_BCPSIS = 42, DHARA_F_BCPSIN = 43,
    DHARA_F_BCPSIB = 44,
    /* int32 fields */
    DHARA_FI_BCW = 64, DHARA_FI_BCE = 65,   /* FWE */
    DHARA_FI_BCS = 66, DHARA_FI_BCN = 67,   /* FSN */
    DHARA_FI_BCB = 68, DHARA_FI_BCT = 69,   /* C */
    DHARA_FI_PROCMAP = 70,                   /* C */
    /* root density table, double, nproc*nz (set with dhara_set_roots) */
    DHARA_F_ROOT = 80
} dhara_field;

typedef struct dhara_handle dhara_handle;

typedef struct {
    int64_t steps;                  /* time steps completed */
    int64_t picard_iters_total;     /* Picard iterations over all steps */
    int64_t krylov_iters_total;     /* inner (FP32 in mixed mode) Krylov iterations */
    int64_t refine_iters_total;     /* FP64 residual recomputes (mixed mode) */
    int64_t overland_iters_total;
    int32_t picard_iters_last;
    int32_t krylov_iters_last;      /* over all Picard iterations of the last step */
    int32_t picard_nonconverged;    /* steps that hit picard_maxiter */
    int32_t krylov_nonconverged;    /* linear solves that hit their iteration cap */
    int32_t overland_nonconverged;
    int32_t nonfinite;              /* 1 if NaN/Inf was seen */
    double mb_subsurface_last;      /* reference water balance of the last step, m (src/subsurface.cu:809-826) */
    double mb_subsurface_cum;       /* sum over steps of the above */
    double storage_change_cum;      /* sum dz*(theta^{n+1}-theta^n) + specific storage, m per column area */
    double top_inflow_cum;          /* sum dt*sum(q_top), m (column-summed) */
    double bottom_outflow_cum;      /* sum dt*sum(q_bottom), m */
    double rain_cum;                /* sum over columns of rain per step, m */
    double overland_boundary_out_cum;   /* water leaving through the fixed ring, m */
    double overland_clip_cum;       /* water created by h = max(H-z,0), m */
    double ponded_volume;           /* sum h over columns after the last step, m */
    double picard_err_last;         /* last Picard difference measure */
    double krylov_relres_last;      /* last ||r||/||b|| of the 3D solve */
    /* With record_branches: an order-independent 64-bit hash-sum over every
     * discrete decision of the run -- the top-flux selection per column and
     * step (src/global.cu:236-251), the ponding clip (src/subsurface.cu:480),
     * saturation (psi >= 0) of every cell at every closure evaluation
     * (src/global.cu:79-97), Manning's wet/slope test per face
     * (src/overland.cu:279-297), the overland depth clip
     * (src/overland.cu:378) and the Picard iteration count.  Each comparison
     * is recorded as below / on / above its boundary, "on" meaning within a
     * rounding band (1e-9 relative, or 1e-9 m / 1e-9 for depths, heads and
     * slopes), so a comparison that ties up to rounding records the same in
     * every run.  Two runs with equal signatures took the same branches
     * everywhere, so a finite difference between them differentiates one
     * smooth piece.  0 when not recorded. */
    uint64_t branch_signature;
    /* accepted steps and sub-steps (dt_halvings), and all attempts including
     * the undone ones; equal to steps when no step was halved */
    int64_t substeps_total;
    int64_t step_attempts_total;
    double reserved[3];
} dhara_diagnostics;

/* ---- lifetime ---------------------------------------------------------- */

/* Creates a handle for ndomains independent domains, params[d] each.  All
 * domains must share one precision and the same Picard/Krylov caps.  The
 * handle owns all device memory.  device < 0 uses the current device. */
int dhara_create(const dhara_params *params, int ndomains, int device, dhara_handle **out);
int dhara_destroy(dhara_handle *h);

/* The parameters domain `domain` of the handle was created with. */
int dhara_get_params(dhara_handle *h, int domain, dhara_params *out);

/* Message of the last failing call on this thread (never NULL). */
const char *dhara_last_error(void);
int dhara_abi_version(void);

/* ---- data in / out (host buffers; copies complete before return) ------ */

int dhara_upload(dhara_handle *h, int domain, int field, const double *src, int64_t count);
int dhara_upload_int(dhara_handle *h, int domain, int field, const int32_t *src, int64_t count);
int dhara_download(dhara_handle *h, int domain, int field, double *dst, int64_t count);
/* The same with device pointers (caller-owned device arrays, reference
 * layout); ordered on the handle's stream and complete on return. */
int dhara_upload_device(dhara_handle *h, int domain, int field, const double *dsrc, int64_t count);
int dhara_download_device(dhara_handle *h, int domain, int field, double *ddst, int64_t count);
/* Root density table rda[proc*nz + k] (src/subsurface.cu:115). */
int dhara_set_roots(dhara_handle *h, int domain, const double *rda, int nproc);
/* Optional per-step rain for graph-replayed runs: mm per step, uniform over
 * the domain, used instead of the PPT field for steps [0, nsteps). */
int dhara_set_rain_schedule(dhara_handle *h, int domain, const double *mm_per_step, int nsteps);

/* ---- the hot path -------------------------------------------------------- */

/* CopyDataToDevice's theta->psi conversion, vanGenuchtenInverse
 * (src/device.cu:327, src/global.cu:32-52): psi := psi(theta) for every domain. */
int dhara_psi_from_theta(dhara_handle *h);

/* PreRunningFlowModel (src/global.cu:270-296): evaluates theta, K, C at psi
 * and resets per-step state.  Must follow the uploads, precede stepping. */
int dhara_prepare(dhara_handle *h);

/* One reference SubsurfaceFlowModel call for every domain (no host sync). */
int dhara_subsurface_step(dhara_handle *h);
/* One reference OverlandFlowModel call for every domain (no host sync). */
int dhara_overland_step(dhara_handle *h);
/* nsteps x (subsurface step + overland step).  use_graph != 0 captures one
 * step into a CUDA graph on first use and replays it. */
int dhara_step(dhara_handle *h, int nsteps, int use_graph);

int dhara_synchronize(dhara_handle *h);
int dhara_get_diagnostics(dhara_handle *h, int domain, dhara_diagnostics *out);
/* The cudaStream_t of the handle, for callers that time or order work. */
int dhara_get_stream(dhara_handle *h, void **stream);

/* Per-kernel CUDA-event timing (off by default).  kernel: 0 = 3D Krylov solve,
 * 1 = Picard assembly, 2 = Picard check, 3 = step epilogue, 4 = overland solve,
 * 5 = overland set-up/finish, 6 = step prologue, 7 = the adjoint's own kernels
 * (its linear solves count under 0 and 4), 8 = the fused subsurface step
 * (dhara_launch_config.fused_step: kernels 0-3 and 6 run inside it). */
int dhara_set_kernel_timing(dhara_handle *h, int enable);
int dhara_get_kernel_timing(dhara_handle *h, int kernel, int64_t *launches, double *total_ms);
int dhara_reset_kernel_timing(dhara_handle *h);
/* Kernel launches this handle has issued (graph replays count their nodes). */
int dhara_get_launch_count(dhara_handle *h, int64_t *count);
/* Algorithmic HBM bytes moved by the 3D Krylov kernel so far (the count the
 * roofline figure divides by time), and the inner iterations they cover. */
int dhara_get_krylov_traffic(dhara_handle *h, double *bytes, int64_t *iterations);

/* ---- block schedules ---------------------------------------------------------
 * The persistent solvers' block schedules and the 3D kernels' tile shape: the
 * column tiles every 3D kernel works on (32 x 4 or 16 x 8 columns of 128
 * threads, per domain or for all), how many co-resident blocks per SM the 3D
 * Krylov solve launches (its tiles are strided over them), and whether the
 * overland solve keeps each segment's vectors in shared memory (one block per
 * segment, when they fit) or streams them with a given number of blocks per
 * SM.  dhara_autotune times the candidates on this handle's own data --
 * trial_steps steps per candidate from the current state, which it restores
 * afterwards -- and keeps the fastest; *chosen (may be NULL) receives the
 * result.  Defaults: tiles per domain, the most blocks per SM that fit,
 * overland resident when possible.  Results agree across schedules to
 * rounding (reductions run over tiles in a fixed order; a different tile
 * shape groups the sums differently), and bit for bit across block counts. */
typedef struct {
    int32_t krylov_blocks_per_sm;
    int32_t overland_resident;
    int32_t overland_blocks_per_sm;
    /* column tiles of the 3D kernels: 1 = 32 x 4 for every domain, 2 = 16 x 8,
     * 0 = per domain whichever needs fewer tiles (fewer idle threads in the
     * ragged tiles of narrow domains; 32 x 4 on a tie) -- the default */
    int32_t tile_shape;
    double krylov_ms;     /* per trial step of the chosen schedule (autotune only) */
    double overland_ms;
    /* 1: each subsurface step is one persistent launch (prologue, every Picard
     * iteration's assembly, solve and check, epilogue) -- the default where
     * that kernel runs as many blocks per SM as the Krylov kernel; 0: a launch
     * per kernel (per-kernel timing then names every phase).  Results are the
     * same bit for bit. */
    int32_t fused_step;
    int32_t pad;
} dhara_launch_config;

int dhara_autotune(dhara_handle *h, int trial_steps, dhara_launch_config *chosen);
int dhara_get_launch_config(dhara_handle *h, dhara_launch_config *out);
int dhara_set_launch_config(dhara_handle *h, const dhara_launch_config *cfg);

/* ---- output ----------------------------------------------------------------
 * The reference's outputs (SaveModelResults, src/io.cc:854-915, and
 * SaveResultEntirePeriod, src/io.cc:962-996) without its blocking per-step
 * copies (src/subsurface.cu:842-846).
 *
 * Statistics: after every step the layer sums of the new head and of
 * theta(new head) over all cells of the layer but its last (the reference's
 * CopyLayers range, src/device.cu:135-147; written as pressure_mean and
 * moisture_mean) and the step's water balance (mb_subsurfaceW) are kept on
 * the device for up to max_steps steps per domain (counted by the domain's
 * step counter).  dhara_get_statistics copies them out: mb_subsurfaceW[t],
 * pressure_sum[t*nz + k], moisture_sum[t*nz + k] for t < *nsteps; any output
 * pointer may be NULL. */
int dhara_enable_statistics(dhara_handle *h, int max_steps);
int dhara_get_statistics(dhara_handle *h, int domain, int64_t *nsteps, double *mb_subsurfaceW,
                         double *pressure_sum, double *moisture_sum);

/* Snapshot of one domain's state (water_elevation, water_depth: nx*ny;
 * pressure_head, moisture: nx*ny*nz in the reference layout; any may be NULL):
 * queued on the handle's stream as a device copy into one of two staging
 * slots, then copied to the host buffers on a second stream, so the steps
 * queued after it run while the copy drains (pin the host buffers for that
 * overlap).  The buffers hold the snapshot once dhara_snapshot_wait returns;
 * with two sets of buffers a caller can snapshot every step. */
int dhara_snapshot(dhara_handle *h, int domain, double *water_elevation, double *water_depth,
                   double *pressure_head, double *moisture);
int dhara_snapshot_wait(dhara_handle *h);

/* ---- NetCDF result files -----------------------------------------------------
 * The reference's output files (SaveModelResults, src/io.cc:854-906, and the
 * flow-model part of SaveResultEntirePeriod, src/io.cc:962-996, through its
 * SaveOutput1D/2D/3D, src/io.cc:696-850) in NetCDF classic format, written by
 * the library (no netCDF library needed); 64-bit-offset format when a file
 * exceeds 2 GiB.  Variables and dimensions as the reference defines them:
 *   file2d: water_elevation, water_depth   [ny][nx], dimensions named "x", "y"
 *           (SaveOutput2D's names: "x" is the slower dimension)
 *   file3d: pressure_head, moisture        [nz][ny][nx], dimensions "z", "y", "x"
 *   file1d: mb_subsurfaceW                 [nsteps], dimension "time_series"
 *   file_stat: pressure_mean, moisture_mean [nsteps][nz], dimensions "x", "y"
 *           (CopyLayers' per-layer sums, src/device.cu:135-147)
 * Any file argument may be NULL (not written).  The writers take host
 * arrays in the reference layout; the dhara_save_* forms take them from a
 * handle (the current state, and the statistics of dhara_enable_statistics). */
int dhara_write_netcdf_state(const char *file2d, const char *file3d, int nx, int ny, int nz,
                             const double *water_elevation, const double *water_depth,
                             const double *pressure_head, const double *moisture);
int dhara_write_netcdf_statistics(const char *file1d, const char *file_stat, int nsteps, int nz,
                                  const double *mb_subsurfaceW, const double *pressure_sum,
                                  const double *moisture_sum);
int dhara_save_netcdf_state(dhara_handle *h, int domain, const char *file2d, const char *file3d);
int dhara_save_netcdf_statistics(dhara_handle *h, int domain, const char *file1d, const char *file_stat);

/* ---- checkpoint and restart -------------------------------------------------
 * The reference has no restart path (it runs one time loop from the initial
 * condition, src/device.cu:374-475); these save and restore the state a step
 * starts from, for every domain of the handle: psi^n, theta^n, the top
 * layer's K, the ponded depth, the overland depth and elevation, the Picard
 * control record (step counter, last iteration counts) and the cumulative
 * diagnostics.  Inputs that do not change during a run (soil and surface
 * fields, boundary conditions, rain schedule, roots) are not part of it: a
 * restart uploads them as the original run did, calls dhara_prepare, then
 * dhara_restore, and its steps then match the original handle's bit for bit.
 * The buffer is host memory the caller owns; the layout is private to this
 * library version (a header records the domain sizes, and a checkpoint from
 * a handle with other domains is rejected with DHARA_ERR_INVALID).  Both
 * calls synchronise the handle's stream and need dhara_prepare first. */
/* ---- failure detection self-check ---------------------------------------------
 * No counterpart in the reference (which exits on any CUDA error).  Every
 * device-side wait of the persistent solvers (grid barriers, TMA stage
 * waits) is bounded: past its limit the kernel raises an error flag and
 * returns, and the host reports DHARA_ERR_TIMEOUT instead of hanging.  This
 * runs one such wait on `device` that nothing can satisfy, with the given
 * limit (0 < limit_ms <= 10000), and sets *timed_out = 1 when the wait gave
 * up, flagged the error and returned and the context still worked after. */
int dhara_selftest_bounded_wait(int device, double limit_ms, int *timed_out);

int dhara_checkpoint_size(dhara_handle *h, int64_t *bytes);
int dhara_checkpoint(dhara_handle *h, void *buf, int64_t bytes);
int dhara_restore(dhara_handle *h, const void *buf, int64_t bytes);

/* ---- configuration file ----------------------------------------------------
 * The reference's "KEY = value" configuration file (parsed by
 * ParserConfigFile, src/parser.cc:39-72; keys read by LoadFlowModelConfig,
 * src/io.cc:236-274, and the boundary keys of src/host.cc:93-112).  Lines
 * starting with '#' are comments; the first occurrence of a key wins; keys
 * absent from the file keep the value dhara_default_params gives.  Units are
 * the reference's: ALPHA is read in 1/cm (stored in 1/m), TIME_STEP_DATA is
 * the model time step in the reference's device time unit (hours) and sets
 * dt and sec_p_mm2dt_p_m = dt * 3600 / 1000 as include/devconst.h pairs them.
 * picard_tol is TOLERANCE_PRESSURE for PICARD_METHOD 0 and TOLERANCE_THETA
 * for PICARD_METHOD 1.  The grid size comes from the caller (the reference
 * reads it from the topography file). */
typedef struct {
    /* faces in the order top, bottom, north, south, east, west */
    int32_t type[6];     /* BOUNDARY_TYPE_*: 0 Dirichlet, 1 free flow, 2 no flow */
    double psi[6];       /* PRESSURE_HEAD_* */
    double flux[6];      /* FLUX_* */
    int32_t found;       /* number of recognised keys read from the file */
    int32_t pad;
} dhara_config_bc;

/* Fills *p (and *bc when not NULL) from the file.  As in the reference
 * (src/host.cc:101-109), PRESSURE_HEAD_BOTTOM and FLUX_BOTTOM land on the top
 * face and PRESSURE_HEAD_TOP and FLUX_TOP on the bottom face.  Returns
 * DHARA_ERR_INVALID if the file cannot be read. */
int dhara_params_from_config(const char *path, int nx, int ny, int nz, dhara_params *p, dhara_config_bc *bc);

/* Uploads the face types and values of *bc as the boundary arrays of one
 * domain (constant over each face). */
int dhara_apply_boundary_config(dhara_handle *h, int domain, const dhara_config_bc *bc);

/* ---- discrete adjoint ------------------------------------------------------
 * No counterpart in the reference.  Gradient of a soil-moisture / outflow
 * misfit with respect to per-cell log Ks, alpha (1/m) and n, by the discrete
 * adjoint of the implicit time steps with checkpointing: the forward run keeps
 * the state every checkpoint_every steps; the reverse sweep recomputes each
 * segment from its checkpoint, recording every Picard iterate, and runs the
 * adjoint kernels backwards through it (each linear solve reversed by a solve
 * with the same symmetric matrix).
 *
 *   L = sum_t sum_{k<3} sum_c (theta_{t,k,c} - theta_target_{t,k,c})^2
 *     + w_q * sum_t (Q_t - q_target_t)^2
 *
 * theta_{t,k,c}: moisture of layer k (k = 0 the top) of column c after step t;
 * Q_t: the overland flow into the fixed boundary ring during step t (depth in
 * m summed over columns).  Scope: a single-domain handle; top flux condition,
 * free-drainage bottom, no-flux sides (no Dirichlet faces); zero ET and
 * transpiration. */
typedef struct {
    int32_t struct_size;         /* sizeof(dhara_adjoint_desc) */
    int32_t nsteps;              /* time steps of the run (>= 1) */
    int32_t checkpoint_every;    /* steps per checkpoint segment (>= 1) */
    int32_t pad;
    const double *theta_target;  /* host, [nsteps][3][nx*ny] */
    const double *q_target;      /* host, [nsteps] */
    double w_q;                  /* weight of the outflow misfit */
    double reserved[4];
} dhara_adjoint_desc;

/* Runs desc->nsteps steps forward from the handle's current state (the state
 * advances exactly as with dhara_step) and returns the loss in *loss.  When
 * grad_logks, grad_alpha and grad_n are all non-NULL it also runs the reverse
 * sweep and writes dL/dlog(Ks), dL/dalpha and dL/dn per cell in the reference
 * 3D layout (nx*ny*nz values each); when they are all NULL only the loss is
 * computed. */
int dhara_adjoint(dhara_handle *h, const dhara_adjoint_desc *desc, double *loss, double *grad_logks,
                  double *grad_alpha, double *grad_n);

/* ---- allocation-free overland step ---------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they step (a host model that owns every GPU buffer and leaves
 * none spare, a loop that forbids allocation after start-up): one overland
 * step of one domain -- the computation of
 * dhara_overland_step -- on the caller's device arrays.  waterdepth is read
 * as the depth before the step and overwritten with the depth after it;
 * waterelev receives H = h + z after the solve; ztopo and mann are read.
 * Uses nx, ny, dx, dy, dt, delta, hmin, K0, overland_tol, overland_maxiter of
 * *p.  Work is queued on `stream` (a cudaStream_t; NULL = default stream).
 * All scratch is one fixed device array of DHARA_NOALLOC_MAX_COLUMNS columns
 * that every GPU loading the library keeps until exit; larger domains return
 * DHARA_ERR_UNSUPPORTED.  Calls share that array: calls whose GPU work
 * overlaps race, so order them on one stream.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress) and keeps it for the
 * life of the process; make it before any stream capture, and do not call
 * again on a device after cudaDeviceReset.  waterdepth and waterelev must not
 * overlap each other, ztopo or mann (DHARA_ERR_INVALID).  Convergence is not
 * reported: the solve stops at overland_tol or overland_maxiter and returns
 * DHARA_OK either way.  Nothing is allocated, nothing is synchronised. */
#define DHARA_NOALLOC_MAX_COLUMNS 16384
int dhara_overland_step_noalloc(const dhara_params *p, double *waterdepth, const double *ztopo,
                                const double *mann, double *waterelev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DHARA_GPU_H */
