// internal.h -- shared host/device definitions of the B200 flow solver.
//
// Data model: all domains of a handle are concatenated in struct-of-arrays
// device buffers in the reference layout (k-major, k = 0 top).  Work is
// organised in COLUMN TILES of TILE_X x TILE_Y columns; a CUDA block owns one
// tile at a time and each thread marches down one (i, j) column, so the
// z-neighbours of the 7-point stencil stay in registers and the x/y
// neighbours are coalesced loads along the same k-plane.
#pragma once

#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/dhara_gpu.h"

// Default tile shape; a domain may use 16 x 8 instead (DomainDesc::tx, ty:
// tx * ty = TILE_THREADS always, tx a power of two)
#define TILE_X 32
#define TILE_Y 4
#define TILE_THREADS (TILE_X * TILE_Y)
#define NZ_MAX 64
// planes per TMA-staged chunk: inner sweep (by inner precision) and the FP64
// residual (compile-time; -D overrides them for timing alternatives)
#ifndef CHUNK_F32
#define CHUNK_F32 2
#endif
#ifndef CHUNK_F64
#define CHUNK_F64 2
#endif
#ifndef CH_R
#define CH_R 2
#endif
// TMA staging buffers per block (chunks in flight ahead of the one being computed: STAGES - 1)
#ifndef STAGES
#define STAGES 2
#endif
// storage of the column preconditioner's factors 1/den and c': narrower than
// the inner precision (bf16 in mixed mode, FP32 in FP64 mode) when set
#ifndef FACTOR_NARROW_F32
#define FACTOR_NARROW_F32 0
#endif
#ifndef FACTOR_NARROW_F64
#define FACTOR_NARROW_F64 1
#endif
// bytes of one stored factor
#define FACTOR_BYTES(mixed) ((mixed) ? (FACTOR_NARROW_F32 ? 2 : 4) : (FACTOR_NARROW_F64 ? 4 : 8))
// inner sweep: chunks prefetched into L2 beyond the staged ones (0: none).
// Measured per FP32 / FP64 inner iteration on the 512x512x40 storm: 0 chunks
// 0.1681 / 0.2595 ms, 1 chunk 0.1644 / 0.2548, 2 chunks 0.1664 / 0.2609,
// 4 chunks 0.1749 / 0.2868 (prefetching further evicts the neighbour tiles'
// halo planes from L2 before they are read).
#ifndef PF_DIST
#define PF_DIST 1
#endif
// Krylov kernel: blocks per SM it is compiled for (register budget), and
// whether the FP32 column solve keeps its forward-sweep values d' in shared
// memory (1) or in the t array it then overwrites (0)
#ifndef KRYLOV_BLOCKS_F32
#define KRYLOV_BLOCKS_F32 7
#endif
#ifndef KRYLOV_BLOCKS_F64
#define KRYLOV_BLOCKS_F64 4
#endif
#ifndef KRYLOV_DSMEM_F32
#define KRYLOV_DSMEM_F32 0
#endif

// Tensor maps of one domain (index = dom * NMAP + id): halo boxes
// (TILE_X + 32 bytes) x (TILE_Y + 2) x chunk, own boxes TILE_X x TILE_Y x chunk.
// The inner iteration's vectors z, t = M^-1 A p and p are double buffered
// (the sweep reads the previous iteration's at the halo and writes the new
// one's at its own columns).
enum {
    MAP_P0_H = 0, MAP_P1_H, MAP_Z0_H, MAP_Z1_H, MAP_T0_H, MAP_T1_H, MAP_K_H,  // inner precision, halo
    MAP_D_O, MAP_DD_O, MAP_INV_O, MAP_C_O,                                    // inner precision, own
    MAP_X64_H, MAP_K64_H, MAP_D64_O, MAP_B_O,                                 // FP64 outer residual
    NMAP
};

// Per-domain constants (device copy in DevPtrs::dom).  3D arrays are stored
// k-major like the reference, with the row pitch nxp = nx rounded up to a
// multiple of 4 and every domain's base 128-byte aligned, so rows and planes
// start on 16-byte boundaries (the TMA stride rule); columns i >= nx are
// padding that no kernel reads as data.
struct DomainDesc {
    int nx, ny, nz, has_alpha;
    int has_n, picard_rule, theta_update, picard_maxiter;
    int krylov_maxiter, inner_maxiter, overland_maxiter, sched_len;
    int tile_begin, tile_end, closure_fp32, nxp;  // nxp: row pitch of 3D arrays (nx rounded up to 4)
    int closure_fast, has_dirichlet;              // reformulated FP64 closure (mixed mode); any type-0 face
    int record_branches, tx, ty, tx_log2;         // accumulate DevDiag::branch_sig; tile shape
    long long off3, off2, offWE, offSN, sched_off;
    double dx, dy, dz, dt;
    double alpha, n, theta_s, theta_r, porosity, Ss, am;
    double delta, hmin, K0, sec;
    double picard_tol, krylov_tol, inner_tol, overland_tol;
    // time-step halving (dt_halvings): dt above is the length of the step
    // being attempted; sub_frac its share of the full step (the rain of a
    // step is spread in proportion), step_advance 0 while sub-stepping (the
    // host advances the step counter once the full step is done), frozen 1
    // for a domain that has finished the step while others still sub-step
    // (its Picard iteration and overland solve are skipped; the host restores
    // its state after the round)
    double sub_frac;
    int step_advance, frozen;
};

struct TileDesc {
    int dom, x0, y0, pad;
};

// Per-domain solver control, written by exactly one block at a time (the last
// block to finish a reduction for that domain) and read by all blocks after a
// grid barrier.
struct KrylovCtrl {
    double bb;          // ||b||^2 of the 3D system
    double rr64;        // ||b - A x||^2 at the last outer check
    double rz;          // preconditioned residual norm r.M^-1 r after the last inner iteration
    double alpha, beta; // step of the last inner iteration (its x update is pending) and the next beta
    double inner_target2;  // the inner solve stops when rz falls to this
    double rho_last;    // z.M z of the last inner iteration (the rho its direction p was formed with)
    int active;         // outer solve still running
    int inner_active;   // inner PCG running
    int inner_iter;     // inner iterations in the current cycle
    int total_iter;     // inner iterations this solve
    int cycles;         // outer residual recomputes this solve
    int parity;         // which z/t/p buffers hold the last iteration's vectors
    int first_inner;    // next sweep is a cycle's first: z from phase R, no pending update
    int keep_p;         // ... and it continues the previous cycle's direction p (beta != 0)
};

struct PicardCtrl {
    int iter;           // Picard iterations done this step
    int done;           // converged or capped
    int converged;
    int step;           // steps done (indexes the rain schedule)
    double err;
};

struct OverlandCtrl {
    double bb, rr;  // ||b||^2 and the final ||r||^2 of the domain's last solve
    int iter, pad;  // its iteration count
};

// The overland solve works on segments: up to OLF_SEG consecutive surface
// cells of one domain, one segment per block at a time, OLF_CPT cells per
// thread.  A domain's segments are consecutive in the segment list.
#define OLF_SEG 1024
#define OLF_THREADS 256
#define OLF_CPT (OLF_SEG / OLF_THREADS)
// per-cell vectors kept in shared memory when every segment has its own block
enum { OV_X, OV_R, OV_W, OV_Z, OV_S, OV_P, OV_M, OV_CW, OV_CE, OV_CS, OV_CN, OV_DG, OV_N };

struct OlfSeg {
    long long begin;  // global surface index of the first cell
    int dom;
    int l0;           // index of the first cell within its domain
    int count;        // cells in the segment
    int first;        // index of the domain's first segment
    int nseg;         // segments of the domain
    int pad;
};

// Scalars of the pipelined CG recurrence for one segment.  Every segment of a
// domain computes the same values from the same domain sums.
struct OlfSegState {
    double gamma_prev, alpha_prev, bb;
    int iter, active;
};

// Multigrid hierarchy of the overland solve (overland_mg.cu).  Level 0 is a
// domain's interior surface grid (the fixed ring eliminated); each coarser
// level halves every dimension that still has at least 3 points, vertex-
// centred (coarse point I sits on fine point 2I+1), until a level has at most
// MG_DENSE_PTS points, which is solved exactly (a dense inverse).
#define MG_MAXLEV 20
#define MG_DENSE_PTS 16      // the coarsest level: at most this many points, solved by its inverse
#define MG_SMEM_PTS 1248     // a domain's coarsest levels, up to this many points together, run in one block
// their operators (5), smoother weights, vectors b, x, t and interpolation
// weights (4 floats) per point, and the coarsest level's inverse
#define MG_SMEM_BYTES ((MG_SMEM_PTS * 11 + MG_DENSE_PTS * MG_DENSE_PTS) * 8)
#ifndef MG_CHUNK0
#define MG_CHUNK0 (4 * OLF_THREADS)  // points of a level-0 chunk (the CG's vectors), four per thread
#endif
struct MgDom {
    int nlev;                      // levels; 0 when the domain has no interior cell
    int lc;                        // first level run by the domain's block (levels lc .. nlev-1)
    int nx;                        // surface row length (level 0 indexing)
    int c0_first, c0_count;        // the domain's level-0 chunks (CG partial sums)
    int pad;
    int m[MG_MAXLEV], n[MG_MAXLEV];             // points per level in x and y
    unsigned char hx[MG_MAXLEV], hy[MG_MAXLEV]; // level l+1 halves x (y) of level l
    long long off[MG_MAXLEV];      // level 0: the domain's surface offset; else first coarse point
    long long pwo[MG_MAXLEV];      // first interpolation-weight slot of level l (l < nlev - 1)
    long long dio;                 // first entry of the coarsest level's inverse
};
// A run of up to OLF_THREADS (level 0: MG_CHUNK0) consecutive points of one
// level of one domain.
struct MgChunk {
    int dom, lev, first, count;
};
struct MgCtrl {
    int active, pad;
};

// Diagnostics accumulated on the device (copied into dhara_diagnostics).
struct DevDiag {
    long long picard_iters_total, krylov_iters_total, refine_iters_total, overland_iters_total;
    int picard_iters_last, krylov_iters_last, picard_nonconverged, krylov_nonconverged;
    int overland_nonconverged, nonfinite, pad0, pad1;
    double mb_last, mb_cum, storage_cum, top_cum, bottom_cum, rain_cum;
    double olf_out_cum, olf_clip_cum, ponded, picard_err_last, krylov_relres_last;
    unsigned long long branch_sig;  // hash-sum of the run's discrete decisions (record_branches)
};

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int error;
    int pad;
};

// Global counters for the persistent kernels.
struct GlobalCtrl {
    int n_active;        // domains with an active outer solve
    int n_inner_active;  // domains with an active inner solve
    int n_olf_active;
    unsigned int olf_bar;  // arrivals at the resident overland solve's barrier
    int olf_live[4];     // domains still iterating, rotating over three phases
    int n_picard;        // domains whose Picard iteration is not done this step (k_step)
    int pad_g;
};

// Number of double partial sums per tile kept for reductions.
#define NPART 12

// Device pointers of a handle.  T-typed buffers are float in mixed mode and
// double in FP64 mode; they are stored as void* and cast in the kernels.
struct DevPtrs {
    const DomainDesc *dom;
    const TileDesc *tiles;
    int ntiles, ndom;
    int smem_nz;         // column capacity of the d' buffer of the column solves in shared memory
    int pad_smem;
    // 3D double state
    double *psin, *thetan, *psim, *x, *b, *ksat, *alpha, *nvg;
    // FP64 coefficients of the outer residual (alias K, D in FP64 mode)
    double *K64, *D64;
    // 3D inner-precision buffers: stencil coefficients, the inner solve's
    // double-buffered z (preconditioned residual), t = M^-1 A p and p, its
    // solution increment d, and the column preconditioner's stored
    // L D L^T factors (1/den, c' = c/den), computed once per outer cycle
    void *K, *D, *p0, *p1, *z0, *z1, *t0, *t1, *d, *finv, *fc;
    // 2D double
    double *ztopo, *mann, *h, *H, *ph, *ppt, *esoil, *tr, *hpoten, *qtop, *ktop, *bcqb;
    double *olf_k;       // 4*C: kw, ke, ks, kn per column (row-based)
    double *olf_b, *olf_r, *olf_p0, *olf_p1, *olf_z;
    double *olf_w, *olf_s, *olf_p;
    const OlfSeg *oseg;  // [nseg]
    OlfSegState *osst;   // [nseg]
    double *olf_part;    // [2][3][nseg] recurrence sums + [nseg] ||b||^2 partials
    int nseg, pad_seg;
    // multigrid-preconditioned overland CG (overland_mg.cu)
    const MgDom *mgd;    // [ndom]
    const MgChunk *mgc;  // chunk lists: level l's at mg_lchunk[l] .. mg_lchunk[l+1]-1
    int mg_lchunk[MG_MAXLEV + 2];
    int mg_lg;           // levels run as grid phases: the largest lc of any domain
    int mg_nchunk0;      // level-0 chunks (every domain with an interior)
    int n_frozen;        // domains with DomainDesc::frozen set (time-step halving)
    long long mg_nc;     // coarse points of all domains and levels
    double *mg_a;        // [5][mg_nc]: C, E, N, NE, NW of every coarse row
    double *mg_w, *mg_b, *mg_x, *mg_t;  // [mg_nc] 1/smoother weight, rhs, pre- and post-smoothed
    double *mg_w0;       // [C] level 0's smoother weights 0.8 / a_ii (surface indexing)
    float4 *mg_pw;       // interpolation weights of every fine point to its (up to) four parents
    double *mg_r;        // [25][mg_nc] restriction stencils P^T (I - A W^-1) of the grid levels' coarse points
    double *mg_dinv;     // the coarsest level's inverse of every domain (row-major, symmetric)
    double *mg_part;     // [5][mg_nchunk0] chunk partials: p.q, r.r, r.z (two slots), b.b
    MgCtrl *mgctl;       // [ndom]
    // faces
    double *bcqw, *bcqe, *bcqs, *bcqn;
    // Dirichlet faces: 1 where the face is type 0, and the fixed heads
    unsigned char *dir_w, *dir_e, *dir_s, *dir_n, *dir_b;
    double *psi_w, *psi_e, *psi_s, *psi_n, *psi_b;
    int *procmap;
    double *rda;         // [ndom][nproc_max*nz_max]
    int nproc_max, rda_stride;
    double *rain_sched;
    // control
    KrylovCtrl *kctrl;
    PicardCtrl *pctrl;
    OverlandCtrl *octrl;
    DevDiag *diag;
    GlobalCtrl *gctrl;
    GridBarrier *barrier;
    double *partials;    // [NPART][ntiles] (structure of arrays)
    unsigned int *arrive;// [ndom][4]
    double *step_acc;    // [ndom][16] per-step sums
    const CUtensorMap *tmaps;  // [ndom][NMAP] TMA descriptors of the 3D arrays
};

// Host-side launchers (subsurface.cu / overland.cu).
struct LaunchCfg {
    int coop_blocks_3d;   // resident blocks for the persistent 3D solve
    int coop_blocks_2d;
    int olf_res_blocks;    // co-resident blocks of the shared-memory-resident overland solve
    int olf_stream_blocks; // co-resident blocks of the streaming overland solve
    // block schedule (dhara_autotune): blocks per SM actually launched
    int sms;
    int krylov_per_sm_max, krylov_per_sm;
    int olf_stream_per_sm_max, olf_stream_per_sm;
    int olf_allow_resident;
    int smem_3d;          // dynamic shared memory bytes of the 3D solve
    int nz_max;
    int mixed;
    int step_per_sm;      // co-resident blocks per SM of the fused step kernel
    int fused_step;       // run the subsurface step as one launch (k_step)
    int uniform_tx;       // the tile width shared by every domain (32 or 16), 0 if they differ
    int olf_mg;           // overland solve: 1 multigrid-preconditioned CG, 0 pipelined Jacobi-PCG
    int mg_blocks;        // co-resident blocks of the multigrid solve
};

cudaError_t launch_psi_from_theta(const DevPtrs &P, cudaStream_t s);
cudaError_t launch_prepare(const DevPtrs &P, int mixed, cudaStream_t s);
cudaError_t launch_prologue(const DevPtrs &P, cudaStream_t s);
cudaError_t launch_assemble(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s);
cudaError_t launch_krylov(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s);
// prologue, Picard loop (assembly, Dirichlet passes, solve, check) and
// epilogue of a subsurface step in one persistent launch
cudaError_t launch_step(const DevPtrs &P, const LaunchCfg &L, int maxiter, int dirichlet, cudaStream_t s);
cudaError_t launch_dirichlet(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s);
cudaError_t launch_picard_check(const DevPtrs &P, cudaStream_t s);
cudaError_t launch_epilogue(const DevPtrs &P, const LaunchCfg &L, cudaStream_t s);
cudaError_t launch_eval_fields(const DevPtrs &P, int which, double *out, cudaStream_t s);
// Saves (action 1) or restores (action 2) each domain's step state -- psi^n,
// theta^n, K_top, ponding, depth, elevation and its diagnostics -- to or from
// the copy in S; a restore also resets the Picard and Krylov initial guesses.
struct StepState {
    double *psin, *thetan, *ktop, *ph, *h, *H;
    DevDiag *diag;
    const int *action;  // [ndom]
};
cudaError_t launch_step_state(const DevPtrs &P, const StepState &S, cudaStream_t s);
cudaError_t launch_advance_step(const DevPtrs &P, cudaStream_t s);
cudaError_t launch_overland_setup(const DevPtrs &P, long long ctot, cudaStream_t s);
cudaError_t launch_overland_solve(const DevPtrs &P, const LaunchCfg &L, long long ctot, cudaStream_t s);
cudaError_t launch_overland_finish(const DevPtrs &P, long long ctot, cudaStream_t s);
// Multigrid hierarchy of the overland solve for the given domains: per-domain
// levels, the chunk lists (level by level) and the number of coarse points.
cudaError_t launch_overland_mg(const DevPtrs &P, const LaunchCfg &L, long long ctot, cudaStream_t s);
bool mg_plan(const std::vector<DomainDesc> &doms, std::vector<MgDom> &mgd, std::vector<MgChunk> &chunks,
             int (&lchunk)[MG_MAXLEV + 2], int &lg, long long &nc, long long &npw, long long &ndinv);
cudaError_t configure_mg(LaunchCfg &L, int device);
// Discrete adjoint (adjoint.cu).  Tape of one checkpoint segment, the
// carried adjoint state and the gradient accumulators; 3D arrays in the
// pitched layout of the handle, 2D arrays dense.
struct AdjPtrs {
    long long np, nc;          // 3D (pitched) and 2D array lengths
    int maxiter;               // Picard iterations stored per step
    int step_in_seg;           // slot of the step being reversed
    // tape, per step slot s: inputs of the step, every Picard iterate, the
    // overland input depth and solution, the theta misfit seed
    double *t_psin, *t_thetan;         // [S][np]
    double *t_ktop, *t_ph;             // [S][nc]
    double *t_psim, *t_xm;             // [S][maxiter][np]
    double *t_hin, *t_hsol;            // [S][nc]
    double *t_thseed;                  // [S][3][nc]
    int *t_iters;                      // [S]
    // loss
    const double *theta_target;        // [nsteps][3][nc]
    const double *q_target;            // [nsteps]
    double *qhist;                     // [nsteps]
    double *q_prev;                    // [1] boundary outflow total before the step
    double *loss;                      // [1]
    double w_q;
    // carried adjoint of the state after the step being reversed
    double *psibar_next, *thbar_next;  // [np]
    double *ktopbar_next, *phbar;      // [nc]
    // per Picard iteration
    double *xbar, *psimbar, *thmbar, *cmbar;  // [np]
    // accumulated adjoint of the step's inputs
    double *psinbar, *thnbar;          // [np]
    double *qtbar, *hpbar, *phsub_bar; // [nc]
    double *olf_Hbar, *olf_hbar;       // [nc]
    // gradients (pitched 3D)
    double *g_lk, *g_al, *g_n;
};

cudaError_t launch_adj_loss(const DevPtrs &P, const AdjPtrs &A, int t, int seed_slot, cudaStream_t s);
cudaError_t launch_adj_olf_rhs(const DevPtrs &P, const AdjPtrs &A, int t, cudaStream_t s);
cudaError_t launch_adj_olf_coef(const DevPtrs &P, const AdjPtrs &A, int t, long long ctot, cudaStream_t s);
cudaError_t launch_adj_olf_finish(const DevPtrs &P, const AdjPtrs &A, cudaStream_t s);
cudaError_t launch_adj_epilogue(const DevPtrs &P, const AdjPtrs &A, int slot, int iters, cudaStream_t s);
cudaError_t launch_adj_matrix(const DevPtrs &P, const AdjPtrs &A, int slot, int m, int zero_guess, int mixed,
                              cudaStream_t s);
cudaError_t launch_adj_picard(const DevPtrs &P, const AdjPtrs &A, int slot, int m, cudaStream_t s);
cudaError_t launch_adj_prologue(const DevPtrs &P, const AdjPtrs &A, int slot, cudaStream_t s);
cudaError_t launch_adj_initial(const DevPtrs &P, const AdjPtrs &A, cudaStream_t s);

cudaError_t launch_layer_stats(const DevPtrs &P, double *part, int nz_max, double *hist, int max_steps,
                               cudaStream_t s);

cudaError_t configure_3d(LaunchCfg &L, int device, int ntiles);
cudaError_t configure_2d(LaunchCfg &L, int device);
