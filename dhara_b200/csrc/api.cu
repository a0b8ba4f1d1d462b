// api.cu -- the C ABI of include/dhara_gpu.h: handle lifetime, device memory
// layout, uploads/downloads, and the launch sequence of one coupled step.
//
// One time step for every domain of a handle (the reference's
// SubsurfaceFlowModel then OverlandFlowModel, src/device.cu:450-458) is a
// fixed launch sequence with no host synchronisation:
//   k_prologue; [k_assemble, k_krylov (persistent), k_picard_check] x maxiter;
//   k_epilogue; k_olf_setup, k_olf_pcg_res or k_olf_pcg (persistent), k_olf_finish
// Domains whose Picard loop has converged skip the remaining iterations on the
// device, so the sequence can be captured once into a CUDA graph and replayed.
#include "internal.h"

#include <cudaTypedefs.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err = "no error";

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(DHARA_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
    } while (0)

enum { KT_KRYLOV = 0, KT_ASSEMBLE, KT_CHECK, KT_EPILOGUE, KT_OLF_SOLVE, KT_OLF_AUX, KT_PROLOGUE, KT_ADJOINT, KT_STEP, KT_N };

}  // namespace

struct dhara_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int ndom = 0;
    int mixed = 0;
    int nz_max = 1;
    int maxiter_picard = 1;
    std::vector<dhara_params> params;
    std::vector<DomainDesc> hdom;
    std::vector<TileDesc> htiles;
    int tile_mode = 0;      // dhara_launch_config::tile_shape in effect
    size_t tiles_cap = 0;   // capacity of the device tile list and per-tile partials
    std::vector<OlfSeg> hsegs;
    long long Ntot = 0, Ctot = 0, WEtot = 0, SNtot = 0;
    DevPtrs P{};
    LaunchCfg L{};
    std::vector<void *> allocs;
    double *scratch = nullptr;
    DomainDesc *d_dom = nullptr;
    std::vector<int> nproc;
    std::vector<std::vector<double>> roots;
    std::vector<std::vector<double>> sched;
    std::vector<unsigned> uploaded;  // bitmask per domain
    bool prepared = false;
    // time-step halving (dt_halvings): the saved step state, per-domain
    // actions, and the accepted / attempted step counts per domain
    int max_halvings = 0;
    StepState substate{};
    int *d_action = nullptr;
    std::vector<long long> substeps, attempts;
    // graph replay
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_failed = false;
    long long graph_launches = 0;  // kernels in the captured step
    // timing
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[KT_N];
    std::vector<cudaEvent_t> event_pool;
    double total_ms[KT_N] = {};
    long long launches[KT_N] = {};
    long long launch_count = 0;
    std::vector<int> adj_step_host;  // step counters uploaded by the adjoint sweep
    bool any_dirichlet = false;      // some domain has a type-0 face
    std::vector<std::vector<bool>> face_dirichlet;  // [domain][W, E, S, N, B]
    // per-step statistics (dhara_enable_statistics)
    int stats_steps = 0;
    double *stats_part = nullptr, *stats_hist = nullptr;
    // snapshots (dhara_snapshot): two device staging slots drained by a copy stream
    cudaStream_t copy_stream = nullptr;
    double *snap[2] = {nullptr, nullptr};
    cudaEvent_t snap_ready[2] = {nullptr, nullptr}, snap_done[2] = {nullptr, nullptr};
    bool snap_used[2] = {false, false};
    int snap_slot = 0;
};

namespace {

enum { UP_PSI = 1, UP_THETA = 2, UP_KSAT = 4, UP_ZTOPO = 8 };

template <typename T>
int dalloc(dhara_handle *h, T **p, size_t count) {
    void *q = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DHARA_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                    cudaGetErrorString(e));
    }
    h->allocs.push_back(q);
    *p = (T *)q;
    return DHARA_OK;
}

int dalloc_void(dhara_handle *h, void **p, size_t bytes) {
    char *q = nullptr;
    int rc = dalloc(h, &q, bytes);
    *p = q;
    return rc;
}

int validate(const dhara_params &p, int d) {
    if (p.struct_size != (int)sizeof(dhara_params))
        return fail(DHARA_ERR_INVALID, "domain %d: struct_size %d != sizeof(dhara_params) %d", d,
                    p.struct_size, (int)sizeof(dhara_params));
    if (p.nx < 1 || p.ny < 1 || p.nz < 1)
        return fail(DHARA_ERR_INVALID, "domain %d: grid %dx%dx%d must be positive", d, p.nx, p.ny, p.nz);
    if (p.nz > NZ_MAX)
        return fail(DHARA_ERR_UNSUPPORTED, "domain %d: nz=%d exceeds the column limit %d", d, p.nz, NZ_MAX);
    if (!(p.dx > 0) || !(p.dy > 0) || !(p.dz > 0) || !(p.dt > 0))
        return fail(DHARA_ERR_INVALID, "domain %d: dx, dy, dz, dt must be > 0", d);
    if (!(p.theta_s > p.theta_r) || !(p.n > 1.0) || !(p.alpha > 0) || !(p.porosity > 0) || !(p.Ss >= 0))
        return fail(DHARA_ERR_INVALID, "domain %d: invalid van Genuchten parameters", d);
    if (p.picard_maxiter < 1 || p.krylov_maxiter < 1 || p.overland_maxiter < 0)
        return fail(DHARA_ERR_INVALID, "domain %d: iteration caps must be positive", d);
    if (!(p.am >= 0.0 && p.am < 1.0))
        return fail(DHARA_ERR_INVALID, "domain %d: am must be in [0, 1)", d);
    if (p.picard_rule < 0 || p.picard_rule > 2 || p.theta_update < 0 || p.theta_update > 2)
        return fail(DHARA_ERR_INVALID, "domain %d: unknown picard_rule / theta_update", d);
    if (p.precision != DHARA_FP64 && p.precision != DHARA_MIXED)
        return fail(DHARA_ERR_INVALID, "domain %d: unknown precision %d", d, p.precision);
    if (!(p.krylov_tol > 0) || !(p.overland_tol > 0) || !(p.picard_tol > 0))
        return fail(DHARA_ERR_INVALID, "domain %d: tolerances must be > 0", d);
    if (p.overland_solver < 0 || p.overland_solver > 1)
        return fail(DHARA_ERR_INVALID, "domain %d: unknown overland_solver %d", d, p.overland_solver);
    if (p.dt_halvings < 0 || p.dt_halvings > 20)
        return fail(DHARA_ERR_INVALID, "domain %d: dt_halvings must be in [0, 20]", d);
    return DHARA_OK;
}

int set_dev(dhara_handle *h) {
    CK(cudaSetDevice(h->device));
    return DHARA_OK;
}

cudaEvent_t get_event(dhara_handle *h) {
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

struct Timed {
    dhara_handle *h;
    int kind;
    cudaEvent_t a = nullptr, b = nullptr;
    Timed(dhara_handle *hh, int k) : h(hh), kind(k) {
        h->launch_count += 1;
        h->launches[kind] += 1;
        if (h->timing) {
            a = get_event(h);
            b = get_event(h);
            cudaEventRecord(a, h->stream);
        }
    }
    ~Timed() {
        if (h->timing) {
            cudaEventRecord(b, h->stream);
            h->pending[kind].push_back({a, b});
        }
    }
};

void collect_timing(dhara_handle *h) {
    for (int k = 0; k < KT_N; ++k) {
        for (auto &pr : h->pending[k]) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) h->total_ms[k] += ms;
            h->event_pool.push_back(pr.first);
            h->event_pool.push_back(pr.second);
        }
        h->pending[k].clear();
    }
}

#define LAUNCH(kind, call)                                                                     \
    do {                                                                                       \
        Timed t_(h, kind);                                                                     \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(DHARA_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

// With a tape (the adjoint's recompute sweep), every Picard iterate psi^m and
// solution x^m is copied into the tape slot after its solve, so the step runs
// as separate launches; otherwise, with the fused schedule, as one k_step.
int enqueue_subsurface(dhara_handle *h, const AdjPtrs *tape = nullptr, int slot = 0) {
    const DevPtrs &P = h->P;
    cudaStream_t s = h->stream;
    if (!tape && h->L.fused_step) {
        LAUNCH(KT_STEP, launch_step(P, h->L, h->maxiter_picard, h->any_dirichlet ? 1 : 0, s));
        if (h->stats_steps > 0) {
            LAUNCH(KT_EPILOGUE, launch_layer_stats(P, h->stats_part, h->nz_max, h->stats_hist, h->stats_steps, s));
            h->launch_count += 1;  // the statistics are two kernels
        }
        return DHARA_OK;
    }
    LAUNCH(KT_PROLOGUE, launch_prologue(P, s));
    for (int m = 0; m < h->maxiter_picard; ++m) {
        LAUNCH(KT_ASSEMBLE, launch_assemble(P, h->L, s));
        if (h->any_dirichlet) {
            LAUNCH(KT_ASSEMBLE, launch_dirichlet(P, h->L, s));
            h->launch_count += 1;  // two kernels
        }
        LAUNCH(KT_KRYLOV, launch_krylov(P, h->L, s));
        if (tape) {
            const size_t off = ((size_t)slot * tape->maxiter + m) * tape->np;
            CK(cudaMemcpyAsync(tape->t_psim + off, P.psim, tape->np * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(tape->t_xm + off, P.x, tape->np * 8, cudaMemcpyDeviceToDevice, s));
        }
        LAUNCH(KT_CHECK, launch_picard_check(P, s));
    }
    LAUNCH(KT_EPILOGUE, launch_epilogue(P, h->L, s));
    if (h->stats_steps > 0) {
        LAUNCH(KT_EPILOGUE, launch_layer_stats(P, h->stats_part, h->nz_max, h->stats_hist, h->stats_steps, s));
        h->launch_count += 1;  // the statistics are two kernels
    }
    return DHARA_OK;
}

int enqueue_overland(dhara_handle *h) {
    const DevPtrs &P = h->P;
    cudaStream_t s = h->stream;
    LAUNCH(KT_OLF_AUX, launch_overland_setup(P, h->Ctot, s));
    LAUNCH(KT_OLF_SOLVE, launch_overland_solve(P, h->L, h->Ctot, s));
    LAUNCH(KT_OLF_AUX, launch_overland_finish(P, h->Ctot, s));
    return DHARA_OK;
}

int check_device_error(dhara_handle *h) {
    GridBarrier gb;
    CK(cudaMemcpyAsync(&gb, h->P.barrier, sizeof(gb), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (gb.error)
        return fail(DHARA_ERR_TIMEOUT, "a persistent kernel's grid barrier timed out; results are invalid");
    return DHARA_OK;
}

struct FieldLoc {
    void *ptr;
    long long count;
    size_t elt;
    bool is_int;
    bool computed;  // download evaluates the closure
    int which;
    bool is3d;      // pitched 3D array (rows of nx values at pitch nxp)
};

int locate(dhara_handle *h, int dom, int field, FieldLoc *out) {
    if (dom < 0 || dom >= h->ndom) return fail(DHARA_ERR_INVALID, "domain %d out of range", dom);
    const DomainDesc &D = h->hdom[dom];
    const long long N = (long long)D.nx * D.ny * D.nz, C = (long long)D.nx * D.ny;
    const long long WE = (long long)D.nz * D.ny, SN = (long long)D.nz * D.nx;
    DevPtrs &P = h->P;
    FieldLoc f{nullptr, 0, sizeof(double), false, false, 0, false};
    switch (field) {
        case DHARA_F_PSI: f.ptr = P.psin + D.off3; f.count = N; break;
        case DHARA_F_THETA: f.ptr = P.thetan + D.off3; f.count = N; break;
        case DHARA_F_KSAT: f.ptr = P.ksat + D.off3; f.count = N; break;
        case DHARA_F_ALPHA:
            if (!P.alpha && dalloc(h, &P.alpha, (size_t)h->Ntot)) return DHARA_ERR_NOMEM;
            f.ptr = P.alpha + D.off3; f.count = N; break;
        case DHARA_F_NVG:
            if (!P.nvg && dalloc(h, &P.nvg, (size_t)h->Ntot)) return DHARA_ERR_NOMEM;
            f.ptr = P.nvg + D.off3; f.count = N; break;
        case DHARA_F_K: f.count = N; f.computed = true; f.which = 1; break;
        case DHARA_F_C: f.count = N; f.computed = true; f.which = 2; break;
        case DHARA_F_THETA_NEW: f.count = N; f.computed = true; f.which = 0; break;
        case DHARA_F_ZTOPO: f.ptr = P.ztopo + D.off2; f.count = C; break;
        case DHARA_F_MANN: f.ptr = P.mann + D.off2; f.count = C; break;
        case DHARA_F_WATERDEPTH: f.ptr = P.h + D.off2; f.count = C; break;
        case DHARA_F_WATERELEV: f.ptr = P.H + D.off2; f.count = C; break;
        case DHARA_F_PONDING: f.ptr = P.ph + D.off2; f.count = C; break;
        case DHARA_F_PPT: f.ptr = P.ppt + D.off2; f.count = C; break;
        case DHARA_F_ESOIL: f.ptr = P.esoil + D.off2; f.count = C; break;
        case DHARA_F_TR: f.ptr = P.tr + D.off2; f.count = C; break;
        case DHARA_F_HPOTEN: f.ptr = P.hpoten + D.off2; f.count = C; break;
        case DHARA_F_QTOP: f.ptr = P.qtop + D.off2; f.count = C; break;
        case DHARA_F_BCQB: f.ptr = P.bcqb + D.off2; f.count = C; break;
        case DHARA_F_BCQW: f.ptr = P.bcqw + D.offWE; f.count = WE; break;
        case DHARA_F_BCQE: f.ptr = P.bcqe + D.offWE; f.count = WE; break;
        case DHARA_F_BCQS: f.ptr = P.bcqs + D.offSN; f.count = SN; break;
        case DHARA_F_BCQN: f.ptr = P.bcqn + D.offSN; f.count = SN; break;
        case DHARA_F_BCPSIW: f.ptr = P.psi_w + D.offWE; f.count = WE; break;
        case DHARA_F_BCPSIE: f.ptr = P.psi_e + D.offWE; f.count = WE; break;
        case DHARA_F_BCPSIS: f.ptr = P.psi_s + D.offSN; f.count = SN; break;
        case DHARA_F_BCPSIN: f.ptr = P.psi_n + D.offSN; f.count = SN; break;
        case DHARA_F_BCPSIB: f.ptr = P.psi_b + D.off2; f.count = C; break;
        case DHARA_FI_BCW: case DHARA_FI_BCE: f.count = WE; f.is_int = true; f.elt = 4; break;
        case DHARA_FI_BCS: case DHARA_FI_BCN: f.count = SN; f.is_int = true; f.elt = 4; break;
        case DHARA_FI_BCB: case DHARA_FI_BCT: f.count = C; f.is_int = true; f.elt = 4; break;
        case DHARA_FI_PROCMAP: f.ptr = P.procmap + D.off2; f.count = C; f.is_int = true; f.elt = 4; break;
        default: return fail(DHARA_ERR_INVALID, "unknown field id %d", field);
    }
    f.is3d = field <= DHARA_F_THETA_NEW;
    *out = f;
    return DHARA_OK;
}

int upload_dom_desc(dhara_handle *h) {
    CK(cudaMemcpyAsync(h->d_dom, h->hdom.data(), sizeof(DomainDesc) * h->ndom, cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DHARA_OK;
}

// Tiles of a domain with shape tx x ty.
size_t tile_count(const DomainDesc &D, int tx, int ty) {
    return (size_t)((D.nx + tx - 1) / tx) * (size_t)((D.ny + ty - 1) / ty);
}

// Tile shape of each domain and the tile list for `mode` (dhara_launch_config
// tile_shape): 1 all 32 x 4, 2 all 16 x 8, 0 per domain the shape with fewer
// tiles (fewer idle threads in ragged tiles; 32 x 4 on a tie, its rows being
// whole 128-byte lines).  Tiles of a domain are consecutive, row by row.
void plan_tiles(dhara_handle *h, int mode) {
    h->htiles.clear();
    for (int d = 0; d < h->ndom; ++d) {
        DomainDesc &D = h->hdom[d];
        bool narrow = mode == 2;
        if (mode == 0) narrow = tile_count(D, 16, 8) < tile_count(D, TILE_X, TILE_Y);
        D.tx = narrow ? 16 : TILE_X;
        D.ty = narrow ? 8 : TILE_Y;
        D.tx_log2 = narrow ? 4 : 5;
        D.tile_begin = (int)h->htiles.size();
        for (int y0 = 0; y0 < D.ny; y0 += D.ty)
            for (int x0 = 0; x0 < D.nx; x0 += D.tx) h->htiles.push_back({d, x0, y0, 0});
        D.tile_end = (int)h->htiles.size();
    }
    h->tile_mode = mode;
    h->L.uniform_tx = h->hdom[0].tx;
    for (const DomainDesc &D : h->hdom)
        if (D.tx != h->L.uniform_tx) h->L.uniform_tx = 0;
}

int build_tensor_maps(dhara_handle *h);

// Uploads the tile list and the domain table of the current plan and re-encodes
// the TMA boxes (their extents are the tile shape's); any captured step graph
// holds the old grid sizes and is dropped.
int apply_tiles(dhara_handle *h) {
    if (h->htiles.size() > h->tiles_cap) return fail(DHARA_ERR_INVALID, "internal: tile list exceeds capacity");
    CK(cudaMemcpyAsync((void *)h->P.tiles, h->htiles.data(), sizeof(TileDesc) * h->htiles.size(),
                       cudaMemcpyHostToDevice, h->stream));
    h->P.ntiles = (int)h->htiles.size();
    int rc = upload_dom_desc(h);
    if (!rc) rc = build_tensor_maps(h);
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    return rc;
}


// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// One 3D tiled map over a domain's part of a pitched array: dims (nx, ny, nz),
// row pitch nxp; box (tx + 2*xoff, ty + 2, chunk) for halo reads or
// (tx, ty, chunk) for own-column reads, tx x ty the domain's tile shape.
// Out-of-range elements read as zero.
int encode_map(CUtensorMap *m, const void *array, size_t elt, const DomainDesc &D, bool halo, int chunk) {
    const int TX = D.tx, TY = D.ty;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return fail(DHARA_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[3] = {(cuuint64_t)D.nx, (cuuint64_t)D.ny, (cuuint64_t)D.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)D.nxp * elt, (cuuint64_t)D.nxp * D.ny * elt};
    const int xoff = (int)(16 / elt);
    const cuuint32_t box[3] = {(cuuint32_t)(halo ? TX + 2 * xoff : TX), (cuuint32_t)(halo ? TY + 2 : TY),
                               (cuuint32_t)chunk};
    const cuuint32_t estr[3] = {1, 1, 1};
    void *base = (void *)((const char *)array + (size_t)D.off3 * elt);
    if (((uintptr_t)base & 15) != 0 || (strides[0] & 15) != 0)
        return fail(DHARA_ERR_INVALID, "internal: unaligned 3D array for TMA");
    const CUtensorMapDataType dt = elt == 2   ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                   : elt == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                              : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUresult r = enc(m, dt, 3, base,
                     dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(DHARA_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return DHARA_OK;
}

int build_tensor_maps(dhara_handle *h) {
    const DevPtrs &P = h->P;
    const size_t sT = h->mixed ? 4 : 8;
    const int chi = h->mixed ? CHUNK_F32 : CHUNK_F64;
    std::vector<CUtensorMap> maps((size_t)h->ndom * NMAP);
    for (int d = 0; d < h->ndom; ++d) {
        const DomainDesc &D = h->hdom[d];
        CUtensorMap *m = &maps[(size_t)d * NMAP];
        int rc = 0;
        rc |= encode_map(m + MAP_P0_H, P.p0, sT, D, true, chi);
        rc |= encode_map(m + MAP_P1_H, P.p1, sT, D, true, chi);
        rc |= encode_map(m + MAP_Z0_H, P.z0, sT, D, true, chi);
        rc |= encode_map(m + MAP_Z1_H, P.z1, sT, D, true, chi);
        rc |= encode_map(m + MAP_T0_H, P.t0, sT, D, true, chi);
        rc |= encode_map(m + MAP_T1_H, P.t1, sT, D, true, chi);
        rc |= encode_map(m + MAP_K_H, P.K, sT, D, true, chi);
        rc |= encode_map(m + MAP_D_O, P.D, sT, D, false, chi);
        rc |= encode_map(m + MAP_DD_O, P.d, sT, D, false, chi);
        rc |= encode_map(m + MAP_INV_O, P.finv, FACTOR_BYTES(h->mixed), D, false, chi);
        rc |= encode_map(m + MAP_C_O, P.fc, FACTOR_BYTES(h->mixed), D, false, chi);
        rc |= encode_map(m + MAP_X64_H, P.x, 8, D, true, CH_R);
        rc |= encode_map(m + MAP_K64_H, P.K64, 8, D, true, CH_R);
        rc |= encode_map(m + MAP_D64_O, P.D64, 8, D, false, CH_R);
        rc |= encode_map(m + MAP_B_O, P.b, 8, D, false, CH_R);
        if (rc) return rc;
    }
    CUtensorMap *dm = const_cast<CUtensorMap *>(h->P.tmaps);
    if (!dm && dalloc(h, &dm, maps.size())) return DHARA_ERR_NOMEM;
    CK(cudaMemcpyAsync(dm, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->P.tmaps = dm;
    return DHARA_OK;
}

}  // namespace

// Lets the library's other translation units report through dhara_last_error
// (not exported).
__attribute__((visibility("hidden"))) int dhara_internal_fail(int code, const char *msg) {
    g_err = msg;
    return code;
}

// ====================================================================== ABI
extern "C" {

const char *dhara_last_error(void) { return g_err.c_str(); }

int dhara_enable_statistics(dhara_handle *h, int max_steps) {
    if (!h || max_steps < 1) return fail(DHARA_ERR_INVALID, "need a handle and max_steps >= 1");
    if (h->stats_steps > 0) return fail(DHARA_ERR_STATE, "statistics are already enabled");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    const size_t row = 1 + 2 * (size_t)h->nz_max;
    if (dalloc(h, &h->stats_part, h->tiles_cap * h->nz_max * 2)) return DHARA_ERR_NOMEM;
    if (dalloc(h, &h->stats_hist, (size_t)h->ndom * max_steps * row)) return DHARA_ERR_NOMEM;
    CK(cudaMemsetAsync(h->stats_hist, 0, (size_t)h->ndom * max_steps * row * 8, h->stream));
    h->stats_steps = max_steps;
    if (h->graph_exec) {  // the step sequence changed
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    return DHARA_OK;
}

int dhara_get_statistics(dhara_handle *h, int domain, int64_t *nsteps, double *mb_subsurfaceW,
                         double *pressure_sum, double *moisture_sum) {
    if (!h || !nsteps) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (domain < 0 || domain >= h->ndom) return fail(DHARA_ERR_INVALID, "domain %d out of range", domain);
    if (h->stats_steps < 1) return fail(DHARA_ERR_STATE, "statistics are not enabled");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    PicardCtrl pc;
    CK(cudaMemcpyAsync(&pc, &h->P.pctrl[domain], sizeof(pc), cudaMemcpyDeviceToHost, h->stream));
    const size_t row = 1 + 2 * (size_t)h->nz_max;
    std::vector<double> hist((size_t)h->stats_steps * row);
    CK(cudaMemcpyAsync(hist.data(), h->stats_hist + (size_t)domain * h->stats_steps * row, hist.size() * 8,
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int n = std::min(pc.step, h->stats_steps);
    const int nz = h->hdom[domain].nz;
    *nsteps = n;
    for (int t = 0; t < n; ++t) {
        const double *r = hist.data() + (size_t)t * row;
        if (mb_subsurfaceW) mb_subsurfaceW[t] = r[0];
        for (int k = 0; k < nz; ++k) {
            if (pressure_sum) pressure_sum[(size_t)t * nz + k] = r[1 + k];
            if (moisture_sum) moisture_sum[(size_t)t * nz + k] = r[1 + h->nz_max + k];
        }
    }
    return DHARA_OK;
}

int dhara_snapshot(dhara_handle *h, int domain, double *water_elevation, double *water_depth,
                   double *pressure_head, double *moisture) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (domain < 0 || domain >= h->ndom) return fail(DHARA_ERR_INVALID, "domain %d out of range", domain);
    if (set_dev(h)) return DHARA_ERR_CUDA;
    const DomainDesc &D = h->hdom[domain];
    const size_t np = (size_t)D.nxp * D.ny * D.nz, nc = (size_t)D.nx * D.ny;
    const size_t slot_len = 2 * np + 2 * nc;
    if (!h->copy_stream) {
        CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CK(cudaEventCreateWithFlags(&h->snap_ready[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&h->snap_done[k], cudaEventDisableTiming));
        }
    }
    // staging slots sized for the largest domain of the handle
    if (!h->snap[0]) {
        size_t most = 0;
        for (const DomainDesc &E : h->hdom)
            most = std::max(most, 2 * (size_t)E.nxp * E.ny * E.nz + 2 * (size_t)E.nx * E.ny);
        for (int k = 0; k < 2; ++k)
            if (dalloc(h, &h->snap[k], most)) return DHARA_ERR_NOMEM;
    }
    (void)slot_len;
    const int k = h->snap_slot;
    h->snap_slot ^= 1;
    double *st = h->snap[k];
    const DevPtrs &P = h->P;
    cudaStream_t s = h->stream;
    // the slot's previous copy-out must be finished before it is overwritten
    if (h->snap_used[k]) CK(cudaStreamWaitEvent(s, h->snap_done[k], 0));
    CK(cudaMemcpyAsync(st, P.psin + D.off3, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st + np, P.thetan + D.off3, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st + 2 * np, P.H + D.off2, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st + 2 * np + nc, P.h + D.off2, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaEventRecord(h->snap_ready[k], s));
    cudaStream_t c = h->copy_stream;
    CK(cudaStreamWaitEvent(c, h->snap_ready[k], 0));
    const size_t row = (size_t)D.nx * 8, pitch = (size_t)D.nxp * 8;
    if (pressure_head)
        CK(cudaMemcpy2DAsync(pressure_head, row, st, pitch, row, (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost, c));
    if (moisture)
        CK(cudaMemcpy2DAsync(moisture, row, st + np, pitch, row, (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost, c));
    if (water_elevation) CK(cudaMemcpyAsync(water_elevation, st + 2 * np, nc * 8, cudaMemcpyDeviceToHost, c));
    if (water_depth) CK(cudaMemcpyAsync(water_depth, st + 2 * np + nc, nc * 8, cudaMemcpyDeviceToHost, c));
    CK(cudaEventRecord(h->snap_done[k], c));
    h->snap_used[k] = true;
    return DHARA_OK;
}

int dhara_snapshot_wait(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (!h->copy_stream) return DHARA_OK;
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->copy_stream));
    return DHARA_OK;
}

int dhara_get_params(dhara_handle *h, int domain, dhara_params *out) {
    if (!h || !out) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (domain < 0 || domain >= h->ndom) return fail(DHARA_ERR_INVALID, "domain %d out of range", domain);
    *out = h->params[domain];
    return DHARA_OK;
}
int dhara_abi_version(void) { return DHARA_ABI_VERSION; }

void dhara_default_params(dhara_params *p, int nx, int ny, int nz, double dx, double dy, double dz,
                          double dt) {
    std::memset(p, 0, sizeof(*p));
    p->struct_size = (int32_t)sizeof(dhara_params);
    p->nx = nx; p->ny = ny; p->nz = nz;
    p->dx = dx; p->dy = dy; p->dz = dz; p->dt = dt;
    // include/devconst.h:13-31, alpha 0.02 /cm = 2.0 /m
    p->alpha = 2.0; p->n = 1.8; p->theta_s = 0.45; p->theta_r = 0.1; p->porosity = 0.45; p->Ss = 5e-4;
    p->airdry = -5.0; p->psimin = 5e-3; p->am = 0.0;
    p->delta = 1e-7; p->hmin = 1e-5; p->hcri = 0.0; p->K0 = 1e-5;
    p->sec_p_mm2dt_p_m = dt / 1000.0;
    // MAXIMUM_ITERATIONS, PICARD_METHOD, TOLERANCE_PRESSURE (examples/1-EBI/ebi.cfg)
    p->picard_maxiter = 10; p->picard_rule = DHARA_PICARD_PSI_RELATIVE; p->picard_tol = 1e-8;
    // cusp::monitor(rhs, 100, 1e-8) and (rhs2d, 100, 1e-9): src/subsurface.cu:750, overland.cu:410
    p->krylov_maxiter = 100; p->krylov_tol = 1e-8; p->theta_update = DHARA_THETA_REFERENCE;
    p->overland_maxiter = 100; p->overland_tol = 1e-9; p->precision = DHARA_FP64;
    p->inner_tol = 1e-4; p->inner_maxiter = 60;
}

int dhara_create(const dhara_params *params, int ndomains, int device, dhara_handle **out) {
    if (!out) return fail(DHARA_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!params || ndomains < 1) return fail(DHARA_ERR_INVALID, "need at least one domain");
    for (int d = 0; d < ndomains; ++d) {
        int rc = validate(params[d], d);
        if (rc) return rc;
        if (params[d].precision != params[0].precision)
            return fail(DHARA_ERR_INVALID, "all domains of a handle must share one precision");
        if (params[d].overland_solver != params[0].overland_solver)
            return fail(DHARA_ERR_INVALID, "all domains of a handle must share one overland solver");
    }
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0) CK(cudaGetDevice(&device));
    if (device >= ndev) return fail(DHARA_ERR_INVALID, "device %d of %d", device, ndev);
    dhara_handle *h = new dhara_handle();
    h->device = device;
    h->ndom = ndomains;
    h->params.assign(params, params + ndomains);
    h->mixed = params[0].precision == DHARA_MIXED;
    auto bail = [&](int rc) {
        dhara_destroy(h);
        return rc;
    };
    if (set_dev(h)) return bail(DHARA_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(DHARA_ERR_CUDA, "cudaStreamCreate failed"));

    // domains, offsets and tiles
    h->hdom.resize(ndomains);
    for (int d = 0; d < ndomains; ++d) {
        const dhara_params &p = params[d];
        DomainDesc &D = h->hdom[d];
        std::memset(&D, 0, sizeof(D));
        D.nx = p.nx; D.ny = p.ny; D.nz = p.nz;
        D.picard_rule = p.picard_rule; D.theta_update = p.theta_update;
        D.picard_maxiter = p.picard_maxiter; D.krylov_maxiter = p.krylov_maxiter;
        D.overland_maxiter = p.overland_maxiter;
        D.inner_maxiter = h->mixed ? (p.inner_maxiter > 0 ? p.inner_maxiter : p.krylov_maxiter) : p.krylov_maxiter;
        D.nxp = (p.nx + 7) & ~7;  // rows of every array 16-byte aligned, 2-byte factors included
        h->Ntot = (h->Ntot + 31) & ~31LL;  // 128-byte aligned base for FP32 and FP64
        D.off3 = h->Ntot; D.off2 = h->Ctot; D.offWE = h->WEtot; D.offSN = h->SNtot;
        h->Ntot += (long long)D.nxp * p.ny * p.nz;
        h->Ctot += (long long)p.nx * p.ny;
        h->WEtot += (long long)p.nz * p.ny;
        h->SNtot += (long long)p.nz * p.nx;
        D.dx = p.dx; D.dy = p.dy; D.dz = p.dz; D.dt = p.dt;
        D.alpha = p.alpha; D.n = p.n; D.theta_s = p.theta_s; D.theta_r = p.theta_r;
        D.porosity = p.porosity; D.Ss = p.Ss; D.am = p.am;
        D.delta = p.delta; D.hmin = p.hmin; D.K0 = p.K0; D.sec = p.sec_p_mm2dt_p_m;
        D.picard_tol = p.picard_tol; D.krylov_tol = p.krylov_tol;
        D.inner_tol = h->mixed ? (p.inner_tol > 0 ? p.inner_tol : 1e-4) : 0.0;
        D.overland_tol = p.overland_tol;
        D.closure_fp32 = (h->mixed && p.closure_fp32) ? 1 : 0;
        D.closure_fast = (h->mixed && !p.closure_fp32) ? 1 : 0;
        D.record_branches = p.record_branches & 127;
        D.sub_frac = 1.0;
        D.step_advance = 1;
        h->max_halvings = std::max(h->max_halvings, (int)p.dt_halvings);
        // overland segments: runs of up to OLF_SEG surface cells of this domain
        {
            const int first = (int)h->hsegs.size();
            const int C2 = p.nx * p.ny;
            const int nseg = (C2 + OLF_SEG - 1) / OLF_SEG;
            for (int k = 0; k < nseg; ++k) {
                OlfSeg sg;
                std::memset(&sg, 0, sizeof(sg));
                sg.begin = D.off2 + (long long)k * OLF_SEG;
                sg.dom = d;
                sg.l0 = k * OLF_SEG;
                sg.count = std::min(OLF_SEG, C2 - k * OLF_SEG);
                sg.first = first;
                sg.nseg = nseg;
                h->hsegs.push_back(sg);
            }
        }
        if (p.nz > h->nz_max) h->nz_max = p.nz;
        if (p.picard_maxiter > h->maxiter_picard) h->maxiter_picard = p.picard_maxiter;
    }
    // the inner sweeps index cells with 32-bit offsets
    if (h->Ntot >= (1LL << 31))
        return bail(fail(DHARA_ERR_UNSUPPORTED, "a handle holds at most 2^31 - 1 cells (with row padding); got %lld",
                         (long long)h->Ntot));
    // tile lists: room for either shape's list, the per-domain plan by default
    for (int d = 0; d < ndomains; ++d)
        h->tiles_cap += std::max(tile_count(h->hdom[d], TILE_X, TILE_Y), tile_count(h->hdom[d], 16, 8));
    plan_tiles(h, 0);
    h->nproc.assign(ndomains, 1);
    h->roots.assign(ndomains, std::vector<double>());
    h->sched.assign(ndomains, std::vector<double>());
    h->uploaded.assign(ndomains, 0u);
    h->face_dirichlet.assign(ndomains, std::vector<bool>(5, false));

    DevPtrs &P = h->P;
    const size_t N = (size_t)h->Ntot, C = (size_t)h->Ctot;
    const size_t sT = h->mixed ? sizeof(float) : sizeof(double);
    int rc = 0;
    rc |= dalloc(h, &h->d_dom, ndomains);
    TileDesc *d_tiles = nullptr;
    rc |= dalloc(h, &d_tiles, h->tiles_cap);
    for (double **q : {&P.psin, &P.thetan, &P.psim, &P.x, &P.b, &P.ksat}) rc |= dalloc(h, q, N);
    for (void **q : {&P.K, &P.D, &P.p0, &P.p1, &P.z0, &P.z1, &P.t0, &P.t1, &P.d})
        rc |= dalloc_void(h, q, N * sT);
    const size_t sF = FACTOR_BYTES(h->mixed);
    for (void **q : {&P.finv, &P.fc}) rc |= dalloc_void(h, q, N * sF);
    if (h->mixed) {
        rc |= dalloc(h, &P.K64, N);
        rc |= dalloc(h, &P.D64, N);
    } else {
        P.K64 = (double *)P.K;
        P.D64 = (double *)P.D;
    }
    for (double **q : {&P.ztopo, &P.mann, &P.h, &P.H, &P.ph, &P.ppt, &P.esoil, &P.tr, &P.hpoten, &P.qtop,
                       &P.ktop, &P.bcqb, &P.olf_b, &P.olf_r, &P.olf_p0, &P.olf_p1, &P.olf_z, &P.olf_w,
                       &P.olf_s, &P.olf_p})
        rc |= dalloc(h, q, C);
    // multigrid hierarchy of the overland solve
    std::vector<MgDom> mgd;
    std::vector<MgChunk> mgc;
    int lchunk[MG_MAXLEV + 2];
    int mg_lg = 0;
    long long mg_nc = 0, mg_npw = 0, mg_ndinv = 0;
    if (!mg_plan(h->hdom, mgd, mgc, lchunk, mg_lg, mg_nc, mg_npw, mg_ndinv))
        return bail(fail(DHARA_ERR_UNSUPPORTED, "a surface grid needs more than %d multigrid levels", MG_MAXLEV));
    MgDom *d_mgd = nullptr;
    MgChunk *d_mgc = nullptr;
    const int nchunk0 = lchunk[1] - lchunk[0];
    rc |= dalloc(h, &d_mgd, ndomains);
    rc |= dalloc(h, &d_mgc, std::max<size_t>(mgc.size(), 1));
    rc |= dalloc(h, &P.mg_a, 5 * (size_t)std::max(mg_nc, 1LL));
    for (double **q : {&P.mg_w, &P.mg_b, &P.mg_x, &P.mg_t}) rc |= dalloc(h, q, (size_t)std::max(mg_nc, 1LL));
    rc |= dalloc(h, &P.mg_w0, C);
    rc |= dalloc(h, &P.mg_pw, (size_t)std::max(mg_npw, 1LL));
    rc |= dalloc(h, &P.mg_r, 25 * (size_t)std::max(mg_nc, 1LL));
    rc |= dalloc(h, &P.mg_dinv, (size_t)std::max(mg_ndinv, 1LL));
    rc |= dalloc(h, &P.mg_part, 5 * (size_t)std::max(nchunk0, 1));
    rc |= dalloc(h, &P.mgctl, ndomains);
    OlfSeg *d_oseg = nullptr;
    rc |= dalloc(h, &d_oseg, h->hsegs.size());
    rc |= dalloc(h, &P.osst, h->hsegs.size());
    rc |= dalloc(h, &P.olf_part, 7 * h->hsegs.size());
    rc |= dalloc(h, &P.olf_k, 4 * C);
    rc |= dalloc(h, &P.bcqw, (size_t)h->WEtot);
    rc |= dalloc(h, &P.bcqe, (size_t)h->WEtot);
    rc |= dalloc(h, &P.bcqs, (size_t)h->SNtot);
    rc |= dalloc(h, &P.bcqn, (size_t)h->SNtot);
    rc |= dalloc(h, &P.psi_w, (size_t)h->WEtot);
    rc |= dalloc(h, &P.psi_e, (size_t)h->WEtot);
    rc |= dalloc(h, &P.psi_s, (size_t)h->SNtot);
    rc |= dalloc(h, &P.psi_n, (size_t)h->SNtot);
    rc |= dalloc(h, &P.psi_b, C);
    rc |= dalloc(h, &P.dir_w, (size_t)h->WEtot);
    rc |= dalloc(h, &P.dir_e, (size_t)h->WEtot);
    rc |= dalloc(h, &P.dir_s, (size_t)h->SNtot);
    rc |= dalloc(h, &P.dir_n, (size_t)h->SNtot);
    rc |= dalloc(h, &P.dir_b, C);
    rc |= dalloc(h, &P.procmap, C);
    P.nproc_max = 1;
    P.rda_stride = h->nz_max;
    rc |= dalloc(h, &P.rda, (size_t)ndomains * P.rda_stride);
    rc |= dalloc(h, &P.kctrl, ndomains);
    rc |= dalloc(h, &P.pctrl, ndomains);
    rc |= dalloc(h, &P.octrl, ndomains);
    rc |= dalloc(h, &P.diag, ndomains);
    rc |= dalloc(h, &P.gctrl, 1);
    rc |= dalloc(h, &P.barrier, 1);
    rc |= dalloc(h, &P.partials, h->tiles_cap * NPART);
    rc |= dalloc(h, &P.arrive, (size_t)ndomains * 4);
    rc |= dalloc(h, &P.step_acc, (size_t)ndomains * 16);
    if (rc) return bail(DHARA_ERR_NOMEM);
    P.dom = h->d_dom;
    P.tiles = d_tiles;
    P.oseg = d_oseg;
    P.nseg = (int)h->hsegs.size();
    P.mgd = d_mgd;
    P.mgc = d_mgc;
    std::memcpy(P.mg_lchunk, lchunk, sizeof(lchunk));
    P.mg_lg = mg_lg;
    P.mg_nchunk0 = nchunk0;
    P.mg_nc = mg_nc;
    P.ntiles = (int)h->htiles.size();
    P.ndom = ndomains;
    P.smem_nz = h->nz_max;
    P.alpha = P.nvg = nullptr;
    P.rain_sched = nullptr;

    // zero everything so unset inputs are defined (fluxes 0, procmap 0, roots 0)
    for (void *q : h->allocs) {
        (void)q;
    }
    auto zero = [&](void *p, size_t bytes) { return cudaMemsetAsync(p, 0, bytes, h->stream); };
    cudaError_t e = cudaSuccess;
    for (double *q : {P.psin, P.thetan, P.psim, P.x, P.b, P.ksat}) e = e ? e : zero(q, N * 8);
    for (void *q : {P.K, P.D, P.p0, P.p1, P.z0, P.z1, P.t0, P.t1, P.d}) e = e ? e : zero(q, N * sT);
    for (void *q : {P.finv, P.fc}) e = e ? e : zero(q, N * sF);
    for (double *q : {P.K64, P.D64}) e = e ? e : zero(q, N * 8);
    for (double *q : {P.ztopo, P.mann, P.h, P.H, P.ph, P.ppt, P.esoil, P.tr, P.hpoten, P.qtop, P.ktop, P.bcqb,
                      P.olf_b, P.olf_r, P.olf_p0, P.olf_p1, P.olf_z, P.olf_w, P.olf_s, P.olf_p})
        e = e ? e : zero(q, C * 8);
    e = e ? e : zero(P.osst, h->hsegs.size() * sizeof(OlfSegState));
    e = e ? e : zero(P.olf_part, 7 * h->hsegs.size() * 8);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_oseg, h->hsegs.data(), sizeof(OlfSeg) * h->hsegs.size(), cudaMemcpyHostToDevice,
                            h->stream);
    e = e ? e : zero(P.olf_k, 4 * C * 8);
    e = e ? e : zero(P.mgctl, ndomains * sizeof(MgCtrl));
    e = e ? e : zero(P.mg_part, 5 * (size_t)std::max(nchunk0, 1) * 8);
    for (double *q : {P.mg_a, P.mg_w, P.mg_b, P.mg_x, P.mg_t})
        e = e ? e : zero(q, (q == P.mg_a ? 5 : 1) * (size_t)std::max(mg_nc, 1LL) * 8);
    e = e ? e : zero(P.mg_w0, C * 8);
    e = e ? e : zero(P.mg_pw, (size_t)std::max(mg_npw, 1LL) * sizeof(float4));
    e = e ? e : zero(P.mg_r, 25 * (size_t)std::max(mg_nc, 1LL) * 8);
    e = e ? e : zero(P.mg_dinv, (size_t)std::max(mg_ndinv, 1LL) * 8);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_mgd, mgd.data(), sizeof(MgDom) * mgd.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && !mgc.empty())
        e = cudaMemcpyAsync(d_mgc, mgc.data(), sizeof(MgChunk) * mgc.size(), cudaMemcpyHostToDevice, h->stream);
    e = e ? e : zero(P.bcqw, (size_t)h->WEtot * 8);
    e = e ? e : zero(P.bcqe, (size_t)h->WEtot * 8);
    e = e ? e : zero(P.bcqs, (size_t)h->SNtot * 8);
    e = e ? e : zero(P.bcqn, (size_t)h->SNtot * 8);
    for (double *q : {P.psi_w, P.psi_e}) e = e ? e : zero(q, (size_t)h->WEtot * 8);
    for (double *q : {P.psi_s, P.psi_n}) e = e ? e : zero(q, (size_t)h->SNtot * 8);
    e = e ? e : zero(P.psi_b, C * 8);
    for (unsigned char *q : {P.dir_w, P.dir_e}) e = e ? e : zero(q, (size_t)h->WEtot);
    for (unsigned char *q : {P.dir_s, P.dir_n}) e = e ? e : zero(q, (size_t)h->SNtot);
    e = e ? e : zero(P.dir_b, C);
    e = e ? e : zero(P.procmap, C * 4);
    e = e ? e : zero(P.rda, (size_t)ndomains * P.rda_stride * 8);
    e = e ? e : zero(P.kctrl, ndomains * sizeof(KrylovCtrl));
    e = e ? e : zero(P.pctrl, ndomains * sizeof(PicardCtrl));
    e = e ? e : zero(P.octrl, ndomains * sizeof(OverlandCtrl));
    e = e ? e : zero(P.diag, ndomains * sizeof(DevDiag));
    e = e ? e : zero(P.gctrl, sizeof(GlobalCtrl));
    e = e ? e : zero(P.barrier, sizeof(GridBarrier));
    e = e ? e : zero(P.partials, h->tiles_cap * NPART * 8);
    e = e ? e : zero(P.arrive, (size_t)ndomains * 4 * 4);
    e = e ? e : zero(P.step_acc, (size_t)ndomains * 16 * 8);
    if (e != cudaSuccess) return bail(fail(DHARA_ERR_CUDA, "initialising device memory: %s", cudaGetErrorString(e)));
    if (cudaMemcpyAsync(d_tiles, h->htiles.data(), sizeof(TileDesc) * h->htiles.size(), cudaMemcpyHostToDevice,
                        h->stream) != cudaSuccess)
        return bail(fail(DHARA_ERR_CUDA, "tile upload failed"));
    if (upload_dom_desc(h)) return bail(DHARA_ERR_CUDA);
    {
        const int rc2 = build_tensor_maps(h);
        if (rc2) return bail(rc2);
    }

    h->substeps.assign(ndomains, 0);
    h->attempts.assign(ndomains, 0);
    if (h->max_halvings > 0) {
        StepState &S = h->substate;
        rc |= dalloc(h, &S.psin, N);
        rc |= dalloc(h, &S.thetan, N);
        for (double **q : {&S.ktop, &S.ph, &S.h, &S.H}) rc |= dalloc(h, q, C);
        rc |= dalloc(h, &S.diag, ndomains);
        rc |= dalloc(h, &h->d_action, ndomains);
        if (rc) return bail(DHARA_ERR_NOMEM);
        S.action = h->d_action;
    }
    h->L.nz_max = h->nz_max;
    h->L.mixed = h->mixed;
    h->L.olf_mg = params[0].overland_solver == 0 ? 1 : 0;
    e = configure_3d(h->L, device, P.ntiles);
    if (e == cudaSuccess) e = configure_2d(h->L, device);
    if (e == cudaSuccess) e = configure_mg(h->L, device);
    if (e != cudaSuccess) return bail(fail(DHARA_ERR_CUDA, "kernel configuration: %s", cudaGetErrorString(e)));
    *out = h;
    return DHARA_OK;
}

void dhara_internal_forget(dhara_handle *h);  // dropin.cu

int dhara_destroy(dhara_handle *h) {
    if (!h) return DHARA_OK;
    dhara_internal_forget(h);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    for (int k = 0; k < KT_N; ++k)
        for (auto &pr : h->pending[k]) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    for (cudaEvent_t ev : h->event_pool) cudaEventDestroy(ev);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    for (int k = 0; k < 2; ++k) {
        if (h->snap_ready[k]) cudaEventDestroy(h->snap_ready[k]);
        if (h->snap_done[k]) cudaEventDestroy(h->snap_done[k]);
    }
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    for (void *q : h->allocs) cudaFree(q);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return DHARA_OK;
}

int dhara_upload(dhara_handle *h, int domain, int field, const double *src, int64_t count) {
    if (!h || !src) return fail(DHARA_ERR_INVALID, "NULL handle or source");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    FieldLoc f;
    int rc = locate(h, domain, field, &f);
    if (rc) return rc;
    if (f.is_int) return fail(DHARA_ERR_INVALID, "field %d is an int32 field", field);
    if (f.computed) return fail(DHARA_ERR_INVALID, "field %d is output-only", field);
    if (count != f.count) return fail(DHARA_ERR_INVALID, "field %d expects %lld values, got %lld", field,
                                      (long long)f.count, (long long)count);
    for (int64_t i = 0; i < count; ++i)
        if (!std::isfinite(src[i]))
            return fail(DHARA_ERR_NONFINITE, "field %d value %lld is not finite", field, (long long)i);
    if (!f.ptr) return DHARA_OK;  // Dirichlet values: only meaningful with Dirichlet faces
    if (f.is3d) {
        const DomainDesc &D = h->hdom[domain];
        CK(cudaMemcpy2DAsync(f.ptr, (size_t)D.nxp * sizeof(double), src, (size_t)D.nx * sizeof(double),
                             (size_t)D.nx * sizeof(double), (size_t)D.ny * D.nz, cudaMemcpyHostToDevice,
                             h->stream));
    } else {
        CK(cudaMemcpyAsync(f.ptr, src, count * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    if (field == DHARA_F_ALPHA || field == DHARA_F_NVG) {
        if (field == DHARA_F_ALPHA) h->hdom[domain].has_alpha = 1;
        else h->hdom[domain].has_n = 1;
        if (upload_dom_desc(h)) return DHARA_ERR_CUDA;
    }
    if (field == DHARA_F_PSI) h->uploaded[domain] |= UP_PSI;
    if (field == DHARA_F_THETA) h->uploaded[domain] |= UP_THETA;
    if (field == DHARA_F_KSAT) h->uploaded[domain] |= UP_KSAT;
    if (field == DHARA_F_ZTOPO) h->uploaded[domain] |= UP_ZTOPO;
    return DHARA_OK;
}

int dhara_upload_int(dhara_handle *h, int domain, int field, const int32_t *src, int64_t count) {
    if (!h || !src) return fail(DHARA_ERR_INVALID, "NULL handle or source");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    FieldLoc f;
    int rc = locate(h, domain, field, &f);
    if (rc) return rc;
    if (!f.is_int) return fail(DHARA_ERR_INVALID, "field %d is a double field", field);
    if (count != f.count) return fail(DHARA_ERR_INVALID, "field %d expects %lld values, got %lld", field,
                                      (long long)f.count, (long long)count);
    if (field == DHARA_FI_PROCMAP) {
        for (int64_t i = 0; i < count; ++i)
            if (src[i] < 0 || src[i] >= h->nproc[domain])
                return fail(DHARA_ERR_INVALID, "procmap[%lld]=%d outside [0, %d) (call dhara_set_roots first)",
                            (long long)i, src[i], h->nproc[domain]);
        CK(cudaMemcpyAsync(f.ptr, src, count * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return DHARA_OK;
    }
    if (field == DHARA_FI_BCT) return DHARA_OK;  // the top is always a flux face (src/global.cu:236-251)
    // side and bottom faces: 1 where the face is Dirichlet (type 0)
    DevPtrs &P = h->P;
    DomainDesc &D = h->hdom[domain];
    unsigned char *dst = nullptr;
    switch (field) {
        case DHARA_FI_BCW: dst = P.dir_w + D.offWE; break;
        case DHARA_FI_BCE: dst = P.dir_e + D.offWE; break;
        case DHARA_FI_BCS: dst = P.dir_s + D.offSN; break;
        case DHARA_FI_BCN: dst = P.dir_n + D.offSN; break;
        case DHARA_FI_BCB: dst = P.dir_b + D.off2; break;
        default: return fail(DHARA_ERR_INVALID, "field %d is not a boundary type field", field);
    }
    std::vector<unsigned char> flags((size_t)count);
    bool any = false;
    for (int64_t i = 0; i < count; ++i) {
        flags[(size_t)i] = src[i] == 0 ? 1 : 0;
        any = any || src[i] == 0;
    }
    CK(cudaMemcpyAsync(dst, flags.data(), (size_t)count, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->face_dirichlet[domain][field - DHARA_FI_BCW] = any;
    bool dom_any = false;
    for (bool b : h->face_dirichlet[domain]) dom_any = dom_any || b;
    if ((D.has_dirichlet != 0) != dom_any) {
        D.has_dirichlet = dom_any ? 1 : 0;
        if (upload_dom_desc(h)) return DHARA_ERR_CUDA;
    }
    h->any_dirichlet = false;
    for (const DomainDesc &E : h->hdom) h->any_dirichlet = h->any_dirichlet || E.has_dirichlet;
    if (h->graph_exec) {  // the step sequence may change
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    return DHARA_OK;
}

int dhara_download(dhara_handle *h, int domain, int field, double *dst, int64_t count) {
    if (!h || !dst) return fail(DHARA_ERR_INVALID, "NULL handle or destination");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    FieldLoc f;
    int rc = locate(h, domain, field, &f);
    if (rc) return rc;
    if (f.is_int) return fail(DHARA_ERR_INVALID, "field %d is an int32 field", field);
    if (count != f.count) return fail(DHARA_ERR_INVALID, "field %d holds %lld values, asked %lld", field,
                                      (long long)f.count, (long long)count);
    const DomainDesc &D = h->hdom[domain];
    if (f.computed) {
        if (!h->scratch && dalloc(h, &h->scratch, (size_t)h->Ntot)) return DHARA_ERR_NOMEM;
        CK(launch_eval_fields(h->P, f.which, h->scratch, h->stream));
        f.ptr = h->scratch + D.off3;
    }
    if (!f.ptr) return fail(DHARA_ERR_INVALID, "field %d is not stored on the GPU path", field);
    if (f.is3d) {
        CK(cudaMemcpy2DAsync(dst, (size_t)D.nx * sizeof(double), f.ptr, (size_t)D.nxp * sizeof(double),
                             (size_t)D.nx * sizeof(double), (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost,
                             h->stream));
    } else {
        CK(cudaMemcpyAsync(dst, f.ptr, count * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return DHARA_OK;
}

int dhara_upload_device(dhara_handle *h, int domain, int field, const double *dsrc, int64_t count) {
    if (!h || !dsrc) return fail(DHARA_ERR_INVALID, "NULL handle or source");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    FieldLoc f;
    int rc = locate(h, domain, field, &f);
    if (rc) return rc;
    if (f.is_int || f.computed) return fail(DHARA_ERR_INVALID, "field %d cannot be uploaded from the device", field);
    if (count != f.count) return fail(DHARA_ERR_INVALID, "field %d expects %lld values, got %lld", field,
                                      (long long)f.count, (long long)count);
    if (!f.ptr) return DHARA_OK;
    const DomainDesc &D = h->hdom[domain];
    if (f.is3d)
        CK(cudaMemcpy2DAsync(f.ptr, (size_t)D.nxp * sizeof(double), dsrc, (size_t)D.nx * sizeof(double),
                             (size_t)D.nx * sizeof(double), (size_t)D.ny * D.nz, cudaMemcpyDeviceToDevice,
                             h->stream));
    else
        CK(cudaMemcpyAsync(f.ptr, dsrc, count * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (field == DHARA_F_PSI) h->uploaded[domain] |= UP_PSI;
    if (field == DHARA_F_THETA) h->uploaded[domain] |= UP_THETA;
    if (field == DHARA_F_KSAT) h->uploaded[domain] |= UP_KSAT;
    if (field == DHARA_F_ZTOPO) h->uploaded[domain] |= UP_ZTOPO;
    return DHARA_OK;
}

int dhara_download_device(dhara_handle *h, int domain, int field, double *ddst, int64_t count) {
    if (!h || !ddst) return fail(DHARA_ERR_INVALID, "NULL handle or destination");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    FieldLoc f;
    int rc = locate(h, domain, field, &f);
    if (rc) return rc;
    if (f.is_int) return fail(DHARA_ERR_INVALID, "field %d is an int32 field", field);
    if (count != f.count) return fail(DHARA_ERR_INVALID, "field %d holds %lld values, asked %lld", field,
                                      (long long)f.count, (long long)count);
    const DomainDesc &D = h->hdom[domain];
    if (f.computed) {
        if (!h->scratch && dalloc(h, &h->scratch, (size_t)h->Ntot)) return DHARA_ERR_NOMEM;
        CK(launch_eval_fields(h->P, f.which, h->scratch, h->stream));
        f.ptr = h->scratch + D.off3;
    }
    if (!f.ptr) return fail(DHARA_ERR_INVALID, "field %d is not stored on the GPU path", field);
    if (f.is3d)
        CK(cudaMemcpy2DAsync(ddst, (size_t)D.nx * sizeof(double), f.ptr, (size_t)D.nxp * sizeof(double),
                             (size_t)D.nx * sizeof(double), (size_t)D.ny * D.nz, cudaMemcpyDeviceToDevice,
                             h->stream));
    else
        CK(cudaMemcpyAsync(ddst, f.ptr, count * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DHARA_OK;
}

int dhara_set_roots(dhara_handle *h, int domain, const double *rda, int nproc) {
    if (!h || !rda || nproc < 1) return fail(DHARA_ERR_INVALID, "bad arguments");
    if (domain < 0 || domain >= h->ndom) return fail(DHARA_ERR_INVALID, "domain out of range");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    const int nz = h->hdom[domain].nz;
    h->nproc[domain] = nproc;
    h->roots[domain].assign(rda, rda + (size_t)nproc * nz);
    int nproc_max = 1;
    for (int n : h->nproc) nproc_max = n > nproc_max ? n : nproc_max;
    const int stride = nproc_max * h->nz_max;
    std::vector<double> all((size_t)h->ndom * stride, 0.0);
    for (int d = 0; d < h->ndom; ++d)
        for (size_t q = 0; q < h->roots[d].size(); ++q) all[(size_t)d * stride + q] = h->roots[d][q];
    if (stride != h->P.rda_stride) {
        double *p = nullptr;
        if (dalloc(h, &p, all.size())) return DHARA_ERR_NOMEM;
        h->P.rda = p;
        h->P.rda_stride = stride;
        h->P.nproc_max = nproc_max;
        if (h->graph_exec) { cudaGraphExecDestroy(h->graph_exec); h->graph_exec = nullptr; }
    }
    CK(cudaMemcpyAsync(h->P.rda, all.data(), all.size() * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return DHARA_OK;
}

int dhara_set_rain_schedule(dhara_handle *h, int domain, const double *mm, int nsteps) {
    if (!h || (nsteps > 0 && !mm) || nsteps < 0) return fail(DHARA_ERR_INVALID, "bad arguments");
    if (domain < 0 || domain >= h->ndom) return fail(DHARA_ERR_INVALID, "domain out of range");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    h->sched[domain].assign(mm, mm + nsteps);
    std::vector<double> all;
    for (int d = 0; d < h->ndom; ++d) {
        h->hdom[d].sched_off = (long long)all.size();
        h->hdom[d].sched_len = (int)h->sched[d].size();
        all.insert(all.end(), h->sched[d].begin(), h->sched[d].end());
    }
    double *p = nullptr;
    if (dalloc(h, &p, all.size())) return DHARA_ERR_NOMEM;
    if (!all.empty())
        CK(cudaMemcpyAsync(p, all.data(), all.size() * 8, cudaMemcpyHostToDevice, h->stream));
    h->P.rain_sched = p;
    if (h->graph_exec) { cudaGraphExecDestroy(h->graph_exec); h->graph_exec = nullptr; }
    return upload_dom_desc(h);
}

int dhara_psi_from_theta(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    for (int d = 0; d < h->ndom; ++d)
        if (!(h->uploaded[d] & UP_THETA)) return fail(DHARA_ERR_STATE, "domain %d: theta not uploaded", d);
    CK(launch_psi_from_theta(h->P, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int d = 0; d < h->ndom; ++d) h->uploaded[d] |= UP_PSI;
    return DHARA_OK;
}

int dhara_prepare(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    for (int d = 0; d < h->ndom; ++d) {
        const unsigned need = UP_PSI | UP_KSAT | UP_ZTOPO;
        if ((h->uploaded[d] & need) != need)
            return fail(DHARA_ERR_STATE, "domain %d: psi (or theta + dhara_psi_from_theta), ksat and ztopo "
                                         "must be uploaded before dhara_prepare", d);
    }
    const DevPtrs &P = h->P;
    CK(cudaMemsetAsync(P.pctrl, 0, h->ndom * sizeof(PicardCtrl), h->stream));
    CK(cudaMemsetAsync(P.kctrl, 0, h->ndom * sizeof(KrylovCtrl), h->stream));
    CK(cudaMemsetAsync(P.octrl, 0, h->ndom * sizeof(OverlandCtrl), h->stream));
    CK(cudaMemsetAsync(P.diag, 0, h->ndom * sizeof(DevDiag), h->stream));
    CK(cudaMemsetAsync(P.gctrl, 0, sizeof(GlobalCtrl), h->stream));
    CK(cudaMemsetAsync(P.barrier, 0, sizeof(GridBarrier), h->stream));
    CK(cudaMemsetAsync(P.arrive, 0, (size_t)h->ndom * 16, h->stream));
    CK(launch_prepare(P, h->mixed, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->prepared = true;
    return DHARA_OK;
}

int dhara_subsurface_step(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    return enqueue_subsurface(h);
}

int dhara_overland_step(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    return enqueue_overland(h);
}

namespace {

// Steps with time-step halving: every round of attempts advances each domain
// that still has time left in the step by its current sub-step, dt / 2^k.  A
// domain whose Picard iteration converged (or that is at its smallest
// sub-step) keeps the result and saves it; one that did not is restored to
// its last saved state and halves.  A domain that has finished the step is
// frozen for the further rounds (no Picard iteration, no overland solve with
// the multigrid solver) and restored after each.  The host reads the Picard
// outcome once per round.
int step_halving(dhara_handle *h, int nsteps) {
    const DevPtrs &P = h->P;
    cudaStream_t s = h->stream;
    if (h->stats_steps > 0) return fail(DHARA_ERR_UNSUPPORTED, "layer statistics are not kept with dt_halvings");
    const int nd = h->ndom, K = h->max_halvings;
    std::vector<int> act(nd), k(nd);
    std::vector<long long> rem(nd);
    std::vector<PicardCtrl> pc(nd);
    auto run_actions = [&]() -> int {
        CK(cudaMemcpyAsync(h->d_action, act.data(), sizeof(int) * nd, cudaMemcpyHostToDevice, s));
        LAUNCH(KT_EPILOGUE, launch_step_state(P, h->substate, s));
        return DHARA_OK;
    };
    for (int st = 0; st < nsteps; ++st) {
        std::fill(act.begin(), act.end(), 1);
        int rc = run_actions();
        if (rc) return rc;
        std::fill(k.begin(), k.end(), 0);
        std::fill(rem.begin(), rem.end(), 1LL << K);  // the step in units of dt / 2^K
        for (;;) {
            bool left = false;
            for (int d = 0; d < nd; ++d) left = left || rem[d] > 0;
            if (!left) break;
            h->P.n_frozen = 0;
            for (int d = 0; d < nd; ++d) {
                DomainDesc &D = h->hdom[d];
                D.sub_frac = std::ldexp(1.0, -k[d]);
                D.dt = h->params[d].dt * D.sub_frac;
                // ||b|| of the 3D system grows as 1/dt (the storage term), so the
                // relative tolerance shrinks with the sub-step to keep the water
                // a step's solves may leave unbalanced the same
                D.krylov_tol = h->params[d].krylov_tol * D.sub_frac;
                D.step_advance = 0;
                D.frozen = rem[d] == 0 ? 1 : 0;
                h->P.n_frozen += D.frozen;
            }
            if (upload_dom_desc(h)) return DHARA_ERR_CUDA;
            rc = enqueue_subsurface(h);
            if (!rc) rc = enqueue_overland(h);
            if (rc) return rc;
            CK(cudaMemcpyAsync(pc.data(), P.pctrl, sizeof(PicardCtrl) * nd, cudaMemcpyDeviceToHost, s));
            rc = check_device_error(h);  // synchronises
            if (rc) return rc;
            for (int d = 0; d < nd; ++d) {
                if (rem[d] == 0) {
                    act[d] = 2;
                    continue;
                }
                h->attempts[d] += 1;
                if (pc[d].converged || k[d] >= h->params[d].dt_halvings) {
                    rem[d] -= 1LL << (K - k[d]);
                    h->substeps[d] += 1;
                    act[d] = 1;
                } else {
                    act[d] = 2;
                    k[d] += 1;
                }
            }
            rc = run_actions();
            if (rc) return rc;
        }
        LAUNCH(KT_EPILOGUE, launch_advance_step(P, s));
    }
    h->P.n_frozen = 0;
    for (int d = 0; d < nd; ++d) {
        DomainDesc &D = h->hdom[d];
        D.sub_frac = 1.0;
        D.dt = h->params[d].dt;
        D.krylov_tol = h->params[d].krylov_tol;
        D.step_advance = 1;
        D.frozen = 0;
    }
    if (upload_dom_desc(h)) return DHARA_ERR_CUDA;
    return DHARA_OK;
}

}  // namespace

int dhara_step(dhara_handle *h, int nsteps, int use_graph) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (nsteps < 0) return fail(DHARA_ERR_INVALID, "nsteps < 0");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    if (h->max_halvings > 0) return step_halving(h, nsteps);
    for (int d = 0; d < h->ndom; ++d) {
        h->substeps[d] += nsteps;
        h->attempts[d] += nsteps;
    }
    if (use_graph && !h->timing && !h->graph_failed && !h->graph_exec) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const long long lc = h->launch_count;
        int rc = enqueue_subsurface(h);
        if (!rc) rc = enqueue_overland(h);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        h->graph_launches = h->launch_count - lc;  // the kernels one replay runs
        h->launch_count = lc;
        if (rc == DHARA_OK && e == cudaSuccess) e = cudaGraphInstantiate(&h->graph_exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (rc != DHARA_OK || e != cudaSuccess) {
            cudaGetLastError();
            h->graph_exec = nullptr;
            h->graph_failed = true;
        }
    }
    for (int s = 0; s < nsteps; ++s) {
        if (use_graph && h->graph_exec && !h->timing) {
            CK(cudaGraphLaunch(h->graph_exec, h->stream));
            h->launch_count += h->graph_launches;
        } else {
            int rc = enqueue_subsurface(h);
            if (rc) return rc;
            rc = enqueue_overland(h);
            if (rc) return rc;
        }
    }
    return DHARA_OK;
}

int dhara_synchronize(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    return check_device_error(h);
}

int dhara_get_diagnostics(dhara_handle *h, int domain, dhara_diagnostics *out) {
    if (!h || !out) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (domain < 0 || domain >= h->ndom) return fail(DHARA_ERR_INVALID, "domain out of range");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    DevDiag dg;
    PicardCtrl pc;
    CK(cudaMemcpyAsync(&dg, h->P.diag + domain, sizeof(dg), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&pc, h->P.pctrl + domain, sizeof(pc), cudaMemcpyDeviceToHost, h->stream));
    int rc = check_device_error(h);
    std::memset(out, 0, sizeof(*out));
    out->steps = pc.step;
    out->substeps_total = h->substeps[domain];
    out->step_attempts_total = h->attempts[domain];
    out->picard_iters_total = dg.picard_iters_total;
    out->krylov_iters_total = dg.krylov_iters_total;
    out->refine_iters_total = dg.refine_iters_total;
    out->overland_iters_total = dg.overland_iters_total;
    out->picard_iters_last = dg.picard_iters_last;
    out->krylov_iters_last = dg.krylov_iters_last;
    out->picard_nonconverged = dg.picard_nonconverged;
    out->krylov_nonconverged = dg.krylov_nonconverged;
    out->overland_nonconverged = dg.overland_nonconverged;
    out->nonfinite = dg.nonfinite;
    out->mb_subsurface_last = dg.mb_last;
    out->mb_subsurface_cum = dg.mb_cum;
    out->storage_change_cum = dg.storage_cum;
    out->top_inflow_cum = dg.top_cum;
    out->bottom_outflow_cum = dg.bottom_cum;
    out->rain_cum = dg.rain_cum;
    out->overland_boundary_out_cum = dg.olf_out_cum;
    out->overland_clip_cum = dg.olf_clip_cum;
    out->ponded_volume = dg.ponded;
    out->picard_err_last = pc.err;
    out->krylov_relres_last = dg.krylov_relres_last;
    out->branch_signature = dg.branch_sig;
    return rc;
}

int dhara_get_stream(dhara_handle *h, void **stream) {
    if (!h || !stream) return fail(DHARA_ERR_INVALID, "NULL argument");
    *stream = (void *)h->stream;
    return DHARA_OK;
}

int dhara_set_kernel_timing(dhara_handle *h, int enable) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    collect_timing(h);
    h->timing = enable != 0;
    return DHARA_OK;
}

int dhara_get_kernel_timing(dhara_handle *h, int kernel, int64_t *launches, double *total_ms) {
    if (!h || kernel < 0 || kernel >= KT_N) return fail(DHARA_ERR_INVALID, "bad kernel id");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    collect_timing(h);
    if (launches) *launches = h->launches[kernel];
    if (total_ms) *total_ms = h->total_ms[kernel];
    return DHARA_OK;
}

int dhara_reset_kernel_timing(dhara_handle *h) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    collect_timing(h);
    for (int k = 0; k < KT_N; ++k) {
        h->total_ms[k] = 0;
        h->launches[k] = 0;
    }
    h->launch_count = 0;
    return DHARA_OK;
}

int dhara_get_launch_count(dhara_handle *h, int64_t *count) {
    if (!h || !count) return fail(DHARA_ERR_INVALID, "NULL argument");
    *count = h->launch_count;
    return DHARA_OK;
}

int dhara_get_krylov_traffic(dhara_handle *h, double *bytes, int64_t *iterations) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    const double sT = h->mixed ? 4.0 : 8.0, sF = (double)FACTOR_BYTES(h->mixed);
    double total = 0.0;
    int64_t iters = 0;
    for (int d = 0; d < h->ndom; ++d) {
        dhara_diagnostics dg;
        int rc = dhara_get_diagnostics(h, d, &dg);
        if (rc) return rc;
        const DomainDesc &D = h->hdom[d];
        const double N = (double)D.nx * D.ny * D.nz;
        const double solves = (double)dg.picard_iters_total;
        const double cycles = (double)dg.refine_iters_total;
        const double upd = cycles > solves ? cycles - solves : 0.0;
        // inner iteration (one sweep): reads the previous z, t, p and K, D, d
        // and the factors 1/den, c', and writes z, t, p, d (10 T-words and 2
        // factors; the back sweep's second read of c' follows the staged read
        // and is not counted); the first sweep of a cycle reads no previous t,
        // p or d (3 T-words fewer).  Outer residual R: x, b, K64, D64 (f64) +
        // writes z (T) and the two factors + c' read back; update U: x
        // read+write (f64) + d, p (2 T).
        total += N * ((10.0 * sT + 2.0 * sF) * (double)dg.krylov_iters_total - 3.0 * sT * upd +
                      (32.0 + sT + 3.0 * sF) * cycles + (16.0 + 2.0 * sT) * upd);
        iters += dg.krylov_iters_total;
    }
    if (bytes) *bytes = total;
    if (iterations) *iterations = iters;
    return DHARA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ adjoint
namespace {

struct DevScratch {
    std::vector<void *> ptrs;
    ~DevScratch() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <typename T>
    int get(T **p, size_t count) {
        void *q = nullptr;
        if (cudaMalloc(&q, (count ? count : 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return fail(DHARA_ERR_NOMEM, "adjoint: cudaMalloc of %zu bytes failed", count * sizeof(T));
        }
        ptrs.push_back(q);
        *p = (T *)q;
        return DHARA_OK;
    }
};

// The state a step starts from: psi^n, theta^n, K(psi^n) of the top layer,
// the ponded depth (= overland depth) and the step counter.  The Krylov warm
// start equals psi^n and the overland elevation is rebuilt from the depth.
struct StateCopy {
    double *psin, *thetan, *ktop, *ph, *h, *H;
};

int copy_state(dhara_handle *h, const StateCopy &dst, bool to_handle, int step) {
    const DevPtrs &P = h->P;
    const size_t np = (size_t)h->Ntot * 8, nc = (size_t)h->Ctot * 8;
    cudaStream_t s = h->stream;
    auto cp = [&](double *handle_arr, double *copy, size_t bytes) {
        return to_handle ? cudaMemcpyAsync(handle_arr, copy, bytes, cudaMemcpyDeviceToDevice, s)
                         : cudaMemcpyAsync(copy, handle_arr, bytes, cudaMemcpyDeviceToDevice, s);
    };
    CK(cp(P.psin, dst.psin, np));
    CK(cp(P.thetan, dst.thetan, np));
    CK(cp(P.ktop, dst.ktop, nc));
    CK(cp(P.ph, dst.ph, nc));
    CK(cp(P.h, dst.h, nc));
    if (dst.H) CK(cp(P.H, dst.H, nc));
    if (to_handle) {
        CK(cudaMemcpyAsync(P.x, dst.psin, np, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(P.psim, dst.psin, np, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(&P.pctrl[0].step, &h->adj_step_host[step], sizeof(int), cudaMemcpyHostToDevice, s));
    }
    return DHARA_OK;
}

}  // namespace

int dhara_adjoint(dhara_handle *h, const dhara_adjoint_desc *desc, double *loss, double *grad_logks,
                  double *grad_alpha, double *grad_n) {
    if (!h || !desc || !loss) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (desc->struct_size != (int)sizeof(dhara_adjoint_desc))
        return fail(DHARA_ERR_INVALID, "struct_size %d != sizeof(dhara_adjoint_desc) %d", desc->struct_size,
                    (int)sizeof(dhara_adjoint_desc));
    if (h->ndom != 1) return fail(DHARA_ERR_UNSUPPORTED, "the adjoint runs on single-domain handles");
    if (h->any_dirichlet) return fail(DHARA_ERR_UNSUPPORTED, "the adjoint does not cover Dirichlet faces");
    if (h->max_halvings > 0) return fail(DHARA_ERR_UNSUPPORTED, "the adjoint does not cover dt_halvings");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (desc->nsteps < 1 || desc->checkpoint_every < 1 || !desc->theta_target || !desc->q_target)
        return fail(DHARA_ERR_INVALID, "adjoint: need nsteps >= 1, checkpoint_every >= 1 and both targets");
    const bool want_grad = grad_logks && grad_alpha && grad_n;
    if (!want_grad && (grad_logks || grad_alpha || grad_n))
        return fail(DHARA_ERR_INVALID, "adjoint: pass all three gradient arrays or none");
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    const DevPtrs &P = h->P;
    const DomainDesc &D = h->hdom[0];
    cudaStream_t s = h->stream;
    const int nsteps = desc->nsteps, K = desc->checkpoint_every;
    const int nseg = (nsteps + K - 1) / K;
    const int S = K < nsteps ? K : nsteps;
    const size_t np = (size_t)h->Ntot, nc = (size_t)h->Ctot, C = (size_t)D.nx * D.ny;
    const int M = h->maxiter_picard;

    DevScratch mem;
    AdjPtrs A;
    std::memset(&A, 0, sizeof(A));
    A.np = (long long)np;
    A.nc = (long long)nc;
    A.maxiter = M;
    A.w_q = desc->w_q;
    int rc = 0;
    double *theta_target = nullptr, *q_target = nullptr;
    rc |= mem.get(&theta_target, (size_t)nsteps * 3 * C);
    rc |= mem.get(&q_target, (size_t)nsteps);
    rc |= mem.get(&A.qhist, (size_t)nsteps);
    rc |= mem.get(&A.q_prev, 1);
    rc |= mem.get(&A.loss, 1);
    std::vector<StateCopy> ckpt(nseg + 1);
    for (int k = 0; k <= nseg && !rc; ++k) {
        rc |= mem.get(&ckpt[k].psin, np);
        rc |= mem.get(&ckpt[k].thetan, np);
        rc |= mem.get(&ckpt[k].ktop, nc);
        rc |= mem.get(&ckpt[k].ph, nc);
        rc |= mem.get(&ckpt[k].h, nc);
        ckpt[k].H = nullptr;
    }
    double *final_H = nullptr;
    rc |= mem.get(&final_H, nc);
    // the overland solution and depth of every step: the recompute sweep
    // restores them instead of solving the overland system again
    double *olf_H_all = nullptr, *olf_h_all = nullptr;
    if (want_grad) {
        rc |= mem.get(&olf_H_all, (size_t)nsteps * nc);
        rc |= mem.get(&olf_h_all, (size_t)nsteps * nc);
    }
    if (rc) return DHARA_ERR_NOMEM;
    A.theta_target = theta_target;
    A.q_target = q_target;
    CK(cudaMemcpyAsync(theta_target, desc->theta_target, (size_t)nsteps * 3 * C * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(q_target, desc->q_target, (size_t)nsteps * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(A.loss, 0, 8, s));
    CK(cudaMemcpyAsync(A.q_prev, &P.diag[0].olf_out_cum, 8, cudaMemcpyDeviceToDevice, s));

    // step counters of the checkpoints (host copies uploaded when restoring)
    PicardCtrl pc0;
    CK(cudaMemcpyAsync(&pc0, &P.pctrl[0], sizeof(pc0), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    h->adj_step_host.assign(nsteps + 1, 0);
    for (int t = 0; t <= nsteps; ++t) h->adj_step_host[t] = pc0.step + t;

    // ---- tape and adjoint buffers
    if (want_grad) {
        rc |= mem.get(&A.t_psin, (size_t)S * np);
        rc |= mem.get(&A.t_thetan, (size_t)S * np);
        rc |= mem.get(&A.t_ktop, (size_t)S * nc);
        rc |= mem.get(&A.t_ph, (size_t)S * nc);
        rc |= mem.get(&A.t_psim, (size_t)S * M * np);
        rc |= mem.get(&A.t_xm, (size_t)S * M * np);
        rc |= mem.get(&A.t_hin, (size_t)S * nc);
        rc |= mem.get(&A.t_hsol, (size_t)S * nc);
        rc |= mem.get(&A.t_thseed, (size_t)S * 3 * nc);
        rc |= mem.get(&A.t_iters, (size_t)S);
        for (double **q : {&A.psibar_next, &A.thbar_next, &A.xbar, &A.psimbar, &A.thmbar, &A.cmbar, &A.psinbar,
                           &A.thnbar, &A.g_lk, &A.g_al, &A.g_n})
            rc |= mem.get(q, np);
        for (double **q : {&A.ktopbar_next, &A.phbar, &A.qtbar, &A.hpbar, &A.phsub_bar, &A.olf_Hbar, &A.olf_hbar})
            rc |= mem.get(q, nc);
        if (rc) return DHARA_ERR_NOMEM;
    }

    // One step of the segment starting at t0, recorded into tape slot sl.
    // One step of the segment starting at t0, recorded into tape slot sl.  In
    // the first (forward) sweep the overland step runs and its results are
    // kept; in the recompute sweep they are restored.
    auto taped_step = [&](int t0, int sl, bool first_sweep) -> int {
        const size_t t = (size_t)(t0 + sl);
        CK(cudaMemcpyAsync(A.t_psin + sl * np, P.psin, np * 8, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(A.t_thetan + sl * np, P.thetan, np * 8, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(A.t_ktop + sl * nc, P.ktop, nc * 8, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(A.t_ph + sl * nc, P.ph, nc * 8, cudaMemcpyDeviceToDevice, s));
        int r = enqueue_subsurface(h, &A, sl);
        if (r) return r;
        CK(cudaMemcpyAsync(A.t_iters + sl, &P.pctrl[0].iter, sizeof(int), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(A.t_hin + sl * nc, P.h, nc * 8, cudaMemcpyDeviceToDevice, s));
        if (first_sweep) {
            r = enqueue_overland(h);
            if (r) return r;
        } else {
            CK(cudaMemcpyAsync(P.H, olf_H_all + t * nc, nc * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(P.h, olf_h_all + t * nc, nc * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(P.ph, olf_h_all + t * nc, nc * 8, cudaMemcpyDeviceToDevice, s));
        }
        CK(cudaMemcpyAsync(A.t_hsol + sl * nc, P.H, nc * 8, cudaMemcpyDeviceToDevice, s));
        LAUNCH(KT_ADJOINT, launch_adj_loss(P, A, t0 + sl, sl, s));
        return DHARA_OK;
    };

    // ---- forward sweep: checkpoints, the loss, and the tape of the last
    // segment (the first one reversed, so it needs no recompute)
    const int t0_last = (nseg - 1) * K;
    for (int t = 0; t < nsteps; ++t) {
        if (t % K == 0) {
            rc = copy_state(h, ckpt[t / K], false, 0);
            if (rc) return rc;
        }
        if (want_grad && t >= t0_last) {
            rc = taped_step(t0_last, t - t0_last, true);
        } else {
            rc = enqueue_subsurface(h);
            if (!rc) rc = enqueue_overland(h);
        }
        if (rc) return rc;
        if (want_grad) {
            CK(cudaMemcpyAsync(olf_H_all + (size_t)t * nc, P.H, nc * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(olf_h_all + (size_t)t * nc, P.h, nc * 8, cudaMemcpyDeviceToDevice, s));
        }
        LAUNCH(KT_ADJOINT, launch_adj_loss(P, A, t, -1, s));
    }
    CK(cudaMemcpyAsync(loss, A.loss, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    rc = check_device_error(h);
    if (rc || !want_grad) return rc;

    // the final state and diagnostics, restored after the reverse sweep
    rc = copy_state(h, ckpt[nseg], false, 0);
    if (rc) return rc;
    CK(cudaMemcpyAsync(final_H, P.H, nc * 8, cudaMemcpyDeviceToDevice, s));
    DevDiag diag_final;
    CK(cudaMemcpyAsync(&diag_final, &P.diag[0], sizeof(DevDiag), cudaMemcpyDeviceToHost, s));
    for (double *q : {A.psibar_next, A.thbar_next, A.g_lk, A.g_al, A.g_n}) CK(cudaMemsetAsync(q, 0, np * 8, s));
    for (double *q : {A.ktopbar_next, A.phbar}) CK(cudaMemsetAsync(q, 0, nc * 8, s));

    std::vector<int> iters(S);
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * K, t1 = std::min(t0 + K, nsteps), ns = t1 - t0;
        if (seg != nseg - 1) {
            // recompute the segment from its checkpoint, recording the tape
            rc = copy_state(h, ckpt[seg], true, t0);
            if (rc) return rc;
            for (int sl = 0; sl < ns; ++sl) {
                rc = taped_step(t0, sl, false);
                if (rc) return rc;
            }
        }
        CK(cudaMemcpyAsync(iters.data(), A.t_iters, ns * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        rc = check_device_error(h);
        if (rc) return rc;
        // reverse through the segment
        for (int sl = ns - 1; sl >= 0; --sl) {
            const int t = t0 + sl;
            A.step_in_seg = sl;
            CK(cudaMemcpyAsync(P.psin, A.t_psin + sl * np, np * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(P.thetan, A.t_thetan + sl * np, np * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(P.ktop, A.t_ktop + sl * nc, nc * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(P.ph, A.t_ph + sl * nc, nc * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(&P.pctrl[0].step, &h->adj_step_host[t], sizeof(int), cudaMemcpyHostToDevice, s));
            LAUNCH(KT_PROLOGUE, launch_prologue(P, s));
            // overland
            CK(cudaMemcpyAsync(P.h, A.t_hin + sl * nc, nc * 8, cudaMemcpyDeviceToDevice, s));
            LAUNCH(KT_OLF_AUX, launch_overland_setup(P, h->Ctot, s));
            LAUNCH(KT_ADJOINT, launch_adj_olf_rhs(P, A, t, s));
            LAUNCH(KT_OLF_SOLVE, launch_overland_solve(P, h->L, h->Ctot, s));
            LAUNCH(KT_ADJOINT, launch_adj_olf_coef(P, A, t, h->Ctot, s));
            LAUNCH(KT_ADJOINT, launch_adj_olf_finish(P, A, s));
            // subsurface
            const int Mi = iters[sl] < 1 ? 1 : (iters[sl] > M ? M : iters[sl]);
            LAUNCH(KT_ADJOINT, launch_adj_epilogue(P, A, sl, Mi, s));
            for (int m = Mi - 1; m >= 0; --m) {
                CK(cudaMemsetAsync(&P.gctrl->n_active, 0, 2 * sizeof(int), s));
                LAUNCH(KT_ADJOINT, launch_adj_matrix(P, A, sl, m, m == Mi - 1, h->mixed, s));
                LAUNCH(KT_KRYLOV, launch_krylov(P, h->L, s));
                LAUNCH(KT_ADJOINT, launch_adj_picard(P, A, sl, m, s));
            }
            LAUNCH(KT_ADJOINT, launch_adj_prologue(P, A, sl, s));
            std::swap(A.psibar_next, A.psinbar);
            std::swap(A.thbar_next, A.thnbar);
        }
    }
    LAUNCH(KT_ADJOINT, launch_adj_initial(P, A, s));
    CK(cudaStreamSynchronize(s));
    rc = check_device_error(h);
    if (rc) return rc;

    // gradients to the caller (pitched -> reference layout)
    const size_t row = (size_t)D.nx * 8, pitch = (size_t)D.nxp * 8;
    CK(cudaMemcpy2DAsync(grad_logks, row, A.g_lk + D.off3, pitch, row, (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpy2DAsync(grad_alpha, row, A.g_al + D.off3, pitch, row, (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpy2DAsync(grad_n, row, A.g_n + D.off3, pitch, row, (size_t)D.ny * D.nz, cudaMemcpyDeviceToHost, s));
    // restore the state after the forward run
    rc = copy_state(h, ckpt[nseg], true, nsteps);
    if (rc) return rc;
    CK(cudaMemcpyAsync(P.H, final_H, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(&P.diag[0], &diag_final, sizeof(DevDiag), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return DHARA_OK;
}

// ---------------------------------------------------------------- autotune
namespace {

struct SavedState {
    std::vector<void *> bufs;
    double *psin = nullptr, *thetan = nullptr, *ktop = nullptr, *ph = nullptr, *hh = nullptr, *H = nullptr;
    std::vector<PicardCtrl> pctrl;
    std::vector<DevDiag> diag;
    ~SavedState() {
        for (void *p : bufs) cudaFree(p);
    }
};

int save_state(dhara_handle *h, SavedState &st) {
    const size_t np = (size_t)h->Ntot, nc = (size_t)h->Ctot;
    for (double **q : {&st.psin, &st.thetan}) {
        if (cudaMalloc((void **)q, np * 8) != cudaSuccess) return fail(DHARA_ERR_NOMEM, "autotune: no memory");
        st.bufs.push_back(*q);
    }
    for (double **q : {&st.ktop, &st.ph, &st.hh, &st.H}) {
        if (cudaMalloc((void **)q, nc * 8) != cudaSuccess) return fail(DHARA_ERR_NOMEM, "autotune: no memory");
        st.bufs.push_back(*q);
    }
    const DevPtrs &P = h->P;
    cudaStream_t s = h->stream;
    CK(cudaMemcpyAsync(st.psin, P.psin, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st.thetan, P.thetan, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st.ktop, P.ktop, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st.ph, P.ph, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st.hh, P.h, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(st.H, P.H, nc * 8, cudaMemcpyDeviceToDevice, s));
    st.pctrl.resize(h->ndom);
    st.diag.resize(h->ndom);
    CK(cudaMemcpyAsync(st.pctrl.data(), P.pctrl, h->ndom * sizeof(PicardCtrl), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(st.diag.data(), P.diag, h->ndom * sizeof(DevDiag), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return DHARA_OK;
}

int restore_state(dhara_handle *h, const SavedState &st) {
    const size_t np = (size_t)h->Ntot, nc = (size_t)h->Ctot;
    const DevPtrs &P = h->P;
    cudaStream_t s = h->stream;
    CK(cudaMemcpyAsync(P.psin, st.psin, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.x, st.psin, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.psim, st.psin, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.thetan, st.thetan, np * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.ktop, st.ktop, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.ph, st.ph, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.h, st.hh, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.H, st.H, nc * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.pctrl, st.pctrl.data(), h->ndom * sizeof(PicardCtrl), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(P.diag, st.diag.data(), h->ndom * sizeof(DevDiag), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return DHARA_OK;
}

void fill_config(const dhara_handle *h, dhara_launch_config *out) {
    std::memset(out, 0, sizeof(*out));
    out->krylov_blocks_per_sm = h->L.krylov_per_sm;
    out->overland_resident = h->L.olf_allow_resident;
    out->overland_blocks_per_sm = h->L.olf_stream_per_sm;
    out->tile_shape = h->tile_mode;
    out->fused_step = h->L.fused_step;
}

}  // namespace

int dhara_get_launch_config(dhara_handle *h, dhara_launch_config *out) {
    if (!h || !out) return fail(DHARA_ERR_INVALID, "NULL argument");
    fill_config(h, out);
    return DHARA_OK;
}

int dhara_set_launch_config(dhara_handle *h, const dhara_launch_config *cfg) {
    if (!h || !cfg) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (cfg->krylov_blocks_per_sm < 1 || cfg->krylov_blocks_per_sm > h->L.krylov_per_sm_max ||
        cfg->overland_blocks_per_sm < 1 || cfg->overland_blocks_per_sm > h->L.olf_stream_per_sm_max)
        return fail(DHARA_ERR_INVALID, "blocks per SM must be in [1, %d] (Krylov) and [1, %d] (overland)",
                    h->L.krylov_per_sm_max, h->L.olf_stream_per_sm_max);
    if (cfg->tile_shape < 0 || cfg->tile_shape > 2)
        return fail(DHARA_ERR_INVALID, "tile_shape must be 0 (per domain), 1 (32 x 4) or 2 (16 x 8)");
    if (cfg->fused_step && h->L.step_per_sm < cfg->krylov_blocks_per_sm)
        return fail(DHARA_ERR_INVALID, "the fused step runs at most %d blocks per SM", h->L.step_per_sm);
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    if (cfg->tile_shape != h->tile_mode) {
        plan_tiles(h, cfg->tile_shape);
        const int rc = apply_tiles(h);
        if (rc) return rc;
    }
    h->L.krylov_per_sm = cfg->krylov_blocks_per_sm;
    h->L.fused_step = cfg->fused_step ? 1 : 0;
    h->L.olf_allow_resident = cfg->overland_resident ? 1 : 0;
    h->L.olf_stream_per_sm = cfg->overland_blocks_per_sm;
    if (h->graph_exec) {  // launch dimensions are baked into the graph
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    return DHARA_OK;
}

int dhara_autotune(dhara_handle *h, int trial_steps, dhara_launch_config *chosen) {
    if (!h) return fail(DHARA_ERR_INVALID, "NULL handle");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (trial_steps < 1) trial_steps = 1;
    if (set_dev(h)) return DHARA_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    SavedState st;
    int rc = save_state(h, st);
    if (rc) return rc;
    const bool timing_was = h->timing;
    double saved_ms[KT_N];
    long long saved_n[KT_N];
    collect_timing(h);
    std::memcpy(saved_ms, h->total_ms, sizeof(saved_ms));
    std::memcpy(saved_n, h->launches, sizeof(saved_n));
    const long long saved_count = h->launch_count;
    h->timing = true;
    // kind < 0: every kernel of the step
    auto timed_ms = [&](int kind) {
        if (kind >= 0) return h->total_ms[kind];
        double s = 0.0;
        for (int k = 0; k < KT_N; ++k) s += h->total_ms[k];
        return s;
    };
    auto trial = [&](int kind, double *ms) -> int {
        int r = restore_state(h, st);
        if (r) return r;
        collect_timing(h);
        const double before = timed_ms(kind);
        for (int t = 0; t < trial_steps && !r; ++t) {
            r = enqueue_subsurface(h);
            if (!r) r = enqueue_overland(h);
        }
        if (r) return r;
        CK(cudaStreamSynchronize(h->stream));
        r = check_device_error(h);
        if (r) return r;
        collect_timing(h);
        *ms = (timed_ms(kind) - before) / trial_steps;
        return DHARA_OK;
    };
    LaunchCfg &L = h->L;
    L.fused_step = 0;  // the stages below time kernels by name
    // tile shape: the whole step's time (every 3D kernel works on the tiles);
    // plans that come out the same for every domain are timed once
    {
        const int mode0 = h->tile_mode;
        int best_mode = mode0;
        double best_ms = 1e300;
        std::vector<std::vector<int>> seen;
        for (int mode = 0; mode <= 2 && !rc; ++mode) {
            plan_tiles(h, mode);
            std::vector<int> shape;
            for (const DomainDesc &D : h->hdom) shape.push_back(D.tx);
            bool dup = false;
            for (const auto &s2 : seen) dup = dup || s2 == shape;
            if (dup) continue;
            seen.push_back(shape);
            rc = apply_tiles(h);
            double ms = 0;
            if (!rc) rc = trial(-1, &ms);
            if (!rc && ms < best_ms) { best_ms = ms; best_mode = mode; }
        }
        plan_tiles(h, rc ? mode0 : best_mode);
        const int r2 = apply_tiles(h);
        if (!rc) rc = r2;
    }
    // 3D Krylov: blocks per SM
    int best_k = L.krylov_per_sm;
    double best_kms = 1e300;
    for (int b = 1; b <= L.krylov_per_sm_max && !rc; ++b) {
        L.krylov_per_sm = b;
        double ms = 0;
        rc = trial(KT_KRYLOV, &ms);
        if (!rc && ms < best_kms) { best_kms = ms; best_k = b; }
    }
    L.krylov_per_sm = best_k;
    // overland (the Jacobi solver): resident (when the segments fit) or
    // streaming with b blocks per SM; the multigrid solve has one schedule
    int best_res = L.olf_allow_resident, best_ob = L.olf_stream_per_sm;
    double best_oms = 1e300;
    if (L.olf_mg && !rc) rc = trial(KT_OLF_SOLVE, &best_oms);
    if (!L.olf_mg && !rc && h->P.nseg <= L.olf_res_blocks) {
        L.olf_allow_resident = 1;
        double ms = 0;
        rc = trial(KT_OLF_SOLVE, &ms);
        if (!rc && ms < best_oms) { best_oms = ms; best_res = 1; }
    }
    for (int b = 1; b <= L.olf_stream_per_sm_max && !rc && !L.olf_mg; ++b) {
        L.olf_allow_resident = 0;
        L.olf_stream_per_sm = b;
        double ms = 0;
        rc = trial(KT_OLF_SOLVE, &ms);
        if (!rc && ms < best_oms) { best_oms = ms; best_res = 0; best_ob = b; }
    }
    L.olf_allow_resident = best_res;
    L.olf_stream_per_sm = best_ob;
    // one launch per subsurface step, or one per kernel: the whole step's time
    if (!rc && L.step_per_sm >= L.krylov_per_sm) {
        double ms_sep = 0, ms_fused = 0;
        L.fused_step = 0;
        rc = trial(-1, &ms_sep);
        if (!rc) {
            L.fused_step = 1;
            rc = trial(-1, &ms_fused);
        }
        L.fused_step = (!rc && ms_fused < ms_sep) ? 1 : 0;
    }
    h->timing = timing_was;
    const int rr = restore_state(h, st);
    std::memcpy(h->total_ms, saved_ms, sizeof(saved_ms));
    std::memcpy(h->launches, saved_n, sizeof(saved_n));
    h->launch_count = saved_count;
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    if (rc) return rc;
    if (rr) return rr;
    if (chosen) {
        fill_config(h, chosen);
        chosen->krylov_ms = best_kms;
        chosen->overland_ms = best_oms;
    }
    return DHARA_OK;
}

// ---------------------------------------------------------- checkpoint
namespace {

// Header of a checkpoint buffer; the arrays follow it in this order:
// psi^n, theta^n (Ntot doubles each, the handle's pitched layout), top-layer
// K, ponded depth, overland depth, overland elevation (Ctot doubles each),
// then ndom PicardCtrl and ndom DevDiag records.
struct CkptHeader {
    char magic[8];
    int32_t version, ndom;
    int64_t ntot, ctot;
    int32_t pctrl_bytes, diag_bytes;
};
constexpr int32_t CKPT_VERSION = 2;
constexpr int CKPT_DIM_INTS = 3;  // nx, ny, nz per domain, after the header

size_t ckpt_bytes(const dhara_handle *h) {
    return sizeof(CkptHeader) + (size_t)h->ndom * CKPT_DIM_INTS * sizeof(int32_t) +
           ((size_t)2 * h->Ntot + (size_t)4 * h->Ctot) * sizeof(double) +
           (size_t)h->ndom * (sizeof(PicardCtrl) + sizeof(DevDiag) + 2 * sizeof(int64_t));
}

// The device arrays of the checkpoint, in buffer order, with their lengths.
void ckpt_arrays(const dhara_handle *h, double *(&arr)[6], size_t (&len)[6]) {
    const DevPtrs &P = h->P;
    double *a[6] = {P.psin, P.thetan, P.ktop, P.ph, P.h, P.H};
    for (int i = 0; i < 6; ++i) {
        arr[i] = a[i];
        len[i] = (size_t)(i < 2 ? h->Ntot : h->Ctot);
    }
}

}  // namespace

int dhara_checkpoint_size(dhara_handle *h, int64_t *bytes) {
    if (!h || !bytes) return fail(DHARA_ERR_INVALID, "NULL argument");
    *bytes = (int64_t)ckpt_bytes(h);
    return DHARA_OK;
}

int dhara_checkpoint(dhara_handle *h, void *buf, int64_t bytes) {
    if (!h || !buf) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (bytes < (int64_t)ckpt_bytes(h))
        return fail(DHARA_ERR_INVALID, "checkpoint buffer of %lld bytes is smaller than %lld", (long long)bytes,
                    (long long)ckpt_bytes(h));
    if (set_dev(h)) return DHARA_ERR_CUDA;
    unsigned char *q = (unsigned char *)buf;
    CkptHeader hd{};
    std::memcpy(hd.magic, "DHARACK", 8);
    hd.version = CKPT_VERSION;
    hd.ndom = h->ndom;
    hd.ntot = h->Ntot;
    hd.ctot = h->Ctot;
    hd.pctrl_bytes = (int32_t)sizeof(PicardCtrl);
    hd.diag_bytes = (int32_t)sizeof(DevDiag);
    std::memcpy(q, &hd, sizeof(hd));
    q += sizeof(hd);
    for (int d = 0; d < h->ndom; ++d) {
        const int32_t dims[CKPT_DIM_INTS] = {h->hdom[d].nx, h->hdom[d].ny, h->hdom[d].nz};
        std::memcpy(q, dims, sizeof(dims));
        q += sizeof(dims);
    }
    double *arr[6];
    size_t len[6];
    ckpt_arrays(h, arr, len);
    cudaStream_t s = h->stream;
    for (int i = 0; i < 6; ++i) {
        CK(cudaMemcpyAsync(q, arr[i], len[i] * sizeof(double), cudaMemcpyDeviceToHost, s));
        q += len[i] * sizeof(double);
    }
    CK(cudaMemcpyAsync(q, h->P.pctrl, h->ndom * sizeof(PicardCtrl), cudaMemcpyDeviceToHost, s));
    q += h->ndom * sizeof(PicardCtrl);
    CK(cudaMemcpyAsync(q, h->P.diag, h->ndom * sizeof(DevDiag), cudaMemcpyDeviceToHost, s));
    q += h->ndom * sizeof(DevDiag);
    // the accepted sub-step and attempt counts (host side)
    for (int d = 0; d < h->ndom; ++d) {
        const int64_t c[2] = {h->substeps[d], h->attempts[d]};
        std::memcpy(q, c, sizeof(c));
        q += sizeof(c);
    }
    CK(cudaStreamSynchronize(s));
    return check_device_error(h);
}

int dhara_restore(dhara_handle *h, const void *buf, int64_t bytes) {
    if (!h || !buf) return fail(DHARA_ERR_INVALID, "NULL argument");
    if (!h->prepared) return fail(DHARA_ERR_STATE, "dhara_prepare has not been called");
    if (bytes < (int64_t)sizeof(CkptHeader)) return fail(DHARA_ERR_INVALID, "checkpoint buffer too small");
    const unsigned char *q = (const unsigned char *)buf;
    CkptHeader hd;
    std::memcpy(&hd, q, sizeof(hd));
    if (std::memcmp(hd.magic, "DHARACK", 8) != 0 || hd.version != CKPT_VERSION)
        return fail(DHARA_ERR_INVALID, "not a checkpoint of this library version");
    if (hd.ndom != h->ndom || hd.ntot != h->Ntot || hd.ctot != h->Ctot ||
        hd.pctrl_bytes != (int32_t)sizeof(PicardCtrl) || hd.diag_bytes != (int32_t)sizeof(DevDiag))
        return fail(DHARA_ERR_INVALID, "checkpoint of %d domains / %lld cells does not match this handle "
                    "(%d / %lld)", hd.ndom, (long long)hd.ntot, h->ndom, (long long)h->Ntot);
    if (bytes < (int64_t)ckpt_bytes(h))
        return fail(DHARA_ERR_INVALID, "checkpoint buffer of %lld bytes is smaller than %lld", (long long)bytes,
                    (long long)ckpt_bytes(h));
    q += sizeof(hd);
    for (int d = 0; d < h->ndom; ++d) {
        int32_t dims[CKPT_DIM_INTS];
        std::memcpy(dims, q, sizeof(dims));
        q += sizeof(dims);
        if (dims[0] != h->hdom[d].nx || dims[1] != h->hdom[d].ny || dims[2] != h->hdom[d].nz)
            return fail(DHARA_ERR_INVALID, "checkpoint domain %d is %dx%dx%d, the handle's is %dx%dx%d", d,
                        dims[0], dims[1], dims[2], h->hdom[d].nx, h->hdom[d].ny, h->hdom[d].nz);
    }
    if (set_dev(h)) return DHARA_ERR_CUDA;
    double *arr[6];
    size_t len[6];
    ckpt_arrays(h, arr, len);
    cudaStream_t s = h->stream;
    const DevPtrs &P = h->P;
    for (int i = 0; i < 6; ++i) {
        CK(cudaMemcpyAsync(arr[i], q, len[i] * sizeof(double), cudaMemcpyHostToDevice, s));
        q += len[i] * sizeof(double);
    }
    // the Krylov warm start and the Picard iterate of a step's first
    // iteration are psi^n
    CK(cudaMemcpyAsync(P.x, P.psin, (size_t)h->Ntot * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.psim, P.psin, (size_t)h->Ntot * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(P.pctrl, q, h->ndom * sizeof(PicardCtrl), cudaMemcpyHostToDevice, s));
    q += h->ndom * sizeof(PicardCtrl);
    CK(cudaMemcpyAsync(P.diag, q, h->ndom * sizeof(DevDiag), cudaMemcpyHostToDevice, s));
    q += h->ndom * sizeof(DevDiag);
    for (int d = 0; d < h->ndom; ++d) {
        int64_t c[2];
        std::memcpy(c, q, sizeof(c));
        q += sizeof(c);
        h->substeps[d] = c[0];
        h->attempts[d] = c[1];
    }
    CK(cudaStreamSynchronize(s));
    return DHARA_OK;
}
