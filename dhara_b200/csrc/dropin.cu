// dropin.cu -- the reference's SubsurfaceFlowModel / OverlandFlowModel entry
// points (src/subsurface.cu:686-847, src/overland.cu:387-419) over a solver
// handle, for host code written against the reference.  See
// include/dhara_dropin.h for what each call reads and writes.
#include "../../include/dhara_dropin.h"

#include <cstdio>
#include <mutex>
#include <set>
#include <vector>

namespace {

std::mutex g_bound_mutex;
std::set<dhara_handle *> g_bound;  // handles whose state was loaded from the structs

void report(const char *where, int rc) {
    if (rc) fprintf(stderr, "dhara %s: %s (status %d)\n", where, dhara_last_error(), rc);
}

// int32 face/column arrays: device -> host -> dhara_upload_int (validated).
int upload_int_from_device(dhara_handle *h, int field, const int *dsrc, size_t count) {
    if (!dsrc) return DHARA_OK;
    std::vector<int32_t> tmp(count);
    if (cudaMemcpy(tmp.data(), dsrc, count * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return DHARA_ERR_CUDA;
    return dhara_upload_int(h, 0, field, tmp.data(), (int64_t)count);
}

int bind_state(dhara_handle *h, OverlandFlowClass *od, SubsurfaceFlowClass *sd, int procsize, int3 g) {
    const size_t N = (size_t)g.x * g.y * g.z, C = (size_t)g.x * g.y;
    const size_t WE = (size_t)g.z * g.y, SN = (size_t)g.z * g.x;
    int rc = 0;
    if (sd->rda && procsize > 0) {
        std::vector<double> rda((size_t)procsize * g.z);
        if (cudaMemcpy(rda.data(), sd->rda, rda.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return DHARA_ERR_CUDA;
        rc = dhara_set_roots(h, 0, rda.data(), procsize);
        if (rc) return rc;
    }
    if ((rc = upload_int_from_device(h, DHARA_FI_PROCMAP, sd->procmap, C))) return rc;
    if ((rc = upload_int_from_device(h, DHARA_FI_BCW, sd->bcw, WE))) return rc;
    if ((rc = upload_int_from_device(h, DHARA_FI_BCE, sd->bce, WE))) return rc;
    if ((rc = upload_int_from_device(h, DHARA_FI_BCS, sd->bcs, SN))) return rc;
    if ((rc = upload_int_from_device(h, DHARA_FI_BCN, sd->bcn, SN))) return rc;
    if ((rc = upload_int_from_device(h, DHARA_FI_BCB, sd->bcb, C))) return rc;
    struct {
        int field;
        const double *src;
        size_t n;
    } items[] = {
        {DHARA_F_PSI, sd->psin, N},        {DHARA_F_KSAT, sd->ksat, N},     {DHARA_F_ZTOPO, od->ztopo, C},
        {DHARA_F_MANN, od->mann, C},       {DHARA_F_WATERDEPTH, od->waterdepth, C},
        {DHARA_F_PONDING, od->ph, C},      {DHARA_F_BCQW, sd->bcqw, WE},    {DHARA_F_BCQE, sd->bcqe, WE},
        {DHARA_F_BCQS, sd->bcqs, SN},      {DHARA_F_BCQN, sd->bcqn, SN},
    };
    for (auto &it : items)
        if (it.src && (rc = dhara_upload_device(h, 0, it.field, it.src, (int64_t)it.n))) return rc;
    return dhara_prepare(h);
}

int copy_out(dhara_handle *h, int field, double *ddst, size_t n) {
    return ddst ? dhara_download_device(h, 0, field, ddst, (int64_t)n) : DHARA_OK;
}

}  // namespace

// Called by dhara_destroy so a later handle at the same address starts unbound
// (not exported).
extern "C" __attribute__((visibility("hidden"))) void dhara_internal_forget(dhara_handle *h) {
    std::lock_guard<std::mutex> lock(g_bound_mutex);
    g_bound.erase(h);
}

void dhara_params_from_reference(dhara_params *p, const SubsurfaceFlowClass *sh, const OverlandFlowClass *oh,
                                 int3 g) {
    dhara_default_params(p, g.x, g.y, g.z, sh->dx, sh->dy, sh->dz, sh->dt);
    p->alpha = sh->alpha * 100.0;  // ALPHA is in 1/cm (src/global.cu:79-97)
    p->n = sh->poresize;
    p->theta_s = sh->theta_s;
    p->theta_r = sh->theta_r;
    p->porosity = sh->porosity;
    p->Ss = sh->Ss;
    p->airdry = sh->airdry;
    p->psimin = sh->psimin;
    p->am = sh->am;
    p->picard_maxiter = sh->maxiter;
    p->picard_rule = sh->picardmethod == 1 ? DHARA_PICARD_THETA_RELATIVE : DHARA_PICARD_PSI_RELATIVE;
    p->picard_tol = sh->picardmethod == 1 ? sh->tolerance_theta : sh->tolerance_psi;
    if (oh) {
        p->delta = oh->delta;
        p->hmin = oh->hmin;
        p->hcri = oh->hcri;
        p->K0 = oh->K0;
    }
}

void SubsurfaceFlowModel(TimeForcingClass *&timeforcings, OverlandFlowClass *&overland_host,
                         OverlandFlowClass *&overland_dev, SubsurfaceFlowClass *&subsurface_host,
                         SubsurfaceFlowClass *&subsurface_dev, dhara_handle *solver, int rank, int procsize,
                         int3 globsize, int t, int num_steps) {
    (void)timeforcings;
    (void)overland_host;
    (void)rank;
    (void)num_steps;
    dhara_handle *h = solver;
    OverlandFlowClass *od = overland_dev;
    SubsurfaceFlowClass *sd = subsurface_dev, *sh = subsurface_host;
    const size_t N = (size_t)globsize.x * globsize.y * globsize.z, C = (size_t)globsize.x * globsize.y;
    int rc = 0;
    {
        std::lock_guard<std::mutex> lock(g_bound_mutex);
        if (!g_bound.count(h)) {
            rc = bind_state(h, od, sd, procsize, globsize);
            report("SubsurfaceFlowModel (loading state)", rc);
            if (rc) return;
            g_bound.insert(h);
        }
    }
    // forcing gathered by the caller (GatherFluxesDomain, src/subsurface.cu:632-662)
    if (sd->ppt_ground && (rc = dhara_upload_device(h, 0, DHARA_F_PPT, sd->ppt_ground, (int64_t)C))) goto fail;
    if (sd->E_soil && (rc = dhara_upload_device(h, 0, DHARA_F_ESOIL, sd->E_soil, (int64_t)C))) goto fail;
    if (sd->TR && (rc = dhara_upload_device(h, 0, DHARA_F_TR, sd->TR, (int64_t)C))) goto fail;
    if ((rc = dhara_subsurface_step(h))) goto fail;
    // what the reference's structs hold after the step (src/subsurface.cu:833-846)
    if ((rc = copy_out(h, DHARA_F_PSI, sd->psin, N)) || (rc = copy_out(h, DHARA_F_PSI, sd->psinp1mp1, N)) ||
        (rc = copy_out(h, DHARA_F_PSI, sd->psinp1m, N)) || (rc = copy_out(h, DHARA_F_THETA, sd->thetan, N)) ||
        (rc = copy_out(h, DHARA_F_THETA, sd->thetanp1m, N)) ||
        (rc = copy_out(h, DHARA_F_THETA_NEW, sd->thetanp1mp1, N)) || (rc = copy_out(h, DHARA_F_K, sd->knp1m, N)) ||
        (rc = copy_out(h, DHARA_F_C, sd->cnp1m, N)) || (rc = copy_out(h, DHARA_F_QTOP, sd->bcqt, C)) ||
        (rc = copy_out(h, DHARA_F_QTOP, sd->qss, C)) || (rc = copy_out(h, DHARA_F_BCQB, sd->bcqb, C)) ||
        (rc = copy_out(h, DHARA_F_PONDING, od->ph, C)) || (rc = copy_out(h, DHARA_F_PONDING, od->waterdepth, C)) ||
        (rc = copy_out(h, DHARA_F_HPOTEN, od->hpoten, C)))
        goto fail;
    if (sh && sh->mb_subsurfaceW) {
        dhara_diagnostics dg;
        if ((rc = dhara_get_diagnostics(h, 0, &dg))) goto fail;
        sh->mb_subsurfaceW[t] = dg.mb_subsurface_last;
    }
    if (sd->psiout && (rc = dhara_download(h, 0, DHARA_F_PSI, sd->psiout, (int64_t)N))) goto fail;
    if (sd->thetaout && (rc = dhara_download(h, 0, DHARA_F_THETA, sd->thetaout, (int64_t)N))) goto fail;
    return;
fail:
    report("SubsurfaceFlowModel", rc);
}

void OverlandFlowModel(TimeForcingClass *&timeforcings, OverlandFlowClass *&overland_dev,
                       SubsurfaceFlowClass *&subsurface_dev, dhara_handle *solver, int rank, int procsize,
                       int3 globsize, int t, int num_steps) {
    (void)timeforcings;
    (void)subsurface_dev;
    (void)rank;
    (void)procsize;
    (void)t;
    (void)num_steps;
    dhara_handle *h = solver;
    OverlandFlowClass *od = overland_dev;
    const size_t C = (size_t)globsize.x * globsize.y;
    int rc = dhara_overland_step(h);
    if (!rc) rc = copy_out(h, DHARA_F_WATERELEV, od->waterelev, C);
    if (!rc) rc = copy_out(h, DHARA_F_WATERDEPTH, od->waterdepth, C);
    if (!rc) rc = copy_out(h, DHARA_F_WATERDEPTH, od->ph, C);
    report("OverlandFlowModel", rc);
}
