/*
 * dhara_dropin.h -- drop-in replacements for the reference's two flow entry
 * points, for host code written against the reference (src/device.cu's time
 * loop, RunCoupledFlowModel, src/device.cu:374-475).
 *
 *   reference                                      here
 *   SubsurfaceFlowModel(...)  src/subsurface.cu:686-694
 *   OverlandFlowModel(...)    src/overland.cu:387-390
 *
 * The signatures keep the reference's struct-pointer arguments, rank,
 * procsize, globsize, t and num_steps; the CUSP/Thrust containers they took
 * (cuspdev_diamat, cuspdev_1d, cuspdev_idoper, thrustdev..., include/
 * cusplib.h:26-30) are replaced by one solver handle that owns the linear
 * system storage.  The structs are the reference's (include/class.h:74-217),
 * declared here with the same members in the same order so the reference's
 * host code and this library agree on their layout; arrays in the *_dev
 * structs are device pointers allocated by the caller with the sizes of
 * src/numerical.cc:38-192, exactly as for the reference.
 *
 * Per call, SubsurfaceFlowModel reads the caller's device forcing
 * (subsurface_dev->ppt_ground, E_soil, TR) and writes back what the reference
 * leaves in the structs after a step: psin, thetan, psinp1m, psinp1mp1,
 * knp1m, cnp1m, thetanp1mp1, bcqt, bcqb, qss (subsurface_dev), ph, hpoten,
 * waterdepth (overland_dev), mb_subsurfaceW[t] (subsurface_host) and the host
 * copies psiout/thetaout.  OverlandFlowModel writes waterelev, waterdepth and
 * ph.  The first SubsurfaceFlowModel call on a handle loads the state from the
 * caller's device arrays (ksat, psin, ztopo, mann, waterdepth, ph, BC arrays,
 * procmap) and runs PreRunningFlowModel's closure evaluation.
 */
#ifndef DHARA_DROPIN_H
#define DHARA_DROPIN_H

#include <cuda_runtime.h>

#include "dhara_gpu.h"

#ifndef PROJECTCLASS_H
#define PROJECTCLASS_H
/* include/class.h:3-33: the output settings SaveModelResults and
 * SaveResultEntirePeriod read (SAVE_*, OUTPUT_* keys, src/io.cc:466-493). */
class ProjectClass {
  public:
    const char *name;
    const char *folderoutput;
    const char *mlcanoutput;
    const char *olfoutput;
    const char *ssfoutput;
    const char *ssf1doutput;
    const char *statoutput;

    int co2elevation;
    int numberofplants;
    int planttype;
    int savemlcan;
    int saveolf;
    int savessf;
    int savestat;
    int saveinterval;
    int printiterval;
    int num_steps;

    int verbose;
    int version;

    double co2concentration;
    double dtimehr;
    double dx_meter;
    double dy_meter;
    double dz_meter;
};
#endif

#ifndef TIMEFORCINGCLASS_H
#define TIMEFORCINGCLASS_H
class TimeForcingClass {
  public:
    int *doy;
    int *years;
    double *rg;
    double *pa;
    double *lwdn;
    double *zen;
    double *u;
    double *ppt;
    double *ta;
    double *ea;
    double *lai;
    double *vpd;
    double *decdoy;
    double *hour;
};
#endif

#ifndef OVERLANDFLOWCLASS_H
#define OVERLANDFLOWCLASS_H
class OverlandFlowClass {
  public:
    double *a2d;
    double *hpoten;
    double *ke;
    double *kn;
    double *ks;
    double *kw;
    double *mann;
    double *ph;
    double *rhs2d;
    double *qcapa;
    double *u;
    double *v;
    double *waterdepth;
    double *waterelev;
    double *ztopo;

    double delta;
    double dx;
    double dy;
    double dt;
    double hmin;
    double hcri;
    double K0;
    double hn;
    double hs;
    double hw;
    double he;
};
#endif

#ifndef SUBSURFACEFLOWCLASS_H
#define SUBSURFACEFLOWCLASS_H
class SubsurfaceFlowClass {
  public:
    int *bcb;
    int *bce;
    int *bcn;
    int *bcs;
    int *bct;
    int *bcw;
    int *type;
    int *procmap;

    double *bcpsib;
    double *bcpsie;
    double *bcpsin;
    double *bcpsis;
    double *bcpsit;
    double *bcpsiw;
    double *bcqb;
    double *bcqe;
    double *bcqn;
    double *bcqs;
    double *bcqt;
    double *bcqw;

    double *a3d;
    double *deltam;
    double *cnp1m;
    double *knp1m;
    double *ksat;
    double *psin;
    double *psinp1m;
    double *psinp1mp1;
    double *psiout;
    double *qss;
    double *rhs3d;
    double *thetan;
    double *thetanp1m;
    double *thetanp1mp1;
    double *thetaout;

    double *quflux;
    double *qdflux;
    double *qwflux;
    double *qeflux;
    double *qsflux;
    double *qnflux;
    double *dtheta;
    double *transp;
    double *evapo;
    double *ssflux;
    double *mb_subsurfaceW;

    double *TR;
    double *TR_root;
    double *ppt_ground;
    double *ppt_root;
    double *E_soil;
    double *E_soil_root;
    double *rda;
    double *psi_col;
    double *theta_col;

    int maxiter;
    int picardmethod;
    double alpha;
    double am;
    double airdry;
    double dx;
    double dy;
    double dz;
    double dt;
    double poresize;
    double porosity;
    double psimin;
    double Ss;
    double theta_s;
    double theta_r;
    double tolerance_psi;
    double tolerance_theta;
};
#endif

/* Parameters of a handle from the reference's host structs (the values
 * LoadFlowModelConfig reads, src/io.cc:236-274); alpha is converted from the
 * reference's 1/cm to 1/m.  Solver tolerances keep dhara_default_params. */
void dhara_params_from_reference(dhara_params *p, const SubsurfaceFlowClass *subsurface_host,
                                 const OverlandFlowClass *overland_host, int3 globsize);

void SubsurfaceFlowModel(TimeForcingClass *&timeforcings, OverlandFlowClass *&overland_host,
                         OverlandFlowClass *&overland_dev, SubsurfaceFlowClass *&subsurface_host,
                         SubsurfaceFlowClass *&subsurface_dev, dhara_handle *solver, int rank, int procsize,
                         int3 globsize, int t, int num_steps);

void OverlandFlowModel(TimeForcingClass *&timeforcings, OverlandFlowClass *&overland_dev,
                       SubsurfaceFlowClass *&subsurface_dev, dhara_handle *solver, int rank, int procsize,
                       int3 globsize, int t, int num_steps);

/* SaveModelResults (src/io.cc:854-906): every saveinterval steps, copies
 * waterelev/waterdepth (when saveolf) and psin/thetan (when savessf) from the
 * device structs into the host structs' arrays (waterelev, waterdepth,
 * psiout, thetaout) and writes <folderoutput>/<olfoutput>_<timestep>.nc and
 * <folderoutput>/<ssfoutput>_<timestep>.nc with the reference's variables
 * (dhara_write_netcdf_state). */
void SaveModelResults(ProjectClass *project, OverlandFlowClass *overland_host, OverlandFlowClass *overland_dev,
                      SubsurfaceFlowClass *subsurface_host, SubsurfaceFlowClass *subsurface_dev, int3 globsize,
                      int timestep);

/* The flow-model part of SaveResultEntirePeriod (src/io.cc:962-996; the
 * MLCan part and its MPI arguments are out of scope): when savestat, writes
 * <folderoutput>/<ssf1doutput>.nc (mb_subsurfaceW over num_steps) and
 * <folderoutput>/<statoutput>.nc (psi_col, theta_col as pressure_mean,
 * moisture_mean [num_steps][nz]) from the host struct. */
void SaveResultEntirePeriod(ProjectClass *project, SubsurfaceFlowClass *subsurface_host, int3 globsize);

#endif
