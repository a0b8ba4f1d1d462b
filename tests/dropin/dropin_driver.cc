// A host program written the way the reference's own host code drives the
// flow model (src/device.cu:374-475, src/numerical.cc:38-192): it fills the
// reference's structs, allocates their device arrays with cudaMalloc, and
// calls SubsurfaceFlowModel and OverlandFlowModel once per step -- here
// through include/dhara_dropin.h and libdhara_b200.so.  Used by
// tests/test_dropin.py.
//
//   dropin_driver <dir> <nsteps>
// reads <dir>/params.bin (a dhara_params), psi.bin, ksat.bin, ztopo.bin,
// mann.bin, rain.bin (mm per step); writes out_psi.bin, out_theta.bin,
// out_ph.bin, out_H.bin, out_mb.bin.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "dhara_dropin.h"

static std::vector<double> load(const std::string &path, size_t n) {
    std::vector<double> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(double), n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path.c_str());
        exit(2);
    }
    fclose(f);
    return v;
}

static void save(const std::string &path, const std::vector<double> &v) {
    FILE *f = fopen(path.c_str(), "wb");
    fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
}

template <typename T>
static T *dev(size_t n, const T *host = nullptr) {
    T *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) exit(3);
    if (host) cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice);
    else cudaMemset(p, 0, n * sizeof(T));
    return p;
}

int main(int argc, char **argv) {
    if (argc < 3) return 1;
    const std::string dir = argv[1];
    const int nsteps = atoi(argv[2]);
    dhara_params cfg;
    {
        FILE *f = fopen((dir + "/params.bin").c_str(), "rb");
        if (!f || fread(&cfg, sizeof(cfg), 1, f) != 1) return 2;
        fclose(f);
    }
    const int3 g = make_int3(cfg.nx, cfg.ny, cfg.nz);
    const size_t N = (size_t)g.x * g.y * g.z, C = (size_t)g.x * g.y;
    const size_t WE = (size_t)g.z * g.y, SN = (size_t)g.z * g.x;
    const int procsize = 1;

    // host-side config, as LoadFlowModelConfig leaves it (src/io.cc:236-274)
    SubsurfaceFlowClass sh = {};
    OverlandFlowClass oh = {};
    sh.dx = cfg.dx; sh.dy = cfg.dy; sh.dz = cfg.dz; sh.dt = cfg.dt;
    sh.alpha = cfg.alpha / 100.0;  // ALPHA is given in 1/cm
    sh.poresize = cfg.n; sh.theta_s = cfg.theta_s; sh.theta_r = cfg.theta_r; sh.porosity = cfg.porosity;
    sh.Ss = cfg.Ss; sh.am = cfg.am; sh.airdry = cfg.airdry; sh.psimin = cfg.psimin;
    sh.maxiter = cfg.picard_maxiter; sh.picardmethod = 0; sh.tolerance_psi = cfg.picard_tol;
    oh.delta = cfg.delta; oh.hmin = cfg.hmin; oh.hcri = cfg.hcri; oh.K0 = cfg.K0;
    std::vector<double> mb(nsteps, 0.0);
    sh.mb_subsurfaceW = mb.data();

    dhara_params p;
    dhara_params_from_reference(&p, &sh, &oh, g);
    // solver controls that the reference hard-codes are taken from the test's config
    p.picard_rule = cfg.picard_rule;
    p.krylov_tol = cfg.krylov_tol; p.krylov_maxiter = cfg.krylov_maxiter;
    p.overland_tol = cfg.overland_tol; p.overland_maxiter = cfg.overland_maxiter;
    p.theta_update = cfg.theta_update; p.precision = cfg.precision;
    p.sec_p_mm2dt_p_m = cfg.sec_p_mm2dt_p_m;

    // device structs (src/numerical.cc:59-188)
    const std::vector<double> psi = load(dir + "/psi.bin", N), ksat = load(dir + "/ksat.bin", N);
    const std::vector<double> z = load(dir + "/ztopo.bin", C), mann = load(dir + "/mann.bin", C);
    const std::vector<double> rain = load(dir + "/rain.bin", nsteps);
    std::vector<int> ones_we(WE, 1), ones_sn(SN, 1), ones_c(C, 1), zeros_c(C, 0);
    std::vector<double> rda((size_t)procsize * g.z, 0.0);
    SubsurfaceFlowClass sd = {};
    OverlandFlowClass od = {};
    sd.bcw = dev(WE, ones_we.data()); sd.bce = dev(WE, ones_we.data());
    sd.bcs = dev(SN, ones_sn.data()); sd.bcn = dev(SN, ones_sn.data());
    sd.bcb = dev(C, ones_c.data()); sd.bct = dev(C, ones_c.data()); sd.procmap = dev(C, zeros_c.data());
    sd.bcqw = dev<double>(WE); sd.bcqe = dev<double>(WE); sd.bcqs = dev<double>(SN); sd.bcqn = dev<double>(SN);
    sd.bcqt = dev<double>(C); sd.bcqb = dev<double>(C);
    sd.ksat = dev(N, ksat.data()); sd.psin = dev(N, psi.data());
    sd.psinp1m = dev<double>(N); sd.psinp1mp1 = dev<double>(N); sd.thetan = dev<double>(N);
    sd.thetanp1m = dev<double>(N); sd.thetanp1mp1 = dev<double>(N); sd.knp1m = dev<double>(N);
    sd.cnp1m = dev<double>(N); sd.qss = dev<double>(C);
    sd.TR = dev<double>(C); sd.E_soil = dev<double>(C); sd.ppt_ground = dev<double>(C); sd.rda = dev(rda.size(), rda.data());
    std::vector<double> psiout(N), thetaout(N);
    sd.psiout = psiout.data(); sd.thetaout = thetaout.data();
    od.ztopo = dev(C, z.data()); od.mann = dev(C, mann.data()); od.waterdepth = dev<double>(C);
    od.waterelev = dev<double>(C); od.ph = dev<double>(C); od.hpoten = dev<double>(C);

    dhara_handle *solver = nullptr;
    if (dhara_create(&p, 1, 0, &solver) != DHARA_OK) {
        fprintf(stderr, "dhara_create: %s\n", dhara_last_error());
        return 4;
    }
    TimeForcingClass tf = {};
    TimeForcingClass *tfp = &tf;
    OverlandFlowClass *ohp = &oh, *odp = &od;
    SubsurfaceFlowClass *shp = &sh, *sdp = &sd;
    std::vector<double> ppt(C);
    for (int t = 0; t < nsteps; ++t) {
        // the forcing GatherFluxesDomain would scatter to the grid
        for (size_t c = 0; c < C; ++c) ppt[c] = rain[t];
        cudaMemcpy(sd.ppt_ground, ppt.data(), C * sizeof(double), cudaMemcpyHostToDevice);
        SubsurfaceFlowModel(tfp, ohp, odp, shp, sdp, solver, 0, procsize, g, t, nsteps);
        OverlandFlowModel(tfp, odp, sdp, solver, 0, procsize, g, t, nsteps);
    }
    std::vector<double> ph(C), H(C);
    cudaMemcpy(ph.data(), od.ph, C * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(H.data(), od.waterelev, C * sizeof(double), cudaMemcpyDeviceToHost);
    save(dir + "/out_psi.bin", psiout);
    save(dir + "/out_theta.bin", thetaout);
    save(dir + "/out_ph.bin", ph);
    save(dir + "/out_H.bin", H);
    save(dir + "/out_mb.bin", mb);
    // the reference's result files after the last step (SaveModelResults,
    // SaveResultEntirePeriod), from the structs as the reference's loop leaves them
    {
        ProjectClass proj = {};
        proj.folderoutput = dir.c_str();
        proj.olfoutput = "olf";
        proj.ssfoutput = "ssf";
        proj.ssf1doutput = "ssf1d";
        proj.statoutput = "stat";
        proj.saveolf = proj.savessf = proj.savestat = 1;
        proj.saveinterval = 1;
        proj.num_steps = nsteps;
        std::vector<double> elev(C), depth(C), psi_col((size_t)nsteps * g.z, 0.0), theta_col((size_t)nsteps * g.z, 0.0);
        std::vector<double> psi_host(N), theta_host(N);
        oh.waterelev = elev.data();
        oh.waterdepth = depth.data();
        // SaveModelResults copies into the host struct's psiout/thetaout
        // (src/io.cc:889-894), which the reference allocates beside the
        // device struct's (src/numerical.cc:38-192)
        sh.psiout = psi_host.data();
        sh.thetaout = theta_host.data();
        sh.psi_col = psi_col.data();
        sh.theta_col = theta_col.data();
        SaveModelResults(&proj, &oh, &od, &sh, &sd, g, nsteps);
        SaveResultEntirePeriod(&proj, &sh, g);
    }
    dhara_destroy(solver);
    printf("dropin ok\n");
    return 0;
}
