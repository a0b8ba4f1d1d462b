// config.cu -- the reference's configuration file onto dhara_params and the
// per-face boundary settings (host code only).
//
// Keys and their meaning follow LoadFlowModelConfig (src/io.cc:236-274) and
// the boundary section of src/host.cc:93-112; the file format follows
// ParserConfigFile (src/parser.cc:39-72): one "KEY = value" per line, '#'
// starting a comment line, surrounding blanks trimmed, first occurrence wins.
#include "../../include/dhara_gpu.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

int dhara_internal_fail(int code, const char *msg);  // api.cu

namespace {

std::string trim(const std::string &s) {
    const char *ws = " \t\r\n";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

bool read_config(const char *path, std::map<std::string, std::string> &kv) {
    FILE *f = fopen(path, "r");
    if (!f) return false;
    std::string line;
    char buf[4096];
    while (fgets(buf, sizeof(buf), f)) {
        line = buf;
        if (!line.empty() && line[0] == '#') continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = trim(line.substr(0, eq));
        if (key.empty() || kv.count(key)) continue;
        kv[key] = trim(line.substr(eq + 1));
    }
    fclose(f);
    return true;
}

}  // namespace

extern "C" int dhara_params_from_config(const char *path, int nx, int ny, int nz, dhara_params *p,
                                        dhara_config_bc *bc) {
    if (!path || !p) return dhara_internal_fail(DHARA_ERR_INVALID, "NULL path or params");
    std::map<std::string, std::string> kv;
    if (!read_config(path, kv)) return dhara_internal_fail(DHARA_ERR_INVALID, "cannot read the configuration file");
    // defaults, then the file on top (the reference's device constants,
    // include/devconst.h, are the defaults of dhara_default_params)
    dhara_default_params(p, nx, ny, nz, 1.2, 1.2, 0.2, 0.5);
    int found = 0;
    auto num = [&](const char *key, double &dst) {
        auto it = kv.find(key);
        if (it == kv.end()) return false;
        dst = strtod(it->second.c_str(), nullptr);
        ++found;
        return true;
    };
    auto inum = [&](const char *key, int &dst) {
        auto it = kv.find(key);
        if (it == kv.end()) return false;
        dst = (int)strtol(it->second.c_str(), nullptr, 10);
        ++found;
        return true;
    };
    int maxiter = p->picard_maxiter, method = 0;
    inum("MAXIMUM_ITERATIONS", maxiter);
    inum("PICARD_METHOD", method);
    p->picard_maxiter = maxiter;
    p->picard_rule = method == 1 ? DHARA_PICARD_THETA_RELATIVE : DHARA_PICARD_PSI_RELATIVE;
    double tol_psi = p->picard_tol, tol_theta = p->picard_tol;
    num("TOLERANCE_PRESSURE", tol_psi);
    num("TOLERANCE_THETA", tol_theta);
    p->picard_tol = method == 1 ? tol_theta : tol_psi;
    num("DRY_AIR_PRESSURE", p->airdry);
    num("MINIMUM_PRESSURE_HEAD", p->psimin);
    num("WEIGHTED_SCHEME", p->am);
    double alpha_cm = p->alpha / 100.0;
    if (num("ALPHA", alpha_cm)) p->alpha = alpha_cm * 100.0;
    num("PORE_SIZE_DISTRIBUTION", p->n);
    num("POROSITY", p->porosity);
    num("SPECIFIC_STORAGE", p->Ss);
    num("RESIDUAL_WATER_CONTENT", p->theta_r);
    num("SATURATED_WATER_CONTENT", p->theta_s);
    if (num("TIME_STEP_DATA", p->dt)) p->sec_p_mm2dt_p_m = p->dt * 3600.0 / 1000.0;
    num("GRID_SIZE.DX", p->dx);
    num("GRID_SIZE.DY", p->dy);
    num("GRID_SIZE.DZ", p->dz);
    num("DELTA", p->delta);
    num("WATERDEPTH_MINIMUM", p->hmin);
    num("WATERDEPTH_CRITICAL", p->hcri);
    num("KZERO", p->K0);
    if (bc) {
        std::memset(bc, 0, sizeof(*bc));
        const char *types[6] = {"BOUNDARY_TYPE_TOP", "BOUNDARY_TYPE_BOTTOM", "BOUNDARY_TYPE_NORTH",
                                "BOUNDARY_TYPE_SOUTH", "BOUNDARY_TYPE_EAST", "BOUNDARY_TYPE_WEST"};
        // src/host.cc:101-114 reads the *_BOTTOM values into the top face and
        // the *_TOP values into the bottom face
        const char *psis[6] = {"PRESSURE_HEAD_BOTTOM", "PRESSURE_HEAD_TOP", "PRESSURE_HEAD_NORTH",
                               "PRESSURE_HEAD_SOUTH", "PRESSURE_HEAD_EAST", "PRESSURE_HEAD_WEST"};
        const char *fluxes[6] = {"FLUX_BOTTOM", "FLUX_TOP", "FLUX_NORTH", "FLUX_SOUTH", "FLUX_EAST", "FLUX_WEST"};
        for (int f = 0; f < 6; ++f) {
            int t = 1;
            inum(types[f], t);
            bc->type[f] = t;
            num(psis[f], bc->psi[f]);
            num(fluxes[f], bc->flux[f]);
        }
    }
    if (bc) bc->found = found;
    return DHARA_OK;
}

extern "C" int dhara_apply_boundary_config(dhara_handle *h, int domain, const dhara_config_bc *bc) {
    if (!h || !bc) return dhara_internal_fail(DHARA_ERR_INVALID, "NULL handle or boundary settings");
    dhara_params p;
    // the domain's grid: read back through the public field sizes
    int rc = dhara_get_params(h, domain, &p);
    if (rc) return rc;
    const int64_t C = (int64_t)p.nx * p.ny, WE = (int64_t)p.nz * p.ny, SN = (int64_t)p.nz * p.nx;
    struct Face {
        int type_field, psi_field, q_field;
        int64_t n;
    } faces[6] = {{DHARA_FI_BCT, -1, -1, C},
                  {DHARA_FI_BCB, DHARA_F_BCPSIB, DHARA_F_BCQB, C},
                  {DHARA_FI_BCN, DHARA_F_BCPSIN, DHARA_F_BCQN, SN},
                  {DHARA_FI_BCS, DHARA_F_BCPSIS, DHARA_F_BCQS, SN},
                  {DHARA_FI_BCE, DHARA_F_BCPSIE, DHARA_F_BCQE, WE},
                  {DHARA_FI_BCW, DHARA_F_BCPSIW, DHARA_F_BCQW, WE}};
    for (int f = 0; f < 6; ++f) {
        std::vector<int32_t> t((size_t)faces[f].n, bc->type[f]);
        rc = dhara_upload_int(h, domain, faces[f].type_field, t.data(), faces[f].n);
        if (rc) return rc;
        if (faces[f].psi_field >= 0) {
            std::vector<double> v((size_t)faces[f].n, bc->psi[f]);
            rc = dhara_upload(h, domain, faces[f].psi_field, v.data(), faces[f].n);
            if (rc) return rc;
        }
        if (faces[f].q_field >= 0) {
            std::vector<double> v((size_t)faces[f].n, bc->flux[f]);
            rc = dhara_upload(h, domain, faces[f].q_field, v.data(), faces[f].n);
            if (rc) return rc;
        }
    }
    return DHARA_OK;
}
