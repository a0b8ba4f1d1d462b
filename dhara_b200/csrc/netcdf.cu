// netcdf.cu -- the reference's result files in NetCDF classic format
// (SaveModelResults, src/io.cc:854-906; SaveResultEntirePeriod's flow-model
// part, src/io.cc:962-996; the writers SaveOutput1D/2D/3D, src/io.cc:696-850),
// written by the library itself.  Host code only.
//
// The format is the published NetCDF classic specification (magic "CDF" and a
// version byte, then the dimension list, global attributes, variable list
// and the variables' big-endian data, every item padded to 4 bytes).  Version
// 1 (32-bit offsets) is what the reference's nc_create(path, NC_CLOBBER)
// makes; version 2 (64-bit offsets) is used when a variable would start
// beyond 2^31 - 1 bytes.  No netCDF library is needed or linked.
//
// File contents, as the reference defines them:
//   snapshot 2D: water_elevation, water_depth   dims ("x" = ny, "y" = nx)
//   snapshot 3D: pressure_head, moisture        dims ("z" = nz, "y" = ny, "x" = nx)
//   1D:          mb_subsurfaceW                 dim  ("time_series" = steps)
//   statistics:  pressure_mean, moisture_mean   dims ("x" = steps, "y" = nz)
// The 2D names follow SaveOutput2D, which calls the first (slower) dimension
// "x" and the second "y" whatever they hold; the data layout is the row-major
// [ny][nx] (or [steps][nz]) the reference writes.  pressure_mean and
// moisture_mean hold CopyLayers' per-layer sums (src/device.cu:135-147).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dhara_dropin.h"

int dhara_internal_fail(int code, const char *msg);  // api.cu

namespace {

struct NcDim {
    std::string name;
    uint32_t len;
};

struct NcVar {
    std::string name;
    std::vector<int> dims;  // indexes into the file's dimensions
    const double *data;     // row-major, product of the dimension lengths
};

class Buf {
public:
    std::vector<unsigned char> b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void name(const std::string &s) {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        while (b.size() % 4) b.push_back(0);
    }
};

uint64_t count_of(const NcVar &v, const std::vector<NcDim> &dims) {
    uint64_t n = 1;
    for (int d : v.dims) n *= dims[d].len;
    return n;
}

// The header with every variable's offset `begin` (data follow the header in order).
Buf header(const std::vector<NcDim> &dims, const std::vector<NcVar> &vars, bool offset64,
           const std::vector<uint64_t> &begin) {
    Buf h;
    h.b = {'C', 'D', 'F', (unsigned char)(offset64 ? 2 : 1)};
    h.u32(0);                // numrecs: no record variables
    h.u32(0x0A);             // NC_DIMENSION
    h.u32((uint32_t)dims.size());
    for (const NcDim &d : dims) {
        h.name(d.name);
        h.u32(d.len);
    }
    h.u32(0);                // global attributes: ABSENT
    h.u32(0);
    h.u32(0x0B);             // NC_VARIABLE
    h.u32((uint32_t)vars.size());
    for (size_t i = 0; i < vars.size(); ++i) {
        const NcVar &v = vars[i];
        h.name(v.name);
        h.u32((uint32_t)v.dims.size());
        for (int d : v.dims) h.u32((uint32_t)d);
        h.u32(0);            // variable attributes: ABSENT
        h.u32(0);
        h.u32(6);            // NC_DOUBLE
        const uint64_t vsize = count_of(v, dims) * 8;
        h.u32(vsize > 0xFFFFFFFCull ? 0xFFFFFFFFu : (uint32_t)vsize);
        if (offset64) h.u64(begin[i]);
        else h.u32((uint32_t)begin[i]);
    }
    return h;
}

int write_classic(const char *path, const std::vector<NcDim> &dims, const std::vector<NcVar> &vars) {
    // offsets depend on the header's size, which depends on the offset width
    bool offset64 = false;
    std::vector<uint64_t> begin(vars.size(), 0);
    for (int pass = 0; pass < 2; ++pass) {
        const size_t hsize = header(dims, vars, offset64, begin).b.size();
        uint64_t at = hsize;
        for (size_t i = 0; i < vars.size(); ++i) {
            begin[i] = at;
            at += count_of(vars[i], dims) * 8;
        }
        const bool need64 = !vars.empty() && begin.back() > 0x7FFFFFFFull;
        if (need64 == offset64) break;
        offset64 = need64;
    }
    const Buf h = header(dims, vars, offset64, begin);
    FILE *f = fopen(path, "wb");
    if (!f) {
        std::string m = std::string("cannot create NetCDF file ") + path;
        return dhara_internal_fail(DHARA_ERR_INVALID, m.c_str());
    }
    bool ok = fwrite(h.b.data(), 1, h.b.size(), f) == h.b.size();
    std::vector<unsigned char> chunk;
    for (size_t i = 0; ok && i < vars.size(); ++i) {
        const uint64_t n = count_of(vars[i], dims);
        const size_t CH = 1 << 16;
        for (uint64_t k0 = 0; ok && k0 < n; k0 += CH) {
            const size_t m = (size_t)std::min<uint64_t>(CH, n - k0);
            chunk.resize(m * 8);
            for (size_t k = 0; k < m; ++k) {
                uint64_t u;
                std::memcpy(&u, vars[i].data + k0 + k, 8);
                for (int s = 0; s < 8; ++s) chunk[k * 8 + s] = (unsigned char)(u >> (56 - 8 * s));
            }
            ok = fwrite(chunk.data(), 1, chunk.size(), f) == chunk.size();
        }
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        std::string m = std::string("cannot write NetCDF file ") + path;
        return dhara_internal_fail(DHARA_ERR_INVALID, m.c_str());
    }
    return DHARA_OK;
}

}  // namespace

extern "C" int dhara_write_netcdf_state(const char *file2d, const char *file3d, int nx, int ny, int nz,
                                        const double *water_elevation, const double *water_depth,
                                        const double *pressure_head, const double *moisture) {
    if (nx < 1 || ny < 1 || nz < 1) return dhara_internal_fail(DHARA_ERR_INVALID, "invalid grid size");
    if (file2d) {
        if (!water_elevation || !water_depth)
            return dhara_internal_fail(DHARA_ERR_INVALID, "NULL 2D array for a 2D file");
        const std::vector<NcDim> dims = {{"x", (uint32_t)ny}, {"y", (uint32_t)nx}};
        const int rc = write_classic(file2d, dims, {{"water_elevation", {0, 1}, water_elevation},
                                                    {"water_depth", {0, 1}, water_depth}});
        if (rc) return rc;
    }
    if (file3d) {
        if (!pressure_head || !moisture)
            return dhara_internal_fail(DHARA_ERR_INVALID, "NULL 3D array for a 3D file");
        const std::vector<NcDim> dims = {{"x", (uint32_t)nx}, {"y", (uint32_t)ny}, {"z", (uint32_t)nz}};
        const int rc = write_classic(file3d, dims, {{"pressure_head", {2, 1, 0}, pressure_head},
                                                    {"moisture", {2, 1, 0}, moisture}});
        if (rc) return rc;
    }
    return DHARA_OK;
}

extern "C" int dhara_write_netcdf_statistics(const char *file1d, const char *file_stat, int nsteps, int nz,
                                             const double *mb_subsurfaceW, const double *pressure_sum,
                                             const double *moisture_sum) {
    if (nsteps < 0 || nz < 1) return dhara_internal_fail(DHARA_ERR_INVALID, "invalid step count or nz");
    if (file1d) {
        if (!mb_subsurfaceW && nsteps) return dhara_internal_fail(DHARA_ERR_INVALID, "NULL mb_subsurfaceW");
        const int rc = write_classic(file1d, {{"time_series", (uint32_t)nsteps}},
                                     {{"mb_subsurfaceW", {0}, mb_subsurfaceW}});
        if (rc) return rc;
    }
    if (file_stat) {
        if ((!pressure_sum || !moisture_sum) && nsteps)
            return dhara_internal_fail(DHARA_ERR_INVALID, "NULL layer statistics");
        const std::vector<NcDim> dims = {{"x", (uint32_t)nsteps}, {"y", (uint32_t)nz}};
        const int rc = write_classic(file_stat, dims, {{"pressure_mean", {0, 1}, pressure_sum},
                                                       {"moisture_mean", {0, 1}, moisture_sum}});
        if (rc) return rc;
    }
    return DHARA_OK;
}

extern "C" int dhara_save_netcdf_state(dhara_handle *h, int domain, const char *file2d, const char *file3d) {
    dhara_params p;
    int rc = dhara_get_params(h, domain, &p);
    if (rc) return rc;
    const size_t C = (size_t)p.nx * p.ny, N = C * p.nz;
    std::vector<double> H, hd, psi, th;
    if (file2d) {
        H.resize(C);
        hd.resize(C);
        if ((rc = dhara_download(h, domain, DHARA_F_WATERELEV, H.data(), (int64_t)C))) return rc;
        if ((rc = dhara_download(h, domain, DHARA_F_WATERDEPTH, hd.data(), (int64_t)C))) return rc;
    }
    if (file3d) {
        psi.resize(N);
        th.resize(N);
        if ((rc = dhara_download(h, domain, DHARA_F_PSI, psi.data(), (int64_t)N))) return rc;
        if ((rc = dhara_download(h, domain, DHARA_F_THETA, th.data(), (int64_t)N))) return rc;
    }
    return dhara_write_netcdf_state(file2d, file3d, p.nx, p.ny, p.nz, H.data(), hd.data(), psi.data(), th.data());
}

extern "C" int dhara_save_netcdf_statistics(dhara_handle *h, int domain, const char *file1d, const char *file_stat) {
    dhara_params p;
    int rc = dhara_get_params(h, domain, &p);
    if (rc) return rc;
    int64_t n = 0;
    if ((rc = dhara_get_statistics(h, domain, &n, nullptr, nullptr, nullptr))) return rc;
    std::vector<double> mb((size_t)n), ps((size_t)n * p.nz), th((size_t)n * p.nz);
    if (n && (rc = dhara_get_statistics(h, domain, &n, mb.data(), ps.data(), th.data()))) return rc;
    return dhara_write_netcdf_statistics(file1d, file_stat, (int)n, p.nz, mb.data(), ps.data(), th.data());
}

// ---- the reference's entry points (include/dhara_dropin.h) ---------------------
void SaveModelResults(ProjectClass *project, OverlandFlowClass *overland_host, OverlandFlowClass *overland_dev,
                      SubsurfaceFlowClass *subsurface_host, SubsurfaceFlowClass *subsurface_dev, int3 globsize,
                      int timestep) {
    if (!project || project->saveinterval <= 0 || timestep % project->saveinterval != 0) return;
    const size_t C = (size_t)globsize.x * globsize.y, N = C * globsize.z;
    char f2[1024], f3[1024];
    int rc = DHARA_OK;
    if (project->saveolf && overland_host && overland_dev) {
        cudaMemcpy(overland_host->waterelev, overland_dev->waterelev, C * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(overland_host->waterdepth, overland_dev->waterdepth, C * sizeof(double), cudaMemcpyDeviceToHost);
        snprintf(f2, sizeof(f2), "%s/%s_%d.nc", project->folderoutput, project->olfoutput, timestep);
        rc = dhara_write_netcdf_state(f2, nullptr, globsize.x, globsize.y, globsize.z, overland_host->waterelev,
                                      overland_host->waterdepth, nullptr, nullptr);
    }
    if (!rc && project->savessf && subsurface_host && subsurface_dev) {
        cudaMemcpy(subsurface_host->psiout, subsurface_dev->psin, N * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(subsurface_host->thetaout, subsurface_dev->thetan, N * sizeof(double), cudaMemcpyDeviceToHost);
        snprintf(f3, sizeof(f3), "%s/%s_%d.nc", project->folderoutput, project->ssfoutput, timestep);
        rc = dhara_write_netcdf_state(nullptr, f3, globsize.x, globsize.y, globsize.z, nullptr, nullptr,
                                      subsurface_host->psiout, subsurface_host->thetaout);
    }
    if (rc) fprintf(stderr, "dhara SaveModelResults: %s (status %d)\n", dhara_last_error(), rc);
}

void SaveResultEntirePeriod(ProjectClass *project, SubsurfaceFlowClass *subsurface_host, int3 globsize) {
    if (!project || !subsurface_host || !project->savestat) return;
    char f1[1024], fs[1024];
    snprintf(f1, sizeof(f1), "%s/%s.nc", project->folderoutput, project->ssf1doutput);
    snprintf(fs, sizeof(fs), "%s/%s.nc", project->folderoutput, project->statoutput);
    const int rc = dhara_write_netcdf_statistics(f1, fs, project->num_steps, globsize.z,
                                                 subsurface_host->mb_subsurfaceW, subsurface_host->psi_col,
                                                 subsurface_host->theta_col);
    if (rc) fprintf(stderr, "dhara SaveResultEntirePeriod: %s (status %d)\n", dhara_last_error(), rc);
}
