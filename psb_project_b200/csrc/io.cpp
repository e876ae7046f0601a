// io.cpp -- particle and surface file formats, and checkpoints.
//
// Writers for the formats the reference's front end exports, so files made
// here open wherever the reference's did:
//   * Txt particles (ParticleExporter_Txt.cpp:27-33): "SPH <n>", then one
//     "-p x y z -m m -d rho" line per particle;
//   * XML particles (ParticleExporter_XML.cpp:130-185): <Particles name dt
//     count>, a <Gravity X Y Z Amp/> element, and one <Particle> per
//     particle with the SPH attributes and <position>, <velocity>,
//     <velocityInterAv>, <velocityInterAp> and <color> children;
//   * Mitsuba grid volumes (_exportData, UniformGrid.cu:266-300): "VOL",
//     version 3, encoding 1 (float32), resolution, one channel, the bounding
//     box, then the values;
//   * Wavefront OBJ surfaces (SurfaceSPH::exportOBJ, SurfaceSPH.cpp:234-276).
// Numbers are written with 9 significant digits, enough to give back every
// float exactly; the reference's writers round to 6 (printf %f, %.5f).
// The array-level writers take host arrays; the psb_export_* calls download
// a context's state and call them. Checkpoints are this library's own
// binary format: the complete state a PCISPH or WCSPH step continues from.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "psb.h"

namespace {

struct File {
    FILE* f;
    explicit File(const char* path, const char* mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
    bool ok() const { return f != nullptr; }
};

// The state of a context in particle-id order, as doubles (what the
// reference's m_hPos[1], m_hVel[1], m_hVelInterAp hold) plus density and
// pressure.
struct Snapshot {
    psb_scene sc{};
    int32_t n = 0;
    int64_t steps = 0;
    std::vector<double> pos, vel, vel_half;
    std::vector<float> density, pressure;
};

int snapshot(psb_ctx* c, Snapshot& s) {
    int rc = psb_context_info(c, &s.sc, &s.n, &s.steps);
    if (rc != PSB_OK) return rc;
    if (s.n <= 0) return PSB_ESTATE;
    const size_t n = (size_t)s.n;
    s.pos.resize(3 * n);
    s.vel.resize(3 * n);
    s.vel_half.resize(3 * n);
    s.density.resize(n);
    s.pressure.resize(n);
    rc = psb_download_aos_f64(c, s.pos.data(), s.vel.data(), s.vel_half.data(), 0);
    if (rc != PSB_OK) return rc;
    return psb_download(c, nullptr, nullptr, nullptr, s.density.data(), s.pressure.data());
}

}  // namespace

extern "C" {

int psb_write_txt(const char* path, int32_t n, const double* pos, double mass, const float* density) {
    if (!path || n < 0 || (n > 0 && (!pos || !density))) return PSB_EINVAL;
    File f(path, "w");
    if (!f.ok()) return PSB_EINVAL;
    std::fprintf(f.f, "SPH %d\n", n);
    for (int32_t i = 0; i < n; ++i)
        std::fprintf(f.f, "-p %.9g %.9g %.9g -m %.9g -d %.9g\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mass,
                     (double)density[i]);
    return std::ferror(f.f) ? PSB_EINVAL : PSB_OK;
}

int psb_write_xml(const char* path, const psb_scene* sc, int32_t n, const double* pos, const double* vel,
                  const double* vel_half, const int32_t* nbr_count) {
    if (!path || !sc || n < 0 || (n > 0 && (!pos || !vel || !vel_half))) return PSB_EINVAL;
    File f(path, "w");
    if (!f.ok()) return PSB_EINVAL;
    const double g[3] = {sc->gravity[0], sc->gravity[1], sc->gravity[2]};
    const double amp = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const double dir[3] = {amp > 0 ? g[0] / amp : 0.0, amp > 0 ? g[1] / amp : 0.0, amp > 0 ? g[2] / amp : 0.0};
    std::fprintf(f.f, "<?xml version=\"1.0\" ?>\n");
    std::fprintf(f.f, "<Particles name=\"SPH System\" dt=\"%.9g\" count=\"%d\">\n", (double)sc->dt, n);
    std::fprintf(f.f, "    <Gravity X=\"%.9g\" Y=\"%.9g\" Z=\"%.9g\" Amp=\"%.9g\" />\n", dir[0], dir[1], dir[2], amp);
    for (int32_t i = 0; i < n; ++i) {
        const double* x = pos + 3 * i;
        const double* v = vel + 3 * i;
        const double* vp = vel_half + 3 * i;
        // the previous half-step velocity, from the interpolated v = (v- + v+)/2
        const double vm[3] = {2 * v[0] - vp[0], 2 * v[1] - vp[1], 2 * v[2] - vp[2]};
        std::fprintf(f.f,
                     "    <Particle index=\"%d\" mass=\"%.9g\" radius=\"%.9g\" kernelParticles=\"%d\" "
                     "interactionRadius=\"%.9g\" restDensity=\"%.9g\" gasStiffness=\"%.9g\" threshold=\"%.9g\" "
                     "surfaceTension=\"%.9g\" viscosity=\"%.9g\">\n",
                     i, sc->mass, (double)sc->particle_radius, nbr_count ? nbr_count[i] : 0, sc->h, sc->rho0, sc->k,
                     sc->l, sc->sigma, sc->mu);
        std::fprintf(f.f, "        <position X=\"%.9g\" Y=\"%.9g\" Z=\"%.9g\" />\n", x[0], x[1], x[2]);
        std::fprintf(f.f, "        <velocity X=\"%.9g\" Y=\"%.9g\" Z=\"%.9g\" />\n", v[0], v[1], v[2]);
        std::fprintf(f.f, "        <velocityInterAv X=\"%.9g\" Y=\"%.9g\" Z=\"%.9g\" />\n", vm[0], vm[1], vm[2]);
        std::fprintf(f.f, "        <velocityInterAp X=\"%.9g\" Y=\"%.9g\" Z=\"%.9g\" />\n", vp[0], vp[1], vp[2]);
        std::fprintf(f.f, "        <color X=\"0\" Y=\"0\" Z=\"1\" />\n");
        std::fprintf(f.f, "    </Particle>\n");
    }
    std::fprintf(f.f, "</Particles>\n");
    return std::ferror(f.f) ? PSB_EINVAL : PSB_OK;
}

int psb_write_vol(const char* path, const double* field, const int32_t dims[3], const float bmin[3],
                  const float bmax[3], int32_t reference_layout) {
    if (!path || !field || !dims || !bmin || !bmax || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return PSB_EINVAL;
    // The reference writes its grid's z resolution for all three axes and
    // loops x outermost, z innermost; that layout is only defined for a cube
    if (reference_layout && !(dims[0] == dims[1] && dims[1] == dims[2])) return PSB_EINVAL;
    File f(path, "wb");
    if (!f.ok()) return PSB_EINVAL;
    const char magic[3] = {'V', 'O', 'L'};
    const uint8_t version = 3;
    const uint32_t encoding = 1, channels = 1;
    const uint32_t res[3] = {(uint32_t)dims[0], (uint32_t)dims[1], (uint32_t)dims[2]};
    std::fwrite(magic, 1, 3, f.f);
    std::fwrite(&version, 1, 1, f.f);
    std::fwrite(&encoding, 4, 1, f.f);
    std::fwrite(res, 4, 3, f.f);
    std::fwrite(&channels, 4, 1, f.f);
    std::fwrite(bmin, 4, 3, f.f);
    std::fwrite(bmax, 4, 3, f.f);
    const size_t nx = (size_t)dims[0], ny = (size_t)dims[1], nz = (size_t)dims[2];
    std::vector<float> row(reference_layout ? nz : nx);
    if (!reference_layout) {     // Mitsuba's order: x fastest, then y, then z
        for (size_t k = 0; k < nz; ++k)
            for (size_t j = 0; j < ny; ++j) {
                for (size_t i = 0; i < nx; ++i) row[i] = (float)field[i + nx * (j + ny * k)];
                std::fwrite(row.data(), 4, nx, f.f);
            }
    } else {                     // the reference's loop order (UniformGrid.cu:290-297)
        for (size_t i = 0; i < nx; ++i)
            for (size_t j = 0; j < ny; ++j) {
                for (size_t k = 0; k < nz; ++k) row[k] = (float)field[i + nx * (j + ny * k)];
                std::fwrite(row.data(), 4, nz, f.f);
            }
    }
    return std::ferror(f.f) ? PSB_EINVAL : PSB_OK;
}

int psb_write_obj(const char* path, const float* vertices, int64_t n_vertices, const int32_t* triangles,
                  int64_t n_triangles) {
    if (!path || n_vertices < 0 || n_triangles < 0 || (n_vertices > 0 && !vertices) || (n_triangles > 0 && !triangles))
        return PSB_EINVAL;
    for (int64_t t = 0; t < 3 * n_triangles; ++t)
        if (triangles[t] < 0 || triangles[t] >= n_vertices) return PSB_EINVAL;
    // vertex normals: the area-weighted sum of the adjacent faces' normals
    std::vector<double> nrm(3 * (size_t)n_vertices, 0.0);
    for (int64_t t = 0; t < n_triangles; ++t) {
        const int32_t* q = triangles + 3 * t;
        const float* a = vertices + 3 * (size_t)q[0];
        const float* b = vertices + 3 * (size_t)q[1];
        const float* c = vertices + 3 * (size_t)q[2];
        const double u[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
        const double v[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
        const double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        for (int k = 0; k < 3; ++k)
            for (int e = 0; e < 3; ++e) nrm[3 * (size_t)q[k] + e] += cr[e];
    }
    File f(path, "w");
    if (!f.ok()) return PSB_EINVAL;
    std::fprintf(f.f, "# psb isosurface: %lld vertices, %lld triangles\n", (long long)n_vertices, (long long)n_triangles);
    std::fprintf(f.f, "o isosurface\n");
    for (int64_t i = 0; i < n_vertices; ++i)
        std::fprintf(f.f, "v %.9g %.9g %.9g\n", (double)vertices[3 * i], (double)vertices[3 * i + 1],
                     (double)vertices[3 * i + 2]);
    for (int64_t i = 0; i < n_vertices; ++i) {
        const double* m = &nrm[3 * (size_t)i];
        const double l = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        const double s = l > 0 ? 1.0 / l : 0.0;
        std::fprintf(f.f, "vn %.6f %.6f %.6f\n", m[0] * s, m[1] * s, m[2] * s);
    }
    std::fprintf(f.f, "s off\n");
    for (int64_t t = 0; t < n_triangles; ++t) {
        const long long a = triangles[3 * t] + 1LL, b = triangles[3 * t + 1] + 1LL, c = triangles[3 * t + 2] + 1LL;
        std::fprintf(f.f, "f %lld//%lld %lld//%lld %lld//%lld\n", a, a, b, b, c, c);
    }
    return std::ferror(f.f) ? PSB_EINVAL : PSB_OK;
}

int psb_export_txt(psb_ctx* c, const char* path) {
    Snapshot s;
    int rc = snapshot(c, s);
    if (rc != PSB_OK) return rc;
    return psb_write_txt(path, s.n, s.pos.data(), s.sc.mass, s.density.data());
}

int psb_export_xml(psb_ctx* c, const char* path) {
    Snapshot s;
    int rc = snapshot(c, s);
    if (rc != PSB_OK) return rc;
    std::vector<int32_t> nbr((size_t)s.n);
    if (psb_read_field(c, PSB_FIELD_NBR_COUNT, nbr.data(), sizeof(int32_t) * nbr.size()) != PSB_OK)
        std::fill(nbr.begin(), nbr.end(), 0);     // no lists built yet
    return psb_write_xml(path, &s.sc, s.n, s.pos.data(), s.vel.data(), s.vel_half.data(), nbr.data());
}

// ---- checkpoints -------------------------------------------------------------
// Layout (little-endian): 8-byte magic "PSBCHK01"; int32 version (1); the
// psb_scene the context was created with (bytes); int32 n; int64 steps
// taken; then float32 arrays in particle-id order: pos (3n), vel (3n),
// vel_half (3n), pressure (n), density (n). The carried pressure is part of
// the state: warm starts read it, and a checkpoint continues bit for bit.

static const char kMagic[8] = {'P', 'S', 'B', 'C', 'H', 'K', '0', '1'};

// Field by field (the struct has padding), every field but n_max.
static bool same_scene(const psb_scene& a, const psb_scene& b) {
    for (int i = 0; i < 3; ++i)
        if (a.box_min[i] != b.box_min[i] || a.box_max[i] != b.box_max[i] || a.grid_min[i] != b.grid_min[i] ||
            a.dims[i] != b.dims[i] || a.gravity[i] != b.gravity[i])
            return false;
    return a.cell == b.cell && a.h == b.h && a.mass == b.mass && a.rho0 == b.rho0 && a.k == b.k && a.mu == b.mu &&
           a.sigma == b.sigma && a.l == b.l && a.particle_radius == b.particle_radius && a.dt == b.dt &&
           a.profile == b.profile && a.method == b.method && a.min_iters == b.min_iters &&
           a.max_iters == b.max_iters && a.eta == b.eta && a.wall_k == b.wall_k && a.wall_c == b.wall_c &&
           a.nbr_cap == b.nbr_cap && a.warm_start == b.warm_start && a.spacing == b.spacing && a.skin == b.skin &&
           a.xsph == b.xsph && a.dem_spring == b.dem_spring && a.dem_damping == b.dem_damping &&
           a.dem_shear == b.dem_shear && a.dem_attraction == b.dem_attraction;
}

int psb_checkpoint_save(psb_ctx* c, const char* path) {
    if (!c || !path) return PSB_EINVAL;
    psb_scene sc{};
    int32_t n = 0;
    int64_t steps = 0;
    int rc = psb_context_info(c, &sc, &n, &steps);
    if (rc != PSB_OK) return rc;
    if (n <= 0) return PSB_ESTATE;
    std::vector<float> pos(3 * (size_t)n), vel(3 * (size_t)n), vh(3 * (size_t)n), p((size_t)n), rho((size_t)n);
    rc = psb_download(c, pos.data(), vel.data(), vh.data(), rho.data(), p.data());
    if (rc != PSB_OK) return rc;
    File f(path, "wb");
    if (!f.ok()) return PSB_EINVAL;
    const int32_t version = 1;
    std::fwrite(kMagic, 1, 8, f.f);
    std::fwrite(&version, 4, 1, f.f);
    std::fwrite(&sc, sizeof(sc), 1, f.f);
    std::fwrite(&n, 4, 1, f.f);
    std::fwrite(&steps, 8, 1, f.f);
    std::fwrite(pos.data(), 4, pos.size(), f.f);
    std::fwrite(vel.data(), 4, vel.size(), f.f);
    std::fwrite(vh.data(), 4, vh.size(), f.f);
    std::fwrite(p.data(), 4, p.size(), f.f);
    std::fwrite(rho.data(), 4, rho.size(), f.f);
    return std::ferror(f.f) ? PSB_EINVAL : PSB_OK;
}

int psb_checkpoint_load(psb_ctx* c, const char* path) {
    if (!c || !path) return PSB_EINVAL;
    File f(path, "rb");
    if (!f.ok()) return PSB_EINVAL;
    char magic[8];
    int32_t version = 0, n = 0;
    int64_t steps = 0;
    psb_scene sc{}, mine{};
    int32_t n_now = 0;
    int64_t steps_now = 0;
    if (std::fread(magic, 1, 8, f.f) != 8 || std::memcmp(magic, kMagic, 8) != 0) return PSB_EINVAL;
    if (std::fread(&version, 4, 1, f.f) != 1 || version != 1) return PSB_EINVAL;
    if (std::fread(&sc, sizeof(sc), 1, f.f) != 1) return PSB_EINVAL;
    if (std::fread(&n, 4, 1, f.f) != 1 || std::fread(&steps, 8, 1, f.f) != 1 || n <= 0) return PSB_EINVAL;
    int rc = psb_context_info(c, &mine, &n_now, &steps_now);
    if (rc != PSB_OK) return rc;
    // the same physics: every scene parameter but the capacity must agree
    if (!same_scene(sc, mine) || n > mine.n_max) return PSB_EINVAL;
    std::vector<float> pos(3 * (size_t)n), vel(3 * (size_t)n), vh(3 * (size_t)n), p((size_t)n), rho((size_t)n);
    if (std::fread(pos.data(), 4, pos.size(), f.f) != pos.size() || std::fread(vel.data(), 4, vel.size(), f.f) != vel.size() ||
        std::fread(vh.data(), 4, vh.size(), f.f) != vh.size() || std::fread(p.data(), 4, p.size(), f.f) != p.size() ||
        std::fread(rho.data(), 4, rho.size(), f.f) != rho.size())
        return PSB_EINVAL;
    rc = psb_upload(c, n, pos.data(), vel.data(), vh.data(), p.data());
    if (rc != PSB_OK) return rc;
    return psb_set_step_count(c, steps);
}

}  // extern "C"
