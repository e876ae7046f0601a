// reference_caller.cpp -- a caller written the way the reference's system
// classes are: it declares the reference's types (Vector3 with its user-
// provided copy constructor, the polymorphic ForceExt objects, UniformGrid,
// partVoisine) and every extern "C" launcher with the signatures of the
// reference's headers (SphSystem.cuh, PciSphSystem.cuh, CudaSystem.cuh,
// System.cuh, UniformGrid.cuh, ForceExt.cuh, MarchingCube.cuh, common.cuh
// and the collision launchers), and links against libpsb.so alone.
//
//   reference_caller link            resolve every symbol and exit 0
//   reference_caller run in out      the first half of SPHSystem::update and
//                                    the surface extraction on the scene in
//                                    `in`, every output written to `out`
//
// Built and run by tests/test_compat_link.py (with -Wl,-z,now, so that a
// missing launcher fails the link or the start, never a later call).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <vector_types.h>

typedef unsigned int uint;

// ---- the reference's types ------------------------------------------------------------
class Vector3 {      // Vector3.h: one double e[3]; its copy constructor is user-provided
public:
    Vector3() { e[0] = 0; e[1] = 0; e[2] = 0; }
    Vector3(double e0, double e1, double e2) { e[0] = e0; e[1] = e1; e[2] = e2; }
    inline Vector3(const Vector3& v) { e[0] = v.e[0]; e[1] = v.e[1]; e[2] = v.e[2]; }
    double x() const { return e[0]; }
    double y() const { return e[1]; }
    double z() const { return e[2]; }
    double e[3];
};

class ForceExt {     // ForceExt.h
public:
    ForceExt() {}
    ~ForceExt() {}
    virtual void draw() = 0;
};

class ForceExt_Constante : public ForceExt {     // ForceExt_Constante.h
public:
    ForceExt_Constante(Vector3 d, float a) : direction(d), amplitude(a) {}
    void draw() {}
    Vector3 getDirection() { return direction; }
    float getAmplitude() { return amplitude; }
private:
    Vector3 direction;
    float amplitude;
};

class ForceExt_Periodic : public ForceExt {      // ForceExt_Periodic.h
public:
    ForceExt_Periodic(float a, float lam, float kk, float th, float ww, float ff, float ph, float t)
        : A(a), lambda(lam), k(kk), theta(th), w(ww), f(ff), phi(ph), time(t) {}
    void draw() {}
private:
    float A, lambda, k, theta, w, f, phi, time;
};

class ForceExt_Trochoide : public ForceExt_Periodic {     // ForceExt_Trochoide.h
public:
    using ForceExt_Periodic::ForceExt_Periodic;
};

typedef struct {     // SphKernel.cuh
    int* nbVoisines;
    int* listeVoisine;
} partVoisine;

typedef struct {     // UniformGrid.cuh
    float3 Min;
    float3 Max;
    float sizeCell;
    double l, h, d;
    int* indexParticles;
    int* nbParticles;
    double3* m_dPos;
    double* m_hPos;
    float* m_dIsoVal;
    float* m_hIsoVal;
    float* m_dIsoNorm;
    float* m_hIsoNorm;
    int nbCellsX;
    int nbCellsY;
    int nbCellsZ;
} UniformGrid;

struct cudaGraphicsResource;

// ---- the reference's launchers, as its headers declare them ----------------------------
extern "C" {
void createGrid(double xC, double yC, double zC, double length, double width, double depth, float sizeCell, UniformGrid* grid);
void reinitCells(UniformGrid* grid);
void _finalizeGrid(UniformGrid* grid);
void storeParticles(UniformGrid* grid, double* pos, unsigned int nbBodies);
void searchNeighbooring(double* pos, double* radius, UniformGrid* grid, double scale, partVoisine voisines, unsigned int nbBodies);
void evaluateIso_CUDA(double* posMC, uint nbCellsX_MC, uint nbCellsY_MC, uint nbCellsZ_MC, double scale,
                      UniformGrid* grid, double* pos, double* radius, uint nbBodies);
void computeNormales_Vertex_CUDA(double* posV, double* normales, float scale, uint nbV, UniformGrid* grid, double* pos,
                                 double* radius, double* mass, double* densities, uint nbBodies);
void displayGrid(UniformGrid* grid);
void integrateSPHSystem(double* velInterAv, double* velInterAp, double* oldPos, double* newPos, double* forces,
                        double* densities, double dt, int numBodies);
void interpolateSPHVelocities(double* velInterAv, double* velInterAp, double* oldVel, double* newVel, int numBodies);
void evaluate_densities_forces(double* pos, double* vel, double* mass, double* radius, double* densities, double* pressure,
                               double* normales, double* restDensities, double* viscosities, double* k, double* threshold,
                               double* surfaceTension, int numBodies, double* fPressure, double* fViscosity,
                               double* fSurface, double* forcesAccum, partVoisine voisines);
void pci_SPH_update(double* oldPos, double* pos, double* vel, double* velInterAv, double* velInterAp,
                    double* restore_oldPos, double* restore_pos, double* restore_velInterAv, double* restore_velInterAp,
                    double* mass, double* radius, double* density, double* restDensity, double* densityError,
                    double* pressure, double* k, double* viscosity, double* l, double* surfaceTension, double threshold,
                    partVoisine voisines, double* normales, double* forceViscosity, double* forceSurface,
                    double* forcePressure, double* forceAccum, float dt, uint nbBodies);
void interactionSystem(double* oldPos, double* oldVel, double* forces, double* interactionRadius, double* spring,
                       double* damping, double* shear, double* attraction, partVoisine voisines, int numBodies);
void integrateSystem(double* oldPos, double* newPos, double* oldVel, double* newVel, double* forces, double* mass,
                     double dt, int start, int numBodies);
void evaluate_ForceExt_Constante(uint nbBodies, double* accumForceBuffer, double* mass, ForceExt_Constante* FC);
void evaluate_ForceExt_Trochoide(uint nbBodies, double* oldPos, double* accumForceBuffer, double* mass,
                                 ForceExt_Trochoide* T);
void collisionSystem_Box_CUDA(double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                              int nbBodiesP, Vector3 Min, Vector3 Max, bool container, float elast);
void collisionPlan_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, Vector3 A, Vector3 B, Vector3 C,
                        Vector3 D, Vector3 N, float elast, float dt, int nbBodiesP);
void collisionSystem_Sphere_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle,
                                 float dt, int nbBodies, Vector3 origin, float radius, float elast, bool container);
void collisionCylinder_CUDA(double* newPos, double* newVel, float radiusParticle, float dt, int nbBodiesP,
                            Vector3 center, Vector3 direction, double radius, double length, float elast, bool container);
void collisionMesh_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                        uint nbFaces, float* fA, float* fB, float* fC, float* fN, float elast, int nbBodiesP);
void collisionSystem_Linear_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel,
                                                      double radiusParticle, float dt, uint nbBodiesP, double a,
                                                      double b, Vector3 Min, Vector3 Max, float elast);
void collisionSystem_Gaussian_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel,
                                                        double radiusParticle, float dt, uint nbBodiesP, double A,
                                                        double x0, double z0, double p1, double p2, Vector3 Min,
                                                        Vector3 Max, float elast);
void collisionSystem_Periodic_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel,
                                                        double radiusParticle, float dt, uint nbBodiesP, uint nbFunc,
                                                        double* A, double* k, double* theta, double* phi, Vector3 Min,
                                                        Vector3 Max, float elast);
void createGrid_MarchingCube_CUDA(Vector3 C, double l, double w, double d, float sizeCell, uint nbPosX, uint nbPosY,
                                  uint nbPosZ, double* grid, int* m_nbIndex);
void polygonize_MarchingCube_CUDA(double* grid, uint nbPosX, uint nbPosY, uint nbPosZ, double isoLevel, int* m_nbIndex,
                                  double* m_vertex, double* m_normales, int* m_index);
int getcudaEnabledDeviceCount();
bool cudaInit(int argc, char** argv);
void cudaGLInit(int argc, char** argv);
void allocateArray(void** devPtr, size_t size);
void freeArray(void* devPtr);
void threadSync();
void copyArrayToDevice(void* device, const void* host, int offset, int size);
void copyArrayDeviceToDevice(void* device, const void* host, int offset, int size);
void copyArrayFromDevice(void* host, const void* device, struct cudaGraphicsResource** cuda_vbo_resource, int size);
int iDivUp(int a, int b);
void computeGridSize(int blockSize, int& numBlocks, int& numThreads);
}

// Every launcher above, so that linking proves each one resolves.
static void* const kAll[] = {
    (void*)&createGrid, (void*)&reinitCells, (void*)&_finalizeGrid, (void*)&storeParticles, (void*)&searchNeighbooring,
    (void*)&evaluateIso_CUDA, (void*)&computeNormales_Vertex_CUDA, (void*)&displayGrid, (void*)&integrateSPHSystem,
    (void*)&interpolateSPHVelocities, (void*)&evaluate_densities_forces, (void*)&pci_SPH_update,
    (void*)&interactionSystem, (void*)&integrateSystem, (void*)&evaluate_ForceExt_Constante,
    (void*)&evaluate_ForceExt_Trochoide, (void*)&collisionSystem_Box_CUDA, (void*)&collisionPlan_CUDA,
    (void*)&collisionSystem_Sphere_CUDA, (void*)&collisionCylinder_CUDA, (void*)&collisionMesh_CUDA,
    (void*)&collisionSystem_Linear_HeightFieldCollision_CUDA, (void*)&collisionSystem_Gaussian_HeightFieldCollision_CUDA,
    (void*)&collisionSystem_Periodic_HeightFieldCollision_CUDA, (void*)&createGrid_MarchingCube_CUDA,
    (void*)&polygonize_MarchingCube_CUDA, (void*)&getcudaEnabledDeviceCount, (void*)&cudaInit, (void*)&cudaGLInit,
    (void*)&allocateArray, (void*)&freeArray, (void*)&threadSync, (void*)&copyArrayToDevice,
    (void*)&copyArrayDeviceToDevice, (void*)&copyArrayFromDevice, (void*)&iDivUp, (void*)&computeGridSize,
};

// ---- run: the scene file and the outputs -------------------------------------------------
struct Reader {
    FILE* f;
    template <class T> T get() { T v{}; if (std::fread(&v, sizeof(T), 1, f) != 1) std::exit(3); return v; }
    template <class T> std::vector<T> get(size_t n) {
        std::vector<T> v(n);
        if (n && std::fread(v.data(), sizeof(T), n, f) != n) std::exit(3);
        return v;
    }
};

struct Writer {
    FILE* f;
    template <class T> void put(const std::vector<T>& v) { std::fwrite(v.data(), sizeof(T), v.size(), f); }
    template <class T> void put(T v) { std::fwrite(&v, sizeof(T), 1, f); }
};

template <class T>
static T* dev(const std::vector<T>& h) {
    void* d = nullptr;
    allocateArray(&d, sizeof(T) * (h.size() ? h.size() : 1));
    if (h.size()) copyArrayToDevice(d, h.data(), 0, (int)(sizeof(T) * h.size()));
    return (T*)d;
}
template <class T>
static std::vector<T> host(const T* d, size_t n) {
    std::vector<T> h(n);
    if (n) copyArrayFromDevice(h.data(), d, nullptr, (int)(sizeof(T) * n));
    return h;
}

int main(int argc, char** argv) {
    if (argc >= 2 && !std::strcmp(argv[1], "link")) {
        std::printf("%zu launchers resolved\n", sizeof(kAll) / sizeof(kAll[0]));
        return 0;
    }
    if (argc < 4 || std::strcmp(argv[1], "run")) return 2;
    if (!cudaInit(argc, argv)) return 4;
    Reader in{std::fopen(argv[2], "rb")};
    if (!in.f) return 3;
    const int n = in.get<int32_t>();
    std::vector<double> pos = in.get<double>(3 * (size_t)n), vel = in.get<double>(3 * (size_t)n);
    const double h = in.get<double>(), m = in.get<double>(), rho0 = in.get<double>(), kk = in.get<double>(),
                 mu = in.get<double>(), l = in.get<double>(), sigma = in.get<double>();
    std::vector<double> gc = in.get<double>(3), gl = in.get<double>(3);
    const float cell = in.get<float>();
    std::vector<double> gdir = in.get<double>(3);
    const float gamp = in.get<float>();
    std::vector<float> tro = in.get<float>(8);
    std::vector<int32_t> mcn = in.get<int32_t>(3);
    std::vector<double> mcc = in.get<double>(3), mcl = in.get<double>(3);
    const float mccell = in.get<float>();
    const double scale = in.get<double>(), level = in.get<double>();
    std::vector<double> bmin = in.get<double>(3), bmax = in.get<double>(3);
    const float prad = in.get<float>(), dt = in.get<float>();
    std::fclose(in.f);

    const std::vector<double> ones(n, 1.0);
    auto scaled = [&](double v) { std::vector<double> a(ones); for (double& x : a) x *= v; return a; };
    double *d_pos = dev(pos), *d_vel = dev(vel), *d_mass = dev(scaled(m)), *d_rad = dev(scaled(h)),
           *d_rho0 = dev(scaled(rho0)), *d_k = dev(scaled(kk)), *d_mu = dev(scaled(mu)), *d_l = dev(scaled(l)),
           *d_sig = dev(scaled(sigma));
    const std::vector<double> z3(3 * (size_t)n, 0.0), z1(n, 0.0);
    double *d_rho = dev(z1), *d_p = dev(z1), *d_nrm = dev(z3), *d_fp = dev(z3), *d_fv = dev(z3), *d_fs = dev(z3),
           *d_acc = dev(z3);
    int *d_cnt = dev(std::vector<int>(n, 0)), *d_list = dev(std::vector<int>(200 * (size_t)n, 0));
    partVoisine v{d_cnt, d_list};
    Writer out{std::fopen(argv[3], "wb")};
    if (!out.f) return 3;

    // SPHSystem::update, first half (SphSystem.cpp:273-320): grid, lists,
    // densities and internal forces, the constant force with the density as mass
    UniformGrid grid{};
    createGrid(gc[0], gc[1], gc[2], gl[0], gl[1], gl[2], cell, &grid);
    reinitCells(&grid);
    storeParticles(&grid, d_pos, n);
    searchNeighbooring(d_pos, d_rad, &grid, 1.0, v, n);
    evaluate_densities_forces(d_pos, d_vel, d_mass, d_rad, d_rho, d_p, d_nrm, d_rho0, d_mu, d_k, d_l, d_sig, n, d_fp, d_fv,
                              d_fs, d_acc, v);
    out.put(host(d_cnt, n));
    for (double* a : {d_rho, d_p}) out.put(host(a, n));
    for (double* a : {d_fp, d_fv, d_fs, d_nrm, d_acc}) out.put(host(a, 3 * (size_t)n));
    ForceExt_Constante gravity(Vector3(gdir[0], gdir[1], gdir[2]), gamp);
    evaluate_ForceExt_Constante(n, d_acc, d_rho, &gravity);
    out.put(host(d_acc, 3 * (size_t)n));
    ForceExt_Trochoide wave(tro[0], tro[1], tro[2], tro[3], tro[4], tro[5], tro[6], tro[7]);
    double* d_tro = dev(z3);
    evaluate_ForceExt_Trochoide(n, d_pos, d_tro, d_mass, &wave);
    out.put(host(d_tro, 3 * (size_t)n));
    // the box, Vector3 bounds passed by value
    double *d_bx = dev(pos), *d_bv = dev(vel);
    collisionSystem_Box_CUDA(d_bx, d_bv, d_bv, prad, dt, n, Vector3(bmin[0], bmin[1], bmin[2]),
                             Vector3(bmax[0], bmax[1], bmax[2]), true, 0.f);
    out.put(host(d_bx, 3 * (size_t)n));
    out.put(host(d_bv, 3 * (size_t)n));

    // SurfaceSPH::extract (SurfaceSPH.cpp:29-110): node grid, iso field,
    // marching cubes, vertex normals
    const uint nx = mcn[0], ny = mcn[1], nz = mcn[2];
    const size_t nn = (size_t)nx * ny * nz;
    double* d_nodes = dev(std::vector<double>(4 * nn, 0.0));
    int* d_nb = dev(std::vector<int>(nn, 0));
    createGrid_MarchingCube_CUDA(Vector3(mcc[0], mcc[1], mcc[2]), mcl[0], mcl[1], mcl[2], mccell, nx, ny, nz, d_nodes, d_nb);
    evaluateIso_CUDA(d_nodes, nx, ny, nz, scale, &grid, d_pos, d_rad, n);
    out.put(host(d_nodes, 4 * nn));
    const size_t slots = 200;
    double* d_vert = dev(std::vector<double>(3 * slots * nn, 0.0));
    double* d_vnrm = dev(std::vector<double>(3 * slots * nn, 0.0));
    int* d_idx = dev(std::vector<int>(slots * nn, 0));
    polygonize_MarchingCube_CUDA(d_nodes, nx, ny, nz, level, d_nb, d_vert, d_vnrm, d_idx);
    std::vector<int> nb = host(d_nb, nn), idx = host(d_idx, slots * nn);
    std::vector<double> vert = host(d_vert, 3 * slots * nn);
    std::vector<double> verts;
    for (size_t c = 0; c < nn; ++c)
        for (int k = 0; k < nb[c]; ++k) {
            if (idx[c * slots + k] != k) return 5;
            for (int a = 0; a < 3; ++a) verts.push_back(vert[3 * (c * slots + k) + a]);
        }
    out.put(nb);
    const uint nv = (uint)(verts.size() / 3);
    double* d_v = dev(verts);
    double* d_vn = dev(std::vector<double>(verts.size(), 0.0));
    computeNormales_Vertex_CUDA(d_v, d_vn, 1.f, nv, &grid, d_pos, d_rad, d_mass, d_rho, n);
    out.put(verts);
    out.put(host(d_vn, verts.size()));
    // launch sizing and the device count, as the reference computes them
    int blocks = 0, threads = 0;
    computeGridSize(1000, blocks, threads);
    out.put((int32_t)blocks);
    out.put((int32_t)threads);
    out.put((int32_t)iDivUp(1000, 256));
    out.put((int32_t)(getcudaEnabledDeviceCount() > 0));
    std::fclose(out.f);
    threadSync();
    _finalizeGrid(&grid);
    return 0;
}
