/*
 * Headless harness around the reference simulator's own substep -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * The reference's src/simulator/MPMCUDA.cu (kernels P2G, VelUpdate,
 * InterpolateAndMove and MPMSimulator::step(), MPMCUDA.cu:310-925) is
 * compiled unmodified from the reference tree by oracle/Makefile and linked
 * with this file.  The reference constructor (MPMSimulator.cpp:178-285)
 * cannot run headless: it loads .obj meshes through a class whose destructor
 * calls OpenGL (model.cpp:159-163) and needs mesh_query, which ships without
 * a Makefile.  This file therefore supplies its own definitions of
 * MPMSimulator::MPMSimulator / ~MPMSimulator that only set the scalar
 * members and allocate the FP64 grid, and a C API that appends particle
 * groups from caller arrays (pMass and pVol passed explicitly, which also
 * sidesteps the seeding's pVol = h^3 issue at MPMSimulator.cpp:252,263).
 *
 * Everything step() touches is laid out exactly as the reference's own
 * initParticles (MPMSimulator.cpp:10-120) would: FP64 AoS pos[3N], vel[3N],
 * Fe[9N], Fp[9N] (snow), J[N] (water), C[9N], dgDiff[N].
 */
#include "MPMSimulator.cuh"

#include <cuda_runtime.h>
#include <cstring>
#include <vector>

MPMSimulator::MPMSimulator(double gap, double dt, unsigned int nodeNumDimX,
                           unsigned int nodeNumDimY, unsigned int nodeNumDimZ,
                           unsigned int /*particleNumPerCell*/,
                           std::vector<ObjInitInfo>& /*objInitInfoVec*/) {
    max_dt = dt;
    adp_dt = dt;
    ext_gravity = -9.8; /* MPMSimulator.cpp:186 */
    current_frame = 0;
    current_time = 0.0;
    mGrid.h = gap;
    mGrid.nodeNumDimX = nodeNumDimX;
    mGrid.nodeNumDimY = nodeNumDimY;
    mGrid.nodeNumDimZ = nodeNumDimZ;
    mGrid.originCorner = {0.0, 0.0, 0.0};
    size_t G = size_t(nodeNumDimX) * nodeNumDimY * nodeNumDimZ;
    mGrid.massVecByteSize = G * sizeof(double);
    mGrid.velVecByteSize = G * 3 * sizeof(double);
    mGrid.nodeMassVec = nullptr;
    mGrid.nodeVelVec = nullptr;
    cudaMalloc((void**)&mGrid.nodeMassVec, mGrid.massVecByteSize);
    cudaMalloc((void**)&mGrid.nodeVelVec, mGrid.velVecByteSize);
}

MPMSimulator::~MPMSimulator() {
    cudaFree(mGrid.nodeMassVec);
    cudaFree(mGrid.nodeVelVec);
    for (auto& g : mParticlesGroupsVec) {
        cudaFree(g.pPosVecGRAM);
        cudaFree(g.pVelVecGRAM);
        cudaFree(g.pElasiticityDeformationGradientGRAM);
        cudaFree(g.pPlasiticityDeformationGradientGRAM);
        cudaFree(g.pAffineVelGRAM);
        cudaFree(g.pDeformationGradientDiffGRAM);
        cudaFree(g.pJVecGRAM);
    }
}

namespace {

int upload(double** dst, const double* src, size_t bytes) {
    if (cudaMalloc((void**)dst, bytes) != cudaSuccess) return -1;
    if (src) {
        if (cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    } else {
        if (cudaMemset(*dst, 0, bytes) != cudaSuccess) return -1;
    }
    return 0;
}

}  // namespace

extern "C" {

void* mpmref_create(double h, double dt, unsigned nx, unsigned ny, unsigned nz) {
    std::vector<ObjInitInfo> none;
    auto* sim = new MPMSimulator(h, dt, nx, ny, nz, 1, none);
    if (!sim->mGrid.nodeMassVec || !sim->mGrid.nodeVelVec) {
        delete sim;
        return nullptr;
    }
    return sim;
}

void mpmref_destroy(void* s) { delete static_cast<MPMSimulator*>(s); }

/* Appends one particle group.  type: 0 jello, 1 snow, 2 water.  Arrays are
 * FP64 AoS host arrays; Fp is read for snow, J for water. */
int mpmref_add_group(void* s, int type, double E, double nu, double rho, double p_mass,
                     double p_vol, unsigned n, const double* pos, const double* vel,
                     const double* F, const double* Fp, const double* J, const double* C) {
    auto* sim = static_cast<MPMSimulator*>(s);
    ParticleGroup pg{};
    pg.particleNum = n;
    pg.mParticleMass = p_mass;
    pg.mParticleVolume = p_vol;
    pg.mMaterial = Material(E, nu, rho, MaterialType(type));
    pg.particlePosVec.assign(pos, pos + 3 * size_t(n));
    pg.posVecByteSize = size_t(n) * 3 * sizeof(double);
    pg.velVecByteSize = size_t(n) * 3 * sizeof(double);
    pg.eDgVecByteSize = size_t(n) * 9 * sizeof(double);
    pg.affineVelVecByteSize = size_t(n) * 9 * sizeof(double);
    pg.dgDiffVecByteSize = size_t(n) * sizeof(double);
    pg.pDgVecByteSize = 0;
    pg.JVecByteSize = 0;
    pg.pPlasiticityDeformationGradientGRAM = nullptr;
    pg.pJVecGRAM = nullptr;
    int rc = 0;
    rc |= upload(&pg.pPosVecGRAM, pos, pg.posVecByteSize);
    rc |= upload(&pg.pVelVecGRAM, vel, pg.velVecByteSize);
    rc |= upload(&pg.pElasiticityDeformationGradientGRAM, F, pg.eDgVecByteSize);
    rc |= upload(&pg.pAffineVelGRAM, C, pg.affineVelVecByteSize);
    rc |= upload(&pg.pDeformationGradientDiffGRAM, nullptr, pg.dgDiffVecByteSize);
    if (type == SNOW) {
        pg.pDgVecByteSize = pg.eDgVecByteSize;
        rc |= upload(&pg.pPlasiticityDeformationGradientGRAM, Fp, pg.pDgVecByteSize);
    } else if (type == WATER) {
        pg.JVecByteSize = size_t(n) * sizeof(double);
        rc |= upload(&pg.pJVecGRAM, J, pg.JVecByteSize);
    }
    sim->mParticlesGroupsVec.push_back(pg);
    return rc;
}

/* Runs n reference substeps (MPMSimulator::step, unmodified). */
int mpmref_step(void* s, int n) {
    auto* sim = static_cast<MPMSimulator*>(s);
    for (int i = 0; i < n; ++i) sim->step();
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

/* Times n substeps with CUDA events on the default stream (the stream the
 * reference launches on); returns milliseconds in *ms. */
int mpmref_time_steps(void* s, int n, float* ms) {
    auto* sim = static_cast<MPMSimulator*>(s);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a, 0);
    for (int i = 0; i < n; ++i) sim->step();
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* Copies one group's FP64 state back.  Null pointers skip a field. */
int mpmref_get_group(void* s, int gidx, double* pos, double* vel, double* F, double* Fp,
                     double* J, double* C) {
    auto* sim = static_cast<MPMSimulator*>(s);
    if (gidx < 0 || gidx >= int(sim->mParticlesGroupsVec.size())) return -1;
    auto& g = sim->mParticlesGroupsVec[gidx];
    int rc = 0;
    auto get = [&](double* dst, const double* src, size_t bytes) {
        if (dst && src && bytes)
            rc |= cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
    };
    get(pos, g.pPosVecGRAM, g.posVecByteSize);
    get(vel, g.pVelVecGRAM, g.velVecByteSize);
    get(F, g.pElasiticityDeformationGradientGRAM, g.eDgVecByteSize);
    get(Fp, g.pPlasiticityDeformationGradientGRAM, g.pDgVecByteSize);
    get(J, g.pJVecGRAM, g.JVecByteSize);
    get(C, g.pAffineVelGRAM, g.affineVelVecByteSize);
    return rc;
}

/* Copies the grid (mass, and momentum/velocity as left by the last step). */
int mpmref_get_grid(void* s, double* mass, double* vel) {
    auto* sim = static_cast<MPMSimulator*>(s);
    int rc = 0;
    if (mass)
        rc |= cudaMemcpy(mass, sim->mGrid.nodeMassVec, sim->mGrid.massVecByteSize,
                         cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
    if (vel)
        rc |= cudaMemcpy(vel, sim->mGrid.nodeVelVec, sim->mGrid.velVecByteSize,
                         cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
    return rc;
}

}  // extern "C"
