// mpm_simulator.hpp -- the reference simulator's C++ interface over the C ABI.
//
// A header-only stand-in for the reference's MPMSimulator class
// (src/simulator/MPMSimulator.cuh:66-102), its ObjInitInfo (:19-27), Material /
// MaterialType (src/simulator/material/Elasiticity.cuh:10-45) and OutputBego
// (src/utilities/FilesIO.h:10), with the same names and signatures, so that
// the reference's main() (src/main.cpp:161-221) compiles against it.  Every
// call forwards to include/mpm_b200.h; errors throw std::runtime_error (the
// reference calls exit(1)).
//
// Seeding follows MPMSimulator.cpp:198-267: the object's model matrix is
// translate * scale * rotate (model.cpp:202-207), its world bounding box must
// lie inside the grid, and every grid cell of that box gets `ppc` uniformly
// jittered samples kept when they fall inside the object.  `objPath` is
//   "builtin:cube"      the cube [-0.5, 0.5]^3
//   "builtin:sphere"    the ball of radius 0.5 at the origin
//   "builtin:cylinder"  radius 0.5, height 1 along y, centred at the origin
//   anything else       a Wavefront .obj file (v / f records), closed mesh,
//                       inside test by ray-crossing parity (on the GPU)
// Differences from the reference: particle volume is h^3 / ppc (the reference
// assigns h^3, MPMSimulator.cpp:252,263; set Options::reference_volume to
// reproduce it); the samples are drawn on the GPU by mpm_seed from a seeded
// counter hash instead of rand(); positions are float on the device.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpm_b200.h"

// Elasiticity.cuh:10-11 (same enumerator values)
enum MaterialType { JELLO = MPM_JELLO, SNOW = MPM_SNOW, WATER = MPM_WATER, SAND = MPM_SAND };

// Elasiticity.cuh:19-45.  The constants the reference hard-codes in its
// kernels are public members with the reference's values as defaults.
class Material {
   private:
    double mYoungsModulus;
    double mPoissonRatio;

   public:
    double mLambda;
    double mMu;
    double mDensity;
    MaterialType mType;
    double mXi = 10.0;       // snow hardening (MPMCUDA.cu:344)
    double mThetaC = 8e-2;   // snow clamp below 1 (MPMCUDA.cu:658-660)
    double mThetaS = 2e-2;   // snow clamp above 1
    double mBulkK = 2.51;    // water pressure scale (MPMCUDA.cu:353)
    double mGamma = 7.0;     // water exponent

    Material() : mYoungsModulus(0.0), mPoissonRatio(0.0), mLambda(0.0), mMu(0.0), mDensity(0.0), mType(JELLO) {}

    Material(double iYM, double iPR, double iDensity, MaterialType iType) : mType(iType) {
        mYoungsModulus = iYM;
        mPoissonRatio = iPR;
        if (mYoungsModulus < 0) throw std::invalid_argument("Youngs Modulus is out of range.");
        if (mPoissonRatio < 0 || mPoissonRatio > 0.5) throw std::invalid_argument("Poison Ratio is out of range.");
        mMu = mYoungsModulus / (2 * (1 + mPoissonRatio));
        mLambda = mYoungsModulus * mPoissonRatio / ((1 + mPoissonRatio) * (1 - 2 * mPoissonRatio));
        mDensity = iDensity;
    }
    double youngsModulus() const { return mYoungsModulus; }
    double poissonRatio() const { return mPoissonRatio; }
};

namespace mpm_shim {

// float3 that also accepts glm::vec3 (anything indexable by [0..2])
struct vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
    vec3() = default;
    vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    template <class V, class = decltype(std::declval<const V&>()[0])>
    vec3(const V& v) : x((float)v[0]), y((float)v[1]), z((float)v[2]) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

struct Mat3 {
    double m[9];
};

// rotation by `deg` degrees about the (normalised) axis, Rodrigues' formula
inline Mat3 rotation(double deg, vec3 axis) {
    const double pi = 3.14159265358979323846;
    double ax = axis.x, ay = axis.y, az = axis.z;
    const double n = std::sqrt(ax * ax + ay * ay + az * az);
    Mat3 r{{1, 0, 0, 0, 1, 0, 0, 0, 1}};
    if (n == 0.0 || deg == 0.0) return r;
    ax /= n;
    ay /= n;
    az /= n;
    const double a = deg * pi / 180.0, c = std::cos(a), s = std::sin(a), t = 1.0 - c;
    r.m[0] = t * ax * ax + c;      r.m[1] = t * ax * ay - s * az; r.m[2] = t * ax * az + s * ay;
    r.m[3] = t * ax * ay + s * az; r.m[4] = t * ay * ay + c;      r.m[5] = t * ay * az - s * ax;
    r.m[6] = t * ax * az - s * ay; r.m[7] = t * ay * az + s * ax; r.m[8] = t * az * az + c;
    return r;
}

// closed triangle mesh (Wavefront .obj v / f records); its inside test runs
// on the GPU in mpm_seed
struct Mesh {
    std::vector<double> v;     // xyz
    std::vector<int> tri;      // 3 indices per triangle
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};

    static Mesh load_obj(const std::string& path) {
        std::ifstream f(path);
        if (!f) throw std::runtime_error("cannot open " + path);
        Mesh m;
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string tag;
            ss >> tag;
            if (tag == "v") {
                double a, b, c;
                ss >> a >> b >> c;
                m.v.insert(m.v.end(), {a, b, c});
            } else if (tag == "f") {
                std::vector<int> idx;
                std::string tok;
                while (ss >> tok) {
                    int k = std::stoi(tok.substr(0, tok.find('/')));
                    idx.push_back(k > 0 ? k - 1 : (int)(m.v.size() / 3) + k);
                }
                for (size_t j = 1; j + 1 < idx.size(); ++j) m.tri.insert(m.tri.end(), {idx[0], idx[j], idx[j + 1]});
            }
        }
        if (m.tri.empty()) throw std::runtime_error(path + ": no faces");
        for (size_t i = 0; i < m.v.size(); i += 3)
            for (int a = 0; a < 3; ++a) {
                m.lo[a] = std::min(m.lo[a], m.v[i + a]);
                m.hi[a] = std::max(m.hi[a], m.v[i + a]);
            }
        return m;
    }
};

}  // namespace mpm_shim

// MPMSimulator.cuh:19-27
struct ObjInitInfo {
    std::array<double, 3> initVel{};
    mpm_shim::vec3 initTranslation;
    mpm_shim::vec3 initRotationAxis{0.f, 1.f, 0.f};
    mpm_shim::vec3 initScale{1.f};
    float initRotationDegree = 0.f;
    std::string objPath;
    Material mMaterial;
};

// MPMSimulator.cuh:66-102
class MPMSimulator {
   public:
    struct Options {
        // wall band of the reference's VelUpdate: the normal component zeroed at
        // nodes within 10 h of a wall by its FP64 position test (MPMCUDA.cu:845-850,
        // 462-469); ref_band = 0 uses the node-count thresholds bc_lo / bc_hi
        int bc_type = MPM_BC_SLIP;
        double ref_band = 10.0;
        int bc_lo = 11, bc_hi = 10;
        double gravity_y = -9.8;           // MPMSimulator.cpp:186
        double mass_eps = 2.220446049250313e-16;  // MPMCUDA.cu:444
        bool reference_volume = false;     // particle volume h^3 as the reference seeds
        unsigned seed = 1234;              // jitter generator
        int p2g_mode = MPM_P2G_ATOMIC;
        int device = 0;
    };

    // the grid fields of the reference's Grid (MPMSimulator.cuh:54-64) that its
    // viewer reads (main.cpp:170-175); the grid arrays live on the device
    struct Grid {
        double h = 0.0;
        unsigned int nodeNumDimX = 0, nodeNumDimY = 0, nodeNumDimZ = 0;
        std::array<double, 3> originCorner{{0.0, 0.0, 0.0}};
    };

    double adp_dt;
    double current_time;
    int current_frame;
    Grid mGrid{};

    MPMSimulator(double gap, double dt, unsigned int nodeNumDimX, unsigned int nodeNumDimY,
                 unsigned int nodeNumDimZ, unsigned int particleNumPerCell,
                 std::vector<ObjInitInfo>& objInitInfoVec)
        : MPMSimulator(gap, dt, nodeNumDimX, nodeNumDimY, nodeNumDimZ, particleNumPerCell, objInitInfoVec,
                       Options()) {}

    MPMSimulator(double gap, double dt, unsigned int nx, unsigned int ny, unsigned int nz, unsigned int ppc,
                 std::vector<ObjInitInfo>& objs, const Options& opt)
        : adp_dt(dt), current_time(0.0), current_frame(0) {
        mGrid.h = gap;
        mGrid.nodeNumDimX = nx;
        mGrid.nodeNumDimY = ny;
        mGrid.nodeNumDimZ = nz;
        std::vector<std::vector<float>> pos(objs.size());
        std::vector<mpm_group_desc> groups(objs.size());
        const unsigned n[3] = {nx, ny, nz};
        for (size_t k = 0; k < objs.size(); ++k) {
            const ObjInitInfo& o = objs[k];
            seed_object(o, gap, n, ppc, opt.seed + (unsigned)k, opt.device, pos[k]);
            const Material& m = o.mMaterial;
            mpm_group_desc& g = groups[k];
            g = mpm_group_desc{};
            g.material.type = m.mType;
            g.material.E = m.youngsModulus();
            g.material.nu = m.poissonRatio();
            g.material.rho = m.mDensity;
            g.material.xi = m.mXi;
            g.material.theta_c = m.mThetaC;
            g.material.theta_s = m.mThetaS;
            g.material.bulk_k = m.mBulkK;
            g.material.gamma = m.mGamma;
            g.p_vol = opt.reference_volume ? gap * gap * gap : gap * gap * gap / ppc;
            g.p_mass = m.mDensity * g.p_vol;
            g.n = (int64_t)(pos[k].size() / 3);
            g.x = pos[k].data();
            for (int a = 0; a < 3; ++a) g.init_v[a] = o.initVel[a];
        }
        mpm_scene_desc sc{};
        sc.dim = 3;
        sc.n[0] = (int)nx;
        sc.n[1] = (int)ny;
        sc.n[2] = (int)nz;
        sc.h = gap;
        sc.dt = dt;
        sc.gravity[1] = opt.gravity_y;
        sc.bc_type = opt.bc_type;
        sc.bc_lo = opt.bc_lo;
        sc.bc_hi = opt.bc_hi;
        sc.ref_band = opt.ref_band;
        sc.mass_eps = opt.mass_eps;
        sc.n_groups = (int)groups.size();
        sc.groups = groups.data();
        mpm_options mo;
        mpm_default_options(&mo);
        mo.p2g_mode = opt.p2g_mode;
        mo.device = opt.device;
        check(mpm_create(&sc, 1, &mo, &h_), nullptr);
    }

    MPMSimulator(const MPMSimulator&) = delete;
    MPMSimulator& operator=(const MPMSimulator&) = delete;

    ~MPMSimulator() {
        if (h_) mpm_destroy(h_);
    }

    // MPMCUDA.cu:793-925: one substep of every particle group
    void step() {
        check(mpm_step(h_, 1), h_);
        ++current_frame;
        current_time += adp_dt;
    }

    int totalParticlesNum() {
        int64_t n = 0;
        check(mpm_num_particles(h_, -1, &n), h_);
        return (int)n;
    }

    // MPMSimulator.cpp:362-371: positions of every group, in group order
    void getGLParticlesPos(std::vector<float>& oPosVec) {
        oPosVec.resize((size_t)totalParticlesNum() * 3);
        check(mpm_get_positions(h_, 0, oPosVec.data(), oPosVec.size()), h_);
    }

    mpm_handle* handle() { return h_; }

   private:
    mpm_handle* h_ = nullptr;

    static void check(int rc, mpm_handle* h) {
        if (rc == MPM_OK) return;
        char buf[512];
        mpm_last_error(h, buf, sizeof(buf));
        throw std::runtime_error(std::string("mpm_b200: ") + buf);
    }

    // Seeds one object on the GPU (mpm_seed): the object's world bounding box
    // must lie inside the grid (the reference's checks, MPMSimulator.cpp:214-223)
    static void seed_object(const ObjInitInfo& o, double gap, const unsigned* n, unsigned ppc, unsigned seed,
                            int device, std::vector<float>& out) {
        using mpm_shim::Mesh;
        const mpm_shim::Mat3 R = mpm_shim::rotation(o.initRotationDegree, o.initRotationAxis);
        mpm_seed_object so{};
        for (int a = 0; a < 9; ++a) so.rotation[a] = R.m[a];
        so.scale[0] = o.initScale.x;
        so.scale[1] = o.initScale.y;
        so.scale[2] = o.initScale.z;
        so.translation[0] = o.initTranslation.x;
        so.translation[1] = o.initTranslation.y;
        so.translation[2] = o.initTranslation.z;
        Mesh mesh;
        std::vector<float> verts;
        std::vector<int32_t> tris;
        double llo[3] = {-0.5, -0.5, -0.5}, lhi[3] = {0.5, 0.5, 0.5};
        if (o.objPath == "builtin:cube") so.shape = MPM_SHAPE_CUBE;
        else if (o.objPath == "builtin:sphere") so.shape = MPM_SHAPE_SPHERE;
        else if (o.objPath == "builtin:cylinder") so.shape = MPM_SHAPE_CYLINDER;
        else {
            so.shape = MPM_SHAPE_MESH;
            mesh = Mesh::load_obj(o.objPath);
            verts.assign(mesh.v.begin(), mesh.v.end());
            tris.assign(mesh.tri.begin(), mesh.tri.end());
            so.vertices = verts.data();
            so.n_vertices = (int64_t)(verts.size() / 3);
            so.triangles = tris.data();
            so.n_triangles = (int64_t)(tris.size() / 3);
            for (int a = 0; a < 3; ++a) {
                llo[a] = mesh.lo[a];
                lhi[a] = mesh.hi[a];
            }
        }
        // world bounding box of the transformed local box (model.cpp:202-222)
        for (int a = 0; a < 3; ++a) {
            double lo = 1e300, hi = -1e300;
            for (int c = 0; c < 8; ++c) {
                const double p[3] = {(c & 1) ? lhi[0] : llo[0], (c & 2) ? lhi[1] : llo[1], (c & 4) ? lhi[2] : llo[2]};
                const double w = so.translation[a] +
                                 so.scale[a] * (R.m[a * 3] * p[0] + R.m[a * 3 + 1] * p[1] + R.m[a * 3 + 2] * p[2]);
                lo = std::min(lo, w);
                hi = std::max(hi, w);
            }
            if (lo < 0.0) throw std::runtime_error("ERROR: OBJ lower bound is smaller than grid's origin.");
            if (hi > (n[a] - 1) * gap) throw std::runtime_error("ERROR: OBJ upper bound is out of the grid.");
        }
        int64_t cnt = 0;
        check(mpm_seed(&so, 3, gap, nullptr, (int)ppc, seed, device, nullptr, 0, &cnt), nullptr);
        out.resize((size_t)cnt * 3);
        if (cnt > 0) check(mpm_seed(&so, 3, gap, nullptr, (int)ppc, seed, device, out.data(), out.size(), &cnt), nullptr);
    }
};

// FilesIO.h:10 -- writes positions (x y z per particle) as a .bgeo file
inline void OutputBego(const std::string& fileNamePath, const std::vector<float>& outPosData) {
    if (mpm_write_bgeo_positions(fileNamePath.c_str(), outPosData.data(), (int64_t)(outPosData.size() / 3)) != MPM_OK)
        throw std::runtime_error("OutputBego: cannot write " + fileNamePath);
}
