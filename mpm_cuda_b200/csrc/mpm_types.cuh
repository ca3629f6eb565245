// Device-side descriptors shared by the kernels and the C-ABI layer.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {

// material type values match the reference enum (Elasiticity.cuh:10-11)
enum : int { JELLO = 0, SNOW = 1, WATER = 2, SAND = 3 };
enum : int { BC_STICKY = 0, BC_SLIP = 1, BC_SEPARATE = 2 };
enum : unsigned { ERR_OUT_OF_GRID = 1u, ERR_NONFINITE = 2u, ERR_DET = 4u, ERR_BINNING = 8u, ERR_TIMEOUT = 16u,
                  ERR_POOL = 32u };

// One particle group: material + per-particle mass/volume (ParticleGroup,
// MPMSimulator.cuh:30-52; Material, Elasiticity.cuh:19-45).
struct GroupParams {
    int scene;
    int type;
    float mu, lambda;
    float xi, theta_c, theta_s;
    float bulk_k, gamma;
    float p_mass, p_vol;
    int surrogate;  // stress from the learned surrogate (MPM_STRESS_SURROGATE)
    float wave;     // signal speed of the material at rest: sqrt((lambda + 2 mu) / rho)
                    // for solids, sqrt(K gamma / rho) for water (adaptive dt)
};

// One scene's grid and integration constants (Grid, MPMSimulator.cuh:54-64).
struct SceneParams {
    int n[3];
    int dim;
    float h, inv_h;
    float origin[3];
    float dt;  // current substep (grid update, G2P, advection)
    float gravity[3];
    int bc_type;
    int bc_lo[3], bc_hi[3];  // per axis: node i is a wall node if i < bc_lo or i >= n - bc_hi
    float mass_eps;
    long long node_off;  // first node of the scene in the global grid arrays
    long long n_nodes;
    // 4^3 (or 4^2) node blocks: blocks per axis and first block index
    int nb[3];
    float dt_next;  // next substep: the fused pass's P2G for it (equal to dt unless adaptive)
    long long block_off;
    long long n_blocks;
    // adaptive dt (MPM_P2G_ATOMIC): dt_next = clamp(cfl h / max(|v| + wave), dt_min, dt_max)
    float dt_max, dt_min, cfl;
    int adaptive;
};

// Compact index of each present material in the binning's per-cell
// counters, which hold n slots of 64 cells per block.
struct MatSlots {
    int s[4];
    int n;
};

// Particle state: component planes of one FP32 buffer, plane stride `cap`.
//   planes [0, D)              x
//   planes [D, 2D)             v
//   planes [2D, 2D + D^2)      C (row-major)
//   planes [2D + D^2, 2D+2D^2) F (row-major)
//   plane  2D + 2D^2           aux: det Fp (snow) / J (water)
template <int D>
struct Planes {
    static constexpr int X = 0;
    static constexpr int V = D;
    static constexpr int C = 2 * D;
    static constexpr int F = 2 * D + D * D;
    static constexpr int AUX = 2 * D + 2 * D * D;
    static constexpr int COUNT = 2 * D + 2 * D * D + 1;
};

// Paged grid (mpm_options.grid_pool_blocks > 0).  The grid arrays hold a
// pool of `trash` physical 64-node blocks plus one trash block (index
// `trash`); page[v] is the physical block of virtual block v (the dense
// block index, scene block_off included) or `trash` when v has none.  Every
// address a kernel forms stays inside the pool: a block without a page reads
// as empty and writes land in the trash block, which nothing reads.
struct GridPages {
    int* page;        // [virtual blocks]
    int* slot_block;  // [trash]: virtual block of each physical block, -1 when free
    int* free_slots;  // stack of free physical blocks
    int* n_free;      // its height
    int trash;        // pool capacity = index of the trash block
};

struct ParticleBuf {
    float* s;          // COUNT planes
    long long cap;     // plane stride (elements)
    uint16_t* grp;     // group index per particle
    uint32_t* id;      // creation index per particle
};

}  // namespace mpm
