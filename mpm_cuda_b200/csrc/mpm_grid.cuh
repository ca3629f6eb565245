// Grid layout and the grid update.
//
// Each scene owns a dense grid stored in 64-node blocks: 4x4x4 nodes in 3D,
// 8x8 nodes in 2D.  A node is one float4: (momentum or velocity xyz, mass).
// Blocks of a scene are x-fastest; nodes inside a block are x-fastest.  The
// blocked order keeps a stencil, a shared-memory tile and a grid-update CTA
// on a few contiguous 1 KB runs.
#pragma once

#include <cmath>

#include "mpm_types.cuh"

namespace mpm {

template <int D>
struct BlockShape {
    static constexpr int SIDE = (D == 3) ? 4 : 8;
    static constexpr int SHIFT = (D == 3) ? 2 : 3;
    static constexpr int NODES = 64;
};

template <int D>
__device__ __forceinline__ long long node_index(const SceneParams& sc, int ix, int iy, int iz) {
    constexpr int S = BlockShape<D>::SHIFT;
    constexpr int M = BlockShape<D>::SIDE - 1;
    long long blk = (long long)(ix >> S) + (long long)sc.nb[0] * ((iy >> S) + (long long)sc.nb[1] * (iz >> S));
    int in = (ix & M) + BlockShape<D>::SIDE * ((iy & M) + BlockShape<D>::SIDE * (iz & M));
    return sc.node_off + blk * 64 + in;
}

// Node indices of a 3^D stencil, relative to the scene's first node.  The
// blocked index is separable per axis, so index(ox, oy, oz) = x[ox] + y[oy] +
// z[oz] (equal to node_index - node_off): 9 offsets computed once instead of
// the block/local split of 27 nodes.  A scene has fewer than 2^31 nodes
// (checked at creation), so the offsets are 32-bit.
template <int D>
struct StencilIndex {
    int x[3], y[3], z[3];
    __device__ __forceinline__ StencilIndex(const SceneParams& sc, const int* base) {
        constexpr int S = BlockShape<D>::SHIFT;
        constexpr int M = BlockShape<D>::SIDE - 1;
        constexpr int SIDE = BlockShape<D>::SIDE;
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            const int ix = base[0] + o, iy = base[1] + o;
            x[o] = (ix >> S) * 64 + (ix & M);
            y[o] = (iy >> S) * sc.nb[0] * 64 + (iy & M) * SIDE;
            if (D == 3) {
                const int iz = base[2] + o;
                z[o] = (iz >> S) * sc.nb[0] * sc.nb[1] * 64 + (iz & M) * SIDE * SIDE;
            } else {
                z[o] = 0;
            }
        }
    }
    __device__ __forceinline__ int operator()(int ox, int oy, int oz) const { return x[ox] + y[oy] + z[oz]; }
};

// ---------------------------------------------------------- paged grid --
//
// With PAGED = false every virtual block is its own physical block (the dense
// grid) and none of the page machinery is compiled in.

// physical block of virtual block v (trash when a paged block has no page;
// a page being claimed by a concurrent page-in reads as trash too, so every
// address formed from it stays inside the pool)
template <bool PAGED>
__device__ __forceinline__ long long phys_block(const GridPages& gp, long long v) {
    if constexpr (PAGED) return min(gp.page[v], gp.trash);
    else return v;
}

// Gives virtual block v a physical block if it has none: claims the page,
// pops a free block and clears its momentum and velocity.  Several threads
// of one kernel may ask for the same block; one claims it, the others see
// the claim and return.  Kernels launched later see the page.  An empty pool
// leaves v without a page and sets ERR_POOL.
__device__ __forceinline__ void page_in(const GridPages& gp, long long v, float4* grid_mom, float4* grid_vel,
                                        unsigned* err) {
    int* pv = gp.page + v;
    if (*pv != gp.trash) return;  // has a page, or another thread is claiming it
    if (atomicCAS(pv, gp.trash, gp.trash + 1) != gp.trash) return;
    const int t = atomicSub(gp.n_free, 1) - 1;
    if (t < 0) {
        atomicAdd(gp.n_free, 1);
        atomicExch(pv, gp.trash);
        atomicOr(err, ERR_POOL);
        return;
    }
    const int slot = gp.free_slots[t];
    gp.slot_block[slot] = (int)v;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; k < 64; ++k) {
        grid_mom[(long long)slot * 64 + k] = z;
        grid_vel[(long long)slot * 64 + k] = z;
    }
    atomicExch(pv, slot);
}

// virtual block of node (ix, iy, iz) of scene sc and the node's index in it
template <int D>
__device__ __forceinline__ long long virtual_block(const SceneParams& sc, int ix, int iy, int iz, int& in) {
    constexpr int S = BlockShape<D>::SHIFT;
    constexpr int M = BlockShape<D>::SIDE - 1;
    constexpr int SIDE = BlockShape<D>::SIDE;
    in = (ix & M) + SIDE * ((iy & M) + SIDE * (iz & M));
    return sc.block_off + (long long)(ix >> S) + (long long)sc.nb[0] * ((iy >> S) + (long long)sc.nb[1] * (iz >> S));
}

// index of node (ix, iy, iz) in the grid arrays (a node of a paged block
// without a page lands in the trash block)
template <int D, bool PAGED>
__device__ __forceinline__ long long grid_node(const SceneParams& sc, const GridPages& gp, int ix, int iy, int iz) {
    int in;
    const long long v = virtual_block<D>(sc, ix, iy, iz, in);
    return phys_block<PAGED>(gp, v) * 64 + in;
}

// value of node (ix, iy, iz); zero for a paged block without a page
template <int D, bool PAGED>
__device__ __forceinline__ float4 grid_read(const float4* g, const SceneParams& sc, const GridPages& gp, int ix, int iy,
                                            int iz) {
    int in;
    const long long v = virtual_block<D>(sc, ix, iy, iz, in);
    const long long b = phys_block<PAGED>(gp, v);
    if (PAGED && b >= gp.trash) return make_float4(0.f, 0.f, 0.f, 0.f);
    return g[b * 64 + in];
}

// Linear velocity layout.  The single-scene dense fused path keeps grid
// velocities x-fastest row by row (node (ix, iy, iz) at node_off + ix +
// n0 (iy + n1 iz)), so the fused kernel's window is one box of a tensor that
// the copy engine (TMA) loads whole; momentum keeps the blocked layout.  The
// scene's linear nodes fit in its blocked range (n0 n1 n2 <= 64 blocks).
template <int D>
__device__ __forceinline__ long long lin_node(const SceneParams& sc, int ix, int iy, int iz) {
    return sc.node_off + ix + (long long)sc.n[0] * (iy + (D == 3 ? (long long)sc.n[1] * iz : 0LL));
}

// scene owning global block `b` (binary search over block_off)
__device__ __forceinline__ int scene_of_block(const SceneParams* scenes, int n_scenes, long long b) {
    int lo = 0, hi = n_scenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (scenes[mid].block_off <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Grid update of one node (VelUpdate, MPMCUDA.cu:435-472): momentum to
// velocity when mass > mass_eps, gravity, wall boundary.  `g` holds
// (momentum, mass) on entry and (velocity, mass) on return.
template <int D>
__device__ __forceinline__ float4 grid_node_update(float4 g, const SceneParams& sc, int ix, int iy,
                                                   int iz) {
    const float m = g.w;
    if (!(m > sc.mass_eps)) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float im = 1.f / m;
    float v[3] = {fmaf(g.x, im, 0.f), fmaf(g.y, im, 0.f), fmaf(g.z, im, 0.f)};
#pragma unroll
    for (int a = 0; a < D; ++a) v[a] = fmaf(sc.dt, sc.gravity[a], v[a]);
    const int id[3] = {ix, iy, iz};
    bool lo[3], hi[3], any = false;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        lo[a] = id[a] < sc.bc_lo[a];
        hi[a] = id[a] >= sc.n[a] - sc.bc_hi[a];
        any |= lo[a] | hi[a];
    }
    if (sc.bc_type == BC_STICKY) {
        if (any) v[0] = v[1] = v[2] = 0.f;
    } else if (sc.bc_type == BC_SLIP) {
#pragma unroll
        for (int a = 0; a < D; ++a)
            if (lo[a] || hi[a]) v[a] = 0.f;
    } else {
#pragma unroll
        for (int a = 0; a < D; ++a) {
            if (lo[a] && v[a] < 0.f) v[a] = 0.f;
            if (hi[a] && v[a] > 0.f) v[a] = 0.f;
        }
    }
    if (D == 2) v[2] = 0.f;
    return make_float4(v[0], v[1], v[2], m);
}

// Wall thresholds of one axis (host): bc_lo / bc_hi as given, or, with
// ref_band > 0, the nodes the reference's FP64 position test marks
// (MPMCUDA.cu:462-469): node i sits at fma(i, h, origin) (the kernel's
// origin + i * h, contracted), the bounds are origin + band * h and
// (origin + h * n) - band * h, each operation rounded once as in the
// reference's host code (MPMCUDA.cu:845-850).  The marked nodes are a prefix
// and a suffix of the axis (positions increase with i).
inline void axis_walls(int n, double h, double origin, double ref_band, int bc_lo, int bc_hi, int& lo, int& hi) {
    if (!(ref_band > 0.0)) {
        lo = bc_lo;
        hi = bc_hi;
        return;
    }
    const volatile double bh = ref_band * h;  // volatile: no contraction into an FMA
    const volatile double nh = h * (double)n;
    const volatile double top = origin + nh;
    const double lower = origin + bh;
    const double upper = top - bh;
    lo = 0;
    while (lo < n && std::fma((double)lo, h, origin) <= lower) ++lo;
    hi = 0;
    while (hi < n && std::fma((double)(n - 1 - hi), h, origin) >= upper) ++hi;
}

// coordinates of node `in` (0..63) of block `blk` of scene `sc`
template <int D>
__device__ __forceinline__ void block_node_coords(const SceneParams& sc, long long blk, int in, int& ix,
                                                  int& iy, int& iz) {
    constexpr int S = BlockShape<D>::SIDE;
    // 32-bit division: a scene has fewer than 2^31 nodes, so fewer than 2^25 blocks
    const int lb = (int)blk;
    const int bx = lb % sc.nb[0];
    const int r = lb / sc.nb[0];
    const int by = r % sc.nb[1];
    const int bz = r / sc.nb[1];
    ix = bx * S + (in % S);
    iy = by * S + ((in / S) % S);
    iz = (D == 3) ? bz * S + in / (S * S) : 0;
}

}  // namespace mpm
