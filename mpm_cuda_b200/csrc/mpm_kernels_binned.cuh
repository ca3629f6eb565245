// Binned substep: particles ordered by home grid block, one fused kernel per
// substep and material that gathers (G2P) from a shared-memory window of the
// grid velocities, updates the particle, evaluates the stress and scatters
// (P2G) for the next substep with float4 reductions into global memory, and a
// grid update that visits only the blocks P2G touched.
//
// Home block: the 4x4x4 node block (8x8 in 2D) that holds a particle's base
// node at the last re-binning.  Inside a block the particles are ordered by
// (material, rank inside their cell, cell): a warp's 32 consecutive particles
// then sit in 32 different cells, so the 32 lanes of every scatter hit 32
// different nodes, and the window layout below puts the gather's nodes in
// different banks.  A chunk is up to CTA size x rounds particles of one block
// and one material, contiguous in the ordered state.  The window of a chunk is
// the node range [S b - 1, S b + S + 3) per axis (S = block side): it holds the
// stencil of every particle whose base node is within one node of the home
// block.  Particles that drifted further since the last re-binning use global
// memory directly, so results never depend on how stale the binning is.
#pragma once

#include <cuda.h>  // CUtensorMap

#include "mpm_config.cuh"
#include "mpm_grid.cuh"
#include "mpm_kernels_direct.cuh"
#include "mpm_particle.cuh"

namespace mpm {

constexpr int kMats = 3;        // JELLO, SNOW, WATER

struct Chunk {
    int block;  // global block index (scene block_off + local block)
    int start;  // first sorted particle
    int count;  // particles in this chunk
    int mat;    // material of every particle of the chunk
    int scene;  // scene of the block
    int o[3];   // window origin: the home block's first node minus one per axis
};

// Tile layout.  3D: window 8^3, stored densely (strides 1, 8, 64); 2D:
// window 12^2, stride 12 -- the layout a tensor-map box load writes (an XOR
// swizzle of x on odd y, against bank conflicts of the gather, measured no
// faster).
template <int D>
struct TileShape;

template <>
struct TileShape<3> {
    static constexpr int SIDE = 4;
    static constexpr int T = 8;
    static constexpr int N = 512;
    static constexpr int VY = 8, VZ = 64, VN = 512;
    static constexpr bool SWIZZLE = false;
};

template <>
struct TileShape<2> {
    static constexpr int SIDE = 8;
    static constexpr int T = 12;
    static constexpr int N = 144;
    static constexpr int VY = 12, VZ = 0, VN = 144;
    static constexpr bool SWIZZLE = false;
};

// ------------------------------------------------------------- binning --

template <int D>
__device__ __forceinline__ void home_of(const SceneParams& sc, const float* x, long long& blk, int& cell) {
    constexpr int S = BlockShape<D>::SHIFT;
    constexpr int M = BlockShape<D>::SIDE - 1;
    int b[3] = {0, 0, 0}, c[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const float gx = (x[a] - sc.origin[a]) * sc.inv_h;
        int base = isfinite(gx) ? (int)floorf(gx - 0.5f) : 0;
        base = min(max(base, 0), sc.n[a] - 3);
        b[a] = base >> S;
        c[a] = base & M;
    }
    blk = sc.block_off + (long long)b[0] + (long long)sc.nb[0] * (b[1] + (long long)sc.nb[1] * b[2]);
    cell = c[0] + BlockShape<D>::SIDE * (c[1] + BlockShape<D>::SIDE * c[2]);  // 0..63
}

// Binning by counting, without a sort.  The particles of each (home block,
// material) segment are ordered rank-major (first every cell's rank-0
// particle, cells ascending, then every rank-1 particle, and so on, so the
// lanes of a warp sit in distinct cells) or cell-major (cells ascending, a
// cell's particles together).

// Pass 1: home block b, cell c and material m of every particle, its rank
// among the particles of (b, m, c) and the size of segment (b, m).
// (PAGED: the cell counters of a block live at its physical block.)  The
// particles arrive in the last binning's order, so the lanes of a warp mostly
// share a segment, and in cell-major order (CELL_MAJOR) runs of lanes share a
// cell: those counter updates are aggregated per warp (one atomic per distinct
// counter, each lane's rank the group's base plus its place among the group's
// lanes).  In rank-major order the lanes sit in distinct cells and update
// their cell counters one by one.
template <int D, bool PAGED, bool CELL_MAJOR>
__global__ void __launch_bounds__(256) k_bin_count(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                   const SceneParams* __restrict__ scenes, MatSlots ms,
                                                   unsigned long long* __restrict__ key, int* __restrict__ rank,
                                                   int* __restrict__ cell_count, int* __restrict__ seg_count,
                                                   GridPages gp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x[a] = pb.s[(Planes<D>::X + a) * pb.cap + i];
    const GroupParams& g = groups[pb.grp[i]];
    const SceneParams& sc = scenes[g.scene];
    long long b;
    int c;
    home_of<D>(sc, x, b, c);
    const unsigned act = __activemask();  // the lanes with a particle (the rest returned above)
    const long long cell = (phys_block<PAGED>(gp, b) * ms.n + ms.s[g.type]) * 64 + c;
    if constexpr (CELL_MAJOR) {
        const unsigned lane_lt = (1u << (threadIdx.x & 31)) - 1u;
        const unsigned in_cell = __match_any_sync(act, cell);
        const int lead_c = __ffs(in_cell) - 1;
        int base = 0;
        if ((int)(threadIdx.x & 31) == lead_c) base = atomicAdd(&cell_count[cell], __popc(in_cell));
        rank[i] = __shfl_sync(in_cell, base, lead_c) + __popc(in_cell & lane_lt);
    } else {
        rank[i] = atomicAdd(&cell_count[cell], 1);
    }
    const long long seg = b * 4 + g.type;
    const unsigned in_seg = __match_any_sync(act, seg);
    if ((int)(threadIdx.x & 31) == __ffs(in_seg) - 1) atomicAdd(&seg_count[seg], __popc(in_seg));
    key[i] = ((unsigned long long)b << 8) | ((unsigned long long)g.type << 6) | (unsigned long long)c;
}

// Pass 2 (after the scan of the segment sizes): with n_c' the segment's cell
// counts, the slot of particle (r, c) in its segment is, rank-major,
//   sum over cells c' of min(n_c', r)   (particles of lower rank)
// + #{c' < c : n_c' > r}                (rank r in lower cells),
// and, cell-major, sum over c' < c of n_c' + r; the particle's state moves
// there (move_vc = 0: all but the v and C planes -- inside the substep loop
// the fused kernels never read them, they rewrite the v planes and rebuild
// both on demand).  Ranks are exact, so the slots are a permutation of the
// segment; a slot outside it (inconsistent counts) is reported, not written.
template <int D, bool PAGED, bool CELL_MAJOR>
__global__ void __launch_bounds__(256) k_bin_place(ParticleBuf src, ParticleBuf dst, long long n,
                                                   const unsigned long long* __restrict__ key,
                                                   const int* __restrict__ rank, const int* __restrict__ cell_count,
                                                   const int* __restrict__ seg_count,
                                                   const int* __restrict__ seg_start, MatSlots ms,
                                                   int move_vc, unsigned* __restrict__ err, GridPages gp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = key[i];
    const long long b = (long long)(k >> 8);
    const int m = (int)((k >> 6) & 3), c = (int)(k & 63);
    const int r = rank[i];
    const int4* cnt = reinterpret_cast<const int4*>(cell_count + (phys_block<PAGED>(gp, b) * ms.n + ms.s[m]) * 64);
    int off = CELL_MAJOR ? r : 0;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int4 v = cnt[q];
        const int nc[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if constexpr (CELL_MAJOR) off += (4 * q + t < c) ? nc[t] : 0;  // the cells below, then the rank
            else off += min(nc[t], r) + ((4 * q + t < c && nc[t] > r) ? 1 : 0);  // lower ranks, then rank r below c
        }
    }
    const int seg = (int)(b * 4 + m);
    if (off < 0 || off >= seg_count[seg]) {
        atomicOr(err, ERR_BINNING);
        return;
    }
    const long long j = (long long)seg_start[seg] + off;
#pragma unroll
    for (int p = 0; p < Planes<D>::COUNT; ++p)
        if (move_vc || p < Planes<D>::V || p >= Planes<D>::F) dst.s[p * dst.cap + j] = src.s[p * src.cap + i];
    dst.grp[j] = src.grp[i];
    dst.id[j] = src.id[i];
}

// window origin of a chunk's home block: one node below the block
template <int D>
__device__ __forceinline__ void tile_origin(const SceneParams& sc, long long lb, int* o) {
    constexpr int SIDE = TileShape<D>::SIDE;
    o[0] = (int)(lb % sc.nb[0]) * SIDE - 1;
    o[1] = (int)((lb / sc.nb[0]) % sc.nb[1]) * SIDE - 1;
    o[2] = (D == 3) ? (int)(lb / ((long long)sc.nb[0] * sc.nb[1])) * SIDE - 1 : 0;
}

// one chunk per `chunk` particles of every non-empty (block, material)
// segment, appended to that material's list, with its scene and window
// origin (the block's coordinates, divided out once here)
template <int D>
__global__ void __launch_bounds__(256) k_make_chunks(const int* __restrict__ seg_count,
                                                     const int* __restrict__ seg_start, long long n_segs,
                                                     Chunk* __restrict__ chunks, long long list_cap,
                                                     int* __restrict__ n_chunks, int chunk,
                                                     const SceneParams* __restrict__ scenes, int n_scenes,
                                                     unsigned* __restrict__ err) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_segs) return;
    const int c = seg_count[s];
    if (c == 0) return;
    const int mat = (int)(s & 3);
    const int nch = (c + chunk - 1) / chunk;
    const int at = atomicAdd(&n_chunks[mat], nch);
    if (at + nch > list_cap) {  // cannot happen with the list sized for the smallest chunk
        atomicOr(err, ERR_BINNING);
        return;
    }
    Chunk ch;
    ch.block = (int)(s >> 2);
    ch.mat = mat;
    ch.scene = scene_of_block(scenes, n_scenes, ch.block);
    const SceneParams& sc = scenes[ch.scene];
    tile_origin<D>(sc, ch.block - sc.block_off, ch.o);
    for (int j = 0; j < nch; ++j) {
        ch.start = seg_start[s] + j * chunk;
        ch.count = min(chunk, c - j * chunk);
        chunks[mat * list_cap + at + j] = ch;
    }
}

// zero the cell and segment counters that k_bin_count touched
template <bool PAGED>
__global__ void __launch_bounds__(256) k_bin_reset(const unsigned long long* __restrict__ key, long long n,
                                                   MatSlots ms, int* __restrict__ cell_count,
                                                   int* __restrict__ seg_count, GridPages gp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = key[i];
    const long long b = (long long)(k >> 8);
    const int m = (int)((k >> 6) & 3);
    cell_count[(phys_block<PAGED>(gp, b) * ms.n + ms.s[m]) * 64 + (int)(k & 63)] = 0;
    seg_count[b * 4 + m] = 0;
}

static __global__ void k_count_rebin(int* counter) { *counter += 1; }

// ------------------------------------------------------ block activity --

// marks global block gb as touched by P2G and appends it to the active list.
// Most callers find the block marked already (every particle of a block marks
// the same few blocks): a read at L2 first spares them the contended exchange;
// a stale zero only costs the exchange, which decides.
__device__ __forceinline__ void mark_block(unsigned* blk_flag, int* active, int* n_active, long long gb) {
    if (__ldcg(&blk_flag[gb]) != 0u) return;
    if (atomicExch(&blk_flag[gb], 1u) == 0u) active[atomicAdd(n_active, 1)] = (int)gb;
}

template <int D>
__device__ __forceinline__ long long block_of_node(const SceneParams& sc, int ix, int iy, int iz) {
    constexpr int S = BlockShape<D>::SHIFT;
    return sc.block_off + (long long)(ix >> S) + (long long)sc.nb[0] * ((iy >> S) + (long long)sc.nb[1] * (iz >> S));
}

// true when every block the stencil at `base` covers has a physical block
// (the stencil spans at most 2 blocks per axis: its corner nodes decide)
template <int D>
__device__ __forceinline__ bool stencil_paged(const SceneParams& sc, const GridPages& gp, const int* base) {
    bool ok = true;
#pragma unroll
    for (int c = 0; c < (D == 3 ? 8 : 4); ++c) {
        int in;
        const long long v = virtual_block<D>(sc, base[0] + 2 * (c & 1), base[1] + 2 * ((c >> 1) & 1),
                                             D == 3 ? base[2] + 2 * (c >> 2) : 0, in);
        ok = ok && phys_block<true>(gp, v) < gp.trash;
    }
    return ok;
}

// P2G of one particle straight to global memory, marking touched blocks.
// PAGED: node addresses through the page table; a stencil reaching a block
// without a page (the pool ran out, or a particle moved more than a cell in a
// substep) sets ERR_POOL, and its writes land in the trash block.
template <int D, bool PAGED = false>
__device__ __forceinline__ void p2g_global(const Stencil<D>& st, const P2GSource<D>& src, const SceneParams& sc,
                                           float4* grid_mom, unsigned* blk_flag, int* active, int* n_active,
                                           const GridPages& gp, unsigned* err_word) {
    if constexpr (PAGED) {
        if (!stencil_paged<D>(sc, gp, st.base)) atomicOr(err_word, ERR_POOL);
        p2g_scatter<D>(st, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 c) {
            atomicAdd(&grid_mom[grid_node<D, true>(sc, gp, st.base[0] + ox, st.base[1] + oy,
                                                   D == 3 ? st.base[2] + oz : 0)], c);
        });
    } else {
        const StencilIndex<D> ix(sc, st.base);
        float4* g = grid_mom + sc.node_off;
        p2g_scatter<D>(st, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 c) {
            atomicAdd(&g[ix(ox, oy, D == 3 ? oz : 0)], c);
        });
    }
    // the stencil spans at most 2 blocks per axis: mark its corner blocks
#pragma unroll
    for (int cx = 0; cx < 2; ++cx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < (D == 3 ? 2 : 1); ++cz) {
                const int ix = st.base[0] + 2 * cx, iy = st.base[1] + 2 * cy, iz = D == 3 ? st.base[2] + 2 * cz : 0;
                mark_block(blk_flag, active, n_active, block_of_node<D>(sc, ix, iy, iz));
            }
}

// First P2G of a state (after creation or set_state): direct atomics.
template <int D, bool PAGED>
__global__ void __launch_bounds__(128) k_p2g_prologue(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                      const SceneParams* __restrict__ scenes, float4* __restrict__ grid_mom,
                                                      unsigned* __restrict__ blk_flag, int* __restrict__ active,
                                                      int* __restrict__ n_active, unsigned* err_word, GridPages gp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[D], v[D], C[D * D], F[D * D], aux;
    load_particle<D>(pb, i, x, v, C, F, aux);
    const GroupParams g = groups[pb.grp[i]];
    const SceneParams& sc = scenes[g.scene];
    unsigned err = 0;
    Stencil<D> st;
    if (!make_stencil<D>(x, sc, st, err)) {
        atomicOr(err_word, err);
        return;
    }
    P2GSource<D> src;
    particle_stress_source<D>(v, C, F, aux, g, sc, src);
    p2g_global<D, PAGED>(st, src, sc, grid_mom, blk_flag, active, n_active, gp, err_word);
}

// Paged grid: gives every block a particle's stencil covers a physical block
// (before the first P2G of a state)
template <int D>
__global__ void __launch_bounds__(256) k_page_in_particles(ParticleBuf pb, long long n,
                                                           const GroupParams* __restrict__ groups,
                                                           const SceneParams* __restrict__ scenes,
                                                           float4* __restrict__ grid_mom, float4* __restrict__ grid_vel,
                                                           GridPages gp, unsigned* err_word) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x[a] = pb.s[(Planes<D>::X + a) * pb.cap + i];
    const SceneParams& sc = scenes[groups[pb.grp[i]].scene];
    unsigned err = 0;
    Stencil<D> st;
    if (!make_stencil<D>(x, sc, st, err)) return;  // the P2G reports it
#pragma unroll
    for (int c = 0; c < (D == 3 ? 8 : 4); ++c) {
        int in;
        const long long v = virtual_block<D>(sc, st.base[0] + 2 * (c & 1), st.base[1] + 2 * ((c >> 1) & 1),
                                             D == 3 ? st.base[2] + 2 * (c >> 2) : 0, in);
        page_in(gp, v, grid_mom, grid_vel, err_word);
    }
}

// Paged grid, at each re-binning: returns to the free stack the physical
// block of every virtual block with nothing active in its 3^D neighbourhood
// (no block there touched by the pending P2G nor stamped by the last two
// grid updates).  Blocks next to active ones keep their pages: the next P2G
// may reach them.  One thread per physical block.
template <int D>
__global__ void __launch_bounds__(256) k_pool_reclaim(GridPages gp, const unsigned* __restrict__ blk_flag,
                                                      const int* __restrict__ blk_epoch, const int* __restrict__ epoch,
                                                      const SceneParams* __restrict__ scenes, int n_scenes) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= gp.trash) return;
    const int v = gp.slot_block[slot];
    if (v < 0) return;
    const int recent = *epoch - 2;
    const SceneParams& sc = scenes[scene_of_block(scenes, n_scenes, v)];
    const int lb = v - (int)sc.block_off;
    const int b[3] = {lb % sc.nb[0], (lb / sc.nb[0]) % sc.nb[1], D == 3 ? lb / (sc.nb[0] * sc.nb[1]) : 0};
    bool live = false;
    for (int t = 0; t < (D == 3 ? 27 : 9) && !live; ++t) {
        const int q[3] = {b[0] + t % 3 - 1, b[1] + (t / 3) % 3 - 1, D == 3 ? b[2] + t / 9 - 1 : 0};
        if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= sc.nb[0] || q[1] >= sc.nb[1] || q[2] >= sc.nb[2]) continue;
        const long long w = sc.block_off + q[0] + (long long)sc.nb[0] * (q[1] + (long long)sc.nb[1] * q[2]);
        live = blk_flag[w] != 0u || blk_epoch[w] >= recent;
    }
    if (live) return;
    gp.page[v] = gp.trash;
    gp.slot_block[slot] = -1;
    gp.free_slots[atomicAdd(gp.n_free, 1)] = slot;
}

// -------------------------------------------------------- grid update --

// Grid update of the active blocks: velocity into grid_vel, momentum buffer
// cleared for the next P2G, block flag reset, block epoch stamped.
// 64 threads per block, 4 blocks per CTA, persistent over the list.
// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start before the kernel ahead of it in the stream ends;
// pdl_wait blocks until that kernel has completed and its writes are visible
// (immediately when launched without the attribute), pdl_trigger lets the
// next kernel in the stream begin launching.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Grid update of the blocks P2G touched.  The last CTA to finish resets the
// active-block count and the fused kernels' chunk cursors for the next pass
// (every CTA has read the count before it counts itself done).
// FIXED: the one scene of a fixed-dt run comes from the kernel parameters
// (fixed_scene), as in the fused kernel.  vel_linear (dense grid): velocities
// in the linear layout (lin_node; nodes of a block beyond the grid's edge are
// not written).  PAGED: a block's nodes through its physical block, and every
// neighbour of an updated block gets a physical block (the next P2G reaches
// at most one block further).
template <int D, bool FIXED, bool PAGED>
__global__ void __launch_bounds__(256) k_grid_update_active(float4* __restrict__ grid_mom, float4* __restrict__ grid_vel,
                                                            const int* __restrict__ active, int* __restrict__ n_active,
                                                            unsigned* __restrict__ blk_flag, int* __restrict__ blk_epoch,
                                                            const int* __restrict__ epoch,
                                                            const SceneParams* __restrict__ scenes, int n_scenes,
                                                            int* __restrict__ cursors, int n_cursors,
                                                            unsigned* __restrict__ done, SceneParams fixed_scene,
                                                            int vel_linear, GridPages gp, unsigned* __restrict__ err_word) {
    pdl_wait();
    const int na = *n_active;
    const int ep = *epoch;
    const int lane = threadIdx.x & 63;
    for (int e = blockIdx.x * 4 + (threadIdx.x >> 6); e < na; e += gridDim.x * 4) {
        const int b = active[e];
        const SceneParams& sc = FIXED ? fixed_scene : scenes[scene_of_block(scenes, n_scenes, b)];
        int ix, iy, iz;
        block_node_coords<D>(sc, b - sc.block_off, lane, ix, iy, iz);
        // (a block without a page -- the pool ran out -- may be claimed by a
        // neighbour's page-in below while it is read here: any value from
        // trash up means no page)
        const long long pb = phys_block<PAGED>(gp, b);
        if (!PAGED || pb < gp.trash) {
            const long long gi = pb * 64 + lane;
            const float4 g = grid_mom[gi];
            const float4 v = grid_node_update<D>(g, sc, ix, iy, iz);
            if (PAGED || !vel_linear) grid_vel[gi] = v;
            else if (ix < sc.n[0] && iy < sc.n[1] && (D == 2 || iz < sc.n[2])) grid_vel[lin_node<D>(sc, ix, iy, iz)] = v;
            grid_mom[gi] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if constexpr (PAGED) {
            if (lane < (D == 3 ? 27 : 9)) {
                // neighbour (lane % 3 - 1, lane / 3 % 3 - 1, lane / 9 - 1) of this block
                const int lb = b - (int)sc.block_off;
                const int bx = lb % sc.nb[0] + lane % 3 - 1, by = (lb / sc.nb[0]) % sc.nb[1] + (lane / 3) % 3 - 1;
                const int bz = D == 3 ? lb / (sc.nb[0] * sc.nb[1]) + lane / 9 - 1 : 0;
                if (bx >= 0 && by >= 0 && bz >= 0 && bx < sc.nb[0] && by < sc.nb[1] && bz < sc.nb[2])
                    page_in(gp, sc.block_off + bx + (long long)sc.nb[0] * (by + (long long)sc.nb[1] * bz), grid_mom,
                            grid_vel, err_word);
            }
        }
        if (lane == 0) {
            blk_flag[b] = 0u;
            blk_epoch[b] = ep;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(done, 1u) == gridDim.x - 1) {
        *n_active = 0;
        for (int k = 0; k < n_cursors; ++k) cursors[k] = 0;
        *done = 0u;
    }
    pdl_trigger();
}

// ------------------------------------------------------------ G2P2G --

struct FusedArgs {
    const Chunk* chunks;  // this material's chunk list
    const int* n_chunks;  // its length
    int* cursor;          // next chunk to hand out (zeroed before every launch)
    const GroupParams* groups;
    const SceneParams* scenes;
    int n_scenes;
    const float4* grid_vel;
    float4* grid_mom;
    unsigned* blk_flag;
    int* active;
    int* n_active;
    int* epoch;      // bumped once per substep (by the launch with bump_epoch)
    int bump_epoch;
    unsigned* err_word;
    unsigned* fallback;  // count of particles that used global memory
    unsigned* speed_max; // adaptive dt: per scene max of |v| + wave (float bits); null when off
    int rounds;          // particles per thread and chunk (a chunk holds CTA size x rounds)
    int defer_vc;        // store the pre-advection position in the v planes and no C (k_recover_vc)
    // the one scene of a single-scene run with a fixed dt, read by the kernels
    // built with FIXED = true from their parameters (constant bank operands,
    // no loads) instead of from `scenes`
    SceneParams scene;
    // one_group != 0: every particle of this launch's material belongs to
    // `group`, which the FIXED kernels then take from their parameters instead
    // of loading each particle's group index and group record
    int one_group;
    GroupParams group;
    GridPages pages;  // paged grid (the PAGED kernels)
    // FIXED dense kernels: grid_vel in the linear layout as a tensor of
    // (component, x, y[, z]) float32, box = one chunk window; the kernels take
    // FusedArgs as a __grid_constant__ parameter, so the copy engine reads the
    // map from the parameter space
    CUtensorMap vel_map;
};

// the group record of particle i of a fused launch
template <bool FIXED>
__device__ __forceinline__ GroupParams particle_group(const FusedArgs& A, const ParticleBuf& pb, long long i) {
    if (FIXED && A.one_group) return A.group;
    return A.groups[pb.grp[i]];
}

// the scene of chunk's scene index si: from the kernel parameters when FIXED
template <bool FIXED>
__device__ __forceinline__ const SceneParams& chunk_scene(const FusedArgs& A, int si) {
    if constexpr (FIXED) return A.scene;
    else return A.scenes[si];
}

template <int D>
__device__ __forceinline__ int tv_idx(int x, int y, int z) {
    if constexpr (TileShape<D>::SWIZZLE) x ^= (y & 1) << 2;
    return x + TileShape<D>::VY * y + TileShape<D>::VZ * z;
}

// ---- pieces of the fused pass (shared by the plain and surrogate kernels)


// 16-byte asynchronous global -> shared copy (cp.async.cg), zero-filled
// when `valid` is false (source size 0: nothing is read)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- window by tensor-map box load (FIXED dense kernels)

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
}

// Waits for phase `parity` of the barrier; false after ~2 s (2^32 cycles)
// without completion, which only a broken copy can cause
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const unsigned a = smem_addr(bar);
    const long long t0 = clock64();
    for (;;) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
        if (clock64() - t0 > (1LL << 32)) return false;
    }
}

// One thread: the window of origin o as one box of the velocity tensor map
// into tv (zero outside the grid), completing on `bar`.  The box starts on a
// component index of 0, so its innermost coordinate is 16-byte aligned; the
// x, y, z coordinates may be -1 or reach past the grid (zero fill).
template <int D>
__device__ __forceinline__ void tma_window(const CUtensorMap* map, float4* tv, unsigned long long* bar, const int* o) {
    constexpr unsigned bytes = TileShape<D>::VN * sizeof(float4);
    const unsigned dst = smem_addr(tv), mb = smem_addr(bar);
    // the window's previous contents were read through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mb), "r"(bytes) : "memory");
    if constexpr (D == 3) {
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
            ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(o[0]), "r"(o[1]), "r"(o[2]), "r"(mb)
            : "memory");
    } else {
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
            ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(o[0]), "r"(o[1]), "r"(mb)
            : "memory");
    }
}

// starts the asynchronous copy of chunk c's grid-velocity window into tv
// (zero outside the grid), NT threads, and keeps the chunk's record in
// *s_ch for the chunk's pass.  PAGED: through the page table (zero for a
// block without a page), and the physical blocks of the window's 3^D blocks
// (trash outside the scene) into s27 for the chunk's scatter.
template <int D, int NT, bool FIXED, bool PAGED>
__device__ __forceinline__ void prefetch_velocity_tile(const FusedArgs& A, int c, float4* tv, int* s27,
                                                       Chunk* s_ch, unsigned long long* bar) {
    constexpr int T = TileShape<D>::T;
    constexpr int S = BlockShape<D>::SHIFT;
    constexpr int M = BlockShape<D>::SIDE - 1;
    constexpr int SIDE = BlockShape<D>::SIDE;
    if constexpr (FIXED && !PAGED) {
        // one box load of the linear velocity tensor, issued by one thread
        if (threadIdx.x == 0) {
            const Chunk ch = A.chunks[c];
            *s_ch = ch;
            tma_window<D>(&A.vel_map, tv, bar, ch.o);
        }
        return;
    }
    const Chunk ch = A.chunks[c];
    if (threadIdx.x == 0) *s_ch = ch;
    const SceneParams& sc = chunk_scene<FIXED>(A, ch.scene);
    const float4* g = A.grid_vel + sc.node_off;
    if constexpr (PAGED) {
        if ((int)threadIdx.x < (D == 3 ? 27 : 9)) {
            const int t = threadIdx.x;
            const int bx = (ch.o[0] + 1) / SIDE - 1 + t % 3, by = (ch.o[1] + 1) / SIDE - 1 + (t / 3) % 3;
            const int bz = D == 3 ? (ch.o[2] + 1) / SIDE - 1 + t / 9 : 0;
            const bool inb = bx >= 0 && by >= 0 && bz >= 0 && bx < sc.nb[0] && by < sc.nb[1] && bz < sc.nb[2];
            s27[t] = inb ? (int)phys_block<true>(A.pages,
                                                 sc.block_off + bx + (long long)sc.nb[0] * (by + (long long)sc.nb[1] * bz))
                         : A.pages.trash;
        }
    }
    for (int t = threadIdx.x; t < TileShape<D>::N; t += NT) {
        const int tx = t % T, ty = (t / T) % T, tz = (D == 3) ? t / (T * T) : 0;
        const int ix = ch.o[0] + tx, iy = ch.o[1] + ty, iz = ch.o[2] + tz;
        bool in = ix >= 0 && iy >= 0 && ix < sc.n[0] && iy < sc.n[1];
        if (D == 3) in = in && iz >= 0 && iz < sc.n[2];
        const float4* src = A.grid_vel;  // not read when outside the grid
        if (in) {
            if constexpr (PAGED) {
                int nin;
                const long long pb = phys_block<true>(A.pages, virtual_block<D>(sc, ix, iy, iz, nin));
                in = pb < A.pages.trash;
                src = A.grid_vel + pb * 64 + nin;
            } else {
                // blocked node index relative to the scene (< 2^31 nodes), as in node_index
                int idx = (ix >> S) * 64 + (ix & M) + ((iy >> S) * sc.nb[0] * 64 + (iy & M) * SIDE);
                if (D == 3) idx += (iz >> S) * sc.nb[0] * sc.nb[1] * 64 + (iz & M) * SIDE * SIDE;
                src = g + idx;
            }
        }
        cp_async16(&tv[tv_idx<D>(tx, ty, tz)], in ? src : A.grid_vel, in);
    }
}

// true when the stencil at `base` lies inside the chunk's window
template <int D>
__device__ __forceinline__ bool in_window(const int* base, const int* o) {
    bool in = true;
#pragma unroll
    for (int a = 0; a < D; ++a) in = in && (base[a] - o[a] >= 0) && (base[a] - o[a] <= TileShape<D>::T - 3);
    return in;
}

// G2P of one particle from the window, or from global memory for a particle
// that drifted out of it since the last re-binning (LIN: grid_vel in the
// linear layout)
template <int D, bool PAGED = false, bool LIN = false>
__device__ __forceinline__ void g2p_window(const Stencil<D>& st, const int* o, const float4* tv, const SceneParams& sc,
                                           const FusedArgs& A, G2PAcc<D>& acc) {
    if (in_window<D>(st.base, o)) {
        const int b0 = st.base[0] - o[0], b1 = st.base[1] - o[1], b2 = D == 3 ? st.base[2] - o[2] : 0;
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) {
            return tv[tv_idx<D>(b0 + ox, b1 + oy, b2 + oz)];
        }, acc);
    } else if constexpr (PAGED) {
        atomicAdd(A.fallback, 1u);
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) {
            return grid_read<D, true>(A.grid_vel, sc, A.pages, st.base[0] + ox, st.base[1] + oy,
                                      D == 3 ? st.base[2] + oz : 0);
        }, acc);
    } else if constexpr (LIN) {
        atomicAdd(A.fallback, 1u);
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) {
            return A.grid_vel[lin_node<D>(sc, st.base[0] + ox, st.base[1] + oy, D == 3 ? st.base[2] + oz : 0)];
        }, acc);
    } else {
        atomicAdd(A.fallback, 1u);
        const StencilIndex<D> ix(sc, st.base);
        const float4* g = A.grid_vel + sc.node_off;
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) { return g[ix(ox, oy, D == 3 ? oz : 0)]; }, acc);
    }
}

// Particle update after G2P (F / Jp / J, advection, new C) and store of the
// new state; x, v, Cn, F, aux hold it on return.  defer_vc: the v planes get
// the pre-advection position instead of v, and C is not stored; k_recover_vc
// rebuilds both from it and the grid velocities when they are read.
template <int D, int MAT>
__device__ __forceinline__ unsigned update_and_store(const G2PAcc<D>& acc, const SceneParams& sc, const GroupParams& g,
                                                     float* __restrict__ S, long long cap, long long i, float* x,
                                                     float* v, float* Cn, float* F, float& aux,
                                                     ElasticSVD<D>* keep = nullptr, bool defer_vc = false) {
    using P = Planes<D>;
    aux = 1.f;
    if (MAT != JELLO) aux = S[P::AUX * cap + i];
    if (MAT != WATER) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) F[k] = S[(P::F + k) * cap + i];
    } else {
#pragma unroll
        for (int k = 0; k < D * D; ++k) F[k] = (k % (D + 1) == 0) ? 1.f : 0.f;
    }
    const unsigned err = material_update<D, MAT>(acc, sc.dt, g, F, aux, keep);
    const float c4 = 4.f * sc.inv_h;
    float x0[D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        x0[a] = x[a];
        v[a] = acc.v[a];
        x[a] = fmaf(sc.dt, acc.v[a], x[a]);
#pragma unroll
        for (int b = 0; b < D; ++b) Cn[a * D + b] = c4 * acc.B[a * D + b];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
        S[(P::X + a) * cap + i] = x[a];
        S[(P::V + a) * cap + i] = defer_vc ? x0[a] : v[a];
    }
    if (!defer_vc) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) S[(P::C + k) * cap + i] = Cn[k];
    }
    if (MAT != WATER) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) S[(P::F + k) * cap + i] = F[k];
    }
    if (MAT != JELLO) S[P::AUX * cap + i] = aux;
    return err;
}

// neighbour-block slots covered by a stencil whose base is local node l of
// the window: the window starts one node below the home block, so local node
// l lies in block slot (l + SIDE - 1) / SIDE (0: home - 1, 1: home, 2: home + 1)
template <int D>
__device__ __forceinline__ unsigned touched_bits(int l0, int l1, int l2) {
    constexpr int SIDE = TileShape<D>::SIDE;
    unsigned bits = 0u;
#pragma unroll
    for (int cx = 0; cx < 2; ++cx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < (D == 3 ? 2 : 1); ++cz) {
                const int sx = (l0 + 2 * cx + SIDE - 1) / SIDE;
                const int sy = (l1 + 2 * cy + SIDE - 1) / SIDE;
                const int sz = D == 3 ? (l2 + 2 * cz + SIDE - 1) / SIDE : 0;
                bits |= 1u << (sx + 3 * (sy + 3 * sz));
            }
    return bits;
}

// P2G scatter of the next substep straight to global memory with float4
// reductions; a stencil inside the window records the blocks it covers in
// `touched`, one outside it marks them itself
// Node offsets of a stencil inside a chunk's window in a paged grid: for
// node (ox, oy, oz), x[ox] + y[oy] + z[oz] packs the window block (0..26,
// low byte) and the node inside it (bits 8..) of the physical address
// s27[block] * 64 + node.
template <int D>
struct PagedStencilIndex {
    int x[3], y[3], z[3];
    __device__ __forceinline__ PagedStencilIndex(const int* base, const int* o) {
        constexpr int S = BlockShape<D>::SHIFT;
        constexpr int M = BlockShape<D>::SIDE - 1;
        constexpr int SIDE = BlockShape<D>::SIDE;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            // window origin o = home block * SIDE - 1: block of node g relative
            // to the one below the home block is (g >> S) - (o + 1) / SIDE + 1
            const int gx = base[0] + k, gy = base[1] + k;
            x[k] = ((gx >> S) - (o[0] + 1) / SIDE + 1) + ((gx & M) << 8);
            y[k] = 3 * ((gy >> S) - (o[1] + 1) / SIDE + 1) + (((gy & M) * SIDE) << 8);
            if (D == 3) {
                const int gz = base[2] + k;
                z[k] = 9 * ((gz >> S) - (o[2] + 1) / SIDE + 1) + (((gz & M) * SIDE * SIDE) << 8);
            } else {
                z[k] = 0;
            }
        }
    }
    // physical node index of stencil node (ox, oy, oz)
    __device__ __forceinline__ long long operator()(const int* s27, int ox, int oy, int oz) const {
        const int p = x[ox] + y[oy] + z[oz];
        return (long long)s27[p & 255] * 64 + (p >> 8);
    }
};

template <int D, bool PAGED = false>
__device__ __forceinline__ void scatter_global(const Stencil<D>& sn, const P2GSource<D>& src, const SceneParams& sc,
                                               const int* o, const FusedArgs& A, unsigned* touched,
                                               const int* s27 = nullptr) {
    if (in_window<D>(sn.base, o)) {
        if constexpr (PAGED) {
            const PagedStencilIndex<D> ix(sn.base, o);
            // a block the stencil covers has no page: the pool ran out or the
            // particle moved more than a cell since the last grid update
            bool ok = true;
#pragma unroll
            for (int c = 0; c < (D == 3 ? 8 : 4); ++c)
                ok = ok && s27[(ix.x[2 * (c & 1)] + ix.y[2 * ((c >> 1) & 1)] + ix.z[D == 3 ? 2 * (c >> 2) : 0]) & 255] <
                               A.pages.trash;
            if (!ok) atomicOr(A.err_word, ERR_POOL);
            p2g_scatter<D>(sn, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 cc) {
                atomicAdd(&A.grid_mom[ix(s27, ox, oy, D == 3 ? oz : 0)], cc);
            });
        } else {
            const StencilIndex<D> ix(sc, sn.base);
            float4* g = A.grid_mom + sc.node_off;
            p2g_scatter<D>(sn, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 cc) {
                atomicAdd(&g[ix(ox, oy, D == 3 ? oz : 0)], cc);
            });
        }
        atomicOr(touched, touched_bits<D>(sn.base[0] - o[0], sn.base[1] - o[1], D == 3 ? sn.base[2] - o[2] : 0));
    } else {
        atomicAdd(A.fallback, 1u);
        p2g_global<D, PAGED>(sn, src, sc, A.grid_mom, A.blk_flag, A.active, A.n_active, A.pages, A.err_word);
    }
}

// marks the neighbour blocks recorded in `touched` (threads 0 .. 3^D - 1)
template <int D>
__device__ __forceinline__ void mark_touched(unsigned touched, const SceneParams& sc, const int* o, const FusedArgs& A) {
    constexpr int SIDE = TileShape<D>::SIDE;
    if ((int)threadIdx.x < (D == 3 ? 27 : 9) && ((touched >> threadIdx.x) & 1u)) {
        const int sx = threadIdx.x % 3, sy = (threadIdx.x / 3) % 3, sz = threadIdx.x / 9;
        const long long bx = (o[0] + 1) / SIDE - 1 + sx, by = (o[1] + 1) / SIDE - 1 + sy;
        const long long bz = D == 3 ? (o[2] + 1) / SIDE - 1 + sz : 0;
        const long long gb = sc.block_off + bx + (long long)sc.nb[0] * (by + (long long)sc.nb[1] * bz);
        mark_block(A.blk_flag, A.active, A.n_active, gb);
    }
}

// ---- segmented scatter (SCATTER_SEGMENTED)
//
// P2G of a warp's particles with one reduction per (run of lanes sharing a
// stencil base, node) instead of one per (lane, node).  In cell-major order
// the particles of a cell are consecutive, so the lanes of a warp form a few
// runs (about 4 at 8 particles per cell) whose members scatter into the same
// 3^D nodes.  Each lane writes its 3^D node values to its column of the
// warp's staging buffer V[row = node][column = lane]; then lane `row` walks
// the columns in order, summing the values of row `row` over each run, and at
// a run's last column reduces the sum into that run's node `row` of the grid
// (red.global.add.v4.f32).  The walk is the same for every lane (run limits
// are warp-uniform bit masks), so it has no divergence.  Lanes whose stencil
// left the chunk's window scatter directly to global memory and do not take
// part; a lane whose base differs from its neighbour's starts a new run, so
// results do not depend on the order.  Every lane of the warp must call this.

// staging-buffer slot of (row, column): the column XOR-ed with the row's low
// three bits, so a column write (fixed row, 32 lanes) and a row read (fixed
// column, one row per lane) both touch distinct 16-byte bank groups
__device__ __forceinline__ int seg_slot(int row, int col) { return row * 32 + (col ^ (row & 7)); }

template <int D>
__device__ __forceinline__ void scatter_segmented(bool valid, const Stencil<D>& sn, const P2GSource<D>& src,
                                                  const SceneParams& sc, const int* o, const FusedArgs& A,
                                                  unsigned* touched, float4* __restrict__ V) {
    constexpr int R = seg_rows(D);
    constexpr int S = BlockShape<D>::SHIFT;
    constexpr int M = BlockShape<D>::SIDE - 1;
    constexpr int SIDE = BlockShape<D>::SIDE;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool inw = valid && in_window<D>(sn.base, o);
    if (valid && !inw) {
        atomicAdd(A.fallback, 1u);
        p2g_global<D>(sn, src, sc, A.grid_mom, A.blk_flag, A.active, A.n_active, A.pages, A.err_word);
    }
    const unsigned part = __ballot_sync(FULL, inw);
    if (part == 0u) return;
    // stencil base in window coordinates (0 .. T - 3 per axis, 4 bits each)
    const int l0 = sn.base[0] - o[0], l1 = sn.base[1] - o[1], l2 = D == 3 ? sn.base[2] - o[2] : 0;
    const int key = inw ? l0 + 16 * (l1 + 16 * l2) : -1;
    if (inw) {
        p2g_scatter<D>(sn, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 c) {
            V[seg_slot(D == 3 ? (ox * 3 + oy) * 3 + oz : ox * 3 + oy, lane)] = c;
        });
    }
    const int kprev = __shfl_up_sync(FULL, key, 1);
    const bool head = inw && (lane == 0 || kprev != key);
    const unsigned heads = __ballot_sync(FULL, head);
    if (head) atomicOr(touched, touched_bits<D>(l0, l1, l2));
    const unsigned ends = part & ~((part & ~heads) >> 1);  // the next lane does not continue the run
    __syncwarp();
    // this lane's row: stencil node (rx, ry, rz)
    const int row = lane;
    const bool has_row = row < R;
    const int rx = D == 3 ? row / 9 : row / 3, ry = D == 3 ? (row / 3) % 3 : row % 3, rz = D == 3 ? row % 3 : 0;
    const int px = o[0] + rx, py = o[1] + ry, pz = o[2] + rz;
    const int sy = sc.nb[0] * 64, sz = sc.nb[0] * sc.nb[1] * 64;
    float4* g = A.grid_mom + sc.node_off;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int m = 0; m < 32; ++m) {
        if (!((part >> m) & 1u)) continue;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (has_row) v = V[seg_slot(row, m)];
        if ((heads >> m) & 1u) {
            acc = v;
        } else {
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
        }
        if ((ends >> m) & 1u) {
            const int km = __shfl_sync(FULL, key, m);
            if (has_row) {
                const int gx = px + (km & 15), gy = py + ((km >> 4) & 15);
                int idx = (gx >> S) * 64 + (gx & M) + (gy >> S) * sy + (gy & M) * SIDE;
                if (D == 3) {
                    const int gz = pz + (km >> 8);
                    idx += (gz >> S) * sz + (gz & M) * SIDE * SIDE;
                }
                atomicAdd(&g[idx], acc);
            }
        }
    }
    __syncwarp();  // the buffer is rewritten by the next call
}

// Per-CTA maximum of the particles' signal speed |v| + wave for adaptive dt:
// warps reduce into a shared word during a chunk, thread 0 folds it into a
// running maximum of the current scene after the chunk and sends one global
// atomicMax when the scene changes and at the end (chunks are ordered by block,
// so a CTA meets few scene changes and the global word sees few atomics).
__device__ __forceinline__ void speed_warp_reduce(unsigned bits, unsigned* shared_word) {
    bits = __reduce_max_sync(0xffffffffu, bits);
    if ((threadIdx.x & 31) == 0 && bits) atomicMax(shared_word, bits);
}
struct SpeedFlush {
    int scene = -1;
    unsigned best = 0u;
    __device__ __forceinline__ void fold(int si, unsigned* shared_word, unsigned* global_max) {
        if (threadIdx.x != 0 || !global_max) return;
        const unsigned v = *shared_word;
        *shared_word = 0u;
        if (si != scene) {
            if (scene >= 0 && best) atomicMax(&global_max[scene], best);
            scene = si;
            best = v;
        } else {
            best = max(best, v);
        }
    }
    __device__ __forceinline__ void flush(unsigned* global_max) {
        if (threadIdx.x == 0 && global_max && scene >= 0 && best) atomicMax(&global_max[scene], best);
    }
};

// Persistent loop of a CTA over a material's chunk list.  Chunks come from a
// global cursor (chunk sizes vary); the index of the chunk after next and the
// next chunk's record and velocity window are fetched while the current chunk
// is processed, so the cursor atomic and the L2 round trips of the record and
// the window are off the critical path.  body(ch, sc, o, tv, touched) runs
// with chunk ch's window in tv; every thread of the CTA calls it; post(scene
// index) runs after the body's barrier.  Two barriers per chunk: (1) window
// landed, the chunk's record and the cleared touched word published; (2) body
// done (touched complete, window free), the index of the chunk after next
// published.  Shared words of parity b = k & 1 are rewritten two chunks
// later, after both barriers of the chunk in between.  PAGED: the window's
// physical blocks (s27) are fetched with the window.
template <int D, int NT, bool FIXED = false, bool PAGED = false, class Body, class Post>
__device__ __forceinline__ void chunk_loop(const FusedArgs& A, float4 (&tv)[2][TileShape<D>::VN], int (&s27)[2][27],
                                           unsigned (&touched)[2], int (&s_cn)[2], Body body, Post post) {
    constexpr bool TMA = FIXED && !PAGED;  // windows by tensor-map box loads
    __shared__ Chunk s_ch[2];  // the records of the current and the next chunk
    // TMA: completion of window b's loads; window b's n-th load completes
    // phase n, so chunk k waits for parity (k >> 1) & 1 of barrier k & 1
    __shared__ __align__(8) unsigned long long s_bar[2];
    const int nch = *A.n_chunks;
    if (threadIdx.x == 0) {
        s_cn[0] = atomicAdd(A.cursor, 1);
        s_cn[1] = atomicAdd(A.cursor, 1);
        if constexpr (TMA) {
            mbar_init(&s_bar[0]);
            mbar_init(&s_bar[1]);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
    }
    __syncthreads();
    int cur = s_cn[0], nxt = s_cn[1];
    __syncthreads();  // s_cn is rewritten below
    if (cur < nch) prefetch_velocity_tile<D, NT, FIXED, PAGED>(A, cur, tv[0], s27[0], &s_ch[0], &s_bar[0]);
    cp_async_commit();
    for (int k = 0; cur < nch; ++k) {
        const int b = k & 1;
        if (nxt < nch)
            prefetch_velocity_tile<D, NT, FIXED, PAGED>(A, nxt, tv[b ^ 1], s27[b ^ 1], &s_ch[b ^ 1], &s_bar[b ^ 1]);
        cp_async_commit();
        // the chunk after next: thread 0 keeps the cursor's answer in a
        // register and publishes it before barrier (2), so the atomic's round
        // trip overlaps the chunk's pass
        int after_next = 0;
        if (threadIdx.x == 0) {
            after_next = atomicAdd(A.cursor, 1);
            touched[b] = 0u;
        }
        cp_async_wait<1>();  // this thread's copies of the current window
        // (1) everyone's copies landed; s_ch[b] and touched[b] published
        if constexpr (TMA) {
            const bool ok = mbar_wait(&s_bar[b], (unsigned)(k >> 1) & 1u);
            if (__syncthreads_or(!ok)) {  // a window that never arrived: report it and stop
                if (threadIdx.x == 0) atomicOr(A.err_word, ERR_TIMEOUT);
                break;
            }
        } else {
            __syncthreads();
        }
        const Chunk ch = s_ch[b];
        const int si = ch.scene;
        const SceneParams& sc = chunk_scene<FIXED>(A, si);
        const int o[3] = {ch.o[0], ch.o[1], ch.o[2]};
        body(ch, sc, o, tv[b], &touched[b], s27[b]);
        if (threadIdx.x == 0) s_cn[b] = after_next;
        __syncthreads();     // (2) s_cn[b] published
        mark_touched<D>(touched[b], sc, o, A);
        post(si);
        cur = nxt;
        nxt = s_cn[b];
    }
    cp_async_wait<0>();
}

// One substep for the particles of each chunk of material MAT: G2P from the
// velocity tile, F / Jp / J update, advection, stress, and P2G of the next
// substep (MPMCUDA.cu:310-741 in one pass: the reference runs P2G, VelUpdate
// and InterpolateAndMove as three kernels with full-grid sweeps and host
// syncs between them).  The P2G scatter reduces into global memory with
// float4 vector reductions (red.global.add.v4.f32), per particle
// (SCATTER_DIRECT) or per run of a warp's lanes sharing a stencil base
// (SCATTER_SEGMENTED, staging buffer in dynamic shared memory).  FIXED: the
// scene comes from A.scene (one scene, dt fixed for the run).
template <int D, int MAT, int CHUNK, int MINB, bool FIXED, int SCATTER, bool PAGED>
__global__ void __launch_bounds__(CHUNK, MINB) k_g2p2g(ParticleBuf pb, const __grid_constant__ FusedArgs A) {
    using P = Planes<D>;
    using TS = TileShape<D>;
    static_assert(!(PAGED && SCATTER == SCATTER_SEGMENTED), "the segmented scatter addresses a dense grid");
    __shared__ __align__(128) float4 tv[2][TS::VN];  // grid velocity windows (double-buffered; box-load targets)
    __shared__ int s27[2][27];                      // PAGED: the windows' physical blocks
    __shared__ unsigned touched[2];                 // 3^D neighbour-block bits
    __shared__ int s_cn[2];
    __shared__ unsigned s_speed;                    // adaptive dt: this chunk's max signal speed
    extern __shared__ __align__(16) float4 seg_stage[];  // SCATTER_SEGMENTED: per-warp staging buffers
    float4* V = seg_stage + (threadIdx.x >> 5) * (seg_rows(D) * 32);

    pdl_wait();     // the grid update ahead of this launch has finished
    pdl_trigger();  // the next pass may launch; it waits for this one to end
    if (A.bump_epoch && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.epoch, 1);
    if (threadIdx.x == 0) s_speed = 0u;
    SpeedFlush speed;
    chunk_loop<D, CHUNK, FIXED, PAGED>(A, tv, s27, touched, s_cn,
                                       [&](const Chunk& ch, const SceneParams& sc, const int* o, const float4* w,
                                           unsigned* tb, const int* wpages) {
        unsigned speed_bits = 0u;
#pragma unroll 1
        for (int r = 0; r < A.rounds; ++r) {
            const int li = (int)threadIdx.x + r * CHUNK;  // this round's particle of the chunk
            // SCATTER_SEGMENTED: sn and src are scattered after the particle's
            // branch, by every lane of the warp together; SCATTER_DIRECT
            // scatters inside it (fewer live registers across the branch)
            bool scatter = false;
            Stencil<D> sn;
            P2GSource<D> src;
            if constexpr (SCATTER == SCATTER_SEGMENTED) sn.base[0] = sn.base[1] = sn.base[2] = 0;
            if (li < ch.count) {
                const long long i = (long long)ch.start + li;
                float* S = pb.s;
                const long long cap = pb.cap;
                unsigned err = 0;
                float x[D];
#pragma unroll
                for (int a = 0; a < D; ++a) x[a] = S[(P::X + a) * cap + i];
                Stencil<D> st;
                if (make_stencil<D>(x, sc, st, err)) {
                    G2PAcc<D> acc;
                    g2p_window<D, PAGED, FIXED && !PAGED>(st, o, w, sc, A, acc);
                    // loaded after the gather, its register peak
                    const GroupParams g = particle_group<FIXED>(A, pb, i);
                    float F[D * D], Cn[D * D], v[D], aux;
                    ElasticSVD<D> esvd;  // snow: the plasticity step's decomposition, reused by the stress
                    err |= update_and_store<D, MAT>(acc, sc, g, S, cap, i, x, v, Cn, F, aux,
                                                    MAT == SNOW ? &esvd : nullptr, A.defer_vc != 0);
                    if (A.speed_max) speed_bits = max(speed_bits, __float_as_uint(signal_speed<D, MAT>(v, g, aux)));

                    // ---- stress + P2G of the next substep (its dt is dt_next)
                    if (make_stencil<D>(x, sc, sn, err)) {
                        if (MAT == SNOW) snow_stress_source<D>(v, Cn, esvd, aux, g, sc.dt_next, src);
                        else particle_stress_source<D, MAT>(v, Cn, F, aux, g, sc.dt_next, src);
                        if constexpr (SCATTER == SCATTER_SEGMENTED) scatter = true;
                        else scatter_global<D, PAGED>(sn, src, sc, o, A, tb, wpages);
                    }
                }
                if (err) atomicOr(A.err_word, err);
            }
            if constexpr (SCATTER == SCATTER_SEGMENTED) scatter_segmented<D>(scatter, sn, src, sc, o, A, tb, V);
        }
        if (A.speed_max) speed_warp_reduce(speed_bits, &s_speed);
    }, [&](int si) { speed.fold(si, &s_speed, A.speed_max); });
    speed.flush(A.speed_max);
}

// v and C of the last substep for particles whose fused pass deferred them:
// the v planes hold the position the pass's G2P used, and grid_vel still holds
// the velocities it gathered (the next grid update has not run), so the same
// gather gives the same v and C = 4/h B (vel_linear: grid_vel in the linear
// layout).  A particle whose stencil left the grid (the pass reported it)
// keeps its planes.
template <int D, bool PAGED>
__global__ void __launch_bounds__(256) k_recover_vc(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                    const SceneParams* __restrict__ scenes,
                                                    const float4* __restrict__ grid_vel, int vel_linear,
                                                    GridPages gp) {
    using P = Planes<D>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* S = pb.s;
    const long long cap = pb.cap;
    const SceneParams& sc = scenes[groups[pb.grp[i]].scene];
    float x0[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x0[a] = S[(P::V + a) * cap + i];
    Stencil<D> st;
    unsigned err = 0;
    if (!make_stencil<D>(x0, sc, st, err)) return;
    G2PAcc<D> acc;
    if constexpr (PAGED) {
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) {
            return grid_read<D, true>(grid_vel, sc, gp, st.base[0] + ox, st.base[1] + oy, D == 3 ? st.base[2] + oz : 0);
        }, acc);
    } else if (vel_linear) {
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) {
            return grid_vel[lin_node<D>(sc, st.base[0] + ox, st.base[1] + oy, D == 3 ? st.base[2] + oz : 0)];
        }, acc);
    } else {
        const StencilIndex<D> ix(sc, st.base);
        const float4* g = grid_vel + sc.node_off;
        g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) { return g[ix(ox, oy, D == 3 ? oz : 0)]; }, acc);
    }
    const float c4 = 4.f * sc.inv_h;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        S[(P::V + a) * cap + i] = acc.v[a];
#pragma unroll
        for (int b = 0; b < D; ++b) S[(P::C + a * D + b) * cap + i] = c4 * acc.B[a * D + b];
    }
}

// Adaptive dt, once per substep after the fused pass (one thread per scene):
// the substep that ran advances the scene's time; the next one uses the dt its
// P2G was built with; the one after gets clamp(cfl h / max(|v| + wave),
// dt_min, dt_max) from the speeds this pass saw.  (The reference computes a
// max(J, 1/J)^3 factor for this and never applies it, MPMCUDA.cu:915-920.)
static __global__ void k_adapt_dt(SceneParams* scenes, int n_scenes, unsigned* speed_max, double* scene_time) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_scenes) return;
    SceneParams& sc = scenes[s];
    scene_time[s] += (double)sc.dt;
    const float v = __uint_as_float(speed_max[s]);
    speed_max[s] = 0u;
    float dtn = sc.dt_max;
    if (v > 0.f) dtn = fminf(dtn, sc.cfl * sc.h / v);
    dtn = fmaxf(dtn, sc.dt_min);
    sc.dt = sc.dt_next;
    sc.dt_next = dtn;
}

}  // namespace mpm
