// Binned substep: particles sorted by home grid block, one fused kernel per
// substep that gathers (G2P), updates the particle, evaluates the stress and
// scatters (P2G) for the next substep through shared-memory grid tiles, and
// a grid update that visits only the blocks P2G touched.
//
// Home block: the 4x4x4 node block (8x8 in 2D) that holds a particle's base
// node at the last re-binning.  A chunk is up to CHUNK particles of one home
// block, contiguous in the sorted state.  The tile of a chunk is the node
// window [4b - 1, 4b + 7) per axis: it holds the stencil of every particle
// whose base node is within one node of the home block.  Particles that
// drifted further since the last re-binning use global memory directly, so
// results never depend on how stale the binning is.
#pragma once

#include "mpm_grid.cuh"
#include "mpm_kernels_direct.cuh"
#include "mpm_particle.cuh"

namespace mpm {

struct Chunk {
    int block;   // global block index (scene block_off + local block)
    int start;   // first sorted particle
    int count;   // particles in this chunk
    int pad;
};

template <int D>
struct TileShape {
    static constexpr int SIDE = BlockShape<D>::SIDE;
    static constexpr int T = SIDE + 4;                    // window width per axis
    static constexpr int N = (D == 3) ? T * T * T : T * T; // nodes per tile
};

constexpr int kChunk = 256;  // particles per chunk = threads per fused CTA

// ------------------------------------------------------------- binning --

template <int D>
__device__ __forceinline__ long long home_block_of(const SceneParams& sc, const float* x) {
    constexpr int S = BlockShape<D>::SHIFT;
    int b[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const float gx = (x[a] - sc.origin[a]) * sc.inv_h;
        int base = isfinite(gx) ? (int)floorf(gx - 0.5f) : 0;
        base = min(max(base, 0), sc.n[a] - 3);
        b[a] = base >> S;
    }
    return sc.block_off + (long long)b[0] + (long long)sc.nb[0] * (b[1] + (long long)sc.nb[1] * b[2]);
}

// key = home block; rank = arrival order inside the block
template <int D>
__global__ void __launch_bounds__(256) k_bin_count(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                   const SceneParams* __restrict__ scenes, int* __restrict__ key,
                                                   int* __restrict__ rank, int* __restrict__ blk_count) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x[a] = pb.s[(Planes<D>::X + a) * pb.cap + i];
    const SceneParams& sc = scenes[groups[pb.grp[i]].scene];
    const long long b = home_block_of<D>(sc, x);
    key[i] = (int)b;
    rank[i] = atomicAdd(&blk_count[b], 1);
}

// moves every particle to blk_start[key] + rank in the other buffer
template <int D>
__global__ void __launch_bounds__(256) k_bin_scatter(ParticleBuf src, ParticleBuf dst, long long n,
                                                     const int* __restrict__ key, const int* __restrict__ rank,
                                                     const int* __restrict__ blk_start) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = (long long)blk_start[key[i]] + rank[i];
#pragma unroll
    for (int p = 0; p < Planes<D>::COUNT; ++p) dst.s[p * dst.cap + j] = src.s[p * src.cap + i];
    dst.grp[j] = src.grp[i];
    dst.id[j] = src.id[i];
}

// one chunk list entry per kChunk particles of every non-empty block
__global__ void __launch_bounds__(256) k_make_chunks(const int* __restrict__ blk_count, const int* __restrict__ blk_start,
                                                     long long total_blocks, Chunk* __restrict__ chunks,
                                                     int* __restrict__ n_chunks) {
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= total_blocks) return;
    const int c = blk_count[b];
    if (c == 0) return;
    const int nch = (c + kChunk - 1) / kChunk;
    const int o = atomicAdd(n_chunks, nch);
    for (int j = 0; j < nch; ++j) {
        Chunk ch;
        ch.block = (int)b;
        ch.start = blk_start[b] + j * kChunk;
        ch.count = min(kChunk, c - j * kChunk);
        ch.pad = 0;
        chunks[o + j] = ch;
    }
}

__global__ void k_count_rebin(int* counter) { *counter += 1; }

// ------------------------------------------------------ block activity --

// marks global block gb as touched by P2G and appends it to the active list
__device__ __forceinline__ void mark_block(unsigned* blk_flag, int* active, int* n_active, long long gb) {
    if (atomicExch(&blk_flag[gb], 1u) == 0u) active[atomicAdd(n_active, 1)] = (int)gb;
}

template <int D>
__device__ __forceinline__ long long block_of_node(const SceneParams& sc, int ix, int iy, int iz) {
    constexpr int S = BlockShape<D>::SHIFT;
    return sc.block_off + (long long)(ix >> S) + (long long)sc.nb[0] * ((iy >> S) + (long long)sc.nb[1] * (iz >> S));
}

// P2G of one particle straight to global memory, marking touched blocks
template <int D>
__device__ __forceinline__ void p2g_global(const Stencil<D>& st, const P2GSource<D>& src, const SceneParams& sc,
                                           float4* grid_mom, unsigned* blk_flag, int* active, int* n_active) {
#pragma unroll
    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
            for (int oz = 0; oz < (D == 3 ? 3 : 1); ++oz) {
                const int o[3] = {ox, oy, oz};
                const float4 c = p2g_node<D>(st, src, o, sc.h, sc.inv_h);
                const int ix = st.base[0] + ox, iy = st.base[1] + oy, iz = D == 3 ? st.base[2] + oz : 0;
                atomicAdd(&grid_mom[node_index<D>(sc, ix, iy, iz)], c);
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
template <int D>
__global__ void __launch_bounds__(128) k_p2g_prologue(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                      const SceneParams* __restrict__ scenes, float4* __restrict__ grid_mom,
                                                      unsigned* __restrict__ blk_flag, int* __restrict__ active,
                                                      int* __restrict__ n_active, unsigned* err_word) {
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
    p2g_global<D>(st, src, sc, grid_mom, blk_flag, active, n_active);
}

// -------------------------------------------------------- grid update --

// Grid update of the active blocks: velocity into grid_vel, momentum buffer
// cleared for the next P2G, block flag reset, block epoch stamped.
// 64 threads per block, 4 blocks per CTA, persistent over the list.
template <int D>
__global__ void __launch_bounds__(256) k_grid_update_active(float4* __restrict__ grid_mom, float4* __restrict__ grid_vel,
                                                            const int* __restrict__ active, const int* __restrict__ n_active,
                                                            unsigned* __restrict__ blk_flag, int* __restrict__ blk_epoch,
                                                            const int* __restrict__ epoch,
                                                            const SceneParams* __restrict__ scenes, int n_scenes) {
    const int na = *n_active;
    const int ep = *epoch;
    const int lane = threadIdx.x & 63;
    for (int e = blockIdx.x * 4 + (threadIdx.x >> 6); e < na; e += gridDim.x * 4) {
        const int b = active[e];
        const int s = scene_of_block(scenes, n_scenes, b);
        const SceneParams& sc = scenes[s];
        int ix, iy, iz;
        block_node_coords<D>(sc, b - sc.block_off, lane, ix, iy, iz);
        const long long gi = (long long)b * 64 + lane;
        const float4 g = grid_mom[gi];
        grid_vel[gi] = grid_node_update<D>(g, sc, ix, iy, iz);
        grid_mom[gi] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (lane == 0) {
            blk_flag[b] = 0u;
            blk_epoch[b] = ep;
        }
    }
}

// ------------------------------------------------------------ G2P2G --

struct FusedArgs {
    const Chunk* chunks;
    const int* n_chunks;
    int* cursor;  // next chunk to hand out (zeroed before every launch)
    const GroupParams* groups;
    const SceneParams* scenes;
    int n_scenes;
    const float4* grid_vel;
    float4* grid_mom;
    unsigned* blk_flag;
    int* active;
    int* n_active;
    int* epoch;
    unsigned* err_word;
    unsigned* fallback;  // count of particles that used global memory
};

// One substep for the particles of each chunk: G2P from the velocity tile,
// F / Jp / J update, advection, stress, and P2G of the next substep into a
// shared momentum tile flushed with float4 atomics (MPMCUDA.cu:310-741 in
// one pass: the reference runs P2G, VelUpdate and InterpolateAndMove as
// three kernels with full-grid sweeps and host syncs between them).
template <int D>
__global__ void __launch_bounds__(kChunk, 2) k_g2p2g(ParticleBuf pb, FusedArgs A) {
    using P = Planes<D>;
    using TS = TileShape<D>;
    constexpr int T = TS::T;
    constexpr int TN = TS::N;
    constexpr int SIDE = TS::SIDE;
    __shared__ float4 tv[TN];      // grid velocity window
    __shared__ float tm[4][TN];    // next-substep momentum / mass window
    __shared__ unsigned touched;   // 3^D neighbour-block bits

    __shared__ int s_chunk;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.epoch, 1);
    const int nch = *A.n_chunks;
    // persistent CTAs take chunks from a global cursor (chunk sizes vary)
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(A.cursor, 1);
        __syncthreads();
        const int c = s_chunk;
        if (c >= nch) break;
        const Chunk ch = A.chunks[c];
        const int s = scene_of_block(A.scenes, A.n_scenes, ch.block);
        const SceneParams& sc = A.scenes[s];
        const long long lb = ch.block - sc.block_off;
        int o[3];
        o[0] = (int)(lb % sc.nb[0]) * SIDE - 1;
        o[1] = (int)((lb / sc.nb[0]) % sc.nb[1]) * SIDE - 1;
        o[2] = (D == 3) ? (int)(lb / ((long long)sc.nb[0] * sc.nb[1])) * SIDE - 1 : 0;
        if (threadIdx.x == 0) touched = 0u;
        for (int t = threadIdx.x; t < TN; t += blockDim.x) {
            const int tx = t % T, ty = (t / T) % T, tz = (D == 3) ? t / (T * T) : 0;
            const int ix = o[0] + tx, iy = o[1] + ty, iz = o[2] + tz;
            bool in = ix >= 0 && iy >= 0 && ix < sc.n[0] && iy < sc.n[1];
            if (D == 3) in = in && iz >= 0 && iz < sc.n[2];
            tv[t] = in ? A.grid_vel[node_index<D>(sc, ix, iy, iz)] : make_float4(0.f, 0.f, 0.f, 0.f);
            tm[0][t] = 0.f;
            tm[1][t] = 0.f;
            tm[2][t] = 0.f;
            tm[3][t] = 0.f;
        }
        __syncthreads();

        if ((int)threadIdx.x < ch.count) {
            const long long i = (long long)ch.start + threadIdx.x;
            float* S = pb.s;
            const long long cap = pb.cap;
            const GroupParams g = A.groups[pb.grp[i]];
            unsigned err = 0;
            float x[D];
#pragma unroll
            for (int a = 0; a < D; ++a) x[a] = S[(P::X + a) * cap + i];
            Stencil<D> st;
            if (make_stencil<D>(x, sc, st, err)) {
                // ---- G2P
                G2PAcc<D> acc;
                g2p_zero<D>(acc);
                bool local = true;
#pragma unroll
                for (int a = 0; a < D; ++a) local = local && (st.base[a] - o[a] >= 0) && (st.base[a] - o[a] <= T - 3);
                if (local) {
                    const int l0 = st.base[0] - o[0], l1 = st.base[1] - o[1], l2 = D == 3 ? st.base[2] - o[2] : 0;
#pragma unroll
                    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                            for (int oz = 0; oz < (D == 3 ? 3 : 1); ++oz) {
                                const int off[3] = {ox, oy, oz};
                                const int t = (l0 + ox) + T * ((l1 + oy) + (D == 3 ? T * (l2 + oz) : 0));
                                g2p_node<D>(st, off, tv[t], sc.inv_h, acc);
                            }
                } else {
                    atomicAdd(A.fallback, 1u);
#pragma unroll
                    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                            for (int oz = 0; oz < (D == 3 ? 3 : 1); ++oz) {
                                const int off[3] = {ox, oy, oz};
                                const long long gi = node_index<D>(sc, st.base[0] + ox, st.base[1] + oy,
                                                                   D == 3 ? st.base[2] + oz : 0);
                                g2p_node<D>(st, off, A.grid_vel[gi], sc.inv_h, acc);
                            }
                }
                // ---- particle update
                float F[D * D], Cn[D * D], v[D];
                float aux = S[P::AUX * cap + i];
                if (g.type != WATER) {
#pragma unroll
                    for (int k = 0; k < D * D; ++k) F[k] = S[(P::F + k) * cap + i];
                } else {
#pragma unroll
                    for (int k = 0; k < D * D; ++k) F[k] = (k % (D + 1) == 0) ? 1.f : 0.f;
                }
                err |= material_update<D>(acc, sc.dt, g, F, aux);
                const float c4 = 4.f * sc.inv_h;
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    v[a] = acc.v[a];
                    x[a] = fmaf(sc.dt, acc.v[a], x[a]);
#pragma unroll
                    for (int b = 0; b < D; ++b) Cn[a * D + b] = c4 * acc.B[a * D + b];
                }
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    S[(P::X + a) * cap + i] = x[a];
                    S[(P::V + a) * cap + i] = v[a];
                }
#pragma unroll
                for (int k = 0; k < D * D; ++k) S[(P::C + k) * cap + i] = Cn[k];
                if (g.type != WATER) {
#pragma unroll
                    for (int k = 0; k < D * D; ++k) S[(P::F + k) * cap + i] = F[k];
                }
                S[P::AUX * cap + i] = aux;

                // ---- stress + P2G of the next substep
                Stencil<D> sn;
                if (make_stencil<D>(x, sc, sn, err)) {
                    P2GSource<D> src;
                    particle_stress_source<D>(v, Cn, F, aux, g, sc, src);
                    bool in_tile = true;
#pragma unroll
                    for (int a = 0; a < D; ++a)
                        in_tile = in_tile && (sn.base[a] - o[a] >= 0) && (sn.base[a] - o[a] <= T - 3);
                    if (in_tile) {
                        const int l0 = sn.base[0] - o[0], l1 = sn.base[1] - o[1], l2 = D == 3 ? sn.base[2] - o[2] : 0;
                        unsigned bits = 0u;
#pragma unroll
                        for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                            for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                                for (int oz = 0; oz < (D == 3 ? 3 : 1); ++oz) {
                                    const int off[3] = {ox, oy, oz};
                                    const float4 cc = p2g_node<D>(sn, src, off, sc.h, sc.inv_h);
                                    const int t = (l0 + ox) + T * ((l1 + oy) + (D == 3 ? T * (l2 + oz) : 0));
                                    atomicAdd(&tm[0][t], cc.x);
                                    atomicAdd(&tm[1][t], cc.y);
                                    if (D == 3) atomicAdd(&tm[2][t], cc.z);
                                    atomicAdd(&tm[3][t], cc.w);
                                }
                        // neighbour-block slots covered by the stencil: the window starts
                        // one node below the home block, so local node l lies in block slot
                        // (l + SIDE - 1) / SIDE (0: home - 1, 1: home, 2: home + 1)
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
                        atomicOr(&touched, bits);
                    } else {
                        atomicAdd(A.fallback, 1u);
                        p2g_global<D>(sn, src, sc, A.grid_mom, A.blk_flag, A.active, A.n_active);
                    }
                }
            }
            if (err) atomicOr(A.err_word, err);
        }
        __syncthreads();

        // ---- flush the momentum window
        for (int t = threadIdx.x; t < TN; t += blockDim.x) {
            const float m = tm[3][t];
            const float mx = tm[0][t], my = tm[1][t], mz = tm[2][t];
            if (m != 0.f || mx != 0.f || my != 0.f || mz != 0.f) {
                const int tx = t % T, ty = (t / T) % T, tz = (D == 3) ? t / (T * T) : 0;
                const int ix = o[0] + tx, iy = o[1] + ty, iz = o[2] + tz;
                atomicAdd(&A.grid_mom[node_index<D>(sc, ix, iy, iz)], make_float4(mx, my, mz, m));
            }
        }
        if ((int)threadIdx.x < (D == 3 ? 27 : 9) && ((touched >> threadIdx.x) & 1u)) {
            const int sx = threadIdx.x % 3, sy = (threadIdx.x / 3) % 3, sz = threadIdx.x / 9;
            const long long bx = (o[0] + 1) / SIDE - 1 + sx, by = (o[1] + 1) / SIDE - 1 + sy;
            const long long bz = D == 3 ? (o[2] + 1) / SIDE - 1 + sz : 0;
            const long long gb = sc.block_off + bx + (long long)sc.nb[0] * (by + (long long)sc.nb[1] * bz);
            mark_block(A.blk_flag, A.active, A.n_active, gb);
        }
        __syncthreads();
    }
}

}  // namespace mpm
