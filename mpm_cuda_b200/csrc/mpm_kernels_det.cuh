// Deterministic P2G (MPM_P2G_DETERMINISTIC): bitwise identical results from
// run to run.
//
// FP32 atomics make the order of a node's additions depend on scheduling.  This
// mode never adds floats atomically: every particle writes its P2G source
// record (stencil fractions, m v, m C, -dt V tau, m) and the id of its base
// node; a stable radix sort groups the records by base node (the key of a
// particle whose stencil left the grid is the node count, which sorts last).
// The records are copied into sorted order (k_det_permute), each record whole,
// so a base node's records form one contiguous run.  One thread per run sums,
// particle by particle in sorted order, the run's contributions to each of the
// 3^D nodes of its stencil (k_det_partials: a partial sum per (base node,
// offset)); then each grid node adds, in a fixed offset order, the partials of
// the 3^D base nodes whose stencils cover it (k_det_sum), and stores the sum.
// Particles stay in creation order in this mode and the grid update visits the
// blocks the stencils touched, as in the binned path.
#pragma once

#include "mpm_grid.cuh"
#include "mpm_kernels_binned.cuh"
#include "mpm_particle.cuh"

namespace mpm {

// P2G source records, component planes of stride `cap`:
//   [0, D) fx   [D, 2D) m v   [2D, 2D + D^2) m C   then A (D^2)   then m
// (the sorted copy holds each record whole: STRIDE floats, the same order)
template <int D>
struct SrcPlanes {
    static constexpr int FX = 0, MV = D, MC = 2 * D, A = 2 * D + D * D, M = 2 * D + 2 * D * D;
    static constexpr int COUNT = 2 * D + 2 * D * D + 1;
    // a record of the sorted copy: COUNT floats padded to whole float4s
    static constexpr int STRIDE = (COUNT + 3) / 4 * 4;
};

template <int D>
__global__ void __launch_bounds__(128) k_det_source(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                    const SceneParams* __restrict__ scenes, float* __restrict__ src,
                                                    long long cap, unsigned long long* __restrict__ keys,
                                                    unsigned long long no_cell,
                                                    unsigned* __restrict__ vals, unsigned* __restrict__ blk_flag,
                                                    int* __restrict__ active, int* __restrict__ n_active,
                                                    unsigned* err_word) {
    using SP = SrcPlanes<D>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vals[i] = (unsigned)i;
    float x[D], v[D], C[D * D], F[D * D], aux;
    load_particle<D>(pb, i, x, v, C, F, aux);
    const GroupParams g = groups[pb.grp[i]];
    const SceneParams& sc = scenes[g.scene];
    unsigned err = 0;
    Stencil<D> st;
    if (!make_stencil<D>(x, sc, st, err)) {
        keys[i] = no_cell;
        atomicOr(err_word, err);
        return;
    }
    P2GSource<D> s;
    particle_stress_source<D>(v, C, F, aux, g, sc, s);
#pragma unroll
    for (int a = 0; a < D; ++a) {
        src[(SP::FX + a) * cap + i] = st.fx[a];
        src[(SP::MV + a) * cap + i] = s.mv[a];
    }
#pragma unroll
    for (int k = 0; k < D * D; ++k) {
        src[(SP::MC + k) * cap + i] = s.mC[k];
        src[(SP::A + k) * cap + i] = s.A[k];
    }
    src[SP::M * cap + i] = s.m;
    keys[i] = (unsigned long long)node_index<D>(sc, st.base[0], st.base[1], D == 3 ? st.base[2] : 0);
#pragma unroll
    for (int cx = 0; cx < 2; ++cx)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < (D == 3 ? 2 : 1); ++cz)
                mark_block(blk_flag, active, n_active,
                           block_of_node<D>(sc, st.base[0] + 2 * cx, st.base[1] + 2 * cy,
                                            D == 3 ? st.base[2] + 2 * cz : 0));
}

// [cell_start, cell_end) of every base node in the sorted records
__global__ void __launch_bounds__(256) k_det_ranges(const unsigned long long* __restrict__ keys, long long n,
                                                    unsigned long long no_cell, int* __restrict__ cell_start,
                                                    int* __restrict__ cell_end) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long k = keys[j];
    if (k == no_cell) return;
    if (j == 0 || keys[j - 1] != k) cell_start[k] = (int)j;
    if (j == n - 1 || keys[j + 1] != k) cell_end[k] = (int)j + 1;
}

__global__ void __launch_bounds__(256) k_det_reset(const unsigned long long* __restrict__ keys, long long n,
                                                   unsigned long long no_cell, int* __restrict__ cell_start,
                                                   int* __restrict__ cell_end) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long k = keys[j];
    if (k == no_cell) return;
    cell_start[k] = 0;
    cell_end[k] = 0;
}

// The records in sorted order: record j of `dst` (STRIDE floats, planes in
// the same order) gets the record of particle order[j] (the out-of-grid
// particles, sorted last, copy records nobody reads)
template <int D>
__global__ void __launch_bounds__(256) k_det_permute(const float* __restrict__ src, float4* __restrict__ dst,
                                                     long long cap, const unsigned* __restrict__ order, long long n) {
    using SP = SrcPlanes<D>;
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const long long p = order[j];
    float r[SP::STRIDE];
#pragma unroll
    for (int k = 0; k < SP::STRIDE; ++k) r[k] = k < SP::COUNT ? src[k * cap + p] : 0.f;
#pragma unroll
    for (int q = 0; q < SP::STRIDE / 4; ++q)
        dst[j * (SP::STRIDE / 4) + q] = make_float4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
}

// Run starts in the sorted keys (the out-of-grid particles, sorted last, start none)
struct RunStart {
    const unsigned long long* keys;
    unsigned long long no_cell;
    __device__ __forceinline__ bool operator()(int j) const {
        return keys[j] != no_cell && (j == 0 || keys[j - 1] != keys[j]);
    }
};

// One thread per run of records sharing a base node (runs[r] = its first
// sorted position j0): the run's P2G contributions to each stencil node,
// summed particle by particle in sorted order, stored as partial[j0 * 3^D + k]
// with k = (ox * 3 + oy) * 3 + oz (3D) or ox * 3 + oy (2D).
template <int D>
__global__ void __launch_bounds__(64, 4) k_det_partials(const float4* __restrict__ src,
                                                        const unsigned long long* __restrict__ keys,
                                                        const int* __restrict__ runs, const int* __restrict__ n_runs,
                                                        const int* __restrict__ cell_end,
                                                        const SceneParams* __restrict__ scenes, int n_scenes,
                                                        float4* __restrict__ partial) {
    using SP = SrcPlanes<D>;
    constexpr int K = D == 3 ? 27 : 9;
    const int nr = *n_runs;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += gridDim.x * blockDim.x) {
        const int j0 = runs[r];
        const unsigned long long key = keys[j0];
        const int j1 = cell_end[key];
        const SceneParams& sc = scenes[scene_of_block(scenes, n_scenes, (long long)(key >> 6))];
        float4 acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int j = j0; j < j1; ++j) {
            float rec[SP::STRIDE];
#pragma unroll
            for (int q = 0; q < SP::STRIDE / 4; ++q) {
                const float4 v = src[(long long)j * (SP::STRIDE / 4) + q];
                rec[4 * q] = v.x;
                rec[4 * q + 1] = v.y;
                rec[4 * q + 2] = v.z;
                rec[4 * q + 3] = v.w;
            }
            Stencil<D> st;
            P2GSource<D> s;
#pragma unroll
            for (int a = 0; a < D; ++a) {
                st.fx[a] = rec[SP::FX + a];
                s.mv[a] = rec[SP::MV + a];
            }
#pragma unroll
            for (int k = 0; k < D * D; ++k) {
                s.mC[k] = rec[SP::MC + k];
                s.A[k] = rec[SP::A + k];
            }
            s.m = rec[SP::M];
            p2g_scatter<D>(st, s, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 c) {
                float4& t = acc[D == 3 ? (ox * 3 + oy) * 3 + oz : ox * 3 + oy];
                t.x += c.x;
                t.y += c.y;
                t.z += c.z;
                t.w += c.w;
            });
        }
#pragma unroll
        for (int k = 0; k < K; ++k) partial[(long long)j0 * K + k] = acc[k];
    }
}

// Every node of the listed blocks adds, in the order of the stencil offset o,
// the partial sums of the base nodes node - o, o in {0,1,2}^D, and stores the
// total.
template <int D>
__global__ void __launch_bounds__(256) k_det_sum(const float4* __restrict__ partial,
                                                 const int* __restrict__ cell_start,
                                                 const int* __restrict__ cell_end, const int* __restrict__ blocks,
                                                 const int* __restrict__ n_blocks,
                                                 const SceneParams* __restrict__ scenes, int n_scenes,
                                                 float4* __restrict__ grid_mom) {
    constexpr int K = D == 3 ? 27 : 9;
    const int na = *n_blocks;
    const int lane = threadIdx.x & 63;
    for (int e = blockIdx.x * 4 + (threadIdx.x >> 6); e < na; e += gridDim.x * 4) {
        const int b = blocks[e];
        const SceneParams& sc = scenes[scene_of_block(scenes, n_scenes, b)];
        int id[3];
        block_node_coords<D>(sc, b - sc.block_off, lane, id[0], id[1], id[2]);
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        const bool in_grid = id[0] < sc.n[0] && id[1] < sc.n[1] && (D == 2 || id[2] < sc.n[2]);
        if (in_grid) {
#pragma unroll
            for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                    for (int oz = 0; oz < (D == 3 ? 3 : 1); ++oz) {
                        const int bx = id[0] - ox, by = id[1] - oy, bz = D == 3 ? id[2] - oz : 0;
                        if (bx < 0 || by < 0 || bz < 0) continue;
                        const long long cell = node_index<D>(sc, bx, by, bz);
                        const int j0 = cell_start[cell];
                        if (cell_end[cell] <= j0) continue;  // no particle has this base node
                        const float4 c = partial[(long long)j0 * K + (D == 3 ? (ox * 3 + oy) * 3 + oz : ox * 3 + oy)];
                        acc.x += c.x;
                        acc.y += c.y;
                        acc.z += c.z;
                        acc.w += c.w;
                    }
        }
        grid_mom[(long long)b * 64 + lane] = acc;
    }
}

}  // namespace mpm
