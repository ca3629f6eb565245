// Deterministic P2G (MPM_P2G_DETERMINISTIC): bitwise identical results from
// run to run.
//
// FP32 atomics make the order of a node's additions depend on scheduling.  This
// mode never adds floats atomically: every particle writes its P2G source
// record (stencil fractions, m v, m C, -dt V tau, m) and the id of its base
// node; a stable radix sort groups the records by base node; then each grid
// node sums, in a fixed order (stencil offset, then sorted position), the
// records of the 27 base nodes whose stencils cover it, and stores the sum.
// The records are copied into sorted order once (k_det_permute), each record
// contiguous, so the sum reads each base node's records as one contiguous run
// of whole records (a few float4 loads each).
// Particles stay in creation order in this mode and the grid update visits the
// blocks the stencils touched, as in the binned path.
#pragma once

#include "mpm_grid.cuh"
#include "mpm_kernels_binned.cuh"
#include "mpm_particle.cuh"

namespace mpm {

// P2G source records, component planes of stride `cap`:
//   [0, D) fx   [D, 2D) m v   [2D, 2D + D^2) m C   then A (D^2)   then m
template <int D>
struct SrcPlanes {
    static constexpr int FX = 0, MV = D, MC = 2 * D, A = 2 * D + D * D, M = 2 * D + 2 * D * D;
    static constexpr int COUNT = 2 * D + 2 * D * D + 1;
    // a record of the sorted copy: COUNT floats padded to whole float4s
    static constexpr int STRIDE = (COUNT + 3) / 4 * 4;
};

constexpr unsigned long long kNoCell = ~0ull;

template <int D>
__global__ void __launch_bounds__(128) k_det_source(ParticleBuf pb, long long n, const GroupParams* __restrict__ groups,
                                                    const SceneParams* __restrict__ scenes, float* __restrict__ src,
                                                    long long cap, unsigned long long* __restrict__ keys,
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
        keys[i] = kNoCell;
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
                                                    int* __restrict__ cell_start, int* __restrict__ cell_end) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long k = keys[j];
    if (k == kNoCell) return;
    if (j == 0 || keys[j - 1] != k) cell_start[k] = (int)j;
    if (j == n - 1 || keys[j + 1] != k) cell_end[k] = (int)j + 1;
}

__global__ void __launch_bounds__(256) k_det_reset(const unsigned long long* __restrict__ keys, long long n,
                                                   int* __restrict__ cell_start, int* __restrict__ cell_end) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long k = keys[j];
    if (k == kNoCell) return;
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

// Every node of the active blocks sums the records of the base nodes
// node - o, o in {0,1,2}^D, in the order (o, sorted position), and stores it
// (src: the records in sorted order, k_det_permute's layout).
template <int D>
__global__ void __launch_bounds__(256) k_det_gather(const float4* __restrict__ src,
                                                    const int* __restrict__ cell_start,
                                                    const int* __restrict__ cell_end, const int* __restrict__ active,
                                                    const int* __restrict__ n_active,
                                                    const SceneParams* __restrict__ scenes, int n_scenes,
                                                    float4* __restrict__ grid_mom) {
    using SP = SrcPlanes<D>;
    const int na = *n_active;
    const int lane = threadIdx.x & 63;
    for (int e = blockIdx.x * 4 + (threadIdx.x >> 6); e < na; e += gridDim.x * 4) {
        const int b = active[e];
        const SceneParams& sc = scenes[scene_of_block(scenes, n_scenes, b)];
        int id[3];
        block_node_coords<D>(sc, b - sc.block_off, lane, id[0], id[1], id[2]);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        bool in_grid = id[0] < sc.n[0] && id[1] < sc.n[1] && (D == 2 || id[2] < sc.n[2]);
#pragma unroll 1
        for (int ox = 0; ox < 3; ++ox)
#pragma unroll 1
            for (int oy = 0; oy < 3; ++oy)
#pragma unroll 1
                for (int oz = 0; oz < (D == 3 ? 3 : 1); ++oz) {
                    const int bx = id[0] - ox, by = id[1] - oy, bz = D == 3 ? id[2] - oz : 0;
                    if (!in_grid || bx < 0 || by < 0 || bz < 0) continue;
                    const long long cell = node_index<D>(sc, bx, by, bz);
                    const int j1 = cell_end[cell];
                    const int o[3] = {ox, oy, oz};
                    for (int j = cell_start[cell]; j < j1; ++j) {
                        float r[SP::STRIDE];
#pragma unroll
                        for (int q = 0; q < SP::STRIDE / 4; ++q) {
                            const float4 v = src[(long long)j * (SP::STRIDE / 4) + q];
                            r[4 * q] = v.x;
                            r[4 * q + 1] = v.y;
                            r[4 * q + 2] = v.z;
                            r[4 * q + 3] = v.w;
                        }
                        Stencil<D> st;
                        P2GSource<D> s;
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            st.fx[a] = r[SP::FX + a];
                            s.mv[a] = r[SP::MV + a];
                        }
#pragma unroll
                        for (int k = 0; k < D * D; ++k) {
                            s.mC[k] = r[SP::MC + k];
                            s.A[k] = r[SP::A + k];
                        }
                        s.m = r[SP::M];
                        const float4 c = p2g_node<D>(st, s, o, sc.h, sc.inv_h);
                        acc[0] += c.x;
                        acc[1] += c.y;
                        acc[2] += c.z;
                        acc[3] += c.w;
                    }
                }
        grid_mom[(long long)b * 64 + lane] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    }
}

}  // namespace mpm
