// Unbinned kernels: one thread per particle, stencil traffic straight to
// global memory.  Used for the first P2G of a scene, as the reference-order
// path of the deterministic mode's checks, and as the fallback when the
// binned path is disabled.
#pragma once

#include "mpm_grid.cuh"
#include "mpm_particle.cuh"

namespace mpm {

template <int D>
__device__ __forceinline__ void load_particle(const ParticleBuf& pb, long long i, float* x, float* v,
                                              float* C, float* F, float& aux) {
    using P = Planes<D>;
    const float* s = pb.s;
    const long long cap = pb.cap;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        x[a] = s[(P::X + a) * cap + i];
        v[a] = s[(P::V + a) * cap + i];
    }
#pragma unroll
    for (int k = 0; k < D * D; ++k) {
        C[k] = s[(P::C + k) * cap + i];
        F[k] = s[(P::F + k) * cap + i];
    }
    aux = s[P::AUX * cap + i];
}

// P2G straight to global memory with float4 vector atomics (MPMCUDA.cu:310-433)
template <int D>
__global__ void __launch_bounds__(128) k_p2g_direct(ParticleBuf pb, long long n,
                                                    const GroupParams* __restrict__ groups,
                                                    const SceneParams* __restrict__ scenes,
                                                    float4* __restrict__ grid, unsigned* err_word) {
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
    const StencilIndex<D> ix(sc, st.base);
    float4* gs = grid + sc.node_off;
    p2g_scatter<D>(st, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 c) {
        atomicAdd(&gs[ix(ox, oy, D == 3 ? oz : 0)], c);
    });
}

// Dense grid update over every node of every scene (VelUpdate,
// MPMCUDA.cu:435-472).  Writes (velocity, mass) into `vel` and, when
// `clear_src`, zeroes the momentum buffer for the next P2G.
template <int D>
__global__ void __launch_bounds__(256) k_grid_update_dense(float4* __restrict__ mom, float4* __restrict__ vel,
                                                           long long total_blocks,
                                                           const SceneParams* __restrict__ scenes,
                                                           int n_scenes, int clear_src) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long b = t >> 6;
    const int in = (int)(t & 63);
    if (b >= total_blocks) return;
    const int s = scene_of_block(scenes, n_scenes, b);
    const SceneParams& sc = scenes[s];
    int ix, iy, iz;
    block_node_coords<D>(sc, b - sc.block_off, in, ix, iy, iz);
    const long long gi = b * 64 + in;
    const float4 g = mom[gi];
    vel[gi] = grid_node_update<D>(g, sc, ix, iy, iz);
    if (clear_src) mom[gi] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// G2P + F update + advection straight from global memory
// (InterpolateAndMove, MPMCUDA.cu:474-741).
template <int D>
__global__ void __launch_bounds__(128) k_g2p_direct(ParticleBuf pb, long long n,
                                                    const GroupParams* __restrict__ groups,
                                                    const SceneParams* __restrict__ scenes,
                                                    const float4* __restrict__ grid, unsigned* err_word) {
    using P = Planes<D>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* s = pb.s;
    const long long cap = pb.cap;
    float x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x[a] = s[(P::X + a) * cap + i];
    const GroupParams g = groups[pb.grp[i]];
    const SceneParams& sc = scenes[g.scene];
    unsigned err = 0;
    Stencil<D> st;
    if (!make_stencil<D>(x, sc, st, err)) {
        atomicOr(err_word, err);
        return;
    }
    G2PAcc<D> acc;
    const float inv_h = sc.inv_h;
    const StencilIndex<D> ix(sc, st.base);
    const float4* gs = grid + sc.node_off;
    g2p_gather<D>(st, inv_h, [&](int ox, int oy, int oz) { return __ldg(&gs[ix(ox, oy, D == 3 ? oz : 0)]); }, acc);
    float F[D * D], aux = s[P::AUX * cap + i];
    if (g.type != WATER) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) F[k] = s[(P::F + k) * cap + i];
    }
    err |= material_update<D>(acc, sc.dt, g, F, aux);
    if (g.type != WATER) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) s[(P::F + k) * cap + i] = F[k];
    }
    s[P::AUX * cap + i] = aux;
    const float c4 = 4.f * inv_h;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const float xn = fmaf(sc.dt, acc.v[a], x[a]);
        if (!isfinite(xn)) err |= ERR_NONFINITE;
        s[(P::X + a) * cap + i] = xn;
        s[(P::V + a) * cap + i] = acc.v[a];
#pragma unroll
        for (int b = 0; b < D; ++b) s[(P::C + a * D + b) * cap + i] = c4 * acc.B[a * D + b];
    }
    if (err) atomicOr(err_word, err);
}

}  // namespace mpm
