// Fused substep with the learned stress (MPM_STRESS_SURROGATE), 3D jello.
// (Snow's exact stress costs no decomposition of its own: it reuses the one of
// its plasticity clamp, so snow keeps the plain kernel.)  Same pass as
// k_g2p2g (G2P, particle update, stress, P2G of the next substep) with the
// stress of eligible particles taken from the BF16 MLP (mpm_mlp.cuh) instead
// of the decomposition in kirchhoff_fcr (MPMCUDA.cu:229-264):
//   1. every thread: G2P, update, store the new state (v and C deferred as in
//      k_g2p2g), keep x, v, C, F in its shared stash row and write its network
//      input (X = F F^T - I, J - 1) to its network row;
//   2. every warp: forward pass of its 32 rows on the tensor cores, in place;
//   3. every thread: stress from the prediction when F is inside the training
//      envelope and the error estimate is below tolerance, else from the
//      decomposition; scatter.
// The stash keeps the network's registers from adding to the G2P registers
// without a round trip of the state through L2.  Launched with programmatic
// dependent launch like k_g2p2g; FIXED: the scene from the kernel parameters.
#pragma once

#include "mpm_kernels_binned.cuh"
#include "mpm_mlp.cuh"

namespace mpm {

// row strides (floats) of the per-particle network rows and stash rows in
// shared memory: odd, so the rows of a warp's 32 particles start in 32
// different banks
constexpr int kSurRowStride = mlp::IN_PAD + 1;
constexpr int kSurStashStride = 25;  // x[3], v[3], C[9], F[9]
// dynamic shared memory of k_g2p2g_sur for a chunk size
constexpr int sur_dyn_smem(int chunk) { return chunk * (kSurRowStride + kSurStashStride) * (int)sizeof(float); }

struct SurArgs {
    const mlp::Forward* weights;
    mlp::Meta meta;
    unsigned long long* counts;  // [0] stresses from the network, [1] SVD fallbacks
};

template <int CHUNK, int MINB, bool FIXED, bool PAGED>
__global__ void __launch_bounds__(CHUNK, MINB) k_g2p2g_sur(ParticleBuf pb, const __grid_constant__ FusedArgs A,
                                                            SurArgs SA) {
    constexpr int D = 3;
    constexpr int MAT = JELLO;
    using TS = TileShape<D>;
    static_assert(CHUNK % 32 == 0, "whole warps");
    constexpr int XS = kSurRowStride, SS = kSurStashStride;
    __shared__ __align__(128) float4 tv[2][TS::VN];  // grid velocity windows (double-buffered; box-load targets)
    __shared__ int s27[2][27];                      // PAGED: the windows' physical blocks
    __shared__ __align__(16) mlp::Forward W;        // network weights
    extern __shared__ float sxy[];                  // CHUNK network rows (inputs, then outputs), CHUNK stash rows
    __shared__ unsigned touched[2];
    __shared__ int s_cn[2];
    __shared__ unsigned s_speed;  // adaptive dt: this chunk's max signal speed

    pdl_wait();     // the grid update ahead of this launch has finished
    pdl_trigger();  // the next pass may launch; it waits for this one to end
    if (A.bump_epoch && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.epoch, 1);
    {
        const int4* src = reinterpret_cast<const int4*>(SA.weights);
        int4* dst = reinterpret_cast<int4*>(&W);
        for (int k = threadIdx.x; k < (int)(sizeof(mlp::Forward) / 16); k += CHUNK) dst[k] = src[k];
    }  // published by the first barrier of chunk_loop
    const int lane = threadIdx.x & 31, w0 = threadIdx.x & ~31;
    float* row = sxy + threadIdx.x * XS;
    float* stash = sxy + CHUNK * XS + threadIdx.x * SS;
    unsigned n_net = 0, n_svd = 0;
    if (threadIdx.x == 0) s_speed = 0u;
    SpeedFlush speed;
    chunk_loop<D, CHUNK, FIXED, PAGED>(A, tv, s27, touched, s_cn,
                                       [&](const Chunk& ch, const SceneParams& sc, const int* o, const float4* w,
                                           unsigned* tb, const int* wpages) {
        unsigned speed_bits = 0u;
        // every thread runs every round (the network step is warp-synchronous)
#pragma unroll 1
        for (int r = 0; r < A.rounds; ++r) {
            const int li = (int)threadIdx.x + r * CHUNK;  // this round's particle of the chunk
            unsigned err = 0;
            bool next = false;      // the particle scatters into the next substep
            bool eligible = false;  // its group takes the network's stress
            int gi = 0;             // its group (re-read after the network: fewer live registers)
            if (li < ch.count) {
                const long long i = (long long)ch.start + li;
                float* S = pb.s;
                const long long cap = pb.cap;
                gi = pb.grp[i];
                float x[D];
#pragma unroll
                for (int a = 0; a < D; ++a) x[a] = S[(Planes<D>::X + a) * cap + i];
                Stencil<D> st;
                if (make_stencil<D>(x, sc, st, err)) {
                    G2PAcc<D> acc;
                    g2p_window<D, PAGED, FIXED && !PAGED>(st, o, w, sc, A, acc);
                    const GroupParams g = A.groups[gi];
                    float F[D * D], Cn[D * D], v[D], aux;
                    err |= update_and_store<D, MAT>(acc, sc, g, S, cap, i, x, v, Cn, F, aux, nullptr,
                                                    A.defer_vc != 0);
                    if (A.speed_max) speed_bits = max(speed_bits, __float_as_uint(signal_speed<D, MAT>(v, g, aux)));
                    Stencil<D> sn;
                    next = make_stencil<D>(x, sc, sn, err);
                    if (next) {
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            stash[a] = x[a];
                            stash[3 + a] = v[a];
                        }
#pragma unroll
                        for (int k = 0; k < D * D; ++k) {
                            stash[6 + k] = Cn[k];
                            stash[15 + k] = F[k];
                        }
                    }
                    eligible = next && g.surrogate != 0;
                    if (eligible) mlp::features(F, det<3>(F), SA.meta, row);
                }
            }
            if (!eligible) {
#pragma unroll
                for (int k = 0; k < mlp::IN_PAD; ++k) row[k] = 0.f;
            }
            __syncwarp();
            // ---- network: 32 rows per warp, two 16-row tiles, in place
            if (__any_sync(0xffffffffu, eligible)) {
                mlp::forward_tile<XS>(W, sxy + w0 * XS, sxy + w0 * XS, lane);
                mlp::forward_tile<XS>(W, sxy + (w0 + 16) * XS, sxy + (w0 + 16) * XS, lane);
            }
            __syncwarp();
            if (next) {
                float x[D], v[D], Cn[D * D], F[D * D];
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    x[a] = stash[a];
                    v[a] = stash[3 + a];
                }
#pragma unroll
                for (int k = 0; k < D * D; ++k) {
                    Cn[k] = stash[6 + k];
                    F[k] = stash[15 + k];
                }
                const GroupParams g = A.groups[gi];
                Stencil<D> sn;
                make_stencil<D>(x, sc, sn, err);  // the stencil found above
                float tau[D * D];
                bool use = false;
                if (eligible) {
                    const float J = det<3>(F);
                    use = mlp::in_envelope(F, J, SA.meta) &&
                          mlp::tau_from_prediction(row, F, J, g.mu, g.lambda, SA.meta, tau);
                }
                P2GSource<D> src;
                if (use) {
                    source_from_tau<D>(v, Cn, tau, g, sc.dt_next, src);
                    ++n_net;
                } else {
                    particle_stress_source<D, MAT>(v, Cn, F, 1.f, g, sc.dt_next, src);
                    ++n_svd;
                }
                scatter_global<D, PAGED>(sn, src, sc, o, A, tb, wpages);
            }
            if (err) atomicOr(A.err_word, err);
            __syncwarp();  // the rows are rewritten by the next round
        }
        if (A.speed_max) speed_warp_reduce(speed_bits, &s_speed);
    }, [&](int si) { speed.fold(si, &s_speed, A.speed_max); });
    speed.flush(A.speed_max);
    n_net = __reduce_add_sync(0xffffffffu, n_net);
    n_svd = __reduce_add_sync(0xffffffffu, n_svd);
    if (lane == 0 && (n_net | n_svd)) {
        atomicAdd(&SA.counts[0], (unsigned long long)n_net);
        atomicAdd(&SA.counts[1], (unsigned long long)n_svd);
    }
}

}  // namespace mpm
