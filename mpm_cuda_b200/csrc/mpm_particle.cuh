// Per-particle pieces of the substep shared by every kernel variant:
// stencil setup, the P2G contribution (momentum + stress force), the G2P
// accumulation and the material update.  All FP32, register resident.
#pragma once

#include "mpm_math.cuh"
#include "mpm_types.cuh"

namespace mpm {

template <int D>
struct Stencil {
    int base[3];
    float fx[3];
    float w[3][3];
    float dw[3][3];
};

// Returns false (and sets error bits) when the 3^D stencil leaves the grid
// or the position is not finite (the reference asserts instead,
// MPMCUDA.cu:376-386).
template <int D>
__device__ __forceinline__ bool make_stencil(const float* x, const SceneParams& sc, Stencil<D>& st,
                                             unsigned& err) {
    bool ok = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const float gx = (x[a] - sc.origin[a]) * sc.inv_h;
        if (!isfinite(gx)) {
            err |= ERR_NONFINITE;
            ok = false;
            st.base[a] = 0;
            continue;
        }
        Axis ax = axis_weights(gx);
        st.base[a] = ax.base;
        st.fx[a] = ax.fx;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            st.w[a][k] = ax.w[k];
            st.dw[a][k] = ax.dw[k];
        }
        if (ax.base < 0 || ax.base + 2 >= sc.n[a]) {
            err |= ERR_OUT_OF_GRID;
            ok = false;
        }
    }
    return ok;
}

// The affine P2G source of one particle.  Node contribution:
//   (m v_i, m_i) += (w (m v + m C dx_i) + A grad w_i,  w m)
// with dx_i = x_i - x_p and A = -dt V tau (solids) or dt V p J I (water):
//   f_ip = -V tau grad w (MPMCUDA.cu:409-411), f_ip = V p J grad w (:412-414)
template <int D>
struct P2GSource {
    float mv[D];     // m v
    float mC[D * D]; // m C
    float A[D * D];  // -dt V tau_eff
    float m;
};

template <int D>
__device__ __forceinline__ void particle_stress_source(const float* v, const float* C, const float* F,
                                                       float aux, const GroupParams& g,
                                                       const SceneParams& sc, P2GSource<D>& src) {
    float tau[D * D];
    if (g.type == WATER) {
        // p = K (J^-gamma - 1) (MPMCUDA.cu:353, MPMWater.py:92); tau_eff = -p J I
        const float J = aux;
        const float p = g.bulk_k * (powf(J, -g.gamma) - 1.f);
#pragma unroll
        for (int i = 0; i < D * D; ++i) tau[i] = (i % (D + 1) == 0) ? -p * J : 0.f;
    } else {
        float mu = g.mu, la = g.lambda;
        if (g.type == SNOW) {
            // hardening exp(xi (1 - Jp)), Jp = det Fp (MPMCUDA.cu:342-347)
            const float hc = expf(g.xi * (1.f - aux));
            mu *= hc;
            la *= hc;
        }
        kirchhoff_fcr<D>(F, mu, la, tau);
    }
    const float k = -sc.dt * g.p_vol;
#pragma unroll
    for (int i = 0; i < D * D; ++i) {
        src.A[i] = k * tau[i];
        src.mC[i] = g.p_mass * C[i];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) src.mv[a] = g.p_mass * v[a];
    src.m = g.p_mass;
}

// contribution of the source to stencil node `o` (offsets 0..2 per axis)
template <int D>
__device__ __forceinline__ float4 p2g_node(const Stencil<D>& st, const P2GSource<D>& src,
                                           const int* o, float h, float inv_h) {
    float wa[3], dwa[3];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        wa[a] = st.w[a][o[a]];
        dwa[a] = st.dw[a][o[a]];
    }
    float w = wa[0] * wa[1];
    float gw[D];
    if constexpr (D == 3) {
        w *= wa[2];
        gw[0] = inv_h * dwa[0] * wa[1] * wa[2];
        gw[1] = inv_h * wa[0] * dwa[1] * wa[2];
        gw[2] = inv_h * wa[0] * wa[1] * dwa[2];
    } else {
        gw[0] = inv_h * dwa[0] * wa[1];
        gw[1] = inv_h * wa[0] * dwa[1];
    }
    float dx[D];
#pragma unroll
    for (int a = 0; a < D; ++a) dx[a] = ((float)o[a] - st.fx[a]) * h;
    float out[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        float cdx = src.mv[a];
#pragma unroll
        for (int b = 0; b < D; ++b) cdx = fmaf(src.mC[a * D + b], dx[b], cdx);
        float f = 0.f;
#pragma unroll
        for (int b = 0; b < D; ++b) f = fmaf(src.A[a * D + b], gw[b], f);
        out[a] = fmaf(w, cdx, f);
    }
    return make_float4(out[0], out[1], out[2], w * src.m);
}

// G2P accumulators (InterpolateAndMove, MPMCUDA.cu:500-587)
template <int D>
struct G2PAcc {
    float v[D];
    float B[D * D];  // sum w v_i (o - fx)^T   (C = 4/h * B)
    float G[D * D];  // sum v_i grad w^T      (velocity gradient)
};

template <int D>
__device__ __forceinline__ void g2p_zero(G2PAcc<D>& acc) {
#pragma unroll
    for (int a = 0; a < D; ++a) acc.v[a] = 0.f;
#pragma unroll
    for (int i = 0; i < D * D; ++i) {
        acc.B[i] = 0.f;
        acc.G[i] = 0.f;
    }
}

template <int D>
__device__ __forceinline__ void g2p_node(const Stencil<D>& st, const int* o, float4 gv, float inv_h,
                                         G2PAcc<D>& acc) {
    float wa[3], dwa[3];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        wa[a] = st.w[a][o[a]];
        dwa[a] = st.dw[a][o[a]];
    }
    float w = wa[0] * wa[1];
    float gw[D];
    if constexpr (D == 3) {
        w *= wa[2];
        gw[0] = inv_h * dwa[0] * wa[1] * wa[2];
        gw[1] = inv_h * wa[0] * dwa[1] * wa[2];
        gw[2] = inv_h * wa[0] * wa[1] * dwa[2];
    } else {
        gw[0] = inv_h * dwa[0] * wa[1];
        gw[1] = inv_h * wa[0] * dwa[1];
    }
    const float vi[3] = {gv.x, gv.y, gv.z};
    float d[D];
#pragma unroll
    for (int a = 0; a < D; ++a) d[a] = (float)o[a] - st.fx[a];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const float wv = w * vi[a];
        acc.v[a] += wv;
#pragma unroll
        for (int b = 0; b < D; ++b) {
            acc.B[a * D + b] = fmaf(wv, d[b], acc.B[a * D + b]);
            acc.G[a * D + b] = fmaf(vi[a], gw[b], acc.G[a * D + b]);
        }
    }
}

// Material update after G2P (MPMCUDA.cu:588-713, MPMSnow.py:135-150,
// MPMWater.py:138).  Updates F / aux in place, returns error bits.
template <int D>
__device__ __forceinline__ unsigned material_update(const G2PAcc<D>& acc, float dt,
                                                    const GroupParams& g, float* F, float& aux) {
    unsigned err = 0;
    if (g.type == WATER) {
        float div = 0.f;
#pragma unroll
        for (int a = 0; a < D; ++a) div += acc.G[a * D + a];
        aux = fmaf(dt * div, aux, aux);  // J <- (1 + dt div v) J
        if (!(aux > 0.f)) err |= ERR_DET;
        return err;
    }
    float L[D * D];
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
        for (int b = 0; b < D; ++b) L[a * D + b] = (a == b ? 1.f : 0.f) + dt * acc.G[a * D + b];
    float Fn[D * D];
    matmul<D>(L, F, Fn);  // F <- (I + dt grad v) F
    if (g.type == SNOW) {
        // Stomakhin et al. 2013 clamp of the trial elastic F
        float U[D * D], s[D], V[D * D];
        svd<D>(Fn, U, s, V);
        const float det_trial = det<D>(Fn);
        float det_new = 1.f;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            s[k] = fminf(fmaxf(s[k], 1.f - g.theta_c), 1.f + g.theta_s);
            det_new *= s[k];
        }
        // Fe = U diag(s*) V^T
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
            for (int j = 0; j < D; ++j) {
                float acc2 = 0.f;
#pragma unroll
                for (int k = 0; k < D; ++k) acc2 = fmaf(U[i * D + k] * s[k], V[j * D + k], acc2);
                F[i * D + j] = acc2;
            }
        // det Fp_new = det(Fe_new^-1 Fe_trial Fp) = det_trial / det_new * det Fp
        aux = aux * (det_trial / det_new);
        if (!(aux > 0.f)) err |= ERR_DET;
    } else {
#pragma unroll
        for (int i = 0; i < D * D; ++i) F[i] = Fn[i];
        if (!(det<D>(F) > 0.f)) err |= ERR_DET;
    }
    return err;
}

}  // namespace mpm
