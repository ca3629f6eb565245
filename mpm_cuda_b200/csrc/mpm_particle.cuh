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
    // quadratic B-spline weight and derivative (d/dx in cell units) of node
    // base + k along axis a, recomputed from fx where used (the same
    // arithmetic as axis_weights) instead of held in 18 registers
    __device__ __forceinline__ float w(int a, int k) const {
        const float f = fx[a];
        if (k == 0) {
            const float t0 = 1.5f - f;
            return 0.5f * t0 * t0;
        }
        if (k == 1) {
            const float t1 = f - 1.f;
            return 0.75f - t1 * t1;
        }
        const float t2 = f - 0.5f;
        return 0.5f * t2 * t2;
    }
    __device__ __forceinline__ float dw(int a, int k) const {
        const float f = fx[a];
        if (k == 0) return -(1.5f - f);
        if (k == 1) return -2.f * (f - 1.f);
        return f - 0.5f;
    }
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
        // base > n - 3 rather than base + 2 >= n: a huge finite coordinate
        // converts to INT_MAX, and base + 2 would wrap around
        if (ax.base < 0 || ax.base > sc.n[a] - 3) {
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

// MAT >= 0 compiles only that material's branch (the caller guarantees
// g.type == MAT); MAT = -1 dispatches on g.type at run time.
template <int MAT>
__device__ __forceinline__ bool is_mat(const GroupParams& g, int m) {
    return MAT >= 0 ? MAT == m : g.type == m;
}

template <int D, int MAT = -1>
__device__ __forceinline__ void particle_stress_source(const float* v, const float* C, const float* F,
                                                       float aux, const GroupParams& g, float dt,
                                                       P2GSource<D>& src) {
    float tau[D * D];
    if (is_mat<MAT>(g, WATER)) {
        // p = K (J^-gamma - 1) (MPMCUDA.cu:353, MPMWater.py:92); tau_eff = -p J I
        const float J = aux;
        const float p = g.bulk_k * (powf(J, -g.gamma) - 1.f);
#pragma unroll
        for (int i = 0; i < D * D; ++i) tau[i] = (i % (D + 1) == 0) ? -p * J : 0.f;
    } else {
        float mu = g.mu, la = g.lambda;
        if (is_mat<MAT>(g, SNOW)) {
            // hardening exp(xi (1 - Jp)), Jp = det Fp (MPMCUDA.cu:342-347)
            const float hc = expf(g.xi * (1.f - aux));
            mu *= hc;
            la *= hc;
        }
        kirchhoff_fcr<D>(F, mu, la, tau);
    }
    const float k = -dt * g.p_vol;
#pragma unroll
    for (int i = 0; i < D * D; ++i) {
        src.A[i] = k * tau[i];
        src.mC[i] = g.p_mass * C[i];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) src.mv[a] = g.p_mass * v[a];
    src.m = g.p_mass;
}

// the same with the scene's current substep
template <int D, int MAT = -1>
__device__ __forceinline__ void particle_stress_source(const float* v, const float* C, const float* F,
                                                       float aux, const GroupParams& g, const SceneParams& sc,
                                                       P2GSource<D>& src) {
    particle_stress_source<D, MAT>(v, C, F, aux, g, sc.dt, src);
}

// Left singular vectors and clamped singular values of snow's new elastic F
// (Fe = U diag(s) V^T), kept by material_update for the stress of the next
// P2G: tau(Fe) = U diag(2 mu s (s - 1)) U^T + lambda J (J - 1) I, J = prod s,
// needs no second decomposition.
template <int D>
struct ElasticSVD {
    float U[D * D];
    float s[D];
};

// Snow's source from the decomposition its plasticity step kept (equal to
// particle_stress_source of Fe = U diag(s) V^T): hardening exp(xi (1 - Jp))
// (MPMCUDA.cu:342-347) and the fixed-corotated stress of U, s.
template <int D>
__device__ __forceinline__ void snow_stress_source(const float* v, const float* C, const ElasticSVD<D>& e,
                                                   float aux, const GroupParams& g, float dt, P2GSource<D>& src) {
    const float hc = expf(g.xi * (1.f - aux));
    const float mu = g.mu * hc, la = g.lambda * hc;
    float J = 1.f, dg[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        J *= e.s[k];
        dg[k] = 2.f * mu * e.s[k] * (e.s[k] - 1.f);
    }
    const float iso = la * J * (J - 1.f);
    const float kf = -dt * g.p_vol;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float acc = (i == j) ? iso : 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) acc = fmaf(e.U[i * D + k] * dg[k], e.U[j * D + k], acc);
            src.A[i * D + j] = kf * acc;
            src.mC[i * D + j] = g.p_mass * C[i * D + j];
        }
#pragma unroll
    for (int a = 0; a < D; ++a) src.mv[a] = g.p_mass * v[a];
    src.m = g.p_mass;
}

// the same source from a given Kirchhoff stress (the surrogate path)
template <int D>
__device__ __forceinline__ void source_from_tau(const float* v, const float* C, const float* tau, const GroupParams& g,
                                                float dt, P2GSource<D>& src) {
    const float k = -dt * g.p_vol;
#pragma unroll
    for (int i = 0; i < D * D; ++i) {
        src.A[i] = k * tau[i];
        src.mC[i] = g.p_mass * C[i];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) src.mv[a] = g.p_mass * v[a];
    src.m = g.p_mass;
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
        wa[a] = st.w(a, o[a]);
        dwa[a] = st.dw(a, o[a]);
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

// ------------------------------------------------ factorised stencil loops
//
// The stencil weight of node o is separable, w(o) = wx[ox] wy[oy] wz[oz], so
// the G2P sums are contracted one axis at a time.  Per velocity component,
// with per-axis vectors w, wo = w * o and dw:
//   z:  A0 = sum wz v,  A1 = sum wo_z v,  A2 = sum dwz v           (per ox, oy)
//   y:  B00 = sum wy A0, B10 = sum wo_y A0, B20 = sum dwy A0,
//       B01 = sum wy A1, B02 = sum wy A2                            (per ox)
//   x:  v = sum wx B00, Sx = sum wo_x B00, Gx = sum dwx B00,
//       Sy = sum wx B10, Gy = sum wx B20, Sz = sum wx B01, Gz = sum wx B02
// giving v = sum w v_i, S_b = sum w v_i o_b and G_b = h sum v_i dw/dx_b;
// then B_ab = S_b[a] - fx_b v[a] (C = 4/h B) and grad v_ab = G_b[a] / h.
// About half the multiply-adds of the node-by-node form.
template <int D, class Fetch>
__device__ __forceinline__ void g2p_gather(const Stencil<D>& st, float inv_h, Fetch fetch, G2PAcc<D>& out) {
    float v[3] = {0.f, 0.f, 0.f}, S[3][3], G[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            S[a][b] = 0.f;
            G[a][b] = 0.f;
        }
    if constexpr (D == 3) {
        // Components x and y as one pair on the paired FP32 instructions of
        // sm_100 (FFMA2: two independent lanes per instruction, each rounded
        // like fmaf), z scalar.  A "3-vector" below is a (float2 xy, float z).
        struct V3 {
            float2 xy;
            float z;
        };
        auto zero = [] { return V3{make_float2(0.f, 0.f), 0.f}; };
        // acc + s * x, per component
        auto fma3 = [](float s, const V3& x, const V3& acc) {
            return V3{__ffma2_rn(make_float2(s, s), x.xy, acc.xy), fmaf(s, x.z, acc.z)};
        };
        V3 vs = zero(), Sv[3] = {zero(), zero(), zero()}, Gv[3] = {zero(), zero(), zero()};
        // both outer loops stay rolled (9 copies of the z row instead of 27):
        // smaller code, fewer instruction-fetch stalls in the fused kernels
#pragma unroll 1
        for (int ox = 0; ox < 3; ++ox) {
            V3 B00 = zero(), B10 = zero(), B20 = zero(), B01 = zero(), B02 = zero();
            // the y loop stays rolled: fully unrolled, the 27 hoisted tile
            // loads and the partial sums exceed the register budget of the
            // high-occupancy launch configurations and spill
#pragma unroll 1
            for (int oy = 0; oy < 3; ++oy) {
                V3 A0 = zero(), A1 = zero(), A2 = zero();
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    const float4 g = fetch(ox, oy, oz);
                    const V3 vi{make_float2(g.x, g.y), g.z};
                    const float wz = st.w(2, oz), dz = st.dw(2, oz);
                    A0 = fma3(wz, vi, A0);
                    if (oz > 0) A1 = fma3((float)oz * wz, vi, A1);
                    A2 = fma3(dz, vi, A2);
                }
                const float wy = st.w(1, oy), dy = st.dw(1, oy), wyo = (float)oy * wy;
                B00 = fma3(wy, A0, B00);
                if (oy > 0) B10 = fma3(wyo, A0, B10);
                B20 = fma3(dy, A0, B20);
                B01 = fma3(wy, A1, B01);
                B02 = fma3(wy, A2, B02);
            }
            const float wx = st.w(0, ox), dx = st.dw(0, ox), wxo = (float)ox * wx;
            vs = fma3(wx, B00, vs);
            if (ox > 0) Sv[0] = fma3(wxo, B00, Sv[0]);
            Gv[0] = fma3(dx, B00, Gv[0]);
            Sv[1] = fma3(wx, B10, Sv[1]);
            Gv[1] = fma3(wx, B20, Gv[1]);
            Sv[2] = fma3(wx, B01, Sv[2]);
            Gv[2] = fma3(wx, B02, Gv[2]);
        }
        v[0] = vs.xy.x;
        v[1] = vs.xy.y;
        v[2] = vs.z;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            S[0][b] = Sv[b].xy.x;
            S[1][b] = Sv[b].xy.y;
            S[2][b] = Sv[b].z;
            G[0][b] = Gv[b].xy.x;
            G[1][b] = Gv[b].xy.y;
            G[2][b] = Gv[b].z;
        }
    } else {
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            float A0[2] = {0.f, 0.f}, A1[2] = {0.f, 0.f}, A2[2] = {0.f, 0.f};
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float4 g = fetch(ox, oy, 0);
                const float vi[2] = {g.x, g.y};
                const float wy = st.w(1, oy), dy = st.dw(1, oy);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    A0[c] = fmaf(wy, vi[c], A0[c]);
                    if (oy > 0) A1[c] = fmaf((float)oy * wy, vi[c], A1[c]);
                    A2[c] = fmaf(dy, vi[c], A2[c]);
                }
            }
            const float wx = st.w(0, ox), dx = st.dw(0, ox), wxo = (float)ox * wx;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                v[c] = fmaf(wx, A0[c], v[c]);
                if (ox > 0) S[c][0] = fmaf(wxo, A0[c], S[c][0]);
                G[c][0] = fmaf(dx, A0[c], G[c][0]);
                S[c][1] = fmaf(wx, A1[c], S[c][1]);
                G[c][1] = fmaf(wx, A2[c], G[c][1]);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
        out.v[a] = v[a];
#pragma unroll
        for (int b = 0; b < D; ++b) {
            out.B[a * D + b] = fmaf(-st.fx[b], v[a], S[a][b]);
            out.G[a * D + b] = inv_h * G[a][b];
        }
    }
}

// P2G contributions of one particle to its 3^D nodes, with the separable
// parts precomputed per stencil row.  Node value for component c:
//   w (alpha_c + sum_b beta_cb o_b) + sum_b A'_cb g_b(o),
// alpha = m v - h (m C) fx, beta = h m C, A' = A / h, g_b = dw_b prod_{a!=b} w_a.
// In 3D, with P = wx wy per (ox, oy) row, the value factors over z as
//   wz (P (lin_c + oz beta_c2) + K_c) + dwz P A'_c2,
// lin_c = alpha_c + ox beta_c0 + oy beta_c1, K_c = A'_c0 dwx wy + A'_c1 wx dwy:
// per row U_c = P lin_c + K_c, V_c = P beta_c2, W_c = P A'_c2, then per node
// two operations a component (offsets 0, 1, 2 as no-op, add, fma).
// emit(ox, oy, oz, float4(momentum, mass)) receives each node's value.
template <int D, class Emit>
__device__ __forceinline__ void p2g_scatter(const Stencil<D>& st, const P2GSource<D>& src, float h, float inv_h,
                                            Emit emit) {
    float alpha[D], beta[D][D], Ap[D][D];
#pragma unroll
    for (int c = 0; c < D; ++c) {
        float a0 = src.mv[c];
#pragma unroll
        for (int b = 0; b < D; ++b) {
            a0 = fmaf(-h * src.mC[c * D + b], st.fx[b], a0);
            beta[c][b] = h * src.mC[c * D + b];
            Ap[c][b] = inv_h * src.A[c * D + b];
        }
        alpha[c] = a0;
    }
    if constexpr (D == 3) {
        // The x and y components as one pair on the paired FP32 instructions
        // of sm_100 (FFMA2 / FMUL2 / FADD2: two independent lanes per
        // instruction, each rounded like its scalar form); z and the mass stay
        // scalar.
        float2 beta_xy[3], Ap_xy[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            beta_xy[b] = make_float2(beta[0][b], beta[1][b]);
            Ap_xy[b] = make_float2(Ap[0][b], Ap[1][b]);
        }
        const float2 alpha_xy = make_float2(alpha[0], alpha[1]);
        // x + k b for a stencil offset k = 0, 1, 2 without a multiply by 0 or 1
        auto off = [](float x, float b, int k) { return k == 0 ? x : (k == 1 ? x + b : fmaf(2.f, b, x)); };
        auto off2 = [](float2 x, float2 b, int k) {
            return k == 0 ? x : (k == 1 ? __fadd2_rn(x, b) : __ffma2_rn(make_float2(2.f, 2.f), b, x));
        };
        auto dup = [](float s) { return make_float2(s, s); };
#pragma unroll
        for (int ox = 0; ox < 3; ++ox)
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float wx = st.w(0, ox), wy = st.w(1, oy);
                const float P = wx * wy, Qx = st.dw(0, ox) * wy, Qy = wx * st.dw(1, oy);
                const float Pm = P * src.m;
                const float2 P2 = dup(P);
                const float2 lin_xy = off2(off2(alpha_xy, beta_xy[0], ox), beta_xy[1], oy);
                const float2 U_xy =
                    __ffma2_rn(P2, lin_xy, __ffma2_rn(Ap_xy[1], dup(Qy), __fmul2_rn(Ap_xy[0], dup(Qx))));
                const float2 V_xy = __fmul2_rn(P2, beta_xy[2]), W_xy = __fmul2_rn(P2, Ap_xy[2]);
                const float lin_z = off(off(alpha[2], beta[2][0], ox), beta[2][1], oy);
                const float U_z = fmaf(P, lin_z, fmaf(Ap[2][1], Qy, Ap[2][0] * Qx));
                const float V_z = P * beta[2][2], W_z = P * Ap[2][2];
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    const float wz = st.w(2, oz), dz = st.dw(2, oz);
                    const float2 o_xy = __ffma2_rn(dup(wz), off2(U_xy, V_xy, oz), __fmul2_rn(dup(dz), W_xy));
                    emit(ox, oy, oz, make_float4(o_xy.x, o_xy.y, fmaf(wz, off(U_z, V_z, oz), dz * W_z), Pm * wz));
                }
            }
    } else {
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const float wx = st.w(0, ox), dx = st.dw(0, ox);
            float lin[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) lin[c] = fmaf(beta[c][0], (float)ox, alpha[c]);
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float wy = st.w(1, oy);
                const float w = wx * wy, gx = dx * wy, gy = wx * st.dw(1, oy);
                float out[2];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float t = fmaf(beta[c][1], (float)oy, lin[c]);
                    out[c] = fmaf(Ap[c][1], gy, fmaf(Ap[c][0], gx, w * t));
                }
                emit(ox, oy, 0, make_float4(out[0], out[1], 0.f, w * src.m));
            }
        }
    }
}

// |v| plus the material's signal speed, for adaptive dt.  Snow's hardening
// scales its stiffness by exp(xi (1 - Jp)), so its wave speed by the square
// root of that.
template <int D, int MAT>
__device__ __forceinline__ float signal_speed(const float* v, const GroupParams& g, float aux) {
    float vv = 0.f;
#pragma unroll
    for (int a = 0; a < D; ++a) vv = fmaf(v[a], v[a], vv);
    float c = g.wave;
    if (MAT == SNOW) c *= expf(0.5f * g.xi * (1.f - aux));
    return sqrtf(vv) + c;
}

// Material update after G2P (MPMCUDA.cu:588-713, MPMSnow.py:135-150,
// MPMWater.py:138).  Updates F / aux in place, returns error bits.
template <int D, int MAT = -1>
__device__ __forceinline__ unsigned material_update(const G2PAcc<D>& acc, float dt,
                                                    const GroupParams& g, float* F, float& aux,
                                                    ElasticSVD<D>* keep = nullptr) {
    unsigned err = 0;
    if (is_mat<MAT>(g, WATER)) {
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
    if (is_mat<MAT>(g, SNOW)) {
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
        if (keep) {
#pragma unroll
            for (int k = 0; k < D * D; ++k) keep->U[k] = U[k];
#pragma unroll
            for (int k = 0; k < D; ++k) keep->s[k] = s[k];
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
