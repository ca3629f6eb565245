// Warp-level BF16 tensor-core MLP for the learned stress surrogate:
// 10 -> 64 -> 64 -> 9 with SiLU, BF16 weights and activations, FP32
// accumulation, evaluated 32 samples per warp with
// mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32.
//
// What the network predicts.  The fixed-corotated Kirchhoff stress
// (MPMCUDA.cu:229-264) is tau = 2 mu (F - R) F^T + lambda J (J - 1) I.  With
// F = R S (polar), R F^T = R S R^T = sqrt(B), B = F F^T, so
//   tau = 2 mu (B - sqrt(B)) + lambda J (J - 1) I,
// and the SVD is only needed for sqrt(B).  With X = B - I,
//   sqrt(B) = I + X/2 - X^2/8 + r(X),
// where the residual r(X) is O(|X|^3) and is what the network learns:
// inputs (X / in_scale as 9 entries, (J - 1) / in_scale), outputs r / out_scale
// as a full 3x3 matrix.  Then
//   tau = mu (X + X^2/4 - 2 sym(r)) + lambda J (J - 1) I,
// which is symmetric by construction and does not depend on lambda/mu, so one
// network serves every Poisson ratio (and snow's hardened mu, lambda).  The
// skew part of the predicted r (zero for the exact residual) is the error
// estimate.  B is invariant under rotations of the material frame, and a rigid
// rotation leaves X at zero, so the inputs carry strain, not rotation.
//
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace mpm {
namespace mlp {

constexpr int IN = 10, IN_PAD = 16, HID = 64, OUT = 9, OUT_PAD = 16;
constexpr int S16 = 24, S64 = 72;  // padded row strides (bf16 elements)

// BF16 weights of the forward pass (device and shared memory use the same
// layout); 15,168 bytes, a multiple of 16
struct Forward {
    __nv_bfloat16 w1[HID * S16];       // [64 x 16]
    __nv_bfloat16 w2[HID * S64];       // [64 x 64]
    __nv_bfloat16 w3[OUT_PAD * S64];   // [16 x 64]
    float b1[HID], b2[HID], b3[OUT_PAD];
};
// plus the transposed copies the backward pass multiplies with
struct Weights {
    Forward f;
    __nv_bfloat16 w2t[HID * S64];      // W2 transposed
    __nv_bfloat16 w3t[HID * S16];      // W3 transposed [64 x 16]
};
static_assert(sizeof(Forward) % 16 == 0 && sizeof(Weights) % 16 == 0, "16-byte copies");

// model constants that travel with the weights
struct Meta {
    float in_scale;    // features: X / in_scale, (J - 1) / in_scale
    float out_scale;   // residual r = out_scale * y
    float env_c;       // envelope: max |X| entry seen in training
    float env_jlo, env_jhi;  // envelope: J range seen in training
    float skew_tol;    // error estimate: 2 out_scale |skew(y)| above skew_tol (|tau/mu| + tau_floor) -> fallback
    float tau_floor;   // absolute floor of that test (units of tau / mu)
    float pad;
};

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma16816(float* c, const unsigned* a, unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment of n-tile `nt`, k-tile `kt` of a row-major [N x K] weight with row stride S
template <int S>
__device__ __forceinline__ void load_b(const __nv_bfloat16* w, int nt, int kt, int lane, unsigned& b0, unsigned& b1) {
    const int g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* row = w + (nt * 8 + g) * S + kt * 16 + 2 * t;
    b0 = *reinterpret_cast<const unsigned*>(row);
    b1 = *reinterpret_cast<const unsigned*>(row + 8);
}

// SiLU x * sigmoid(x), sigmoid(x) = (1 + tanh(x / 2)) / 2 with the hardware
// tanh approximation (PTX tanh.approx.f32); training uses the same function.
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu(float x) {
    const float s = fmaf(0.5f, tanh_approx(0.5f * x), 0.5f);
    return x * s;
}
// d silu / dx = s + x s (1 - s)
__device__ __forceinline__ float silu_grad(float x) {
    const float s = fmaf(0.5f, tanh_approx(0.5f * x), 0.5f);
    return fmaf(x * s, 1.f - s, s);
}

// A fragments of one 16-row tile of the input (row stride 16 floats)
__device__ __forceinline__ void load_a_input(const float* x, int lane, unsigned* a) {
    const int g = lane >> 2, t = lane & 3;
    const float* r0 = x + g * IN_PAD;
    const float* r1 = x + (g + 8) * IN_PAD;
    a[0] = pack_bf16(r0[2 * t], r0[2 * t + 1]);
    a[1] = pack_bf16(r1[2 * t], r1[2 * t + 1]);
    a[2] = pack_bf16(r0[2 * t + 8], r0[2 * t + 9]);
    a[3] = pack_bf16(r1[2 * t + 8], r1[2 * t + 9]);
}

// SiLU of two values on the packed BF16 pipe: z rounded to bf16x2, then
// z * (1/2 + tanh(z/2)/2) with tanh.approx.bf16x2, fma.rn.bf16x2 and
// mul.rn.bf16x2; a -> low half, b -> high half (the A-fragment order).  Half
// the MUFU operations of two FP32 tanh; the result is a BF16 MMA operand
// anyway.
__device__ __forceinline__ unsigned silu2_bf16(float a, float b) {
    const unsigned z = pack_bf16(a, b);
    const unsigned half = 0x3f003f00u;  // (0.5, 0.5)
    unsigned h, t, s, y;
    asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(h) : "r"(z), "r"(half));
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
    asm("fma.rn.bf16x2 %0, %1, %2, %2;" : "=r"(s) : "r"(t), "r"(half));
    asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(y) : "r"(z), "r"(s));
    return y;
}

// accumulator tiles (nt, nt+1) -> SiLU -> A fragment of one 16-wide k slice
__device__ __forceinline__ void acc_to_a_silu(const float* c0, const float* c1, unsigned* a) {
    a[0] = silu2_bf16(c0[0], c0[1]);
    a[1] = silu2_bf16(c0[2], c0[3]);
    a[2] = silu2_bf16(c1[0], c1[1]);
    a[3] = silu2_bf16(c1[2], c1[3]);
}

// accumulator tiles (nt, nt+1) -> A fragment of one 16-wide k slice, after f
template <class Fn>
__device__ __forceinline__ void acc_to_a(const float* c0, const float* c1, unsigned* a, Fn f) {
    a[0] = pack_bf16(f(c0[0]), f(c0[1]));
    a[1] = pack_bf16(f(c0[2]), f(c0[3]));
    a[2] = pack_bf16(f(c1[0]), f(c1[1]));
    a[3] = pack_bf16(f(c1[2]), f(c1[3]));
}

// accumulators initialised with the bias of their columns
template <int NT>
__device__ __forceinline__ void init_bias(float (*acc)[4], const float* b, int lane) {
    const int t = lane & 3;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        acc[j][0] = acc[j][2] = b[8 * j + 2 * t];
        acc[j][1] = acc[j][3] = b[8 * j + 2 * t + 1];
    }
}

// Forward pass of one 16-row tile.  x: 16 rows of 16 features, y: 16 rows of
// 16 outputs (columns >= 9 are padding), both with row stride XS floats in
// shared memory (an odd XS keeps the per-particle row accesses free of bank
// conflicts); y may alias x.  All 32 lanes of the warp must call it together.
template <int XS = IN_PAD>
__device__ __forceinline__ void forward_tile(const Forward& W, const float* x, float* y, int lane) {
    const int g = lane >> 2, t = lane & 3;
    unsigned a[4];
    {
        const float* r0 = x + g * XS;
        const float* r1 = x + (g + 8) * XS;
        a[0] = pack_bf16(r0[2 * t], r0[2 * t + 1]);
        a[1] = pack_bf16(r1[2 * t], r1[2 * t + 1]);
        a[2] = pack_bf16(r0[2 * t + 8], r0[2 * t + 9]);
        a[3] = pack_bf16(r1[2 * t + 8], r1[2 * t + 9]);
    }
    float h1[8][4];
    init_bias<8>(h1, W.b1, lane);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        unsigned b0, b1;
        load_b<S16>(W.w1, j, 0, lane, b0, b1);
        mma16816(h1[j], a, b0, b1);
    }
    unsigned a2[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) acc_to_a_silu(h1[2 * kk], h1[2 * kk + 1], a2[kk]);
    float h2[8][4];
    init_bias<8>(h2, W.b2, lane);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            unsigned b0, b1;
            load_b<S64>(W.w2, j, kk, lane, b0, b1);
            mma16816(h2[j], a2[kk], b0, b1);
        }
    unsigned a3[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) acc_to_a_silu(h2[2 * kk], h2[2 * kk + 1], a3[kk]);
    float o[2][4];
    init_bias<2>(o, W.b3, lane);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            unsigned b0, b1;
            load_b<S64>(W.w3, j, kk, lane, b0, b1);
            mma16816(o[j], a3[kk], b0, b1);
        }
    __syncwarp();  // y may alias x: every lane has read its inputs
    // only the 9 real outputs are stored (columns 0..8)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int col = 8 * j + 2 * t + (e & 1), row = (e < 2) ? g : g + 8;
            if (col < OUT) y[row * XS + col] = o[j][e];
        }
}

// ------------------------------------------------------ features / stress --

// X = F F^T - I (row-major, symmetric)
__device__ __forceinline__ void strain_b(const float* F, float* X) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const float c = fmaf(F[i * 3 + 0], F[j * 3 + 0], fmaf(F[i * 3 + 1], F[j * 3 + 1], F[i * 3 + 2] * F[j * 3 + 2]));
            X[i * 3 + j] = X[j * 3 + i] = c - (i == j ? 1.f : 0.f);
        }
}

// network input of one deformation gradient (J = det F)
__device__ __forceinline__ void features(const float* F, float J, const Meta& m, float* x) {
    const float s = 1.f / m.in_scale;
    float X[9];
    strain_b(F, X);
#pragma unroll
    for (int k = 0; k < 9; ++k) x[k] = X[k] * s;
    x[9] = (J - 1.f) * s;
#pragma unroll
    for (int k = 10; k < IN_PAD; ++k) x[k] = 0.f;
}

// inside the training envelope: max |X| entry and J range
__device__ __forceinline__ bool in_envelope(const float* F, float J, const Meta& m) {
    if (!(J >= m.env_jlo && J <= m.env_jhi)) return false;
    float X[9];
    strain_b(F, X);
    float e = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) e = fmaxf(e, fabsf(X[k]));
    return e <= m.env_c;
}

// Kirchhoff stress from the prediction y (9 outputs):
//   tau = mu (X + X^2/4 - 2 out_scale sym(y)) + lambda J (J - 1) I.
// Returns false when the error estimate is above the model's tolerance.
__device__ __forceinline__ bool tau_from_prediction(const float* y, const float* F, float J, float mu, float lambda,
                                                    const Meta& m, float* tau) {
    float X[9];
    strain_b(F, X);
    float nrm = 0.f, skew = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float x2 = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) x2 = fmaf(X[i * 3 + k], X[k * 3 + j], x2);
            const float r = m.out_scale * (y[i * 3 + j] + y[j * 3 + i]);  // 2 out_scale sym(y)
            const float d = m.out_scale * (y[i * 3 + j] - y[j * 3 + i]);  // 2 out_scale skew(y)
            const float t = fmaf(0.25f, x2, X[i * 3 + j]) - r;          // tau / mu without the volume term
            tau[i * 3 + j] = mu * t;
            nrm = fmaf(t, t, nrm);
            skew = fmaf(d, d, skew);
        }
    const float vol = lambda * J * (J - 1.f);
    tau[0] += vol;
    tau[4] += vol;
    tau[8] += vol;
    const float lim = m.skew_tol * (sqrtf(nrm) + m.tau_floor);
    return skew <= lim * lim;
}

// training / evaluation target: the residual r = sqrt(B) - I - X/2 + X^2/8 of
// F = U diag(s) V^T, computed spectrally as U diag(f(s)) U^T with
// f(s) = s - 1 - (s^2 - 1)/2 + (s^2 - 1)^2/8 (s >= 0)
__device__ __forceinline__ void residual_target(const float* U, const float* s, float* r) {
    float f[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float a = fabsf(s[k]), q = fmaf(a, a, -1.f);
        f[k] = fmaf(0.125f * q, q, fmaf(-0.5f, q, a - 1.f));
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r[i * 3 + j] = fmaf(U[i * 3 + 0] * f[0], U[j * 3 + 0],
                                fmaf(U[i * 3 + 1] * f[1], U[j * 3 + 1], U[i * 3 + 2] * f[2] * U[j * 3 + 2]));
}

}  // namespace mlp
}  // namespace mpm
