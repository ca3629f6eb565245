// Register-resident FP32 math for the MPM substep: small matrices, the 2x2 /
// 3x3 SVD with the reference's PolarSVD sign convention, the material stress
// models and the quadratic B-spline stencil.
//
// Matrices are row-major in float[9] (3D) or float[4] (2D) and live in
// registers once the callers are fully unrolled.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#define MPM_HD __host__ __device__ __forceinline__

namespace mpm {

// ---------------------------------------------------------------- helpers --

template <int D>
MPM_HD float det(const float* A) {
    if constexpr (D == 2) {
        return A[0] * A[3] - A[1] * A[2];
    } else {
        return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
               A[2] * (A[3] * A[7] - A[4] * A[6]);
    }
}

template <int D>
MPM_HD void matmul(const float* A, const float* B, float* Cm) {
    float T[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) s = fmaf(A[i * D + k], B[k * D + j], s);
            T[i * D + j] = s;
        }
#pragma unroll
    for (int i = 0; i < D * D; ++i) Cm[i] = T[i];
}

// inverse through the adjugate; caller guarantees det != 0
template <int D>
MPM_HD void inverse(const float* A, float* Ai) {
    float id = 1.f / det<D>(A);
    if constexpr (D == 2) {
        float a = A[0], b = A[1], c = A[2], d = A[3];
        Ai[0] = d * id; Ai[1] = -b * id; Ai[2] = -c * id; Ai[3] = a * id;
    } else {
        float T[9];
        T[0] = (A[4] * A[8] - A[5] * A[7]) * id;
        T[1] = (A[2] * A[7] - A[1] * A[8]) * id;
        T[2] = (A[1] * A[5] - A[2] * A[4]) * id;
        T[3] = (A[5] * A[6] - A[3] * A[8]) * id;
        T[4] = (A[0] * A[8] - A[2] * A[6]) * id;
        T[5] = (A[2] * A[3] - A[0] * A[5]) * id;
        T[6] = (A[3] * A[7] - A[4] * A[6]) * id;
        T[7] = (A[1] * A[6] - A[0] * A[7]) * id;
        T[8] = (A[0] * A[4] - A[1] * A[3]) * id;
#pragma unroll
        for (int i = 0; i < 9; ++i) Ai[i] = T[i];
    }
}

// ------------------------------------------------------------------- SVD --
//
// F = U diag(s) V^T with det U = det V = +1 and s0 >= s1 >= |s2|; the last
// singular value carries the sign of det F.  This is the convention of the
// reference's PolarSVD (MPMCUDA.cu:87-134).  The reference calls the McAdams
// et al. (UW-Madison TR1690) FP32 routine; this is an independent routine:
//   1. S = F^T F
//   2. up to 4 cyclic Jacobi sweeps with exact rotation angles (Golub & Van
//      Loan, Matrix Computations, Alg. 8.4.1-8.4.2), accumulating V; after two,
//      a sweep is skipped once the off-diagonal mass is below the FP32
//      resolution of the diagonal (jacobi_converged; the method converges
//      quadratically, so a near-rotation F is done after two)
//   3. one Newton-Schulz polish of V:  V <- V (3 I - V^T V) / 2
//   4. sort by eigenvalue, B = F V, Gram-Schmidt QR of B -> U, s

// x / y with the hardware's approximate division on the device (y a normal
// magnitude here); exact division on the host
MPM_HD float fast_div(float x, float y) {
#ifdef __CUDA_ARCH__
    return __fdividef(x, y);
#else
    return x / y;
#endif
}

// one Jacobi rotation on the (p,q) pair of the symmetric S (stored as 3x3)
template <int P, int Q>
MPM_HD void jacobi_rotate(float* S, float* V) {
    constexpr int R = 3 - P - Q;  // the remaining index
    const float spq = S[P * 3 + Q];
    const float diff = S[Q * 3 + Q] - S[P * 3 + P];
    // tan of the rotation angle (0 when the pair is already diagonal).  The
    // approximate square root and quotient only perturb the angle: c and s
    // below form an exact rotation for any t, so orthogonality does not suffer
    // (below 1e-30 the pair counts as diagonal: keeps both operations on
    // normal numbers)
    const float q = fmaf(diff, diff, 4.f * spq * spq);
    const float root = q > 1e-30f ? q * rsqrtf(q) : 0.f;
    const float den = fabsf(diff) + root;
    float t = den > 1e-30f ? fast_div(2.f * spq, den) : 0.f;
    t = diff < 0.f ? -t : t;
    const float c = rsqrtf(fmaf(t, t, 1.f));
    const float s = t * c;
    S[P * 3 + P] -= t * spq;
    S[Q * 3 + Q] += t * spq;
    S[P * 3 + Q] = 0.f;
    S[Q * 3 + P] = 0.f;
    const float srp = S[R * 3 + P], srq = S[R * 3 + Q];
    const float nrp = c * srp - s * srq, nrq = s * srp + c * srq;
    S[R * 3 + P] = nrp; S[P * 3 + R] = nrp;
    S[R * 3 + Q] = nrq; S[Q * 3 + R] = nrq;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float vkp = V[k * 3 + P], vkq = V[k * 3 + Q];
        V[k * 3 + P] = c * vkp - s * vkq;
        V[k * 3 + Q] = s * vkp + c * vkq;
    }
}

// the off-diagonal mass of S is below the FP32 resolution of its diagonal:
// a further sweep would change nothing at FP32 precision
MPM_HD bool jacobi_converged(const float* S) {
    const float off = S[1] * S[1] + S[2] * S[2] + S[5] * S[5];
    const float dg = S[0] * S[0] + S[4] * S[4] + S[8] * S[8];
    return off <= 1e-14f * dg;
}

MPM_HD void swap_cols_neg(float* V, float* lam, int a, int b) {
    // swap columns a and b and negate one so det V keeps its sign
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float t = V[k * 3 + a];
        V[k * 3 + a] = -V[k * 3 + b];
        V[k * 3 + b] = t;
    }
    float t = lam[a]; lam[a] = lam[b]; lam[b] = t;
}

MPM_HD void svd3(const float* F, float* U, float* s, float* V) {
    float S[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            S[i * 3 + j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] +
                           F[2 * 3 + i] * F[2 * 3 + j];
#pragma unroll
    for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? 1.f : 0.f;
    // the sweep loop stays rolled: one copy of the three rotations keeps the
    // fused kernels' code small (instruction-fetch stalls)
#pragma unroll 1
    for (int sweep = 0; sweep < 4; ++sweep) {
        if (sweep >= 2 && jacobi_converged(S)) break;
        jacobi_rotate<0, 1>(S, V);
        jacobi_rotate<0, 2>(S, V);
        jacobi_rotate<1, 2>(S, V);
    }
    // Newton-Schulz polish: V <- V (3I - V^T V) / 2
    {
        float G[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                G[i * 3 + j] = ((i == j) ? 1.5f : 0.f) -
                               0.5f * (V[0 * 3 + i] * V[0 * 3 + j] + V[1 * 3 + i] * V[1 * 3 + j] +
                                       V[2 * 3 + i] * V[2 * 3 + j]);
        matmul<3>(V, G, V);
    }
    float lam[3] = {S[0], S[4], S[8]};
    if (lam[0] < lam[1]) swap_cols_neg(V, lam, 0, 1);
    if (lam[0] < lam[2]) swap_cols_neg(V, lam, 0, 2);
    if (lam[1] < lam[2]) swap_cols_neg(V, lam, 1, 2);
    float B[9];
    matmul<3>(F, V, B);
    // u0 = b0 / |b0|
    float b0[3] = {B[0], B[3], B[6]}, b1[3] = {B[1], B[4], B[7]}, b2[3] = {B[2], B[5], B[8]};
    float n0 = b0[0] * b0[0] + b0[1] * b0[1] + b0[2] * b0[2];
    float u0[3];
    if (n0 > 1e-30f) {
        float r = rsqrtf(n0);
        u0[0] = b0[0] * r; u0[1] = b0[1] * r; u0[2] = b0[2] * r;
    } else {
        u0[0] = 1.f; u0[1] = 0.f; u0[2] = 0.f;
    }
    float d01 = u0[0] * b1[0] + u0[1] * b1[1] + u0[2] * b1[2];
    float u1[3] = {b1[0] - d01 * u0[0], b1[1] - d01 * u0[1], b1[2] - d01 * u0[2]};
    float n1 = u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2];
    if (n1 > 1e-30f) {
        float r = rsqrtf(n1);
        u1[0] *= r; u1[1] *= r; u1[2] *= r;
    } else {
        // any unit vector orthogonal to u0: cross with the axis least aligned
        float ax[3] = {0.f, 0.f, 0.f};
        float a0 = fabsf(u0[0]), a1 = fabsf(u0[1]), a2 = fabsf(u0[2]);
        int m = (a0 <= a1 && a0 <= a2) ? 0 : ((a1 <= a2) ? 1 : 2);
        ax[m] = 1.f;
        float c[3] = {u0[1] * ax[2] - u0[2] * ax[1], u0[2] * ax[0] - u0[0] * ax[2],
                      u0[0] * ax[1] - u0[1] * ax[0]};
        float r = rsqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        u1[0] = c[0] * r; u1[1] = c[1] * r; u1[2] = c[2] * r;
    }
    float u2[3] = {u0[1] * u1[2] - u0[2] * u1[1], u0[2] * u1[0] - u0[0] * u1[2],
                   u0[0] * u1[1] - u0[1] * u1[0]};
    s[0] = u0[0] * b0[0] + u0[1] * b0[1] + u0[2] * b0[2];
    s[1] = u1[0] * b1[0] + u1[1] * b1[1] + u1[2] * b1[2];
    s[2] = u2[0] * b2[0] + u2[1] * b2[1] + u2[2] * b2[2];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        U[r * 3 + 0] = u0[r];
        U[r * 3 + 1] = u1[r];
        U[r * 3 + 2] = u2[r];
    }
}

// 2x2: closed-form polar rotation R (angle atan2(c - b, a + d)), then the
// symmetric eigenproblem of S = R^T F.  U = R W, V = W, det U = det V = +1.
MPM_HD void svd2(const float* F, float* U, float* s, float* V) {
    const float a = F[0], b = F[1], c = F[2], d = F[3];
    float x = a + d, y = c - b;
    float rn = x * x + y * y;
    float co = 1.f, si = 0.f;
    if (rn > 1e-30f) {
        float r = rsqrtf(rn);
        co = x * r;
        si = y * r;
    }
    // S = R^T F (symmetric up to round-off)
    const float s00 = co * a + si * c, s01 = co * b + si * d;
    const float s11 = -si * b + co * d;
    const float s10 = -si * a + co * c;
    const float sym01 = 0.5f * (s01 + s10);
    // eigen-rotation of [[s00, sym01], [sym01, s11]]
    const float diff = s11 - s00;
    const float root = sqrtf(fmaf(diff, diff, 4.f * sym01 * sym01));
    const float den = fabsf(diff) + root;
    float t = den > 0.f ? (2.f * sym01) / den : 0.f;
    t = diff < 0.f ? -t : t;
    const float wc = rsqrtf(fmaf(t, t, 1.f)), ws = t * wc;
    float l0 = s00 - t * sym01, l1 = s11 + t * sym01;
    // W columns: (wc, -ws), (ws, wc)
    float w00 = wc, w01 = ws, w10 = -ws, w11 = wc;
    if (l0 < l1) {  // order so that s0 >= s1; swap columns and negate one
        float t0 = l0; l0 = l1; l1 = t0;
        float c0 = w00, c1 = w10;
        w00 = -w01; w10 = -w11;
        w01 = c0; w11 = c1;
    }
    V[0] = w00; V[1] = w01; V[2] = w10; V[3] = w11;
    // U = R W
    U[0] = co * w00 - si * w10; U[1] = co * w01 - si * w11;
    U[2] = si * w00 + co * w10; U[3] = si * w01 + co * w11;
    s[0] = l0;
    s[1] = l1;
}

template <int D>
MPM_HD void svd(const float* F, float* U, float* s, float* V) {
    if constexpr (D == 2) svd2(F, U, s, V);
    else svd3(F, U, s, V);
}

// ---------------------------------------------------------------- stress --
//
// Fixed-corotated Kirchhoff stress (kirchoff_FCR, MPMCUDA.cu:229-264;
// MPMJello.py:28-29):  tau = 2 mu (F - R) F^T + lambda J (J - 1) I,
// R = U V^T, J = det F.  With F = U S V^T, (F - R) F^T = U (S^2 - S) U^T, so
// only U and s are needed:  tau = U diag(2 mu s_i (s_i - 1)) U^T
//                                 + lambda J (J - 1) I.
//
// In 3D the left singular vectors and singular values come from the
// eigendecomposition of B = F F^T = U diag(s^2) U^T (the same cyclic Jacobi
// sweeps as svd3, accumulating U instead of V), so V, its polish and the
// Gram-Schmidt step are not needed: s_i = sqrt(eig_i), and when det F < 0 the
// smallest one is negated (the convention of the SVD: s0 >= s1 >= |s2|, the
// last carrying the sign of det F).  The sum over k does not depend on the
// order of the eigenpairs, so they are not sorted.
MPM_HD void kirchhoff_fcr3(const float* F, float mu, float lambda, float* tau) {
    float S[9], U[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            S[i * 3 + j] = F[i * 3 + 0] * F[j * 3 + 0] + F[i * 3 + 1] * F[j * 3 + 1] + F[i * 3 + 2] * F[j * 3 + 2];
#pragma unroll
    for (int i = 0; i < 9; ++i) U[i] = (i % 4 == 0) ? 1.f : 0.f;
#pragma unroll 1  // rolled, as in svd3
    for (int sweep = 0; sweep < 4; ++sweep) {
        if (sweep >= 2 && jacobi_converged(S)) break;
        jacobi_rotate<0, 1>(S, U);
        jacobi_rotate<0, 2>(S, U);
        jacobi_rotate<1, 2>(S, U);
    }
    const float J = det<3>(F);
    float s[3] = {sqrtf(fmaxf(S[0], 0.f)), sqrtf(fmaxf(S[4], 0.f)), sqrtf(fmaxf(S[8], 0.f))};
    if (J < 0.f) {
        const int k = (S[0] <= S[4] && S[0] <= S[8]) ? 0 : (S[4] <= S[8] ? 1 : 2);
        s[k] = -s[k];
    }
    const float iso = lambda * J * (J - 1.f);
    float dg[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) dg[k] = 2.f * mu * s[k] * (s[k] - 1.f);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = (i == j) ? iso : 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc = fmaf(U[i * 3 + k] * dg[k], U[j * 3 + k], acc);
            tau[i * 3 + j] = acc;
        }
}

template <int D>
MPM_HD void kirchhoff_fcr(const float* F, float mu, float lambda, float* tau) {
    if constexpr (D == 3) {
        kirchhoff_fcr3(F, mu, lambda, tau);
    } else {
        float U[4], s[2], V[4];
        svd2(F, U, s, V);
        const float J = det<2>(F);
        const float iso = lambda * J * (J - 1.f);
        float dg[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) dg[k] = 2.f * mu * s[k] * (s[k] - 1.f);
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float acc = (i == j) ? iso : 0.f;
#pragma unroll
                for (int k = 0; k < 2; ++k) acc = fmaf(U[i * 2 + k] * dg[k], U[j * 2 + k], acc);
                tau[i * 2 + j] = acc;
            }
    }
}

// ------------------------------------------------------------- B-spline --
//
// Quadratic B-spline weights of the 3 stencil nodes along one axis for a
// particle at grid coordinate gx = (x - origin) / h.  The base node is
// floor(gx - 0.5) (MPMCUDA.cu:356, MPMJello.py:42); with fx = gx - base in
// [0.5, 1.5) the weights N(fx - k) and derivatives N'(fx - k) are
//   w  = { (1.5 - fx)^2 / 2,  0.75 - (fx - 1)^2,  (fx - 0.5)^2 / 2 }
//   dw = { fx - 1.5,          -2 (fx - 1),        fx - 0.5 }
// (MPMJello.py:46-47; equal to the piecewise form of MPMCUDA.cu:267-290).
struct Axis {
    int base;
    float fx;
    float w[3];
    float dw[3];
};

MPM_HD Axis axis_weights(float gx) {
    Axis a;
    a.base = (int)floorf(gx - 0.5f);
    const float fx = gx - (float)a.base;
    a.fx = fx;
    const float t0 = 1.5f - fx, t1 = fx - 1.f, t2 = fx - 0.5f;
    a.w[0] = 0.5f * t0 * t0;
    a.w[1] = 0.75f - t1 * t1;
    a.w[2] = 0.5f * t2 * t2;
    a.dw[0] = -t0;
    a.dw[1] = -2.f * t1;
    a.dw[2] = t2;
    return a;
}

}  // namespace mpm
