// Training, evaluation and storage of the learned stress surrogate.
//
// The network (mpm_mlp.cuh) predicts the residual r(X) of sqrt(B) beyond its
// second-order series in X = B - I, B = F F^T, from which the fixed-corotated
// Kirchhoff stress follows without an SVD (MPMCUDA.cu:229-264 computes it
// with one).
//
// Training data: deformation gradients harvested from plain runs, perturbed
// as U diag(sigma + N(0, s^2)) V^T where U, V come from the plain path's own
// FP32 SVD (svd3) of the harvested F and, for a given fraction of the samples,
// U is replaced by a rotation drawn uniformly on SO(3).  The target residual
// is U diag(f(sigma)) U^T, exact for the constructed F.  Training runs on the
// GPU: a warp-level forward + backward pass (mma.sync BF16 tensor cores, FP32
// accumulation), split-K weight-gradient GEMMs on the same tensor cores, and
// Adam on FP32 master weights.  The plain path's kirchhoff_fcr is the
// reference for the trained network's stress error (mpm_surrogate_eval).
#include "mpm_b200.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "mpm_math.cuh"
#include "mpm_surrogate.cuh"

namespace mpm {

void set_thread_error(const char* msg);

namespace {

using namespace mlp;

// ------------------------------------------------------------ random --
// splitmix64 finaliser (Steele, Lea, Flood 2014) as a counter-based hash
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float u01(unsigned long long h) { return ((float)(h >> 40) + 0.5f) * (1.f / 16777216.f); }
__device__ __forceinline__ float gauss(unsigned long long h) {
    const float a = u01(h), b = u01(mix64(h));
    return sqrtf(-2.f * logf(a)) * cospif(2.f * b);
}
// rotation uniform on SO(3): unit quaternion from four normal deviates
__device__ __forceinline__ void haar_rotation(unsigned long long h, float* R) {
    float q[4];
    for (int k = 0; k < 4; ++k) q[k] = gauss(mix64(h + 0x1000ull * (k + 1)));
    const float n = rsqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3] + 1e-30f);
    const float w = q[0] * n, x = q[1] * n, y = q[2] * n, z = q[3] * n;
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z);     R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);     R[7] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}

// training samples: F, J and the residual target; envelope statistics as
// float bits (max |X| entry, min J, max J) and sums of squares for the scales
__global__ void k_gen_samples(const float* __restrict__ seedF, long long n_seed, long long n, unsigned long long seed,
                              float sigma, float rot_frac, float* __restrict__ Fo, float* __restrict__ Jo,
                              float* __restrict__ Ro, unsigned* __restrict__ env, double* __restrict__ sums) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)i));
    const long long idx = (long long)(mix64(h + 1) % (unsigned long long)n_seed);
    float F0[9], U[9], s[3], V[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F0[k] = seedF[idx * 9 + k];
    svd3(F0, U, s, V);
    if (u01(mix64(h + 2)) < rot_frac) haar_rotation(mix64(h + 3), U);
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = fmaxf(fabsf(s[k]) + sigma * gauss(mix64(h + 5 + k)), 0.3f);
    float F[9], X[9], r[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            F[a * 3 + b] = fmaf(U[a * 3 + 0] * s[0], V[b * 3 + 0], fmaf(U[a * 3 + 1] * s[1], V[b * 3 + 1],
                                                                      U[a * 3 + 2] * s[2] * V[b * 3 + 2]));
    strain_b(F, X);
    residual_target(U, s, r);
    const float J = det<3>(F);
    float e = 0.f, sx = 0.f, sr = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        Fo[i * 9 + k] = F[k];
        Ro[i * 9 + k] = r[k];
        e = fmaxf(e, fabsf(X[k]));
        sx = fmaf(X[k], X[k], sx);
        sr = fmaf(r[k], r[k], sr);
    }
    Jo[i] = J;
    atomicMax(&env[0], __float_as_uint(e));
    atomicMin(&env[1], __float_as_uint(J));
    atomicMax(&env[2], __float_as_uint(J));
    atomicAdd(&sums[0], (double)sx);
    atomicAdd(&sums[1], (double)sr);
}

// master parameters -> BF16 weights (with the transposed copies)
__global__ void k_refresh(const float* __restrict__ p, Weights* __restrict__ W) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N_PARAMS; i += gridDim.x * blockDim.x) {
        const float v = p[i];
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        if (i < OFF_W2) {
            const int o = i / IN_PAD, k = i % IN_PAD;
            W->f.w1[o * S16 + k] = b;
        } else if (i < OFF_W3) {
            const int j = i - OFF_W2, o = j / HID, k = j % HID;
            W->f.w2[o * S64 + k] = b;
            W->w2t[k * S64 + o] = b;
        } else if (i < OFF_B1) {
            const int j = i - OFF_W3, o = j / HID, k = j % HID;
            W->f.w3[o * S64 + k] = b;
            W->w3t[k * S16 + o] = b;
        } else if (i < OFF_B2) {
            W->f.b1[i - OFF_B1] = v;
        } else if (i < OFF_B3) {
            W->f.b2[i - OFF_B2] = v;
        } else {
            W->f.b3[i - OFF_B3] = v;
        }
    }
}

template <class T>
__device__ __forceinline__ void copy_weights(const T* __restrict__ g, T& s) {
    const int4* src = reinterpret_cast<const int4*>(g);
    int4* dst = reinterpret_cast<int4*>(&s);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 16); i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ unsigned short bf16_bits(float v) {
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    return __bfloat16_as_ushort(b);
}

// column sums over the 16 rows of an accumulator tile: rows g and g + 8 of
// lanes with the same t, reduced over g (lane bits 2..4)
__device__ __forceinline__ float colsum(float a, float b) {
    float v = a + b;
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// Forward + backward of one mini-batch, 32 samples per warp.  Stores the BF16
// activations and deltas each weight gradient needs (rows = batch position)
// and accumulates the bias gradients and the loss (mean squared error over the
// 9 outputs of the batch, in units of out_scale).  Samples are drawn at random
// from the n training samples, or taken in order (`sequential`).  Features come
// from F, J, or, when Xraw is given, directly from Xraw (10 per sample);
// targets Ts (9 per sample) are multiplied by inv_out.
__global__ void __launch_bounds__(128) k_train_fb(const Weights* __restrict__ Wg, Meta meta, const float* __restrict__ Fs,
                                                  const float* __restrict__ Js, const float* __restrict__ Xraw,
                                                  const float* __restrict__ Ps, float inv_out, long long n,
                                                  unsigned long long seed, long long step, int sequential, int batch,
                                                  unsigned short* __restrict__ bX, unsigned short* __restrict__ bH1,
                                                  unsigned short* __restrict__ bH2, unsigned short* __restrict__ bdZ1,
                                                  unsigned short* __restrict__ bdZ2, unsigned short* __restrict__ bdY,
                                                  float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ __align__(16) Weights W;
    __shared__ float sx[128][IN_PAD];
    __shared__ long long sidx[128];
    copy_weights(Wg, W);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long row = (long long)blockIdx.x * 128 + threadIdx.x;
    long long j = 0;
    if (row < batch) {
        j = sequential ? row : (long long)(mix64(seed ^ mix64(0x5eedull + step) ^ mix64((unsigned long long)row)) %
                                           (unsigned long long)n);
        if (Xraw) {
            for (int k = 0; k < IN_PAD; ++k) sx[threadIdx.x][k] = k < IN ? Xraw[j * IN + k] : 0.f;
        } else {
            features(Fs + j * 9, Js[j], meta, sx[threadIdx.x]);
        }
    } else {
        for (int k = 0; k < IN_PAD; ++k) sx[threadIdx.x][k] = 0.f;
    }
    sidx[threadIdx.x] = row < batch ? j : -1;
    __syncthreads();
    const int g = lane >> 2, t = lane & 3;
    const float dscale = 2.f / ((float)batch * OUT);
    float lsum = 0.f;
    for (int mt = 0; mt < 2; ++mt) {
        const int r0 = warp * 32 + mt * 16;  // first row of the tile in the CTA
        const float* x = sx[r0];
        unsigned a[4];
        load_a_input(x, lane, a);
        float z1[8][4];
        init_bias<8>(z1, W.f.b1, lane);
#pragma unroll
        for (int jn = 0; jn < 8; ++jn) {
            unsigned b0, b1;
            load_b<S16>(W.f.w1, jn, 0, lane, b0, b1);
            mma16816(z1[jn], a, b0, b1);
        }
        unsigned a2[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) acc_to_a_silu(z1[2 * kk], z1[2 * kk + 1], a2[kk]);
        float z2[8][4];
        init_bias<8>(z2, W.f.b2, lane);
#pragma unroll
        for (int jn = 0; jn < 8; ++jn)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                unsigned b0, b1;
                load_b<S64>(W.f.w2, jn, kk, lane, b0, b1);
                mma16816(z2[jn], a2[kk], b0, b1);
            }
        unsigned a3[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) acc_to_a_silu(z2[2 * kk], z2[2 * kk + 1], a3[kk]);
        float o[2][4];
        init_bias<2>(o, W.f.b3, lane);
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                unsigned b0, b1;
                load_b<S64>(W.f.w3, jn, kk, lane, b0, b1);
                mma16816(o[jn], a3[kk], b0, b1);
            }
        // loss gradient, masked to the 9 outputs and to rows of the batch
        const long long gr0 = (long long)blockIdx.x * 128 + r0 + g, gr1 = gr0 + 8;
        const long long s0 = sidx[r0 + g], s1 = sidx[r0 + g + 8];
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = 8 * jn + 2 * t + (e & 1);
                const long long sidx_e = (e < 2) ? s0 : s1;
                float d = 0.f;
                if (col < OUT && sidx_e >= 0) {
                    d = o[jn][e] - Ps[sidx_e * 9 + col] * inv_out;
                    lsum = fmaf(d, d, lsum);
                }
                o[jn][e] = d * dscale;
            }
        // dH2 = dY W3, dZ2 = dH2 * silu'(Z2)
        unsigned ady[4];
        acc_to_a(o[0], o[1], ady, [](float v) { return v; });
        float dz2[8][4];
#pragma unroll
        for (int jn = 0; jn < 8; ++jn) {
            dz2[jn][0] = dz2[jn][1] = dz2[jn][2] = dz2[jn][3] = 0.f;
            unsigned b0, b1;
            load_b<S16>(W.w3t, jn, 0, lane, b0, b1);
            mma16816(dz2[jn], ady, b0, b1);
#pragma unroll
            for (int e = 0; e < 4; ++e) dz2[jn][e] *= silu_grad(z2[jn][e]);
        }
        // dH1 = dZ2 W2, dZ1 = dH1 * silu'(Z1)
        unsigned adz2[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) acc_to_a(dz2[2 * kk], dz2[2 * kk + 1], adz2[kk], [](float v) { return v; });
        float dz1[8][4];
#pragma unroll
        for (int jn = 0; jn < 8; ++jn) {
            dz1[jn][0] = dz1[jn][1] = dz1[jn][2] = dz1[jn][3] = 0.f;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                unsigned b0, b1;
                load_b<S64>(W.w2t, jn, kk, lane, b0, b1);
                mma16816(dz1[jn], adz2[kk], b0, b1);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) dz1[jn][e] *= silu_grad(z1[jn][e]);
        }
        // store activations and deltas (BF16, batch-row major) for the weight gradients
        if (gr0 < batch || gr1 < batch) {
            // hidden activations exactly as the forward pass fed them on:
            // fragment q of k slice kk holds row g (q even) or g + 8 (q odd) and
            // columns 8 (2 kk + q / 2) + 2t, + 1
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const long long r = (q & 1) ? gr1 : gr0;
                    if (r >= batch) continue;
                    const int col = 8 * (2 * kk + (q >> 1)) + 2 * t;
                    *reinterpret_cast<unsigned*>(bH1 + r * HID + col) = a2[kk][q];
                    *reinterpret_cast<unsigned*>(bH2 + r * HID + col) = a3[kk][q];
                }
#pragma unroll
            for (int jn = 0; jn < 8; ++jn)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const long long r = (e < 2) ? gr0 : gr1;
                    if (r >= batch) continue;
                    const int col = 8 * jn + 2 * t + (e & 1);
                    bdZ1[r * HID + col] = bf16_bits(dz1[jn][e]);
                    bdZ2[r * HID + col] = bf16_bits(dz2[jn][e]);
                }
#pragma unroll
            for (int jn = 0; jn < 2; ++jn)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const long long r = (e < 2) ? gr0 : gr1;
                    if (r >= batch) continue;
                    const int col = 8 * jn + 2 * t + (e & 1);
                    bdY[r * OUT_PAD + col] = bf16_bits(o[jn][e]);
                    bX[r * IN_PAD + col] = bf16_bits(sx[r0 + ((e < 2) ? g : g + 8)][col]);
                }
        }
        // bias gradients: column sums of the deltas
#pragma unroll
        for (int jn = 0; jn < 8; ++jn) {
            const float c1a = colsum(dz1[jn][0], dz1[jn][2]), c1b = colsum(dz1[jn][1], dz1[jn][3]);
            const float c2a = colsum(dz2[jn][0], dz2[jn][2]), c2b = colsum(dz2[jn][1], dz2[jn][3]);
            if (g == 0) {
                atomicAdd(&grad[OFF_B1 + 8 * jn + 2 * t], c1a);
                atomicAdd(&grad[OFF_B1 + 8 * jn + 2 * t + 1], c1b);
                atomicAdd(&grad[OFF_B2 + 8 * jn + 2 * t], c2a);
                atomicAdd(&grad[OFF_B2 + 8 * jn + 2 * t + 1], c2b);
            }
        }
#pragma unroll
        for (int jn = 0; jn < 2; ++jn) {
            const float ca = colsum(o[jn][0], o[jn][2]), cb = colsum(o[jn][1], o[jn][3]);
            if (g == 0) {
                atomicAdd(&grad[OFF_B3 + 8 * jn + 2 * t], ca);
                atomicAdd(&grad[OFF_B3 + 8 * jn + 2 * t + 1], cb);
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if (lane == 0) atomicAdd(loss, lsum / ((float)batch * OUT));
}

__device__ __forceinline__ unsigned pack_bits(unsigned short lo, unsigned short hi) {
    return (unsigned)lo | ((unsigned)hi << 16);
}

// Weight gradients dW = delta^T act over a slice of the batch on the tensor
// cores (split-K), added to the FP32 gradient: warp w owns rows 16w..16w+15 of
// dW1 [64 x 16] and dW2 [64 x 64] and columns 16w..16w+15 of dW3 [16 x 64].
__global__ void __launch_bounds__(128) k_train_wgrad(const unsigned short* __restrict__ bX,
                                                     const unsigned short* __restrict__ bH1,
                                                     const unsigned short* __restrict__ bH2,
                                                     const unsigned short* __restrict__ bdZ1,
                                                     const unsigned short* __restrict__ bdZ2,
                                                     const unsigned short* __restrict__ bdY, int batch, int kslice,
                                                     float* __restrict__ grad) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int k_begin = blockIdx.x * kslice, k_end = min(batch, k_begin + kslice);
    float d1[2][4] = {}, d2[8][4] = {}, d3[2][4] = {};
    const int m = 16 * w + g;
    for (int k0 = k_begin; k0 < k_end; k0 += 16) {
        const int ka = k0 + 2 * t, kb = k0 + 2 * t + 8;
        // A = delta^T rows m, m+8; k = samples
        unsigned a1[4], a2[4], a3[4];
        a1[0] = pack_bits(bdZ1[(long long)ka * HID + m], bdZ1[(long long)(ka + 1) * HID + m]);
        a1[1] = pack_bits(bdZ1[(long long)ka * HID + m + 8], bdZ1[(long long)(ka + 1) * HID + m + 8]);
        a1[2] = pack_bits(bdZ1[(long long)kb * HID + m], bdZ1[(long long)(kb + 1) * HID + m]);
        a1[3] = pack_bits(bdZ1[(long long)kb * HID + m + 8], bdZ1[(long long)(kb + 1) * HID + m + 8]);
        a2[0] = pack_bits(bdZ2[(long long)ka * HID + m], bdZ2[(long long)(ka + 1) * HID + m]);
        a2[1] = pack_bits(bdZ2[(long long)ka * HID + m + 8], bdZ2[(long long)(ka + 1) * HID + m + 8]);
        a2[2] = pack_bits(bdZ2[(long long)kb * HID + m], bdZ2[(long long)(kb + 1) * HID + m]);
        a2[3] = pack_bits(bdZ2[(long long)kb * HID + m + 8], bdZ2[(long long)(kb + 1) * HID + m + 8]);
        // dW3 rows are the 16 (padded) outputs
        a3[0] = pack_bits(bdY[(long long)ka * OUT_PAD + g], bdY[(long long)(ka + 1) * OUT_PAD + g]);
        a3[1] = pack_bits(bdY[(long long)ka * OUT_PAD + g + 8], bdY[(long long)(ka + 1) * OUT_PAD + g + 8]);
        a3[2] = pack_bits(bdY[(long long)kb * OUT_PAD + g], bdY[(long long)(kb + 1) * OUT_PAD + g]);
        a3[3] = pack_bits(bdY[(long long)kb * OUT_PAD + g + 8], bdY[(long long)(kb + 1) * OUT_PAD + g + 8]);
#pragma unroll
        for (int jn = 0; jn < 2; ++jn) {  // dW1 columns: the 16 inputs
            const int col = 8 * jn + g;
            const unsigned b0 = pack_bits(bX[(long long)ka * IN_PAD + col], bX[(long long)(ka + 1) * IN_PAD + col]);
            const unsigned b1 = pack_bits(bX[(long long)kb * IN_PAD + col], bX[(long long)(kb + 1) * IN_PAD + col]);
            mma16816(d1[jn], a1, b0, b1);
        }
#pragma unroll
        for (int jn = 0; jn < 8; ++jn) {  // dW2 columns: hidden layer 1
            const int col = 8 * jn + g;
            const unsigned b0 = pack_bits(bH1[(long long)ka * HID + col], bH1[(long long)(ka + 1) * HID + col]);
            const unsigned b1 = pack_bits(bH1[(long long)kb * HID + col], bH1[(long long)(kb + 1) * HID + col]);
            mma16816(d2[jn], a2, b0, b1);
        }
#pragma unroll
        for (int jn = 0; jn < 2; ++jn) {  // dW3 columns 16w.. of hidden layer 2
            const int col = 16 * w + 8 * jn + g;
            const unsigned b0 = pack_bits(bH2[(long long)ka * HID + col], bH2[(long long)(ka + 1) * HID + col]);
            const unsigned b1 = pack_bits(bH2[(long long)kb * HID + col], bH2[(long long)(kb + 1) * HID + col]);
            mma16816(d3[jn], a3, b0, b1);
        }
    }
#pragma unroll
    for (int jn = 0; jn < 2; ++jn)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = 16 * w + g + ((e < 2) ? 0 : 8), col = 8 * jn + 2 * t + (e & 1);
            atomicAdd(&grad[OFF_W1 + row * IN_PAD + col], d1[jn][e]);
        }
#pragma unroll
    for (int jn = 0; jn < 8; ++jn)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = 16 * w + g + ((e < 2) ? 0 : 8), col = 8 * jn + 2 * t + (e & 1);
            atomicAdd(&grad[OFF_W2 + row * HID + col], d2[jn][e]);
        }
#pragma unroll
    for (int jn = 0; jn < 2; ++jn)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = g + ((e < 2) ? 0 : 8), col = 16 * w + 8 * jn + 2 * t + (e & 1);
            atomicAdd(&grad[OFF_W3 + row * HID + col], d3[jn][e]);
        }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; clears the gradient
__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, float* __restrict__ g,
                       float lr, float b1, float b2, float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N_PARAMS; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        g[i] = 0.f;
    }
}

// surrogate Kirchhoff stress tau / mu (lambda / mu = lam_mu) of n samples and
// whether the fused stress pass would accept it (envelope and error estimate)
__global__ void __launch_bounds__(128) k_eval(const Forward* __restrict__ Wg, Meta meta, const float* __restrict__ Fs,
                                              long long n, float lam_mu, float* __restrict__ Tout,
                                              unsigned char* __restrict__ ok) {
    __shared__ __align__(16) Forward W;
    __shared__ float sxy[128][IN_PAD];
    copy_weights(Wg, W);
    const long long i = (long long)blockIdx.x * 128 + threadIdx.x;
    float F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (i < n)
        for (int k = 0; k < 9; ++k) F[k] = Fs[i * 9 + k];
    const float J = det<3>(F);
    features(F, J, meta, sxy[threadIdx.x]);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    forward_tile(W, sxy[warp * 32], sxy[warp * 32], lane);
    forward_tile(W, sxy[warp * 32 + 16], sxy[warp * 32 + 16], lane);
    __syncwarp();
    if (i < n) {
        float tau[9];
        const bool good = tau_from_prediction(sxy[threadIdx.x], F, J, 1.f, lam_mu, meta, tau);
        for (int k = 0; k < 9; ++k) Tout[i * 9 + k] = tau[k];
        ok[i] = (good && in_envelope(F, J, meta)) ? 1 : 0;
    }
}

// the plain path's tau / mu (its FP32 SVD) of n samples
__global__ void k_ref_tau(const float* __restrict__ Fs, long long n, float lam_mu, float* __restrict__ Tout) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float F[9], tau[9];
    for (int k = 0; k < 9; ++k) F[k] = Fs[i * 9 + k];
    kirchhoff_fcr<3>(F, 1.f, lam_mu, tau);
    for (int k = 0; k < 9; ++k) Tout[i * 9 + k] = tau[k];
}

// zero-stress calibration: b3 -= y(X = 0, J = 1), so that an undeformed
// particle gets exactly zero stress from the network (one warp)
__global__ void k_calibrate_rest(const Forward* __restrict__ Wg, float* __restrict__ master) {
    __shared__ __align__(16) Forward W;
    __shared__ float sxy[16][IN_PAD];
    copy_weights(Wg, W);
    for (int k = threadIdx.x; k < 16 * IN_PAD; k += blockDim.x) sxy[k / IN_PAD][k % IN_PAD] = 0.f;
    __syncthreads();
    if (threadIdx.x < 32) forward_tile(W, sxy[0], sxy[0], threadIdx.x);
    __syncthreads();
    if (threadIdx.x < OUT) master[OFF_B3 + threadIdx.x] -= sxy[0][threadIdx.x];
}

int fail(mpm::Surrogate* s, int code, const char* msg) {
    if (s) s->last_error = msg;
    set_thread_error(msg);
    return code;
}

#define SUR_TRY(expr, what)                                                      \
    do {                                                                         \
        cudaError_t e_ = (expr);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            char b_[256];                                                        \
            std::snprintf(b_, sizeof(b_), "%s: %s", what, cudaGetErrorString(e_)); \
            return ::mpm::fail(s, MPM_ERR_CUDA, b_);                             \
        }                                                                        \
    } while (0)

}  // namespace

int Surrogate::init(int dev, uint64_t seed) {
    Surrogate* s = this;
    device = dev;
    SUR_TRY(cudaSetDevice(dev), "cudaSetDevice");
    SUR_TRY(cudaMalloc((void**)&master, N_PARAMS * sizeof(float)), "alloc");
    SUR_TRY(cudaMalloc((void**)&adam_m, N_PARAMS * sizeof(float)), "alloc");
    SUR_TRY(cudaMalloc((void**)&adam_v, N_PARAMS * sizeof(float)), "alloc");
    SUR_TRY(cudaMalloc((void**)&grad, N_PARAMS * sizeof(float)), "alloc");
    SUR_TRY(cudaMalloc((void**)&weights, sizeof(Weights)), "alloc");
    SUR_TRY(cudaMemset(weights, 0, sizeof(Weights)), "memset");
    SUR_TRY(cudaMemset(adam_m, 0, N_PARAMS * sizeof(float)), "memset");
    SUR_TRY(cudaMemset(adam_v, 0, N_PARAMS * sizeof(float)), "memset");
    SUR_TRY(cudaMemset(grad, 0, N_PARAMS * sizeof(float)), "memset");
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) on the real inputs / outputs;
    // the padding rows and columns stay zero (their gradients are zero)
    std::mt19937_64 rng(seed);
    std::vector<float> p(N_PARAMS, 0.f);
    auto fill = [&](int off, int cols, int real_rows, int real_cols, int fan_in) {
        std::uniform_real_distribution<float> U(-1.f / std::sqrt((float)fan_in), 1.f / std::sqrt((float)fan_in));
        for (int r = 0; r < real_rows; ++r)
            for (int c = 0; c < real_cols; ++c) p[off + r * cols + c] = U(rng);
    };
    fill(OFF_W1, IN_PAD, HID, IN, IN);
    fill(OFF_W2, HID, HID, HID, HID);
    fill(OFF_W3, HID, OUT, HID, HID);
    meta = Meta{};
    meta.in_scale = 1.f;
    meta.out_scale = 1.f;
    meta.env_c = -1.f;  // empty envelope until trained: every particle falls back
    meta.env_jlo = 1.f;
    meta.env_jhi = 1.f;
    meta.skew_tol = 0.01f;
    meta.tau_floor = 0.f;
    adam_t = 0;
    return upload_master(p.data());
}

void Surrogate::release() {
    cudaSetDevice(device);
    cudaFree(master);
    cudaFree(adam_m);
    cudaFree(adam_v);
    cudaFree(grad);
    cudaFree(weights);
    master = adam_m = adam_v = grad = nullptr;
    weights = nullptr;
}

int Surrogate::refresh_weights(cudaStream_t st) {
    Surrogate* s = this;
    k_refresh<<<8, 256, 0, st>>>(master, weights);
    SUR_TRY(cudaGetLastError(), "refresh launch");
    return MPM_OK;
}

int Surrogate::upload_master(const float* host) {
    Surrogate* s = this;
    SUR_TRY(cudaSetDevice(device), "cudaSetDevice");
    SUR_TRY(cudaMemcpy(master, host, N_PARAMS * sizeof(float), cudaMemcpyHostToDevice), "upload");
    int rc = refresh_weights(0);
    if (rc != MPM_OK) return rc;
    SUR_TRY(cudaDeviceSynchronize(), "sync");
    return MPM_OK;
}

int Surrogate::download_master(float* host) {
    Surrogate* s = this;
    SUR_TRY(cudaSetDevice(device), "cudaSetDevice");
    SUR_TRY(cudaMemcpy(host, master, N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost), "download");
    return MPM_OK;
}

}  // namespace mpm

struct mpm_surrogate {
    mpm::Surrogate s;
};

using mpm::Surrogate;
namespace ml = mpm::mlp;

extern "C" {

void mpm_surrogate_default_train_options(mpm_surrogate_train_options* o) {
    if (!o) return;
    o->n_samples = 1 << 21;
    o->epochs = 8;
    o->batch = 8192;
    o->lr = 3e-3f;
    o->lr_final = 3e-5f;
    o->sigma = 0.05f;
    o->rotation_fraction = 0.5f;
    o->skew_tol = 0.01f;
    o->seed = 1234;
}

int mpm_surrogate_create(int device, uint64_t seed, mpm_surrogate** out) {
    if (!out) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_create: NULL out");
    auto* h = new (std::nothrow) mpm_surrogate();
    if (!h) return mpm::fail(nullptr, MPM_ERR_NOMEM, "mpm_surrogate_create: host allocation");
    const int rc = h->s.init(device, seed);
    if (rc != MPM_OK) {
        h->s.release();
        delete h;
        return rc;
    }
    *out = h;
    return MPM_OK;
}

int mpm_surrogate_destroy(mpm_surrogate* h) {
    if (!h) return MPM_OK;
    h->s.release();
    delete h;
    return MPM_OK;
}

int mpm_surrogate_train(mpm_surrogate* h, const float* F_seed, int64_t n_seed, const mpm_surrogate_train_options* opt,
                        float* final_loss) {
    if (!h || !F_seed || n_seed <= 0) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_train: bad argument");
    Surrogate* s = &h->s;
    mpm_surrogate_train_options o;
    mpm_surrogate_default_train_options(&o);
    if (opt) o = *opt;
    if (o.n_samples < 1024 || o.batch < 128 || o.batch % 128 || o.batch > (1 << 20) || o.epochs < 1 ||
        !(o.lr > 0.f) || !(o.lr_final > 0.f) || !(o.sigma >= 0.f) || !(o.skew_tol > 0.f))
        return mpm::fail(s, MPM_ERR_INVALID,
                         "mpm_surrogate_train: need n_samples >= 1024, 128 <= batch <= 2^20 a multiple of 128, "
                         "epochs >= 1, lr, lr_final, skew_tol > 0, sigma >= 0");
    SUR_TRY(cudaSetDevice(s->device), "cudaSetDevice");
    const long long n = o.n_samples;
    float *dSeed = nullptr, *dF = nullptr, *dJ = nullptr, *dR = nullptr, *dLoss = nullptr;
    unsigned* dEnv = nullptr;
    double* dSums = nullptr;
    unsigned short* act = nullptr;
    const size_t per_row = ml::IN_PAD + 4 * ml::HID + ml::OUT_PAD;  // X, H1, H2, dZ1, dZ2, dY
    auto cleanup = [&]() {
        cudaFree(dSeed); cudaFree(dF); cudaFree(dJ); cudaFree(dR); cudaFree(dLoss);
        cudaFree(dEnv); cudaFree(dSums); cudaFree(act);
    };
    cudaError_t e = cudaMalloc((void**)&dSeed, n_seed * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dF, n * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dJ, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dR, n * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dLoss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dEnv, 3 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dSums, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&act, (size_t)o.batch * per_row * sizeof(unsigned short));
    if (e == cudaSuccess) e = cudaMemcpy(dSeed, F_seed, n_seed * 9 * sizeof(float), cudaMemcpyHostToDevice);
    const unsigned env0[3] = {0u, 0x7f7fffffu, 0u};
    if (e == cudaSuccess) e = cudaMemcpy(dEnv, env0, sizeof(env0), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dSums, 0, 2 * sizeof(double));
    if (e != cudaSuccess) {
        cleanup();
        return mpm::fail(s, MPM_ERR_NOMEM, "mpm_surrogate_train: device allocation");
    }
    mpm::k_gen_samples<<<(unsigned)((n + 255) / 256), 256>>>(dSeed, n_seed, n, o.seed, o.sigma, o.rotation_fraction,
                                                             dF, dJ, dR, dEnv, dSums);
    unsigned env[3];
    double sums[2];
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(env, dEnv, sizeof(env), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sums, dSums, sizeof(sums), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cleanup();
        return mpm::fail(s, MPM_ERR_CUDA, "mpm_surrogate_train: sample generation failed");
    }
    auto bits = [](unsigned u) {
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    };
    s->meta.in_scale = (float)std::sqrt(sums[0] / (9.0 * n)) + 1e-6f;
    s->meta.out_scale = (float)std::sqrt(sums[1] / (9.0 * n)) + 1e-9f;
    s->meta.env_c = bits(env[0]);
    s->meta.env_jlo = bits(env[1]);
    s->meta.env_jhi = bits(env[2]);
    s->meta.skew_tol = o.skew_tol;
    s->meta.tau_floor = 0.05f * s->meta.in_scale;
    const float inv_out = 1.f / s->meta.out_scale;
    unsigned short* bX = act;
    unsigned short* bH1 = bX + (size_t)o.batch * ml::IN_PAD;
    unsigned short* bH2 = bH1 + (size_t)o.batch * ml::HID;
    unsigned short* bdZ1 = bH2 + (size_t)o.batch * ml::HID;
    unsigned short* bdZ2 = bdZ1 + (size_t)o.batch * ml::HID;
    unsigned short* bdY = bdZ2 + (size_t)o.batch * ml::HID;
    const long long steps_per_epoch = std::max<long long>(1, n / o.batch);
    const long long total = steps_per_epoch * o.epochs;
    const int kslice = 256;
    const unsigned wgrad_ctas = (unsigned)((o.batch + kslice - 1) / kslice);
    float loss = 0.f;
    if (e == cudaSuccess) e = cudaMemset(s->grad, 0, ml::N_PARAMS * sizeof(float));
    for (long long stp = 0; stp < total && e == cudaSuccess; ++stp) {
        if (stp % steps_per_epoch == 0) cudaMemsetAsync(dLoss, 0, sizeof(float));
        mpm::k_train_fb<<<o.batch / 128, 128>>>(s->weights, s->meta, dF, dJ, nullptr, dR, inv_out, n, o.seed, stp, 0,
                                                o.batch, bX, bH1, bH2, bdZ1, bdZ2, bdY, s->grad, dLoss);
        mpm::k_train_wgrad<<<wgrad_ctas, 128>>>(bX, bH1, bH2, bdZ1, bdZ2, bdY, o.batch, kslice, s->grad);
        ++s->adam_t;
        // cosine decay from lr to lr_final
        const double frac = (double)stp / std::max<long long>(1, total - 1);
        const float lr = (float)(o.lr_final + 0.5 * (o.lr - o.lr_final) * (1.0 + std::cos(3.14159265358979 * frac)));
        const float b1 = 0.9f, b2 = 0.999f;
        const float bc1 = 1.f - std::pow(b1, (float)s->adam_t), bc2 = 1.f - std::pow(b2, (float)s->adam_t);
        mpm::k_adam<<<8, 256>>>(s->master, s->adam_m, s->adam_v, s->grad, lr, b1, b2, 1e-8f, bc1, bc2);
        mpm::k_refresh<<<8, 256>>>(s->master, s->weights);
        e = cudaGetLastError();
        if (e == cudaSuccess && (stp + 1) % steps_per_epoch == 0) {
            e = cudaMemcpy(&loss, dLoss, sizeof(float), cudaMemcpyDeviceToHost);
            loss /= (float)steps_per_epoch;
        }
    }
    if (e == cudaSuccess) {
        mpm::k_calibrate_rest<<<1, 128>>>(&s->weights->f, s->master);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        mpm::k_refresh<<<8, 256>>>(s->master, s->weights);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cleanup();
    if (e != cudaSuccess) return mpm::fail(s, MPM_ERR_CUDA, "mpm_surrogate_train: training kernels failed");
    ++s->version;
    if (final_loss) *final_loss = loss;
    return MPM_OK;
}

int mpm_surrogate_eval(mpm_surrogate* h, const float* F, int64_t n, float lam_over_mu, float* tau_pred,
                       float* tau_ref, uint8_t* accepted) {
    if (!h || !F || n <= 0) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_eval: bad argument");
    Surrogate* s = &h->s;
    SUR_TRY(cudaSetDevice(s->device), "cudaSetDevice");
    float *dF = nullptr, *dP = nullptr, *dR = nullptr;
    unsigned char* dE = nullptr;
    cudaError_t e = cudaMalloc((void**)&dF, n * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dP, n * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dR, n * 9 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dE, n);
    if (e == cudaSuccess) e = cudaMemcpy(dF, F, n * 9 * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        mpm::k_eval<<<(unsigned)((n + 127) / 128), 128>>>(&s->weights->f, s->meta, dF, n, lam_over_mu, dP, dE);
        mpm::k_ref_tau<<<(unsigned)((n + 255) / 256), 256>>>(dF, n, lam_over_mu, dR);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && tau_pred) e = cudaMemcpy(tau_pred, dP, n * 9 * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && tau_ref) e = cudaMemcpy(tau_ref, dR, n * 9 * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && accepted) e = cudaMemcpy(accepted, dE, n, cudaMemcpyDeviceToHost);
    cudaFree(dF);
    cudaFree(dP);
    cudaFree(dR);
    cudaFree(dE);
    if (e != cudaSuccess) return mpm::fail(s, MPM_ERR_CUDA, "mpm_surrogate_eval failed");
    return MPM_OK;
}

int mpm_surrogate_gradients(mpm_surrogate* h, const float* x, const float* y_target, int64_t n, float* grads,
                            float* loss) {
    if (!h || !x || !y_target || n <= 0 || n % 128 || n > (1 << 20))
        return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_gradients: n must be a positive multiple of 128");
    Surrogate* s = &h->s;
    SUR_TRY(cudaSetDevice(s->device), "cudaSetDevice");
    float *dX = nullptr, *dY = nullptr, *dLoss = nullptr;
    unsigned short* act = nullptr;
    const size_t per_row = ml::IN_PAD + 4 * ml::HID + ml::OUT_PAD;
    cudaError_t e = cudaMalloc((void**)&dX, n * ml::IN * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dY, n * ml::OUT * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dLoss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&act, (size_t)n * per_row * sizeof(unsigned short));
    if (e == cudaSuccess) e = cudaMemcpy(dX, x, n * ml::IN * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dY, y_target, n * ml::OUT * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dLoss, 0, sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(s->grad, 0, ml::N_PARAMS * sizeof(float));
    if (e == cudaSuccess) {
        unsigned short* bX = act;
        unsigned short* bH1 = bX + (size_t)n * ml::IN_PAD;
        unsigned short* bH2 = bH1 + (size_t)n * ml::HID;
        unsigned short* bdZ1 = bH2 + (size_t)n * ml::HID;
        unsigned short* bdZ2 = bdZ1 + (size_t)n * ml::HID;
        unsigned short* bdY = bdZ2 + (size_t)n * ml::HID;
        mpm::k_train_fb<<<(unsigned)(n / 128), 128>>>(s->weights, s->meta, nullptr, nullptr, dX, dY, 1.f, n, 0, 0, 1,
                                                       (int)n, bX, bH1, bH2, bdZ1, bdZ2, bdY, s->grad, dLoss);
        mpm::k_train_wgrad<<<(unsigned)((n + 255) / 256), 128>>>(bX, bH1, bH2, bdZ1, bdZ2, bdY, (int)n, 256, s->grad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && grads) e = cudaMemcpy(grads, s->grad, ml::N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && loss) e = cudaMemcpy(loss, dLoss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(s->grad, 0, ml::N_PARAMS * sizeof(float));
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dLoss);
    cudaFree(act);
    if (e != cudaSuccess) return mpm::fail(s, MPM_ERR_CUDA, "mpm_surrogate_gradients failed");
    return MPM_OK;
}

int mpm_surrogate_num_params(void) { return ml::N_PARAMS; }
int mpm_surrogate_num_meta(void) { return (int)(sizeof(ml::Meta) / sizeof(float)); }

int mpm_surrogate_get_params(mpm_surrogate* h, float* params, float* meta) {
    if (!h) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_get_params: NULL");
    if (params) {
        const int rc = h->s.download_master(params);
        if (rc != MPM_OK) return rc;
    }
    if (meta) std::memcpy(meta, &h->s.meta, sizeof(ml::Meta));
    return MPM_OK;
}

int mpm_surrogate_set_params(mpm_surrogate* h, const float* params, const float* meta) {
    if (!h) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_set_params: NULL");
    if (meta) std::memcpy(&h->s.meta, meta, sizeof(ml::Meta));
    ++h->s.version;
    if (params) return h->s.upload_master(params);
    return MPM_OK;
}

int mpm_surrogate_save(mpm_surrogate* h, const char* path) {
    if (!h || !path) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_save: bad argument");
    std::vector<float> p(ml::N_PARAMS);
    int rc = h->s.download_master(p.data());
    if (rc != MPM_OK) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) return mpm::fail(&h->s, MPM_ERR_IO, "mpm_surrogate_save: cannot open file");
    const char magic[8] = {'M', 'P', 'M', 'S', 'U', 'R', '0', '2'};
    const int np = ml::N_PARAMS;
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&np, 4, 1, f) == 1 &&
              std::fwrite(&h->s.meta, sizeof(ml::Meta), 1, f) == 1 &&
              std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? MPM_OK : mpm::fail(&h->s, MPM_ERR_IO, "mpm_surrogate_save: write failed");
}

int mpm_surrogate_load(const char* path, int device, mpm_surrogate** out) {
    if (!path || !out) return mpm::fail(nullptr, MPM_ERR_INVALID, "mpm_surrogate_load: bad argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return mpm::fail(nullptr, MPM_ERR_IO, "mpm_surrogate_load: cannot open file");
    char magic[8];
    int np = 0;
    ml::Meta meta{};
    std::vector<float> p(ml::N_PARAMS);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "MPMSUR02", 8) == 0 &&
              std::fread(&np, 4, 1, f) == 1 && np == ml::N_PARAMS && std::fread(&meta, sizeof(meta), 1, f) == 1 &&
              std::fread(p.data(), sizeof(float), p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) return mpm::fail(nullptr, MPM_ERR_IO, "mpm_surrogate_load: not a surrogate file");
    mpm_surrogate* h = nullptr;
    int rc = mpm_surrogate_create(device, 0, &h);
    if (rc != MPM_OK) return rc;
    h->s.meta = meta;
    rc = h->s.upload_master(p.data());
    if (rc != MPM_OK) {
        mpm_surrogate_destroy(h);
        return rc;
    }
    *out = h;
    return MPM_OK;
}

}  // extern "C"

namespace mpm {
Surrogate* surrogate_of(mpm_surrogate* h) { return h ? &h->s : nullptr; }
}  // namespace mpm
