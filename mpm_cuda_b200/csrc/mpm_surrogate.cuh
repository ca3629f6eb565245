// The learned stress surrogate object shared by the training runtime
// (mpm_surrogate.cu) and the substep kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "mpm_b200.h"
#include "mpm_mlp.cuh"

namespace mpm {

// FP32 master parameters, packed: W1 [64 x 16], W2 [64 x 64], W3 [16 x 64],
// b1 [64], b2 [64], b3 [16]
namespace mlp {
constexpr int OFF_W1 = 0;
constexpr int OFF_W2 = OFF_W1 + HID * IN_PAD;
constexpr int OFF_W3 = OFF_W2 + HID * HID;
constexpr int OFF_B1 = OFF_W3 + OUT_PAD * HID;
constexpr int OFF_B2 = OFF_B1 + HID;
constexpr int OFF_B3 = OFF_B2 + HID;
constexpr int N_PARAMS = OFF_B3 + OUT_PAD;
}  // namespace mlp

struct Surrogate {
    int device = 0;
    mlp::Meta meta{};
    float* master = nullptr;  // FP32 parameters (device)
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    float* grad = nullptr;
    mlp::Weights* weights = nullptr;  // BF16 copy used by the kernels (device)
    long long adam_t = 0;
    long long version = 0;  // bumped whenever the weights or meta change
    std::string last_error;

    int init(int dev, uint64_t seed);
    void release();
    int upload_master(const float* host);   // host FP32 params -> master + BF16 copy
    int download_master(float* host);
    int refresh_weights(cudaStream_t s);    // master -> BF16 copy
};

Surrogate* surrogate_of(::mpm_surrogate* h);

}  // namespace mpm
