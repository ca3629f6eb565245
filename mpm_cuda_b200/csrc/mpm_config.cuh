// Launch configurations of the fused substep kernel (the autotuner's search
// space), shared by the kernels and the C-ABI layer.
#pragma once

namespace mpm {

// particles per chunk (= threads per CTA), the minimum resident CTAs per SM
// given to __launch_bounds__ (which caps registers at
// 65536 / (chunk * min_ctas)), and the P2G scatter variant (0: shared-memory
// window with shared atomics, flushed once per chunk; 1: float4 reductions
// straight to global memory)
struct FusedCfg {
    int chunk;
    int min_ctas;
    int scatter;
};
constexpr int kNumFusedCfgs = 8;
constexpr FusedCfg kFusedCfgs[kNumFusedCfgs] = {{128, 4, 0}, {128, 5, 0}, {64, 8, 0},  {64, 10, 0},
                                                {128, 4, 1}, {128, 6, 1}, {64, 10, 1}, {64, 12, 1}};

}  // namespace mpm
