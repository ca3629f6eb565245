// Launch configurations of the fused substep kernel (the autotuner's search
// space), shared by the kernels and the C-ABI layer.
#pragma once

namespace mpm {

// particles per chunk (= threads per CTA) and the minimum resident CTAs per
// SM given to __launch_bounds__ (which caps registers at
// 65536 / (chunk * min_ctas))
struct FusedCfg {
    int chunk;
    int min_ctas;
};
constexpr int kNumFusedCfgs = 8;
constexpr FusedCfg kFusedCfgs[kNumFusedCfgs] = {{128, 4}, {128, 5}, {128, 6}, {64, 8},
                                                {64, 10}, {64, 12}, {256, 2}, {256, 3}};

}  // namespace mpm
