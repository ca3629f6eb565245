// Instantiations of the fused substep kernel with the learned stress (3D
// jello) for every launch configuration.
#include "mpm_dispatch.cuh"

namespace mpm {

// the surrogate kernel of a fused-kernel configuration (same chunk and
// launch-bound occupancy as its direct-scatter instantiation)
template <int K>
static constexpr auto sur_kernel() {
    return &k_g2p2g_sur<kFusedKernels[K].chunk, kFusedKernels[K].min_ctas>;
}

SurFn sur_fn(int ci) {
    static_assert(kNumFusedKernels == 12, "update the dispatch table");
    // the learned-stress kernel scatters directly: a segmented configuration
    // runs it with the direct instantiation of its chunk
    switch (direct_kernel_of(kFusedCfgs[ci].kernel)) {
        case 0: return sur_kernel<0>();
        case 1: return sur_kernel<1>();
        case 2: return sur_kernel<2>();
        case 3: return sur_kernel<3>();
        case 4: return sur_kernel<4>();
        case 5: return sur_kernel<5>();
        case 6: return sur_kernel<6>();
        default: return sur_kernel<7>();
    }
}

}  // namespace mpm
