// Instantiations of the fused substep kernel with the learned stress (3D
// jello and snow) for every launch configuration.
#include "mpm_dispatch.cuh"

namespace mpm {

// the surrogate kernel of a fused-kernel configuration (same chunk and
// launch-bound occupancy)
template <int MAT, int CI>
static constexpr auto sur_kernel() {
    return &k_g2p2g_sur<MAT, kFusedCfgs[CI].chunk, kFusedCfgs[CI].min_ctas>;
}

template <int MAT>
static void (*sur_for(int ci))(ParticleBuf, FusedArgs, SurArgs) {
    switch (ci) {
        case 0: return sur_kernel<MAT, 0>();
        case 1: return sur_kernel<MAT, 1>();
        case 2: return sur_kernel<MAT, 2>();
        case 3: return sur_kernel<MAT, 3>();
        case 4: return sur_kernel<MAT, 4>();
        case 5: return sur_kernel<MAT, 5>();
        case 6: return sur_kernel<MAT, 6>();
        default: return sur_kernel<MAT, 7>();
    }
}

SurFn sur_fn(int mat, int ci) {
    return mat == SNOW ? sur_for<SNOW>(ci) : sur_for<JELLO>(ci);
}

}  // namespace mpm
