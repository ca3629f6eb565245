// Instantiations of the fused substep kernel for every dimension, material
// and launch configuration (the autotuner's search space), in their own
// translation unit so that they compile in parallel with the rest.
#include "mpm_dispatch.cuh"

namespace mpm {

// the fused kernel instantiations, indexed [material][config]
template <int D, int MAT, int CI>
static constexpr auto fused_kernel() {
    return &k_g2p2g<D, MAT, kFusedCfgs[CI].chunk, kFusedCfgs[CI].min_ctas>;
}

template <int D, int MAT>
static void (*fused_for(int ci))(ParticleBuf, FusedArgs) {
    static_assert(kNumFusedCfgs == 8, "update the dispatch table");
    switch (ci) {
        case 0: return fused_kernel<D, MAT, 0>();
        case 1: return fused_kernel<D, MAT, 1>();
        case 2: return fused_kernel<D, MAT, 2>();
        case 3: return fused_kernel<D, MAT, 3>();
        case 4: return fused_kernel<D, MAT, 4>();
        case 5: return fused_kernel<D, MAT, 5>();
        case 6: return fused_kernel<D, MAT, 6>();
        default: return fused_kernel<D, MAT, 7>();
    }
}

template <int D>
static void (*fused_for_mat(int mat, int ci))(ParticleBuf, FusedArgs) {
    if (mat == JELLO) return fused_for<D, JELLO>(ci);
    if (mat == SNOW) return fused_for<D, SNOW>(ci);
    return fused_for<D, WATER>(ci);
}

FusedFn fused_fn(int dim, int mat, int ci) {
    return dim == 3 ? fused_for_mat<3>(mat, ci) : fused_for_mat<2>(mat, ci);
}

}  // namespace mpm
