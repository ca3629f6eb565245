// Table of the fused substep kernel's instantiations for one scene source
// (FIXED: the scene from the kernel parameters, else from the device table),
// indexed by dimension, material and launch configuration (configurations
// that differ only in rounds or particle order share an instantiation).  Each source's
// table is instantiated in its own translation unit so they compile in
// parallel.
#pragma once

#include "mpm_dispatch.cuh"

namespace mpm {

template <int D, int MAT, int K, bool FIXED>
static constexpr auto fused_kernel() {
    return &k_g2p2g<D, MAT, kFusedKernels[K].chunk, kFusedKernels[K].min_ctas, FIXED, kFusedKernels[K].scatter>;
}

template <int D, int MAT, bool FIXED>
static FusedFn fused_for(int ci) {
    static_assert(kNumFusedKernels == 12, "update the dispatch table");
    switch (kFusedCfgs[ci].kernel) {
        case 0: return fused_kernel<D, MAT, 0, FIXED>();
        case 1: return fused_kernel<D, MAT, 1, FIXED>();
        case 2: return fused_kernel<D, MAT, 2, FIXED>();
        case 3: return fused_kernel<D, MAT, 3, FIXED>();
        case 4: return fused_kernel<D, MAT, 4, FIXED>();
        case 5: return fused_kernel<D, MAT, 5, FIXED>();
        case 6: return fused_kernel<D, MAT, 6, FIXED>();
        case 7: return fused_kernel<D, MAT, 7, FIXED>();
        case 8: return fused_kernel<D, MAT, 8, FIXED>();
        case 9: return fused_kernel<D, MAT, 9, FIXED>();
        case 10: return fused_kernel<D, MAT, 10, FIXED>();
        default: return fused_kernel<D, MAT, 11, FIXED>();
    }
}

template <int D, bool FIXED>
static FusedFn fused_for_mat(int mat, int ci) {
    if (mat == JELLO) return fused_for<D, JELLO, FIXED>(ci);
    if (mat == SNOW) return fused_for<D, SNOW, FIXED>(ci);
    return fused_for<D, WATER, FIXED>(ci);
}

template <bool FIXED>
static FusedFn fused_table(int dim, int mat, int ci) {
    return dim == 3 ? fused_for_mat<3, FIXED>(mat, ci) : fused_for_mat<2, FIXED>(mat, ci);
}

}  // namespace mpm
