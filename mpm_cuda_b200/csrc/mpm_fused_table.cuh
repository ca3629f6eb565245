// Table of the fused substep kernel's instantiations for one scene source
// (FIXED: the scene from the kernel parameters, else from the device table),
// indexed by dimension, material and launch configuration (configurations
// that differ only in rounds or particle order share an instantiation).  Each source's
// table is instantiated in its own translation unit so they compile in
// parallel.
#pragma once

#include "mpm_dispatch.cuh"

namespace mpm {

template <int D, int MAT, int K, bool FIXED, bool PAGED>
static constexpr FusedFn fused_kernel() {
    if constexpr (PAGED && kFusedKernels[K].scatter == SCATTER_SEGMENTED) {
        return nullptr;  // the segmented scatter addresses a dense grid
    } else {
        return &k_g2p2g<D, MAT, kFusedKernels[K].chunk, kFusedKernels[K].min_ctas, FIXED, kFusedKernels[K].scatter,
                        PAGED>;
    }
}

template <int D, int MAT, bool FIXED, bool PAGED>
static FusedFn fused_for(int ci) {
    static_assert(kNumFusedKernels == 12, "update the dispatch table");
    switch (kFusedCfgs[ci].kernel) {
        case 0: return fused_kernel<D, MAT, 0, FIXED, PAGED>();
        case 1: return fused_kernel<D, MAT, 1, FIXED, PAGED>();
        case 2: return fused_kernel<D, MAT, 2, FIXED, PAGED>();
        case 3: return fused_kernel<D, MAT, 3, FIXED, PAGED>();
        case 4: return fused_kernel<D, MAT, 4, FIXED, PAGED>();
        case 5: return fused_kernel<D, MAT, 5, FIXED, PAGED>();
        case 6: return fused_kernel<D, MAT, 6, FIXED, PAGED>();
        case 7: return fused_kernel<D, MAT, 7, FIXED, PAGED>();
        case 8: return fused_kernel<D, MAT, 8, FIXED, PAGED>();
        case 9: return fused_kernel<D, MAT, 9, FIXED, PAGED>();
        case 10: return fused_kernel<D, MAT, 10, FIXED, PAGED>();
        default: return fused_kernel<D, MAT, 11, FIXED, PAGED>();
    }
}

template <int D, bool FIXED, bool PAGED>
static FusedFn fused_for_mat(int mat, int ci) {
    if (mat == JELLO) return fused_for<D, JELLO, FIXED, PAGED>(ci);
    if (mat == SNOW) return fused_for<D, SNOW, FIXED, PAGED>(ci);
    return fused_for<D, WATER, FIXED, PAGED>(ci);
}

template <bool FIXED, bool PAGED>
static FusedFn fused_table(int dim, int mat, int ci) {
    return dim == 3 ? fused_for_mat<3, FIXED, PAGED>(mat, ci) : fused_for_mat<2, FIXED, PAGED>(mat, ci);
}

}  // namespace mpm
