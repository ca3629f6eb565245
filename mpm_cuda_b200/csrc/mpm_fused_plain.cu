// Instantiations of the fused substep kernel that read each chunk's scene
// from the device scene table (several scenes, or adaptive dt), for every
// dimension, material and launch configuration (the autotuner's search space).
#include "mpm_fused_table.cuh"

namespace mpm {

FusedFn fused_fn_fixed(int dim, int mat, int ci);         // mpm_fused_fixed.cu
FusedFn fused_fn_paged(int dim, int mat, int ci, bool fixed);  // mpm_fused_paged.cu

FusedFn fused_fn(int dim, int mat, int ci, bool fixed_scene, bool paged) {
    if (paged) return fused_fn_paged(dim, mat, ci, fixed_scene);
    return fixed_scene ? fused_fn_fixed(dim, mat, ci) : fused_table<false, false>(dim, mat, ci);
}

}  // namespace mpm
