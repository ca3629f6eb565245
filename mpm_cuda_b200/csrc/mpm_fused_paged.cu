// Instantiations of the fused substep kernel for a paged grid
// (mpm_options.grid_pool_blocks > 0), direct-scatter configurations, reading
// the scene from the device table (several scenes or adaptive dt).
#include "mpm_fused_table.cuh"

namespace mpm {

FusedFn fused_fn_paged_fixed(int dim, int mat, int ci);  // mpm_fused_paged_fixed.cu

FusedFn fused_fn_paged(int dim, int mat, int ci, bool fixed) {
    return fixed ? fused_fn_paged_fixed(dim, mat, ci) : fused_table<false, true>(dim, mat, ci);
}

}  // namespace mpm
