// Instantiations of the fused substep kernel for a single scene with a fixed
// dt: the scene's constants come from the kernel parameters, so the kernel
// neither loads them nor keeps them in registers.
#include "mpm_fused_table.cuh"

namespace mpm {

FusedFn fused_fn_fixed(int dim, int mat, int ci) { return fused_table<true, false>(dim, mat, ci); }

}  // namespace mpm
