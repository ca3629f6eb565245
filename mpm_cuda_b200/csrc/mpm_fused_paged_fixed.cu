// Instantiations of the fused substep kernel for a paged grid and a single
// scene with a fixed dt (the scene from the kernel parameters).
#include "mpm_fused_table.cuh"

namespace mpm {

FusedFn fused_fn_paged_fixed(int dim, int mat, int ci) { return fused_table<true, true>(dim, mat, ci); }

}  // namespace mpm
