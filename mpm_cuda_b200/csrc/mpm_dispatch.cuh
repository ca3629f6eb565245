// Kernel tables of the fused substep: the plain and surrogate-stress kernels
// for a (dimension, material, launch configuration).
#pragma once

#include "mpm_config.cuh"
#include "mpm_kernels_binned.cuh"
#include "mpm_kernels_surrogate.cuh"

namespace mpm {

using FusedFn = void (*)(ParticleBuf, FusedArgs);
using SurFn = void (*)(ParticleBuf, FusedArgs, SurArgs);

// k_g2p2g<dim, mat, kFusedCfgs[ci], fixed_scene, paged>; fixed_scene: one
// scene whose parameters do not change during the run, passed in
// FusedArgs::scene; paged: a paged grid (direct-scatter configurations only:
// nullptr for the others)
FusedFn fused_fn(int dim, int mat, int ci, bool fixed_scene, bool paged);
// k_g2p2g_sur with `cta` threads (64 or 128), fixed_scene, paged (3D jello)
SurFn sur_fn(int cta, bool fixed_scene, bool paged);

}  // namespace mpm
