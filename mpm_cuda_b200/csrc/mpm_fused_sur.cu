// Instantiations of the fused substep kernel with the learned stress (3D
// jello) for every launch configuration.
#include "mpm_dispatch.cuh"

namespace mpm {

// The learned-stress kernel for a CTA size (64 or 128 threads; the engine
// picks 128 when the chunk holds a multiple of 128 particles), with launch
// bounds at the CTAs per SM its shared memory allows (velocity windows,
// network weights, network and stash rows: 5 CTAs of 64, 4 of 128 threads),
// so its registers are not capped below what that occupancy leaves them.
template <int CHUNK, bool FIXED, bool PAGED>
static constexpr auto sur_kernel() {
    return &k_g2p2g_sur<CHUNK, CHUNK == 64 ? 5 : 4, FIXED, PAGED>;
}

template <bool PAGED>
static SurFn sur_for(int cta, bool fixed_scene) {
    if (cta == 64) return fixed_scene ? sur_kernel<64, true, PAGED>() : sur_kernel<64, false, PAGED>();
    return fixed_scene ? sur_kernel<128, true, PAGED>() : sur_kernel<128, false, PAGED>();
}

SurFn sur_fn(int cta, bool fixed_scene, bool paged) {
    return paged ? sur_for<true>(cta, fixed_scene) : sur_for<false>(cta, fixed_scene);
}

}  // namespace mpm
