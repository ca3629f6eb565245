// Launch configurations of the fused substep kernel (the autotuner's search
// space), shared by the kernels and the C-ABI layer.
#pragma once

namespace mpm {

// chunk: threads per CTA; min_ctas: the minimum resident CTAs per SM given to
// __launch_bounds__ (which caps registers at 65536 / (chunk * min_ctas));
// rounds: particles each thread processes per chunk, one after the other, so a
// chunk holds chunk * rounds particles and one velocity window and one pair of
// CTA barriers serve them all; kernel: the instantiation the configuration
// launches (configurations differing only in rounds share one).
struct FusedCfg {
    int chunk;
    int min_ctas;
    int rounds;
    int kernel;
};
constexpr int kNumFusedKernels = 8;
constexpr int kNumFusedCfgs = 12;
constexpr FusedCfg kFusedCfgs[kNumFusedCfgs] = {
    {128, 4, 1, 0}, {128, 5, 1, 1}, {128, 6, 1, 2}, {64, 8, 1, 3},  {64, 10, 1, 4},  {64, 12, 1, 5},
    {256, 2, 1, 6}, {256, 3, 1, 7}, {128, 5, 2, 1}, {128, 6, 2, 2}, {64, 10, 2, 4}, {256, 3, 2, 7}};
// fewest particles a chunk of any configuration holds (sizes the chunk lists)
constexpr int kMinChunkParticles = 64;

constexpr bool fused_cfgs_consistent() {
    for (int i = 0; i < kNumFusedCfgs; ++i) {
        const FusedCfg& c = kFusedCfgs[i];
        const FusedCfg& k = kFusedCfgs[c.kernel];
        if (c.kernel >= kNumFusedKernels || k.chunk != c.chunk || k.min_ctas != c.min_ctas || k.rounds != 1 ||
            c.chunk * c.rounds < kMinChunkParticles || c.chunk % 32 != 0)
            return false;
    }
    return true;
}
static_assert(fused_cfgs_consistent(), "each configuration names the instantiation of its chunk and CTAs per SM");

}  // namespace mpm
