// Launch configurations of the fused substep kernel (the autotuner's search
// space), shared by the kernels and the C-ABI layer.
#pragma once

namespace mpm {

// Instantiations of the fused kernel.  chunk: threads per CTA; min_ctas: the
// minimum resident CTAs per SM given to __launch_bounds__ (which caps
// registers at 65536 / (chunk * min_ctas)); scatter: how the P2G of the next
// substep reaches the grid -- SCATTER_DIRECT: every particle reduces its 3^D
// node values into global memory (red.global.add.v4.f32); SCATTER_SEGMENTED:
// the lanes of a warp that share a stencil base (a cell, in cell-major order)
// are summed in shared memory first and each sum is reduced once (the
// per-warp staging buffer limits these kernels to fewer CTAs per SM).
enum : int { SCATTER_DIRECT = 0, SCATTER_SEGMENTED = 1 };
struct FusedKernel {
    int chunk;
    int min_ctas;
    int scatter;
};
constexpr int kNumFusedKernels = 12;
constexpr FusedKernel kFusedKernels[kNumFusedKernels] = {
    {128, 4, 0}, {128, 5, 0}, {128, 6, 0}, {64, 8, 0}, {64, 10, 0}, {64, 12, 0}, {256, 2, 0}, {256, 3, 0},
    {64, 5, 1},  {128, 3, 1}, {64, 4, 1},  {128, 2, 1}};

// A launch configuration (the autotuner's search space): an instantiation,
// rounds -- particles each thread processes per chunk, one after the other,
// so a chunk holds chunk * rounds particles and one velocity window and one
// pair of CTA barriers serve them all -- and order: how the re-binning orders
// the particles of a (block, material) segment.  ORDER_RANK: rank-major
// (every cell's first particle, then every cell's second, ...), so a warp's
// 32 lanes sit in 32 different cells and every scatter instruction hits 32
// different nodes; ORDER_CELL: cell-major (a cell's particles together), so
// the lanes of one cell gather the same nodes (shared-memory broadcasts) and
// scatter into the same nodes.
enum : int { ORDER_RANK = 0, ORDER_CELL = 1 };
struct FusedCfg {
    int chunk;
    int min_ctas;
    int rounds;
    int kernel;
    int order;
    int scatter;
};
struct FusedCfgTable {
    static constexpr int N = 36;
    FusedCfg c[N];
    // 0..11 direct scatter, rank-major; 12..23 the same shapes cell-major;
    // 24..31 segmented scatter (cell-major), one and two rounds; 32..35 the
    // 64-thread, 10-CTA direct kernel with three and four rounds, rank-major
    // and cell-major (fewer window loads and barrier pairs per particle; on
    // the 2M-particle scenes 3-4 % faster than two rounds)
    constexpr FusedCfgTable() : c{} {
        constexpr int kr[12][2] = {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {4, 1}, {5, 1},
                                   {6, 1}, {7, 1}, {1, 2}, {2, 2}, {4, 2}, {7, 2}};
        constexpr int sr[8][2] = {{8, 1}, {9, 1}, {10, 1}, {11, 1}, {8, 2}, {9, 2}, {10, 2}, {11, 2}};
        for (int i = 0; i < 24; ++i) {
            const int k = kr[i % 12][0];
            c[i] = FusedCfg{kFusedKernels[k].chunk, kFusedKernels[k].min_ctas, kr[i % 12][1], k,
                            i < 12 ? ORDER_RANK : ORDER_CELL, SCATTER_DIRECT};
        }
        for (int i = 0; i < 8; ++i) {
            const int k = sr[i][0];
            c[24 + i] = FusedCfg{kFusedKernels[k].chunk, kFusedKernels[k].min_ctas, sr[i][1], k, ORDER_CELL,
                                 SCATTER_SEGMENTED};
        }
        for (int i = 0; i < 4; ++i)
            c[32 + i] = FusedCfg{kFusedKernels[4].chunk, kFusedKernels[4].min_ctas, 3 + i % 2, 4,
                                 i < 2 ? ORDER_RANK : ORDER_CELL, SCATTER_DIRECT};
    }
    constexpr const FusedCfg& operator[](int i) const { return c[i]; }
};
constexpr FusedCfgTable kFusedCfgs{};
constexpr int kNumFusedCfgs = FusedCfgTable::N;
// fewest particles a chunk of any configuration holds (sizes the chunk lists)
constexpr int kMinChunkParticles = 64;

// dynamic shared memory of a fused kernel: the segmented scatter's staging
// buffer, 3^D node values of each of a warp's 32 lanes
constexpr int seg_rows(int dim) { return dim == 3 ? 27 : 9; }
constexpr int fused_dyn_smem(int dim, int kernel) {
    return kFusedKernels[kernel].scatter == SCATTER_SEGMENTED
               ? kFusedKernels[kernel].chunk / 32 * seg_rows(dim) * 32 * 16
               : 0;
}

// the direct-scatter instantiation with a kernel's chunk (the learned-stress
// kernel, which scatters directly, runs with that shape)
constexpr int direct_kernel_of(int kernel) {
    return kFusedKernels[kernel].scatter == SCATTER_DIRECT ? kernel : (kFusedKernels[kernel].chunk == 64 ? 3 : 0);
}

constexpr bool fused_cfgs_consistent() {
    for (int i = 0; i < kNumFusedCfgs; ++i) {
        const FusedCfg& c = kFusedCfgs[i];
        if (c.kernel < 0 || c.kernel >= kNumFusedKernels) return false;
        const FusedKernel& k = kFusedKernels[c.kernel];
        if (k.chunk != c.chunk || k.min_ctas != c.min_ctas || k.scatter != c.scatter ||
            (c.order != ORDER_RANK && c.order != ORDER_CELL) ||
            (c.scatter == SCATTER_SEGMENTED && c.order != ORDER_CELL) ||
            c.chunk * c.rounds < kMinChunkParticles || c.chunk % 32 != 0)
            return false;
    }
    for (int k = 0; k < kNumFusedKernels; ++k)
        if (kFusedKernels[direct_kernel_of(k)].scatter != SCATTER_DIRECT ||
            kFusedKernels[direct_kernel_of(k)].chunk != kFusedKernels[k].chunk)
            return false;
    return true;
}
static_assert(fused_cfgs_consistent(), "each configuration names the instantiation of its launch shape");

}  // namespace mpm
