// Engine behind the C-ABI handle: device memory, stream, substep graphs.
#pragma once

#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "mpm_b200.h"
#include "mpm_types.cuh"

namespace mpm {

int write_bgeo(const char* path, const float* x, int64_t n, int dim);

struct Chunk;
struct FusedArgs;
struct Surrogate;

struct Engine {
    int dim = 3;
    int device = 0;
    cudaStream_t stream = nullptr;
    mpm_options opt{};
    int num_sms = 148;

    // host copies of the tables
    std::vector<SceneParams> scenes_h;
    std::vector<GroupParams> groups_h;
    std::vector<long long> scene_begin, scene_count;  // creation-order ranges
    long long n_particles = 0;
    long long cap = 0;
    int n_planes = 0;
    long long total_blocks = 0;

    // particle state: two buffers (sorted / re-binning target)
    int cur = 0;
    float* st[2] = {nullptr, nullptr};
    uint16_t* gp[2] = {nullptr, nullptr};
    uint32_t* ids[2] = {nullptr, nullptr};

    GroupParams* groups_d = nullptr;
    SceneParams* scenes_d = nullptr;
    float4* grid_mom = nullptr;  // P2G accumulation (momentum, mass)
    float4* grid_vel = nullptr;  // after the grid update (velocity, mass)
    unsigned* err_d = nullptr;

    // binning and block activity
    // binning: keys[0] = (home block, material, cell) and vals[0] = rank in
    // the cell of each particle; the deterministic mode sorts keys / vals
    unsigned long long* keys[2] = {nullptr, nullptr};
    unsigned* vals[2] = {nullptr, nullptr};
    // binning: per (block, present material) 64 cell counts; the
    // deterministic mode: per base node of every block
    int* cell_count = nullptr;
    MatSlots mat_slots{};       // compact index of each present material
    int* cell_end = nullptr;    // deterministic mode: end of each base node's records
    float* det_src = nullptr;   // deterministic mode: P2G source records
    float* det_sorted = nullptr;  // the same records in sorted order
    int* det_blocks = nullptr;    // the blocks they mark, ascending
    int* det_runs = nullptr;      // first sorted position of each run sharing a base node
    float4* det_partial = nullptr;  // per (run, stencil offset) partial sums (allocated on first use)
    int det_key_bits = 64;
    // sort key of a particle whose stencil left the grid: one past the last node
    unsigned long long det_no_cell() const { return (unsigned long long)total_blocks * 64; }
    bool sorted_order = false;  // particles permuted away from creation order
    int* seg_count = nullptr;   // per (block, material)
    int* seg_start = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    void* scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    Chunk* chunks = nullptr;    // kMats lists of list_cap entries
    long long list_cap = 0;
    bool mat_present[3] = {false, false, false};
    int* counters = nullptr;    // see CNT_* in mpm_engine.cu
    unsigned* blk_flag = nullptr;
    int* active = nullptr;
    int* blk_epoch = nullptr;
    float* pos_out = nullptr;  // gathered positions (creation order)
    // asynchronous position reads: a ring of staging buffers, each gathered on
    // `stream` and copied to the host on `copy_stream`; created on first use
    static constexpr int kPosSlots = 3;
    struct PosSlot {
        float* dev = nullptr;
        cudaEvent_t gathered = nullptr;  // gather done (recorded on stream)
        cudaEvent_t copied = nullptr;    // host copy done (recorded on copy_stream)
        long long ticket = -1;           // last ticket that used the slot
    };
    PosSlot pos_slots[kPosSlots];
    cudaStream_t copy_stream = nullptr;
    long long next_ticket = 0;
    int fused_ctas[3] = {0, 0, 0};  // persistent CTAs per material kernel
    int cfg = 1;                     // index into kFusedCfgs
    // particles per chunk of the current configuration (CTA size x rounds)
    int chunk_particles() const;
    bool fixed_scene = false;        // one scene, fixed dt: fused kernels take it as a parameter
    // paged grid (mpm_options.grid_pool_blocks > 0): the grid arrays hold
    // pool_cap physical blocks plus the trash block; `pages` points at the
    // device page table, the physical-to-virtual map and the free stack
    bool paged = false;
    long long pool_cap = 0;
    GridPages pages{};
    long long grid_blocks_alloc() const { return paged ? pool_cap + 1 : total_blocks; }
    // the state's v planes hold the last G2P positions and C is stale: the
    // fused kernels deferred them (k_recover_vc rebuilds both)
    bool vc_deferred = false;
    bool defer_vc_now() const;
    // the single-scene dense fused path keeps grid velocities in the linear
    // layout and loads its windows as boxes of vel_map (encoded at creation);
    // vel_lin_state: the layout of what grid_vel holds now (the last grid
    // update's), for the readers outside the fused pass
    CUtensorMap vel_map{};
    bool vel_lin_state = false;
    bool vel_linear_mode() const { return fixed_scene && !paged && fused(); }
    int encode_vel_map();
    int recover_vc();
    // learned stress (MPM_STRESS_SURROGATE): the network, the version of its
    // weights the graphs were captured with, per-material persistent CTAs and
    // the network / fallback counters
    Surrogate* sur = nullptr;
    long long sur_version = -1;
    int sur_ctas[3] = {0, 0, 0};
    unsigned long long* sur_counts = nullptr;
    // adaptive dt: per scene max signal speed of the last pass (float bits) and
    // simulated time (the device owns the clock when dt adapts)
    unsigned* speed_max = nullptr;
    double* scene_time = nullptr;
    int update_ctas = 0;
    int steps_since_rebin = 0;

    // substep graphs: [parity][rebin first]
    cudaGraphExec_t graphs[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    // per parity: the rebin_interval - 1 plain substeps between two re-binnings
    cudaGraphExec_t run_graphs[2] = {nullptr, nullptr};
    bool grid_dirty = true;  // grid_mom does not hold the P2G of the current state

    double current_time = 0.0;
    long long current_frame = 0;
    std::string last_error;
    std::string launch_error;  // first failed launch since the last check

    int create(const mpm_scene_desc* scenes, int n_scenes, const mpm_options& o, std::string& msg);
    void release();
    int step(int n);
    int sync_and_check();
    int read_errors(uint32_t* bits);
    int clear_errors();
    int get_state(int scene, float* x, float* v, float* C, float* F, float* aux);
    int set_state(int scene, const float* x, const float* v, const float* C, const float* F,
                  const float* aux);
    int get_grid(int scene, float* mass, float* vel);
    int count_active_nodes(int scene, int64_t* n);
    int set_p2g_mode(int mode);
    int alloc_det_partials();
    int set_stress_mode(int mode, Surrogate* s);
    int stress_stats(int64_t* net, int64_t* fallback);
    int scene_time_of(int scene, double* t, float* dt);
    int profile_stages(int n, float* out_ms, int n_out, int* n_written);
    int get_positions(int scene, float* out);
    int get_positions_async(int scene, float* out, long long* ticket);
    int wait_positions(long long ticket);
    int bin_stats(int64_t* fallbacks, int64_t* rebins);
    int grid_pool(int64_t* capacity, int64_t* in_use);
    void set_config(int ci);
    int autotune(int steps, float* best_ms);
    int cached_config() const;

   private:
    int cuda_fail(cudaError_t e, const char* what);
    void note_launch(const char* what);
    void note_launch_status(const char* what, cudaError_t e);
    int take_launch_error();
    ParticleBuf buf(int p) const { return ParticleBuf{st[p], cap, gp[p], ids[p]}; }
    void enqueue_direct_substep();
    void enqueue_rebin(int from, bool in_loop = true);
    void enqueue_page_in_particles();
    int download_grid(const SceneParams& sc, std::vector<float4>& blk);
    void enqueue_fused_substep(int parity);
    void enqueue_grid_update();
    void enqueue_adapt_dt();
    void enqueue_g2p2g(int parity);
    FusedArgs fused_args(int mat, bool bump);
    int prologue();
    int build_graph(int parity, int rebin, int count, cudaGraphExec_t* out);
    void drop_graphs();
    int unpermute_to_alt();
    bool fused() const { return opt.p2g_mode == MPM_P2G_ATOMIC; }
    bool deterministic() const { return opt.p2g_mode == MPM_P2G_DETERMINISTIC; }
    bool direct() const { return opt.p2g_mode == MPM_P2G_DIRECT; }
    // jello only: snow's exact stress reuses its plasticity decomposition
    bool sur_kernel(int mat) const { return sur && dim == 3 && mat == JELLO; }
    void sur_occupancy();
    int sur_chunk() const;
    int sur_refresh();
    void enqueue_det_p2g();
    void enqueue_det_substep();
    int canonical_order();
};

}  // namespace mpm
