// Engine behind the C-ABI handle: device memory, stream, substep graph.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "mpm_b200.h"
#include "mpm_types.cuh"

namespace mpm {

int write_bgeo(const char* path, const float* x, int64_t n, int dim);

struct Engine {
    int dim = 3;
    int device = 0;
    cudaStream_t stream = nullptr;
    mpm_options opt{};

    // host copies of the tables
    std::vector<SceneParams> scenes_h;
    std::vector<GroupParams> groups_h;
    std::vector<long long> scene_begin, scene_count;  // creation-order ranges
    long long n_particles = 0;
    long long cap = 0;
    int n_planes = 0;
    long long total_blocks = 0;

    // device memory
    float* state = nullptr;      // current particle planes
    float* state_alt = nullptr;  // scratch / sort target
    uint16_t* grp = nullptr;
    uint16_t* grp_alt = nullptr;
    uint32_t* id = nullptr;
    uint32_t* id_alt = nullptr;
    GroupParams* groups_d = nullptr;
    SceneParams* scenes_d = nullptr;
    float4* grid_mom = nullptr;  // P2G accumulation (momentum, mass)
    float4* grid_vel = nullptr;  // after the grid update (velocity, mass)
    unsigned* err_d = nullptr;

    cudaGraphExec_t graph_exec = nullptr;
    bool graph_dirty = true;

    double current_time = 0.0;
    long long current_frame = 0;
    std::string last_error;

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
    int profile_stages(int n, float* out_ms, int n_out, int* n_written);

   private:
    int cuda_fail(cudaError_t e, const char* what);
    void enqueue_substep();
    int build_graph();
    void drop_graph();
    int unpermute_to_alt();
};

}  // namespace mpm
