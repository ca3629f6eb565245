// C-ABI of the B200 MPM substep (declared in include/mpm_b200.h).
//
// A handle owns: the particle state of every scene (FP32 component planes,
// all scenes concatenated), the per-scene blocked grids, the group/scene
// parameter tables, a CUDA stream and the CUDA graph of one substep.
#include "mpm_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mpm_config.cuh"
#include "mpm_engine.cuh"
#include "mpm_surrogate.cuh"

namespace {

thread_local std::string g_thread_error;

}  // namespace

using mpm::Engine;

namespace mpm {
// error text of calls that have no handle (read back by mpm_last_error(NULL))
void set_thread_error(const char* msg) { g_thread_error = msg ? msg : ""; }
}  // namespace mpm

struct mpm_handle {
    Engine eng;
};

static int fail(mpm_handle* h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->eng.last_error = buf;
    else g_thread_error = buf;
    return code;
}

extern "C" {

void mpm_default_options(mpm_options* opt) {
    if (!opt) return;
    opt->p2g_mode = MPM_P2G_ATOMIC;
    opt->stress_mode = MPM_STRESS_PLAIN;
    opt->adaptive_dt = 0;
    opt->cfl = 0.5f;
    opt->use_graph = 1;
    opt->block_threads = 0;
    opt->device = 0;
    opt->rebin_interval = 0;
    opt->kernel_config = -1;
    opt->grid_pool_blocks = 0;
}

int mpm_create(const mpm_scene_desc* scenes, int n_scenes, const mpm_options* opt,
               mpm_handle** out) {
    if (!out) return fail(nullptr, MPM_ERR_INVALID, "mpm_create: out is NULL");
    *out = nullptr;
    mpm_options o;
    mpm_default_options(&o);
    if (opt) o = *opt;
    auto* h = new (std::nothrow) mpm_handle();
    if (!h) return fail(nullptr, MPM_ERR_NOMEM, "mpm_create: host allocation failed");
    std::string msg;
    int rc = h->eng.create(scenes, n_scenes, o, msg);
    if (rc != MPM_OK) {
        g_thread_error = msg;
        delete h;
        return rc;
    }
    *out = h;
    return MPM_OK;
}

int mpm_destroy(mpm_handle* h) {
    if (!h) return MPM_OK;
    h->eng.release();
    delete h;
    return MPM_OK;
}

int mpm_step(mpm_handle* h, int n) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_step: NULL handle");
    int rc = h->eng.step(n);
    if (rc != MPM_OK) return rc;
    return h->eng.sync_and_check();
}

int mpm_step_async(mpm_handle* h, int n) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_step_async: NULL handle");
    return h->eng.step(n);
}

int mpm_synchronize(mpm_handle* h) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_synchronize: NULL handle");
    return h->eng.sync_and_check();
}

int mpm_get_device_errors(mpm_handle* h, uint32_t* bits) {
    if (!h || !bits) return fail(h, MPM_ERR_INVALID, "mpm_get_device_errors: bad argument");
    return h->eng.read_errors(bits);
}

int mpm_clear_device_errors(mpm_handle* h) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_clear_device_errors: NULL handle");
    return h->eng.clear_errors();
}

int mpm_get_stream(mpm_handle* h, void** stream) {
    if (!h || !stream) return fail(h, MPM_ERR_INVALID, "mpm_get_stream: bad argument");
    *stream = (void*)h->eng.stream;
    return MPM_OK;
}

int mpm_num_particles(mpm_handle* h, int scene, int64_t* n) {
    if (!h || !n) return fail(h, MPM_ERR_INVALID, "mpm_num_particles: bad argument");
    if (scene < 0) {
        *n = h->eng.n_particles;
        return MPM_OK;
    }
    if (scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_num_particles: scene %d out of range", scene);
    *n = h->eng.scene_count[scene];
    return MPM_OK;
}

int mpm_get_positions(mpm_handle* h, int scene, float* x, size_t cap) {
    if (!h || !x) return fail(h, MPM_ERR_INVALID, "mpm_get_positions: bad argument");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_get_positions: scene %d out of range", scene);
    size_t need = (size_t)h->eng.scene_count[scene] * h->eng.dim;
    if (cap < need)
        return fail(h, MPM_ERR_INVALID, "mpm_get_positions: cap %zu < %zu floats", cap, need);
    return h->eng.get_positions(scene, x);
}

int mpm_get_positions_async(mpm_handle* h, int scene, float* x, size_t cap, int64_t* ticket) {
    if (!h || !x) return fail(h, MPM_ERR_INVALID, "mpm_get_positions_async: bad argument");
    if (scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_get_positions_async: scene %d out of range", scene);
    size_t need = (size_t)(scene < 0 ? h->eng.n_particles : h->eng.scene_count[scene]) * h->eng.dim;
    if (cap < need)
        return fail(h, MPM_ERR_INVALID, "mpm_get_positions_async: cap %zu < %zu floats", cap, need);
    long long t = -1;
    const int rc = h->eng.get_positions_async(scene, x, &t);
    if (ticket) *ticket = t;
    return rc;
}

int mpm_wait_positions(mpm_handle* h, int64_t ticket) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_wait_positions: NULL handle");
    return h->eng.wait_positions(ticket);
}

int mpm_get_state(mpm_handle* h, int scene, float* x, float* v, float* C, float* F, float* aux) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_state: NULL handle");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_get_state: scene %d out of range", scene);
    return h->eng.get_state(scene, x, v, C, F, aux);
}

int mpm_set_state(mpm_handle* h, int scene, const float* x, const float* v, const float* C,
                  const float* F, const float* aux) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_set_state: NULL handle");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_set_state: scene %d out of range", scene);
    return h->eng.set_state(scene, x, v, C, F, aux);
}

int mpm_get_grid(mpm_handle* h, int scene, float* mass, float* vel) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_grid: NULL handle");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_get_grid: scene %d out of range", scene);
    return h->eng.get_grid(scene, mass, vel);
}

int mpm_count_active_nodes(mpm_handle* h, int scene, int64_t* n) {
    if (!h || !n) return fail(h, MPM_ERR_INVALID, "mpm_count_active_nodes: bad argument");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_count_active_nodes: scene %d out of range", scene);
    return h->eng.count_active_nodes(scene, n);
}

int mpm_get_bin_stats(mpm_handle* h, int64_t* fallbacks, int64_t* rebins) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_bin_stats: NULL handle");
    return h->eng.bin_stats(fallbacks, rebins);
}

int mpm_get_grid_pool(mpm_handle* h, int64_t* capacity, int64_t* in_use) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_grid_pool: NULL handle");
    return h->eng.grid_pool(capacity, in_use);
}

int mpm_num_kernel_configs(void) { return mpm::kNumFusedCfgs; }

int mpm_kernel_config_info(int config, int* chunk, int* min_ctas, int* rounds) {
    if (config < 0 || config >= mpm::kNumFusedCfgs)
        return fail(nullptr, MPM_ERR_INVALID, "mpm_kernel_config_info: config %d out of range", config);
    if (chunk) *chunk = mpm::kFusedCfgs[config].chunk;
    if (min_ctas) *min_ctas = mpm::kFusedCfgs[config].min_ctas;
    if (rounds) *rounds = mpm::kFusedCfgs[config].rounds;
    return MPM_OK;
}

int mpm_kernel_config_scatter(int config, int* cell_major, int* segmented) {
    if (config < 0 || config >= mpm::kNumFusedCfgs)
        return fail(nullptr, MPM_ERR_INVALID, "mpm_kernel_config_scatter: config %d out of range", config);
    if (cell_major) *cell_major = mpm::kFusedCfgs[config].order == mpm::ORDER_CELL ? 1 : 0;
    if (segmented) *segmented = mpm::kFusedCfgs[config].scatter == mpm::SCATTER_SEGMENTED ? 1 : 0;
    return MPM_OK;
}

int mpm_get_kernel_config(mpm_handle* h, int* config) {
    if (!h || !config) return fail(h, MPM_ERR_INVALID, "mpm_get_kernel_config: bad argument");
    *config = h->eng.cfg;
    return MPM_OK;
}

int mpm_set_kernel_config(mpm_handle* h, int config) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_set_kernel_config: NULL handle");
    if (config < 0 || config >= mpm::kNumFusedCfgs)
        return fail(h, MPM_ERR_INVALID, "mpm_set_kernel_config: config %d out of range", config);
    if (h->eng.paged && mpm::kFusedCfgs[config].scatter != mpm::SCATTER_DIRECT)
        return fail(h, MPM_ERR_UNSUPPORTED, "mpm_set_kernel_config: config %d scatters into a dense grid", config);
    h->eng.set_config(config);
    return MPM_OK;
}

int mpm_autotune(mpm_handle* h, int n_substeps, int* chosen, float* ms_per_substep) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_autotune: NULL handle");
    int rc = h->eng.autotune(n_substeps, ms_per_substep);
    if (rc == MPM_OK && chosen) *chosen = h->eng.cfg;
    return rc;
}

int mpm_get_time(mpm_handle* h, double* t, int64_t* frame) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_time: NULL handle");
    if (frame) *frame = h->eng.current_frame;
    if (!t) return MPM_OK;
    if (h->eng.opt.adaptive_dt) return h->eng.scene_time_of(0, t, nullptr);
    *t = h->eng.current_time;
    return MPM_OK;
}

int mpm_get_scene_time(mpm_handle* h, int scene, double* t, float* dt) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_scene_time: NULL handle");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_get_scene_time: scene %d out of range", scene);
    return h->eng.scene_time_of(scene, t, dt);
}

int mpm_write_bgeo(mpm_handle* h, int scene, const char* path) {
    if (!h || !path) return fail(h, MPM_ERR_INVALID, "mpm_write_bgeo: bad argument");
    if (scene < 0 || scene >= (int)h->eng.scenes_h.size())
        return fail(h, MPM_ERR_INVALID, "mpm_write_bgeo: scene %d out of range", scene);
    std::vector<float> x((size_t)h->eng.scene_count[scene] * h->eng.dim);
    int rc = h->eng.get_state(scene, x.data(), nullptr, nullptr, nullptr, nullptr);
    if (rc != MPM_OK) return rc;
    if (mpm::write_bgeo(path, x.data(), h->eng.scene_count[scene], h->eng.dim) != 0)
        return fail(h, MPM_ERR_IO, "mpm_write_bgeo: cannot write %s", path);
    return MPM_OK;
}

int mpm_write_bgeo_positions(const char* path, const float* x, int64_t n) {
    if (mpm::write_bgeo(path, x, n, 3) != 0)
        return fail(nullptr, MPM_ERR_IO, "mpm_write_bgeo_positions: cannot write %s",
                    path ? path : "(null)");
    return MPM_OK;
}

int mpm_set_p2g_mode(mpm_handle* h, int mode) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_set_p2g_mode: NULL handle");
    if (mode != MPM_P2G_ATOMIC && mode != MPM_P2G_DETERMINISTIC && mode != MPM_P2G_DIRECT)
        return fail(h, MPM_ERR_INVALID, "mpm_set_p2g_mode: bad mode %d", mode);
    return h->eng.set_p2g_mode(mode);
}

int mpm_set_stress_mode(mpm_handle* h, int mode, mpm_surrogate* s) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_set_stress_mode: NULL handle");
    return h->eng.set_stress_mode(mode, mpm::surrogate_of(s));
}

int mpm_get_stress_stats(mpm_handle* h, int64_t* surrogate, int64_t* fallback) {
    if (!h) return fail(nullptr, MPM_ERR_INVALID, "mpm_get_stress_stats: NULL handle");
    return h->eng.stress_stats(surrogate, fallback);
}

int mpm_last_error(mpm_handle* h, char* buf, size_t cap) {
    if (!buf || cap == 0) return MPM_ERR_INVALID;
    const std::string& s = h ? h->eng.last_error : g_thread_error;
    std::snprintf(buf, cap, "%s", s.c_str());
    return MPM_OK;
}

int mpm_profile_stages(mpm_handle* h, int n, float* out_ms, int n_out, int* n_written) {
    if (!h || !out_ms || n <= 0) return fail(h, MPM_ERR_INVALID, "mpm_profile_stages: bad argument");
    return h->eng.profile_stages(n, out_ms, n_out, n_written);
}

}  // extern "C"
