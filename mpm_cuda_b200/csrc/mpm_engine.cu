// Engine implementation: validation, allocation, state I/O and the substep
// launch sequence.
#include "mpm_engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "mpm_kernels_direct.cuh"

namespace mpm {

namespace {

constexpr int kMaxGroups = 65535;

// out[id[i]] = in[i] for every plane (storage order -> creation order)
__global__ void k_unpermute(const float* __restrict__ in, float* __restrict__ out, const uint32_t* __restrict__ id,
                            long long n, long long cap, int planes) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = id[i];
    for (int p = 0; p < planes; ++p) out[p * cap + j] = in[p * cap + i];
}

// out[i] = in[id[i]] for particles whose creation index lies in [lo, hi)
__global__ void k_permute_range(const float* __restrict__ in, float* __restrict__ out, const uint32_t* __restrict__ id,
                                long long n, long long cap, int planes, long long lo, long long hi) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = id[i];
    if (j < lo || j >= hi) return;
    for (int p = 0; p < planes; ++p) out[p * cap + i] = in[p * cap + j];
}

unsigned grid_blocks(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int Engine::cuda_fail(cudaError_t e, const char* what) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    last_error = buf;
    return e == cudaErrorMemoryAllocation ? MPM_ERR_NOMEM : MPM_ERR_CUDA;
}

#define MPM_CUDA_TRY(expr, what)                     \
    do {                                             \
        cudaError_t e_ = (expr);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

int Engine::create(const mpm_scene_desc* scenes, int n_scenes, const mpm_options& o,
                   std::string& msg) {
    opt = o;
    char buf[512];
    auto bad = [&](int code, const char* text) {
        msg = text;
        return code;
    };
    if (!scenes || n_scenes <= 0) return bad(MPM_ERR_INVALID, "mpm_create: no scenes");
    dim = scenes[0].dim;
    if (dim != 2 && dim != 3) return bad(MPM_ERR_INVALID, "mpm_create: dim must be 2 or 3");
    long long total_groups = 0;
    n_particles = 0;
    for (int s = 0; s < n_scenes; ++s) {
        const mpm_scene_desc& d = scenes[s];
        if (d.dim != dim) return bad(MPM_ERR_INVALID, "mpm_create: every scene of a handle must have the same dim");
        for (int a = 0; a < dim; ++a)
            if (d.n[a] < 4) {
                std::snprintf(buf, sizeof(buf), "mpm_create: scene %d has fewer than 4 nodes on axis %d", s, a);
                return bad(MPM_ERR_INVALID, buf);
            }
        if (!(d.h > 0.0) || !(d.dt > 0.0)) {
            std::snprintf(buf, sizeof(buf), "mpm_create: scene %d needs h > 0 and dt > 0", s);
            return bad(MPM_ERR_INVALID, buf);
        }
        if (d.bc_type < MPM_BC_STICKY || d.bc_type > MPM_BC_SEPARATE || d.bc_lo < 0 || d.bc_hi < 0)
            return bad(MPM_ERR_INVALID, "mpm_create: bad boundary descriptor");
        if (d.n_groups < 0 || (d.n_groups > 0 && !d.groups))
            return bad(MPM_ERR_INVALID, "mpm_create: bad group list");
        for (int gi = 0; gi < d.n_groups; ++gi) {
            const mpm_group_desc& g = d.groups[gi];
            const mpm_material_desc& m = g.material;
            if (m.type == MPM_SAND) {
                msg = "mpm_create: SAND is declared by the reference but not implemented";
                return MPM_ERR_UNSUPPORTED;
            }
            if (m.type < MPM_JELLO || m.type > MPM_WATER)
                return bad(MPM_ERR_INVALID, "mpm_create: unknown material type");
            // Elasiticity.cuh:34-41 range checks
            if (m.E < 0.0) return bad(MPM_ERR_INVALID, "mpm_create: Youngs Modulus is out of range");
            if (m.nu < 0.0 || m.nu >= 0.5) return bad(MPM_ERR_INVALID, "mpm_create: Poisson ratio is out of range");
            if (!(g.p_mass > 0.0) || !(g.p_vol > 0.0))
                return bad(MPM_ERR_INVALID, "mpm_create: p_mass and p_vol must be positive");
            if (g.n < 0 || (g.n > 0 && !g.x)) return bad(MPM_ERR_INVALID, "mpm_create: group needs positions");
            if (m.type == MPM_SNOW && (!(m.theta_c >= 0.0) || m.theta_c >= 1.0 || !(m.theta_s >= 0.0)))
                return bad(MPM_ERR_INVALID, "mpm_create: snow clamp thresholds out of range");
            n_particles += g.n;
            ++total_groups;
        }
    }
    if (total_groups > kMaxGroups) return bad(MPM_ERR_INVALID, "mpm_create: too many particle groups");
    if (n_particles > 0x7fffffffLL) return bad(MPM_ERR_INVALID, "mpm_create: too many particles");

    // ---- tables
    scenes_h.resize(n_scenes);
    groups_h.clear();
    scene_begin.assign(n_scenes, 0);
    scene_count.assign(n_scenes, 0);
    long long block_off = 0, p_off = 0;
    constexpr int side3 = 4, side2 = 8;
    const int side = dim == 3 ? side3 : side2;
    for (int s = 0; s < n_scenes; ++s) {
        const mpm_scene_desc& d = scenes[s];
        SceneParams sp{};
        sp.dim = dim;
        for (int a = 0; a < 3; ++a) {
            sp.n[a] = a < dim ? d.n[a] : 1;
            sp.origin[a] = a < dim ? (float)d.origin[a] : 0.f;
            sp.gravity[a] = a < dim ? (float)d.gravity[a] : 0.f;
            sp.nb[a] = a < dim ? (sp.n[a] + side - 1) / side : 1;
        }
        sp.h = (float)d.h;
        sp.inv_h = (float)(1.0 / d.h);
        sp.dt = (float)d.dt;
        sp.bc_type = d.bc_type;
        sp.bc_lo = d.bc_lo;
        sp.bc_hi = d.bc_hi;
        sp.mass_eps = (float)d.mass_eps;
        sp.n_blocks = (long long)sp.nb[0] * sp.nb[1] * sp.nb[2];
        sp.block_off = block_off;
        sp.node_off = block_off * 64;
        sp.n_nodes = sp.n_blocks * 64;
        block_off += sp.n_blocks;
        scenes_h[s] = sp;
        scene_begin[s] = p_off;
        for (int gi = 0; gi < d.n_groups; ++gi) {
            const mpm_group_desc& g = d.groups[gi];
            const mpm_material_desc& m = g.material;
            GroupParams gp{};
            gp.scene = s;
            gp.type = m.type;
            double mu = m.E / (2.0 * (1.0 + m.nu));
            double la = m.E * m.nu / ((1.0 + m.nu) * (1.0 - 2.0 * m.nu));
            gp.mu = (float)mu;
            gp.lambda = (float)la;
            gp.xi = (float)m.xi;
            gp.theta_c = (float)m.theta_c;
            gp.theta_s = (float)m.theta_s;
            gp.bulk_k = (float)m.bulk_k;
            gp.gamma = (float)m.gamma;
            gp.p_mass = (float)g.p_mass;
            gp.p_vol = (float)g.p_vol;
            groups_h.push_back(gp);
            p_off += g.n;
        }
        scene_count[s] = p_off - scene_begin[s];
    }
    total_blocks = block_off;
    current_time = 0.0;
    current_frame = 0;

    // ---- host staging of the particle planes (creation order)
    n_planes = dim == 3 ? Planes<3>::COUNT : Planes<2>::COUNT;
    cap = std::max<long long>(32, (n_particles + 31) / 32 * 32);
    const int D = dim;
    const int PV = D, PC = 2 * D, PF = 2 * D + D * D, PA = 2 * D + 2 * D * D;
    std::vector<float> host((size_t)n_planes * cap, 0.f);
    std::vector<uint16_t> grp_h(cap, 0);
    std::vector<uint32_t> id_h(cap, 0);
    {
        long long i = 0;
        int gidx = 0;
        for (int s = 0; s < n_scenes; ++s) {
            const mpm_scene_desc& d = scenes[s];
            for (int gi = 0; gi < d.n_groups; ++gi, ++gidx) {
                const mpm_group_desc& g = d.groups[gi];
                for (long long k = 0; k < g.n; ++k, ++i) {
                    for (int a = 0; a < D; ++a) {
                        host[(size_t)a * cap + i] = g.x[k * D + a];
                        host[(size_t)(PV + a) * cap + i] = g.v ? g.v[k * D + a] : (float)g.init_v[a];
                    }
                    for (int e = 0; e < D * D; ++e) {
                        host[(size_t)(PC + e) * cap + i] = g.C ? g.C[k * D * D + e] : 0.f;
                        host[(size_t)(PF + e) * cap + i] =
                            g.F ? g.F[k * D * D + e] : ((e % (D + 1) == 0) ? 1.f : 0.f);
                    }
                    host[(size_t)PA * cap + i] = g.aux ? g.aux[k] : 1.f;
                    grp_h[i] = (uint16_t)gidx;
                    id_h[i] = (uint32_t)i;
                }
            }
        }
    }

    // ---- device
    device = opt.device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        msg = std::string("mpm_create: cudaSetDevice: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    auto alloc = [&](void** p, size_t bytes, const char* what) -> int {
        cudaError_t ae = cudaMalloc(p, bytes);
        if (ae != cudaSuccess) {
            msg = std::string("mpm_create: cudaMalloc ") + what + ": " + cudaGetErrorString(ae);
            return ae == cudaErrorMemoryAllocation ? MPM_ERR_NOMEM : MPM_ERR_CUDA;
        }
        return MPM_OK;
    };
    int rc;
    const size_t state_bytes = (size_t)n_planes * cap * sizeof(float);
    if ((rc = alloc((void**)&state, state_bytes, "state")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&state_alt, state_bytes, "state_alt")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&grp, cap * sizeof(uint16_t), "grp")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&grp_alt, cap * sizeof(uint16_t), "grp_alt")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&id, cap * sizeof(uint32_t), "id")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&id_alt, cap * sizeof(uint32_t), "id_alt")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&groups_d, std::max<size_t>(1, groups_h.size()) * sizeof(GroupParams), "groups")) != MPM_OK)
        return rc;
    if ((rc = alloc((void**)&scenes_d, scenes_h.size() * sizeof(SceneParams), "scenes")) != MPM_OK) return rc;
    const size_t grid_bytes = (size_t)total_blocks * 64 * sizeof(float4);
    if ((rc = alloc((void**)&grid_mom, grid_bytes, "grid_mom")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&grid_vel, grid_bytes, "grid_vel")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&err_d, sizeof(unsigned), "err")) != MPM_OK) return rc;
    e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        msg = std::string("mpm_create: stream: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    e = cudaMemcpy(state, host.data(), state_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(grp, grp_h.data(), cap * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(id, id_h.data(), cap * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !groups_h.empty())
        e = cudaMemcpy(groups_d, groups_h.data(), groups_h.size() * sizeof(GroupParams), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(scenes_d, scenes_h.data(), scenes_h.size() * sizeof(SceneParams), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(grid_mom, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(grid_vel, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(err_d, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        msg = std::string("mpm_create: upload: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    graph_dirty = true;
    return MPM_OK;
}

void Engine::release() {
    if (device >= 0) cudaSetDevice(device);
    drop_graph();
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(state);
    cudaFree(state_alt);
    cudaFree(grp);
    cudaFree(grp_alt);
    cudaFree(id);
    cudaFree(id_alt);
    cudaFree(groups_d);
    cudaFree(scenes_d);
    cudaFree(grid_mom);
    cudaFree(grid_vel);
    cudaFree(err_d);
    if (stream) cudaStreamDestroy(stream);
    state = state_alt = nullptr;
    grp = grp_alt = nullptr;
    id = id_alt = nullptr;
    groups_d = nullptr;
    scenes_d = nullptr;
    grid_mom = grid_vel = nullptr;
    err_d = nullptr;
    stream = nullptr;
}

void Engine::drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    graph_dirty = true;
}

void Engine::enqueue_substep() {
    ParticleBuf pb{state, cap, grp, id};
    const int n_scenes = (int)scenes_h.size();
    const long long nodes = total_blocks * 64;
    if (dim == 3) {
        if (n_particles > 0)
            k_p2g_direct<3><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_mom, err_d);
        k_grid_update_dense<3><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                            scenes_d, n_scenes, 1);
        if (n_particles > 0)
            k_g2p_direct<3><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_vel, err_d);
    } else {
        if (n_particles > 0)
            k_p2g_direct<2><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_mom, err_d);
        k_grid_update_dense<2><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                            scenes_d, n_scenes, 1);
        if (n_particles > 0)
            k_g2p_direct<2><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_vel, err_d);
    }
}

int Engine::build_graph() {
    drop_graph();
    cudaGraph_t g = nullptr;
    MPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "graph capture begin");
    enqueue_substep();
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(e, "graph capture end");
    }
    e = cudaGraphInstantiate(&graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        graph_exec = nullptr;
        return cuda_fail(e, "graph instantiate");
    }
    graph_dirty = false;
    return MPM_OK;
}

int Engine::step(int n) {
    if (n < 0) {
        last_error = "mpm_step: negative substep count";
        return MPM_ERR_INVALID;
    }
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    if (opt.use_graph) {
        if (graph_dirty || !graph_exec) {
            int rc = build_graph();
            if (rc != MPM_OK) return rc;
        }
        for (int i = 0; i < n; ++i) MPM_CUDA_TRY(cudaGraphLaunch(graph_exec, stream), "graph launch");
    } else {
        for (int i = 0; i < n; ++i) enqueue_substep();
        MPM_CUDA_TRY(cudaGetLastError(), "kernel launch");
    }
    current_frame += n;
    current_time += (double)n * (scenes_h.empty() ? 0.0 : (double)scenes_h[0].dt);
    return MPM_OK;
}

int Engine::read_errors(uint32_t* bits) {
    unsigned v = 0;
    MPM_CUDA_TRY(cudaMemcpyAsync(&v, err_d, sizeof(unsigned), cudaMemcpyDeviceToHost, stream), "read error word");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    *bits = v;
    return MPM_OK;
}

int Engine::clear_errors() {
    MPM_CUDA_TRY(cudaMemsetAsync(err_d, 0, sizeof(unsigned), stream), "clear error word");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    return MPM_OK;
}

int Engine::sync_and_check() {
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    uint32_t bits = 0;
    int rc = read_errors(&bits);
    if (rc != MPM_OK) return rc;
    if (bits) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "device error word 0x%x (1 out of grid, 2 non-finite, 4 det<=0, 16 timeout)",
                      bits);
        last_error = buf;
        return MPM_ERR_SIM;
    }
    return MPM_OK;
}

int Engine::unpermute_to_alt() {
    if (n_particles == 0) return MPM_OK;
    k_unpermute<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(state, state_alt, id, n_particles, cap, n_planes);
    MPM_CUDA_TRY(cudaGetLastError(), "unpermute launch");
    return MPM_OK;
}

int Engine::get_state(int scene, float* x, float* v, float* C, float* F, float* aux) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    int rc = unpermute_to_alt();
    if (rc != MPM_OK) return rc;
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    const long long b = scene_begin[scene], n = scene_count[scene];
    if (n == 0) return MPM_OK;
    const int D = dim;
    std::vector<float> plane(n);
    auto fetch = [&](int p) -> int {
        MPM_CUDA_TRY(cudaMemcpy(plane.data(), state_alt + (size_t)p * cap + b, n * sizeof(float),
                                cudaMemcpyDeviceToHost),
                     "state download");
        return MPM_OK;
    };
    struct Field {
        float* dst;
        int first, count;
    } fields[5] = {{x, 0, D}, {v, D, D}, {C, 2 * D, D * D}, {F, 2 * D + D * D, D * D}, {aux, 2 * D + 2 * D * D, 1}};
    for (auto& f : fields) {
        if (!f.dst) continue;
        for (int c = 0; c < f.count; ++c) {
            if ((rc = fetch(f.first + c)) != MPM_OK) return rc;
            for (long long i = 0; i < n; ++i) f.dst[i * f.count + c] = plane[i];
        }
    }
    return MPM_OK;
}

int Engine::set_state(int scene, const float* x, const float* v, const float* C, const float* F,
                      const float* aux) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    int rc = unpermute_to_alt();
    if (rc != MPM_OK) return rc;
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    const long long b = scene_begin[scene], n = scene_count[scene];
    if (n == 0) return MPM_OK;
    const int D = dim;
    std::vector<float> plane(n);
    struct Field {
        const float* src;
        int first, count;
    } fields[5] = {{x, 0, D}, {v, D, D}, {C, 2 * D, D * D}, {F, 2 * D + D * D, D * D}, {aux, 2 * D + 2 * D * D, 1}};
    for (auto& f : fields) {
        if (!f.src) continue;
        for (int c = 0; c < f.count; ++c) {
            for (long long i = 0; i < n; ++i) plane[i] = f.src[i * f.count + c];
            MPM_CUDA_TRY(cudaMemcpy(state_alt + (size_t)(f.first + c) * cap + b, plane.data(), n * sizeof(float),
                                    cudaMemcpyHostToDevice),
                         "state upload");
        }
    }
    k_permute_range<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(state_alt, state, id, n_particles, cap,
                                                                       n_planes, b, b + n);
    MPM_CUDA_TRY(cudaGetLastError(), "permute launch");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    return MPM_OK;
}

int Engine::get_grid(int scene, float* mass, float* vel) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    const SceneParams& sc = scenes_h[scene];
    std::vector<float4> blk((size_t)sc.n_nodes);
    MPM_CUDA_TRY(cudaMemcpy(blk.data(), grid_vel + sc.node_off, sc.n_nodes * sizeof(float4), cudaMemcpyDeviceToHost),
                 "grid download");
    const int side = dim == 3 ? 4 : 8;
    const int D = dim;
    for (int iz = 0; iz < sc.n[2]; ++iz)
        for (int iy = 0; iy < sc.n[1]; ++iy)
            for (int ix = 0; ix < sc.n[0]; ++ix) {
                long long b = (ix / side) + (long long)sc.nb[0] * ((iy / side) + (long long)sc.nb[1] * (iz / side));
                int in = (ix % side) + side * ((iy % side) + side * (iz % side));
                const float4 g = blk[(size_t)(b * 64 + in)];
                long long o = (long long)iz * sc.n[0] * sc.n[1] + (long long)iy * sc.n[0] + ix;
                if (mass) mass[o] = g.w;
                if (vel) {
                    vel[o * D + 0] = g.x;
                    vel[o * D + 1] = g.y;
                    if (D == 3) vel[o * D + 2] = g.z;
                }
            }
    return MPM_OK;
}

int Engine::count_active_nodes(int scene, int64_t* n) {
    const SceneParams& sc = scenes_h[scene];
    std::vector<float> mass((size_t)sc.n[0] * sc.n[1] * sc.n[2]);
    int rc = get_grid(scene, mass.data(), nullptr);
    if (rc != MPM_OK) return rc;
    int64_t c = 0;
    for (float m : mass) c += m > 0.f;
    *n = c;
    return MPM_OK;
}

int Engine::set_p2g_mode(int mode) {
    opt.p2g_mode = mode;
    drop_graph();
    return MPM_OK;
}

int Engine::profile_stages(int n, float* out_ms, int n_out, int* n_written) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    ParticleBuf pb{state, cap, grp, id};
    const int n_scenes = (int)scenes_h.size();
    const long long nodes = total_blocks * 64;
    const int n_stages = 3;
    cudaEvent_t ev[n_stages + 1];
    for (auto& e : ev) cudaEventCreate(&e);
    float acc[n_stages] = {0.f, 0.f, 0.f};
    for (int it = 0; it < n; ++it) {
        cudaEventRecord(ev[0], stream);
        if (dim == 3) {
            k_p2g_direct<3><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_mom, err_d);
            cudaEventRecord(ev[1], stream);
            k_grid_update_dense<3><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                                scenes_d, n_scenes, 1);
            cudaEventRecord(ev[2], stream);
            k_g2p_direct<3><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_vel, err_d);
        } else {
            k_p2g_direct<2><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_mom, err_d);
            cudaEventRecord(ev[1], stream);
            k_grid_update_dense<2><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                                scenes_d, n_scenes, 1);
            cudaEventRecord(ev[2], stream);
            k_g2p_direct<2><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                               grid_vel, err_d);
        }
        cudaEventRecord(ev[3], stream);
        cudaEventSynchronize(ev[3]);
        for (int s = 0; s < n_stages; ++s) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[s], ev[s + 1]);
            acc[s] += ms;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    MPM_CUDA_TRY(cudaGetLastError(), "profile launch");
    int w = std::min(n_out, n_stages);
    for (int s = 0; s < w; ++s) out_ms[s] = acc[s] / n;
    if (n_written) *n_written = w;
    current_frame += n;
    current_time += (double)n * (double)scenes_h[0].dt;
    return MPM_OK;
}

}  // namespace mpm
