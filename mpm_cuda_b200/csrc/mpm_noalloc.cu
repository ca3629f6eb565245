// mpm_step_noalloc: the substep for callers that must not allocate device
// memory.
//
// Some callers cannot call cudaMalloc at all: plug-in hosts that hand out a
// fixed device memory budget up front, and real-time loops that forbid
// allocator calls after start-up.  For them this entry point runs whole substeps of one scene
// whose particle state lives in device memory the caller already owns.  The
// only other memory it touches is one fixed scratch area compiled into this
// library: the scene's grid (momentum and velocity) and an error word.
//
// Limits and rules:
//   * the scratch holds at most kScratchNodes = 262,144 grid nodes (64^3 in 3D,
//     512^2 in 2D, counted in whole 64-node blocks); larger grids are rejected
//     with MPM_ERR_INVALID and a message naming both sizes;
//   * the array (8 MiB + 256 B) exists on every GPU that loads the library,
//     for the life of the process;
//   * every call shares it: two calls whose work overlaps on the GPU (two
//     streams, two host threads) race on the grid and give wrong results;
//   * the first call on a device looks up the array's device address with that
//     device current (cudaGetSymbolAddress); make that first call before any
//     stream capture begins.  The address is kept per device ordinal for the
//     life of the process and belongs to the context current at that first call
//     (the device's primary context for runtime-API callers): later calls must
//     run in that context, and a cudaDeviceReset does not refresh it;
//   * each call clears the grid and the error word it uses, so nothing carries
//     over from the previous call except what the caller's state holds.
#include "mpm_b200.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "mpm_grid.cuh"
#include "mpm_particle.cuh"

namespace mpm {

void set_thread_error(const char* msg);

namespace {

constexpr long long kScratchNodes = 1LL << 18;  // 262,144 nodes
constexpr size_t kGridBytes = (size_t)kScratchNodes * sizeof(float4);
constexpr size_t kScratchBytes = 2 * kGridBytes + 256;  // momentum, velocity, error word

// the scratch: grid momentum/mass [0, kGridBytes), grid velocity/mass
// [kGridBytes, 2 kGridBytes), error word at 2 kGridBytes
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// particle i of a caller buffer in the C ABI's plane layout
template <int D>
struct CallerState {
    float* s;
    long long stride;
    __device__ float& at(int plane, long long i) const { return s[plane * stride + i]; }
};

template <int D>
__global__ void __launch_bounds__(128) k_noalloc_p2g(CallerState<D> ps, long long n, SceneParams sc,
                                                     GroupParams g, float4* __restrict__ grid, unsigned* err_word) {
    using P = Planes<D>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[D], v[D], C[D * D], F[D * D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        x[a] = ps.at(P::X + a, i);
        v[a] = ps.at(P::V + a, i);
    }
#pragma unroll
    for (int k = 0; k < D * D; ++k) {
        C[k] = ps.at(P::C + k, i);
        F[k] = ps.at(P::F + k, i);
    }
    const float aux = ps.at(P::AUX, i);
    unsigned err = 0;
    Stencil<D> st;
    if (!make_stencil<D>(x, sc, st, err)) {
        atomicOr(err_word, err);
        return;
    }
    P2GSource<D> src;
    particle_stress_source<D>(v, C, F, aux, g, sc, src);
    p2g_scatter<D>(st, src, sc.h, sc.inv_h, [&](int ox, int oy, int oz, float4 c) {
        atomicAdd(&grid[node_index<D>(sc, st.base[0] + ox, st.base[1] + oy, D == 3 ? st.base[2] + oz : 0)], c);
    });
}

template <int D>
__global__ void __launch_bounds__(256) k_noalloc_grid(const float4* __restrict__ mom, float4* __restrict__ vel,
                                                      long long n_blocks, SceneParams sc) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long b = t >> 6;
    if (b >= n_blocks) return;
    const int in = (int)(t & 63);
    int ix, iy, iz;
    block_node_coords<D>(sc, b, in, ix, iy, iz);
    vel[t] = grid_node_update<D>(mom[t], sc, ix, iy, iz);
}

template <int D>
__global__ void __launch_bounds__(128) k_noalloc_g2p(CallerState<D> ps, long long n, SceneParams sc, GroupParams g,
                                                     const float4* __restrict__ grid, unsigned* err_word) {
    using P = Planes<D>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x[a] = ps.at(P::X + a, i);
    unsigned err = 0;
    Stencil<D> st;
    if (!make_stencil<D>(x, sc, st, err)) {
        atomicOr(err_word, err);
        return;
    }
    G2PAcc<D> acc;
    g2p_gather<D>(st, sc.inv_h, [&](int ox, int oy, int oz) {
        return grid[node_index<D>(sc, st.base[0] + ox, st.base[1] + oy, D == 3 ? st.base[2] + oz : 0)];
    }, acc);
    float F[D * D], aux = ps.at(P::AUX, i);
#pragma unroll
    for (int k = 0; k < D * D; ++k) F[k] = ps.at(P::F + k, i);
    err |= material_update<D>(acc, sc.dt, g, F, aux);
    if (g.type != WATER) {
#pragma unroll
        for (int k = 0; k < D * D; ++k) ps.at(P::F + k, i) = F[k];
    }
    ps.at(P::AUX, i) = aux;
    const float c4 = 4.f * sc.inv_h;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const float xn = fmaf(sc.dt, acc.v[a], x[a]);
        if (!isfinite(xn)) err |= ERR_NONFINITE;
        ps.at(P::X + a, i) = xn;
        ps.at(P::V + a, i) = acc.v[a];
#pragma unroll
        for (int b = 0; b < D; ++b) ps.at(P::C + a * D + b, i) = c4 * acc.B[a * D + b];
    }
    if (err) atomicOr(err_word, err);
}

int fail(int code, const char* msg) {
    set_thread_error(msg);
    return code;
}

// device address of the scratch array on the current device (looked up once)
int scratch_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(MPM_ERR_INVALID, "mpm_step_noalloc: device ordinal too large");
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            char buf[256];
            std::snprintf(buf, sizeof(buf), "mpm_step_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return fail(MPM_ERR_CUDA, buf);
        }
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[dev];
    return MPM_OK;
}

template <int D>
int run(const SceneParams& sc, const GroupParams& g, float* state, long long stride, long long n, int n_substeps,
        cudaStream_t stream, unsigned char* scratch) {
    float4* mom = reinterpret_cast<float4*>(scratch);
    float4* vel = reinterpret_cast<float4*>(scratch + kGridBytes);
    unsigned* err_word = reinterpret_cast<unsigned*>(scratch + 2 * kGridBytes);
    const CallerState<D> ps{state, stride};
    const long long nodes = sc.n_blocks * 64;
    const unsigned pblocks = (unsigned)((n + 127) / 128);
    const unsigned gblocks = (unsigned)((nodes + 255) / 256);
    cudaError_t e = cudaMemsetAsync(err_word, 0, sizeof(unsigned), stream);
    for (int s = 0; s < n_substeps && e == cudaSuccess; ++s) {
        e = cudaMemsetAsync(mom, 0, (size_t)nodes * sizeof(float4), stream);
        if (e != cudaSuccess) break;
        if (n > 0) k_noalloc_p2g<D><<<pblocks, 128, 0, stream>>>(ps, n, sc, g, mom, err_word);
        k_noalloc_grid<D><<<gblocks, 256, 0, stream>>>(mom, vel, sc.n_blocks, sc);
        if (n > 0) k_noalloc_g2p<D><<<pblocks, 128, 0, stream>>>(ps, n, sc, g, vel, err_word);
        e = cudaGetLastError();
    }
    unsigned bits = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, err_word, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "mpm_step_noalloc: %s", cudaGetErrorString(e));
        return fail(MPM_ERR_CUDA, buf);
    }
    if (bits) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "mpm_step_noalloc: device error word 0x%x", bits);
        return fail(MPM_ERR_SIM, buf);
    }
    return MPM_OK;
}

}  // namespace
}  // namespace mpm

extern "C" int mpm_step_noalloc(const mpm_scene_desc* scene, float* state, int64_t plane_stride,
                                int64_t n_particles, int n_substeps, void* stream) {
    using namespace mpm;
    if (!scene) return fail(MPM_ERR_INVALID, "mpm_step_noalloc: scene is NULL");
    const mpm_scene_desc& d = *scene;
    const int dim = d.dim;
    if (dim != 2 && dim != 3) return fail(MPM_ERR_INVALID, "mpm_step_noalloc: dim must be 2 or 3");
    if (d.n_groups != 1 || !d.groups)
        return fail(MPM_ERR_INVALID, "mpm_step_noalloc: the scene must have exactly one particle group");
    if (n_particles < 0 || n_substeps < 0 || (n_particles > 0 && !state) || plane_stride < n_particles)
        return fail(MPM_ERR_INVALID, "mpm_step_noalloc: bad state pointer, particle count or plane stride");
    if (!(d.h > 0.0) || !(d.dt > 0.0)) return fail(MPM_ERR_INVALID, "mpm_step_noalloc: needs h > 0 and dt > 0");
    if (d.bc_type < MPM_BC_STICKY || d.bc_type > MPM_BC_SEPARATE || d.bc_lo < 0 || d.bc_hi < 0 ||
        !(d.ref_band >= 0.0))
        return fail(MPM_ERR_INVALID, "mpm_step_noalloc: bad boundary descriptor");
    const mpm_group_desc& gd = d.groups[0];
    const mpm_material_desc& m = gd.material;
    if (m.type == MPM_SAND) return fail(MPM_ERR_UNSUPPORTED, "mpm_step_noalloc: SAND is not implemented");
    if (m.type < MPM_JELLO || m.type > MPM_WATER) return fail(MPM_ERR_INVALID, "mpm_step_noalloc: unknown material");
    if (m.E < 0.0 || m.nu < 0.0 || m.nu >= 0.5 || !(gd.p_mass > 0.0) || !(gd.p_vol > 0.0))
        return fail(MPM_ERR_INVALID, "mpm_step_noalloc: material or particle mass/volume out of range");

    const int side = dim == 3 ? 4 : 8;
    SceneParams sc{};
    sc.dim = dim;
    for (int a = 0; a < 3; ++a) {
        sc.n[a] = a < dim ? d.n[a] : 1;
        if (a < dim && sc.n[a] < 4) return fail(MPM_ERR_INVALID, "mpm_step_noalloc: fewer than 4 nodes on an axis");
        sc.origin[a] = a < dim ? (float)d.origin[a] : 0.f;
        sc.gravity[a] = a < dim ? (float)d.gravity[a] : 0.f;
        sc.nb[a] = a < dim ? (sc.n[a] + side - 1) / side : 1;
    }
    sc.n_blocks = (long long)sc.nb[0] * sc.nb[1] * sc.nb[2];
    sc.n_nodes = sc.n_blocks * 64;
    if (sc.n_nodes > kScratchNodes) {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "mpm_step_noalloc: the grid needs %lld nodes (whole 64-node blocks) but the static scratch "
                      "holds at most %lld; use mpm_create for larger grids",
                      sc.n_nodes, kScratchNodes);
        return fail(MPM_ERR_INVALID, buf);
    }
    sc.h = (float)d.h;
    sc.inv_h = (float)(1.0 / d.h);
    sc.dt = (float)d.dt;
    sc.bc_type = d.bc_type;
    for (int a = 0; a < 3; ++a) {
        sc.bc_lo[a] = sc.bc_hi[a] = 0;
        if (a < dim) axis_walls(sc.n[a], d.h, d.origin[a], d.ref_band, d.bc_lo, d.bc_hi, sc.bc_lo[a], sc.bc_hi[a]);
    }
    sc.mass_eps = (float)d.mass_eps;
    sc.node_off = 0;
    sc.block_off = 0;

    GroupParams g{};
    g.scene = 0;
    g.type = m.type;
    g.mu = (float)(m.E / (2.0 * (1.0 + m.nu)));
    g.lambda = (float)(m.E * m.nu / ((1.0 + m.nu) * (1.0 - 2.0 * m.nu)));
    g.xi = (float)m.xi;
    g.theta_c = (float)m.theta_c;
    g.theta_s = (float)m.theta_s;
    g.bulk_k = (float)m.bulk_k;
    g.gamma = (float)m.gamma;
    g.p_mass = (float)gd.p_mass;
    g.p_vol = (float)gd.p_vol;

    int dev = 0;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(MPM_ERR_CUDA, "mpm_step_noalloc: cudaGetDevice failed");
    unsigned char* scratch = nullptr;
    const int rc = scratch_address(dev, &scratch);
    if (rc != MPM_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dim == 3 ? run<3>(sc, g, state, plane_stride, n_particles, n_substeps, st, scratch)
                    : run<2>(sc, g, state, plane_stride, n_particles, n_substeps, st, scratch);
}
