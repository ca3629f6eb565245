// Engine implementation: validation, allocation, state I/O and the substep
// launch sequences (binned fused path, unbinned path).
#include "mpm_engine.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "mpm_kernels_binned.cuh"
#include "mpm_kernels_det.cuh"
#include "mpm_kernels_direct.cuh"
#include "mpm_dispatch.cuh"
#include "mpm_surrogate.cuh"

namespace mpm {

namespace {

constexpr int kMaxGroups = 65535;
constexpr int kDefaultRebinInterval = 16;
// device counters: chunk list lengths and cursors per material, active
// block count, grid epoch, tile fallbacks, re-binnings
enum {
    CNT_CHUNKS = 0,
    CNT_ACTIVE = 3,
    CNT_EPOCH = 4,
    CNT_CURSOR = 5,
    CNT_FALLBACK = 8,
    CNT_REBINS = 9,
    CNT_UPDATE_DONE = 10,
    CNT_POOL_FREE = 11,  // paged grid: height of the free stack
    CNT_DET_BLOCKS = 12, // deterministic P2G: length of the ascending list of marked blocks
    CNT_DET_RUNS = 13,   // deterministic P2G: number of runs of records sharing a base node
    CNT_N = 16
};

// out[id[i]] = in[i] for every plane (storage order -> creation order)
__global__ void k_unpermute(const float* __restrict__ in, float* __restrict__ out, const uint32_t* __restrict__ id,
                            long long n, long long cap, int planes) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = id[i];
    for (int p = 0; p < planes; ++p) out[p * cap + j] = in[p * cap + i];
}

// planes, group and creation index of every particle moved to its creation
// index (afterwards id[j] == j)
__global__ void k_canonicalize(const float* __restrict__ in, float* __restrict__ out, const uint16_t* __restrict__ gin,
                               uint16_t* __restrict__ gout, const uint32_t* __restrict__ id, uint32_t* __restrict__ id_out,
                               long long n, long long cap, int planes) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = id[i];
    for (int p = 0; p < planes; ++p) out[p * cap + j] = in[p * cap + i];
    gout[j] = gin[i];
    id_out[j] = (uint32_t)j;
}

// out[i] = in[id[i]] for particles whose creation index lies in [lo, hi)
__global__ void k_permute_range(const float* __restrict__ in, float* __restrict__ out, const uint32_t* __restrict__ id,
                                long long n, long long cap, int planes, long long lo, long long hi) {
    pdl_wait();  // launched early behind the fused pass: wait for its positions
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = id[i];
    if (j < lo || j >= hi) return;
    for (int p = 0; p < planes; ++p) out[p * cap + i] = in[p * cap + j];
}

// positions of creation indices [lo, hi) as interleaved x[(id - lo) * dim + a]
__global__ void k_gather_positions(const float* __restrict__ s, const uint32_t* __restrict__ id, long long n,
                                   long long cap, int dim, long long lo, long long hi, float* __restrict__ out) {
    pdl_wait();  // launched early behind the fused pass: wait for its positions
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = id[i];
    if (j < lo || j >= hi) return;
    for (int a = 0; a < dim; ++a) out[(j - lo) * dim + a] = s[a * cap + i];
}

unsigned grid_blocks(long long n, int threads) { return (unsigned)std::max<long long>(1, (n + threads - 1) / threads); }

// a[i] = value (the page table's "no page")
__global__ void k_fill_int(int* __restrict__ a, long long n, int value) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = value;
}

// the free stack of a fresh pool: every physical block, the lowest on top
__global__ void k_fill_stack(int* __restrict__ s, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) s[i] = (int)(n - 1 - i);
}

}  // namespace

int Engine::cuda_fail(cudaError_t e, const char* what) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    last_error = buf;
    return e == cudaErrorMemoryAllocation ? MPM_ERR_NOMEM : MPM_ERR_CUDA;
}

// records the first failing launch (by name) since the last take_launch_error()
void Engine::note_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess && launch_error.empty()) launch_error = std::string(what) + ": " + cudaGetErrorString(e);
}

// the same for a launch whose status the launch call returned
void Engine::note_launch_status(const char* what, cudaError_t e) {
    if (e != cudaSuccess && launch_error.empty()) launch_error = std::string(what) + ": " + cudaGetErrorString(e);
}

int Engine::take_launch_error() {
    if (launch_error.empty()) return MPM_OK;
    last_error = launch_error;
    launch_error.clear();
    return MPM_ERR_CUDA;
}

#define MPM_CUDA_TRY(expr, what)                           \
    do {                                                   \
        cudaError_t e_ = (expr);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

int Engine::create(const mpm_scene_desc* scenes, int n_scenes, const mpm_options& o, std::string& msg) {
    opt = o;
    if (opt.rebin_interval <= 0) opt.rebin_interval = kDefaultRebinInterval;
    if (opt.p2g_mode < MPM_P2G_ATOMIC || opt.p2g_mode > MPM_P2G_DIRECT) {
        msg = "mpm_create: bad p2g_mode";
        return MPM_ERR_INVALID;
    }
    if (opt.adaptive_dt && opt.p2g_mode != MPM_P2G_ATOMIC) {
        msg = "mpm_create: adaptive dt runs in MPM_P2G_ATOMIC only";
        return MPM_ERR_UNSUPPORTED;
    }
    if (opt.adaptive_dt && !(opt.cfl > 0.f && opt.cfl <= 1.f)) {
        msg = "mpm_create: cfl must be in (0, 1]";
        return MPM_ERR_INVALID;
    }
    if (opt.stress_mode != MPM_STRESS_PLAIN) {
        msg = "mpm_create: select the surrogate stress with mpm_set_stress_mode after creation";
        return MPM_ERR_UNSUPPORTED;
    }
    if (opt.grid_pool_blocks < 0) {
        msg = "mpm_create: grid_pool_blocks must be >= 0";
        return MPM_ERR_INVALID;
    }
    paged = opt.grid_pool_blocks > 0;
    if (paged && opt.p2g_mode != MPM_P2G_ATOMIC) {
        msg = "mpm_create: a paged grid runs in MPM_P2G_ATOMIC only";
        return MPM_ERR_UNSUPPORTED;
    }
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
        if (d.bc_type < MPM_BC_STICKY || d.bc_type > MPM_BC_SEPARATE || d.bc_lo < 0 || d.bc_hi < 0 ||
            !(d.ref_band >= 0.0))
            return bad(MPM_ERR_INVALID, "mpm_create: bad boundary descriptor");
        if (d.n_groups < 0 || (d.n_groups > 0 && !d.groups)) return bad(MPM_ERR_INVALID, "mpm_create: bad group list");
        for (int gi = 0; gi < d.n_groups; ++gi) {
            const mpm_group_desc& g = d.groups[gi];
            const mpm_material_desc& m = g.material;
            if (m.type == MPM_SAND) {
                msg = "mpm_create: SAND is declared by the reference but not implemented";
                return MPM_ERR_UNSUPPORTED;
            }
            if (m.type < MPM_JELLO || m.type > MPM_WATER) return bad(MPM_ERR_INVALID, "mpm_create: unknown material type");
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
    const int side = dim == 3 ? 4 : 8;
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
        for (int a = 0; a < 3; ++a) {
            sp.bc_lo[a] = sp.bc_hi[a] = 0;
            if (a < dim) axis_walls(sp.n[a], d.h, d.origin[a], d.ref_band, d.bc_lo, d.bc_hi, sp.bc_lo[a], sp.bc_hi[a]);
        }
        sp.mass_eps = (float)d.mass_eps;
        sp.n_blocks = (long long)sp.nb[0] * sp.nb[1] * sp.nb[2];
        sp.block_off = block_off;
        sp.node_off = block_off * 64;
        sp.n_nodes = sp.n_blocks * 64;
        if (sp.n_nodes > 0x7fffffffLL) {  // per-scene node offsets are 32-bit in the kernels
            std::snprintf(buf, sizeof(buf), "mpm_create: scene %d has more than 2^31 grid nodes", s);
            return bad(MPM_ERR_INVALID, buf);
        }
        block_off += sp.n_blocks;
        scenes_h[s] = sp;
        scene_begin[s] = p_off;
        double signal = 0.0;
        for (int gi = 0; gi < d.n_groups; ++gi) {
            const mpm_group_desc& g = d.groups[gi];
            const mpm_material_desc& m = g.material;
            GroupParams gp{};
            gp.scene = s;
            gp.type = m.type;
            const double mu = m.E / (2.0 * (1.0 + m.nu));
            const double la = m.E * m.nu / ((1.0 + m.nu) * (1.0 - 2.0 * m.nu));
            gp.mu = (float)mu;
            gp.lambda = (float)la;
            gp.xi = (float)m.xi;
            gp.theta_c = (float)m.theta_c;
            gp.theta_s = (float)m.theta_s;
            gp.bulk_k = (float)m.bulk_k;
            gp.gamma = (float)m.gamma;
            gp.p_mass = (float)g.p_mass;
            gp.p_vol = (float)g.p_vol;
            const double rho = g.p_mass / g.p_vol;
            gp.wave = (float)(m.type == MPM_WATER ? std::sqrt(m.bulk_k * m.gamma / rho) : std::sqrt((la + 2.0 * mu) / rho));
            groups_h.push_back(gp);
            p_off += g.n;
            // fastest initial signal of the scene: wave speed + initial velocity
            double v0 = std::sqrt(g.init_v[0] * g.init_v[0] + g.init_v[1] * g.init_v[1] + g.init_v[2] * g.init_v[2]);
            if (g.v)
                for (int64_t k = 0; k < g.n; ++k) {
                    double vv = 0.0;
                    for (int a = 0; a < dim; ++a) vv += (double)g.v[k * dim + a] * g.v[k * dim + a];
                    v0 = std::max(v0, std::sqrt(vv));
                }
            signal = std::max(signal, gp.wave + v0);
        }
        scene_count[s] = p_off - scene_begin[s];
        // adaptive dt: the scene's dt is the largest; the first substep takes the
        // CFL bound of the initial signal speed
        SceneParams& sq = scenes_h[s];
        sq.adaptive = opt.adaptive_dt ? 1 : 0;
        sq.cfl = opt.cfl;
        sq.dt_max = sq.dt;
        sq.dt_min = sq.dt * 1e-4f;
        if (opt.adaptive_dt && signal > 0.0)
            sq.dt = (float)std::max((double)sq.dt_min, std::min((double)sq.dt_max, opt.cfl * sq.h / signal));
        sq.dt_next = sq.dt;
    }
    if (block_off > 0x7fffffffLL) return bad(MPM_ERR_INVALID, "mpm_create: grids too large");
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
                        host[(size_t)(PF + e) * cap + i] = g.F ? g.F[k * D * D + e] : ((e % (D + 1) == 0) ? 1.f : 0.f);
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
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
    auto alloc = [&](void** p, size_t bytes, const char* what) -> int {
        cudaError_t ae = cudaMalloc(p, std::max<size_t>(bytes, 16));
        if (ae != cudaSuccess) {
            msg = std::string("mpm_create: cudaMalloc ") + what + ": " + cudaGetErrorString(ae);
            return ae == cudaErrorMemoryAllocation ? MPM_ERR_NOMEM : MPM_ERR_CUDA;
        }
        return MPM_OK;
    };
    int rc;
    const size_t state_bytes = (size_t)n_planes * cap * sizeof(float);
    for (int p = 0; p < 2; ++p) {
        if ((rc = alloc((void**)&st[p], state_bytes, "state")) != MPM_OK) return rc;
        if ((rc = alloc((void**)&gp[p], cap * sizeof(uint16_t), "grp")) != MPM_OK) return rc;
        if ((rc = alloc((void**)&ids[p], cap * sizeof(uint32_t), "id")) != MPM_OK) return rc;
    }
    if ((rc = alloc((void**)&groups_d, std::max<size_t>(1, groups_h.size()) * sizeof(GroupParams), "groups")) != MPM_OK)
        return rc;
    if ((rc = alloc((void**)&scenes_d, scenes_h.size() * sizeof(SceneParams), "scenes")) != MPM_OK) return rc;
    // the device scene table never changes in such a run (only adaptive dt
    // writes it), so the fused kernels may carry the scene in their parameters
    fixed_scene = scenes_h.size() == 1 && !opt.adaptive_dt;
    if (paged) {
        pool_cap = std::min<long long>(opt.grid_pool_blocks, total_blocks);
        pages.trash = (int)pool_cap;
        if ((rc = alloc((void**)&pages.page, total_blocks * sizeof(int), "page table")) != MPM_OK) return rc;
        if ((rc = alloc((void**)&pages.slot_block, pool_cap * sizeof(int), "pool map")) != MPM_OK) return rc;
        if ((rc = alloc((void**)&pages.free_slots, pool_cap * sizeof(int), "free blocks")) != MPM_OK) return rc;
    }
    const size_t grid_bytes = (size_t)grid_blocks_alloc() * 64 * sizeof(float4);
    if ((rc = alloc((void**)&grid_mom, grid_bytes, "grid_mom")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&grid_vel, grid_bytes, "grid_vel")) != MPM_OK) return rc;
    // the fixed-scene dense kernels load their windows through vel_map; a
    // driver without tensor maps leaves the run on the table-reading kernels
    if (fixed_scene && !paged && encode_vel_map() != MPM_OK) fixed_scene = false;
    if ((rc = alloc((void**)&err_d, sizeof(unsigned), "err")) != MPM_OK) return rc;
    for (int p = 0; p < 2; ++p) {
        if ((rc = alloc((void**)&keys[p], cap * sizeof(unsigned long long), "sort keys")) != MPM_OK) return rc;
        if ((rc = alloc((void**)&vals[p], cap * sizeof(unsigned), "sort values")) != MPM_OK) return rc;
    }
    for (const GroupParams& g : groups_h) mat_present[g.type] = true;
    mat_slots = MatSlots{};
    for (int m = 0; m < kMats; ++m)
        if (mat_present[m]) mat_slots.s[m] = mat_slots.n++;
    mat_slots.n = std::max(mat_slots.n, 1);
    // the binning's cell counters live at the physical block in a paged grid
    const long long n_cell_counts = grid_blocks_alloc() * 64 * mat_slots.n;
    if ((rc = alloc((void**)&cell_count, n_cell_counts * sizeof(int), "cell counts")) != MPM_OK) return rc;
    // the deterministic path's buffers (it needs a dense grid)
    if ((rc = alloc((void**)&cell_end, paged ? 16 : total_blocks * 64 * sizeof(int), "cell ends")) != MPM_OK)
        return rc;
    {
        const int src_planes = dim == 3 ? SrcPlanes<3>::COUNT : SrcPlanes<2>::COUNT;
        if ((rc = alloc((void**)&det_src, paged ? 16 : (size_t)src_planes * cap * sizeof(float), "source records")) !=
            MPM_OK)
            return rc;
        const int src_stride = dim == 3 ? SrcPlanes<3>::STRIDE : SrcPlanes<2>::STRIDE;
        if ((rc = alloc((void**)&det_sorted, paged ? 16 : (size_t)src_stride * cap * sizeof(float),
                        "sorted source records")) != MPM_OK)
            return rc;
        if ((rc = alloc((void**)&det_blocks, paged ? 16 : total_blocks * sizeof(int), "sorted block list")) != MPM_OK)
            return rc;
        if (deterministic() && (rc = alloc_det_partials()) != MPM_OK) {
            msg = "mpm_create: " + last_error;
            return rc;
        }
    }
    if ((rc = alloc((void**)&seg_count, total_blocks * 4 * sizeof(int), "segment counts")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&seg_start, total_blocks * 4 * sizeof(int), "segment starts")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&blk_flag, total_blocks * sizeof(unsigned), "blk_flag")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&active, total_blocks * sizeof(int), "active")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&blk_epoch, total_blocks * sizeof(int), "blk_epoch")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&counters, CNT_N * sizeof(int), "counters")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&speed_max, scenes_h.size() * sizeof(unsigned), "speed maxima")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&scene_time, scenes_h.size() * sizeof(double), "scene times")) != MPM_OK) return rc;
    // per material: at most n / (particles per chunk) full chunks plus one
    // partial chunk per non-empty block
    list_cap = cap / kMinChunkParticles + std::min<long long>(cap, total_blocks) + 1;
    if ((rc = alloc((void**)&chunks, kMats * list_cap * sizeof(Chunk), "chunks")) != MPM_OK) return rc;
    // bits of the deterministic path's sort keys: node indices and the
    // no-cell key (the node count) are all below 2^det_key_bits
    det_key_bits = 1;
    while (det_key_bits < 64 && (1LL << det_key_bits) <= total_blocks * 64) ++det_key_bits;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp_bytes, keys[0], keys[1], vals[0], vals[1], (int)cap, 0, 64);
    {
        // the deterministic path's ascending list of marked blocks shares the temp space
        size_t sel = 0;
        cub::DeviceSelect::Flagged(nullptr, sel, cub::CountingInputIterator<int>(0), blk_flag, det_blocks,
                                   counters + CNT_DET_BLOCKS, (int)total_blocks);
        sort_tmp_bytes = std::max(sort_tmp_bytes, sel);
        // and the list of runs of sorted records
        cub::DeviceSelect::If(nullptr, sel, cub::CountingInputIterator<int>(0), det_runs, counters + CNT_DET_RUNS,
                              (int)cap, RunStart{keys[1], det_no_cell()});
        sort_tmp_bytes = std::max(sort_tmp_bytes, sel);
    }
    if ((rc = alloc(&sort_tmp, sort_tmp_bytes, "sort temp")) != MPM_OK) return rc;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp_bytes, seg_count, seg_start, (int)(total_blocks * 4));
    if ((rc = alloc(&scan_tmp, scan_tmp_bytes, "scan temp")) != MPM_OK) return rc;
    if ((rc = alloc((void**)&pos_out, cap * D * sizeof(float), "positions")) != MPM_OK) return rc;

    e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        msg = std::string("mpm_create: stream: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    e = cudaMemcpy(st[0], host.data(), state_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(gp[0], grp_h.data(), cap * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ids[0], id_h.data(), cap * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !groups_h.empty())
        e = cudaMemcpy(groups_d, groups_h.data(), groups_h.size() * sizeof(GroupParams), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(scenes_d, scenes_h.data(), scenes_h.size() * sizeof(SceneParams), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(grid_mom, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(grid_vel, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(err_d, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(blk_flag, 0, total_blocks * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(cell_count, 0, n_cell_counts * sizeof(int));
    if (e == cudaSuccess && !paged) e = cudaMemset(cell_end, 0, total_blocks * 64 * sizeof(int));
    if (e == cudaSuccess && paged) {
        k_fill_int<<<grid_blocks(total_blocks, 256), 256>>>(pages.page, total_blocks, pages.trash);
        k_fill_stack<<<grid_blocks(pool_cap, 256), 256>>>(pages.free_slots, pool_cap);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemset(pages.slot_block, 0xff, pool_cap * sizeof(int));
    }
    if (e == cudaSuccess) e = cudaMemset(seg_count, 0, total_blocks * 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(blk_epoch, 0xff, total_blocks * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(counters, 0, CNT_N * sizeof(int));
    if (e == cudaSuccess && paged) {
        const int free0 = (int)pool_cap;
        e = cudaMemcpy(counters + CNT_POOL_FREE, &free0, sizeof(int), cudaMemcpyHostToDevice);
        pages.n_free = counters + CNT_POOL_FREE;
    }
    if (e == cudaSuccess) e = cudaMemset(speed_max, 0, scenes_h.size() * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(scene_time, 0, scenes_h.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        msg = std::string("mpm_create: upload: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    update_ctas = (int)std::max<long long>(1, std::min<long long>((total_blocks + 3) / 4, (long long)num_sms * 8));
    cfg = (opt.kernel_config >= 0 && opt.kernel_config < kNumFusedCfgs) ? opt.kernel_config : 1;
    if (paged && kFusedCfgs[cfg].scatter != SCATTER_DIRECT) {
        msg = "mpm_create: the segmented scatter addresses a dense grid; choose another kernel_config";
        return MPM_ERR_UNSUPPORTED;
    }
    set_config(cfg);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        msg = std::string("mpm_create: pending CUDA error: ") + cudaGetErrorString(e);
        return MPM_ERR_CUDA;
    }
    if (opt.kernel_config < 0 && n_particles > 0) {
        const int cached = cached_config();
        if (cached >= 0) {
            set_config(cached);
        } else {
            const int trc = autotune(8, nullptr);
            if (trc != MPM_OK) {
                msg = "mpm_create: autotune: " + last_error;
                return trc;
            }
        }
    }
    cur = 0;
    grid_dirty = true;
    return MPM_OK;
}

int Engine::chunk_particles() const { return kFusedCfgs[cfg].chunk * kFusedCfgs[cfg].rounds; }

void Engine::set_config(int ci) {
    cfg = ci;
    const int dyn = fused_dyn_smem(dim, kFusedCfgs[ci].kernel);
    for (int mat = 0; mat < kMats; ++mat) {
        int per_sm = 0;
        const FusedFn fn = fused_fn(dim, mat, ci, fixed_scene, paged);
        if (!fn) {  // a configuration the paged grid has no kernel for (rejected before)
            fused_ctas[mat] = num_sms;
            continue;
        }
        // the segmented scatter's staging buffer can exceed the 48 KB a kernel
        // gets without opting in; a failure here shows in the occupancy query
        if (dyn > 0 && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess)
            cudaGetLastError();
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kFusedCfgs[ci].chunk, dyn) != cudaSuccess) {
            cudaGetLastError();  // the query failed: fall back to one CTA per SM
            per_sm = 1;
        }
        fused_ctas[mat] = num_sms * std::max(1, per_sm);
    }
    sur_occupancy();
    drop_graphs();
    grid_dirty = true;  // chunk lists depend on the chunk size
}

// CTA size of the learned-stress kernel: 128 threads when the chunk holds at
// least 128 particles (its shared rows then allow 16 warps per SM; 64-thread
// CTAs measured slower), else 64; it takes ceil(chunk_particles() / that)
// rounds, the last one partly idle when the chunk is not a multiple of it
int Engine::sur_chunk() const { return chunk_particles() >= 128 ? 128 : 64; }

void Engine::sur_occupancy() {
    for (int mat = 0; mat < kMats; ++mat) {
        if (!sur_kernel(mat)) continue;
        const int ch = sur_chunk();
        int per_sm = 0;
        // the network rows live in dynamic shared memory; with the windows and
        // weights they can exceed the 48 KB a kernel gets without opting in
        if (cudaFuncSetAttribute(sur_fn(ch, fixed_scene, paged), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 sur_dyn_smem(ch)) !=
            cudaSuccess)
            cudaGetLastError();  // not fatal here: the occupancy query and the launch report it
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sur_fn(ch, fixed_scene, paged), ch, sur_dyn_smem(ch)) !=
            cudaSuccess) {
            cudaGetLastError();
            per_sm = 1;
        }
        sur_ctas[mat] = num_sms * std::max(1, per_sm);
    }
}

namespace {

// autotuner results of this process, keyed by the workload's shape
struct TuneKey {
    int device, dim, mats;
    long long particles, blocks;
    bool paged;  // a paged grid has its own kernels (and no segmented scatter)
    bool operator<(const TuneKey& o) const {
        if (device != o.device) return device < o.device;
        if (dim != o.dim) return dim < o.dim;
        if (mats != o.mats) return mats < o.mats;
        if (particles != o.particles) return particles < o.particles;
        if (blocks != o.blocks) return blocks < o.blocks;
        return paged < o.paged;
    }
};
std::map<TuneKey, int>& tune_cache() {
    static std::map<TuneKey, int> m;
    return m;
}
std::mutex& tune_mutex() {
    static std::mutex m;
    return m;
}

}  // namespace

// Times `steps` substeps of every fused-kernel configuration on a copy of
// the current state and keeps the fastest; the state, clock and counters are
// restored afterwards, so tuning does not advance the simulation.
int Engine::autotune(int steps, float* best_ms) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    {
        const int rc = recover_vc();  // the backup below must hold real v and C
        if (rc != MPM_OK) return rc;
    }
    if (steps <= 0) steps = 8;
    const size_t state_bytes = (size_t)n_planes * cap * sizeof(float);
    float* bk_state = nullptr;
    uint16_t* bk_grp = nullptr;
    uint32_t* bk_id = nullptr;
    cudaError_t e = cudaMalloc((void**)&bk_state, state_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&bk_grp, cap * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&bk_id, cap * sizeof(uint32_t));
    unsigned err_before = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(&err_before, err_d, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(bk_state, st[cur], state_bytes, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bk_grp, gp[cur], cap * sizeof(uint16_t), cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bk_id, ids[cur], cap * sizeof(uint32_t), cudaMemcpyDeviceToDevice);
    const double t0 = current_time;
    const long long f0 = current_frame;
    // adaptive dt changes the scene table and the scene times: restore them too
    std::vector<SceneParams> bk_scenes(scenes_h.size());
    std::vector<double> bk_time(scenes_h.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(bk_scenes.data(), scenes_d, bk_scenes.size() * sizeof(SceneParams), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(bk_time.data(), scene_time, bk_time.size() * sizeof(double), cudaMemcpyDeviceToHost);
    const int mode0 = opt.p2g_mode;
    opt.p2g_mode = MPM_P2G_ATOMIC;
    int best = cfg;
    float best_t = 1e30f;
    int rc = MPM_OK;
    cudaEvent_t a = nullptr, b = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    // time of n substeps of configuration ci from the saved state (after a
    // warm-up of two that captures its graphs); false on an error (e, rc)
    auto time_cfg = [&](int ci, int n, float& ms) -> bool {
        e = cudaMemcpyAsync(st[cur], bk_state, state_bytes, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(scenes_d, bk_scenes.data(), bk_scenes.size() * sizeof(SceneParams),
                                cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(gp[cur], bk_grp, cap * sizeof(uint16_t), cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ids[cur], bk_id, cap * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return false;
        vc_deferred = false;  // the restored state holds real v and C
        set_config(ci);
        if ((rc = step(2)) != MPM_OK) return false;  // prologue, graph capture, warm-up
        cudaEventRecord(a, stream);
        if ((rc = step(n)) != MPM_OK) return false;
        cudaEventRecord(b, stream);
        e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        return e == cudaSuccess;
    };
    // two passes over the configurations, each keeping its faster time: a
    // single short timing on a shared GPU can pick a configuration that is
    // several per cent slower
    std::vector<float> best_of(kNumFusedCfgs, 1e30f);
    for (int it = 0; it < 2 * kNumFusedCfgs && e == cudaSuccess && rc == MPM_OK; ++it) {
        const int ci = it % kNumFusedCfgs;
        if (paged && kFusedCfgs[ci].scatter != SCATTER_DIRECT) continue;  // the paged grid scatters directly
        float ms = 0.f;
        if (!time_cfg(ci, steps, ms)) break;
        best_of[ci] = std::min(best_of[ci], ms);
    }
    // the three fastest, timed again over four times the substeps (two passes):
    // the leaders are often within a few per cent of each other, closer than a
    // short timing resolves
    std::vector<int> order;
    for (int ci = 0; ci < kNumFusedCfgs; ++ci)
        if (best_of[ci] < 1e30f) order.push_back(ci);
    std::sort(order.begin(), order.end(), [&](int x, int y) { return best_of[x] < best_of[y]; });
    if (order.size() > 3) order.resize(3);
    std::vector<float> long_of(kNumFusedCfgs, 1e30f);
    for (int it = 0; it < 2 * (int)order.size() && e == cudaSuccess && rc == MPM_OK; ++it) {
        const int ci = order[it % order.size()];
        float ms = 0.f;
        if (!time_cfg(ci, 4 * steps, ms)) break;
        long_of[ci] = std::min(long_of[ci], ms / 4.f);
    }
    for (int ci : order)
        if (long_of[ci] < best_t) {
            best_t = long_of[ci];
            best = ci;
        }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    // restore
    cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(st[cur], bk_state, state_bytes, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(gp[cur], bk_grp, cap * sizeof(uint16_t), cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ids[cur], bk_id, cap * sizeof(uint32_t), cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(err_d, &err_before, sizeof(unsigned), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(counters + CNT_FALLBACK, 0, 2 * sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpy(scenes_d, bk_scenes.data(), bk_scenes.size() * sizeof(SceneParams), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(scene_time, bk_time.data(), bk_time.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(speed_max, 0, scenes_h.size() * sizeof(unsigned));
    cudaFree(bk_state);
    cudaFree(bk_grp);
    cudaFree(bk_id);
    vc_deferred = false;
    opt.p2g_mode = mode0;
    current_time = t0;
    current_frame = f0;
    set_config(best);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    if (rc != MPM_OK) return rc;
    if (best_ms) *best_ms = best_t / steps;
    int mats = 0;
    for (int m = 0; m < kMats; ++m) mats |= mat_present[m] ? (1 << m) : 0;
    std::lock_guard<std::mutex> lk(tune_mutex());
    // the cache serves handle creation, which starts on the plain stress: a
    // choice timed with the learned stress is not kept for it
    if (!sur) tune_cache()[TuneKey{device, dim, mats, n_particles, total_blocks, paged}] = best;
    return MPM_OK;
}

int Engine::cached_config() const {
    int mats = 0;
    for (int m = 0; m < kMats; ++m) mats |= mat_present[m] ? (1 << m) : 0;
    std::lock_guard<std::mutex> lk(tune_mutex());
    auto it = tune_cache().find(TuneKey{device, dim, mats, n_particles, total_blocks, paged});
    return it == tune_cache().end() ? -1 : it->second;
}

void Engine::release() {
    if (device >= 0) cudaSetDevice(device);
    drop_graphs();
    if (stream) cudaStreamSynchronize(stream);
    for (int p = 0; p < 2; ++p) {
        cudaFree(st[p]);
        cudaFree(gp[p]);
        cudaFree(ids[p]);
        st[p] = nullptr;
        gp[p] = nullptr;
        ids[p] = nullptr;
    }
    void* ptrs[] = {groups_d, scenes_d, grid_mom, grid_vel, err_d, keys[0], keys[1], vals[0], vals[1],
                    cell_count, seg_count, seg_start, sort_tmp, blk_flag, active, blk_epoch, counters, chunks,
                    scan_tmp, pos_out, cell_end, det_src, det_sorted, det_blocks, det_runs, det_partial,
                    sur_counts, speed_max, scene_time,
                    pages.page, pages.slot_block, pages.free_slots};
    for (void* p : ptrs) cudaFree(p);
    pages = GridPages{};
    groups_d = nullptr;
    scenes_d = nullptr;
    grid_mom = grid_vel = nullptr;
    err_d = nullptr;
    keys[0] = keys[1] = nullptr;
    vals[0] = vals[1] = nullptr;
    cell_count = seg_count = seg_start = cell_end = nullptr;
    det_src = det_sorted = nullptr;
    det_blocks = det_runs = nullptr;
    det_partial = nullptr;
    sort_tmp = nullptr;
    blk_flag = nullptr;
    active = blk_epoch = counters = nullptr;
    chunks = nullptr;
    scan_tmp = nullptr;
    pos_out = nullptr;
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    for (auto& sl : pos_slots) {
        cudaFree(sl.dev);
        if (sl.gathered) cudaEventDestroy(sl.gathered);
        if (sl.copied) cudaEventDestroy(sl.copied);
        sl = PosSlot{};
    }
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
    sur_counts = nullptr;
    speed_max = nullptr;
    scene_time = nullptr;
    sur = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

void Engine::drop_graphs() {
    for (auto& row : graphs)
        for (auto& g : row) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto& g : run_graphs) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// ---------------------------------------------------------- launches --

void Engine::enqueue_direct_substep() {
    const ParticleBuf pb = buf(cur);
    const int n_scenes = (int)scenes_h.size();
    const long long nodes = total_blocks * 64;
    const int bt = opt.block_threads > 0 ? opt.block_threads : 128;
    if (dim == 3) {
        if (n_particles > 0)
            k_p2g_direct<3><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                             grid_mom, err_d);
        k_grid_update_dense<3><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                            scenes_d, n_scenes, 1);
        if (n_particles > 0)
            k_g2p_direct<3><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                             grid_vel, err_d);
    } else {
        if (n_particles > 0)
            k_p2g_direct<2><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                             grid_mom, err_d);
        k_grid_update_dense<2><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                            scenes_d, n_scenes, 1);
        if (n_particles > 0)
            k_g2p_direct<2><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                             grid_vel, err_d);
    }
}

// bins the particles of buffer `from` by (home block, material) into the
// other buffer, in the configuration's order within each segment (counting
// placement, no sort), and builds the chunk lists of the result
void Engine::enqueue_rebin(int from, bool in_loop) {
    // in_loop: a re-binning between two fused passes: the paged grid reclaims
    // blocks, and the v and C planes, which the fused passes never read and the
    // next one rewrites, stay behind
    const bool reclaim = in_loop;
    const int to = 1 - from;
    const long long n_segs = total_blocks * 4;
    int* rank = reinterpret_cast<int*>(vals[0]);
    if (paged && reclaim) {
        // blocks with nothing active near them give their physical block back
        auto k = dim == 3 ? k_pool_reclaim<3> : k_pool_reclaim<2>;
        k<<<grid_blocks(pool_cap, 256), 256, 0, stream>>>(pages, blk_flag, blk_epoch, counters + CNT_EPOCH, scenes_d,
                                                          (int)scenes_h.size());
        note_launch("k_pool_reclaim");
    }
    cudaMemsetAsync(counters + CNT_CHUNKS, 0, kMats * sizeof(int), stream);
    const unsigned nb = grid_blocks(n_particles, 256);
    if (n_particles > 0) {
        // the particles arrive in the order the configuration's last binning gave them
        const bool cm = kFusedCfgs[cfg].order == ORDER_CELL;
        auto k = dim == 3 ? (paged ? (cm ? k_bin_count<3, true, true> : k_bin_count<3, true, false>)
                                   : (cm ? k_bin_count<3, false, true> : k_bin_count<3, false, false>))
                          : (paged ? (cm ? k_bin_count<2, true, true> : k_bin_count<2, true, false>)
                                   : (cm ? k_bin_count<2, false, true> : k_bin_count<2, false, false>));
        k<<<nb, 256, 0, stream>>>(buf(from), n_particles, groups_d, scenes_d, mat_slots, keys[0], rank, cell_count,
                                  seg_count, pages);
        note_launch("k_bin_count");
    }
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_tmp_bytes, seg_count, seg_start, (int)n_segs, stream);
    note_launch("cub::DeviceScan::ExclusiveSum");
    if (n_particles > 0) {
        const bool cm = kFusedCfgs[cfg].order == ORDER_CELL;
        auto k = dim == 3 ? (paged ? (cm ? k_bin_place<3, true, true> : k_bin_place<3, true, false>)
                                   : (cm ? k_bin_place<3, false, true> : k_bin_place<3, false, false>))
                          : (paged ? (cm ? k_bin_place<2, true, true> : k_bin_place<2, true, false>)
                                   : (cm ? k_bin_place<2, false, true> : k_bin_place<2, false, false>));
        k<<<nb, 256, 0, stream>>>(buf(from), buf(to), n_particles, keys[0], rank, cell_count, seg_count, seg_start,
                                  mat_slots, in_loop ? 0 : 1, err_d, pages);
        note_launch("k_bin_place");
    }
    if (dim == 3)
        k_make_chunks<3><<<grid_blocks(n_segs, 256), 256, 0, stream>>>(seg_count, seg_start, n_segs, chunks, list_cap,
                                                                       counters + CNT_CHUNKS, chunk_particles(),
                                                                       scenes_d, (int)scenes_h.size(), err_d);
    else
        k_make_chunks<2><<<grid_blocks(n_segs, 256), 256, 0, stream>>>(seg_count, seg_start, n_segs, chunks, list_cap,
                                                                       counters + CNT_CHUNKS, chunk_particles(),
                                                                       scenes_d, (int)scenes_h.size(), err_d);
    note_launch("k_make_chunks");
    if (n_particles > 0) {
        auto k = paged ? k_bin_reset<true> : k_bin_reset<false>;
        k<<<nb, 256, 0, stream>>>(keys[0], n_particles, mat_slots, cell_count, seg_count, pages);
        note_launch("k_bin_reset");
    }
    k_count_rebin<<<1, 1, 0, stream>>>(counters + CNT_REBINS);
    note_launch("k_count_rebin");
    sorted_order = true;
}

// Tensor map of the single scene's grid velocities in the linear layout:
// float32 (component, x, y[, z]) with strides 16 B, 16 n0 B[, 16 n0 n1 B];
// a box is one chunk window (4 x 8 x 8 x 8, or 4 x 12 x 12 in 2D), zero
// outside the grid.  The encoder comes from the driver through the runtime,
// so the library does not link the driver API.
int Engine::encode_vel_map() {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        cudaGetLastError();
        return MPM_ERR_UNSUPPORTED;
    }
    const SceneParams& sc = scenes_h[0];
    const cuuint32_t rank = dim == 3 ? 4 : 3;
    const cuuint64_t dims[4] = {4, (cuuint64_t)sc.n[0], (cuuint64_t)sc.n[1], (cuuint64_t)sc.n[2]};
    const cuuint64_t strides[3] = {16, 16ull * sc.n[0], 16ull * sc.n[0] * sc.n[1]};
    const cuuint32_t box[4] = {4, (cuuint32_t)TileShape<3>::T, (cuuint32_t)TileShape<3>::T, (cuuint32_t)TileShape<3>::T};
    const cuuint32_t box2[3] = {4, (cuuint32_t)TileShape<2>::T, (cuuint32_t)TileShape<2>::T};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const CUresult r = reinterpret_cast<Encode>(fn)(
        &vel_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, grid_vel + sc.node_off, dims, strides,
        dim == 3 ? box : box2, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MPM_OK : MPM_ERR_UNSUPPORTED;
}

FusedArgs Engine::fused_args(int mat, bool bump) {
    FusedArgs A;
    A.chunks = chunks + mat * list_cap;
    A.n_chunks = counters + CNT_CHUNKS + mat;
    A.cursor = counters + CNT_CURSOR + mat;
    A.groups = groups_d;
    A.scenes = scenes_d;
    A.n_scenes = (int)scenes_h.size();
    A.grid_vel = grid_vel;
    A.grid_mom = grid_mom;
    A.blk_flag = blk_flag;
    A.active = active;
    A.n_active = counters + CNT_ACTIVE;
    A.epoch = counters + CNT_EPOCH;
    A.bump_epoch = bump ? 1 : 0;
    A.err_word = err_d;
    A.fallback = (unsigned*)(counters + CNT_FALLBACK);
    A.speed_max = opt.adaptive_dt ? speed_max : nullptr;
    A.rounds = kFusedCfgs[cfg].rounds;
    A.defer_vc = defer_vc_now() ? 1 : 0;
    A.scene = scenes_h[0];
    // the material's only group, when it has one
    int n_of_mat = 0;
    A.one_group = 0;
    A.group = GroupParams{};
    for (const GroupParams& g : groups_h)
        if (g.type == mat && ++n_of_mat == 1) A.group = g;
    A.one_group = n_of_mat == 1 ? 1 : 0;
    A.pages = pages;
    A.vel_map = vel_map;
    return A;
}

// launch attributes of a kernel that calls pdl_wait before it reads what the
// kernel ahead of it wrote (programmatic dependent launch)
static cudaLaunchConfig_t pdl_config(unsigned grid, unsigned block, size_t smem, cudaStream_t stream,
                                     cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3(grid);
    c.blockDim = dim3(block);
    c.dynamicSmemBytes = smem;
    c.stream = stream;
    attr->id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr->val.programmaticStreamSerializationAllowed = 1;
    c.attrs = attr;
    c.numAttrs = 1;
    return c;
}

void Engine::enqueue_grid_update() {
    const int n_scenes = (int)scenes_h.size();
    // the kernel's last CTA zeroes the active-block count and the chunk
    // cursors, so the fused launches append the next substep's blocks from zero
    cudaLaunchAttribute attr;
    const cudaLaunchConfig_t lc = pdl_config(update_ctas, 256, 0, stream, &attr);
    auto k = paged ? (dim == 3 ? (fixed_scene ? k_grid_update_active<3, true, true> : k_grid_update_active<3, false, true>)
                               : (fixed_scene ? k_grid_update_active<2, true, true> : k_grid_update_active<2, false, true>))
                   : (dim == 3 ? (fixed_scene ? k_grid_update_active<3, true, false> : k_grid_update_active<3, false, false>)
                               : (fixed_scene ? k_grid_update_active<2, true, false>
                                              : k_grid_update_active<2, false, false>));
    const cudaError_t e = cudaLaunchKernelEx(&lc, k, grid_mom, grid_vel, (const int*)active, counters + CNT_ACTIVE,
                                             blk_flag, blk_epoch, (const int*)(counters + CNT_EPOCH),
                                             (const SceneParams*)scenes_d, n_scenes, counters + CNT_CURSOR, (int)kMats,
                                             (unsigned*)(counters + CNT_UPDATE_DONE), scenes_h[0],
                                             vel_linear_mode() ? 1 : 0, pages, err_d);
    note_launch_status("k_grid_update_active", e);
}

void Engine::enqueue_g2p2g(int parity) {
    bool bump = true;
    for (int mat = 0; mat < kMats; ++mat) {
        if (!mat_present[mat]) continue;
        const FusedArgs A = fused_args(mat, bump);
        bump = false;
        if (sur_kernel(mat)) {
            const SurArgs SA{&sur->weights->f, sur->meta, sur_counts};
            const int ch = sur_chunk();
            FusedArgs As = A;
            As.rounds = (chunk_particles() + ch - 1) / ch;
            cudaLaunchAttribute attr;
            const cudaLaunchConfig_t lc = pdl_config(sur_ctas[mat], ch, sur_dyn_smem(ch), stream, &attr);
            const cudaError_t e = cudaLaunchKernelEx(&lc, sur_fn(ch, fixed_scene, paged), buf(parity), As, SA);
            note_launch_status("k_g2p2g_sur", e);
        } else {
            cudaLaunchAttribute attr;
            const cudaLaunchConfig_t lc = pdl_config(fused_ctas[mat], kFusedCfgs[cfg].chunk,
                                                     fused_dyn_smem(dim, kFusedCfgs[cfg].kernel), stream, &attr);
            const cudaError_t e = cudaLaunchKernelEx(&lc, fused_fn(dim, mat, cfg, fixed_scene, paged), buf(parity), A);
            note_launch_status("k_g2p2g", e);
            note_launch("fused_fn");
        }
    }
}

void Engine::enqueue_fused_substep(int parity) {
    enqueue_grid_update();
    enqueue_g2p2g(parity);
    enqueue_adapt_dt();
}

void Engine::enqueue_adapt_dt() {
    if (!opt.adaptive_dt) return;
    const int n_scenes = (int)scenes_h.size();
    k_adapt_dt<<<(n_scenes + 127) / 128, 128, 0, stream>>>(scenes_d, n_scenes, speed_max, scene_time);
    note_launch("k_adapt_dt");
}

// deterministic P2G of the current state into grid_mom (blocks marked active)
void Engine::enqueue_det_p2g() {
    const int n_scenes = (int)scenes_h.size();
    if (n_particles > 0) {
        if (dim == 3)
            k_det_source<3><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(
                buf(cur), n_particles, groups_d, scenes_d, det_src, cap, keys[0], det_no_cell(), vals[0], blk_flag,
                active, counters + CNT_ACTIVE, err_d);
        else
            k_det_source<2><<<grid_blocks(n_particles, 128), 128, 0, stream>>>(
                buf(cur), n_particles, groups_d, scenes_d, det_src, cap, keys[0], det_no_cell(), vals[0], blk_flag,
                active, counters + CNT_ACTIVE, err_d);
        note_launch("k_det_source");
        // keys are node indices below the no-cell key (the node count), which
        // sorts last: the sort needs only the bits that hold the node count
        cub::DeviceRadixSort::SortPairs(sort_tmp, sort_tmp_bytes, keys[0], keys[1], vals[0], vals[1],
                                        (int)n_particles, 0, det_key_bits, stream);
        note_launch("cub::DeviceRadixSort::SortPairs");
        k_det_ranges<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(keys[1], n_particles, det_no_cell(),
                                                                        cell_count, cell_end);
        note_launch("k_det_ranges");
        if (dim == 3)
            k_det_permute<3><<<grid_blocks(n_particles, 256), 256, 0, stream>>>(det_src, (float4*)det_sorted, cap,
                                                                                vals[1], n_particles);
        else
            k_det_permute<2><<<grid_blocks(n_particles, 256), 256, 0, stream>>>(det_src, (float4*)det_sorted, cap,
                                                                                vals[1], n_particles);
        note_launch("k_det_permute");
    }
    if (n_particles > 0) {
        // the runs of records sharing a base node, and their partial sums
        cub::DeviceSelect::If(sort_tmp, sort_tmp_bytes, cub::CountingInputIterator<int>(0), det_runs,
                              counters + CNT_DET_RUNS, (int)n_particles, RunStart{keys[1], det_no_cell()}, stream);
        note_launch("cub::DeviceSelect::If");
        if (dim == 3)
            k_det_partials<3><<<num_sms * 8, 64, 0, stream>>>((const float4*)det_sorted, keys[1], det_runs,
                                                              counters + CNT_DET_RUNS, cell_end, scenes_d, n_scenes,
                                                              det_partial);
        else
            k_det_partials<2><<<num_sms * 8, 64, 0, stream>>>((const float4*)det_sorted, keys[1], det_runs,
                                                              counters + CNT_DET_RUNS, cell_end, scenes_d, n_scenes,
                                                              det_partial);
        note_launch("k_det_partials");
    }
    // the blocks the source records marked, in ascending order
    cub::DeviceSelect::Flagged(sort_tmp, sort_tmp_bytes, cub::CountingInputIterator<int>(0), blk_flag, det_blocks,
                               counters + CNT_DET_BLOCKS, (int)total_blocks, stream);
    note_launch("cub::DeviceSelect::Flagged");
    if (dim == 3)
        k_det_sum<3><<<update_ctas, 256, 0, stream>>>(det_partial, cell_count, cell_end, det_blocks,
                                                      counters + CNT_DET_BLOCKS, scenes_d, n_scenes, grid_mom);
    else
        k_det_sum<2><<<update_ctas, 256, 0, stream>>>(det_partial, cell_count, cell_end, det_blocks,
                                                      counters + CNT_DET_BLOCKS, scenes_d, n_scenes, grid_mom);
    note_launch("k_det_sum");
    if (n_particles > 0) {
        k_det_reset<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(keys[1], n_particles, det_no_cell(),
                                                                       cell_count, cell_end);
        note_launch("k_det_reset");
    }
}

// grid update of the pending P2G, G2P from it, deterministic P2G of the result
void Engine::enqueue_det_substep() {
    enqueue_grid_update();
    const ParticleBuf pb = buf(cur);
    const int bt = opt.block_threads > 0 ? opt.block_threads : 128;
    if (n_particles > 0) {
        if (dim == 3)
            k_g2p_direct<3><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                             grid_vel, err_d);
        else
            k_g2p_direct<2><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                             grid_vel, err_d);
        note_launch("k_g2p_direct");
    }
    // the epoch is bumped once per substep (the fused kernel does it in its path)
    k_count_rebin<<<1, 1, 0, stream>>>(counters + CNT_EPOCH);
    note_launch("epoch");
    enqueue_det_p2g();
}

// moves the particles back to creation order (deterministic mode needs an
// order that does not depend on atomics)
int Engine::canonical_order() {
    if (!sorted_order) return MPM_OK;
    if (n_particles > 0) {
        k_canonicalize<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(st[cur], st[1 - cur], gp[cur], gp[1 - cur],
                                                                          ids[cur], ids[1 - cur], n_particles, cap,
                                                                          n_planes);
        note_launch("k_canonicalize");
        cur = 1 - cur;
    }
    sorted_order = false;
    return take_launch_error();
}

// the fused kernels (plain and learned-stress) defer v and C
bool Engine::defer_vc_now() const { return true; }

// rebuilds the deferred v and C planes (k_recover_vc) before anything reads
// them: the state download and upload, the first P2G of a state, the other
// P2G paths, the autotuner's backup
int Engine::recover_vc() {
    if (!vc_deferred) return MPM_OK;
    if (n_particles > 0) {
        auto k = dim == 3 ? (paged ? k_recover_vc<3, true> : k_recover_vc<3, false>)
                          : (paged ? k_recover_vc<2, true> : k_recover_vc<2, false>);
        k<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(buf(cur), n_particles, groups_d, scenes_d, grid_vel,
                                                             vel_lin_state ? 1 : 0, pages);
        MPM_CUDA_TRY(cudaGetLastError(), "v/C recovery launch");
    }
    vc_deferred = false;
    return MPM_OK;
}

// paged grid: a physical block for every block a particle's stencil covers
void Engine::enqueue_page_in_particles() {
    if (n_particles == 0) return;
    auto k = dim == 3 ? k_page_in_particles<3> : k_page_in_particles<2>;
    k<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(buf(cur), n_particles, groups_d, scenes_d, grid_mom, grid_vel,
                                                         pages, err_d);
    note_launch("k_page_in_particles");
}

// makes grid_mom hold the P2G of the current state (binned path): sorts the
// particles into fresh chunks and scatters them straight to global memory
int Engine::prologue() {
    {
        const int rc = recover_vc();
        if (rc != MPM_OK) return rc;
    }
    const size_t grid_bytes = (size_t)grid_blocks_alloc() * 64 * sizeof(float4);
    MPM_CUDA_TRY(cudaMemsetAsync(grid_mom, 0, grid_bytes, stream), "prologue clear");
    MPM_CUDA_TRY(cudaMemsetAsync(blk_flag, 0, total_blocks * sizeof(unsigned), stream), "prologue flags");
    MPM_CUDA_TRY(cudaMemsetAsync(counters + CNT_ACTIVE, 0, sizeof(int), stream), "prologue counters");
    if (deterministic()) {
        int rc = canonical_order();
        if (rc != MPM_OK) return rc;
        enqueue_det_p2g();
        rc = take_launch_error();
        if (rc != MPM_OK) return rc;
        grid_dirty = false;
        return MPM_OK;
    }
    if (paged) enqueue_page_in_particles();  // the binning counts and the P2G below need the pages
    enqueue_rebin(cur, false);
    cur = 1 - cur;
    steps_since_rebin = 0;
    if (n_particles > 0) {
        auto k = dim == 3 ? (paged ? k_p2g_prologue<3, true> : k_p2g_prologue<3, false>)
                          : (paged ? k_p2g_prologue<2, true> : k_p2g_prologue<2, false>);
        k<<<grid_blocks(n_particles, 128), 128, 0, stream>>>(buf(cur), n_particles, groups_d, scenes_d, grid_mom,
                                                             blk_flag, active, counters + CNT_ACTIVE, err_d, pages);
    }
    note_launch("k_p2g_prologue");
    int lrc = take_launch_error();
    if (lrc != MPM_OK) return lrc;
    grid_dirty = false;
    return MPM_OK;
}

// captures a re-binning and one substep (rebin), or `count` plain substeps
int Engine::build_graph(int parity, int rebin, int count, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    MPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "graph capture begin");
    if (rebin) {
        enqueue_rebin(parity);
        enqueue_fused_substep(1 - parity);
    } else {
        for (int k = 0; k < count; ++k) enqueue_fused_substep(parity);
    }
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        take_launch_error();
        return cuda_fail(e, "graph capture end");
    }
    if (take_launch_error() != MPM_OK) {
        cudaGraphDestroy(g);
        return MPM_ERR_CUDA;
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *out = nullptr;
        return cuda_fail(e, "graph instantiate");
    }
    return MPM_OK;
}

int Engine::step(int n) {
    if (n < 0) {
        last_error = "mpm_step: negative substep count";
        return MPM_ERR_INVALID;
    }
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    sur_refresh();
    if (direct()) {
        if (grid_dirty) {
            MPM_CUDA_TRY(cudaMemsetAsync(grid_mom, 0, (size_t)total_blocks * 64 * sizeof(float4), stream),
                         "grid clear");
            grid_dirty = false;
        }
        if (n > 0) vel_lin_state = false;  // the dense grid update writes the blocked layout
        if (opt.use_graph) {
            if (!graphs[cur][0]) {
                cudaGraph_t g = nullptr;
                MPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture begin");
                enqueue_direct_substep();
                cudaError_t e = cudaStreamEndCapture(stream, &g);
                if (e != cudaSuccess) return cuda_fail(e, "capture end");
                e = cudaGraphInstantiate(&graphs[cur][0], g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
            }
            for (int i = 0; i < n; ++i) MPM_CUDA_TRY(cudaGraphLaunch(graphs[cur][0], stream), "graph launch");
        } else {
            for (int i = 0; i < n; ++i) enqueue_direct_substep();
            MPM_CUDA_TRY(cudaGetLastError(), "kernel launch");
        }
    } else if (deterministic()) {
        if (grid_dirty) {
            int rc = prologue();
            if (rc != MPM_OK) return rc;
        }
        if (n > 0) vel_lin_state = false;  // read back by k_g2p_direct in the blocked layout
        if (opt.use_graph) {
            if (!graphs[cur][0]) {
                cudaGraph_t g = nullptr;
                MPM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture begin");
                enqueue_det_substep();
                cudaError_t e = cudaStreamEndCapture(stream, &g);
                if (e != cudaSuccess) {
                    take_launch_error();
                    return cuda_fail(e, "capture end");
                }
                if (take_launch_error() != MPM_OK) {
                    cudaGraphDestroy(g);
                    return MPM_ERR_CUDA;
                }
                e = cudaGraphInstantiate(&graphs[cur][0], g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
            }
            for (int i = 0; i < n; ++i) MPM_CUDA_TRY(cudaGraphLaunch(graphs[cur][0], stream), "graph launch");
        } else {
            for (int i = 0; i < n; ++i) enqueue_det_substep();
            const int lrc = take_launch_error();
            if (lrc != MPM_OK) return lrc;
        }
    } else {
        if (grid_dirty) {
            int rc = prologue();
            if (rc != MPM_OK) return rc;
        }
        // (after the prologue, whose v/C recovery reads the previous layout)
        if (n > 0) vel_lin_state = vel_linear_mode();
        const int run = opt.rebin_interval - 1;  // plain substeps between two re-binnings
        // set after every launched substep, so an early return below leaves it
        // describing the state the launched substeps produced
        const bool defer = defer_vc_now();
        for (int i = 0; i < n; ++i) {
            const int rebin = steps_since_rebin >= opt.rebin_interval ? 1 : 0;
            if (opt.use_graph && !rebin && run > 1 && steps_since_rebin == 1 && n - i >= run) {
                // the whole stretch up to the next re-binning as one graph
                if (!run_graphs[cur]) {
                    int rc = build_graph(cur, 0, run, &run_graphs[cur]);
                    if (rc != MPM_OK) return rc;
                }
                MPM_CUDA_TRY(cudaGraphLaunch(run_graphs[cur], stream), "graph launch");
                vc_deferred = defer;
                steps_since_rebin += run;
                i += run - 1;
                continue;
            }
            if (opt.use_graph) {
                if (!graphs[cur][rebin]) {
                    int rc = build_graph(cur, rebin, 1, &graphs[cur][rebin]);
                    if (rc != MPM_OK) return rc;
                }
                MPM_CUDA_TRY(cudaGraphLaunch(graphs[cur][rebin], stream), "graph launch");
            } else {
                if (rebin) enqueue_rebin(cur);
                enqueue_fused_substep(rebin ? 1 - cur : cur);
                // kernels of this substep may be queued even if a launch
                // below reports an error
                vc_deferred = defer;
                const int lrc = take_launch_error();
                if (lrc != MPM_OK) return lrc;
                MPM_CUDA_TRY(cudaGetLastError(), "kernel launch");
            }
            vc_deferred = defer;
            if (rebin) {
                cur = 1 - cur;
                steps_since_rebin = 0;
            }
            ++steps_since_rebin;
        }
    }
    if (n > 0 && !fused()) vc_deferred = false;  // the other paths store v and C
    current_frame += n;
    current_time += (double)n * (scenes_h.empty() ? 0.0 : (double)scenes_h[0].dt);
    return MPM_OK;
}

// ----------------------------------------------------------- queries --

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
    if (copy_stream) MPM_CUDA_TRY(cudaStreamSynchronize(copy_stream), "copy stream sync");
    uint32_t bits = 0;
    int rc = read_errors(&bits);
    if (rc != MPM_OK) return rc;
    if (bits) {
        char b[256];
        std::snprintf(b, sizeof(b), "device error word 0x%x (1 out of grid, 2 non-finite, 4 det<=0, 16 timeout)", bits);
        last_error = b;
        return MPM_ERR_SIM;
    }
    return MPM_OK;
}

int Engine::unpermute_to_alt() {
    if (n_particles == 0) return MPM_OK;
    MPM_CUDA_TRY(cudaGetLastError(), "pending error before unpermute");
    k_unpermute<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(st[cur], st[1 - cur], ids[cur], n_particles, cap,
                                                                   n_planes);
    MPM_CUDA_TRY(cudaGetLastError(), "unpermute launch");
    return MPM_OK;
}

int Engine::get_positions(int scene, float* out) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    const long long b = scene_begin[scene], n = scene_count[scene];
    if (n == 0) return MPM_OK;
    k_gather_positions<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(st[cur], ids[cur], n_particles, cap, dim, b,
                                                                          b + n, pos_out);
    MPM_CUDA_TRY(cudaGetLastError(), "gather launch");
    MPM_CUDA_TRY(cudaMemcpyAsync(out, pos_out, (size_t)n * dim * sizeof(float), cudaMemcpyDeviceToHost, stream),
                 "positions download");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    return MPM_OK;
}

// Positions of one scene (creation order) copied to the host without
// blocking: the gather runs on the handle's stream after the substeps enqueued
// so far, the copy on a second stream, so later substeps overlap the copy.
// A ring of kPosSlots staging buffers; a slot is reused only after its
// previous copy finished (a device-side wait of the handle's stream).
int Engine::get_positions_async(int scene, float* out, long long* ticket) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    if (!copy_stream) {  // first use: the stream is created last, so a failed set-up is retried
        for (auto& sl : pos_slots) {
            if (!sl.dev)
                MPM_CUDA_TRY(cudaMalloc((void**)&sl.dev, (size_t)std::max<long long>(cap, 1) * dim * sizeof(float)),
                             "position staging");
            if (!sl.gathered) MPM_CUDA_TRY(cudaEventCreateWithFlags(&sl.gathered, cudaEventDisableTiming), "event");
            if (!sl.copied) MPM_CUDA_TRY(cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming), "event");
        }
        MPM_CUDA_TRY(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "copy stream");
    }
    const long long t = next_ticket++;
    PosSlot& sl = pos_slots[t % kPosSlots];
    if (sl.ticket >= 0) MPM_CUDA_TRY(cudaStreamWaitEvent(stream, sl.copied, 0), "slot reuse wait");
    sl.ticket = t;
    // scene < 0: every scene, concatenated in creation order
    const long long b = scene < 0 ? 0 : scene_begin[scene], n = scene < 0 ? n_particles : scene_count[scene];
    if (n > 0) {
        cudaLaunchAttribute attr;
        const cudaLaunchConfig_t lc = pdl_config(grid_blocks(n_particles, 256), 256, 0, stream, &attr);
        MPM_CUDA_TRY(cudaLaunchKernelEx(&lc, k_gather_positions, (const float*)st[cur], (const uint32_t*)ids[cur],
                                        n_particles, cap, dim, b, b + n, sl.dev),
                     "gather launch");
    }
    MPM_CUDA_TRY(cudaEventRecord(sl.gathered, stream), "event record");
    MPM_CUDA_TRY(cudaStreamWaitEvent(copy_stream, sl.gathered, 0), "copy wait");
    if (n > 0)
        MPM_CUDA_TRY(cudaMemcpyAsync(out, sl.dev, (size_t)n * dim * sizeof(float), cudaMemcpyDeviceToHost, copy_stream),
                     "positions download");
    MPM_CUDA_TRY(cudaEventRecord(sl.copied, copy_stream), "event record");
    if (ticket) *ticket = t;
    return MPM_OK;
}

// Waits until the copy of `ticket` has reached the host.  A slot reused by a
// later ticket is waited for through that later copy, which the handle's
// stream started only after the earlier one had finished.
int Engine::wait_positions(long long ticket) {
    if (ticket < 0 || ticket >= next_ticket) {
        last_error = "mpm_wait_positions: unknown ticket";
        return MPM_ERR_INVALID;
    }
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaEventSynchronize(pos_slots[ticket % kPosSlots].copied), "positions wait");
    return MPM_OK;
}

int Engine::get_state(int scene, float* x, float* v, float* C, float* F, float* aux) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    int rc = recover_vc();
    if (rc != MPM_OK) return rc;
    rc = unpermute_to_alt();
    if (rc != MPM_OK) return rc;
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    const long long b = scene_begin[scene], n = scene_count[scene];
    if (n == 0) return MPM_OK;
    const int D = dim;
    const float* alt = st[1 - cur];
    std::vector<float> plane(n);
    struct Field {
        float* dst;
        int first, count;
    } fields[5] = {{x, 0, D}, {v, D, D}, {C, 2 * D, D * D}, {F, 2 * D + D * D, D * D}, {aux, 2 * D + 2 * D * D, 1}};
    for (auto& f : fields) {
        if (!f.dst) continue;
        for (int c = 0; c < f.count; ++c) {
            MPM_CUDA_TRY(cudaMemcpy(plane.data(), alt + (size_t)(f.first + c) * cap + b, n * sizeof(float),
                                    cudaMemcpyDeviceToHost),
                         "state download");
            for (long long i = 0; i < n; ++i) f.dst[i * f.count + c] = plane[i];
        }
    }
    return MPM_OK;
}

int Engine::set_state(int scene, const float* x, const float* v, const float* C, const float* F, const float* aux) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    int rc = recover_vc();  // the planes this call does not overwrite keep real v and C
    if (rc != MPM_OK) return rc;
    rc = unpermute_to_alt();
    if (rc != MPM_OK) return rc;
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    const long long b = scene_begin[scene], n = scene_count[scene];
    if (n == 0) return MPM_OK;
    const int D = dim;
    float* alt = st[1 - cur];
    std::vector<float> plane(n);
    struct Field {
        const float* src;
        int first, count;
    } fields[5] = {{x, 0, D}, {v, D, D}, {C, 2 * D, D * D}, {F, 2 * D + D * D, D * D}, {aux, 2 * D + 2 * D * D, 1}};
    for (auto& f : fields) {
        if (!f.src) continue;
        for (int c = 0; c < f.count; ++c) {
            for (long long i = 0; i < n; ++i) plane[i] = f.src[i * f.count + c];
            MPM_CUDA_TRY(cudaMemcpy(alt + (size_t)(f.first + c) * cap + b, plane.data(), n * sizeof(float),
                                    cudaMemcpyHostToDevice),
                         "state upload");
        }
    }
    k_permute_range<<<grid_blocks(n_particles, 256), 256, 0, stream>>>(alt, st[cur], ids[cur], n_particles, cap,
                                                                       n_planes, b, b + n);
    MPM_CUDA_TRY(cudaGetLastError(), "permute launch");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    grid_dirty = true;
    return MPM_OK;
}

// the scene's grid velocities in the dense blocked order (a paged block
// without a page reads as zero; a grid in the linear layout is reordered)
int Engine::download_grid(const SceneParams& sc, std::vector<float4>& blk) {
    blk.assign((size_t)sc.n_nodes, make_float4(0.f, 0.f, 0.f, 0.f));
    if (!paged && vel_lin_state) {
        const long long nl = (long long)sc.n[0] * sc.n[1] * (dim == 3 ? sc.n[2] : 1);
        std::vector<float4> lin((size_t)nl);
        MPM_CUDA_TRY(cudaMemcpy(lin.data(), grid_vel + sc.node_off, nl * sizeof(float4), cudaMemcpyDeviceToHost),
                     "grid download");
        const int side = dim == 3 ? 4 : 8, sh = dim == 3 ? 2 : 3;
        for (int iz = 0; iz < (dim == 3 ? sc.n[2] : 1); ++iz)
            for (int iy = 0; iy < sc.n[1]; ++iy)
                for (int ix = 0; ix < sc.n[0]; ++ix) {
                    const long long b = (ix >> sh) + (long long)sc.nb[0] * ((iy >> sh) + (long long)sc.nb[1] * (iz >> sh));
                    const int in = (ix & (side - 1)) + side * ((iy & (side - 1)) + side * (iz & (side - 1)));
                    blk[(size_t)(b * 64 + in)] = lin[(size_t)(ix + (long long)sc.n[0] * (iy + (long long)sc.n[1] * iz))];
                }
        return MPM_OK;
    }
    if (!paged) {
        MPM_CUDA_TRY(cudaMemcpy(blk.data(), grid_vel + sc.node_off, sc.n_nodes * sizeof(float4), cudaMemcpyDeviceToHost),
                     "grid download");
        return MPM_OK;
    }
    std::vector<int> page((size_t)sc.n_blocks);
    std::vector<float4> pool((size_t)pool_cap * 64);
    MPM_CUDA_TRY(cudaMemcpy(page.data(), pages.page + sc.block_off, sc.n_blocks * sizeof(int), cudaMemcpyDeviceToHost),
                 "page table download");
    MPM_CUDA_TRY(cudaMemcpy(pool.data(), grid_vel, pool.size() * sizeof(float4), cudaMemcpyDeviceToHost),
                 "grid pool download");
    for (long long b = 0; b < sc.n_blocks; ++b)
        if (page[b] >= 0 && page[b] < pages.trash)
            std::copy(pool.begin() + (size_t)page[b] * 64, pool.begin() + (size_t)page[b] * 64 + 64,
                      blk.begin() + (size_t)b * 64);
    return MPM_OK;
}

int Engine::get_grid(int scene, float* mass, float* vel) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    const SceneParams& sc = scenes_h[scene];
    std::vector<float4> blk;
    {
        const int rc = download_grid(sc, blk);
        if (rc != MPM_OK) return rc;
    }
    if (!direct()) {
        // blocks not stamped by the last grid update hold stale values
        std::vector<int> ep((size_t)sc.n_blocks);
        int cnt[CNT_N];
        MPM_CUDA_TRY(cudaMemcpy(ep.data(), blk_epoch + sc.block_off, sc.n_blocks * sizeof(int), cudaMemcpyDeviceToHost),
                     "epoch download");
        MPM_CUDA_TRY(cudaMemcpy(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost), "counter download");
        const int last = cnt[CNT_EPOCH] - 1;
        for (long long b = 0; b < sc.n_blocks; ++b)
            if (ep[b] != last)
                for (int k = 0; k < 64; ++k) blk[b * 64 + k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
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

int Engine::grid_pool(int64_t* capacity, int64_t* in_use) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    int n_free = 0;
    if (paged) {
        MPM_CUDA_TRY(cudaMemcpyAsync(&n_free, counters + CNT_POOL_FREE, sizeof(int), cudaMemcpyDeviceToHost, stream),
                     "pool counter download");
        MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    }
    const long long cap_blocks = paged ? pool_cap : total_blocks;
    if (capacity) *capacity = cap_blocks;
    if (in_use) *in_use = cap_blocks - n_free;
    return MPM_OK;
}

int Engine::bin_stats(int64_t* fallbacks, int64_t* rebins) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    int cnt[CNT_N];
    MPM_CUDA_TRY(cudaMemcpy(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost), "counter download");
    if (fallbacks) *fallbacks = (int64_t)(unsigned)cnt[CNT_FALLBACK];
    if (rebins) *rebins = cnt[CNT_REBINS];
    return MPM_OK;
}

// The deterministic path's partial sums (3^D float4 per particle slot) and run
// list, allocated when the path is first chosen
int Engine::alloc_det_partials() {
    if (det_partial) return MPM_OK;
    const int k = dim == 3 ? 27 : 9;
    if (cudaMalloc((void**)&det_partial, (size_t)cap * k * sizeof(float4)) != cudaSuccess ||
        cudaMalloc((void**)&det_runs, (size_t)cap * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(det_partial);
        det_partial = nullptr;
        last_error = "mpm: out of device memory for the deterministic path's partial sums";
        return MPM_ERR_NOMEM;
    }
    return MPM_OK;
}

int Engine::set_p2g_mode(int mode) {
    if (paged && mode != MPM_P2G_ATOMIC) {
        last_error = "mpm_set_p2g_mode: a paged grid runs in MPM_P2G_ATOMIC only";
        return MPM_ERR_UNSUPPORTED;
    }
    if (opt.adaptive_dt && mode != MPM_P2G_ATOMIC) {
        last_error = "mpm_set_p2g_mode: adaptive dt runs in MPM_P2G_ATOMIC only";
        return MPM_ERR_UNSUPPORTED;
    }
    if (sur && mode != MPM_P2G_ATOMIC) {
        last_error = "mpm_set_p2g_mode: the surrogate stress runs in MPM_P2G_ATOMIC only";
        return MPM_ERR_UNSUPPORTED;
    }
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    {
        const int rc = recover_vc();  // the other paths read v and C
        if (rc != MPM_OK) return rc;
    }
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    if (mode == MPM_P2G_DETERMINISTIC) {
        const int rc = alloc_det_partials();
        if (rc != MPM_OK) return rc;
    }
    opt.p2g_mode = mode;
    drop_graphs();
    grid_dirty = true;
    return MPM_OK;
}

int Engine::set_stress_mode(int mode, Surrogate* s) {
    if (mode != MPM_STRESS_PLAIN && mode != MPM_STRESS_SURROGATE) {
        last_error = "mpm_set_stress_mode: bad mode";
        return MPM_ERR_INVALID;
    }
    if (mode == MPM_STRESS_SURROGATE) {
        if (!s) {
            last_error = "mpm_set_stress_mode: MPM_STRESS_SURROGATE needs a surrogate";
            return MPM_ERR_INVALID;
        }
        if (!fused()) {
            last_error = "mpm_set_stress_mode: the surrogate stress runs in MPM_P2G_ATOMIC only";
            return MPM_ERR_UNSUPPORTED;
        }
        if (s->device != device) {
            last_error = "mpm_set_stress_mode: surrogate and handle are on different devices";
            return MPM_ERR_INVALID;
        }
    }
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    if (!sur_counts) MPM_CUDA_TRY(cudaMalloc((void**)&sur_counts, 2 * sizeof(unsigned long long)), "alloc counters");
    MPM_CUDA_TRY(cudaMemset(sur_counts, 0, 2 * sizeof(unsigned long long)), "clear counters");
    sur = mode == MPM_STRESS_SURROGATE ? s : nullptr;
    opt.stress_mode = mode;
    // eligible groups: 3D jello (snow's exact stress reuses its plasticity
    // decomposition, so the network could only cost time there)
    for (auto& g : groups_h) g.surrogate = (sur && dim == 3 && g.type == JELLO) ? 1 : 0;
    MPM_CUDA_TRY(cudaMemcpy(groups_d, groups_h.data(), groups_h.size() * sizeof(GroupParams), cudaMemcpyHostToDevice),
                 "group upload");
    sur_version = sur ? sur->version : -1;
    sur_occupancy();
    drop_graphs();
    return MPM_OK;
}

// captured graphs hold the network's constants by value: re-capture after a
// retraining or set_params
int Engine::sur_refresh() {
    if (sur && sur->version != sur_version) {
        sur_version = sur->version;
        drop_graphs();
    }
    return MPM_OK;
}

// simulated time and current substep of a scene: with adaptive dt the device
// owns the clock (k_adapt_dt), otherwise substeps x dt
int Engine::scene_time_of(int scene, double* t, float* dt) {
    if (!opt.adaptive_dt) {
        if (t) *t = (double)current_frame * scenes_h[scene].dt;
        if (dt) *dt = scenes_h[scene].dt;
        return MPM_OK;
    }
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    if (t) MPM_CUDA_TRY(cudaMemcpy(t, scene_time + scene, sizeof(double), cudaMemcpyDeviceToHost), "time download");
    if (dt) {
        SceneParams sp;
        MPM_CUDA_TRY(cudaMemcpy(&sp, scenes_d + scene, sizeof(sp), cudaMemcpyDeviceToHost), "scene download");
        *dt = sp.dt;
    }
    return MPM_OK;
}

int Engine::stress_stats(int64_t* net, int64_t* fallback) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream), "stream sync");
    unsigned long long c[2] = {0ull, 0ull};
    if (sur_counts) MPM_CUDA_TRY(cudaMemcpy(c, sur_counts, sizeof(c), cudaMemcpyDeviceToHost), "counter download");
    if (net) *net = (int64_t)c[0];
    if (fallback) *fallback = (int64_t)c[1];
    return MPM_OK;
}

int Engine::profile_stages(int n, float* out_ms, int n_out, int* n_written) {
    MPM_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    cudaEvent_t ev[4];
    for (auto& e : ev) cudaEventCreate(&e);
    float acc[3] = {0.f, 0.f, 0.f};
    const int n_scenes = (int)scenes_h.size();
    const long long nodes = total_blocks * 64;
    const int bt = opt.block_threads > 0 ? opt.block_threads : 128;
    if (fused()) {
        if (grid_dirty) {
            int rc = prologue();
            if (rc != MPM_OK) return rc;
        }
        if (n > 0) vel_lin_state = vel_linear_mode();
        // re-binnings at the handle's interval, as in step(); reported per
        // re-binning, the other stages per substep
        int n_rebin = 0;
        for (int it = 0; it < n; ++it) {
            if (it == 0 || steps_since_rebin >= opt.rebin_interval) {
                cudaEventRecord(ev[0], stream);
                enqueue_rebin(cur);
                cudaEventRecord(ev[1], stream);
                cudaEventSynchronize(ev[1]);
                float r = 0.f;
                cudaEventElapsedTime(&r, ev[0], ev[1]);
                acc[0] += r;
                ++n_rebin;
                cur = 1 - cur;
                steps_since_rebin = 0;
            }
            cudaEventRecord(ev[0], stream);
            enqueue_grid_update();
            cudaEventRecord(ev[1], stream);
            enqueue_g2p2g(cur);
            enqueue_adapt_dt();
            cudaEventRecord(ev[2], stream);
            cudaEventSynchronize(ev[2]);
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[0], ev[1]);
            cudaEventElapsedTime(&b, ev[1], ev[2]);
            acc[1] += a;
            acc[2] += b;
            ++steps_since_rebin;
        }
        acc[0] *= (float)n / (float)n_rebin;
    } else if (deterministic()) {
        if (grid_dirty) {
            int rc = prologue();
            if (rc != MPM_OK) return rc;
        }
        if (n > 0) vel_lin_state = false;  // read back by k_g2p_direct in the blocked layout
        const ParticleBuf pb = buf(cur);
        for (int it = 0; it < n; ++it) {
            cudaEventRecord(ev[0], stream);
            enqueue_grid_update();
            cudaEventRecord(ev[1], stream);
            if (dim == 3)
                k_g2p_direct<3><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                                 grid_vel, err_d);
            else
                k_g2p_direct<2><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                                 grid_vel, err_d);
            note_launch("k_g2p_direct");
            k_count_rebin<<<1, 1, 0, stream>>>(counters + CNT_EPOCH);
            cudaEventRecord(ev[2], stream);
            enqueue_det_p2g();
            cudaEventRecord(ev[3], stream);
            cudaEventSynchronize(ev[3]);
            for (int st_i = 0; st_i < 3; ++st_i) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[st_i], ev[st_i + 1]);
                acc[st_i] += ms;
            }
        }
    } else {
        const ParticleBuf pb = buf(cur);
        if (grid_dirty) {
            cudaMemsetAsync(grid_mom, 0, (size_t)total_blocks * 64 * sizeof(float4), stream);
            grid_dirty = false;
        }
        if (n > 0) vel_lin_state = false;  // the dense grid update writes the blocked layout
        for (int it = 0; it < n; ++it) {
            cudaEventRecord(ev[0], stream);
            if (dim == 3) {
                k_p2g_direct<3><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                                 grid_mom, err_d);
                cudaEventRecord(ev[1], stream);
                k_grid_update_dense<3><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                                    scenes_d, n_scenes, 1);
                cudaEventRecord(ev[2], stream);
                k_g2p_direct<3><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                                 grid_vel, err_d);
            } else {
                k_p2g_direct<2><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                                 grid_mom, err_d);
                cudaEventRecord(ev[1], stream);
                k_grid_update_dense<2><<<grid_blocks(nodes, 256), 256, 0, stream>>>(grid_mom, grid_vel, total_blocks,
                                                                                    scenes_d, n_scenes, 1);
                cudaEventRecord(ev[2], stream);
                k_g2p_direct<2><<<grid_blocks(n_particles, bt), bt, 0, stream>>>(pb, n_particles, groups_d, scenes_d,
                                                                                 grid_vel, err_d);
            }
            cudaEventRecord(ev[3], stream);
            cudaEventSynchronize(ev[3]);
            for (int s = 0; s < 3; ++s) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[s], ev[s + 1]);
                acc[s] += ms;
            }
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (n > 0) vc_deferred = fused() && defer_vc_now();
    const int lrc = take_launch_error();
    if (lrc != MPM_OK) return lrc;
    MPM_CUDA_TRY(cudaGetLastError(), "profile launch");
    const int w = std::min(n_out, 3);
    for (int s = 0; s < w; ++s) out_ms[s] = acc[s] / n;
    if (n_written) *n_written = w;
    current_frame += n;
    current_time += (double)n * (double)scenes_h[0].dt;
    return MPM_OK;
}

}  // namespace mpm
