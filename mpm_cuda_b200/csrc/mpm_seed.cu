// Particle seeding on the GPU (mpm_seed), replacing the reference's host loop
// over the grid cells of an object's bounding box with rand() jitter and a
// point-in-mesh test per sample (MPMSimulator.cpp:198-257).
//
// Every cell of the lattice {origin + i h} that the object's world bounding
// box touches gets `ppc` samples at counter-hashed positions inside the cell
// (deterministic for a seed); a sample is kept when it lies inside the object.
// One thread per cell: a count pass that records which samples are kept, an
// exclusive scan, then a write pass that recomputes the kept samples'
// positions, so the output is in cell order (x outermost, then y, z, then the
// sample index), like the reference's loop.
//
// Objects are the unit shapes centred at the origin (cube [-1/2, 1/2]^3, ball
// of radius 1/2, cylinder of radius 1/2 and height 1 along y) or a closed
// triangle mesh, placed by world = translation + scale * (R local) (the model
// matrix translate * scale * rotate of model.cpp:202-207).  The mesh test is
// ray-crossing parity along +z; triangles are binned by their xy bounds so a
// sample only visits the triangles of its bin.  Edges shared by two triangles
// are resolved with a top-left rule so a crossing is counted exactly once.
#include "mpm_b200.h"

#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

namespace mpm {

void set_thread_error(const char* msg);

namespace {

// splitmix64 finaliser (Steele, Lea, Flood 2014) as a counter-based hash
__device__ __forceinline__ unsigned long long seed_mix(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct SeedParams {
    int shape, dim, ppc;
    double R[9], S[3], T[3];  // world = T + S * (R local)
    double h, origin[3];
    int i0[3], ni[3];         // lattice cells [i0, i0 + ni) per axis
    unsigned long long seed;
    // mesh: local vertices, triangles, xy bins (CSR) over [blo, bhi)
    const float* vert;
    const int* tri;
    const int* bin_start;
    const int* bin_tri;
    int nbx, nby;
    double blo[2], bhi[2];
};

// Every floating-point operation that decides which samples are kept is
// rounded explicitly (no multiply-add contraction), so a CPU restatement with
// the same operations reproduces the output bit for bit.
__device__ __forceinline__ double dsub(double a, double b) { return __dadd_rn(a, -b); }
__device__ __forceinline__ double dcross(double a, double b, double c, double d) {
    return dsub(__dmul_rn(a, b), __dmul_rn(c, d));  // a b - c d
}

// 2D edge function with a top-left tie rule: a point on an edge belongs to
// the triangle on one fixed side of it
__device__ __forceinline__ bool edge_in(double ax, double ay, double bx, double by, double px, double py) {
    const double e = dcross(dsub(bx, ax), dsub(py, ay), dsub(by, ay), dsub(px, ax));
    if (e != 0.0) return e > 0.0;
    return (by > ay) || (by == ay && bx < ax);
}

__device__ bool inside_mesh(const SeedParams& P, const double* l) {
    if (!(l[0] >= P.blo[0] && l[0] < P.bhi[0] && l[1] >= P.blo[1] && l[1] < P.bhi[1])) return false;
    const int bx = min(P.nbx - 1, (int)__dmul_rn(__ddiv_rn(dsub(l[0], P.blo[0]), dsub(P.bhi[0], P.blo[0])), P.nbx));
    const int by = min(P.nby - 1, (int)__dmul_rn(__ddiv_rn(dsub(l[1], P.blo[1]), dsub(P.bhi[1], P.blo[1])), P.nby));
    const int b = by * P.nbx + bx;
    int hits = 0;
    for (int k = P.bin_start[b]; k < P.bin_start[b + 1]; ++k) {
        const int t = P.bin_tri[k];
        const float* A = P.vert + 3 * P.tri[3 * t];
        const float* B = P.vert + 3 * P.tri[3 * t + 1];
        const float* Cc = P.vert + 3 * P.tri[3 * t + 2];
        double ax = A[0], ay = A[1], bxx = B[0], byy = B[1], cx = Cc[0], cy = Cc[1];
        double az = A[2], bz = B[2], cz = Cc[2];
        // orient the projected triangle counter-clockwise
        const double area = dcross(dsub(bxx, ax), dsub(cy, ay), dsub(byy, ay), dsub(cx, ax));
        if (area == 0.0) continue;  // seen edge-on by the ray
        if (area < 0.0) {
            double tx = bxx, ty = byy, tz = bz;
            bxx = cx; byy = cy; bz = cz;
            cx = tx; cy = ty; cz = tz;
        }
        if (!edge_in(ax, ay, bxx, byy, l[0], l[1]) || !edge_in(bxx, byy, cx, cy, l[0], l[1]) ||
            !edge_in(cx, cy, ax, ay, l[0], l[1]))
            continue;
        // height of the triangle's plane above the sample
        const double a2 = fabs(area);
        const double wa = __ddiv_rn(dcross(dsub(bxx, l[0]), dsub(cy, l[1]), dsub(byy, l[1]), dsub(cx, l[0])), a2);
        const double wb = __ddiv_rn(dcross(dsub(cx, l[0]), dsub(ay, l[1]), dsub(cy, l[1]), dsub(ax, l[0])), a2);
        const double z = __dadd_rn(__dadd_rn(__dmul_rn(wa, az), __dmul_rn(wb, bz)),
                                   __dmul_rn(dsub(dsub(1.0, wa), wb), cz));
        if (z > l[2]) ++hits;
    }
    return (hits & 1) != 0;
}

// sample k of lattice cell (ix, iy, iz) and whether it lies inside the object
__device__ bool sample(const SeedParams& P, long long cell, int ix, int iy, int iz, int k, float* w) {
    const unsigned long long base = seed_mix(P.seed ^ seed_mix((unsigned long long)cell * 64ull + (unsigned)k));
    const int ic[3] = {ix, iy, iz};
    double q[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < P.dim; ++a) {
        const double u = (double)(seed_mix(base + (unsigned long long)a) >> 11) * (1.0 / 9007199254740992.0);
        // explicitly rounded (no contraction): the same position in every kernel;
        // the float stays inside the cell [lo, hi) when rounding reaches an edge
        const double lo = __dadd_rn(P.origin[a], __dmul_rn((double)ic[a], P.h));
        const double hi = __dadd_rn(P.origin[a], __dmul_rn((double)ic[a] + 1.0, P.h));
        float f = (float)__dadd_rn(P.origin[a], __dmul_rn(__dadd_rn((double)ic[a], u), P.h));
        if ((double)f >= hi) f = nextafterf(f, -INFINITY);
        if ((double)f < lo) f = nextafterf(f, INFINITY);
        w[a] = f;
        q[a] = __ddiv_rn(dsub((double)w[a], P.T[a]), P.S[a]);
    }
    double l[3];
    for (int a = 0; a < 3; ++a)  // R^T q
        l[a] = __dadd_rn(__dadd_rn(__dmul_rn(P.R[a], q[0]), __dmul_rn(P.R[3 + a], q[1])), __dmul_rn(P.R[6 + a], q[2]));
    switch (P.shape) {
        case MPM_SHAPE_CUBE:
            return fabs(l[0]) <= 0.5 && fabs(l[1]) <= 0.5 && (P.dim == 2 || fabs(l[2]) <= 0.5);
        case MPM_SHAPE_SPHERE:
            return __dadd_rn(__dadd_rn(__dmul_rn(l[0], l[0]), __dmul_rn(l[1], l[1])),
                             P.dim == 3 ? __dmul_rn(l[2], l[2]) : 0.0) <= 0.25;
        case MPM_SHAPE_CYLINDER:
            return __dadd_rn(__dmul_rn(l[0], l[0]), __dmul_rn(l[2], l[2])) <= 0.25 && fabs(l[1]) <= 0.5;
        default:
            return inside_mesh(P, l);
    }
}

__device__ __forceinline__ void cell_coords(const SeedParams& P, long long cell, int& ix, int& iy, int& iz) {
    iz = P.i0[2] + (int)(cell % P.ni[2]);
    const long long r = cell / P.ni[2];
    iy = P.i0[1] + (int)(r % P.ni[1]);
    ix = P.i0[0] + (int)(r / P.ni[1]);
}

// count pass: which samples of the cell are kept (bit k), and how many
__global__ void k_seed_count(SeedParams P, long long n_cells, int* __restrict__ counts,
                             unsigned long long* __restrict__ kept) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    int ix, iy, iz;
    cell_coords(P, c, ix, iy, iz);
    unsigned long long mask = 0ull;
    float w[3];
    for (int k = 0; k < P.ppc; ++k)
        if (sample(P, c, ix, iy, iz, k, w)) mask |= 1ull << k;
    kept[c] = mask;
    counts[c] = __popcll(mask);
}

// write pass: the kept samples' positions at the cell's offset (the decision
// comes from the count pass, so a cell writes exactly its count)
__global__ void k_seed_write(SeedParams P, long long n_cells, const int* __restrict__ offsets,
                             const unsigned long long* __restrict__ kept, float* __restrict__ out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    int ix, iy, iz;
    cell_coords(P, c, ix, iy, iz);
    long long o = offsets[c];
    const unsigned long long mask = kept[c];
    float w[3];
    for (int k = 0; k < P.ppc; ++k)
        if ((mask >> k) & 1ull) {
            sample(P, c, ix, iy, iz, k, w);
            for (int a = 0; a < P.dim; ++a) out[o * P.dim + a] = w[a];
            ++o;
        }
}

int seed_fail(int code, const std::string& msg) {
    set_thread_error(msg.c_str());
    return code;
}

}  // namespace
}  // namespace mpm

extern "C" int mpm_seed(const mpm_seed_object* obj, int dim, double h, const double* origin, int ppc, uint64_t seed,
                        int device, float* host_out, size_t cap, int64_t* n_out) {
    using namespace mpm;
    if (!obj || !n_out || !(h > 0.0) || ppc < 1 || ppc > 64 || (dim != 2 && dim != 3))
        return seed_fail(MPM_ERR_INVALID, "mpm_seed: bad argument (h > 0, 1 <= ppc <= 64, dim 2 or 3)");
    if (obj->shape < MPM_SHAPE_CUBE || obj->shape > MPM_SHAPE_MESH)
        return seed_fail(MPM_ERR_INVALID, "mpm_seed: unknown shape");
    if (obj->shape == MPM_SHAPE_MESH && (dim != 3 || !obj->vertices || !obj->triangles || obj->n_vertices <= 0 ||
                                         obj->n_triangles <= 0))
        return seed_fail(MPM_ERR_INVALID, "mpm_seed: a mesh needs dim 3, vertices and triangles");
    for (int a = 0; a < 3; ++a)
        if (!(obj->scale[a] != 0.0)) return seed_fail(MPM_ERR_INVALID, "mpm_seed: zero scale");
    bool finite = std::isfinite(h);
    for (int a = 0; a < 9; ++a) finite = finite && std::isfinite(obj->rotation[a]);
    for (int a = 0; a < 3; ++a)
        finite = finite && std::isfinite(obj->scale[a]) && std::isfinite(obj->translation[a]) &&
                 (!origin || std::isfinite(origin[a]));
    if (!finite) return seed_fail(MPM_ERR_INVALID, "mpm_seed: non-finite placement");
    SeedParams P{};
    P.shape = obj->shape;
    P.dim = dim;
    P.ppc = ppc;
    P.h = h;
    P.seed = seed;
    for (int a = 0; a < 9; ++a) P.R[a] = obj->rotation[a];
    for (int a = 0; a < 3; ++a) {
        P.S[a] = obj->scale[a];
        P.T[a] = obj->translation[a];
        P.origin[a] = origin ? origin[a] : 0.0;
    }
    // local bounds of the object
    double llo[3] = {-0.5, -0.5, -0.5}, lhi[3] = {0.5, 0.5, 0.5};
    std::vector<int> bin_start, bin_tri;
    if (P.shape == MPM_SHAPE_MESH) {
        for (int a = 0; a < 3; ++a) {
            llo[a] = 1e300;
            lhi[a] = -1e300;
        }
        for (int64_t v = 0; v < obj->n_vertices; ++v)
            for (int a = 0; a < 3; ++a) {
                llo[a] = std::min(llo[a], (double)obj->vertices[3 * v + a]);
                lhi[a] = std::max(lhi[a], (double)obj->vertices[3 * v + a]);
            }
        for (int64_t t = 0; t < 3 * obj->n_triangles; ++t)
            if (obj->triangles[t] < 0 || obj->triangles[t] >= obj->n_vertices)
                return seed_fail(MPM_ERR_INVALID, "mpm_seed: triangle index out of range");
        // xy bins over the local bounds (slightly widened), CSR triangle lists
        const int nb = std::max(1, std::min(256, (int)std::sqrt((double)obj->n_triangles)));
        P.nbx = P.nby = nb;
        const double pad = 1e-9 * std::max(1.0, std::max(lhi[0] - llo[0], lhi[1] - llo[1]));
        P.blo[0] = llo[0] - pad;
        P.blo[1] = llo[1] - pad;
        P.bhi[0] = lhi[0] + pad;
        P.bhi[1] = lhi[1] + pad;
        std::vector<std::vector<int>> bins((size_t)nb * nb);
        for (int64_t t = 0; t < obj->n_triangles; ++t) {
            double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
            for (int c = 0; c < 3; ++c) {
                const float* p = obj->vertices + 3 * obj->triangles[3 * t + c];
                x0 = std::min(x0, (double)p[0]);
                x1 = std::max(x1, (double)p[0]);
                y0 = std::min(y0, (double)p[1]);
                y1 = std::max(y1, (double)p[1]);
            }
            auto bin_of = [&](double v, int ax) {
                return std::min(nb - 1, std::max(0, (int)((v - P.blo[ax]) / (P.bhi[ax] - P.blo[ax]) * nb)));
            };
            for (int by = bin_of(y0, 1); by <= bin_of(y1, 1); ++by)
                for (int bx = bin_of(x0, 0); bx <= bin_of(x1, 0); ++bx) bins[(size_t)by * nb + bx].push_back((int)t);
        }
        bin_start.push_back(0);
        for (auto& b : bins) {
            bin_tri.insert(bin_tri.end(), b.begin(), b.end());
            bin_start.push_back((int)bin_tri.size());
        }
    }
    // world bounding box of the transformed local box, then the lattice cells
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; ++c) {
        const double p[3] = {(c & 1) ? lhi[0] : llo[0], (c & 2) ? lhi[1] : llo[1], (c & 4) ? lhi[2] : llo[2]};
        for (int a = 0; a < 3; ++a) {
            const double w = P.T[a] + P.S[a] * (P.R[a * 3] * p[0] + P.R[a * 3 + 1] * p[1] + P.R[a * 3 + 2] * p[2]);
            lo[a] = std::min(lo[a], w);
            hi[a] = std::max(hi[a], w);
        }
    }
    long long n_cells = 1;
    for (int a = 0; a < 3; ++a) {
        if (a >= dim) {
            P.i0[a] = 0;
            P.ni[a] = 1;
            continue;
        }
        const double i0 = std::floor((lo[a] - P.origin[a]) / h), i1 = std::floor((hi[a] - P.origin[a]) / h) + 1.0;
        if (!(i1 - i0 < 1e6)) return seed_fail(MPM_ERR_INVALID, "mpm_seed: object spans too many cells");
        if (!(std::fabs(i0) < 1e9)) return seed_fail(MPM_ERR_INVALID, "mpm_seed: object too far from the origin");
        P.i0[a] = (int)i0;
        P.ni[a] = (int)(i1 - i0);
        n_cells *= P.ni[a];
    }
    if (n_cells > (1LL << 31) / std::max(1, ppc)) return seed_fail(MPM_ERR_INVALID, "mpm_seed: object too large");

    if (cudaSetDevice(device) != cudaSuccess) return seed_fail(MPM_ERR_CUDA, "mpm_seed: cudaSetDevice failed");
    int *counts = nullptr, *offsets = nullptr, *d_bs = nullptr, *d_bt = nullptr, *d_tri = nullptr;
    unsigned long long* kept = nullptr;
    float *d_vert = nullptr, *d_out = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    auto cleanup = [&]() {
        cudaFree(counts); cudaFree(offsets); cudaFree(kept); cudaFree(d_bs); cudaFree(d_bt); cudaFree(d_tri);
        cudaFree(d_vert); cudaFree(d_out); cudaFree(tmp);
    };
    cudaError_t e = cudaMalloc((void**)&counts, (n_cells + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&offsets, (n_cells + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&kept, n_cells * sizeof(unsigned long long));
    if (e == cudaSuccess && P.shape == MPM_SHAPE_MESH) {
        e = cudaMalloc((void**)&d_vert, obj->n_vertices * 3 * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_tri, obj->n_triangles * 3 * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_bs, bin_start.size() * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_bt, std::max<size_t>(1, bin_tri.size()) * sizeof(int));
        if (e == cudaSuccess)
            e = cudaMemcpy(d_vert, obj->vertices, obj->n_vertices * 3 * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_tri, obj->triangles, obj->n_triangles * 3 * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_bs, bin_start.data(), bin_start.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !bin_tri.empty())
            e = cudaMemcpy(d_bt, bin_tri.data(), bin_tri.size() * sizeof(int), cudaMemcpyHostToDevice);
        P.vert = d_vert;
        P.tri = d_tri;
        P.bin_start = d_bs;
        P.bin_tri = d_bt;
    }
    if (e != cudaSuccess) {
        cleanup();
        return seed_fail(MPM_ERR_NOMEM, "mpm_seed: device allocation");
    }
    const unsigned blocks = (unsigned)((n_cells + 255) / 256);
    k_seed_count<<<blocks, 256>>>(P, n_cells, counts, kept);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemset(counts + n_cells, 0, sizeof(int));
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, offsets, (int)(n_cells + 1));
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, offsets, (int)(n_cells + 1));
    int total = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&total, offsets + n_cells, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cleanup();
        return seed_fail(MPM_ERR_CUDA, std::string("mpm_seed: ") + cudaGetErrorString(e));
    }
    *n_out = total;
    if (host_out && total > 0) {
        if (cap < (size_t)total * dim) {
            cleanup();
            return seed_fail(MPM_ERR_INVALID, "mpm_seed: cap smaller than the particle count times dim");
        }
        e = cudaMalloc((void**)&d_out, (size_t)total * dim * sizeof(float));
        if (e == cudaSuccess) {
            k_seed_write<<<blocks, 256>>>(P, n_cells, offsets, kept, d_out);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(host_out, d_out, (size_t)total * dim * sizeof(float), cudaMemcpyDeviceToHost);
    }
    cleanup();
    if (e != cudaSuccess) return seed_fail(MPM_ERR_CUDA, std::string("mpm_seed: ") + cudaGetErrorString(e));
    return MPM_OK;
}
