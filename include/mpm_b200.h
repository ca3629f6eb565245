/*
 * mpm_b200.h -- C ABI of the B200-native explicit MPM substep.
 *
 * This is the drop-in boundary for the substep loop of the reference
 * simulator (JerryYan97/MPM_CUDA).  Each entry point names the reference
 * interface it replaces (path:line within the reference project).  The
 * reference exposes a C++ class; the C++ class with the reference's exact
 * signatures lives in mpm_simulator.hpp and forwards here.
 *
 * Conventions
 *   - Every function returns an int status (MPM_OK = 0, negative on error)
 *     and never calls exit() or throws across the ABI (the reference calls
 *     exit(1) on any CUDA error, e.g. MPMSimulator.cpp:36-39).
 *   - Host arrays are plain float / double pointers with explicit sizes.
 *   - A handle owns all device memory and one CUDA stream.  A handle is not
 *     thread-safe: use one handle per host thread.
 *   - Particle arrays passed across the ABI are per-particle interleaved
 *     (AoS): x[N*dim], v[N*dim], C[N*dim*dim], F[N*dim*dim] (row-major
 *     matrices), aux[N].  aux is det(Fp) for snow, J for water, unused (1)
 *     for jello.
 */
#ifndef MPM_B200_H
#define MPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 1

/* Material types; values match the reference enum MaterialType
 * (src/simulator/material/Elasiticity.cuh:10-11).  SAND is declared there but
 * has no implementation (MPMCUDA.cu:415-416); mpm_create rejects it. */
enum mpm_material_type { MPM_JELLO = 0, MPM_SNOW = 1, MPM_WATER = 2, MPM_SAND = 3 };

/* Wall treatment of the grid update (VelUpdate, MPMCUDA.cu:459-469).
 * A node with index i along an axis is a lower-wall node if i < bc_lo and an
 * upper-wall node if i >= n - bc_hi.  The reference 3D build's walls are a
 * position test instead (MPMCUDA.cu:462-469, band 10 h, :845-850): set
 * mpm_scene_desc.ref_band = 10 with MPM_BC_SLIP to reproduce it exactly. */
enum mpm_boundary_type {
    MPM_BC_STICKY = 0,   /* zero all velocity components of a wall node */
    MPM_BC_SLIP = 1,     /* zero the wall-normal component */
    MPM_BC_SEPARATE = 2  /* zero the wall-normal component only when moving
                            into the wall (MPMJello.py:92-95) */
};

/* P2G reduction modes */
enum mpm_p2g_mode {
    MPM_P2G_ATOMIC = 0,        /* particles binned by grid block; one fused
                                  G2P + stress + P2G kernel per substep that
                                  gathers from a shared-memory window of the
                                  grid velocities and scatters with FP32
                                  vector reductions to global memory (fast;
                                  summation order varies run to run) */
    MPM_P2G_DETERMINISTIC = 1, /* records sorted by base node, summed in a
                                  fixed order (per-run partial sums, then
                                  per-node sums): bitwise identical results
                                  across runs; 27 float4 of partial sums per
                                  particle slot, allocated when first chosen */
    MPM_P2G_DIRECT = 2         /* unbinned: one thread per particle, stencil
                                  straight to global memory (the reference's
                                  kernel structure; for comparison) */
};

/* Stress evaluation modes */
enum mpm_stress_mode {
    MPM_STRESS_PLAIN = 0,     /* 3x3 SVD fixed-corotated stress */
    MPM_STRESS_SURROGATE = 1  /* learned MLP stress with SVD fallback */
};

/* Status codes */
enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_INVALID = -1,     /* bad argument or descriptor */
    MPM_ERR_CUDA = -2,        /* CUDA runtime error (text in mpm_last_error) */
    MPM_ERR_NOMEM = -3,       /* device allocation failed */
    MPM_ERR_UNSUPPORTED = -4, /* valid but not implemented (e.g. SAND) */
    MPM_ERR_SIM = -5,         /* the device error word is non-zero */
    MPM_ERR_IO = -6           /* file output failed */
};

/* Bits of the device error word (replace the reference's device asserts,
 * MPMCUDA.cu:376-386,431,546,614,702,725-739). */
enum mpm_device_error {
    MPM_DEVERR_OUT_OF_GRID = 1, /* a particle's stencil left its grid */
    MPM_DEVERR_NONFINITE = 2,   /* NaN or Inf in particle state */
    MPM_DEVERR_DET = 4,         /* det F <= 0, det Fp <= 0 or J <= 0 */
    MPM_DEVERR_BINNING = 8,     /* internal: particle binning counts disagreed */
    MPM_DEVERR_TIMEOUT = 16,    /* a bounded device-side wait gave up */
    MPM_DEVERR_POOL = 32        /* the paged grid's pool ran out of blocks
                                   (mpm_options.grid_pool_blocks) */
};

typedef struct mpm_material_desc {
    int type;       /* enum mpm_material_type */
    double E, nu;   /* Young's modulus, Poisson ratio -> Lame parameters as
                       Material(E, nu, rho, type), Elasiticity.cuh:30-45 */
    double rho;     /* density (informational; mass comes from p_mass) */
    double xi;      /* snow hardening, mu,lambda *= exp(xi (1 - Jp));
                       reference 10 (MPMCUDA.cu:344) */
    double theta_c; /* snow: sigma clamped to >= 1 - theta_c; reference 8e-2
                       (MPMCUDA.cu:658-660) */
    double theta_s; /* snow: sigma clamped to <= 1 + theta_s; reference 2e-2 */
    double bulk_k;  /* water: p = bulk_k (J^-gamma - 1); reference 2.51
                       (MPMCUDA.cu:353) */
    double gamma;   /* water exponent; reference 7 */
} mpm_material_desc;

/* One particle group (the reference's ParticleGroup, MPMSimulator.cuh:30-52). */
typedef struct mpm_group_desc {
    mpm_material_desc material;
    double p_mass, p_vol;  /* per-particle mass and initial volume */
    int64_t n;             /* number of particles */
    const float *x;        /* [n*dim] positions (required) */
    const float *v;        /* [n*dim] velocities, or NULL -> init_v */
    double init_v[3];
    const float *F;        /* [n*dim*dim] or NULL -> identity */
    const float *C;        /* [n*dim*dim] or NULL -> zero */
    const float *aux;      /* [n] Jp (snow) / J (water), or NULL -> 1 */
} mpm_group_desc;

/* One scene: a grid plus its particle groups (the reference's Grid,
 * MPMSimulator.cuh:54-64, and simulator scalars). */
typedef struct mpm_scene_desc {
    int dim;           /* 2 or 3 */
    int n[3];          /* grid nodes per axis; n[2] = 1 for dim 2 */
    double h;          /* node spacing (the reference's `gap`) */
    double origin[3];  /* grid corner (the reference uses 0) */
    double dt;         /* substep (the reference's adp_dt = max_dt) */
    double gravity[3]; /* the reference adds -9.8 to y (MPMSimulator.cpp:186) */
    int bc_type, bc_lo, bc_hi;
    double mass_eps;   /* nodes with mass <= mass_eps get zero velocity;
                          reference DBL_EPSILON (MPMCUDA.cu:444) */
    int n_groups;
    const mpm_group_desc *groups;
    double ref_band;   /* > 0: the walls are the reference's position test with
                          a band of ref_band cells (MPMCUDA.cu:462-469 with
                          lower = origin + band h, upper = origin + n h - band h,
                          :845-850): node i of an axis is a wall node when
                          origin + i h <= lower or >= upper, evaluated in FP64
                          with the reference's own operations, so a node the
                          reference's rounding puts outside the band (e.g.
                          n - 10 for n = 48, h = 1/48) is outside here too;
                          bc_lo / bc_hi are then ignored.  0: bc_lo / bc_hi. */
} mpm_scene_desc;

typedef struct mpm_options {
    int p2g_mode;       /* enum mpm_p2g_mode */
    int stress_mode;    /* enum mpm_stress_mode */
    int use_graph;      /* capture the substep in a CUDA graph (default 1) */
    int block_threads;  /* threads per CTA for the unbinned kernels; 0 = tuned */
    int device;         /* CUDA device ordinal */
    int rebin_interval; /* substeps between re-binnings of the particles
                           (MPM_P2G_ATOMIC); 0 = tuned default */
    int kernel_config;  /* fused-kernel launch configuration (threads per
                           CTA, CTAs per SM, particles per thread; see
                           mpm_kernel_config_info); -1 = choose with the
                           autotuner at creation */
    int adaptive_dt;    /* MPM_P2G_ATOMIC only: each scene's dt becomes its
                           largest; every substep picks the next from the CFL
                           bound cfl * h / max(|v| + material wave speed), on
                           the device inside the substep graph (the reference
                           computes a dt factor it never applies,
                           MPMCUDA.cu:915-920).  Default 0 (fixed dt). */
    float cfl;          /* CFL number of adaptive dt, (0, 1]; default 0.5 */
    int grid_pool_blocks; /* MPM_P2G_ATOMIC only.  0 (default): each scene's grid
                           is allocated densely (the reference allocates its
                           grid densely, MPMSimulator.cpp:122-146).  > 0: the
                           grid is paged: one pool of this many 64-node blocks
                           (at most the scenes' block count) shared by all
                           scenes, pages
                           assigned on the device to the blocks particles
                           touch and their neighbours and returned when nothing
                           is active near them; a step that needs more blocks
                           than the pool holds sets MPM_DEVERR_POOL.  Each
                           pool block costs 2 KB of grid (momentum and
                           velocity) plus 256 B per material of binning
                           counters. */
} mpm_options;

typedef struct mpm_handle mpm_handle;

/* Fills *opt with defaults (ATOMIC, PLAIN, graphs on, tuned sizes, device 0). */
void mpm_default_options(mpm_options *opt);

/* Replaces MPMSimulator::MPMSimulator(gap, dt, nx, ny, nz, ppc, objs)
 * (src/simulator/MPMSimulator.cuh:92-96, MPMSimulator.cpp:178-285): builds
 * n_scenes independent scenes on one device.  opt may be NULL.  A scene's
 * grid (rounded up to whole blocks) holds fewer than 2^31 nodes. */
int mpm_create(const mpm_scene_desc *scenes, int n_scenes, const mpm_options *opt,
               mpm_handle **out);

/* Replaces ~MPMSimulator() (MPMSimulator.cuh:101, MPMSimulator.cpp:288-352). */
int mpm_destroy(mpm_handle *h);

/* Replaces MPMSimulator::step() (MPMSimulator.cuh:98, MPMCUDA.cu:793-925):
 * advances every scene by n_substeps and waits for completion; returns
 * MPM_ERR_SIM if the device error word became non-zero. */
int mpm_step(mpm_handle *h, int n_substeps);

/* Same as mpm_step but returns right after enqueueing on the handle's
 * stream; call mpm_synchronize to wait and collect the error word. */
int mpm_step_async(mpm_handle *h, int n_substeps);
int mpm_synchronize(mpm_handle *h);

/* Device error word (enum mpm_device_error bits), read after a sync. */
int mpm_get_device_errors(mpm_handle *h, uint32_t *bits);
int mpm_clear_device_errors(mpm_handle *h);

/* The handle's CUDA stream (a cudaStream_t) for event timing. */
int mpm_get_stream(mpm_handle *h, void **stream);

/* Replaces MPMSimulator::totalParticlesNum() (MPMSimulator.cuh:99):
 * scene < 0 counts every scene. */
int mpm_num_particles(mpm_handle *h, int scene, int64_t *n);

/* Replaces MPMSimulator::getGLParticlesPos(std::vector<float>&)
 * (MPMSimulator.cuh:100, MPMSimulator.cpp:362-371): copies a scene's
 * positions, in creation order, as float x[N*dim].  cap is in floats. */
int mpm_get_positions(mpm_handle *h, int scene, float *host_out, size_t cap);

/* Same as mpm_get_positions without blocking: the positions after every
 * substep enqueued so far are gathered on the handle's stream and copied to
 * host_out on a second stream, so that substeps enqueued next run while the
 * copy crosses to the host (the reference copies positions to host memory
 * synchronously in every step(), MPMCUDA.cu:905-909, and reads them each
 * loop iteration, main.cpp:206-210).  host_out should be
 * page-locked for the copy to overlap, and must not be read or freed before
 * mpm_wait_positions(h, *ticket) (or mpm_synchronize) returns.  Up to three
 * copies can be in flight; a fourth waits, on the device, for the oldest.
 * scene < 0 copies every scene's positions, concatenated in scene order. */
int mpm_get_positions_async(mpm_handle *h, int scene, float *host_out, size_t cap,
                            int64_t *ticket);
int mpm_wait_positions(mpm_handle *h, int64_t ticket);

/* Full particle state of one scene in creation order (the reference's device
 * arrays, MPMSimulator.cuh:37-43).  Any pointer may be NULL to skip it. */
int mpm_get_state(mpm_handle *h, int scene, float *x, float *v, float *C, float *F,
                  float *aux);
int mpm_set_state(mpm_handle *h, int scene, const float *x, const float *v,
                  const float *C, const float *F, const float *aux);

/* Grid of one scene after the last grid update: mass[G] and velocity
 * vel[G*dim], x-fastest node order as MPMCUDA.cu:375.  Either may be NULL. */
int mpm_get_grid(mpm_handle *h, int scene, float *mass, float *vel);

/* Simulated time and substep count of a scene (the reference's public
 * current_time / current_frame, MPMSimulator.cuh:86-87). */
int mpm_get_time(mpm_handle *h, double *current_time, int64_t *current_frame);

/* Simulated time and current dt of one scene.  With adaptive dt each scene
 * has its own clock, kept on the device (this call waits for the stream);
 * mpm_get_time then reports scene 0's. */
int mpm_get_scene_time(mpm_handle *h, int scene, double *time, float *dt);

/* ------------------------------------------------------------------------
 * Particle seeding on the GPU.  Replaces the reference's host loop
 * (MPMSimulator.cpp:198-257): every cell of the lattice origin + i h that the
 * object's world bounding box touches gets ppc samples at hashed positions
 * inside the cell (deterministic for a seed; the reference uses rand()), and
 * the samples inside the object are kept, in cell order.  Objects are unit
 * shapes centred at the origin, or a closed triangle mesh (inside test by
 * ray-crossing parity), placed by world = translation + scale * (R local)
 * (the reference's model matrix translate * scale * rotate, model.cpp:202-207).
 * ---------------------------------------------------------------------- */
enum mpm_shape {
    MPM_SHAPE_CUBE = 0,     /* [-1/2, 1/2]^3 */
    MPM_SHAPE_SPHERE = 1,   /* ball of radius 1/2 */
    MPM_SHAPE_CYLINDER = 2, /* radius 1/2, height 1 along y */
    MPM_SHAPE_MESH = 3      /* vertices / triangles below (3D only) */
};

typedef struct mpm_seed_object {
    int shape;              /* enum mpm_shape */
    double rotation[9];     /* R, row-major */
    double scale[3];
    double translation[3];
    const float *vertices;  /* MPM_SHAPE_MESH: n_vertices x 3, local coordinates */
    int64_t n_vertices;
    const int32_t *triangles; /* n_triangles x 3 vertex indices */
    int64_t n_triangles;
} mpm_seed_object;

/* Seeds one object with ppc (1..64) samples per lattice cell of spacing h
 * anchored at origin (NULL = 0) in dim 2 or 3.  *n receives the particle
 * count; with host_out (cap floats, >= n * dim) the positions are written
 * too, so a first call with host_out = NULL sizes the buffer. */
int mpm_seed(const mpm_seed_object *obj, int dim, double h, const double *origin, int ppc,
             uint64_t seed, int device, float *host_out, size_t cap, int64_t *n);

/* Replaces OutputBego(path, positions) (src/utilities/FilesIO.h:10,
 * FilesIO.cpp:6-24): writes the scene's positions as a Houdini .bgeo
 * particle file with one float[3] "position" attribute. */
int mpm_write_bgeo(mpm_handle *h, int scene, const char *path);

/* Writes host positions (x[n*3]) as .bgeo without a handle. */
int mpm_write_bgeo_positions(const char *path, const float *x, int64_t n);

/* Switches the P2G reduction mode (enum mpm_p2g_mode) of a live handle. */
int mpm_set_p2g_mode(mpm_handle *h, int mode);

/* Last error message of the handle (or of the thread when h is NULL). */
int mpm_last_error(mpm_handle *h, char *buf, size_t cap);

/* Per-stage device time of one substep, measured with CUDA events on the
 * handle's stream and averaged over n_substeps (the handle advances by
 * n_substeps).  out_ms[0..n_out) in stage order:
 *   MPM_P2G_ATOMIC:  rebin (time of one re-binning; they run every
 *                    rebin_interval substeps as in mpm_step), grid_update, g2p2g
 *   MPM_P2G_DIRECT:  p2g, grid_update, g2p
 *   MPM_P2G_DETERMINISTIC: grid_update, g2p, p2g (source records, sort,
 *                    partial sums, node sums)
 * *n_written receives the number of stages written. */
int mpm_profile_stages(mpm_handle *h, int n_substeps, float *out_ms, int n_out,
                       int *n_written);

/* Number of grid nodes with non-zero mass in one scene after the last step. */
int mpm_count_active_nodes(mpm_handle *h, int scene, int64_t *n);

/* Launch configurations of the fused substep kernel (the autotuner's search
 * space): configuration i runs *chunk threads per CTA, at least *min_ctas CTAs
 * per SM, and chunks of *chunk x *rounds particles (each thread processes
 * *rounds particles of a chunk in turn).  Any output pointer may be NULL.  No
 * reference counterpart: the reference launches fixed 128-thread blocks
 * (MPMCUDA.cu:813-815). */
int mpm_num_kernel_configs(void);
int mpm_kernel_config_info(int config, int *chunk, int *min_ctas, int *rounds);
/* How a configuration orders and scatters the particles: *cell_major = 1 when
 * the re-binning puts a cell's particles together (else rank-major: a warp's
 * lanes in distinct cells); *segmented = 1 when the lanes of a warp that share
 * a stencil base are summed in shared memory before one reduction per node
 * (else every particle reduces its own 3^D node values).  The reference
 * scatters every particle's values with FP64 atomics (MPMCUDA.cu:388-421). */
int mpm_kernel_config_scatter(int config, int *cell_major, int *segmented);
int mpm_get_kernel_config(mpm_handle *h, int *config);
int mpm_set_kernel_config(mpm_handle *h, int config);

/* Times n_substeps of every configuration on a copy of the state (the
 * simulation does not advance), keeps the fastest and caches it for handles
 * of the same shape in this process.  *chosen / *ms_per_substep may be NULL. */
int mpm_autotune(mpm_handle *h, int n_substeps, int *chosen, float *ms_per_substep);

/* Diagnostics of the binned path: *fallbacks counts particle gathers or
 * scatters that left their block's shared-memory tile (served from global
 * memory) since creation; *rebins counts re-binnings. */
int mpm_get_bin_stats(mpm_handle *h, int64_t *fallbacks, int64_t *rebins);

/* Paged grid (mpm_options.grid_pool_blocks > 0): *capacity = the pool's
 * 64-node blocks, *in_use = the blocks holding a page after the substeps
 * enqueued so far (waits for the stream).  A dense grid reports its block
 * count for both.  The reference allocates its grid densely
 * (MPMSimulator.cpp:122-146) and has no counterpart. */
int mpm_get_grid_pool(mpm_handle *h, int64_t *capacity, int64_t *in_use);

/* Substeps without any device allocation, for callers that cannot allocate:
 * plug-in hosts with a fixed device memory budget, loops that forbid
 * allocator calls after start-up.  No counterpart in the reference (its step() uses grids that its
 * constructor allocated).
 * Runs n_substeps of ONE scene with exactly one particle group (material,
 * p_mass, p_vol from scene->groups[0]; its particle pointers are ignored)
 * on the caller's stream.  `state` is caller-owned device memory in the
 * handle's plane layout: x[dim], v[dim], C[dim*dim], F[dim*dim], aux, each
 * plane `plane_stride` floats after the previous one; it is updated in place.
 * The grid lives in a scratch area compiled into the library (8 MiB + 256 B
 * per GPU, held until process exit) that fits at most 262,144 grid nodes
 * counted in whole 64-node blocks (64^3 in 3D, 512^2 in 2D); larger grids are
 * rejected with MPM_ERR_INVALID.  Every call shares that scratch, so calls
 * whose work overlaps on the GPU race.  The first call on a device looks up the
 * scratch address with that device current; make it before any stream
 * capture begins.  The address is kept per device ordinal for the life of the
 * process: it belongs to the context current at that first call (the device's
 * primary context for runtime-API callers), so later calls must run in that
 * context, and it is not looked up again after a cudaDeviceReset.  Waits for
 * the stream and returns MPM_ERR_SIM if the device error word is set.  Calls
 * no cudaMalloc, cudaFree or allocating routine. */
int mpm_step_noalloc(const mpm_scene_desc *scene, float *state, int64_t plane_stride,
                     int64_t n_particles, int n_substeps, void *stream);

/* ------------------------------------------------------------------------
 * Learned stress surrogate.  No counterpart in the reference, whose stress
 * pass always takes an SVD (MPMCUDA.cu:87-134, 229-264).  A BF16 MLP
 * 10 -> 64 -> 64 -> 9 (SiLU) predicts the residual of sqrt(F F^T) beyond its
 * second-order series; the Kirchhoff stress of jello follows from it without
 * an SVD (snow's stress already reuses the decomposition of its plasticity
 * clamp and keeps the plain path).  Training and inference run on the
 * GPU's tensor cores; particles outside the training envelope, or whose error
 * estimate is above skew_tol, take the SVD path.
 * ---------------------------------------------------------------------- */
typedef struct mpm_surrogate mpm_surrogate;

typedef struct mpm_surrogate_train_options {
    int64_t n_samples;       /* training samples generated from the seeds */
    int epochs;              /* passes over the samples */
    int batch;               /* mini-batch, a multiple of 128 */
    float lr, lr_final;      /* Adam learning rate, cosine-decayed */
    float sigma;             /* std of the singular-value perturbation */
    float rotation_fraction; /* share of samples with a uniformly random rotation */
    float skew_tol;          /* error-estimate tolerance of the fused pass */
    uint64_t seed;
} mpm_surrogate_train_options;

void mpm_surrogate_default_train_options(mpm_surrogate_train_options *opt);

/* Untrained network on a device (its envelope is empty: every particle
 * falls back to the SVD until it is trained or loaded). */
int mpm_surrogate_create(int device, uint64_t seed, mpm_surrogate **out);
int mpm_surrogate_destroy(mpm_surrogate *s);

/* Trains on the GPU from n_seed deformation gradients F_seed[n_seed*9]
 * (row-major, e.g. the F plane of mpm_get_state after plain substeps).  opt
 * may be NULL.  *final_loss (may be NULL) receives the last epoch's mean
 * squared error in units of the output scale. */
int mpm_surrogate_train(mpm_surrogate *s, const float *F_seed, int64_t n_seed,
                        const mpm_surrogate_train_options *opt, float *final_loss);

/* Kirchhoff stress divided by mu of n deformation gradients F[n*9] for
 * lambda/mu = lam_over_mu: tau_pred from the network, tau_ref from the SVD
 * path; accepted[i] = 1 where the fused pass would use the network.  Any
 * output may be NULL. */
int mpm_surrogate_eval(mpm_surrogate *s, const float *F, int64_t n, float lam_over_mu,
                       float *tau_pred, float *tau_ref, uint8_t *accepted);

/* Gradient of the mean squared error over 9 outputs of the batch
 * (x[n*10] network inputs, y_target[n*9] targets, n a multiple of 128,
 * n <= 2^20) with respect to the packed parameters, computed by the training
 * kernels; grads[mpm_surrogate_num_params()], *loss may be NULL. */
int mpm_surrogate_gradients(mpm_surrogate *s, const float *x, const float *y_target, int64_t n,
                            float *grads, float *loss);

/* Packed FP32 parameters: W1[64][16], W2[64][64], W3[16][64], b1[64],
 * b2[64], b3[16] (padding rows and columns zero), and the model constants
 * (in_scale, out_scale, env_c, env_jlo, env_jhi, skew_tol, tau_floor, pad). */
int mpm_surrogate_num_params(void);
int mpm_surrogate_num_meta(void);
int mpm_surrogate_get_params(mpm_surrogate *s, float *params, float *meta);
int mpm_surrogate_set_params(mpm_surrogate *s, const float *params, const float *meta);
int mpm_surrogate_save(mpm_surrogate *s, const char *path);
int mpm_surrogate_load(const char *path, int device, mpm_surrogate **out);

/* Selects the stress of the 3D jello groups: MPM_STRESS_PLAIN, or
 * MPM_STRESS_SURROGATE with network s (kept alive by the caller while the
 * handle uses it; call again after retraining s).  Needs MPM_P2G_ATOMIC;
 * snow, water and 2D scenes keep the plain stress. */
int mpm_set_stress_mode(mpm_handle *h, int mode, mpm_surrogate *s);

/* Particles whose stress came from the network / from the SVD fallback in
 * surrogate mode since the mode was set. */
int mpm_get_stress_stats(mpm_handle *h, int64_t *surrogate, int64_t *fallback);

#ifdef __cplusplus
}
#endif
#endif /* MPM_B200_H */
