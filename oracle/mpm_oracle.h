/*
 * FP64 CPU oracle for the explicit MLS/APIC MPM substep.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * (mpm_cuda_b200/) is compared against.  Only tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py may load it.  The product path never
 * links or calls it.
 *
 * Parity pin: the 3D substep restates MPMSimulator::step() of the reference
 * (src/simulator/MPMCUDA.cu:793-925) and its kernels P2G (:310-433),
 * VelUpdate (:435-472) and InterpolateAndMove (:474-741).  The 2D substep
 * restates the Taichi scripts MPMJello.py:31-120, MPMSnow.py:78-150 and
 * MPMWater.py:71-138.  The 3D oracle is pinned against outputs of the
 * reference's own CUDA build (oracle/_ref, golden fixtures under
 * tests/golden/).  The 2D oracle has no runnable reference here (Taichi is
 * not installed), so its parity rests on this restatement and is cross
 * checked against an independent NumPy restatement in tests/.
 *
 * All arithmetic is FP64, including the stress and its SVD (the reference
 * computes those in FP32; the difference is at FP32 round-off).
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* material type values match the reference enum (Elasiticity.cuh:10-11) */
enum { ORC_JELLO = 0, ORC_SNOW = 1, ORC_WATER = 2, ORC_SAND = 3 };

/* boundary kinds applied in the grid update */
enum {
    ORC_BC_STICKY = 0,   /* zero every component of a wall node (MPMSnow.py:109-111) */
    ORC_BC_SLIP = 1,     /* zero the wall-normal component (MPMCUDA.cu:467-469) */
    ORC_BC_SEPARATE = 2  /* zero the wall-normal component only when it points
                            into the wall (MPMJello.py:92-95) */
};

/* error bits returned by the step functions */
enum {
    ORC_ERR_OUT_OF_GRID = 1,   /* particle stencil leaves the grid */
    ORC_ERR_NONFINITE = 2,     /* NaN/Inf in particle state */
    ORC_ERR_DET = 4,           /* det F <= 0 (jello) or det Fp <= 0 (snow) or J <= 0 */
    ORC_ERR_WEIGHTS = 8        /* |sum w - 1| above 1e-4 */
};

typedef struct {
    int dim;            /* 2 or 3 */
    int n[3];           /* grid nodes per axis (n[2] = 1 in 2D) */
    double h;           /* node spacing */
    double origin[3];
    double dt;
    double gravity[3];
    int bc_type;        /* ORC_BC_* */
    int bc_lo;          /* node index i is a lower-wall node if i < bc_lo */
    int bc_hi;          /* node index i is an upper-wall node if i >= n - bc_hi */
    double mass_eps;    /* nodes with mass <= mass_eps get zero velocity */
    double ref_band;    /* > 0: walls by the reference's FP64 position test with a
                           band of ref_band cells (MPMCUDA.cu:462-469, 845-850);
                           bc_lo / bc_hi are then ignored */
} orc_grid;

typedef struct {
    int type;           /* ORC_JELLO / ORC_SNOW / ORC_WATER */
    double mu, lambda;  /* Lame parameters */
    double xi;          /* snow hardening coefficient (reference: 10) */
    double theta_c;     /* snow clamp: sigma >= 1 - theta_c (reference: 8e-2) */
    double theta_s;     /* snow clamp: sigma <= 1 + theta_s (reference: 2e-2) */
    double bulk_k;      /* water: p = bulk_k * (J^-gamma - 1) (reference: 2.51) */
    double gamma;       /* water exponent (reference: 7) */
    double p_mass, p_vol;
} orc_group;

/*
 * Particle state, AoS per particle, FP64:
 *   x[3N] v[3N] C[9N] F[9N] Fp[9N] J[N] group[N]
 * 2D uses the same strides: x/v components 0..1, matrices in the top-left
 * 2x2 of the row-major 3x3 slot.
 *   F  : elastic deformation gradient (jello, snow)
 *   Fp : plastic deformation gradient (snow)
 *   J  : volume ratio (water)
 */
typedef struct {
    int n;
    double *x, *v, *C, *F, *Fp, *J;
    const int *group;
} orc_particles;

/* Lame parameters from (E, nu), Elasiticity.cuh:42-43 */
void orc_lame(double E, double nu, double *mu, double *lambda);

/* One full substep: clear grid, P2G, grid update, G2P.  grid_mass has
 * n0*n1*n2 entries, grid_mom 3*n0*n1*n2 (x-fastest node index).  After the
 * call grid_mom holds the updated grid velocity.  Returns error bits.
 * nthreads > 1 uses OpenMP over particles (atomics on the grid). */
int orc_substep(const orc_grid *g, const orc_group *groups, orc_particles *p,
                double *grid_mass, double *grid_mom, int nthreads);

/* The three stages separately (same semantics as orc_substep). */
int orc_p2g(const orc_grid *g, const orc_group *groups, const orc_particles *p,
            double *grid_mass, double *grid_mom, int nthreads);
int orc_grid_update(const orc_grid *g, double *grid_mass, double *grid_mom);
int orc_g2p(const orc_grid *g, const orc_group *groups, orc_particles *p,
            const double *grid_vel, int nthreads);

/* Per-particle kernels exposed for unit tests. */
/* Kirchhoff stress of the fixed-corotated model (MPMCUDA.cu:229-264). */
void orc_kirchhoff_fcr(int dim, const double *F, double mu, double lambda, double *tau);
/* F = U diag(s) V^T with det U = det V = +1; s[dim-1] may be negative
 * (PolarSVD, MPMCUDA.cu:87-134). */
void orc_polar_svd(int dim, const double *F, double *U, double *s, double *V);
/* Quadratic B-spline and derivative (MPMCUDA.cu:267-290). */
double orc_bspline(double x);
double orc_bspline_deriv(double x);

/* CPU restatement of the project's particle seeding (mpm_seed in
 * mpm_cuda_b200/csrc/mpm_seed.cu, which replaces the reference's rand()
 * jitter and point-in-mesh loop, MPMSimulator.cpp:198-257): the same
 * splitmix64 jitter per (seed, lattice cell, sample), the same inside tests
 * and the same cell order, every floating-point operation in the same order
 * without contraction, so the positions agree bit for bit.  shape: 0 cube,
 * 1 sphere, 2 cylinder, 3 triangle mesh.  Writes up to cap floats to out
 * (n * dim used) and the particle count to *n_out; returns 0, or -1 on a bad
 * argument or a count above cap / dim. */
int orc_seed(int shape, const double *rotation, const double *scale, const double *translation,
             const float *vertices, long n_vertices, const int *triangles, long n_triangles, int dim,
             double h, const double *origin, int ppc, unsigned long long seed, float *out, long cap,
             long *n_out);

#ifdef __cplusplus
}
#endif
#endif
