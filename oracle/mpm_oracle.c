/*
 * FP64 CPU oracle for the explicit MLS/APIC MPM substep -- TEST
 * INFRASTRUCTURE ONLY (the checker, never the product).  See mpm_oracle.h
 * for the parity pin.
 *
 * Formulas follow, line by line in meaning (not in code):
 *   B-spline N, N'            MPMCUDA.cu:267-308
 *   fixed-corotated Kirchhoff MPMCUDA.cu:229-264
 *   PolarSVD sign convention  MPMCUDA.cu:87-134
 *   P2G                       MPMCUDA.cu:310-433, MPMJello.py:39-78
 *   snow hardening            MPMCUDA.cu:342-349, MPMSnow.py:86-89
 *   water pressure            MPMCUDA.cu:351-354,412-414, MPMWater.py:92
 *   grid update               MPMCUDA.cu:435-472, MPMJello.py:81-95,
 *                             MPMSnow.py:105-114
 *   G2P, F/Fp/J update        MPMCUDA.cu:474-741, MPMSnow.py:116-150,
 *                             MPMWater.py:113-138
 * The SVD is a converged cyclic Jacobi eigen-decomposition of F^T F in FP64
 * (Golub & Van Loan, Matrix Computations, section 8.5), not the reference's
 * FP32 McAdams routine.
 */
#include "mpm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void orc_lame(double E, double nu, double *mu, double *lambda) {
    *mu = E / (2.0 * (1.0 + nu));
    *lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

double orc_bspline(double x) {
    double a = fabs(x);
    if (a < 0.5) return 0.75 - a * a;
    if (a < 1.5) return 0.5 * (1.5 - a) * (1.5 - a);
    return 0.0;
}

double orc_bspline_deriv(double x) {
    if (x > -0.5 && x < 0.5) return -2.0 * x;
    if (x >= 0.5 && x < 1.5) return x - 1.5;
    if (x > -1.5 && x <= -0.5) return 1.5 + x;
    return 0.0;
}

/* ---- small dense helpers on row-major 3x3 slots (dim <= 3) ---- */

static void mat_mul(int d, const double *A, const double *B, double *Cm) {
    double T[9] = {0};
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
            double s = 0.0;
            for (int k = 0; k < d; ++k) s += A[i * 3 + k] * B[k * 3 + j];
            T[i * 3 + j] = s;
        }
    memcpy(Cm, T, sizeof(T));
}

static double mat_det(int d, const double *A) {
    if (d == 2) return A[0] * A[4] - A[1] * A[3];
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}

static void mat_inv(int d, const double *A, double *Ai) {
    double det = mat_det(d, A);
    double id = 1.0 / det;
    double T[9] = {0};
    if (d == 2) {
        T[0] = A[4] * id; T[1] = -A[1] * id;
        T[3] = -A[3] * id; T[4] = A[0] * id;
    } else {
        T[0] = (A[4] * A[8] - A[5] * A[7]) * id;
        T[1] = (A[2] * A[7] - A[1] * A[8]) * id;
        T[2] = (A[1] * A[5] - A[2] * A[4]) * id;
        T[3] = (A[5] * A[6] - A[3] * A[8]) * id;
        T[4] = (A[0] * A[8] - A[2] * A[6]) * id;
        T[5] = (A[2] * A[3] - A[0] * A[5]) * id;
        T[6] = (A[3] * A[7] - A[4] * A[6]) * id;
        T[7] = (A[1] * A[6] - A[0] * A[7]) * id;
        T[8] = (A[0] * A[4] - A[1] * A[3]) * id;
    }
    memcpy(Ai, T, sizeof(T));
}

/* Cyclic Jacobi eigen-decomposition of a symmetric d x d matrix S:
 * S = Q diag(lam) Q^T, columns of Q are eigenvectors. */
static void sym_eig(int d, const double *S_in, double *lam, double *Q) {
    double S[9];
    memcpy(S, S_in, sizeof(S));
    for (int i = 0; i < 9; ++i) Q[i] = 0.0;
    for (int i = 0; i < d; ++i) Q[i * 3 + i] = 1.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < d; ++i)
            for (int j = 0; j < d; ++j) {
                tot += S[i * 3 + j] * S[i * 3 + j];
                if (i != j) off += S[i * 3 + j] * S[i * 3 + j];
            }
        if (off <= 1e-32 * tot || off == 0.0) break;
        for (int p = 0; p < d - 1; ++p)
            for (int q = p + 1; q < d; ++q) {
                double apq = S[p * 3 + q];
                if (apq == 0.0) continue;
                double app = S[p * 3 + p], aqq = S[q * 3 + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                /* S <- J^T S J with J the (p,q) rotation */
                for (int k = 0; k < d; ++k) {
                    double skp = S[k * 3 + p], skq = S[k * 3 + q];
                    S[k * 3 + p] = c * skp - s * skq;
                    S[k * 3 + q] = s * skp + c * skq;
                }
                for (int k = 0; k < d; ++k) {
                    double spk = S[p * 3 + k], sqk = S[q * 3 + k];
                    S[p * 3 + k] = c * spk - s * sqk;
                    S[q * 3 + k] = s * spk + c * sqk;
                }
                for (int k = 0; k < d; ++k) {
                    double qkp = Q[k * 3 + p], qkq = Q[k * 3 + q];
                    Q[k * 3 + p] = c * qkp - s * qkq;
                    Q[k * 3 + q] = s * qkp + c * qkq;
                }
            }
    }
    for (int i = 0; i < d; ++i) lam[i] = S[i * 3 + i];
}

void orc_polar_svd(int d, const double *F, double *U, double *s, double *V) {
    double S[9] = {0};
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
            double a = 0.0;
            for (int k = 0; k < d; ++k) a += F[k * 3 + i] * F[k * 3 + j];
            S[i * 3 + j] = a;
        }
    double lam[3] = {0}, Q[9];
    sym_eig(d, S, lam, Q);
    /* sort eigenpairs by decreasing eigenvalue */
    int idx[3] = {0, 1, 2};
    for (int i = 0; i < d; ++i)
        for (int j = i + 1; j < d; ++j)
            if (lam[idx[j]] > lam[idx[i]]) { int t = idx[i]; idx[i] = idx[j]; idx[j] = t; }
    for (int i = 0; i < 9; ++i) V[i] = 0.0;
    for (int c = 0; c < d; ++c)
        for (int r = 0; r < d; ++r) V[r * 3 + c] = Q[r * 3 + idx[c]];
    if (mat_det(d, V) < 0.0)
        for (int r = 0; r < d; ++r) V[r * 3 + (d - 1)] = -V[r * 3 + (d - 1)];
    /* FV columns */
    double FV[9];
    mat_mul(d, F, V, FV);
    for (int i = 0; i < 9; ++i) U[i] = 0.0;
    double u1[3] = {0}, u2[3] = {0}, u3[3] = {0};
    double n1 = 0.0;
    for (int r = 0; r < d; ++r) n1 += FV[r * 3] * FV[r * 3];
    n1 = sqrt(n1);
    if (n1 > 0.0) for (int r = 0; r < d; ++r) u1[r] = FV[r * 3] / n1;
    else u1[0] = 1.0;
    if (d == 2) {
        u2[0] = -u1[1]; u2[1] = u1[0];
        for (int r = 0; r < 2; ++r) { U[r * 3] = u1[r]; U[r * 3 + 1] = u2[r]; }
        s[0] = u1[0] * FV[0] + u1[1] * FV[3];
        s[1] = u2[0] * FV[1] + u2[1] * FV[4];
        s[2] = 0.0;
        return;
    }
    /* Gram-Schmidt for the second column, cross product for the third */
    double dot = 0.0;
    for (int r = 0; r < 3; ++r) dot += u1[r] * FV[r * 3 + 1];
    for (int r = 0; r < 3; ++r) u2[r] = FV[r * 3 + 1] - dot * u1[r];
    double n2 = sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
    if (n2 > 1e-300 * (n1 + 1e-300)) {
        for (int r = 0; r < 3; ++r) u2[r] /= n2;
    } else {
        /* any unit vector orthogonal to u1 */
        double e[3] = {0, 0, 0};
        int m = (fabs(u1[0]) < fabs(u1[1])) ? (fabs(u1[0]) < fabs(u1[2]) ? 0 : 2)
                                             : (fabs(u1[1]) < fabs(u1[2]) ? 1 : 2);
        e[m] = 1.0;
        double dd = u1[0] * e[0] + u1[1] * e[1] + u1[2] * e[2];
        for (int r = 0; r < 3; ++r) u2[r] = e[r] - dd * u1[r];
        double nn = sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
        for (int r = 0; r < 3; ++r) u2[r] /= nn;
    }
    u3[0] = u1[1] * u2[2] - u1[2] * u2[1];
    u3[1] = u1[2] * u2[0] - u1[0] * u2[2];
    u3[2] = u1[0] * u2[1] - u1[1] * u2[0];
    for (int r = 0; r < 3; ++r) { U[r * 3] = u1[r]; U[r * 3 + 1] = u2[r]; U[r * 3 + 2] = u3[r]; }
    s[0] = s[1] = s[2] = 0.0;
    for (int r = 0; r < 3; ++r) {
        s[0] += u1[r] * FV[r * 3 + 0];
        s[1] += u2[r] * FV[r * 3 + 1];
        s[2] += u3[r] * FV[r * 3 + 2];
    }
}

void orc_kirchhoff_fcr(int d, const double *F, double mu, double lambda, double *tau) {
    double U[9], s[3], V[9], R[9], Vt[9] = {0};
    orc_polar_svd(d, F, U, s, V);
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) Vt[i * 3 + j] = V[j * 3 + i];
    mat_mul(d, U, Vt, R);
    double FmR[9] = {0}, Ft[9] = {0}, T[9];
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
            FmR[i * 3 + j] = F[i * 3 + j] - R[i * 3 + j];
            Ft[i * 3 + j] = F[j * 3 + i];
        }
    mat_mul(d, FmR, Ft, T);
    double J = mat_det(d, F);
    for (int i = 0; i < 9; ++i) tau[i] = 0.0;
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j)
            tau[i * 3 + j] = 2.0 * mu * T[i * 3 + j] + (i == j ? lambda * J * (J - 1.0) : 0.0);
}

static int base_index(double x, double o, double h) {
    double q = (x - o - 0.5 * h) / h;
    if (!(q < 1e9)) q = 1e9; /* far outside: stays out of the grid, no int overflow */
    int b = (int)q;          /* C truncation, as MPMCUDA.cu:356 */
    return b < 0 ? 0 : b;
}

static int finite_all(const double *a, int n) {
    for (int i = 0; i < n; ++i)
        if (!isfinite(a[i])) return 0;
    return 1;
}

int orc_p2g(const orc_grid *g, const orc_group *groups, const orc_particles *p,
            double *grid_mass, double *grid_mom, int nthreads) {
    const int d = g->dim;
    const double h = g->h;
    const long nx = g->n[0], ny = g->n[1], nz = (d == 3) ? g->n[2] : 1;
    int err = 0;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(| : err)
    for (int i = 0; i < p->n; ++i) {
        const orc_group *grp = &groups[p->group ? p->group[i] : 0];
        const double *x = &p->x[3 * i], *v = &p->v[3 * i], *Cp = &p->C[9 * i];
        double tau[9] = {0};
        double water_p = 0.0, water_J = 0.0;
        if (!finite_all(x, d) || !finite_all(v, d)) { err |= ORC_ERR_NONFINITE; continue; }
        if (grp->type == ORC_JELLO) {
            orc_kirchhoff_fcr(d, &p->F[9 * i], grp->mu, grp->lambda, tau);
        } else if (grp->type == ORC_SNOW) {
            double Jp = mat_det(d, &p->Fp[9 * i]);
            double hc = exp(grp->xi * (1.0 - Jp));
            orc_kirchhoff_fcr(d, &p->F[9 * i], grp->mu * hc, grp->lambda * hc, tau);
        } else if (grp->type == ORC_WATER) {
            water_J = p->J[i];
            water_p = grp->bulk_k * (1.0 / pow(water_J, grp->gamma) - 1.0);
        }
        int base[3] = {0, 0, 0};
        for (int a = 0; a < d; ++a) base[a] = base_index(x[a], g->origin[a], h);
        double wsum = 0.0;
        const int kz = (d == 3) ? 3 : 1;
        for (int ox = 0; ox < 3; ++ox)
            for (int oy = 0; oy < 3; ++oy)
                for (int oz = 0; oz < kz; ++oz) {
                    int id[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
                    if (id[0] >= nx || id[1] >= ny || (d == 3 && id[2] >= nz)) {
                        err |= ORC_ERR_OUT_OF_GRID;
                        continue;
                    }
                    double dx[3] = {0}, N[3] = {1, 1, 1}, dN[3] = {0, 0, 0}, bpos[3] = {0};
                    for (int a = 0; a < d; ++a) {
                        bpos[a] = g->origin[a] + id[a] * h;
                        dx[a] = bpos[a] - x[a];
                        double r = (x[a] - bpos[a]) / h;
                        N[a] = orc_bspline(r);
                        dN[a] = orc_bspline_deriv(r);
                    }
                    double w = N[0] * N[1] * N[2];
                    double gw[3] = {0};
                    gw[0] = dN[0] * N[1] * N[2] / h;
                    gw[1] = N[0] * dN[1] * N[2] / h;
                    if (d == 3) gw[2] = N[0] * N[1] * dN[2] / h;
                    long gi = (long)id[2] * nx * ny + (long)id[1] * nx + id[0];
                    double m = w * grp->p_mass;
                    double mom[3] = {0};
                    for (int a = 0; a < d; ++a) {
                        double cdx = 0.0;
                        for (int b = 0; b < d; ++b) cdx += Cp[a * 3 + b] * dx[b];
                        mom[a] = m * (v[a] + cdx);
                    }
                    double f[3] = {0};
                    if (grp->type == ORC_WATER) {
                        for (int a = 0; a < d; ++a) f[a] = grp->p_vol * water_p * water_J * gw[a];
                    } else {
                        for (int a = 0; a < d; ++a) {
                            double s = 0.0;
                            for (int b = 0; b < d; ++b) s += tau[a * 3 + b] * gw[b];
                            f[a] = -grp->p_vol * s;
                        }
                    }
#pragma omp atomic
                    grid_mass[gi] += m;
                    for (int a = 0; a < d; ++a) {
                        double add = mom[a] + g->dt * f[a];
#pragma omp atomic
                        grid_mom[3 * gi + a] += add;
                    }
                    wsum += w;
                }
        if (fabs(wsum - 1.0) > 1e-4) err |= ORC_ERR_WEIGHTS;
    }
    return err;
}

int orc_grid_update(const orc_grid *g, double *grid_mass, double *grid_mom) {
    const int d = g->dim;
    const long nx = g->n[0], ny = g->n[1], nz = (d == 3) ? g->n[2] : 1;
    const long G = nx * ny * nz;
    for (long i = 0; i < G; ++i) {
        double m = grid_mass[i];
        double *vel = &grid_mom[3 * i];
        if (!(m > g->mass_eps)) {
            grid_mass[i] = 0.0;
            vel[0] = vel[1] = vel[2] = 0.0;
            continue;
        }
        for (int a = 0; a < d; ++a) vel[a] = vel[a] / m + g->dt * g->gravity[a];
        long id[3] = {i % nx, (i / nx) % ny, i / (nx * ny)};
        int lo[3], hi[3], any = 0;
        for (int a = 0; a < d; ++a) {
            if (g->ref_band > 0.0) {
                /* MPMCUDA.cu:462-469: node position origin + idx * h (a fused
                 * multiply-add in the reference's kernel) against the bounds
                 * origin + band h and origin + h n - band h, which the
                 * reference's host code computes one rounded operation at a
                 * time (MPMCUDA.cu:845-850) */
                volatile double bh = g->ref_band * g->h;
                volatile double top = g->origin[a] + g->h * (double)g->n[a];
                const double lower = g->origin[a] + bh, upper = top - bh;
                const double pos = fma((double)id[a], g->h, g->origin[a]);
                lo[a] = pos <= lower;
                hi[a] = pos >= upper;
            } else {
                lo[a] = id[a] < g->bc_lo;
                hi[a] = id[a] >= g->n[a] - g->bc_hi;
            }
            any |= lo[a] | hi[a];
        }
        if (g->bc_type == ORC_BC_STICKY) {
            if (any) vel[0] = vel[1] = vel[2] = 0.0;
        } else if (g->bc_type == ORC_BC_SLIP) {
            for (int a = 0; a < d; ++a)
                if (lo[a] || hi[a]) vel[a] = 0.0;
        } else {
            for (int a = 0; a < d; ++a) {
                if (lo[a] && vel[a] < 0.0) vel[a] = 0.0;
                if (hi[a] && vel[a] > 0.0) vel[a] = 0.0;
            }
        }
    }
    return 0;
}

int orc_g2p(const orc_grid *g, const orc_group *groups, orc_particles *p,
            const double *grid_vel, int nthreads) {
    const int d = g->dim;
    const double h = g->h, dt = g->dt;
    const long nx = g->n[0], ny = g->n[1], nz = (d == 3) ? g->n[2] : 1;
    int err = 0;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(| : err)
    for (int i = 0; i < p->n; ++i) {
        const orc_group *grp = &groups[p->group ? p->group[i] : 0];
        double *x = &p->x[3 * i];
        if (!finite_all(x, d)) { err |= ORC_ERR_NONFINITE; continue; }
        int base[3] = {0, 0, 0};
        for (int a = 0; a < d; ++a) base[a] = base_index(x[a], g->origin[a], h);
        double vp[3] = {0}, Cn[9] = {0}, gv[9] = {0}, div = 0.0, wsum = 0.0;
        const int kz = (d == 3) ? 3 : 1;
        for (int ox = 0; ox < 3; ++ox)
            for (int oy = 0; oy < 3; ++oy)
                for (int oz = 0; oz < kz; ++oz) {
                    int id[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
                    if (id[0] >= nx || id[1] >= ny || (d == 3 && id[2] >= nz)) {
                        err |= ORC_ERR_OUT_OF_GRID;
                        continue;
                    }
                    double dx[3] = {0}, N[3] = {1, 1, 1}, dN[3] = {0, 0, 0};
                    for (int a = 0; a < d; ++a) {
                        double bpos = g->origin[a] + id[a] * h;
                        dx[a] = bpos - x[a];
                        double r = (x[a] - bpos) / h;
                        N[a] = orc_bspline(r);
                        dN[a] = orc_bspline_deriv(r);
                    }
                    double w = N[0] * N[1] * N[2];
                    double gw[3] = {0};
                    gw[0] = dN[0] * N[1] * N[2] / h;
                    gw[1] = N[0] * dN[1] * N[2] / h;
                    if (d == 3) gw[2] = N[0] * N[1] * dN[2] / h;
                    long gi = (long)id[2] * nx * ny + (long)id[1] * nx + id[0];
                    const double *vi = &grid_vel[3 * gi];
                    for (int a = 0; a < d; ++a) {
                        vp[a] += w * vi[a];
                        for (int b = 0; b < d; ++b) {
                            Cn[a * 3 + b] += 4.0 * w / (h * h) * vi[a] * dx[b];
                            gv[a * 3 + b] += vi[a] * gw[b];
                        }
                        div += vi[a] * gw[a];
                    }
                    wsum += w;
                }
        if (fabs(wsum - 1.0) > 1e-4) err |= ORC_ERR_WEIGHTS;
        double L[9] = {0};
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) L[a * 3 + b] = (a == b ? 1.0 : 0.0) + dt * gv[a * 3 + b];
        if (grp->type == ORC_JELLO) {
            double *F = &p->F[9 * i];
            mat_mul(d, L, F, F);
            if (!(mat_det(d, F) > 0.0)) err |= ORC_ERR_DET;
        } else if (grp->type == ORC_SNOW) {
            double *Fe = &p->F[9 * i], *Fp = &p->Fp[9 * i];
            double Ft[9], U[9], s[3], V[9];
            mat_mul(d, L, Fe, Ft);
            orc_polar_svd(d, Ft, U, s, V);
            double Us[9] = {0}, Vt[9] = {0}, Fn[9], Fni[9], T[9];
            for (int a = 0; a < d; ++a) {
                double sc = s[a];
                if (sc < 1.0 - grp->theta_c) sc = 1.0 - grp->theta_c;
                if (sc > 1.0 + grp->theta_s) sc = 1.0 + grp->theta_s;
                for (int r = 0; r < d; ++r) Us[r * 3 + a] = U[r * 3 + a] * sc;
                for (int c = 0; c < d; ++c) Vt[a * 3 + c] = V[c * 3 + a];
            }
            mat_mul(d, Us, Vt, Fn);
            mat_inv(d, Fn, Fni);
            mat_mul(d, Fni, Ft, T);
            mat_mul(d, T, Fp, Fp);
            memcpy(Fe, Fn, sizeof(Fn));
            if (!(mat_det(d, Fp) > 0.0)) err |= ORC_ERR_DET;
        } else if (grp->type == ORC_WATER) {
            p->J[i] = (1.0 + dt * div) * p->J[i];
            if (!(p->J[i] > 0.0)) err |= ORC_ERR_DET;
        }
        double *v = &p->v[3 * i];
        double *Cp = &p->C[9 * i];
        for (int a = 0; a < d; ++a) {
            v[a] = vp[a];
            x[a] += dt * vp[a];
            for (int b = 0; b < d; ++b) Cp[a * 3 + b] = Cn[a * 3 + b];
        }
        if (!finite_all(x, d) || !finite_all(v, d)) err |= ORC_ERR_NONFINITE;
    }
    return err;
}

int orc_substep(const orc_grid *g, const orc_group *groups, orc_particles *p,
                double *grid_mass, double *grid_mom, int nthreads) {
    const long G = (long)g->n[0] * g->n[1] * (g->dim == 3 ? g->n[2] : 1);
    memset(grid_mass, 0, sizeof(double) * G);
    memset(grid_mom, 0, sizeof(double) * 3 * G);
    int err = orc_p2g(g, groups, p, grid_mass, grid_mom, nthreads);
    err |= orc_grid_update(g, grid_mass, grid_mom);
    err |= orc_g2p(g, groups, p, grid_mom, nthreads);
    return err;
}


/* ------------------------------------------------------------------ seeding
 * Restatement of mpm_seed (mpm_cuda_b200/csrc/mpm_seed.cu), operation for
 * operation; this file is compiled with -ffp-contract=off. */

/* splitmix64 finaliser (Steele, Lea, Flood 2014) */
static unsigned long long seed_mix(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

typedef struct {
    int shape, dim, ppc;
    double R[9], S[3], T[3], h, origin[3];
    int i0[3], ni[3];
    unsigned long long seed;
    const float *vert;
    const int *tri, *bin_start, *bin_tri;
    int nbx, nby;
    double blo[2], bhi[2];
} seed_params;

static double dcross(double a, double b, double c, double d) { return a * b - c * d; }

static int edge_in(double ax, double ay, double bx, double by, double px, double py) {
    const double e = dcross(bx - ax, py - ay, by - ay, px - ax);
    if (e != 0.0) return e > 0.0;
    return (by > ay) || (by == ay && bx < ax);
}

static int inside_mesh(const seed_params *P, const double *l) {
    if (!(l[0] >= P->blo[0] && l[0] < P->bhi[0] && l[1] >= P->blo[1] && l[1] < P->bhi[1])) return 0;
    int bx = (int)((l[0] - P->blo[0]) / (P->bhi[0] - P->blo[0]) * P->nbx);
    int by = (int)((l[1] - P->blo[1]) / (P->bhi[1] - P->blo[1]) * P->nby);
    if (bx > P->nbx - 1) bx = P->nbx - 1;
    if (by > P->nby - 1) by = P->nby - 1;
    const int b = by * P->nbx + bx;
    int hits = 0;
    for (int k = P->bin_start[b]; k < P->bin_start[b + 1]; ++k) {
        const int t = P->bin_tri[k];
        const float *A = P->vert + 3 * P->tri[3 * t], *B = P->vert + 3 * P->tri[3 * t + 1],
                    *Cc = P->vert + 3 * P->tri[3 * t + 2];
        double ax = A[0], ay = A[1], bxx = B[0], byy = B[1], cx = Cc[0], cy = Cc[1];
        double az = A[2], bz = B[2], cz = Cc[2];
        const double area = dcross(bxx - ax, cy - ay, byy - ay, cx - ax);
        if (area == 0.0) continue;
        if (area < 0.0) {
            double tx = bxx, ty = byy, tz = bz;
            bxx = cx; byy = cy; bz = cz;
            cx = tx; cy = ty; cz = tz;
        }
        if (!edge_in(ax, ay, bxx, byy, l[0], l[1]) || !edge_in(bxx, byy, cx, cy, l[0], l[1]) ||
            !edge_in(cx, cy, ax, ay, l[0], l[1]))
            continue;
        const double a2 = fabs(area);
        const double wa = dcross(bxx - l[0], cy - l[1], byy - l[1], cx - l[0]) / a2;
        const double wb = dcross(cx - l[0], ay - l[1], cy - l[1], ax - l[0]) / a2;
        const double z = (wa * az + wb * bz) + ((1.0 - wa) - wb) * cz;
        if (z > l[2]) ++hits;
    }
    return hits & 1;
}

/* sample k of lattice cell (ix, iy, iz), linear cell index `cell` */
static int seed_sample(const seed_params *P, long long cell, int ix, int iy, int iz, int k, float *w) {
    const unsigned long long base = seed_mix(P->seed ^ seed_mix((unsigned long long)cell * 64ull + (unsigned)k));
    const int ic[3] = {ix, iy, iz};
    double q[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < P->dim; ++a) {
        const double u = (double)(seed_mix(base + (unsigned long long)a) >> 11) * (1.0 / 9007199254740992.0);
        const double lo = P->origin[a] + (double)ic[a] * P->h;
        const double hi = P->origin[a] + ((double)ic[a] + 1.0) * P->h;
        float f = (float)(P->origin[a] + ((double)ic[a] + u) * P->h);
        if ((double)f >= hi) f = nextafterf(f, -INFINITY);
        if ((double)f < lo) f = nextafterf(f, INFINITY);
        w[a] = f;
        q[a] = ((double)w[a] - P->T[a]) / P->S[a];
    }
    double l[3];
    for (int a = 0; a < 3; ++a) l[a] = (P->R[a] * q[0] + P->R[3 + a] * q[1]) + P->R[6 + a] * q[2];
    switch (P->shape) {
        case 0:
            return fabs(l[0]) <= 0.5 && fabs(l[1]) <= 0.5 && (P->dim == 2 || fabs(l[2]) <= 0.5);
        case 1:
            return (l[0] * l[0] + l[1] * l[1]) + (P->dim == 3 ? l[2] * l[2] : 0.0) <= 0.25;
        case 2:
            return l[0] * l[0] + l[2] * l[2] <= 0.25 && fabs(l[1]) <= 0.5;
        default:
            return inside_mesh(P, l);
    }
}

int orc_seed(int shape, const double *rotation, const double *scale, const double *translation,
             const float *vertices, long n_vertices, const int *triangles, long n_triangles, int dim,
             double h, const double *origin, int ppc, unsigned long long seed, float *out, long cap,
             long *n_out) {
    if (!n_out || !(h > 0.0) || ppc < 1 || ppc > 64 || (dim != 2 && dim != 3) || shape < 0 || shape > 3) return -1;
    seed_params P;
    memset(&P, 0, sizeof(P));
    P.shape = shape;
    P.dim = dim;
    P.ppc = ppc;
    P.h = h;
    P.seed = seed;
    for (int a = 0; a < 9; ++a) P.R[a] = rotation[a];
    for (int a = 0; a < 3; ++a) {
        P.S[a] = scale[a];
        P.T[a] = translation[a];
        P.origin[a] = origin ? origin[a] : 0.0;
    }
    double llo[3] = {-0.5, -0.5, -0.5}, lhi[3] = {0.5, 0.5, 0.5};
    int *bin_start = NULL, *bin_tri = NULL;
    if (shape == 3) {
        if (dim != 3 || !vertices || !triangles || n_vertices <= 0 || n_triangles <= 0) return -1;
        for (int a = 0; a < 3; ++a) {
            llo[a] = 1e300;
            lhi[a] = -1e300;
        }
        for (long v = 0; v < n_vertices; ++v)
            for (int a = 0; a < 3; ++a) {
                llo[a] = fmin(llo[a], (double)vertices[3 * v + a]);
                lhi[a] = fmax(lhi[a], (double)vertices[3 * v + a]);
            }
        int nb = (int)sqrt((double)n_triangles);
        if (nb > 256) nb = 256;
        if (nb < 1) nb = 1;
        P.nbx = P.nby = nb;
        const double pad = 1e-9 * fmax(1.0, fmax(lhi[0] - llo[0], lhi[1] - llo[1]));
        P.blo[0] = llo[0] - pad;
        P.blo[1] = llo[1] - pad;
        P.bhi[0] = lhi[0] + pad;
        P.bhi[1] = lhi[1] + pad;
        /* CSR triangle lists of the xy bins, triangles ascending in each bin */
        int *counts = calloc((size_t)nb * nb + 1, sizeof(int));
        int (*span)[4] = malloc((size_t)n_triangles * sizeof(*span));
        for (long t = 0; t < n_triangles; ++t) {
            double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
            for (int c = 0; c < 3; ++c) {
                const float *p = vertices + 3 * triangles[3 * t + c];
                x0 = fmin(x0, (double)p[0]);
                x1 = fmax(x1, (double)p[0]);
                y0 = fmin(y0, (double)p[1]);
                y1 = fmax(y1, (double)p[1]);
            }
            const double ev[4] = {x0, x1, y0, y1};
            for (int e = 0; e < 4; ++e) {
                const int ax = e / 2;
                int bi = (int)((ev[e] - P.blo[ax]) / (P.bhi[ax] - P.blo[ax]) * nb);
                span[t][e] = bi < 0 ? 0 : (bi > nb - 1 ? nb - 1 : bi);
            }
            for (int by = span[t][2]; by <= span[t][3]; ++by)
                for (int bx = span[t][0]; bx <= span[t][1]; ++bx) counts[by * nb + bx + 1]++;
        }
        bin_start = malloc(((size_t)nb * nb + 1) * sizeof(int));
        bin_start[0] = 0;
        for (int b = 0; b < nb * nb; ++b) bin_start[b + 1] = bin_start[b] + counts[b + 1];
        bin_tri = malloc((size_t)(bin_start[nb * nb] > 0 ? bin_start[nb * nb] : 1) * sizeof(int));
        int *fill = calloc((size_t)nb * nb, sizeof(int));
        for (long t = 0; t < n_triangles; ++t)
            for (int by = span[t][2]; by <= span[t][3]; ++by)
                for (int bx = span[t][0]; bx <= span[t][1]; ++bx) {
                    const int b = by * nb + bx;
                    bin_tri[bin_start[b] + fill[b]++] = (int)t;
                }
        free(fill);
        free(span);
        free(counts);
        P.vert = vertices;
        P.tri = triangles;
        P.bin_start = bin_start;
        P.bin_tri = bin_tri;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; ++c) {
        const double p[3] = {(c & 1) ? lhi[0] : llo[0], (c & 2) ? lhi[1] : llo[1], (c & 4) ? lhi[2] : llo[2]};
        for (int a = 0; a < 3; ++a) {
            const double w = P.T[a] + P.S[a] * ((P.R[a * 3] * p[0] + P.R[a * 3 + 1] * p[1]) + P.R[a * 3 + 2] * p[2]);
            lo[a] = fmin(lo[a], w);
            hi[a] = fmax(hi[a], w);
        }
    }
    for (int a = 0; a < 3; ++a) {
        if (a >= dim) {
            P.i0[a] = 0;
            P.ni[a] = 1;
            continue;
        }
        const double i0 = floor((lo[a] - P.origin[a]) / h), i1 = floor((hi[a] - P.origin[a]) / h) + 1.0;
        P.i0[a] = (int)i0;
        P.ni[a] = (int)(i1 - i0);
    }
    long n = 0;
    int rc = 0;
    float w[3];
    for (int ix = 0; ix < P.ni[0]; ++ix)
        for (int iy = 0; iy < P.ni[1]; ++iy)
            for (int iz = 0; iz < P.ni[2]; ++iz) {
                const long long cell = ((long long)ix * P.ni[1] + iy) * P.ni[2] + iz;
                for (int k = 0; k < ppc; ++k)
                    if (seed_sample(&P, cell, P.i0[0] + ix, P.i0[1] + iy, P.i0[2] + iz, k, w)) {
                        if (out) {
                            if ((n + 1) * dim > cap) {
                                rc = -1;
                                continue;
                            }
                            for (int a = 0; a < dim; ++a) out[n * dim + a] = w[a];
                        }
                        ++n;
                    }
            }
    free(bin_start);
    free(bin_tri);
    *n_out = n;
    return rc;
}
