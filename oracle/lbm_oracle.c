/* ============================================================================
 *  lbm_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle). Plain-C restatement
 *  of the reference's D3Q19 TRT + Guo + bounce-back + squirmer algorithm,
 *  operation for operation, so that with one thread it reproduces the
 *  reference bit for bit (both are compiled in ISO mode, where GCC does not
 *  contract a*b+c into FMA). Each function cites the reference lines it
 *  restates. It stores populations the reference's way -- two buffers f and
 *  fnew, push streaming -- and is deliberately not optimised.
 * ==========================================================================*/
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LBO_PI 3.14159265358979323846

/* D3Q19 velocity set in opposite pairs, weights (lattice.hpp:18-30). */
enum { Q = 19 };
static const int cx[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int cy[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int cz[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int opp[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const double w[Q] = {1.0 / 3.0,
                            1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18,
                            1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36,
                            1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
enum { FLUID = 0, WALL = 1, PARTICLE = 2 };

typedef struct {
    double R, B1, beta, M, I;
    int planar;
    double X[3], e[3], U[3], W[3];
    double Fh[3], Th[3], Fc[3], Tc[3], Fw[3];
    double eps, hc, hmin, FS;
    long contacts;
} sqm;

struct lbo_state {
    int NX, NY, NZ;
    size_t N;
    double tau, omPlus, omMinus, nu;
    double F[3];
    int wallsY, wallsZ;
    int massCorrectionEvery, trajEvery;
    double *f, *fnew, *rho, *ux, *uy, *uz;
    unsigned char* flag;
    double wallForce[3];
    int hasSquirmer;
    sqm sq;
    long t;
};

static size_t idx(const lbo_state* s, int x, int y, int z) {
    return (size_t)x + (size_t)s->NX * ((size_t)y + (size_t)s->NY * (size_t)z);
}

/* equilibrium() (lattice.hpp:42-47) */
static double equilibrium(int i, double rho, double ux, double uy, double uz) {
    const double cu = cx[i] * ux + cy[i] * uy + cz[i] * uz;
    const double usq = ux * ux + uy * uy + uz * uz;
    return w[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
}

/* cross() (lattice.hpp:52-56) */
static void cross(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* Squirmer::surfaceVelocity (squirmer.cpp:35-46) */
static void surface_velocity(const sqm* q, const double r[3], double ub[3], int withSlip) {
    double wr[3];
    cross(q->W, r, wr);
    for (int d = 0; d < 3; ++d) ub[d] = q->U[d] + wr[d];
    if (!withSlip) return;
    const double rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (rn < 1e-12) return;
    const double rh[3] = {r[0] / rn, r[1] / rn, r[2] / rn};
    const double ct = q->e[0] * rh[0] + q->e[1] * rh[1] + q->e[2] * rh[2];
    const double amp = q->B1 * (1.0 + q->beta * ct);
    for (int d = 0; d < 3; ++d) ub[d] += amp * (ct * rh[d] - q->e[d]);
}

/* Squirmer::integrate (squirmer.cpp:52-68) */
static void integrate(sqm* q) {
    for (int d = 0; d < 3; ++d) {
        q->U[d] += (q->Fh[d] + q->Fc[d] + q->Fw[d]) / q->M;
        q->W[d] += (q->Th[d] + q->Tc[d]) / q->I;
        q->Fc[d] = q->Tc[d] = 0.0;
    }
    if (q->planar) { q->U[2] = 0.0; q->W[0] = 0.0; q->W[1] = 0.0; }
    for (int d = 0; d < 3; ++d) q->X[d] += q->U[d];
    double we[3];
    cross(q->W, q->e, we);
    for (int d = 0; d < 3; ++d) q->e[d] += we[d];
    if (q->planar) q->e[2] = 0.0;
    const double n = sqrt(q->e[0] * q->e[0] + q->e[1] * q->e[1] + q->e[2] * q->e[2]);
    for (int d = 0; d < 3; ++d) q->e[d] /= n;
}

/* softWallForce (squirmer.cpp:73-77) */
static double soft_wall_force(double h, double eps, double FS, double hc) {
    if (h >= hc) return 0.0;
    const double s = 1.0 - (h > 0.0 ? h : 0.0) / hc;
    return eps * FS * s * s;
}

/* LBM::offsetFromSquirmer (lbm.cpp:100-104) */
static void offset_from_squirmer(const lbo_state* s, double px, double py, double pz, double r[3]) {
    r[0] = px - s->sq.X[0]; r[0] -= s->NX * round(r[0] / s->NX);
    r[1] = py - s->sq.X[1]; if (!s->wallsY) r[1] -= s->NY * round(r[1] / s->NY);
    r[2] = pz - s->sq.X[2]; if (!s->wallsZ) r[2] -= s->NZ * round(r[2] / s->NZ);
}

/* LBM::updateParticleFlags (lbm.cpp:271-320) */
static void update_particle_flags(lbo_state* s, int initial) {
    sqm* q = &s->sq;
    const double R = q->R;
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const size_t N = s->N;
    const int x0 = (int)floor(q->X[0] - R) - 2, x1 = (int)ceil(q->X[0] + R) + 2;
    int y0 = (int)floor(q->X[1] - R) - 2, y1 = (int)ceil(q->X[1] + R) + 2;
    const int z0 = (int)floor(q->X[2] - R) - 2, z1 = (int)ceil(q->X[2] + R) + 2;
    if (s->wallsY) { if (y0 < 0) y0 = 0; if (y1 > NY - 1) y1 = NY - 1; }

    for (int zz = z0; zz <= z1; ++zz)
        for (int yy = y0; yy <= y1; ++yy)
            for (int xx = x0; xx <= x1; ++xx) {
                const int x = ((xx % NX) + NX) % NX;
                const int y = ((yy % NY) + NY) % NY;
                const int z = ((zz % NZ) + NZ) % NZ;
                const size_t n = idx(s, x, y, z);
                if (s->flag[n] == WALL) continue;
                double r[3];
                offset_from_squirmer(s, x, y, z, r);
                const int inside = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < R * R;
                const int was = s->flag[n] == PARTICLE;
                if (inside == was) continue;
                if (initial) { s->flag[n] = inside ? PARTICLE : FLUID; continue; }
                if (inside) {
                    double p[3] = {0, 0, 0}, t[3];
                    for (int i = 0; i < Q; ++i) {
                        const double fv = s->f[(size_t)i * N + n];
                        p[0] += fv * cx[i]; p[1] += fv * cy[i]; p[2] += fv * cz[i];
                    }
                    cross(r, p, t);
                    for (int d = 0; d < 3; ++d) { q->Fc[d] += p[d]; q->Tc[d] += t[d]; }
                    s->flag[n] = PARTICLE;
                } else {
                    double rs = 0; int cnt = 0;
                    for (int i = 1; i < Q; ++i) {
                        const int xn = (x + cx[i] + NX) % NX, yn = (y + cy[i] + NY) % NY,
                                  zn = (z + cz[i] + NZ) % NZ;
                        const size_t nb = idx(s, xn, yn, zn);
                        if (s->flag[nb] == FLUID) { rs += s->rho[nb]; ++cnt; }
                    }
                    const double rr = cnt ? rs / cnt : 1.0;
                    double ub[3];
                    surface_velocity(q, r, ub, 0);
                    for (int i = 0; i < Q; ++i) s->f[(size_t)i * N + n] = equilibrium(i, rr, ub[0], ub[1], ub[2]);
                    s->rho[n] = rr; s->ux[n] = ub[0]; s->uy[n] = ub[1]; s->uz[n] = ub[2];
                    double p[3] = {rr * ub[0], rr * ub[1], rr * ub[2]}, t[3];
                    cross(r, p, t);
                    for (int d = 0; d < 3; ++d) { q->Fc[d] -= p[d]; q->Tc[d] -= t[d]; }
                    s->flag[n] = FLUID;
                }
            }
}

/* LBM::LBM (lbm.cpp:60-94) and Squirmer::init (squirmer.cpp:20-30) */
lbo_state* lbo_create(const lbmgpu_params* p) {
    lbo_state* s = (lbo_state*)calloc(1, sizeof(lbo_state));
    s->NX = p->nx; s->NY = p->ny; s->NZ = p->nz;
    s->N = (size_t)p->nx * p->ny * p->nz;
    s->tau = p->tau;
    s->F[0] = p->fx; s->F[1] = p->fy; s->F[2] = p->fz;
    s->wallsY = p->walls_y; s->wallsZ = p->walls_z;
    s->massCorrectionEvery = p->mass_correction_every;
    s->trajEvery = p->traj_every;
    const size_t N = s->N;
    s->f = (double*)malloc(sizeof(double) * Q * N);
    s->fnew = (double*)malloc(sizeof(double) * Q * N);
    s->rho = (double*)malloc(sizeof(double) * N);
    s->ux = (double*)calloc(N, sizeof(double));
    s->uy = (double*)calloc(N, sizeof(double));
    s->uz = (double*)calloc(N, sizeof(double));
    s->flag = (unsigned char*)malloc(N);
    for (size_t n = 0; n < N; ++n) s->rho[n] = 1.0;

    s->omPlus = 1.0 / s->tau;
    s->omMinus = 1.0 / (0.5 + p->lambda / (s->tau - 0.5));
    s->nu = (s->tau - 0.5) / 3.0;

    for (int z = 0; z < s->NZ; ++z)
        for (int y = 0; y < s->NY; ++y)
            for (int x = 0; x < s->NX; ++x) {
                const int wall = (s->wallsY && (y == 0 || y == s->NY - 1)) ||
                                 (s->wallsZ && (z == 0 || z == s->NZ - 1));
                s->flag[idx(s, x, y, z)] = wall ? WALL : FLUID;
            }
    for (size_t n = 0; n < N; ++n)
        for (int i = 0; i < Q; ++i) s->f[(size_t)i * N + n] = w[i];
    memcpy(s->fnew, s->f, sizeof(double) * Q * N);

    if (p->squirmer) {
        sqm* q = &s->sq;
        s->hasSquirmer = 1;
        q->R = p->radius; q->B1 = p->b1; q->beta = p->beta; q->planar = p->planar;
        q->M = p->rho_p * 4.0 / 3.0 * LBO_PI * q->R * q->R * q->R;
        q->I = 0.4 * q->M * q->R * q->R;
        q->X[0] = p->x0 >= 0 ? p->x0 : 0.5 * (s->NX - 1);
        q->X[1] = p->y0 >= 0 ? p->y0 : 0.5 * (s->NY - 1);
        q->X[2] = p->z0 >= 0 ? p->z0 : 0.5 * (s->NZ - 1);
        if (p->use_orientation) {
            const double n = sqrt(p->ex * p->ex + p->ey * p->ey + p->ez * p->ez);
            q->e[0] = p->ex / n; q->e[1] = p->ey / n; q->e[2] = p->ez / n;
        } else {
            const double a = p->angle * LBO_PI / 180.0;
            q->e[0] = cos(a); q->e[1] = sin(a); q->e[2] = 0.0;
        }
        q->eps = p->eps; q->hc = p->hc; q->hmin = p->hmin;
        q->FS = 6.0 * LBO_PI * s->nu * q->R * (2.0 * q->B1 / 3.0);
        update_particle_flags(s, 1);
    }
    return s;
}

void lbo_destroy(lbo_state* s) {
    if (!s) return;
    free(s->f); free(s->fnew); free(s->rho); free(s->ux); free(s->uy); free(s->uz); free(s->flag);
    free(s);
}

/* LBM::step (lbm.cpp:128-224): moments, TRT + Guo, push streaming, halfway
 * bounce-back with moving-boundary correction, Wen momentum exchange. */
void lbo_step(lbo_state* s) {
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const size_t N = s->N;
    const double omPlus = s->omPlus, omMinus = s->omMinus;
    const double gP = 1.0 - 0.5 * omPlus, gM = 1.0 - 0.5 * omMinus;
    const double Fx = s->F[0], Fy = s->F[1], Fz = s->F[2];
    double FWx = 0, FWy = 0, FWz = 0;
    double FPx = 0, FPy = 0, FPz = 0, TPx = 0, TPy = 0, TPz = 0;
    const double* f = s->f;
    double* fnew = s->fnew;

#pragma omp parallel for collapse(2) schedule(static) reduction(+:FWx,FWy,FWz,FPx,FPy,FPz,TPx,TPy,TPz)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                const size_t n = idx(s, x, y, z);
                if (s->flag[n] != FLUID) continue;
                double fl[Q];
                double r = 0, mx = 0, my = 0, mz = 0;
                for (int i = 0; i < Q; ++i) {
                    fl[i] = f[(size_t)i * N + n];
                    r += fl[i]; mx += cx[i] * fl[i]; my += cy[i] * fl[i]; mz += cz[i] * fl[i];
                }
                const double u = (mx + 0.5 * Fx) / r, v = (my + 0.5 * Fy) / r, wz = (mz + 0.5 * Fz) / r;
                s->rho[n] = r; s->ux[n] = u; s->uy[n] = v; s->uz[n] = wz;
                const double usq = u * u + v * v + wz * wz, uF = u * Fx + v * Fy + wz * Fz;
                for (int i = 0; i < Q; ++i) {
                    const int io = opp[i];
                    const double cu = cx[i] * u + cy[i] * v + cz[i] * wz;
                    const double cF = cx[i] * Fx + cy[i] * Fy + cz[i] * Fz;
                    const double feqP = w[i] * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
                    const double feqM = w[i] * r * 3.0 * cu;
                    const double fP = 0.5 * (fl[i] + fl[io]), fM = 0.5 * (fl[i] - fl[io]);
                    const double SP = w[i] * (9.0 * cu * cF - 3.0 * uF), SM = w[i] * 3.0 * cF;
                    const double fpost = fl[i] - omPlus * (fP - feqP) - omMinus * (fM - feqM) + gP * SP + gM * SM;

                    int xn = x + cx[i], yn = y + cy[i], zn = z + cz[i];
                    if (xn < 0) xn += NX; else if (xn >= NX) xn -= NX;
                    if (yn < 0) yn += NY; else if (yn >= NY) yn -= NY;
                    if (zn < 0) zn += NZ; else if (zn >= NZ) zn -= NZ;
                    const size_t nb = idx(s, xn, yn, zn);
                    const unsigned char t = s->flag[nb];
                    if (t == FLUID) { fnew[(size_t)i * N + nb] = fpost; continue; }

                    double ub[3] = {0, 0, 0}, rb[3] = {0, 0, 0};
                    if (t == PARTICLE) {
                        offset_from_squirmer(s, x + 0.5 * cx[i], y + 0.5 * cy[i], z + 0.5 * cz[i], rb);
                        surface_velocity(&s->sq, rb, ub, 1);
                    }
                    const double cub = cx[i] * ub[0] + cy[i] * ub[1] + cz[i] * ub[2];
                    const double fb = fpost - 6.0 * w[i] * r * cub;
                    fnew[(size_t)io * N + n] = fb;

                    const double sm = fpost + fb, dl = fpost - fb;
                    const double dpx = sm * cx[i] - dl * ub[0];
                    const double dpy = sm * cy[i] - dl * ub[1];
                    const double dpz = sm * cz[i] - dl * ub[2];
                    if (t == WALL) { FWx += dpx; FWy += dpy; FWz += dpz; }
                    else {
                        FPx += dpx; FPy += dpy; FPz += dpz;
                        TPx += rb[1] * dpz - rb[2] * dpy;
                        TPy += rb[2] * dpx - rb[0] * dpz;
                        TPz += rb[0] * dpy - rb[1] * dpx;
                    }
                }
            }
    double* tmp = s->f; s->f = s->fnew; s->fnew = tmp;
    s->wallForce[0] = FWx; s->wallForce[1] = FWy; s->wallForce[2] = FWz;
    if (s->hasSquirmer) {
        s->sq.Fh[0] = FPx; s->sq.Fh[1] = FPy; s->sq.Fh[2] = FPz;
        s->sq.Th[0] = TPx; s->sq.Th[1] = TPy; s->sq.Th[2] = TPz;
    }
}

/* LBM::applyWallPotential (lbm.cpp:231-241) */
static void apply_wall_potential(lbo_state* s) {
    sqm* q = &s->sq;
    q->Fw[0] = q->Fw[1] = q->Fw[2] = 0.0;
    if (s->wallsY) {
        q->Fw[1] += soft_wall_force(q->X[1] - q->R - 0.5, q->eps, q->FS, q->hc);
        q->Fw[1] -= soft_wall_force((s->NY - 1.5) - q->X[1] - q->R, q->eps, q->FS, q->hc);
    }
    if (s->wallsZ) {
        q->Fw[2] += soft_wall_force(q->X[2] - q->R - 0.5, q->eps, q->FS, q->hc);
        q->Fw[2] -= soft_wall_force((s->NZ - 1.5) - q->X[2] - q->R, q->eps, q->FS, q->hc);
    }
}

/* LBM::enforceMinimumGap (lbm.cpp:245-253) */
static void clamp_axis(sqm* q, int d, int Nd) {
    const double lo = 0.5 + q->R + q->hmin, hi = (Nd - 1.5) - q->R - q->hmin;
    if (q->X[d] < lo) { q->X[d] = lo; if (q->U[d] < 0) q->U[d] = 0; ++q->contacts; }
    if (q->X[d] > hi) { q->X[d] = hi; if (q->U[d] > 0) q->U[d] = 0; ++q->contacts; }
}

/* LBM::advanceSquirmer (lbm.cpp:257-263) */
void lbo_advance_squirmer(lbo_state* s) {
    if (!s->hasSquirmer) return;
    apply_wall_potential(s);
    integrate(&s->sq);
    if (s->wallsY) clamp_axis(&s->sq, 1, s->NY);
    if (s->wallsZ) clamp_axis(&s->sq, 2, s->NZ);
    update_particle_flags(s, 0);
}

/* LBM::correctMass (lbm.cpp:324-339) */
void lbo_correct_mass(lbo_state* s) {
    const size_t N = s->N;
    double m = 0; long nf = 0;
#pragma omp parallel for reduction(+:m,nf)
    for (long n = 0; n < (long)N; ++n) {
        if (s->flag[n] != FLUID) continue;
        for (int i = 0; i < Q; ++i) m += s->f[(size_t)i * N + n];
        ++nf;
    }
    if (nf == 0) return;
    const double d = 1.0 - m / nf;
#pragma omp parallel for
    for (long n = 0; n < (long)N; ++n) {
        if (s->flag[n] != FLUID) continue;
        for (int i = 0; i < Q; ++i) s->f[(size_t)i * N + n] += w[i] * d;
    }
}

/* The time-loop body of src/main.cpp:60-64 (no I/O); trajectory rows as in
 * src/utils/io.cpp:79-83. */
int lbo_run(lbo_state* s, int nsteps, double* traj, int max_rows) {
    int rows = 0;
    for (int k = 0; k < nsteps; ++k) {
        const long t = ++s->t;
        lbo_step(s);
        if (s->hasSquirmer) {
            lbo_advance_squirmer(s);
            if (s->massCorrectionEvery > 0 && t % s->massCorrectionEvery == 0) lbo_correct_mass(s);
            if (traj && t % s->trajEvery == 0 && rows < max_rows) {
                const sqm* q = &s->sq;
                double* r = traj + 15 * rows;
                r[0] = (double)t;
                for (int d = 0; d < 3; ++d) {
                    r[1 + d] = q->X[d]; r[4 + d] = q->e[d]; r[7 + d] = q->U[d]; r[10 + d] = q->W[d];
                }
                r[13] = q->Fw[1]; r[14] = q->Fw[2];
                ++rows;
            }
        }
    }
    return rows;
}

long lbo_ncells(const lbo_state* s) { return (long)s->N; }
long lbo_time(const lbo_state* s) { return s->t; }
void lbo_get_f(const lbo_state* s, double* out) { memcpy(out, s->f, sizeof(double) * Q * s->N); }
void lbo_set_f(lbo_state* s, const double* in) { memcpy(s->f, in, sizeof(double) * Q * s->N); }
void lbo_set_flags(lbo_state* s, const unsigned char* flag) { memcpy(s->flag, flag, s->N); }

void lbo_get_fields(const lbo_state* s, unsigned char* flag, double* rho, double* u3) {
    for (size_t n = 0; n < s->N; ++n) {
        if (flag) flag[n] = s->flag[n];
        if (rho) rho[n] = s->rho[n];
        if (u3) { u3[3 * n] = s->ux[n]; u3[3 * n + 1] = s->uy[n]; u3[3 * n + 2] = s->uz[n]; }
    }
}

/* Same layout as ref_squirmer_state in ref_harness.cpp. */
void lbo_squirmer_state(const lbo_state* s, double* o) {
    const sqm* q = &s->sq;
    for (int d = 0; d < 3; ++d) {
        o[d] = q->X[d]; o[3 + d] = q->e[d]; o[6 + d] = q->U[d]; o[9 + d] = q->W[d];
        o[12 + d] = q->Fh[d]; o[15 + d] = q->Th[d]; o[18 + d] = q->Fc[d]; o[21 + d] = q->Tc[d];
        o[24 + d] = q->Fw[d];
    }
    o[27] = (double)q->contacts; o[28] = q->M; o[29] = q->I; o[30] = q->FS;
}

void lbo_set_squirmer_state(lbo_state* s, const double* X, const double* e, const double* U, const double* W) {
    for (int d = 0; d < 3; ++d) { s->sq.X[d] = X[d]; s->sq.e[d] = e[d]; s->sq.U[d] = U[d]; s->sq.W[d] = W[d]; }
}

void lbo_wall_force(const lbo_state* s, double* o) {
    o[0] = s->wallForce[0]; o[1] = s->wallForce[1]; o[2] = s->wallForce[2];
}

/* countFluid, meanDensity, maxSpeed, sumUx (lbm.cpp:342-364) */
void lbo_diag(const lbo_state* s, double* o) {
    long nf = 0; double m = 0, mx = 0, sx = 0;
    for (size_t n = 0; n < s->N; ++n) {
        if (s->flag[n] != FLUID) continue;
        ++nf; m += s->rho[n]; sx += s->ux[n];
        const double sp = sqrt(s->ux[n] * s->ux[n] + s->uy[n] * s->uy[n] + s->uz[n] * s->uz[n]);
        if (sp > mx) mx = sp;
    }
    o[0] = (double)nf; o[1] = nf ? m / nf : 0.0; o[2] = mx; o[3] = sx;
}

/* ductVelocity (analytic.cpp:11-21): series over odd n < 400 */
double lbo_duct_velocity(double y, double z, double a, double b, double G, double mu) {
    double s = 0.0;
    for (int n = 1; n < 400; n += 2) {
        const double k = n * LBO_PI / (2.0 * a), A = k * fabs(z), B = k * b;
        const double ratio = exp(A - B) * (1.0 + exp(-2.0 * A)) / (1.0 + exp(-2.0 * B));
        const double sign = ((n - 1) / 2) % 2 == 0 ? 1.0 : -1.0;
        s += sign * (1.0 - ratio) * cos(k * y) / ((double)n * n * n);
    }
    return 16.0 * a * a * G / (mu * LBO_PI * LBO_PI * LBO_PI) * s;
}

/* poiseuilleError (analytic.cpp:27-60) without the profile files */
double lbo_poiseuille_error(const lbo_state* s) {
    if (!s->wallsY && !s->wallsZ) return -1.0;
    const double mu = s->nu, G = s->F[0];
    const double yc = 0.5 * (s->NY - 1), zc = 0.5 * (s->NZ - 1);
    const double a = 0.5 * (s->NY - 2), b = 0.5 * (s->NZ - 2);
    double num = 0, den = 0;
    for (int z = 0; z < s->NZ; ++z)
        for (int y = 0; y < s->NY; ++y) {
            const size_t n = idx(s, 0, y, z);
            if (s->flag[n] != FLUID) continue;
            double ue;
            if (s->wallsY && s->wallsZ) ue = lbo_duct_velocity(y - yc, z - zc, a, b, G, mu);
            else if (s->wallsY) ue = G / (2.0 * mu) * (a * a - (y - yc) * (y - yc));
            else ue = G / (2.0 * mu) * (b * b - (z - zc) * (z - zc));
            num += (s->ux[n] - ue) * (s->ux[n] - ue);
            den += ue * ue;
        }
    return den > 0 ? sqrt(num / den) : -1.0;
}
