/* artss_oracle.c -- CPU restatement of the ARTSS fractional-step kernels.
 * TEST INFRASTRUCTURE ONLY (see artss_oracle.h).  Serial loops over the
 * reference's index lists, reference expression order, no FMA contraction. */
#include "artss_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

int64_t oracle_size(const oracle_scene *s, int l) { return s->Nx[l] * s->Ny[l] * s->Nz[l]; }

/* DomainBoundary.cpp:42-46 / ObstacleBoundary.cpp:42-48, in program order */
void oracle_apply_bc(const oracle_scene *s, double *f, int level, int ft) {
    const oracle_bc *ops = s->bc[level][ft];
    const int64_t n = s->n_bc[level][ft];
    if (!ops) return;
    for (int64_t q = 0; q < n; q++) f[ops[q].target] = (double) ops[q].sign * f[ops[q].source] + ops[q].value;
}

/* SLAdvect::advect (src/advection/SLAdvect.cpp:34-170) */
void oracle_advect(const oracle_scene *s, double *out, const double *in, const double *u, const double *v,
                   const double *w, double dt, int ft) {
    const int64_t Nx = s->Nx[0], Ny = s->Ny[0];
    const double dtx = dt / s->dx[0], dty = dt / s->dy[0], dtz = dt / s->dz[0];
    const double eps = 1e-6;
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t idx = s->inner[0][l];
        const int64_t k = idx / (Nx * Ny);
        const int64_t j = (idx - k * Nx * Ny) / Nx;
        const int64_t i = idx - k * Nx * Ny - j * Nx;
        const double Ci = dtx * u[idx], Cj = dty * v[idx], Ck = dtz * w[idx];
        int64_t i0 = i, i1 = i, j0 = j, j1 = j, k0 = k, k1 = k;
        double r = 1, sw = 1, t = 1;
        if (Ci > eps) {
            i0 = i - (int64_t) Ci;
            if (i0 < s->i1[0]) i0 = s->i1[0];
            i1 = i0 - 1;
            r = fmod(Ci, 1);
        } else if (Ci < -eps) {
            i0 = i - (int64_t) Ci;
            if (i0 > s->i2[0]) i0 = s->i2[0];
            i1 = i0 + 1;
            r = fmod(-Ci, 1);
        }
        if (Cj > eps) {
            j0 = j - (int64_t) Cj;
            if (j0 < s->j1[0]) j0 = s->j1[0];
            j1 = j0 - 1;
            sw = fmod(Cj, 1);
        } else if (Cj < -eps) {
            j0 = j - (int64_t) Cj;
            if (j0 > s->j2[0]) j0 = s->j2[0];
            j1 = j0 + 1;
            sw = fmod(-Cj, 1);
        }
        if (Ck > eps) {
            k0 = k - (int64_t) Ck;
            if (k0 < s->k1[0]) k0 = s->k1[0];
            k1 = k0 - 1;
            t = fmod(Ck, 1);
        } else if (Ck < -eps) {
            k0 = k - (int64_t) Ck;
            if (k0 > s->k2[0]) k0 = s->k2[0];
            k1 = k0 + 1;
            t = fmod(-Ck, 1);
        }
#define AT(a, b, c) in[(a) + Nx * (b) + Nx * Ny * (c)]
        const double d000 = AT(i0, j0, k0), d100 = AT(i1, j0, k0), d010 = AT(i0, j1, k0), d110 = AT(i1, j1, k0);
        const double d001 = AT(i0, j0, k1), d101 = AT(i1, j0, k1), d011 = AT(i0, j1, k1), d111 = AT(i1, j1, k1);
#undef AT
        const double r100 = d000 + r * (d100 - d000);
        const double r110 = d010 + r * (d110 - d010);
        const double r101 = d001 + r * (d101 - d001);
        const double r111 = d011 + r * (d111 - d011);
        const double s110 = r100 + sw * (r110 - r100);
        const double s111 = r101 + sw * (r111 - r101);
        out[idx] = s110 + t * (s111 - s110);
    }
    oracle_apply_bc(s, out, 0, ft);
}

/* ConstSmagorinsky::calc_turbulent_viscosity (src/turbulence/ConstSmagorinsky.cpp:30-87) */
void oracle_smagorinsky(const oracle_scene *s, double *ev, const double *u, const double *v, const double *w,
                        double cs) {
    const int64_t nj = s->Nx[0], nk = s->Nx[0] * s->Ny[0];
    const double dx = s->dx[0], dy = s->dy[0], dz = s->dz[0];
    const double rdx = 1. / dx, rdy = 1. / dy, rdz = 1. / dz;
    const double delta_s = cbrt(dx * dy * dz);
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t i = s->inner[0][l];
        const double S11 = (u[i + 1] - u[i - 1]) * 0.5 * rdx;
        const double S22 = (v[i + nj] - v[i - nj]) * 0.5 * rdy;
        const double S33 = (w[i + nk] - w[i - nk]) * 0.5 * rdz;
        const double S12 = 0.5 * ((u[i + nj] - u[i - nj]) * 0.5 * rdy + (v[i + 1] - v[i - 1]) * 0.5 * rdx);
        const double S13 = 0.5 * ((u[i + nk] - u[i - nk]) * 0.5 * rdz + (w[i + 1] - w[i - 1]) * 0.5 * rdx);
        const double S23 = 0.5 * ((v[i + nk] - v[i - nk]) * 0.5 * rdz + (w[i + nj] - w[i - nj]) * 0.5 * rdy);
        const double S_bar = sqrt(2. * (S11 * S11 + S22 * S22 + S33 * S33 + 2. * (S12 * S12) + 2. * (S13 * S13) +
                                        2. * (S23 * S23)));
        ev[i] = cs * cs * delta_s * delta_s * S_bar;
    }
    oracle_apply_bc(s, ev, 0, 6);
}

/* IPressure::divergence (src/interfaces/IPressure.cpp:20-110) */
void oracle_divergence(const oracle_scene *s, double *out, const double *u, const double *v, const double *w) {
    const int64_t Nx = s->Nx[0], Ny = s->Ny[0], nj = Nx, nk = Nx * Ny;
    const double rdx = 1. / s->dx[0], rdy = 1. / s->dy[0], rdz = 1. / s->dz[0];
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t i = s->inner[0][l];
        const double a = 0.5 * rdx * (u[i + 1] - u[i - 1]);
        const double b = 0.5 * rdy * (v[i + nj] - v[i - nj]);
        const double c = 0.5 * rdz * (w[i + nk] - w[i - nk]);
        out[i] = a + b + c;
    }
    const int64_t x1 = s->i1[0] - 1, x2 = s->i2[0] + 1, y1 = s->j1[0] - 1, y2 = s->j2[0] + 1;
    const int64_t z1 = s->k1[0] - 1, z2 = s->k2[0] + 1;
    for (int64_t k = z1; k <= z2; k++)
        for (int64_t j = y1; j <= y2; j++)
            for (int64_t i = x1; i <= x2; i++)
                if (i == x1 || i == x2 || j == y1 || j == y2 || k == z1 || k == z2) out[i + Nx * j + Nx * Ny * k] = 0;
}

/* IPressure::projection (src/interfaces/IPressure.cpp:125-172) */
void oracle_projection(const oracle_scene *s, double *u, double *v, double *w, const double *us, const double *vs,
                       const double *ws, const double *p) {
    const int64_t nj = s->Nx[0], nk = s->Nx[0] * s->Ny[0];
    const double rdx = 1. / s->dx[0], rdy = 1. / s->dy[0], rdz = 1. / s->dz[0];
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t i = s->inner[0][l];
        u[i] = us[i] - 0.5 * rdx * (p[i + 1] - p[i - 1]);
        v[i] = vs[i] - 0.5 * rdy * (p[i + nj] - p[i - nj]);
        w[i] = ws[i] - 0.5 * rdz * (p[i + nk] - p[i - nk]);
    }
    oracle_apply_bc(s, u, 0, 1);
    oracle_apply_bc(s, v, 0, 2);
    oracle_apply_bc(s, w, 0, 3);
}

/* ISource::buoyancy_force (src/interfaces/ISource.cpp:26-52) */
void oracle_buoyancy(const oracle_scene *s, double *f, const double *T, const double *Ta, double beta, double g) {
    for (int64_t l = 0; l < s->n_domain[0]; l++) {
        const int64_t i = s->domain[0][l];
        f[i] = -beta * (T[i] - Ta[i]) * g;
    }
}

/* ExplicitEulerSource::add_source (src/source/ExplicitEulerSource.cpp:88-104) */
void oracle_add_source(const oracle_scene *s, double *out, const double *S, double dt, int ft) {
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t i = s->inner[0][l];
        out[i] += dt * S[i];
    }
    oracle_apply_bc(s, out, 0, ft);
}

/* ExplicitDiffuse::ExplicitStep (src/diffusion/ExplicitDiffuse.cpp:50-76, laminar;
 * :79-124, turbulent: face viscosities from EV, no division by the spacing,
 * as the reference writes it) + DomainController::apply_boundary (:28, :45) */
void oracle_diffuse_explicit(const oracle_scene *s, double *out, const double *in, double D, const double *ev,
                             double dt, int ft) {
    const int64_t ni = 1, nj = s->Nx[0], nk = s->Nx[0] * s->Ny[0];
    const double rdx = D / (s->dx[0] * s->dx[0]), rdy = D / (s->dy[0] * s->dy[0]), rdz = D / (s->dz[0] * s->dz[0]);
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t q = s->inner[0][l];
        if (!ev) {
            out[q] = in[q] + dt * ((in[q + ni] - 2 * in[q] + in[q - ni]) * rdx + (in[q + nj] - 2 * in[q] + in[q - nj]) * rdy +
                                   (in[q + nk] - 2 * in[q] + in[q - nk]) * rdz);
        } else {
            const double nu_x1 = 0.5 * (ev[q + ni] + ev[q]) + D, nu_x2 = 0.5 * (ev[q - ni] + ev[q]) + D;
            const double nu_y1 = 0.5 * (ev[q + nj] + ev[q]) + D, nu_y2 = 0.5 * (ev[q - nj] + ev[q]) + D;
            const double nu_z1 = 0.5 * (ev[q + nk] + ev[q]) + D, nu_z2 = 0.5 * (ev[q - nk] + ev[q]) + D;
            const double di0 = in[q] - in[q - ni], di1 = in[q + ni] - in[q];
            const double dj0 = in[q] - in[q - nj], dj1 = in[q + nj] - in[q];
            const double dk0 = in[q] - in[q - nk], dk1 = in[q + nk] - in[q];
            out[q] = in[q] + dt * ((nu_x1 * di0 - nu_x2 * di1) + (nu_y1 * dj0 - nu_y2 * dj1) + (nu_z1 * dk0 - nu_z2 * dk1));
        }
    }
    oracle_apply_bc(s, out, 0, ft);
}

/* ISource::dissipate (src/interfaces/ISource.cpp:63-123) */
void oracle_dissipate(const oracle_scene *s, double *out, const double *u, const double *v, const double *w,
                      double nu, double dt, int ft) {
    const int64_t ni = 1, nj = s->Nx[0], nk = s->Nx[0] * s->Ny[0];
    const double rdx = 1. / s->dx[0], rdy = 1. / s->dy[0], rdz = 1. / s->dz[0];
    for (int64_t l = 0; l < s->n_inner[0]; l++) {
        const int64_t i = s->inner[0][l];
        const double out_h = nu * (2 * (0.5 * rdx * (u[i + ni] - u[i - ni])) * (0.5 * rdx * (u[i + ni] - u[i - ni])) +
                                   2 * (0.5 * rdy * (v[i + nj] - v[i - nj])) * (0.5 * rdy * (v[i + nj] - v[i - nj])) +
                                   2 * (0.5 * rdz * (w[i + nk] - w[i - nk])) * (0.5 * rdz * (w[i + nk] - w[i - nk])) +
                                   ((0.5 * rdx * (v[i + ni] - v[i - ni])) + (0.5 * rdy * (u[i + nj] - u[i - nj]))) *
                                       ((0.5 * rdx * (v[i + ni] - v[i - ni])) + (0.5 * rdy * (u[i + nj] - u[i - nj]))) +
                                   ((0.5 * rdy * (w[i + nj] - w[i - nj])) + (0.5 * rdz * (v[i + nk] - v[i - nk]))) *
                                       ((0.5 * rdy * (w[i + nj] - w[i - nj])) + (0.5 * rdz * (v[i + nk] - v[i - nk]))) +
                                   ((0.5 * rdz * (u[i + nk] - u[i - nk])) + (0.5 * rdx * (w[i + ni] - w[i - ni]))) *
                                       ((0.5 * rdz * (u[i + nk] - u[i - nk])) + (0.5 * rdx * (w[i + ni] - w[i - ni]))));
        out[i] += dt * out_h;
    }
    oracle_apply_bc(s, out, 0, ft);
}

/* ------------------------------------------------------------------ diffusion */

static void parity(const oracle_scene *s, int level, int64_t idx, int *color) {
    const int64_t Nx = s->Nx[level], Ny = s->Ny[level];
    const int64_t k = idx / (Nx * Ny), j = (idx - k * Nx * Ny) / Nx, i = idx - k * Nx * Ny - j * Nx;
    *color = (int) ((i + j + k) % 2);
}

/* colored_gauss_seidel_stencil (src/diffusion/ColoredGaussSeidelDiffuse.cpp:316-341) */
static void cgs_stencil(int64_t q, double *out, const double *b, double ax, double ay, double az, double dsign,
                        double beta, double w, int64_t nj, int64_t nk) {
    const double xp = out[q + 1], xm = out[q - 1], yp = out[q + nj], ym = out[q - nj], zp = out[q + nk],
                 zm = out[q - nk];
    const double r_out = out[q];
    const double out_h = beta * (dsign * b[q] + ax * (xp + xm) + ay * (yp + ym) + az * (zp + zm));
    out[q] = (1 - w) * r_out + w * out_h;
}

/* one red (even i+j+k) then black sweep over a level's inner list
 * (ColoredGaussSeidelDiffuse.cpp:190-295, lists :343-372) */
static void cgs_step(const oracle_scene *s, int level, double *out, const double *b, double ax, double ay,
                     double az, double beta, double dsign, double w, const double *ev, double D, double dt) {
    const int64_t nj = s->Nx[level], nk = s->Nx[level] * s->Ny[level];
    const double rdx = 1. / s->dx[level], rdy = 1. / s->dy[level], rdz = 1. / s->dz[level];
    for (int color = 0; color < 2; color++) {
        for (int64_t l = 0; l < s->n_inner[level]; l++) {
            const int64_t q = s->inner[level][l];
            int c;
            parity(s, level, q, &c);
            if (c != color) continue;
            if (ev) {
                const double aX = (D + ev[q]) * dt * rdx * rdx;
                const double aY = (D + ev[q]) * dt * rdy * rdy;
                const double aZ = (D + ev[q]) * dt * rdz * rdz;
                const double rb = (1. + 2. * (aX + aY + aZ));
                cgs_stencil(q, out, b, aX, aY, aZ, dsign, 1. / rb, w, nj, nk);
            } else {
                cgs_stencil(q, out, b, ax, ay, az, dsign, beta, w, nj, nk);
            }
        }
    }
}

/* ColoredGaussSeidelDiffuse::diffuse (src/diffusion/ColoredGaussSeidelDiffuse.cpp:38-173) */
int64_t oracle_diffuse_cgs(const oracle_scene *s, double *out, double *in, const double *b, double D,
                           const double *ev, double dt, int ft, int64_t max_iter, double tol, double w,
                           double *residual) {
    const int64_t n = oracle_size(s, 0);
    memcpy(out, in, n * sizeof(double));
    const double rdx = 1. / s->dx[0], rdy = 1. / s->dy[0], rdz = 1. / s->dz[0];
    const double ax = D * dt * rdx * rdx, ay = D * dt * rdy * rdy, az = D * dt * rdz * rdz;
    const double rbeta = (1. + 2. * (ax + ay + az));
    const double beta = 1. / rbeta;
    int64_t it = 0;
    double res = 1.;
    while (res > tol && it < max_iter) {
        memcpy(in, out, n * sizeof(double));
        cgs_step(s, 0, out, b, ax, ay, az, beta, 1.0, w, ev, D, dt);
        oracle_apply_bc(s, out, 0, ft);
        double sum = 0;
        for (int64_t l = 0; l < s->n_inner[0]; l++) {
            const int64_t q = s->inner[0][l];
            double rb = rbeta;
            if (ev) {
                const double aX = (D + ev[q]) * dt * rdx * rdx;
                const double aY = (D + ev[q]) * dt * rdy * rdy;
                const double aZ = (D + ev[q]) * dt * rdz * rdz;
                rb = (1. + 2. * (aX + aY + aZ));
            }
            const double r = rb * (out[q] - in[q]);
            sum += r * r;
        }
        res = sqrt(sum);
        it++;
    }
    if (residual) *residual = res;
    return it;
}

/* JacobiDiffuse::diffuse (src/diffusion/JacobiDiffuse.cpp:31-203) with the
 * JacobiStep variants of :222-254 (laminar, divides by reciprocal_beta) and
 * :320-367 (turbulent) */
int64_t oracle_diffuse_jacobi(const oracle_scene *s, double *out, double *in, const double *b, double D,
                              const double *ev, double dt, int ft, int64_t max_iter, double tol, double w,
                              double *residual) {
    const int64_t nj = s->Nx[0], nk = s->Nx[0] * s->Ny[0];
    const double rdx = 1. / s->dx[0], rdy = 1. / s->dy[0], rdz = 1. / s->dz[0];
    const double ax = D * dt * rdx * rdx, ay = D * dt * rdy * rdy, az = D * dt * rdz * rdz;
    const double rbeta = (1. + 2. * (ax + ay + az));
    const double dsign = 1.;
    int64_t it = 0;
    double res = 1.;
    while (res > tol && it < max_iter) {
        for (int64_t l = 0; l < s->n_inner[0]; l++) {
            const int64_t i = s->inner[0][l];
            double out_h;
            if (ev) {
                const double aX = (D + ev[i]) * dt * rdx * rdx;
                const double aY = (D + ev[i]) * dt * rdy * rdy;
                const double aZ = (D + ev[i]) * dt * rdz * rdz;
                const double rb = (1. + 2. * (aX + aY + aZ));
                const double bb = 1. / rb;
                const double d_aX = aX * (in[i + 1] + in[i - 1]);
                const double d_aY = aY * (in[i + nj] + in[i - nj]);
                const double d_aZ = aZ * (in[i + nk] + in[i - nk]);
                out_h = bb * (dsign * b[i] + d_aX + d_aY + d_aZ);
            } else {
                out_h = (dsign * b[i] + ax * (in[i + 1] + in[i - 1]) + ay * (in[i + nj] + in[i - nj]) +
                         az * (in[i + nk] + in[i - nk])) / rbeta;
            }
            out[i] = (1 - w) * in[i] + w * out_h;
        }
        oracle_apply_bc(s, out, 0, ft);
        double sum = 0;
        for (int64_t l = 0; l < s->n_inner[0]; l++) {
            const int64_t i = s->inner[0][l];
            double rb = rbeta;
            if (ev) {
                const double aX = (D + ev[i]) * dt * rdx * rdx;
                const double aY = (D + ev[i]) * dt * rdy * rdy;
                const double aZ = (D + ev[i]) * dt * rdz * rdz;
                rb = (1. + 2. * (aX + aY + aZ));
            }
            const double r = rb * (out[i] - in[i]);
            sum += r * r;
        }
        res = sqrt(sum);
        it++;
        for (int64_t l = 0; l < s->n_domain[0]; l++) in[s->domain[0][l]] = out[s->domain[0][l]];
    }
    if (residual) *residual = res;
    return it;
}

/* ------------------------------------------------------------------ VCycleMG */

struct oracle_mg {
    const oracle_scene *s;
    oracle_mg_cfg cfg;
    double *r0[ORACLE_MAX_LEVEL + 1], *r1[ORACLE_MAX_LEVEL + 1], *e0[ORACLE_MAX_LEVEL + 1];
    double *e1[ORACLE_MAX_LEVEL + 1], *tmp[ORACLE_MAX_LEVEL + 1];
    int64_t last_coarse_it;  /* sweeps of the last coarse solve */
};

static double *zeros(const oracle_scene *s, int l) { return (double *) calloc((size_t) oracle_size(s, l), sizeof(double)); }

/* VCycleMG::VCycleMG field allocation (src/pressure/VCycleMG.cpp:51-99) */
oracle_mg *oracle_mg_create(const oracle_scene *s, const oracle_mg_cfg *cfg) {
    oracle_mg *mg = (oracle_mg *) calloc(1, sizeof(oracle_mg));
    mg->s = s;
    mg->cfg = *cfg;
    mg->r1[0] = zeros(s, 0);
    mg->e1[0] = zeros(s, 0);
    mg->tmp[0] = zeros(s, 0);
    for (int l = 0; l < cfg->n_level; l++) {
        mg->r0[l] = zeros(s, l);
        mg->r1[l + 1] = zeros(s, l + 1);
        mg->e0[l] = zeros(s, l);
        mg->e1[l + 1] = zeros(s, l + 1);
        mg->tmp[l + 1] = zeros(s, l + 1);
    }
    return mg;
}

void oracle_mg_destroy(oracle_mg *mg) {
    if (!mg) return;
    for (int l = 0; l <= ORACLE_MAX_LEVEL; l++) {
        free(mg->r0[l]);
        free(mg->r1[l]);
        free(mg->e0[l]);
        free(mg->e1[l]);
        free(mg->tmp[l]);
    }
    free(mg);
}

static void mg_alphas(const oracle_scene *s, int l, double *ax, double *ay, double *az, double *beta) {
    *ax = 1. / (s->dx[l] * s->dx[l]);
    *ay = 1. / (s->dy[l] * s->dy[l]);
    *az = 1. / (s->dz[l] * s->dz[l]);
    const double rbeta = 2. * (*ax + *ay + *az);
    *beta = 1. / rbeta;
}

/* JacobiDiffuse::JacobiStep, multigrid variant (src/diffusion/JacobiDiffuse.cpp:274-305) */
static void mg_jacobi_step(const oracle_scene *s, int l, double *out, const double *in, const double *b,
                           double ax, double ay, double az, double beta, double dsign, double w) {
    const int64_t nj = s->Nx[l], nk = s->Nx[l] * s->Ny[l];
    for (int64_t q = 0; q < s->n_inner[l]; q++) {
        const int64_t i = s->inner[l][q];
        const double out_h = beta * (dsign * b[i] + ax * (in[i + 1] + in[i - 1]) + ay * (in[i + nj] + in[i - nj]) +
                                     az * (in[i + nk] + in[i - nk]));
        out[i] = (1 - w) * in[i] + w * out_h;
    }
}

/* ||b - A x||_2 on a level's inner list (VCycleMG.cpp:186-194, :668-679, :777-788) */
static double mg_resnorm(const oracle_scene *s, int l, const double *x, const double *b) {
    const int64_t nj = s->Nx[l], nk = s->Nx[l] * s->Ny[l];
    const double rx = 1. / (s->dx[l] * s->dx[l]), ry = 1. / (s->dy[l] * s->dy[l]), rz = 1. / (s->dz[l] * s->dz[l]);
    double sum = 0.;
    for (int64_t q = 0; q < s->n_inner[l]; q++) {
        const int64_t i = s->inner[l][q];
        const double r = b[i] - (rx * (x[i - 1] - 2 * x[i] + x[i + 1]) + ry * (x[i - nj] - 2 * x[i] + x[i + nj]) +
                                 rz * (x[i - nk] - 2 * x[i] + x[i + nk]));
        sum += r * r;
    }
    return sqrt(sum);
}

/* VCycleMG::Smooth + call_smooth_* (VCycleMG.cpp:299-305, :583-723) */
static void mg_smooth(oracle_mg *mg, double *out, double *tmp, const double *b, int l) {
    const oracle_scene *s = mg->s;
    double ax, ay, az, beta;
    mg_alphas(s, l, &ax, &ay, &az, &beta);
    oracle_apply_bc(s, out, l, 4);
    oracle_apply_bc(s, out, l, 4);
    if (mg->cfg.smoother == 1) {
        for (int r = 0; r < mg->cfg.n_relax; r++) {
            cgs_step(s, l, out, b, ax, ay, az, beta, -1., mg->cfg.smoother_w, NULL, 0, 0);
            oracle_apply_bc(s, out, l, 4);
        }
        return;
    }
    memcpy(tmp, out, (size_t) oracle_size(s, l) * sizeof(double));
    double *A = out, *B = tmp;  /* Field::swap exchanges these after every sweep */
    for (int r = 0; r < mg->cfg.n_relax; r++) {
        mg_jacobi_step(s, l, A, B, b, ax, ay, az, beta, -1., mg->cfg.smoother_w);
        oracle_apply_bc(s, A, l, 4);
        double *t = A;
        A = B;
        B = t;
    }
}

/* VCycleMG::Solve + call_solve_* (VCycleMG.cpp:562-581, :620-798) */
static void mg_solve(oracle_mg *mg, double *out, double *tmp, const double *b, int l) {
    const oracle_scene *s = mg->s;
    if (s->Nx[l] <= 4 && s->Ny[l] <= 4) {
        mg_smooth(mg, out, tmp, b, l);
        return;
    }
    double ax, ay, az, beta;
    mg_alphas(s, l, &ax, &ay, &az, &beta);
    oracle_apply_bc(s, out, l, 4);
    int64_t it = 0;
    double res = 10000.;
    if (mg->cfg.smoother == 1) {
        while (res > mg->cfg.smoother_tol_res && it < mg->cfg.smoother_max_iter) {
            cgs_step(s, l, out, b, ax, ay, az, beta, -1., mg->cfg.smoother_w, NULL, 0, 0);
            oracle_apply_bc(s, out, l, 4);
            res = mg_resnorm(s, l, out, b);
            it++;
        }
        mg->last_coarse_it = it;
        return;
    }
    memcpy(tmp, out, (size_t) oracle_size(s, l) * sizeof(double));
    double *A = out, *B = tmp;
    while (res > mg->cfg.smoother_tol_res && it < mg->cfg.smoother_max_iter) {
        mg_jacobi_step(s, l, A, B, b, ax, ay, az, beta, -1., mg->cfg.smoother_w);
        oracle_apply_bc(s, A, l, 4);
        res = mg_resnorm(s, l, A, b);
        double *t = A;
        A = B;
        B = t;
        it++;
    }
    mg->last_coarse_it = it;
}

/* VCycleMG::VCycleMultigrid (VCycleMG.cpp:215-288) with Residuum :319-360,
 * Restrict :370-427 and Prolongate :437-551 */
static void mg_vcycle(oracle_mg *mg, double *out) {
    const oracle_scene *s = mg->s;
    const int L = mg->cfg.n_level;
    if (L == 0) {
        mg_solve(mg, out, mg->tmp[0], mg->r1[0], 0);
        return;
    }
    memcpy(mg->e1[0], out, (size_t) oracle_size(s, 0) * sizeof(double));
    for (int l = 0; l < L; l++) {
        mg_smooth(mg, mg->e1[l], mg->tmp[l], mg->r1[l], l);
        {   /* Residuum */
            const int64_t nj = s->Nx[l], nk = s->Nx[l] * s->Ny[l];
            const double rx = 1. / (s->dx[l] * s->dx[l]), ry = 1. / (s->dy[l] * s->dy[l]);
            const double rz = 1. / (s->dz[l] * s->dz[l]);
            const double *in = mg->e1[l], *b = mg->r1[l];
            double *o = mg->r0[l];
            for (int64_t q = 0; q < s->n_inner[l]; q++) {
                const int64_t i = s->inner[l][q];
                const double weighted = (rx * (in[i - 1] - 2 * in[i] + in[i + 1]) + ry * (in[i - nj] - 2 * in[i] + in[i + nj]) +
                                         rz * (in[i - nk] - 2 * in[i] + in[i + nk]));
                o[i] = b[i] - weighted;
            }
        }
        oracle_apply_bc(s, mg->r0[l], l, 4);
        {   /* Restrict to level l+1 */
            const int c = l + 1;
            const int64_t Nxc = s->Nx[c], Nyc = s->Ny[c], Nxf = s->Nx[l], Nyf = s->Ny[l];
            const double *in = mg->r0[l];
            double *o = mg->r1[c];
            for (int64_t q = 0; q < s->n_inner[c]; q++) {
                const int64_t idx = s->inner[c][q];
                const int64_t k = idx / (Nxc * Nyc), j = (idx - k * Nxc * Nyc) / Nxc, i = idx - k * Nxc * Nyc - j * Nxc;
#define F(a, b2, c2) in[(a) + Nxf * (b2) + Nxf * Nyf * (c2)]
                o[idx] = 0.125 * (F(2 * i - 1, 2 * j - 1, 2 * k - 1) + F(2 * i, 2 * j - 1, 2 * k - 1) +
                                  F(2 * i - 1, 2 * j, 2 * k - 1) + F(2 * i, 2 * j, 2 * k - 1) +
                                  F(2 * i - 1, 2 * j - 1, 2 * k) + F(2 * i, 2 * j - 1, 2 * k) +
                                  F(2 * i - 1, 2 * j, 2 * k) + F(2 * i, 2 * j, 2 * k));
#undef F
            }
        }
        oracle_apply_bc(s, mg->r1[l + 1], l + 1, 4);
        memset(mg->e1[l + 1], 0, (size_t) oracle_size(s, l + 1) * sizeof(double));
    }
    memcpy(out, mg->e0[0], (size_t) oracle_size(s, 0) * sizeof(double));
    for (int l = L; l > 0; l--) {
        {   /* Prolongate level l -> l-1 */
            const int64_t Nxc = s->Nx[l], Nyc = s->Ny[l], Nxf = s->Nx[l - 1], Nyf = s->Ny[l - 1];
            const int64_t ni = 1, nj = Nxc, nk = Nxc * Nyc;
            const double *in = mg->e1[l];
            double *o = mg->e0[l - 1];
            for (int64_t q = 0; q < s->n_inner[l]; q++) {
                const int64_t idx = s->inner[l][q];
                const int64_t k = idx / (Nxc * Nyc), j = (idx - k * Nxc * Nyc) / Nxc, i = idx - k * Nxc * Nyc - j * Nxc;
                for (int c = 0; c < 8; c++) {
                    const int sx = (c & 4) ? -1 : 1, sy = (c & 2) ? -1 : 1, sz = (c & 1) ? -1 : 1;
                    const int64_t fi = sx > 0 ? 2 * i : 2 * i - 1, fj = sy > 0 ? 2 * j : 2 * j - 1;
                    const int64_t fk = sz > 0 ? 2 * k : 2 * k - 1;
                    o[fi + Nxf * fj + Nxf * Nyf * fk] =
                        0.015625 * (27 * in[idx] + 9 * in[idx + sx * ni] + 9 * in[idx + sy * nj] + 9 * in[idx + sz * nk] +
                                    3 * in[idx + sx * ni + sy * nj] + 3 * in[idx + sx * ni + sz * nk] +
                                    3 * in[idx + sy * nj + sz * nk] + in[idx + sx * ni + sy * nj + sz * nk]);
                }
            }
        }
        oracle_apply_bc(s, mg->e0[l - 1], l - 1, 4);
        {
            const int64_t n = oracle_size(s, l - 1);
            for (int64_t q = 0; q < n; q++) mg->e1[l - 1][q] += mg->e0[l - 1][q];
        }
        if (l == L) mg_solve(mg, mg->e1[l - 1], mg->tmp[l - 1], mg->r1[l - 1], l - 1);
        else mg_smooth(mg, mg->e1[l - 1], mg->tmp[l - 1], mg->r1[l - 1], l - 1);
    }
    memcpy(out, mg->e1[0], (size_t) oracle_size(s, 0) * sizeof(double));
    oracle_apply_bc(s, out, 0, 4);
}

/* VCycleMG::pressure (src/pressure/VCycleMG.cpp:142-207) */
int64_t oracle_mg_pressure(oracle_mg *mg, double *p, const double *rhs, int first_step, double *residual) {
    const oracle_scene *s = mg->s;
    const size_t n = (size_t) oracle_size(s, 0) * sizeof(double);
    memcpy(mg->e1[0], p, n);
    memcpy(mg->tmp[0], p, n);
    memcpy(mg->r1[0], rhs, n);
    int64_t cycles = 0;
    double r = -1;
    if (first_step) {
        int64_t set_relax = mg->cfg.n_relax;
        r = 10000.;
        while (r > mg->cfg.tol_res && cycles < mg->cfg.max_cycle && set_relax < mg->cfg.smoother_max_iter) {
            for (int c = 0; c < mg->cfg.n_cycle; c++) {
                mg_vcycle(mg, p);
                cycles++;
            }
            r = mg_resnorm(s, 0, p, rhs);
            set_relax += mg->cfg.n_relax;
        }
    } else {
        for (int c = 0; c < mg->cfg.n_cycle; c++) {
            mg_vcycle(mg, p);
            cycles++;
        }
    }
    if (residual) *residual = r;
    return cycles;
}

int64_t oracle_mg_last_coarse_iterations(const oracle_mg *mg) { return mg->last_coarse_it; }

/* DynamicSmagorinsky::explicit_filtering (src/turbulence/DynamicSmagorinsky.cpp:393-427):
 * trapezoidal 3x3x3 weights, x offset outermost, z innermost */
static void ds_filter(const oracle_scene *s, double *out, const double *in) {
    const int64_t Nx = s->Nx[0], Ny = s->Ny[0];
    const double a[3] = {1. / 4., 1. / 2., 1. / 4.};
    for (int64_t j = 0; j < s->n_inner[0]; j++) {
        const int64_t i = s->inner[0][j];
        double sum = 0;
        for (int64_t l = 0; l < 3; l++)
            for (int64_t m = 0; m < 3; m++)
                for (int64_t n = 0; n < 3; n++)
                    sum = sum + a[l] * a[m] * a[n] * in[i - 1 + l + Nx * (m - 1) + Nx * Ny * (n - 1)];
        out[i] = sum;
    }
}

void oracle_dynamic_smagorinsky(const oracle_scene *s, double *ev, const double *u, const double *v, const double *w,
                                double nu) {
    enum { UF, VF, WF, UU, VV, WW, UV, UW, VW, UUF, VVF, WWF, UVF, UWF, VWF, UFUF, VFVF, WFWF, UFVF, UFWF, VFWF,
           L11, L22, L33, L12, L13, L23, S11, S22, S33, S12, S13, S23, S11F, S22F, S33F, S12F, S13F, S23F,
           P11, P22, P33, P12, P13, P23, P11F, P22F, P33F, P12F, P13F, P23F, M11, M22, M33, M12, M13, M23,
           SBAR, SBARF, CS, NARR };
    const int64_t Nx = s->Nx[0], Ny = s->Ny[0], N = Nx * Ny * s->Nz[0];
    double *f[NARR];
    for (int a = 0; a < NARR; a++) f[a] = (double *) calloc((size_t) N, sizeof(double));
    const double dx = s->dx[0], dy = s->dy[0], dz = s->dz[0];
    const double rdx = 1. / dx, rdy = 1. / dy, rdz = 1. / dz;
    const double alpha = 2.0;
    const double delta_s = cbrt(dx * dy * dz);
    const int64_t n_in = s->n_inner[0];
    const int64_t *lst = s->inner[0];
    ds_filter(s, f[UF], u);
    ds_filter(s, f[VF], v);
    ds_filter(s, f[WF], w);
    for (int64_t j = 0; j < n_in; j++) {
        const int64_t i = lst[j];
        f[UU][i] = f[UF][i] * f[UF][i];
        f[VV][i] = f[VF][i] * f[VF][i];
        f[WW][i] = f[WF][i] * f[WF][i];
        f[UV][i] = f[UF][i] * f[VF][i];
        f[UW][i] = f[UF][i] * f[WF][i];
        f[VW][i] = f[VF][i] * f[WF][i];
        f[UFUF][i] = f[UF][i] * f[UF][i];
        f[VFVF][i] = f[VF][i] * f[VF][i];
        f[WFWF][i] = f[WF][i] * f[WF][i];
        f[UFVF][i] = f[UF][i] * f[VF][i];
        f[UFWF][i] = f[UF][i] * f[WF][i];
        f[VFWF][i] = f[VF][i] * f[WF][i];
    }
    /* the reference filters ww twice and never uw (uw_f keeps its zeros) */
    ds_filter(s, f[UUF], f[UU]);
    ds_filter(s, f[VVF], f[VV]);
    ds_filter(s, f[WWF], f[WW]);
    ds_filter(s, f[UVF], f[UV]);
    ds_filter(s, f[VWF], f[VW]);
    ds_filter(s, f[WWF], f[WW]);
    const double *uf = f[UF], *vf = f[VF], *wf = f[WF];
    for (int64_t j = 0; j < n_in; j++) {
        const int64_t i = lst[j];
        f[L11][i] = f[UUF][i] - f[UFUF][i];
        f[L22][i] = f[VVF][i] - f[VFVF][i];
        f[L33][i] = f[WWF][i] - f[WFWF][i];
        f[L12][i] = f[UVF][i] - f[UFVF][i];
        f[L13][i] = f[UWF][i] - f[UFWF][i];
        f[L23][i] = f[VWF][i] - f[VFWF][i];
        f[S11][i] = (uf[i + 1] - uf[i - 1]) * 0.5 * rdx;
        f[S22][i] = (vf[i + Nx] - vf[i - Nx]) * 0.5 * rdy;
        f[S33][i] = (wf[i + Nx * Ny] - wf[i - Nx * Ny]) * 0.5 * rdz;
        f[S12][i] = 0.5 * ((uf[i + Nx] - uf[i - Nx]) * 0.5 * rdy + (vf[i + 1] - vf[i - 1]) * 0.5 * rdx);
        f[S13][i] = 0.5 * ((uf[i + Nx * Ny] - uf[i - Nx * Ny]) * 0.5 * rdz + (wf[i + 1] - wf[i - 1]) * 0.5 * rdx);
        f[S23][i] = 0.5 * ((vf[i + Nx * Ny] - vf[i - Nx * Ny]) * 0.5 * rdz + (wf[i + Nx] - wf[i - Nx]) * 0.5 * rdy);
        f[SBAR][i] = sqrt(2. * (f[S11][i] * f[S11][i] + f[S22][i] * f[S22][i] + f[S33][i] * f[S33][i] +
                                2. * (f[S12][i] * f[S12][i]) + 2. * (f[S13][i] * f[S13][i]) +
                                2. * (f[S23][i] * f[S23][i])));
        f[P11][i] = f[SBAR][i] * f[S11][i];
        f[P22][i] = f[SBAR][i] * f[S22][i];
        f[P33][i] = f[SBAR][i] * f[S33][i];
        f[P12][i] = f[SBAR][i] * f[S12][i];
        f[P13][i] = f[SBAR][i] * f[S13][i];
        f[P23][i] = f[SBAR][i] * f[S23][i];
    }
    for (int a = 0; a < 6; a++) ds_filter(s, f[S11F + a], f[S11 + a]);
    for (int a = 0; a < 6; a++) ds_filter(s, f[P11F + a], f[P11 + a]);
    double *Cs = f[CS];
    for (int64_t j = 0; j < n_in; j++) {
        const int64_t i = lst[j];
        f[SBARF][i] = sqrt(2. * (f[S11F][i] * f[S11F][i] + f[S22F][i] * f[S22F][i] + f[S33F][i] * f[S33F][i] +
                                 2. * (f[S12F][i] * f[S12F][i]) + 2. * (f[S13F][i] * f[S13F][i]) +
                                 2. * (f[S23F][i] * f[S23F][i])));
        for (int a = 0; a < 6; a++)
            f[M11 + a][i] = 2.0 * delta_s * delta_s * (f[P11F + a][i] - alpha * alpha * f[SBARF][i] * f[S11F + a][i]);
        /* the reference's products (not sums) of the 22 and 33 terms, kept */
        const double num = f[L11][i] * f[M11][i] + f[L22][i] * f[M22][i] * f[L33][i] * f[M33][i] +
                           2.0 * f[L12][i] * f[M12][i] + 2.0 * f[L13][i] * f[M13][i] + 2.0 * f[L23][i] * f[M23][i];
        const double den = f[M11][i] * f[M11][i] + f[M22][i] * f[M22][i] * f[M33][i] * f[M33][i] +
                           2.0 * f[M12][i] * f[M12][i] + 2.0 * f[M13][i] * f[M13][i] + 2.0 * f[M23][i] * f[M23][i];
        Cs[i] = num / den;
    }
    /* local averaging in place, in list order (earlier cells already averaged) */
    for (int64_t j = 0; j < n_in; j++) {
        const int64_t i = lst[j];
        double sum = 0;
        for (int64_t l = 0; l < 3; l++)
            for (int64_t m = 0; m < 3; m++)
                for (int64_t n = 0; n < 3; n++) sum = sum + Cs[i - 1 + l + Nx * (m - 1) + Nx * Ny * (n - 1)];
        Cs[i] = sum / 27.0;
        ev[i] = 2.0 * Cs[i] * delta_s * delta_s * f[SBAR][i];
    }
    for (int64_t j = 0; j < n_in; j++) {
        const int64_t i = lst[j];
        if ((ev[i] + nu) < 0) ev[i] = 0;
    }
    for (int a = 0; a < NARR; a++) free(f[a]);
}
