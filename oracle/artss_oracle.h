/* artss_oracle.h -- CPU restatement of the ARTSS fractional-step kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the B200 path is compared
 * against: tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py may call it; nothing under artss_b200/ links or runs it.
 *
 * Each function restates one reference routine in plain C, serially, in the
 * reference's loop order and expression order (compiled with
 * -ffp-contract=off); the citation is the ARTSS source file:line it follows.
 * Cell sets are the reference's index lists (ascending linear indices
 * i + Nx*j + Nx*Ny*k).  Pinned against the reference serial build
 * (oracle/_ref) by tests/test_oracle.py: full NSTempTurb timesteps agree bit
 * for bit with the reference's dumped fields.
 */
#ifndef ARTSS_ORACLE_H
#define ARTSS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_LEVEL 8

/* x[target] = sign * x[source] + value, in order (DomainBoundary.cpp:42-46) */
typedef struct {
    int64_t target;
    int64_t source;
    double value;
    int32_t sign;
    int32_t reserved;
} oracle_bc;

typedef struct {
    int32_t levels;
    int64_t Nx[ORACLE_MAX_LEVEL + 1], Ny[ORACLE_MAX_LEVEL + 1], Nz[ORACLE_MAX_LEVEL + 1];
    int64_t i1[ORACLE_MAX_LEVEL + 1], i2[ORACLE_MAX_LEVEL + 1];
    int64_t j1[ORACLE_MAX_LEVEL + 1], j2[ORACLE_MAX_LEVEL + 1];
    int64_t k1[ORACLE_MAX_LEVEL + 1], k2[ORACLE_MAX_LEVEL + 1];
    double dx[ORACLE_MAX_LEVEL + 1], dy[ORACLE_MAX_LEVEL + 1], dz[ORACLE_MAX_LEVEL + 1];
    const int64_t *inner[ORACLE_MAX_LEVEL + 1];
    int64_t n_inner[ORACLE_MAX_LEVEL + 1];
    const int64_t *domain[ORACLE_MAX_LEVEL + 1];
    int64_t n_domain[ORACLE_MAX_LEVEL + 1];
    const oracle_bc *bc[ORACLE_MAX_LEVEL + 1][7];   /* per level and field type, NULL: none */
    int64_t n_bc[ORACLE_MAX_LEVEL + 1][7];
} oracle_scene;

typedef struct {
    int32_t n_level, n_cycle, max_cycle, n_relax;
    double tol_res;
    int32_t smoother;  /* 0 Jacobi, 1 colored Gauss-Seidel */
    int32_t reserved;
    int64_t smoother_max_iter;
    double smoother_tol_res, smoother_w;
} oracle_mg_cfg;

int64_t oracle_size(const oracle_scene *s, int level);

void oracle_apply_bc(const oracle_scene *s, double *f, int level, int field_type);

void oracle_advect(const oracle_scene *s, double *out, const double *in, const double *u, const double *v,
                   const double *w, double dt, int field_type);
void oracle_smagorinsky(const oracle_scene *s, double *ev, const double *u, const double *v, const double *w,
                        double cs);
void oracle_divergence(const oracle_scene *s, double *out, const double *u, const double *v, const double *w);
void oracle_projection(const oracle_scene *s, double *u, double *v, double *w, const double *us, const double *vs,
                       const double *ws, const double *p);
void oracle_buoyancy(const oracle_scene *s, double *f, const double *T, const double *Ta, double beta, double g);
void oracle_add_source(const oracle_scene *s, double *out, const double *S, double dt, int field_type);

/* ExplicitDiffuse::diffuse (src/diffusion/ExplicitDiffuse.cpp:27-127): one
 * explicit step out = in + dt * (...) on inner cells, then the boundary
 * program; ev == NULL: laminar. */
void oracle_diffuse_explicit(const oracle_scene *s, double *out, const double *in, double D, const double *ev,
                             double dt, int field_type);
/* DynamicSmagorinsky::calc_turbulent_viscosity (src/turbulence/DynamicSmagorinsky.cpp:172-384)
 * with its explicit_filtering (:384-427), loop by loop: ev on the inner cells
 * (no boundary program).  The reference's work fields start as zero and only
 * their inner cells are written; this restatement allocates them zeroed per
 * call, which gives the same values (every inner cell is written before it is
 * read in a call). */
void oracle_dynamic_smagorinsky(const oracle_scene *s, double *ev, const double *u, const double *v, const double *w,
                                double nu);
/* ISource::dissipate (src/interfaces/ISource.cpp:63-123): out += dt * nu * Phi
 * on inner cells, then the boundary program of field_type. */
void oracle_dissipate(const oracle_scene *s, double *out, const double *u, const double *v, const double *w,
                      double nu, double dt, int field_type);

/* IDiffusion::diffuse; ev == NULL: laminar.  Returns iterations. */
int64_t oracle_diffuse_cgs(const oracle_scene *s, double *out, double *in, const double *b, double D,
                           const double *ev, double dt, int field_type, int64_t max_iter, double tol, double w,
                           double *residual);
int64_t oracle_diffuse_jacobi(const oracle_scene *s, double *out, double *in, const double *b, double D,
                              const double *ev, double dt, int field_type, int64_t max_iter, double tol, double w,
                              double *residual);

/* VCycleMG::pressure; the solver's level arrays persist between calls in *state. */
typedef struct oracle_mg oracle_mg;
oracle_mg *oracle_mg_create(const oracle_scene *s, const oracle_mg_cfg *cfg);
void oracle_mg_destroy(oracle_mg *mg);
int64_t oracle_mg_pressure(oracle_mg *mg, double *p, const double *rhs, int first_step, double *residual);
/* sweeps of the last coarse-level solve (VCycleMG::Solve) */
int64_t oracle_mg_last_coarse_iterations(const oracle_mg *mg);

#ifdef __cplusplus
}
#endif
#endif
