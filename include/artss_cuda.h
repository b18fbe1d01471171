/* artss_cuda.h -- C ABI of the B200 kernels behind the ARTSS plugin interfaces.
 *
 * One entry point per plugin method of the fractional-step timestep
 * (ARTSS src/solver/NSTempTurbSolver.cpp:94-248).  Everything crosses the
 * boundary as plain pointers, sizes and POD structs; device memory is owned by
 * a context and all work of a context is enqueued on its own CUDA stream.
 *
 * Conventions
 *  - Every function returns ARTSS_OK (0) or a negative status; the message of
 *    the last failure on the calling thread is returned by artss_last_error().
 *  - Arrays use the reference layout IX(i,j,k) = i + Nx*j + Nx*Ny*k with one
 *    ghost layer (ARTSS src/utility/GlobalMacrosTypes.h:70), FP64 unless noted.
 *  - "level" is the multigrid level (0 = finest), "field_type" the reference
 *    FieldType (ARTSS src/utility/Mapping.h:52-54) that selects boundary
 *    conditions.
 *  - Iterative solvers never hang: each loop is bounded by its max_iter and
 *    reports the iterations it took.
 *  - A context is not thread-safe; distinct contexts are independent.
 */
#ifndef ARTSS_CUDA_H
#define ARTSS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARTSS_MAX_LEVEL 8 /* multigrid levels 0..ARTSS_MAX_LEVEL */

enum artss_status {
    ARTSS_OK = 0,
    ARTSS_ERR_ARG = -1,       /* invalid argument / size / pointer */
    ARTSS_ERR_CUDA = -2,      /* CUDA runtime error */
    ARTSS_ERR_NOMEM = -3,     /* device allocation failed */
    ARTSS_ERR_STATE = -4,     /* call not valid in the context's state */
    ARTSS_ERR_NO_DEVICE = -5, /* no CUDA device / extension unusable */
    ARTSS_ERR_LIMIT = -6      /* a size exceeds a documented maximum */
};

/* ARTSS FieldType (src/utility/Mapping.h:52-54) */
enum artss_field_type {
    ARTSS_FIELD_RHO = 0, ARTSS_FIELD_U = 1, ARTSS_FIELD_V = 2, ARTSS_FIELD_W = 3,
    ARTSS_FIELD_P = 4, ARTSS_FIELD_T = 5, ARTSS_FIELD_NU = 6, ARTSS_NUM_FIELD_TYPES = 7
};

typedef struct artss_ctx artss_ctx;

/* Per-level grid geometry, as DomainData computes it
 * (ARTSS src/domain/DomainData.cpp:12-56, DomainData.h:144-171). */
typedef struct {
    int32_t n_levels;                    /* coarse levels (reference n_level); levels 0..n_levels */
    int32_t reserved;
    int64_t Nx[ARTSS_MAX_LEVEL + 1];     /* cells incl. ghost layer */
    int64_t Ny[ARTSS_MAX_LEVEL + 1];
    int64_t Nz[ARTSS_MAX_LEVEL + 1];
    int64_t i1[ARTSS_MAX_LEVEL + 1];     /* computational-domain inner index range, inclusive */
    int64_t i2[ARTSS_MAX_LEVEL + 1];
    int64_t j1[ARTSS_MAX_LEVEL + 1];
    int64_t j2[ARTSS_MAX_LEVEL + 1];
    int64_t k1[ARTSS_MAX_LEVEL + 1];
    int64_t k2[ARTSS_MAX_LEVEL + 1];
    double dx[ARTSS_MAX_LEVEL + 1];      /* spacing per level */
    double dy[ARTSS_MAX_LEVEL + 1];
    double dz[ARTSS_MAX_LEVEL + 1];
} artss_grid_desc;

/* One boundary assignment x[target] = sign * x[source] + value, the loop body
 * of DomainBoundary/ObstacleBoundary::apply_boundary_condition
 * (ARTSS src/boundaryCondition/DomainBoundary.cpp:42-46,
 *  src/boundaryCondition/ObstacleBoundary.cpp:42-48). */
typedef struct {
    int64_t target;
    int64_t source;
    double value;
    int32_t sign;   /* +1 or -1 */
    int32_t reserved;
} artss_bc_assign;

/* Iteration control of the diffusion solvers
 * (Settings::solver::diffusion_solvers::{jacobi,colored_gauss_seidel}). */
typedef struct {
    int64_t max_iter;
    double tol_res;
    double w;
} artss_iter_cfg;

typedef struct {
    int64_t iterations;
    double residual;
} artss_iter_stats;

/* VCycleMG settings (Settings::solver::pressure_solvers::vcycle_mg). */
enum artss_smoother { ARTSS_SMOOTHER_JACOBI = 0, ARTSS_SMOOTHER_CGS = 1 };
/* run the coarse solve as separate kernels per sweep (multi-block), not as
 * one single-block kernel; same results, for levels too large for one block
 * the multi-block form is used anyway */
#define ARTSS_MG_NO_FUSED_COARSE 1
/* keep the fused coarse solve in one thread block instead of spreading it
 * over a thread-block cluster (distributed shared memory); same results */
#define ARTSS_MG_NO_CLUSTER_COARSE 2
/* run the Jacobi coarse solve on the cluster with three cluster barriers per
 * sweep (sweep, boundary program, residual) instead of the pipelined form
 * with one; same results */
#define ARTSS_MG_NO_PIPELINED_COARSE 4
typedef struct {
    int32_t n_level;
    int32_t n_cycle;
    int32_t max_cycle;
    int32_t n_relax;
    double tol_res;           /* first-step absolute residual tolerance */
    int32_t smoother;         /* enum artss_smoother */
    int32_t flags;            /* ARTSS_MG_* bits */
    int64_t smoother_max_iter;
    double smoother_tol_res;
    double smoother_w;
} artss_mg_cfg;

typedef struct {
    int64_t cycles;             /* V-cycles run by the call */
    int64_t coarse_iterations;  /* Jacobi/CGS sweeps of the last coarse solve */
    double residual;            /* first-step loop: final absolute ||b - A p||_2, else -1 */
} artss_mg_stats;

typedef struct artss_mg artss_mg;

/* ------------------------------------------------------------------ */
/* context and memory                                                 */
/* ------------------------------------------------------------------ */

/* Replaces DomainData::init + the OpenACC device set-up (src/main.cpp:62-78). */
int artss_ctx_create(const artss_grid_desc *grid, int device, artss_ctx **out);
int artss_ctx_destroy(artss_ctx *ctx);
/* cudaStream_t of the context (all work of the context runs on it). */
void *artss_ctx_stream(artss_ctx *ctx);
int artss_ctx_sync(artss_ctx *ctx);
const char *artss_last_error(void);
/* Number of kernels this context has launched so far. */
int64_t artss_ctx_kernel_launches(artss_ctx *ctx);

/* Per-kernel-family timing.  Families whose bit is set in `mask` (bit k =
 * family k, see artss_kernel_family_name) get a CUDA event pair recorded
 * around every launch on the context's stream; artss_ctx_profile_read
 * synchronises the stream and returns, per family, the launches counted since
 * the last reset (all families, profiled or not) and the summed device time
 * of the profiled ones. */
#define ARTSS_KERNEL_FAMILIES 22
/* Stage timing (no counterpart in the reference, whose benchmark build only
 * prints one wall-clock time for the run, src/TimeIntegration.cpp:59,183).  With
 * enable != 0 the host solvers record one CUDA event on the context stream
 * at each stage boundary of a timestep (not inside graph capture);
 * artss_ctx_stage_read synchronizes the stream and returns the device time
 * summed per stage since the last enable.  Stages of NSTempTurbSolver::do_step
 * (src/solver/NSTempTurbSolver.cpp:94-248): velocity advection, turbulence
 * + velocity diffusion, momentum source, pressure (divergence, solve,
 * projection), temperature (advection, diffusion, source); then the source
 * update and FieldController::update_data of the time loop. */
enum {
    ARTSS_STAGE_ADVECTION = 0,
    ARTSS_STAGE_DIFFUSION = 1,
    ARTSS_STAGE_SOURCE = 2,
    ARTSS_STAGE_PRESSURE = 3,
    ARTSS_STAGE_TEMPERATURE = 4,
    ARTSS_STAGE_UPDATE = 5,
    ARTSS_STAGES = 6
};
#define ARTSS_STAGE_END (-1) /* closes the last stage of a step */
int artss_ctx_stage_timing(artss_ctx *ctx, int enable);
int artss_ctx_stage_mark(artss_ctx *ctx, int stage);
int artss_ctx_stage_read(artss_ctx *ctx, double *ms, int n_stages);
int artss_ctx_profile(artss_ctx *ctx, uint64_t mask);
int artss_ctx_profile_read(artss_ctx *ctx, int64_t *launches, double *ms, int n_families);
int artss_ctx_profile_reset(artss_ctx *ctx);
const char *artss_kernel_family_name(int family);

/* Replaces Field's `new real[]` + `acc enter data` (src/field/Field.cpp:12-53):
 * a zero-filled device array of Nx*Ny*Nz doubles of `level`. */
int artss_field_alloc(artss_ctx *ctx, int level, double **out);
int artss_field_free(artss_ctx *ctx, double *field);
int64_t artss_field_size(artss_ctx *ctx, int level);
/* Field::update_dev / update_host (src/field/Field.h:45-52). */
int artss_upload(artss_ctx *ctx, double *dst, const double *host, int64_t n);
int artss_download(artss_ctx *ctx, double *host, const double *src, int64_t n);
/* The same copies ordered on the context's stream without waiting for them:
 * the copy runs after the work already enqueued and before any later work of
 * the context; `host` must stay valid (and, for overlap, be page-locked) until
 * then.  Field::update_dev / update_host with async = true. */
int artss_upload_async(artss_ctx *ctx, double *dst, const double *host, int64_t n);
int artss_download_async(artss_ctx *ctx, double *host, const double *src, int64_t n);
/* Host transfers overlapped with computation, on a second stream of the
 * context.  artss_copy_upload starts after the work enqueued on the context
 * so far and marks its completion in `slot` (0..7); artss_copy_wait makes the
 * context's later work wait for that slot.  artss_copy_download starts after
 * the work enqueued so far and runs beside later work; artss_copy_join makes
 * the context's later work wait for every transfer of the second stream. */
int artss_copy_upload(artss_ctx *ctx, int slot, double *dst, const double *host, int64_t n);
int artss_copy_wait(artss_ctx *ctx, int slot);
int artss_copy_download(artss_ctx *ctx, double *host, const double *src, int64_t n);
int artss_copy_join(artss_ctx *ctx);

/* Pipelined whole-field transfers (no reference counterpart).  Uploads run on
 * one copy engine and read-backs on the other, so that the inputs of one call
 * go up while the outputs of the previous one come down, both beside the
 * context's work.
 * artss_io_in: the n_in host arrays (n doubles each, page-locked for overlap)
 * are copied into device staging once the previous call's inputs have left
 * it, and from there into `fields`, ordered before the context's later work.
 * artss_io_out: the values of `fields` as of the work enqueued so far are
 * copied into staging (two sets, used alternately) and from there to the
 * host beside later work.  The k-th artss_io_out returns once the (k-2)-th
 * has completed: host arrays given to call pair k-2 may then be reused.
 * artss_io_sync waits for every transfer and for the context's work. */
/* Snapshot read-back for output writers (no counterpart in the reference,
 * whose writers read host mirrors updated by OpenACC): the values of the n
 * `fields` (count doubles each) as of the work enqueued so far are copied into
 * device staging on the context stream and from there, on a copy stream, into
 * page-locked host arrays of the library, beside the context's later work.
 * *ticket identifies the read-back.  artss_readback_wait (callable from
 * another thread) blocks until the copies are on the host and hands out the
 * arrays; artss_readback_release gives them back.  Two read-backs can be in
 * flight: the next call waits until the ticket two before it is released. */
int artss_readback(artss_ctx *ctx, int n, const double *const *fields, int64_t count, int64_t *ticket);
int artss_readback_wait(artss_ctx *ctx, int64_t ticket, const double **host, int n);
int artss_readback_release(artss_ctx *ctx, int64_t ticket);
/* Analysis::calc_CFL (src/analysis/Analysis.cpp:322-351): dt * max over inner
 * cells of |u|/dx + |v|/dy + |w|/dz; synchronizes the stream. */
int artss_cfl(artss_ctx *ctx, const double *u, const double *v, const double *w, double dt, double *cfl);
int artss_io_in(artss_ctx *ctx, int n_in, double *const *fields, const double *const *host, int64_t n);
int artss_io_out(artss_ctx *ctx, int n_out, const double *const *fields, double *const *host, int64_t n);
int artss_io_sync(artss_ctx *ctx);

/* Whole-step graphs.  Between artss_graph_begin and artss_graph_end every
 * call on the context is captured instead of run: its bounded solver loops
 * (diffusion, mixed-precision pressure) become conditional WHILE nodes that
 * test the device loop state, so the captured work needs no host decision;
 * calls that must read results on the host fail inside a capture.
 * artss_graph_launch runs the captured work once more on the context's
 * stream.  Values that change from launch to launch live in parameter slots
 * (artss_param_set, set before the launch) read by kernels such as
 * artss_scale_copy_param (dst = src * param[slot]). */
typedef struct artss_graph artss_graph;
int artss_graph_begin(artss_ctx *ctx);
int artss_graph_end(artss_ctx *ctx, int discard, artss_graph **out);
int artss_graph_launch(artss_graph *g);
int artss_graph_destroy(artss_graph *g);
int artss_graph_capturing(artss_ctx *ctx);
int artss_param_set(artss_ctx *ctx, int slot, double value);
int artss_scale_copy_param(artss_ctx *ctx, double *dst, const double *src, int slot, int level);

/* ------------------------------------------------------------------ */
/* geometry: GPU lists -> device cell flags and boundary programs     */
/* ------------------------------------------------------------------ */

/* Replaces Multigrid::send_domain_lists_to_GPU (src/domain/Multigrid.cpp:520-526):
 * the level's domain-inner list and domain list (inner + boundary cells),
 * sorted ascending as the reference builds them, become per-cell flags. */
int artss_set_cell_lists(artss_ctx *ctx, int level,
                         const int64_t *inner, int64_t n_inner,
                         const int64_t *domain, int64_t n_domain);
/* Device copy of the level's cell flags (bit0 inner, bit1 domain list). */
int artss_get_cell_flags(artss_ctx *ctx, int level, uint8_t *host_out, int64_t n);

/* Replaces Multigrid::apply_boundary_condition's per-patch loops
 * (src/domain/Multigrid.cpp:555-572): the ordered assignments for one field
 * type on one level (obstacles in id order, then domain patches
 * left..back).  The library compiles them into dependency-free waves. */
int artss_set_boundary_program(artss_ctx *ctx, int level, int field_type,
                               const artss_bc_assign *ops, int64_t n_ops);
/* Number of kernel waves the compiled program of (level, field_type) needs. */
int artss_boundary_program_waves(artss_ctx *ctx, int level, int field_type);

/* DomainController::apply_boundary (src/domain/DomainController.cpp:145-147). */
int artss_apply_boundary(artss_ctx *ctx, double *field, int level, int field_type);

/* ------------------------------------------------------------------ */
/* whole-array field operations (src/field/Field.h:64-135)            */
/* ------------------------------------------------------------------ */
int artss_fill(artss_ctx *ctx, double *field, int level, double value);
int artss_copy(artss_ctx *ctx, double *dst, const double *src, int level);
int artss_add_field(artss_ctx *ctx, double *dst, const double *src, int level);   /* dst += src */
int artss_add_scalar(artss_ctx *ctx, double *dst, double x, int level);         /* dst += x */
int artss_scale(artss_ctx *ctx, double *dst, double x, int level);              /* dst *= x */
int artss_scale_copy(artss_ctx *ctx, double *dst, const double *src, double x, int level); /* dst = src * x */
/* FieldController::couple_vector / couple_scalar (src/field/FieldController.cpp:151-186):
 * a0 = a and a_tmp = a for each non-null triple, one pass over memory.  a0 may
 * be NULL (a_tmp = a only), for a caller that knows a0 is rewritten before it
 * is read. */
int artss_couple(artss_ctx *ctx, const double *a, double *a0, double *a_tmp,
                 const double *b, double *b0, double *b_tmp,
                 const double *c, double *c0, double *c_tmp);

/* ------------------------------------------------------------------ */
/* plugins                                                            */
/* ------------------------------------------------------------------ */

/* IAdvection::advect, SLAdvect (src/advection/SLAdvect.cpp:34-170), with the
 * closing apply_boundary(out).  dt is the physical time step. */
int artss_advect_sl(artss_ctx *ctx, double *out, const double *in,
                    const double *u, const double *v, const double *w,
                    double dt, int out_field_type);
/* Three SLAdvect calls sharing one backtrace: out_u <- in_u, out_v <- in_v,
 * out_w <- in_w, all advected with (u, v, w) (NSTempTurbSolver.cpp:129-131). */
int artss_advect_sl_uvw(artss_ctx *ctx, double *out_u, double *out_v, double *out_w,
                        const double *in_u, const double *in_v, const double *in_w,
                        const double *u, const double *v, const double *w, double dt);

/* ITurbulence::calc_turbulent_viscosity, ConstSmagorinsky
 * (src/turbulence/ConstSmagorinsky.cpp:30-87), including apply_boundary(ev). */
int artss_turb_const_smagorinsky(artss_ctx *ctx, double *nu_t,
                                 const double *u, const double *v, const double *w, double cs);
/* ITurbulence::calc_turbulent_viscosity, DynamicSmagorinsky
 * (src/turbulence/DynamicSmagorinsky.cpp:172-427): the dynamic
 * Smagorinsky-Lilly eddy viscosity on the inner cells of level 0, with the
 * reference's filters, its in-place 27-cell averaging of the coefficient in
 * list order and ev = 0 where ev + nu < 0; no boundary program (the reference
 * applies none).  The first call (or the first after the cell lists or
 * boundary programs changed) sets up 40 level-0 work arrays and must not be
 * inside a stream capture. */
int artss_turb_dynamic_smagorinsky(artss_ctx *ctx, double *nu_t, const double *u, const double *v,
                                   const double *w, double nu);

/* IDiffusion::diffuse, ColoredGaussSeidelDiffuse (src/diffusion/ColoredGaussSeidelDiffuse.cpp:38-173).
 * ev == NULL selects the laminar variant.  `in` is overwritten as in the
 * reference (it holds the state before the last sweep) unless flags has
 * ARTSS_DIFFUSE_IN_SCRATCH, in which case its final contents are unspecified.
 * ARTSS_DIFFUSE_OUT_HOLDS_IN: the caller guarantees out already equals in
 * (both coupled from one field), and the reference's out.copy_data(in) is
 * skipped. */
#define ARTSS_DIFFUSE_IN_SCRATCH 1
#define ARTSS_DIFFUSE_OUT_HOLDS_IN 2
int artss_diffuse_cgs(artss_ctx *ctx, double *out, double *in, const double *b,
                      double D, const double *ev, double dt, int field_type,
                      const artss_iter_cfg *cfg, int flags, artss_iter_stats *stats);
/* Autotuner (no counterpart in the reference): the first colored Gauss-Seidel
 * solve on a level shape times the sweep's z-depths (8, 16, 32 planes per
 * block) on its first iteration and keeps the fastest for the context.
 * enable = 0 switches tuning off (16 planes) and forgets earlier choices;
 * artss_cgs_sweep_depth returns the chosen depth, 0 before the first solve. */
int artss_ctx_autotune(artss_ctx *ctx, int enable);
/* Programmatic dependent launch: kernels launched so that they begin while
 * their predecessor finishes (each waits on the device for the predecessor's
 * results before it reads them).  enable = 2 (default): eager launches and
 * the launches captured into whole-step graphs; 1: eager launches only; 0:
 * every kernel starts after its predecessor has completed. */
int artss_ctx_pdl(artss_ctx *ctx, int enable);
int artss_cgs_sweep_depth(artss_ctx *ctx, int turbulent);
/* the tuned sweep variant of level 0 (0-2: two-phase kernel of z-depth 8,
 * 16, 32; 3-5: one-phase kernel; 6-8: row-pair kernel with persistent
 * blocks: 64 x 8 and 64 x 6 tiles two blocks per multiprocessor, 64 x 16
 * tiles one block), -1 before the first solve; artss_cgs_sweep_depth
 * returns -1 for variants 6-8 */
int artss_cgs_sweep_variant(artss_ctx *ctx, int turbulent);
/* Pins the colored Gauss-Seidel sweep variant of artss_diffuse_cgs (0-8 as
 * above; 3-8 need an inner box that starts at an odd x), -1 (default): the
 * autotuner's choice.  No counterpart in the reference. */
int artss_ctx_sweep_variant(artss_ctx *ctx, int variant);
/* IDiffusion::diffuse, ColoredGaussSeidelDiffuse with FP32 sweeps inside FP64
 * defect correction (no counterpart in the reference; mirrors
 * src/diffusion/ColoredGaussSeidelDiffuse.cpp:38-173): each iteration forms
 * the FP64 defect of out, solves for the correction by one red-then-black
 * sweep from zero with the correction in FP32, adds it in FP64 and applies the
 * boundary program; the loop stops on the reference's measure ||rb (x_new -
 * x)||_2 <= tol_res or max_iter.  In exact arithmetic each iteration is the
 * reference's (w must be 1).  Same arguments and flags as artss_diffuse_cgs;
 * not captured into graphs. */
int artss_diffuse_cgs_mixed(artss_ctx *ctx, double *out, double *in, const double *b,
                            double D, const double *ev, double dt, int field_type,
                            const artss_iter_cfg *cfg, int flags, artss_iter_stats *stats);
/* IDiffusion::diffuse, JacobiDiffuse (src/diffusion/JacobiDiffuse.cpp:31-203). */
int artss_diffuse_jacobi(artss_ctx *ctx, double *out, double *in, const double *b,
                         double D, const double *ev, double dt, int field_type,
                         const artss_iter_cfg *cfg, artss_iter_stats *stats);

/* IDiffusion::diffuse, ExplicitDiffuse (src/diffusion/ExplicitDiffuse.cpp:27-127):
 * one explicit Euler step out = in + dt * (D Laplacian(in)) on inner cells
 * (ev != NULL: the reference's turbulent form with face viscosities
 * 0.5 (EV_nb + EV) + D), then the boundary program of field_type on out. */
int artss_diffuse_explicit(artss_ctx *ctx, double *out, const double *in, double D, const double *ev, double dt,
                           int field_type);
/* ISource::dissipate (src/interfaces/ISource.cpp:63-123): out += dt * nu *
 * Phi(u, v, w) (viscous dissipation) on inner cells, then the boundary
 * program of field_type. */
int artss_dissipate(artss_ctx *ctx, double *out, const double *u, const double *v, const double *w, double nu,
                    double dt, int field_type);

/* IPressure::divergence (src/interfaces/IPressure.cpp:20-110): rhs on inner
 * cells and zero on the computational domain's ghost ring. */
int artss_divergence(artss_ctx *ctx, double *rhs, const double *u, const double *v, const double *w);
/* IPressure::projection (src/interfaces/IPressure.cpp:125-172) + BCs of u, v, w. */
int artss_projection(artss_ctx *ctx, double *u, double *v, double *w,
                     const double *u_star, const double *v_star, const double *w_star,
                     const double *p);

/* ISource::buoyancy_force (src/interfaces/ISource.cpp:26-52) on the domain list. */
int artss_buoyancy_force(artss_ctx *ctx, double *force, const double *T, const double *T_ambient,
                         double beta, double g);
/* ExplicitEulerSource::add_source (src/source/ExplicitEulerSource.cpp:25-104):
 * out += dt * S on inner cells, then apply_boundary(out). */
int artss_add_source(artss_ctx *ctx, double *out, const double *S, double dt, int field_type);

/* IPressure::pressure, VCycleMG (src/pressure/VCycleMG.cpp:17-798).
 * The solver owns its level hierarchy (residuals, errors, temporaries). */
int artss_mg_create(artss_ctx *ctx, const artss_mg_cfg *cfg, artss_mg **out);
int artss_mg_destroy(artss_mg *mg);
/* One VCycleMG::pressure call: first_step != 0 reproduces the Nt == 1 branch
 * (cycles until the absolute residual reaches tol_res, max_cycle, or the
 * smoother budget), otherwise n_cycle V-cycles. */
int artss_mg_pressure(artss_mg *mg, double *p, const double *rhs, int first_step, artss_mg_stats *stats);
/* One VCycleMG::VCycleMultigrid on p with the right-hand side last given to
 * artss_mg_pressure / artss_mg_set_rhs. */
int artss_mg_set_rhs(artss_mg *mg, const double *p, const double *rhs);
int artss_mg_vcycle(artss_mg *mg, double *p);
/* VCycleMG iterated to a relative tolerance: V-cycles (VCycleMG.cpp:215-288)
 * on p until ||b - A p||_2 <= rel_tol * ||b||_2 over the level-0 inner cells
 * or max_cycles; the plain FP64 solve the mixed-precision one is measured
 * against.  stats may be NULL. */
typedef struct {
    int64_t cycles;        /* V-cycles done */
    double residual;       /* ||b - A p||_2 at the end */
    double rel_residual;   /* residual / b_norm */
    double b_norm;         /* ||b||_2 over the inner cells */
} artss_solve_stats;
int artss_mg_solve_rel(artss_mg *mg, double *p, const double *rhs, double rel_tol, int64_t max_cycles,
                       artss_solve_stats *stats);

/* Mixed-precision pressure solve; no counterpart in the reference (it plugs
 * in where IPressure::pressure, src/interfaces/IPressure.h:17, is called).
 * FP64 defect correction on level 0 around FP32 V-cycles:
 *     r = b - A p  (FP64);  stop when ||r|| <= rel_tol ||b||;
 *     e = V-cycle(r) in FP32 with zero boundary values, coarsest level solved
 *     in FP64;  p += e  (FP64)
 * With ARTSS_MIXED_REMOVE_MEAN the mean of p over the inner cells is removed
 * at the end (pure-Neumann pressure problems: p is defined up to a constant).
 * b must lie in the range of A; for pure-Neumann scenes with obstacles a
 * mean-free b is not enough (the obstacle edge and corner cells make A
 * non-symmetric) -- artss_laplacian gives consistent right-hand sides. */
#define ARTSS_MIXED_REMOVE_MEAN 1
/* smoothing by red-black Gauss-Seidel (in place, w the over-relaxation
 * weight, boundary program after each colour) instead of weighted Jacobi */
#define ARTSS_MIXED_RBGS 2
/* the FP32 levels launch the boundary program after every sweep; without it
 * (and without ARTSS_MIXED_RBGS) their stencils read boundary neighbours
 * through the program instead (same values, fewer launches) */
#define ARTSS_MIXED_BC_LAUNCH 4
/* solve the coarsest level on a thread-block cluster even where it fits one
 * block (shared memory, register-resident cells and boundary assignments,
 * block barriers only); same iterates, up to the order of the residual sums */
#define ARTSS_MIXED_CLUSTER_COARSE 8
/* prolongate one fine cell per thread (8 coarse loads each) instead of one
 * coarse column per thread updating its 8 children from a register window;
 * same values */
#define ARTSS_MIXED_FINE_PROLONG 16
typedef struct {
    int32_t n_level;          /* V-cycle levels 0 .. n_level-1; the coarse solve is on n_level-1 */
    int32_t n_relax;          /* weighted-Jacobi sweeps before and after each coarse correction */
    int32_t coarse_smoother;  /* ARTSS_SMOOTHER_JACOBI or ARTSS_SMOOTHER_CGS (FP64, one kernel) */
    int32_t flags;            /* ARTSS_MIXED_* */
    double w;                 /* Jacobi weight of the FP32 sweeps */
    double coarse_w;          /* relaxation weight of the coarse solve; <= 0: red-black SOR with the
                               * model problem's optimal weight 2 / (1 + sin(pi / (n + 1))) for CGS,
                               * 2/3 for Jacobi */
    double coarse_rel_tol;    /* coarse solve stops at this fraction of its initial residual ... */
    int64_t coarse_max_iter;  /* ... or after this many sweeps */
    double rel_tol;           /* outer stopping rule */
    int64_t max_cycles;       /* outer V-cycle limit */
} artss_mixed_cfg;
typedef struct artss_mixed artss_mixed;
int artss_mixed_create(artss_ctx *ctx, const artss_mixed_cfg *cfg, artss_mixed **out);
int artss_mixed_destroy(artss_mixed *m);
int artss_mixed_solve(artss_mixed *m, double *p, const double *b, artss_solve_stats *stats);
/* out = A p on the inner cells of `level` (the VCycleMG operator, after the
 * level's pressure boundary program is applied to p); other cells of out are
 * left as they are. */
int artss_laplacian(artss_ctx *ctx, double *out, double *p, int level);

/* ---- learned initial guess: BF16 3-D convolution on the tensor cores ----
 * No counterpart in the reference.  Activations are channels-last [D][H][W][C]
 * bf16 with C a multiple of 16; 3x3x3 kernel, stride 1, zero padding 1:
 *   y[z,y,x,co] = bias[co] + sum_{t,ci} w[t][co][ci] x[z+dz, y+dy, x+dx, ci],
 *   t = 9(dz+1) + 3(dy+1) + (dx+1).
 * w_packed holds w as [27][C_in/8][C_out][8] bf16 (per tap the shared-memory
 * layout of the MMA's B operand); bias (FP32, C_out) may be NULL; relu != 0
 * clamps the output at 0.  Tiles of 128 voxels must fit: W a multiple of
 * 128, or W dividing 128 with H a multiple of 128/W, or W*H dividing 128 with
 * D a multiple of 128/(W*H); C_in and C_out multiples of 16, at most 256.
 * The backward pass w.r.t. the input is this same convolution with the
 * weights flipped in space and C_in, C_out exchanged. */
typedef struct {
    int32_t D, H, W;
    int32_t cin, cout;
    int32_t relu;
} artss_conv_desc;
int artss_conv3d_fwd(artss_ctx *ctx, const artss_conv_desc *d, const void *x, const void *w_packed,
                     const float *bias, void *y);
/* Weight gradient of artss_conv3d_fwd: dw[t][co][ci] += sum over voxels of
 * dy[v][co] * x[v + offset(t)][ci] (FP32, dw zeroed by the caller); x is the
 * forward input, dy the gradient of the forward output (same D, H, W).
 * C_in, C_out multiples of 16, at most 128. */
int artss_conv3d_wgrad(artss_ctx *ctx, const artss_conv_desc *d, const void *x, const void *dy, float *dw);
/* Element-wise and data-movement kernels of the network (bf16 activations
 * [D][H][W][C], FP32 parameters).  relu_bwd: dy *= (y > 0).  pool2: 2x2x2
 * average (backward != 0: x is the coarse gradient, y the fine one, /8).
 * up2: nearest 2x upsampling of x [D][H][W][C] into channels
 * [c_off, c_off + C) of y [2D][2H][2W][c_total] (backward: sum of the 8
 * children).  copy_channels: channel slice copy or add (concatenation).
 * bias_grad: db[c] += sum_v dy[v][c].  pack_weights: FP32 w[27][co][ci] to the
 * convolution's packed BF16 operand (flip != 0: input-gradient weights).
 * adam: Adam with bias correction (step >= 1).  inputs: network input from
 * level arrays over the level's inner box: ch0 = s_r (rhs - A p_prev) (p_prev
 * with its boundary values applied), ch1 = inner-cell mask, ch2 = s_b rhs, the
 * rest 0.  apply: p = p_prev + scale * y[.][0] on inner cells.  mse: 0.5 sum over masked voxels (y[.][0] - target)^2 as block
 * partials and its gradient (times inv_n) in channel 0 of dy. */
int artss_nn_zero(artss_ctx *ctx, void *p, int64_t bytes);
int artss_nn_relu_bwd(artss_ctx *ctx, void *dy, const void *y, int64_t n);
int artss_nn_pool2(artss_ctx *ctx, const void *x, void *y, int D, int H, int W, int C, int backward);
int artss_nn_up2(artss_ctx *ctx, const void *x, void *y, int D, int H, int W, int C, int c_total, int c_off,
                 int backward);
int artss_nn_copy_channels(artss_ctx *ctx, const void *src, int s_total, int s_off, void *dst, int d_total, int d_off,
                           int C, int64_t voxels, int accumulate);
int artss_nn_bias_grad(artss_ctx *ctx, const void *dy, float *db, int64_t voxels, int C);
int artss_nn_pack_weights(artss_ctx *ctx, const float *w, void *packed, int cout, int cin, int flip);
int artss_nn_adam(artss_ctx *ctx, float *w, const float *g, float *m, float *v, int64_t n, float lr, float b1,
                  float b2, float eps, int step);
int artss_nn_inputs(artss_ctx *ctx, int level, const double *rhs, const double *p_prev, double s_r, double s_b,
                    void *out, int C);
int artss_nn_apply(artss_ctx *ctx, int level, const void *y, int C, const double *p_prev, double scale, double *p);
/* training target t = scale (p_star - p_prev) over the inner box (FP32, 0 off the inner list) */
int artss_nn_target(artss_ctx *ctx, int level, const double *p_star, const double *p_prev, double scale, float *t);
int artss_nn_mse(artss_ctx *ctx, const void *y, int C, const float *target, const void *inputs, void *dy,
                 int64_t voxels, float inv_n, float *partials, int n_partials);
/* d <- P^k R^k d for a level-0 correction d: restricted `levels` times with
 * the multigrid restriction and prolongated back with its trilinear
 * prolongation, which keeps only what the coarse level represents (the
 * smooth part); cells outside the prolongation's reach become 0.  Uses
 * context-owned scratch arrays, allocated on first use. */
int artss_coarse_project(artss_ctx *ctx, double *d, int levels);
/* Reads and clears the error flag the network kernels raise when a bounded
 * wait gives up (returns ARTSS_ERR_CUDA then); synchronizes the stream. */
int artss_nn_check(artss_ctx *ctx);

/* ||b - A p||_2 over level-0 inner cells (VCycleMG.cpp:186-194) and ||b||_2. */
int artss_residual_norm(artss_ctx *ctx, const double *p, const double *b, double *res_out, double *b_norm_out);

/* The same two norms for callers that cannot allocate device memory (a host
 * code whose allocator owns the device, a memory pool that must not grow):
 * no context, no allocation.  No counterpart in the reference.
 *  - grid: level 0 of the geometry (positive, finite dx, dy, dz);
 *    flags: device array of the level-0 cell flags (bit 0 = inner cell)
 *    holding Nx*Ny*Nz bytes of level 0, or NULL when every
 *    computational-domain cell is inner; p, b: device arrays of Nx*Ny*Nz
 *    doubles; stream: cudaStream_t or NULL.
 *  - The per-block partial sums live in one fixed 128 KiB device array of
 *    this library, kept on every GPU that loads it until the process exits;
 *    grids with more than 8192 tiles of 64x4 cells in an x-y plane are
 *    rejected with ARTSS_ERR_LIMIT.
 *  - The first call on a device looks the array's address up (with that
 *    device current) and keeps it; do not use this function across a
 *    cudaDeviceReset of that device.
 *  - All calls share the array: calls that overlap on the GPU race.
 *  - Blocks until the results are on the host, so it must not be called on
 *    a stream that is being captured (returns ARTSS_ERR_ARG). */
int artss_residual_norm_static(const artss_grid_desc *grid, const uint8_t *flags, const double *p, const double *b,
                               void *stream, double *res_out, double *b_norm_out);

#ifdef __cplusplus
}
#endif
#endif /* ARTSS_CUDA_H */
