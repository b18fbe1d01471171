/* artss_host.h -- C API of the host runtime (libartss_host.so).
 *
 * The host runtime reads an ARTSS XML file, builds the geometry (multigrid
 * levels, index lists, boundary programs) and drives the timestep of
 * SolverController / TimeIntegration (ARTSS src/solver/SolverController.cpp,
 * src/TimeIntegration.cpp) through the kernels of artss_cuda.h.
 *
 * The artss_geom_* functions need no GPU: they expose the index lists and
 * boundary assignments the host builds, for bit-exact comparison with the
 * reference's lists (ARTSS src/domain/Multigrid.cpp:313-374).
 */
#ifndef ARTSS_HOST_H
#define ARTSS_HOST_H

#include <stddef.h>
#include <stdint.h>
#include "artss_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct artss_geom artss_geom;
typedef struct artss_sim artss_sim;

/* Status of the int-returning functions: ARTSS_OK; ARTSS_ERR_ARG for a
 * pointer, name, level, size or file the call cannot use (an XML file the
 * settings reader refuses included); ARTSS_ERR_STATE for a call the scene's
 * solver or the simulation's state does not allow (a step after t_end);
 * ARTSS_ERR_CUDA for a device error.  The message of the last failure on the
 * calling thread: */
const char *artss_host_last_error(void);

/* ---- geometry (CPU only) ---- */
int artss_geom_create(const char *xml_path, artss_geom **out);
void artss_geom_destroy(artss_geom *g);
int artss_geom_levels(artss_geom *g);
int artss_geom_obstacles(artss_geom *g);
/* name: "inner", "domain", "obst", "bnd_<patch>", "obst<id>_<patch>" with
 * <patch> in left,right,bottom,top,front,back.  The pointer stays valid until
 * artss_geom_destroy. */
int artss_geom_list(artss_geom *g, const char *name, int level, const int64_t **data, int64_t *n);
/* Nx, Ny, Nz of a level */
int artss_geom_dims(artss_geom *g, int level, int64_t *dims3);
/* ordered boundary assignments of (level, field type); *n == 0 when the
 * field type has no boundary conditions */
int artss_geom_boundary_program(artss_geom *g, int level, int field_type, const artss_bc_assign **ops, int64_t *n);
int artss_geom_grid_desc(artss_geom *g, artss_grid_desc *out);

/* ---- simulation (GPU) ---- */
int artss_sim_create(const char *xml_path, int device, artss_sim **out);
void artss_sim_destroy(artss_sim *s);
/* runs up to `steps` timesteps (all remaining when steps < 0); *done = steps run */
int artss_sim_run(artss_sim *s, int64_t steps, int64_t *done);
/* One timestep with its host transfers: the n_in named fields are set from
 * in_host[k] before they are read, the n_out named fields are read into
 * out_host[k] after their last write; transfers run beside the step where
 * the solver allows (NSTempTurbSolver / NSTempSolver: p and T arrive while
 * the velocity is computed, u, v, w, p leave while T is).  Inputs u, v, w
 * and T are the state the step advances: their copies (u0, u_tmp, ..., T0,
 * T_tmp) are set from them, as FieldController::update_data sets them after
 * a step.  Buffers should be page-locked; they are complete when the call
 * returns. */
int artss_sim_step_io(artss_sim *s, int n_in, const char *const *in_names, const double *const *in_host, int n_out,
                      const char *const *out_names, double *const *out_host);
/* The same step, pipelined: the call returns once the inputs, the step and
 * the read-back are enqueued.  Inputs go up on one copy engine while the
 * previous call's outputs come down on the other, beside the steps.  The
 * host arrays of a call may be reused once the call two after it has
 * returned, or after artss_sim_io_sync, which waits for everything.  The
 * fields read back are the step's final values, as from artss_sim_step_io. */
int artss_sim_step_io_async(artss_sim *s, int n_in, const char *const *in_names, const double *const *in_host,
                            int n_out, const char *const *out_names, double *const *out_host);
int artss_sim_io_sync(artss_sim *s);
/* Whole-step graphs on or off (off by default): from the third step on, a
 * step is captured once (its solver loops as conditional WHILE nodes on the
 * device loop state) and replayed per step; a scene whose step cannot be
 * captured (a noisy source, the mixed solver's mean removal) keeps running
 * step by step.  Per-step statistics are not updated while replaying. */
int artss_sim_set_graphs(artss_sim *s, int enable);
/* steps run as one graph launch so far */
int64_t artss_sim_graph_steps(artss_sim *s);
int artss_sim_finished(artss_sim *s);
double artss_sim_time(artss_sim *s);
int64_t artss_sim_step_index(artss_sim *s);
int64_t artss_sim_inner_cells(artss_sim *s);
/* field names: u v w u0 v0 w0 u_tmp v_tmp w_tmp nu_t kappa_t p p0 rhs T T0 T_tmp
 * T_a f_x f_y f_z S_T; n must equal the level-0 array size */
int artss_sim_get_field(artss_sim *s, const char *name, double *host, int64_t n);
int artss_sim_set_field(artss_sim *s, const char *name, const double *host, int64_t n);
int64_t artss_sim_field_size(artss_sim *s);
/* device pointer of a field (for timing or zero-copy use) */
double *artss_sim_field_device(artss_sim *s, const char *name);
artss_ctx *artss_sim_context(artss_sim *s);
/* per-step statistics of the last step: iterations of the u, v, w, T
 * diffusion solves, V-cycles and (first step) residual of the pressure solve */
int artss_sim_last_stats(artss_sim *s, int64_t *diff_iters4, int64_t *mg_cycles, double *mg_residual);
/* Checkpoint and rollback (the reference keeps data-assimilation checkpoints in
 * HDF5, src/dataAssimilation/FieldIO.cpp:44-100, absent here): every field of
 * the simulation, the step index and the time in one raw file (magic
 * "ARTSSCKP", little-endian FP64 arrays).  After artss_sim_restore the run
 * continues from the saved step and its fields equal those of the
 * uninterrupted run. */
int artss_sim_save(artss_sim *s, const char *path);
int artss_sim_restore(artss_sim *s, const char *path);
/* Output of the time loop (src/analysis/Analysis.cpp:360-390,
 * src/visualisation/VTKWriter.cpp:60-106): the fields' values as of the steps
 * run so far leave the device by a snapshot read-back beside the next steps,
 * and a worker thread writes the file.  write_dat: one field, every level-0
 * cell, one value per line in the default stream format (Analysis::write_file);
 * write_vtk: the legacy binary VTK rectilinear grid of VTKWriter::write_numerical
 * (u, v, w, p, rhs as divergence, T, concentration 0, sight, nu_t, S_T and the
 * cell centres).  output_wait returns once every queued file is written (the
 * first failure as its status). */
int artss_sim_write_dat(artss_sim *s, const char *field, const char *path);
int artss_sim_write_vtk(artss_sim *s, const char *path);
int artss_sim_output_wait(artss_sim *s);
/* Analysis::calc_CFL (src/analysis/Analysis.cpp:322-351) of the current
 * velocity, reduced on the device */
int artss_sim_cfl(artss_sim *s, double *cfl);
/* one pressure solve of a PressureSolver scene with the current p and rhs */
int artss_sim_pressure(artss_sim *s, int first_step, int64_t *cycles, double *residual);
/* the multigrid solver of a PressureSolver scene, or NULL */
artss_mg *artss_sim_mg(artss_sim *s);

#ifdef __cplusplus
}
#endif
#endif
