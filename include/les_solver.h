/*
 * les_solver.h -- C host driver around les_gpu.h: the reference's main() time loop
 * (les_combustion_solver.c:4016-4632) with the step body on the GPU.
 *
 * The host keeps what the reference keeps on the host and must stay bit-identical to it:
 * the glibc rand() stream (vortex recycling and inflow white noise, drawn in the reference's
 * order), the SEM vortex positions, the dt formula, and the probe / monitor / checkpoint
 * files in the reference's formats.  Each solver owns an independent rand() state, so many
 * solvers can run in one process (ensembles, serving).
 */
#ifndef LES_SOLVER_H
#define LES_SOLVER_H

#include "les_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* glibc random_r TYPE_3 generator (the algorithm behind srand/rand), one state per user. */
typedef struct les_rng {
    int r[34];
    int f, b;                 /* ring positions of the two taps */
    unsigned long long n;     /* draws so far */
} les_rng;

void les_rng_seed(les_rng* g, unsigned int seed);     /* srand(seed) */
int les_rng_next(les_rng* g);                          /* rand(), 0 .. 2^31-1 */
#define LES_RAND_MAX 2147483647

/* Host-side pieces of the time loop, usable without a solver object.
 * vort is nv x {x, y, z, radius, strength_u, strength_v, strength_w}. */
/* initialize() + setting() (:1085-1285): attribute map and the 11 state fields. */
int les_initial_state(const lesgpu_config* cfg, const lesgpu_species* sp, int* attr, double* const* fields);
/* initialize_vortices (:861-897) and update_vortices (:900-939) on a private rand() stream. */
void les_vortices_init(les_rng* g, const lesgpu_config* cfg, double* vort);
void les_vortices_update(les_rng* g, const lesgpu_config* cfg, double* vort, double dt);
/* Inflow white noise (:2990-2992): 3 draws per inlet cell of attr's i = 0 face, (j,k) order. */
void les_inflow_noise(les_rng* g, const int* attr, int ny, int nz, double* noise);
/* dt formula (:4400-4411) from the three maxima returned by lesgpu_dt_inputs. */
double les_dt(const lesgpu_config* cfg, double umax, double numax, double alphamax);

typedef struct les_solver les_solver;

/* Output switches for les_solver_set_outputs. */
#define LES_OUT_PROBES 1       /* probe_data_flame_region_loc*.csv every step (:4572-4574) */
#define LES_OUT_MONITOR 2      /* simulation_monitor.csv every 10 steps (:4592) */
#define LES_OUT_CHECKPOINT 4   /* checkpoint.bin + restart_info.txt every 50 steps (:4583-4589), with
                                  stats_backup.bin when time averages are on */
#define LES_OUT_POINTS 8       /* LES_point_data_phi*_i*_j*_k*.csv: the point time series
                                  (:4557-4568, flush_point_data :3824-3850) at 4D and 8D, on the
                                  axis and in the shear layer (:3780-3822), flushed every 50 steps,
                                  by les_solver_flush and when the solver is destroyed */
#define LES_OUT_VTK 16         /* Premixed_C3H8_Air_%04d.vtk every 500 steps (:4594-4598) and at
                                  les_solver_flush (:4611) */
#define LES_OUT_PSTAT 32       /* no reference counterpart: the probe-row statistics accumulated on
                                  the device during device-loop runs (les_solver_pstat_*, default
                                  bins) instead of probe files, written as profile_stats.bin by
                                  les_solver_flush and at the end of a served request */

/* Load the species files, create the GPU context, build the attribute map and the initial
 * state exactly as initialize()+setting() (:1085-1285), seed rand() and place the SEM
 * vortices (initialize_vortices, :861-897).  t_loop starts at start_step. */
int les_solver_create(const lesgpu_config* cfg, const char* chem_path, const char* tran_path, int start_step,
                      les_solver** out);
void les_solver_destroy(les_solver* s);
lesgpu_ctx* les_solver_ctx(les_solver* s);
const char* les_solver_last_error(const les_solver* s);

/* Directory (must exist) and LES_OUT_* flags; creates the probe files with their header
 * as initialize_probe_file does (:3373-3398). */
int les_solver_set_outputs(les_solver* s, const char* dir, int flags);

/* One iteration of the time loop (:4390-4603): dt from the GPU maxima, vortex update and
 * noise draws with rand(), the GPU step, then the enabled outputs. */
int les_solver_step(les_solver* s);
int les_solver_run(les_solver* s, int nsteps);
/* The same loop with the host side on the GPU (lesgpu_loop_* in les_gpu.h): nsteps steps
 * queued in chunks of `chunk` steps (<= 0: 64) without a per-step host round trip; results,
 * rand() stream and output files are identical to les_solver_run. */
int les_solver_run_device(les_solver* s, int nsteps, int chunk);
/* The device loop as a session: begin (hands the rand() window and vortices to the GPU,
 * sizes the history for `chunk` steps), any number of runs, end (hands them back).
 * Host-driven steps are refused while a session is open. */
int les_solver_loop_begin(les_solver* s, int chunk);
int les_solver_loop_run(les_solver* s, int nsteps);
int les_solver_loop_end(les_solver* s);
/* The two halves of les_solver_loop_run, for callers that queue the steps themselves (a
 * group graph, les_ensemble_run): next_chunk gives the length of the next chunk of a
 * session with `left` steps to go (history capacity, checkpoint steps); after those steps
 * are queued, loop_collect reads their history back, writes the outputs and advances
 * t_loop. */
int les_solver_next_chunk(const les_solver* s, int left);
int les_solver_loop_collect(les_solver* s, int nsteps);

int les_solver_t_loop(const les_solver* s);
double les_solver_last_dt(const les_solver* s);
double les_solver_last_umax(const les_solver* s);

/* Host copies of the attribute map and the initial state fields (checkpoint order). */
int les_solver_attribute(const les_solver* s, int* out);

/* checkpoint.bin in the reference layout (:3671-3698): int t, then u v w T G rho Y0..Y4.
 * load also restores rho*u momentum as load_quick_checkpoint does (:3716-3726). */
int les_solver_save_checkpoint(les_solver* s, const char* path, int t);
int les_solver_load_checkpoint(les_solver* s, const char* path, int* t_out);

/* End of a run (:4604-4623) and the reference's auto-resume from restart_info.txt +
 * checkpoint.bin (:4138-4193), with the reference's resume defects kept or fixed:
 *
 * LES_RESUME_REFERENCE -- what the reference does, defects included:
 *   - les_solver_finish writes checkpoint.bin and restart_info.txt with step 0 whatever step
 *     was reached (save_quick_checkpoint(0), :4623), so the resumed run starts its step count
 *     (and the t_loop >= 500 switch to the WENO5 flame-front gradient) again at 0;
 *   - les_solver_resume re-seeds rand() with the configured seed and redraws the SEM
 *     vortices (initialize_vortices after the load, :4193) instead of continuing the stream;
 *   - it installs the start-up attribute map (:4123-4136), because a resume never runs
 *     setting(): the j = 0 face is a wall/free face (code 4), not the symmetry plane (code 5);
 *   - the nu/alpha maxima of the first dt after the resume are 0 (not restored, :4401-4408).
 * LES_RESUME_FIXED -- les_solver_finish writes the step reached and, beside checkpoint.bin,
 *   les_resume.bin (the SEM vortices, the rand() state and the nu/alpha maxima);
 *   les_solver_resume restores all of it and keeps setting()'s attribute map, so the resumed
 *   run continues the uninterrupted one exactly.
 *
 * finish also writes what les_solver_flush writes and stats_backup.bin when time averages
 * are on (:4611-4625).  resume reads `dir`/restart_info.txt ("BINARY\n<step>\n"),
 * checkpoint.bin (the step the run continues from is the one stored in it, as :4189 takes)
 * and, with averages on, stats_backup.bin; t_out receives that step. */
#define LES_RESUME_REFERENCE 0
#define LES_RESUME_FIXED 1
int les_solver_finish(les_solver* s, const char* dir, int mode);
int les_solver_resume(les_solver* s, const char* dir, int mode, int* t_out);

/* Profile statistics of the probe rows, accumulated on the device during device-loop runs
 * (lesgpu_pstat_* in les_gpu.h): after les_solver_pstat_begin every chunk of
 * les_solver_run_device / les_solver_loop_run / les_ensemble_run adds its rows, with or
 * without probe files; les_solver_pstat_read returns the sums in lesgpu_pstat_read's layout.
 * NULL edge arrays select the defaults: 0.5 mm flame-distance bins over [-LY, LY] (in mm),
 * the post-processing's G bins (0, 0.05] .. (0.95, 1.0] and the optimiser's [0, 0.05) ..
 * [0.95, 1.0), and 40-bin histograms of u over [-U, 3U] and v over [-2U, 2U] for the inlet
 * velocity U; n_* are then ignored. */
int les_solver_pstat_begin(les_solver* s, const double* y_edges_mm, int n_y, const double* g_rc_edges, int n_grc,
                           const double* g_ho_edges, int n_gho, const double* u_edges, const double* v_edges,
                           int n_pdf);
size_t les_solver_pstat_size(const les_solver* s);
int les_solver_pstat_read(les_solver* s, double* out);
/* profile_stats.bin: int32 magic 0x53505350, int32 n_y, n_grc, n_gho, n_pdf, then the edges
 * (y mm, G right-closed, G half-open, u, v; n + 1 doubles each) and the sums. */
int les_solver_pstat_write(les_solver* s, const char* path);

/* Time averages (update_time_averages, :3166-3191) summed on the device from the step whose
 * t_loop reaches start_step (the reference's start_avg_step); start_step < 0 turns them off.
 * save/load: stats_backup.bin (:3736-3778); reynolds_stresses: the seven fields of
 * calculate_resolved_reynolds_stresses (:3194-3217) -- uu, vv, ww, uv, uw, vw, mean G -- each
 * NX*NY*NZ, and the number of steps summed. */
int les_solver_set_averaging(les_solver* s, int start_step);
int les_solver_save_stats(les_solver* s, const char* path);
int les_solver_load_stats(les_solver* s, const char* path);
int les_solver_reynolds_stresses(les_solver* s, double* const* out, int* count);
/* Write what the end of the reference's run writes and the library still buffers: the VTK
 * file of the current step (with LES_OUT_VTK) and the point rows. */
int les_solver_flush(les_solver* s);
/* output_vtk (:3473-3668) to `path`, from the current device state. */
int les_solver_write_vtk(les_solver* s, const char* path);

/* Vortex table (nv x 7) and rand() draw count, for inspection. */
int les_solver_vortices(const les_solver* s, double* out);
unsigned long long les_solver_rng_draws(const les_solver* s);

/* Ensembles (no reference counterpart as an API: the reference's Bayesian optimiser runs
 * one LES per parameter proposal, bayesian_optimizer.py:568-673).  n solvers with their own
 * configs (grids, model constants, seeds) on one device, all advanced by one multi-stream
 * graph per step (lesgpu_group_*).  autotune != 0 tunes the tiles at creation
 * (lesgpu_autotune, once per grid shape and precision; the other members of that shape get
 * the same tiles).  les_ensemble_run advances every member by nsteps in chunks of
 * `chunk` steps (<= 0: 64), writing each member's enabled outputs as les_solver_run_device
 * does; each member's results equal running it alone with the same tiles. */
typedef struct les_ensemble les_ensemble;
int les_ensemble_create(const lesgpu_config* cfgs, int n, const char* chem_path, const char* tran_path, int autotune,
                        les_ensemble** out);
int les_ensemble_run(les_ensemble* e, int nsteps, int chunk);
/* Step the members with the batched group form (lesgpu_group_create_batched: one launch per
 * RK pass for the members of one grid shape, at most max_per_batch per launch, 0: no cap)
 * instead of the multi-stream graph (enable = 0, the default).  Same results in FP64; in FP32
 * up to the batched kernels' FMA contraction. */
int les_ensemble_set_batched(les_ensemble* e, int enable, int max_per_batch);
int les_ensemble_size(const les_ensemble* e);
les_solver* les_ensemble_member(les_ensemble* e, int i);
const char* les_ensemble_last_error(const les_ensemble* e);
void les_ensemble_destroy(les_ensemble* e);

#ifdef __cplusplus
}
#endif

#endif /* LES_SOLVER_H */
