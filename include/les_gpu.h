/*
 * les_gpu.h -- C ABI of the B200 solver step for the premixed-flame LES of
 * les_combustion_solver.c (naist15421/Combustion-LES-Optimization).
 *
 * The reference has no plugin or FFI layer: its time loop (les_combustion_solver.c:4390-4603)
 * mutates global Grid3D arrays through direct calls.  This header is the boundary that
 * replaces the body of that loop -- the dt reductions (:4399-4411), the SEM inflow plane
 * (:965-1074), the RK4 stages with calculate_RHS (:4420-4544) and
 * apply_boundary_conditions (:4555) -- with calls into a CUDA library, while the caller
 * keeps the host-side pieces (glibc-compatible rand() draws, probe/monitor/checkpoint files).
 *
 * Conventions
 *  - Every field crossing the boundary is a host array of NX*NY*NZ doubles in the
 *    reference's [i][j][k] order (k fastest, les_combustion_solver.c:286).
 *  - State field order is the checkpoint.bin order (:3671-3698):
 *    u, v, w, T, G, rho, Y[C3H8], Y[O2], Y[N2], Y[CO2], Y[H2O].
 *  - The library owns all device memory; host arrays are only read/written during a call.
 *  - Calls return LESGPU_OK (0) or a negative LESGPU_E* code and never exit the process;
 *    lesgpu_last_error() returns a message for the last failure on a context.
 *  - A context is bound to one CUDA device and one stream and is driven by one host thread.
 *    Calls are synchronous unless their comment says otherwise.
 */
#ifndef LES_GPU_H
#define LES_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LESGPU_OK 0
#define LESGPU_EINVAL -1     /* bad argument (null pointer, size mismatch, unknown id) */
#define LESGPU_ECUDA -2      /* a CUDA runtime call failed */
#define LESGPU_ENOMEM -3     /* device allocation failed or over the configured budget */
#define LESGPU_EIO -4        /* file could not be read or has the wrong record layout */
#define LESGPU_ESTATE -5     /* call out of order (e.g. step before a state was uploaded) */
#define LESGPU_ENONFINITE -6 /* a NaN/Inf was found where the reference would abort */

#define LESGPU_NSP 5          /* C3H8, O2, N2, CO2, H2O (les_combustion_solver.c:129-133) */
#define LESGPU_NSTATE 11      /* u v w T G rho Y0..Y4 */

#define LESGPU_FP64 0         /* plain form: everything in double precision */
#define LESGPU_FP32 1         /* precision form: fp32 bulk, fp64 global sums/reductions */

/* Run-time replacement for the reference's compile-time #defines (:46-83, :136-262) and
 * function-local constants (:2701-2703, :2834, :4101). */
typedef struct lesgpu_config {
    int nx, ny, nz, num_vortices;
    int initial_flame_front_i, weno_transition_step;
    unsigned int seed;
    int flame_accel;                  /* USE_FLAME_ACCEL_MODEL (:208) */
    double lx, ly, lz;
    double inlet_radius, rim_outer_radius;
    double inlet_velocity, inlet_temperature, ambient_temperature;
    double turbulence_intensity, length_scale;
    double s_l, burnt_gas_temperature, pr_t, sc_t, d3;
    double courant, courant_diffusion;
    double cs_unburned, cs_burnt, cs_flame_boost;
    double accel_strength, accel_width, accel_center, relax;
    double nu_unburnt, rho_unburnt_approx, rho_burnt_approx, equivalence_ratio;
    int precision;                    /* LESGPU_FP64 or LESGPU_FP32 */
    int device;                       /* CUDA device ordinal */
} lesgpu_config;

/* Species data as the reference's SpeciesData (:292-305) plus the binary-diffusion fits. */
typedef struct lesgpu_species {
    double mw[LESGPU_NSP];            /* g/mol */
    double t_mid[LESGPU_NSP];
    double nasa_high[LESGPU_NSP][7];
    double nasa_low[LESGPU_NSP][7];
    double lambda[LESGPU_NSP][4];     /* ln-polynomial fits, CGS */
    double eta[LESGPU_NSP][4];
    double dcoef[LESGPU_NSP][LESGPU_NSP][4];
} lesgpu_species;

typedef struct lesgpu_ctx lesgpu_ctx;
typedef struct lesgpu_group lesgpu_group;

/* Field ids for lesgpu_get_field: the 11 state fields, then per-step diagnostics. */
enum {
    LESGPU_F_U = 0, LESGPU_F_V, LESGPU_F_W, LESGPU_F_T, LESGPU_F_G, LESGPU_F_RHO,
    LESGPU_F_Y0, LESGPU_F_Y1, LESGPU_F_Y2, LESGPU_F_Y3, LESGPU_F_Y4,
    LESGPU_F_NU_T = 11,               /* eddy viscosity of the last RHS evaluation */
    LESGPU_F_S_MAG = 12,              /* |S| of the last RHS evaluation */
    LESGPU_F_GRAD_G = 13,             /* |grad G| of the last RHS evaluation (lesgpu_keep_grad_g) */
    /* intermediates of the last RHS evaluation (filtered fields, properties, k-arrays) */
    LESGPU_F_U_F = 100, LESGPU_F_V_F, LESGPU_F_W_F, LESGPU_F_T_F, LESGPU_F_G_F, LESGPU_F_RHO_F,
    LESGPU_F_Y0_F, LESGPU_F_Y1_F, LESGPU_F_Y2_F, LESGPU_F_Y3_F, LESGPU_F_Y4_F,
    LESGPU_F_NU, LESGPU_F_MU_MIX, LESGPU_F_ST, LESGPU_F_CP, LESGPU_F_LAMBDA, LESGPU_F_ALPHA,
    LESGPU_F_D0, LESGPU_F_D1, LESGPU_F_D2, LESGPU_F_D3, LESGPU_F_D4,
    LESGPU_F_K_RHOU, LESGPU_F_K_RHOV, LESGPU_F_K_RHOW, LESGPU_F_K_T, LESGPU_F_K_G,
    LESGPU_F_K_Y0, LESGPU_F_K_Y1, LESGPU_F_K_Y2, LESGPU_F_K_Y3, LESGPU_F_K_Y4
};

/* Replaces load_chem_bin + load_tran_bin (:324-382): read the two Fortran-record files. */
int lesgpu_load_species(const char* chem_path, const char* tran_path, lesgpu_species* out);

/* Allocates the device field arena for one grid (replaces the ALLOC_GRID block, :4023-4080). */
int lesgpu_create(const lesgpu_config* cfg, const lesgpu_species* sp, lesgpu_ctx** out);
void lesgpu_destroy(lesgpu_ctx* ctx);
const char* lesgpu_last_error(const lesgpu_ctx* ctx);

/* Cell attribute codes (:1151-1181): 1 inlet, 2 outlet, 3 fluid, 4 wall/free, 5 symmetry,
 * 6 rim.  NX*NY*NZ ints in [i][j][k] order. */
int lesgpu_upload_attribute(lesgpu_ctx* ctx, const int* attr);

/* Replaces the state half of load_quick_checkpoint (:3701-3726): nfields (<= 11) host
 * arrays in checkpoint order; rho*u momentum is derived as the reference does (:3717).
 * Resets the dt-reduction inputs as a restart does (nu/alpha are not part of the state). */
int lesgpu_upload_state(lesgpu_ctx* ctx, const double* const* fields, int nfields);
int lesgpu_download_state(lesgpu_ctx* ctx, double* const* fields, int nfields);
int lesgpu_get_field(lesgpu_ctx* ctx, int field_id, double* out);

/* The three maxima feeding dt (:1472-1485, :4399-4408): max |u| over inlet+fluid cells
 * (INLET_VELOCITY when below 1e-10) and max nu / alpha over fluid cells from the last
 * RHS evaluation (0 before the first step). */
int lesgpu_dt_inputs(lesgpu_ctx* ctx, double* umax, double* numax, double* alphamax);

/* No counterpart in the reference (its nu/alpha arrays are never saved): sets the nu and
 * alpha maxima that the next dt reads, as lesgpu_dt_inputs returned them before a
 * checkpoint, so a run resumed from that checkpoint takes the same dt as the uninterrupted
 * one.  Call after lesgpu_upload_state, which resets them to 0. */
int lesgpu_set_dt_inputs(lesgpu_ctx* ctx, double numax, double alphamax);

/* SEM inflow for the next step (:943-1075 and the white noise of :2987-2997).
 * vortices: nv x {x, y, z, radius, strength_u, strength_v, strength_w} after the host's
 *           update_vortices (:900-939) for this step's dt;
 * noise:    3 x NY x NZ planes of the rand()-derived r1, r2, r3 in [-1, 1] (only inlet
 *           cells are read), drawn in the reference's (j, k) order after the vortex draws. */
int lesgpu_set_inflow(lesgpu_ctx* ctx, const double* vortices, int nv, const double* noise);

/* One time step with the given dt: SEM plane, four RK4 stages of calculate_RHS with the
 * stage updates, the final combine and apply_boundary_conditions.  t_loop selects the
 * central/WENO5 G-gradient switch (:2740-2780).  Asynchronous on the context's stream. */
int lesgpu_step(lesgpu_ctx* ctx, double dt, int t_loop);

/* Device-resident time loop.  The host-driven cycle above (lesgpu_dt_inputs -> host rand()
 * -> lesgpu_set_inflow -> lesgpu_step) needs one host round trip per step.  These calls move
 * that host side onto the GPU: dt is computed from the device maxima, update_vortices
 * (:900-939) and the inflow noise (:2990-2992) draw from the same glibc rand() stream
 * through a jump-ahead table (bit-identical draws), and each step records its dt, |u|max,
 * probe lines and (every 10th step) the monitor values in a history buffer.  One step is
 * captured once as a CUDA graph and replayed.
 *
 * lesgpu_loop_begin: hand over the host's rand() window (the last 31 words of the
 *   generator, oldest first: x[n-31..n-1]), the vortex table and t_loop.
 * lesgpu_loop_config: probe stations / line and the history capacity in steps (default:
 *   the reference's seven stations on k = NZ/2 and 64 steps).
 * lesgpu_run: queue nsteps (<= capacity) steps; asynchronous.
 * lesgpu_loop_history: after a run, per-step dt and |u|max (nsteps each), probe lines
 *   (nsteps x n x NY x 6) and monitor rows (nsteps x 6, written on steps with
 *   t_loop % 10 == 0 only); any pointer may be NULL.
 * lesgpu_loop_end: hand the rand() window, vortices and t_loop back to the host. */
int lesgpu_loop_begin(lesgpu_ctx* ctx, const unsigned int rng_window[31], const double* vortices, int nv, int t_loop);
int lesgpu_loop_config(lesgpu_ctx* ctx, const int* i_stations, int n, int k_line, int capacity_steps);
int lesgpu_run(lesgpu_ctx* ctx, int nsteps);
int lesgpu_loop_history(lesgpu_ctx* ctx, int nsteps, double* dt, double* umax, double* probes, double* monitor);
int lesgpu_loop_end(lesgpu_ctx* ctx, unsigned int rng_window[31], double* vortices, int* t_loop);

/* Groups (no reference counterpart; the reference runs one LES per process, and its
 * Bayesian optimiser runs trials one after another, bayesian_optimizer.py:568-673).  A group
 * advances several contexts of one device together: one step of every member is captured
 * once as a single multi-stream CUDA graph (each member on its own stream, branches
 * independent), so members whose grids are too small to fill the GPU share it.  Every
 * member must be in a device-loop session (lesgpu_loop_begin) with kernel timing off;
 * lesgpu_group_run queues nsteps (<= each member's history capacity) replays and is
 * asynchronous: each member's lesgpu_loop_history / lesgpu_sync waits for it.  A member's
 * results are bit-identical to running it alone with the same tiles.  Changing a member's
 * tiles or history layout after lesgpu_group_create requires a new group. */
int lesgpu_group_create(lesgpu_ctx* const* ctxs, int n, lesgpu_group** out);
/* The batched form of a group: members whose constants agree except the model constants an
 * optimiser varies (CS_UNBURNED, CS_BURNT, CS_FLAME_BOOST, the flame-acceleration strength,
 * width and centre, the nudging coefficient) and whose grid shape, precision and tiles agree
 * form one batch, and each RK pass of a batch is ONE launch over a (member, tile) grid: blocks
 * find their member's field arena, attribute map, reductions and model constants in a member
 * table.  Each member's dt, rand() draws and SEM plane before, and its boundary conditions and
 * history after, run on its own stream; one step of everything is one CUDA graph.  Members need
 * inspection buffers, |grad G| and the staged scalar pass off.  Results are bit-identical to
 * running each member alone with the same tiles in FP64 (in FP32 up to the FMA contraction
 * of the batched kernels, ~1e-7).  max_per_batch > 0 caps a batch's size: smaller batches on
 * their own streams let one batch's passes overlap another's (0: no cap).
 * lesgpu_group_batches: the number of batches (in the multi-stream form, the number of
 * members). */
int lesgpu_group_create_batched(lesgpu_ctx* const* ctxs, int n, int max_per_batch, lesgpu_group** out);
int lesgpu_group_batches(const lesgpu_group* g);
int lesgpu_group_run(lesgpu_group* g, int nsteps);
void lesgpu_group_destroy(lesgpu_group* g);

/* Probe lines for record_flame_region_data (:3403-3471) and the point buffer (:4558-4569):
 * for each of n x-stations, NY rows of {u, v, w, G, nu_t, S_mag} on the line k = k_line.
 * out holds n * NY * 6 doubles. */
int lesgpu_probe_lines(lesgpu_ctx* ctx, const int* i_stations, int n, int k_line, double* out);

/* Monitor reductions of write_monitor_log (:3874-3918): out[0] total mass (sum of
 * rho*DX*DY*DZ), out[1..2] min/max T, out[3..4] min/max G, out[5] min Y[C3H8]. */
int lesgpu_monitor(lesgpu_ctx* ctx, double out[6]);

/* lesgpu_monitor_noalloc -- no counterpart in the reference.  The same six monitor values
 * as lesgpu_monitor, computed from caller-owned device arrays (n FP64 cells each of rho,
 * T, G and Y[C3H8]) into a caller-owned device buffer out[6], asynchronously on `stream`
 * (a cudaStream_t, or NULL for the default stream).  It allocates nothing: for callers that
 * cannot call cudaMalloc -- a serving loop whose HBM is fully handed out to request slots,
 * or a latency-bound path that must not take cudaMalloc's device-wide synchronisation.
 * Its scratch is a fixed 3 MiB __device__ array that every GPU loading the library holds
 * until exit, so n is limited to LESGPU_NOALLOC_MAX_CELLS; larger n returns LESGPU_EINVAL.
 * The first call on a device looks up that array's device address and should come before
 * any stream capture.  All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller.  `stream` and every buffer must belong to the current
 * device (the scratch address is the current device's); otherwise LESGPU_EINVAL. */
#define LESGPU_NOALLOC_MAX_CELLS 16777216
int lesgpu_monitor_noalloc(const double* rho, const double* T, const double* G, const double* Y0, size_t n,
                           double dx, double dy, double dz, double* out, void* stream);

/* Profile statistics of the probe rows on the device -- no counterpart as an API: the
 * reference appends every probe row to a CSV file each step (record_flame_region_data,
 * :3403-3471) and its post-processing reads them back (analysis.py:82-154, :215-257,
 * bayesian_optimizer.py:71-117).  Here the rows stay on the device: after each device-loop
 * chunk, lesgpu_pstat_accumulate bins the rows of the first n_lines history lines (the probe
 * stations; y_flame from the lower G = 0.5 crossing, rows with |y_rel| <= 1 m) and adds their
 * moments to running FP64 sums, deterministically.  Bins (each array holds n + 1 increasing
 * edges): flame distance y_rel in mm, right-closed (e_b, e_b+1]; G right-closed (the
 * conditional stresses); G half-open [e_b, e_b+1) (the optimiser's <u'v'>); u and v
 * histograms [e_b, e_b+1), last bin closed, for G < 0.5 and G >= 0.5.
 * lesgpu_pstat_read writes lesgpu_pstat_size() doubles:
 *   N, sum u, sum v, sum w;
 *   per y bin: n, sum u, v, w, G, uu, vv, ww, uv;
 *   per right-closed G bin: n, sum u, v, w, uu, vv, uv;
 *   per half-open G bin: n, sum u, v, uv;
 *   counts: u unburnt [n_pdf], v unburnt [n_pdf], u burnt [n_pdf], v burnt [n_pdf]. */
int lesgpu_pstat_begin(lesgpu_ctx* ctx, const double* y_edges_mm, int n_y, const double* g_rc_edges, int n_grc,
                       const double* g_ho_edges, int n_gho, const double* u_edges, const double* v_edges, int n_pdf);
int lesgpu_pstat_accumulate(lesgpu_ctx* ctx, int nsteps, int n_lines);
size_t lesgpu_pstat_size(const lesgpu_ctx* ctx);
/* The bin counts and, when `edges` is not NULL, the edges in the order of lesgpu_pstat_begin's
 * arguments (y, G right-closed, G half-open, u, v); *n_edges receives their total count. */
int lesgpu_pstat_layout(const lesgpu_ctx* ctx, int* n_y, int* n_grc, int* n_gho, int* n_pdf, double* edges,
                        size_t* n_edges);
int lesgpu_pstat_read(lesgpu_ctx* ctx, double* out);
int lesgpu_pstat_end(lesgpu_ctx* ctx);

/* check_for_nan (:1289-1305) without exit(): returns LESGPU_ENONFINITE if any u is not finite. */
int lesgpu_check_finite(lesgpu_ctx* ctx, int field_id);

/* Inspection support (no reference counterpart; the reference exposes these intermediates
 * as globals, :457-612).  lesgpu_set_debug(ctx, 1) makes every step keep Cp, lambda,
 * alpha and the stage-1 k-arrays for lesgpu_get_field; lesgpu_eval_rhs evaluates one
 * calculate_RHS (:2494) at the current state, filling all intermediates, without
 * advancing the state. */
int lesgpu_set_debug(lesgpu_ctx* ctx, int enable);
int lesgpu_eval_rhs(lesgpu_ctx* ctx, int t_loop);

/* Kernel timing (observability; the reference only prints a per-step line, :4601).
 * With timing enabled every step records CUDA events around each kernel class on the
 * context's stream and accumulates their durations; lesgpu_kernel_times returns the
 * totals (ms) and launch counts per class and resets them.  Classes: */
enum {
    LESGPU_K_SEM = 0,        /* SEM inflow plane + normalisation */
    LESGPU_K_FILTER = 1,     /* box filter + mixture properties (4 launches per step) */
    LESGPU_K_STRAIN = 2,     /* strain, nu_t, S_T (4 per step) */
    LESGPU_K_RHS_FLOW = 3,   /* momentum and G right-hand sides (4 per step) */
    LESGPU_K_BC = 4,         /* boundary faces + EOS/renormalisation */
    LESGPU_K_RHS_SCALAR = 5, /* species/T right-hand sides + RK4 stage update (4 per step) */
    LESGPU_NK = 6
};
int lesgpu_kernel_timing(lesgpu_ctx* ctx, int enable);
/* Device-time markers on the context's stream (slots 0..15): lesgpu_mark records a CUDA
 * event, lesgpu_elapsed_ms waits for slot b and returns the time between two markers. */
int lesgpu_mark(lesgpu_ctx* ctx, int slot);
int lesgpu_elapsed_ms(lesgpu_ctx* ctx, int slot_a, int slot_b, double* ms);
int lesgpu_kernel_times(lesgpu_ctx* ctx, double* ms, long long* launches, int n);

/* Self-check of the constant-divisor division used by the kernels (x/c evaluated as a
 * reciprocal product with one fma correction): n pseudo-random dividends spanning
 * 2^-60..2^60 for each of nd divisors; *mismatches counts results whose bits differ from
 * IEEE division.  Runs on the current device; allocates a few bytes of device memory. */
int lesgpu_selfcheck_division(const double* divisors, int nd, size_t n, unsigned long long seed,
                              unsigned long long* mismatches);

/* Keep |grad G| of every RHS evaluation in a field (grad_G_magnitude_for_debug, :2783,
 * :2820; written to the VTK files, :3579-3583), readable as LESGPU_F_GRAD_G.  Off by default:
 * one more store per fluid cell and stage. */
int lesgpu_keep_grad_g(lesgpu_ctx* ctx, int enable);

/* Time averages: update_time_averages (:3166-3191) on the device.  lesgpu_avg_begin allocates
 * ten FP64 running sums per cell (zeroed) and from then on every step -- host-driven or
 * device loop -- adds the state after its boundary conditions to them when its t_loop is
 * >= start_step (the reference's start_avg_step, :4382, :4577).  The sums are in the order
 * of stats_backup.bin (:3740-3754): u, v, w, u*u, v*v, w*w, u*v, u*w, v*w, G; `count` is the
 * number of steps summed (time_avg_steps).  download/upload move the sums and the count
 * (save_statistics_backup / load_statistics_backup, :3736-3778). */
int lesgpu_avg_begin(lesgpu_ctx* ctx, int start_step);
int lesgpu_avg_end(lesgpu_ctx* ctx);
int lesgpu_avg_download(lesgpu_ctx* ctx, double* const* sums, int* count);
int lesgpu_avg_upload(lesgpu_ctx* ctx, const double* const* sums, int count);

/* Thread-block tiles of the per-cell kernels (no reference counterpart; the reference is
 * serial C).  tiles[c] for the classes {filter, strain, rhs_flow, rhs_scalar, eos} indexes
 * the LESGPU_NTILES shapes (k extent x j extent x i extent).  256 threads, every class:
 * 0 = 32x8x1, 1 = 64x4x1, 2 = 16x16x1, 3 = 128x2x1, 4 = 32x4x2, 5 = 16x8x2, 6 = 32x2x4,
 * 7 = 16x4x4; 512 threads, the strain, rhs_flow and rhs_scalar classes only (a filter or
 * eos index above 7 is refused with LESGPU_EINVAL): 8 = 32x8x2, 9 = 32x4x4, 10 = 16x8x4,
 * 11 = 16x4x8, 12 = 64x4x2.  lesgpu_autotune times `reps` evaluations of the four stage
 * kernels per shape at the current state, picks the fastest shape per class (eos follows
 * filter), installs it and optionally returns it and the times (ms_out: 4 classes x
 * LESGPU_NTILES, ms per launch; 1e30 where a shape does not serve the class).  It leaves the
 * state, the dt inputs and the step counters as they were.  The tile changes only the launch
 * geometry; results change only through the summation order of the block partials of
 * <rho_f> (rounding level). */
#define LESGPU_NTILES 13
int lesgpu_set_tiles(lesgpu_ctx* ctx, const int tiles[5]);
int lesgpu_get_tiles(const lesgpu_ctx* ctx, int tiles[5]);
int lesgpu_autotune(lesgpu_ctx* ctx, int reps, int tiles_out[5], double* ms_out);
/* The scalar pass with its stencil fields staged in shared memory by tensor copies
 * (cp.async.bulk.tensor, a (32 x 8) tile marching through i-planes; the same arithmetic, so
 * the same bits).  Available when a grid row (NZ values) is a multiple of 16 bytes.  Off
 * by default and left alone by lesgpu_autotune: on B200 it is slower than the plain pass
 * (two resident blocks of 112.5 KB shared memory per SM instead of four). */
int lesgpu_set_scalar_staging(lesgpu_ctx* ctx, int enable);
int lesgpu_get_scalar_staging(const lesgpu_ctx* ctx);

/* Block until all work queued on the context's stream has finished. */
int lesgpu_sync(lesgpu_ctx* ctx);

/* No counterpart in the reference (one host thread).  Make `device` the calling host
 * thread's current CUDA device.  lesgpu_create selects the configured device for the thread
 * that calls it; the other calls use the calling thread's current device, so a thread that
 * drives contexts created by another thread calls this first. */
int lesgpu_bind_device(int device);

/* Bytes of device memory the context holds (for admission by memory budget). */
size_t lesgpu_device_bytes(const lesgpu_ctx* ctx);
size_t lesgpu_bytes_for_grid(int nx, int ny, int nz, int precision);

#ifdef __cplusplus
}
#endif

#endif /* LES_GPU_H */
