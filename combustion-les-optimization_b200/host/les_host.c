/*
 * les_host.c -- C host driver of the GPU solver step (include/les_solver.h).
 *
 * Mirrors the host side of the reference's main() (les_combustion_solver.c:4016-4632):
 * start-up state, the glibc rand() stream that drives the SEM vortex recycling and the
 * inflow white noise, the dt formula, and the probe / monitor / checkpoint files.  All
 * floating-point expressions keep the reference's operation order (built with
 * -ffp-contract=off) so the host-side numbers are bit-identical to the reference's.
 */
#include "les_solver.h"

#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ glibc rand() */
/* srand()/rand() of glibc are random_r's TYPE_3 additive feedback generator: 31 words
 * seeded by the Park-Miller LCG (16807 mod 2^31-1, Schrage's method), the recurrence
 * x[i] = x[i-31] + x[i-3] (mod 2^32), 310 discarded outputs, and x[i] >> 1 returned.
 * Restated here with a private state per solver instead of the process-wide one. */

void les_rng_seed(les_rng* g, unsigned int seed) {
    if (seed == 0) seed = 1;
    g->r[0] = (int)seed;
    int word = (int)seed;   /* the seed word is a signed 32-bit value */
    for (int i = 1; i < 31; i++) {
        long long hi = word / 127773;
        long long lo = word % 127773;
        long long nw = 16807 * lo - 2836 * hi;
        if (nw < 0) nw += 2147483647;
        word = (int)nw;
        g->r[i] = word;
    }
    g->f = 3;     /* front tap: x[i-3] lives at (i-3) mod 31 */
    g->b = 0;     /* back tap:  x[i-31] lives at i mod 31 */
    g->n = 0;
    for (int i = 0; i < 310; i++) (void)les_rng_next(g);
    g->n = 0;
}

int les_rng_next(les_rng* g) {
    unsigned int v = (unsigned int)g->r[g->f] + (unsigned int)g->r[g->b];
    g->r[g->f] = (int)v;
    if (++g->f >= 31) g->f = 0;
    if (++g->b >= 31) g->b = 0;
    g->n++;
    return (int)(v >> 1);
}

static double rng01(les_rng* g) { return (double)les_rng_next(g) / (double)LES_RAND_MAX; }

/* ------------------------------------------------------------------ solver object */

#define LES_MAX_LINES 16      /* probe stations + measurement-point stations */

struct les_solver {
    lesgpu_config cfg;
    lesgpu_species sp;
    lesgpu_ctx* ctx;
    les_rng rng;
    int nx, ny, nz;
    size_t n;
    double dx, dy, dz;
    int* attr;
    double* vort;         /* nv x 7 */
    double* noise;        /* 3 x NY x NZ */
    double inletYk[LESGPU_NSP], ambientYk[LESGPU_NSP];
    double stoich_o2, stoich_co2, stoich_h2o;
    int t_loop;
    double dt, umax;
    char out_dir[1024];
    int out_flags;
    int probe_i[7];
    double* probe_buf;    /* LES_MAX_LINES lines of NY x 6 */
    /* measurement points of setup_measurement_points (:3780-3822) and their buffers */
    int npt;
    int pt_i[4], pt_j[4], pt_line[4], pt_count[4];
    double* pt_buf[4];    /* PT_MAX x {u, v, w, G} */
    /* time averages (lesgpu_avg_*) */
    int avg_on, avg_start;
    /* profile statistics on the device (lesgpu_pstat_*) */
    int ps_on;
    /* device-loop session (les_solver_loop_*) */
    int loop_on, l_chunk, l_m, l_lines;
    int l_st[LES_MAX_LINES], l_slot[LES_MAX_LINES];
    double *l_dt, *l_umax, *l_mon, *l_probe;
    char err[256];
};

static int serr(les_solver* s, int code, const char* msg) {
    if (s) snprintf(s->err, sizeof(s->err), "%s", msg);
    return code;
}

static const double PROBE_X[7] = {0.010, 0.015, 0.020, 0.025, 0.030, 0.035, 0.040};   /* :274 */
#define PT_MAX 50000          /* MAX_DATA_POINTS (:199) */

/* initialize_vortices (:861-897): three discarded test draws, then 7 draws per vortex. */
void les_vortices_init(les_rng* g, const lesgpu_config* c, double* vort) {
    (void)les_rng_next(g);
    (void)les_rng_next(g);
    (void)les_rng_next(g);
    double u_rms = c->inlet_velocity * c->turbulence_intensity;
    for (int i = 0; i < c->num_vortices; i++) {
        double r1 = rng01(g), r2 = rng01(g), r3 = rng01(g), r4 = rng01(g);
        double r5 = rng01(g), r6 = rng01(g), r7 = rng01(g);
        double* v = vort + 7 * (size_t)i;
        v[0] = (r1 - 0.5) * c->length_scale;
        v[1] = r2 * c->ly;
        v[2] = r3 * c->lz;
        double min_r = c->length_scale * 0.5, max_r = c->length_scale * 1.5;
        v[3] = min_r + (max_r - min_r) * r4;
        v[4] = (r5 * 2.0 - 1.0) * u_rms;
        v[5] = (r6 * 2.0 - 1.0) * u_rms;
        v[6] = (r7 * 2.0 - 1.0) * u_rms;
    }
}

/* update_vortices (:900-939): advect at U, recycle with 6 draws each in index order. */
void les_vortices_update(les_rng* g, const lesgpu_config* c, double* vort, double dt) {
    double u_rms = c->inlet_velocity * c->turbulence_intensity;
    double box_x = c->length_scale;
    for (int i = 0; i < c->num_vortices; i++) {
        double* v = vort + 7 * (size_t)i;
        v[0] += c->inlet_velocity * dt;
        if (v[0] > box_x / 2.0) {
            v[0] -= box_x;
            double ry = rng01(g), rz = rng01(g);
            v[1] = ry * c->ly;
            v[2] = rz * c->lz;
            double ru = rng01(g), rv = rng01(g), rw = rng01(g);
            v[4] = (ru * 2.0 - 1.0) * u_rms;
            v[5] = (rv * 2.0 - 1.0) * u_rms;
            v[6] = (rw * 2.0 - 1.0) * u_rms;
            double rr = rng01(g);
            double min_r = c->length_scale * 0.5, max_r = c->length_scale * 1.5;
            v[3] = min_r + (max_r - min_r) * rr;
        }
    }
}

/* The inflow white noise of apply_boundary_conditions (:2990-2992): three draws per inlet
 * cell in (j, k) order, mapped to [-1, 1]; non-inlet entries are left untouched. */
void les_inflow_noise(les_rng* g, const int* attr, int ny, int nz, double* noise) {
    const size_t np = (size_t)ny * nz;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            size_t p = (size_t)j * nz + k;
            if (attr[p] != 1) continue;
            noise[p] = ((double)les_rng_next(g) / LES_RAND_MAX) * 2.0 - 1.0;
            noise[np + p] = ((double)les_rng_next(g) / LES_RAND_MAX) * 2.0 - 1.0;
            noise[2 * np + p] = ((double)les_rng_next(g) / LES_RAND_MAX) * 2.0 - 1.0;
        }
}

double les_dt(const lesgpu_config* c, double umax, double numax, double alphamax) {
    double dx = c->lx / (double)c->nx;
    double dt_conv = c->courant * dx / (umax + 1e-10);
    double dt_nu = c->courant_diffusion * (dx * dx) / (numax + 1e-10);
    double dt_al = c->courant_diffusion * (dx * dx) / (alphamax + 1e-10);
    return fmin(dt_conv, fmin(dt_nu, dt_al));
}

/* initialize() + setting() (:1085-1285): attribute map (symmetry code 5 on j = 0) and the
 * initial burnt/unburnt state with rho from the equation of state. */
int les_initial_state(const lesgpu_config* c, const lesgpu_species* sp, int* attr, double* const* f) {
    if (!c || !sp || !attr || !f) return LESGPU_EINVAL;
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const double dy = c->ly / (double)ny, dz = c->lz / (double)nz;
    /* inlet composition and stoichiometry (:4101-4120) */
    double inletYk[LESGPU_NSP], ambientYk[LESGPU_NSP] = {0.0, 0.232, 0.768, 0.0, 0.0};
    const double phi = c->equivalence_ratio;
    double m_f = 1.0, m_o2 = 5.0 / phi, m_n2 = m_o2 * 3.76;
    double mass_total = m_f * sp->mw[0] + m_o2 * sp->mw[1] + m_n2 * sp->mw[2];
    inletYk[0] = (m_f * sp->mw[0]) / mass_total;
    inletYk[1] = (m_o2 * sp->mw[1]) / mass_total;
    inletYk[2] = (m_n2 * sp->mw[2]) / mass_total;
    inletYk[3] = 0.0; inletYk[4] = 0.0;
    const double st_o2 = (5.0 * sp->mw[1]) / sp->mw[0];
    const double st_co2 = (3.0 * sp->mw[3]) / sp->mw[0];
    const double st_h2o = (4.0 * sp->mw[4]) / sp->mw[0];
    const double icy = 0.0, icz = c->lz / 2.0;
#define CIDX(i, j, k) (((size_t)(i) * (size_t)ny + (size_t)(j)) * (size_t)nz + (size_t)(k))
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                int a;
                if (i == 0) {
                    double y = j * dy, z = k * dz;
                    double d2 = pow(y - icy, 2) + pow(z - icz, 2);
                    if (d2 <= pow(c->inlet_radius, 2)) a = 1;
                    else if (d2 <= pow(c->rim_outer_radius, 2)) a = 6;
                    else a = 4;
                } else if (i == nx - 1) a = 2;
                else if (j == 0) a = 5;
                else if (j == ny - 1 || k == 0 || k == nz - 1) a = 4;
                else a = 3;
                attr[CIDX(i, j, k)] = a;
            }
    double *u = f[0], *v = f[1], *w = f[2], *T = f[3], *G = f[4], *rho = f[5];
    double* const* Y = f + 6;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                size_t id = CIDX(i, j, k);
                u[id] = v[id] = w[id] = 0.0;
                T[id] = 0.0; G[id] = 0.0;
                for (int q = 0; q < LESGPU_NSP; q++) Y[q][id] = 0.0;
                switch (attr[id]) {
                    case 1:
                        u[id] = c->inlet_velocity;
                        T[id] = c->inlet_temperature;
                        for (int q = 0; q < LESGPU_NSP; q++) Y[q][id] = inletYk[q];
                        break;
                    case 4:
                    case 2:
                        T[id] = c->ambient_temperature;
                        for (int q = 0; q < LESGPU_NSP; q++) Y[q][id] = ambientYk[q];
                        break;
                    case 5:
                    case 3:
                        if (i <= c->initial_flame_front_i) {
                            G[id] = 1.0;
                            T[id] = c->burnt_gas_temperature;
                            double cons = inletYk[0];
                            Y[0][id] = inletYk[0] - cons;
                            Y[1][id] = inletYk[1] - cons * st_o2;
                            Y[2][id] = inletYk[2];
                            Y[3][id] = inletYk[3] + cons * st_co2;
                            Y[4][id] = inletYk[4] + cons * st_h2o;
                        } else {
                            T[id] = c->inlet_temperature;
                            for (int q = 0; q < LESGPU_NSP; q++) Y[q][id] = inletYk[q];
                        }
                        break;
                    default:
                        break;
                }
                double syw = 0.0;
                for (int q = 0; q < LESGPU_NSP; q++) syw += Y[q][id] / (sp->mw[q] / 1000.0);
                if (syw > 1e-10 && T[id] > 1.0) {
                    double W = 1.0 / syw;
                    double Rm = 8.314462 / W;
                    rho[id] = 101325.0 / (Rm * T[id]);
                } else {
                    rho[id] = 1.2;
                }
            }
#undef CIDX
    return LESGPU_OK;
}

static int alloc_fields(size_t n, double** f) {
    for (int q = 0; q < LESGPU_NSTATE; q++) {
        f[q] = (double*)malloc(n * sizeof(double));
        if (!f[q]) {
            for (int r = 0; r < q; r++) free(f[r]);
            return -1;
        }
    }
    return 0;
}

static void free_fields(double** f) {
    for (int q = 0; q < LESGPU_NSTATE; q++) free(f[q]);
}

int les_solver_create(const lesgpu_config* cfg, const char* chem_path, const char* tran_path, int start_step,
                      les_solver** out) {
    if (!cfg || !chem_path || !tran_path || !out) return LESGPU_EINVAL;
    *out = NULL;
    les_solver* s = (les_solver*)calloc(1, sizeof(les_solver));
    if (!s) return LESGPU_ENOMEM;
    s->cfg = *cfg;
    int rc = lesgpu_load_species(chem_path, tran_path, &s->sp);
    if (rc) { free(s); return rc; }
    s->nx = cfg->nx; s->ny = cfg->ny; s->nz = cfg->nz;
    s->n = (size_t)s->nx * s->ny * s->nz;
    s->dx = cfg->lx / (double)cfg->nx;
    s->dy = cfg->ly / (double)cfg->ny;
    s->dz = cfg->lz / (double)cfg->nz;
    /* inlet composition and stoichiometry (:4101-4120) */
    const double phi = cfg->equivalence_ratio;
    double m_f = 1.0, m_o2 = 5.0 / phi, m_n2 = m_o2 * 3.76;
    double mass_total = m_f * s->sp.mw[0] + m_o2 * s->sp.mw[1] + m_n2 * s->sp.mw[2];
    s->inletYk[0] = (m_f * s->sp.mw[0]) / mass_total;
    s->inletYk[1] = (m_o2 * s->sp.mw[1]) / mass_total;
    s->inletYk[2] = (m_n2 * s->sp.mw[2]) / mass_total;
    s->inletYk[3] = 0.0; s->inletYk[4] = 0.0;
    s->ambientYk[0] = 0.0; s->ambientYk[1] = 0.232; s->ambientYk[2] = 0.768; s->ambientYk[3] = 0.0; s->ambientYk[4] = 0.0;
    s->stoich_o2 = (5.0 * s->sp.mw[1]) / s->sp.mw[0];
    s->stoich_co2 = (3.0 * s->sp.mw[3]) / s->sp.mw[0];
    s->stoich_h2o = (4.0 * s->sp.mw[4]) / s->sp.mw[0];
    s->attr = (int*)malloc(s->n * sizeof(int));
    s->vort = (double*)calloc(cfg->num_vortices > 0 ? (size_t)cfg->num_vortices * 7 : 7, sizeof(double));
    s->noise = (double*)calloc(3 * (size_t)s->ny * s->nz, sizeof(double));
    s->probe_buf = (double*)malloc(LES_MAX_LINES * (size_t)s->ny * 6 * sizeof(double));
    if (!s->attr || !s->vort || !s->noise || !s->probe_buf) {
        les_solver_destroy(s);
        return LESGPU_ENOMEM;
    }
    double* f[LESGPU_NSTATE];
    if (alloc_fields(s->n, f)) { les_solver_destroy(s); return LESGPU_ENOMEM; }
    les_initial_state(cfg, &s->sp, s->attr, f);
    rc = lesgpu_create(cfg, &s->sp, &s->ctx);
    if (rc == LESGPU_OK) rc = lesgpu_upload_attribute(s->ctx, s->attr);
    if (rc == LESGPU_OK) rc = lesgpu_upload_state(s->ctx, (const double* const*)f, LESGPU_NSTATE);
    free_fields(f);
    if (rc) {
        if (s->ctx) snprintf(s->err, sizeof(s->err), "%s", lesgpu_last_error(s->ctx));
        les_solver_destroy(s);
        return rc;
    }
    /* srand(seed) + initialize_vortices (:4085, :4360) and the inlet mask (:4366-4367) */
    les_rng_seed(&s->rng, cfg->seed);
    les_vortices_init(&s->rng, cfg, s->vort);
    for (int q = 0; q < 7; q++) s->probe_i[q] = (int)(PROBE_X[q] / s->dx);
    /* setup_measurement_points (:3780-3822): at 4D and 8D downstream (D = 2 x inlet radius),
     * on the axis (j = 0) and in the shear layer (j = R / DY), k = NZ/2 */
    {
        const int j_shear = (int)(cfg->inlet_radius / s->dy);
        const int i_locs[2] = {(int)((4.0 * cfg->inlet_radius) / s->dx), (int)((8.0 * cfg->inlet_radius) / s->dx)};
        s->npt = 0;
        for (int q = 0; q < 2; q++) {
            if (i_locs[q] >= s->nx) continue;
            s->pt_i[s->npt] = i_locs[q]; s->pt_j[s->npt] = 0; s->npt++;
            s->pt_i[s->npt] = i_locs[q]; s->pt_j[s->npt] = j_shear; s->npt++;
        }
    }
    s->t_loop = start_step;
    *out = s;
    return LESGPU_OK;
}

static void flush_points(les_solver* s);

void les_solver_destroy(les_solver* s) {
    if (!s) return;
    if (s->loop_on) les_solver_loop_end(s);
    flush_points(s);
    if (s->ctx) lesgpu_destroy(s->ctx);
    free(s->attr); free(s->vort); free(s->noise); free(s->probe_buf);
    for (int q = 0; q < 4; q++) free(s->pt_buf[q]);
    free(s);
}

lesgpu_ctx* les_solver_ctx(les_solver* s) { return s ? s->ctx : NULL; }
const char* les_solver_last_error(const les_solver* s) { return s ? s->err : "null solver"; }
int les_solver_t_loop(const les_solver* s) { return s ? s->t_loop : -1; }
double les_solver_last_dt(const les_solver* s) { return s ? s->dt : 0.0; }
double les_solver_last_umax(const les_solver* s) { return s ? s->umax : 0.0; }
unsigned long long les_solver_rng_draws(const les_solver* s) { return s ? s->rng.n : 0; }

int les_solver_attribute(const les_solver* s, int* out) {
    if (!s || !out) return LESGPU_EINVAL;
    memcpy(out, s->attr, s->n * sizeof(int));
    return LESGPU_OK;
}

int les_solver_vortices(const les_solver* s, double* out) {
    if (!s || !out) return LESGPU_EINVAL;
    memcpy(out, s->vort, (size_t)s->cfg.num_vortices * 7 * sizeof(double));
    return s->cfg.num_vortices;
}

static void join_path(char* dst, size_t cap, const char* dir, const char* name) {
    snprintf(dst, cap, "%s/%s", dir, name);
}

static int write_vtk_step(les_solver* s, int t);

int les_solver_set_outputs(les_solver* s, const char* dir, int flags) {
    if (!s || (flags && !dir)) return LESGPU_EINVAL;
    if (s->loop_on && ((flags ^ s->out_flags) & LES_OUT_VTK))
        return serr(s, LESGPU_ESTATE, "end the device loop before switching VTK output");
    if ((flags & LES_OUT_VTK) != (s->out_flags & LES_OUT_VTK)) {
        int rc = lesgpu_keep_grad_g(s->ctx, (flags & LES_OUT_VTK) ? 1 : 0);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    }
    if ((flags & LES_OUT_PSTAT) && !s->ps_on) {
        int rc = les_solver_pstat_begin(s, NULL, 0, NULL, 0, NULL, 0, NULL, NULL, 0);
        if (rc) return rc;
    }
    s->out_flags = flags;
    if (!dir) return LESGPU_OK;
    snprintf(s->out_dir, sizeof(s->out_dir), "%s", dir);
    if (flags & LES_OUT_PROBES) {
        for (int n = 0; n < 7; n++) {
            char name[128], path[1200];
            snprintf(name, sizeof(name), "probe_data_flame_region_loc%d.csv", n);
            join_path(path, sizeof(path), s->out_dir, name);
            remove(path);
            FILE* fp = fopen(path, "w");
            if (!fp) return serr(s, LESGPU_EIO, "cannot create probe file");
            fprintf(fp, "timestep,x_location,y_flame,y_physical,y_relative,u,v,w,G,nu_t,S_mag\n");
            fclose(fp);
        }
    }
    return LESGPU_OK;
}

/* The x-stations that record_flame_region_data keeps (0 < i < NX-1), with their slot n. */
static int probe_stations(const les_solver* s, int* st, int* slot) {
    int m = 0;
    for (int n = 0; n < 7; n++) {
        int ip = s->probe_i[n];
        if (ip <= 0 || ip >= s->nx - 1) continue;
        st[m] = ip;
        slot[m] = n;
        m++;
    }
    return m;
}

/* record_flame_region_data (:3403-3471): the lower G = 0.5 crossing on the line k = NZ/2
 * at each x-station, then every row within SAMPLING_RANGE (1.0 m, i.e. all rows).
 * lines holds m stations x NY x {u, v, w, G, nu_t, S_mag}. */
static void append_probe_rows(les_solver* s, int t_loop, const double* lines, int m, const int* slot) {
    for (int q = 0; q < m; q++) {
        const double* row = lines + (size_t)q * s->ny * 6;
        double y_flame = -1.0;
        for (int j = 0; j < s->ny - 1; j++) {
            double G1 = row[6 * j + 3], G2 = row[6 * (j + 1) + 3];
            if ((G1 - 0.5) * (G2 - 0.5) <= 0.0) {
                double y1 = j * s->dy, y2 = (j + 1) * s->dy;
                if (fabs(G2 - G1) < 1e-9) y_flame = y1;
                else y_flame = y1 + (0.5 - G1) / (G2 - G1) * (y2 - y1);
                break;
            }
        }
        if (!(y_flame > 0.0)) continue;
        char name[128], path[1200];
        snprintf(name, sizeof(name), "probe_data_flame_region_loc%d.csv", slot[q]);
        join_path(path, sizeof(path), s->out_dir, name);
        FILE* fp = fopen(path, "a");
        if (!fp) continue;
        for (int j = 0; j < s->ny; j++) {
            double yp = j * s->dy, yr = yp - y_flame;
            if (fabs(yr) <= 1.000) {
                const double* r = row + 6 * j;
                fprintf(fp, "%d,%.3f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6e,%.6e\n", t_loop, PROBE_X[slot[q]], y_flame, yp,
                        yr, r[0], r[1], r[2], r[3], r[4], r[5]);
            }
        }
        fclose(fp);
    }
}

/* The lines read back each step: the m probe stations first, then one line per distinct
 * measurement-point station (pt_line maps each point to its line).  Returns the count. */
static int line_stations(les_solver* s, int* st, int* slot, int* m_out) {
    int m = probe_stations(s, st, slot);
    int L = m;
    for (int p = 0; p < s->npt; p++) {
        int found = -1;
        for (int q = m; q < L; q++)
            if (st[q] == s->pt_i[p]) found = q;
        if (found < 0 && L < LES_MAX_LINES) { st[L] = s->pt_i[p]; slot[L] = -1; found = L++; }
        s->pt_line[p] = found;
    }
    *m_out = m;
    return L;
}

/* flush_point_data (:3824-3850): append the buffered rows, then empty the buffers. */
static void flush_points(les_solver* s) {
    if (!(s->out_flags & LES_OUT_POINTS) || !s->out_dir[0]) return;
    for (int p = 0; p < s->npt; p++) {
        if (s->pt_count[p] == 0 || !s->pt_buf[p]) continue;
        char name[160], path[1300];
        snprintf(name, sizeof(name), "LES_point_data_phi%.2f_i%d_j%d_k%d.csv", s->cfg.equivalence_ratio, s->pt_i[p],
                 s->pt_j[p], s->nz / 2);
        join_path(path, sizeof(path), s->out_dir, name);
        FILE* fp = fopen(path, "a");
        if (!fp) continue;
        fseek(fp, 0, SEEK_END);
        if (ftell(fp) == 0) fprintf(fp, "u,v,w,G\n");
        const double* b = s->pt_buf[p];
        for (int q = 0; q < s->pt_count[p]; q++)
            fprintf(fp, "%.6f,%.6f,%.6f,%.6f\n", b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]);
        fclose(fp);
        s->pt_count[p] = 0;
    }
}

/* The point buffer of the time loop (:4557-4568): u, v, w, G of every point after the BC. */
static void record_points(les_solver* s, const double* lines) {
    for (int p = 0; p < s->npt; p++) {
        if (s->pt_line[p] < 0 || s->pt_count[p] >= PT_MAX) continue;
        if (!s->pt_buf[p]) {
            s->pt_buf[p] = (double*)malloc((size_t)PT_MAX * 4 * sizeof(double));
            if (!s->pt_buf[p]) continue;
        }
        const double* r = lines + ((size_t)s->pt_line[p] * s->ny + s->pt_j[p]) * 6;
        double* b = s->pt_buf[p] + 4 * (size_t)s->pt_count[p];
        b[0] = r[0]; b[1] = r[1]; b[2] = r[2]; b[3] = r[3];
        s->pt_count[p]++;
    }
}

static int write_probes(les_solver* s, int t_loop) {
    int st[LES_MAX_LINES], slot[LES_MAX_LINES], m;
    int L = line_stations(s, st, slot, &m);
    if (L == 0) return LESGPU_OK;
    int rc = lesgpu_probe_lines(s->ctx, st, L, s->nz / 2, s->probe_buf);
    if (rc) return rc;
    if ((s->out_flags & LES_OUT_PROBES) && m > 0) append_probe_rows(s, t_loop, s->probe_buf, m, slot);
    if (s->out_flags & LES_OUT_POINTS) record_points(s, s->probe_buf);
    return LESGPU_OK;
}

static void append_monitor_row(les_solver* s, int step, double dt, const double* m) {
    char path[1200];
    join_path(path, sizeof(path), s->out_dir, "simulation_monitor.csv");
    FILE* fp = fopen(path, "a");
    if (!fp) return;
    fseek(fp, 0, SEEK_END);
    if (ftell(fp) == 0) fprintf(fp, "step,dt,total_mass,min_T,max_T,min_G,max_G,min_Y_C3H8\n");
    fprintf(fp, "%d,%.6e,%.6e,%.2f,%.2f,%.4f,%.4f,%.2e\n", step, dt, m[0], m[1], m[2], m[3], m[4], m[5]);
    fclose(fp);
}

/* write_monitor_log (:3874-3924), every 10 steps */
static int write_monitor(les_solver* s, int step, double dt) {
    if (step % 10 != 0) return LESGPU_OK;
    double m[6];
    int rc = lesgpu_monitor(s->ctx, m);
    if (rc) return rc;
    append_monitor_row(s, step, dt, m);
    return LESGPU_OK;
}

/* The checkpoint block of the time loop (:4583-4589) at t > 0, t % 50 == 0:
 * checkpoint.bin + restart_info.txt, stats_backup.bin (time averages on), point data. */
static int checkpoint_step(les_solver* s, int t) {
    if (!(t > 0 && t % 50 == 0) || !s->out_dir[0]) return LESGPU_OK;
    if (s->out_flags & LES_OUT_CHECKPOINT) {
        char path[1200];
        join_path(path, sizeof(path), s->out_dir, "checkpoint.bin");
        int rc = les_solver_save_checkpoint(s, path, t);
        if (rc) return rc;
        if (s->avg_on) {
            join_path(path, sizeof(path), s->out_dir, "stats_backup.bin");
            rc = les_solver_save_stats(s, path);
            if (rc) return rc;
        }
    }
    flush_points(s);
    return LESGPU_OK;
}

int les_solver_step(les_solver* s) {
    if (!s) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "end the device loop before host-driven steps");
    const lesgpu_config* c = &s->cfg;
    /* dt (:4399-4411) */
    double umax, numax, alphamax;
    int rc = lesgpu_dt_inputs(s->ctx, &umax, &numax, &alphamax);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    double dt = les_dt(c, umax, numax, alphamax);
    s->dt = dt;
    s->umax = umax;
    /* SEM vortices for this step, then the inflow noise drawn after the RK stages (:4414, :2990) */
    les_vortices_update(&s->rng, c, s->vort, dt);
    les_inflow_noise(&s->rng, s->attr, s->ny, s->nz, s->noise);
    rc = lesgpu_set_inflow(s->ctx, s->vort, c->num_vortices, s->noise);
    if (rc == LESGPU_OK) rc = lesgpu_step(s->ctx, dt, s->t_loop);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    if ((s->out_flags & (LES_OUT_PROBES | LES_OUT_POINTS)) && s->out_dir[0]) {
        rc = write_probes(s, s->t_loop);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    }
    rc = checkpoint_step(s, s->t_loop);
    if (rc) return rc;
    if ((s->out_flags & LES_OUT_MONITOR) && s->out_dir[0]) {
        rc = write_monitor(s, s->t_loop, dt);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    }
    if (s->t_loop > 0 && s->t_loop % 500 == 0) {
        rc = write_vtk_step(s, s->t_loop);
        if (rc) return rc;
    }
    s->t_loop++;
    return LESGPU_OK;
}

/* The same time loop with the host side on the GPU (lesgpu_loop_*): steps are queued in
 * chunks without a host round trip; between chunks the probe and monitor rows are written
 * from the step history, and checkpoints fall on chunk boundaries. */
static void loop_free(les_solver* s) {
    free(s->l_dt); free(s->l_umax); free(s->l_mon); free(s->l_probe);
    s->l_dt = s->l_umax = s->l_mon = s->l_probe = NULL;
}

int les_solver_loop_begin(les_solver* s, int chunk) {
    if (!s) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "device loop already running");
    if (chunk <= 0) chunk = 64;
    unsigned int win[31];
    for (int j = 0; j < 31; j++) win[j] = (unsigned int)s->rng.r[(s->rng.f + j) % 31];
    int rc = lesgpu_loop_begin(s->ctx, win, s->vort, s->cfg.num_vortices, s->t_loop);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    s->l_lines = line_stations(s, s->l_st, s->l_slot, &s->l_m);
    rc = lesgpu_loop_config(s->ctx, s->l_st, s->l_lines, s->nz / 2, chunk);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    s->l_chunk = chunk;
    s->l_dt = (double*)malloc((size_t)chunk * sizeof(double));
    s->l_umax = (double*)malloc((size_t)chunk * sizeof(double));
    s->l_mon = (double*)malloc((size_t)chunk * 6 * sizeof(double));
    s->l_probe = (double*)malloc((size_t)chunk * (s->l_lines > 0 ? s->l_lines : 1) * s->ny * 6 * sizeof(double));
    if (!s->l_dt || !s->l_umax || !s->l_mon || !s->l_probe) {
        loop_free(s);
        return serr(s, LESGPU_ENOMEM, "host history buffers");
    }
    s->loop_on = 1;
    return LESGPU_OK;
}

/* Length of the next chunk of a session with `left` steps to go: at most the history
 * capacity, and ending on the next checkpoint step (t > 0, t % 50 == 0) when checkpoints
 * are written. */
int les_solver_next_chunk(const les_solver* s, int left) {
    if (!s || left <= 0 || !s->loop_on) return 0;
    int n = left < s->l_chunk ? left : s->l_chunk;
    const int ck = (s->out_flags & LES_OUT_CHECKPOINT) && s->out_dir[0];
    const int vtk = (s->out_flags & LES_OUT_VTK) && s->out_dir[0];
    if (ck || vtk) {
        for (int q = 0; q < n; q++) {
            int t = s->t_loop + q;
            if ((ck && t > 0 && t % 50 == 0) || (vtk && t > 0 && t % 500 == 0)) { n = q + 1; break; }
        }
    }
    return n;
}

/* After n queued device-loop steps: read the step history back, write the probe and
 * monitor rows, advance t_loop and write the checkpoint that ends the chunk. */
int les_solver_loop_collect(les_solver* s, int n) {
    if (!s || n < 0) return LESGPU_EINVAL;
    if (!s->loop_on) return serr(s, LESGPU_ESTATE, "les_solver_loop_begin first");
    if (n > s->l_chunk) return serr(s, LESGPU_EINVAL, "more steps than the history holds");
    if (n == 0) return LESGPU_OK;
    const int want_probes = (s->out_flags & LES_OUT_PROBES) && s->out_dir[0];
    const int want_points = (s->out_flags & LES_OUT_POINTS) && s->out_dir[0];
    const int want_mon = (s->out_flags & LES_OUT_MONITOR) && s->out_dir[0];
    const int m = s->l_m, L = s->l_lines;
    int rc = lesgpu_loop_history(s->ctx, n, s->l_dt, s->l_umax, (want_probes || want_points) ? s->l_probe : NULL,
                                 want_mon ? s->l_mon : NULL);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    /* the rows of this chunk into the device statistics, before the next chunk reuses the slots */
    if (s->ps_on && m > 0) {
        rc = lesgpu_pstat_accumulate(s->ctx, n, m);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    }
    for (int q = 0; q < n; q++) {
        const int t = s->t_loop + q;
        const double* lines = s->l_probe + (size_t)q * L * s->ny * 6;
        if (want_probes && m > 0) append_probe_rows(s, t, lines, m, s->l_slot);
        if (want_points) {
            record_points(s, lines);
            if (t > 0 && t % 50 == 0) flush_points(s);
        }
        if (want_mon && t % 10 == 0) append_monitor_row(s, t, s->l_dt[q], s->l_mon + 6 * (size_t)q);
    }
    s->dt = s->l_dt[n - 1];
    s->umax = s->l_umax[n - 1];
    s->t_loop += n;
    /* checkpoint.bin and stats_backup.bin need the state of their step: les_solver_next_chunk
     * ends every chunk on a checkpoint step when checkpoints are written */
    const int tl = s->t_loop - 1;
    if ((s->out_flags & LES_OUT_CHECKPOINT) && s->out_dir[0] && tl > 0 && tl % 50 == 0) {
        char path[1200];
        join_path(path, sizeof(path), s->out_dir, "checkpoint.bin");
        rc = les_solver_save_checkpoint(s, path, tl);
        if (rc) return rc;
        if (s->avg_on) {
            join_path(path, sizeof(path), s->out_dir, "stats_backup.bin");
            rc = les_solver_save_stats(s, path);
            if (rc) return rc;
        }
    }
    if (tl > 0 && tl % 500 == 0) {
        rc = write_vtk_step(s, tl);
        if (rc) return rc;
    }
    return LESGPU_OK;
}

int les_solver_loop_run(les_solver* s, int nsteps) {
    if (!s || nsteps < 0) return LESGPU_EINVAL;
    if (!s->loop_on) return serr(s, LESGPU_ESTATE, "les_solver_loop_begin first");
    int left = nsteps;
    while (left > 0) {
        const int n = les_solver_next_chunk(s, left);
        int rc = lesgpu_run(s->ctx, n);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
        rc = les_solver_loop_collect(s, n);
        if (rc) return rc;
        left -= n;
    }
    return LESGPU_OK;
}

int les_solver_loop_end(les_solver* s) {
    if (!s) return LESGPU_EINVAL;
    if (!s->loop_on) return LESGPU_OK;
    unsigned int win[31];
    int t_back = 0;
    int rc = lesgpu_loop_end(s->ctx, win, s->vort, &t_back);
    s->loop_on = 0;
    loop_free(s);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    for (int j = 0; j < 31; j++) s->rng.r[j] = (int)win[j];
    s->rng.f = 0;
    s->rng.b = 28;
    return LESGPU_OK;
}

int les_solver_run_device(les_solver* s, int nsteps, int chunk) {
    if (!s || nsteps < 0) return LESGPU_EINVAL;
    if (nsteps == 0) return LESGPU_OK;
    int rc = les_solver_loop_begin(s, chunk);
    if (rc) return rc;
    rc = les_solver_loop_run(s, nsteps);
    int rc2 = les_solver_loop_end(s);
    return rc ? rc : rc2;
}

int les_solver_run(les_solver* s, int nsteps) {
    for (int q = 0; q < nsteps; q++) {
        int rc = les_solver_step(s);
        if (rc) return rc;
    }
    return lesgpu_sync(s->ctx);
}

int les_solver_save_checkpoint(les_solver* s, const char* path, int t) {
    if (!s || !path) return LESGPU_EINVAL;
    double* f[LESGPU_NSTATE];
    if (alloc_fields(s->n, f)) return LESGPU_ENOMEM;
    int rc = lesgpu_download_state(s->ctx, (double* const*)f, LESGPU_NSTATE);
    if (rc) { free_fields(f); return serr(s, rc, lesgpu_last_error(s->ctx)); }
    FILE* fp = fopen(path, "wb");
    if (!fp) { free_fields(f); return serr(s, LESGPU_EIO, "cannot open checkpoint for writing"); }
    int ok = fwrite(&t, sizeof(int), 1, fp) == 1;
    for (int q = 0; q < LESGPU_NSTATE && ok; q++) ok = fwrite(f[q], sizeof(double), s->n, fp) == s->n;
    fclose(fp);
    free_fields(f);
    if (!ok) return serr(s, LESGPU_EIO, "short checkpoint write");
    /* restart_info.txt next to the checkpoint (:3691-3697) */
    char info[1200];
    snprintf(info, sizeof(info), "%s", path);
    char* slash = strrchr(info, '/');
    if (slash) snprintf(slash + 1, sizeof(info) - (size_t)(slash + 1 - info), "restart_info.txt");
    else snprintf(info, sizeof(info), "restart_info.txt");
    FILE* fi = fopen(info, "w");
    if (fi) {
        fprintf(fi, "BINARY\n%d\n", t);
        fclose(fi);
    }
    return LESGPU_OK;
}

int les_solver_load_checkpoint(les_solver* s, const char* path, int* t_out) {
    if (!s || !path) return LESGPU_EINVAL;
    FILE* fp = fopen(path, "rb");
    if (!fp) return serr(s, LESGPU_EIO, "cannot open checkpoint");
    fseek(fp, 0, SEEK_END);
    long sz = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    long want = (long)sizeof(int) + (long)(LESGPU_NSTATE * s->n * sizeof(double));
    if (sz != want) { fclose(fp); return serr(s, LESGPU_EIO, "checkpoint size does not match the grid"); }
    int t = 0;
    double* f[LESGPU_NSTATE];
    if (alloc_fields(s->n, f)) { fclose(fp); return LESGPU_ENOMEM; }
    int ok = fread(&t, sizeof(int), 1, fp) == 1;
    for (int q = 0; q < LESGPU_NSTATE && ok; q++) ok = fread(f[q], sizeof(double), s->n, fp) == s->n;
    fclose(fp);
    if (!ok) { free_fields(f); return serr(s, LESGPU_EIO, "short checkpoint read"); }
    for (int q = 0; q < LESGPU_NSTATE && ok; q++)
        for (size_t i = 0; i < s->n; i++)
            if (!isfinite(f[q][i])) { ok = 0; break; }
    if (!ok) { free_fields(f); return serr(s, LESGPU_ENONFINITE, "checkpoint holds non-finite values"); }
    int rc = lesgpu_upload_state(s->ctx, (const double* const*)f, LESGPU_NSTATE);
    free_fields(f);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    if (t_out) *t_out = t;
    return LESGPU_OK;
}

/* ------------------------------------------------------------------ device profile statistics */

int les_solver_pstat_begin(les_solver* s, const double* y_edges_mm, int n_y, const double* g_rc_edges, int n_grc,
                           const double* g_ho_edges, int n_gho, const double* u_edges, const double* v_edges,
                           int n_pdf) {
    if (!s) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "end the device loop before starting the statistics");
    int rc;
    if (y_edges_mm && g_rc_edges && g_ho_edges && u_edges && v_edges) {
        rc = lesgpu_pstat_begin(s->ctx, y_edges_mm, n_y, g_rc_edges, n_grc, g_ho_edges, n_gho, u_edges, v_edges, n_pdf);
    } else {
        /* defaults; edges are start + b * step, as numpy's arange and linspace compute them */
        const double ly_mm = 1000.0 * s->cfg.ly, U = s->cfg.inlet_velocity;
        const int ny_b = (int)(2.0 * ly_mm / 0.5 + 0.5), ng = 20, np_ = 40;
        double* e = (double*)malloc((size_t)(ny_b + 1 + 2 * (ng + 1) + 2 * (np_ + 1)) * sizeof(double));
        if (!e) return serr(s, LESGPU_ENOMEM, "host buffers");
        double *ey = e, *erc = ey + ny_b + 1, *eho = erc + ng + 1, *eu = eho + ng + 1, *ev = eu + np_ + 1;
        for (int b = 0; b <= ny_b; b++) ey[b] = -ly_mm + b * 0.5;
        for (int b = 0; b <= ng; b++) erc[b] = b * 0.05;
        for (int b = 0; b < ng; b++) eho[b] = b * (1.0 / ng);
        eho[ng] = 1.0;
        for (int b = 0; b < np_; b++) { eu[b] = -U + b * (4.0 * U / np_); ev[b] = -2.0 * U + b * (4.0 * U / np_); }
        eu[np_] = 3.0 * U;
        ev[np_] = 2.0 * U;
        rc = lesgpu_pstat_begin(s->ctx, ey, ny_b, erc, ng, eho, ng, eu, ev, np_);
        free(e);
    }
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    s->ps_on = 1;
    return LESGPU_OK;
}

size_t les_solver_pstat_size(const les_solver* s) { return (s && s->ps_on) ? lesgpu_pstat_size(s->ctx) : 0; }

int les_solver_pstat_write(les_solver* s, const char* path) {
    if (!s || !path) return LESGPU_EINVAL;
    if (!s->ps_on) return serr(s, LESGPU_ESTATE, "les_solver_pstat_begin first");
    int32_t hdr[5] = {0x53505350, 0, 0, 0, 0};
    size_t ne = 0;
    int rc = lesgpu_pstat_layout(s->ctx, &hdr[1], &hdr[2], &hdr[3], &hdr[4], NULL, &ne);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    const size_t ns = lesgpu_pstat_size(s->ctx);
    double* buf = (double*)malloc((ne + ns) * sizeof(double));
    if (!buf) return serr(s, LESGPU_ENOMEM, "host buffers");
    rc = lesgpu_pstat_layout(s->ctx, NULL, NULL, NULL, NULL, buf, &ne);
    if (rc == LESGPU_OK) rc = lesgpu_pstat_read(s->ctx, buf + ne);
    if (rc) { free(buf); return serr(s, rc, lesgpu_last_error(s->ctx)); }
    FILE* fp = fopen(path, "wb");
    if (!fp) { free(buf); return serr(s, LESGPU_EIO, "cannot open profile_stats.bin for writing"); }
    const int ok = fwrite(hdr, sizeof hdr, 1, fp) == 1 && fwrite(buf, sizeof(double), ne + ns, fp) == ne + ns;
    fclose(fp);
    free(buf);
    return ok ? LESGPU_OK : serr(s, LESGPU_EIO, "short profile_stats.bin write");
}

int les_solver_pstat_read(les_solver* s, double* out) {
    if (!s || !out) return LESGPU_EINVAL;
    if (!s->ps_on) return serr(s, LESGPU_ESTATE, "les_solver_pstat_begin first");
    int rc = lesgpu_pstat_read(s->ctx, out);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    return LESGPU_OK;
}

/* ------------------------------------------------------------------ end of run and resume */

#define LES_RESUME_MAGIC 0x5253454cu   /* "LESR" */

/* les_resume.bin: magic, nv, t_loop, the rand() state, the nu/alpha maxima, nv x 7 vortices. */
static int write_resume_sidecar(les_solver* s, const char* path) {
    double umax = 0.0, numax = 0.0, amax = 0.0;
    int rc = lesgpu_dt_inputs(s->ctx, &umax, &numax, &amax);
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    FILE* fp = fopen(path, "wb");
    if (!fp) return serr(s, LESGPU_EIO, "cannot open les_resume.bin for writing");
    const unsigned int magic = LES_RESUME_MAGIC;
    const int nv = s->cfg.num_vortices, t = s->t_loop;
    const size_t nvd = (size_t)(nv > 0 ? nv : 0) * 7;
    int ok = fwrite(&magic, sizeof magic, 1, fp) == 1 && fwrite(&nv, sizeof nv, 1, fp) == 1 &&
             fwrite(&t, sizeof t, 1, fp) == 1 && fwrite(&s->rng, sizeof s->rng, 1, fp) == 1 &&
             fwrite(&numax, sizeof numax, 1, fp) == 1 && fwrite(&amax, sizeof amax, 1, fp) == 1 &&
             (nvd == 0 || fwrite(s->vort, sizeof(double), nvd, fp) == nvd);
    fclose(fp);
    return ok ? LESGPU_OK : serr(s, LESGPU_EIO, "short les_resume.bin write");
}

int les_solver_finish(les_solver* s, const char* dir, int mode) {
    if (!s || !dir || (mode != LES_RESUME_REFERENCE && mode != LES_RESUME_FIXED)) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "end the device loop first");
    int rc = les_solver_flush(s);
    if (rc) return rc;
    char path[1200];
    /* save_quick_checkpoint(0) (:4623) -- or the step reached */
    join_path(path, sizeof(path), dir, "checkpoint.bin");
    rc = les_solver_save_checkpoint(s, path, mode == LES_RESUME_FIXED ? s->t_loop : 0);
    if (rc) return rc;
    if (s->avg_on) {                                   /* save_statistics_backup (:4624) */
        join_path(path, sizeof(path), dir, "stats_backup.bin");
        rc = les_solver_save_stats(s, path);
        if (rc) return rc;
    }
    join_path(path, sizeof(path), dir, "les_resume.bin");
    if (mode == LES_RESUME_FIXED) return write_resume_sidecar(s, path);
    remove(path);                 /* no stale sidecar beside a reference-mode checkpoint */
    return LESGPU_OK;
}

int les_solver_resume(les_solver* s, const char* dir, int mode, int* t_out) {
    if (!s || !dir || (mode != LES_RESUME_REFERENCE && mode != LES_RESUME_FIXED)) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "end the device loop first");
    char path[1200], line[256];
    /* restart detection (:4150-4181): "BINARY" then the step on the next line */
    join_path(path, sizeof(path), dir, "restart_info.txt");
    FILE* fi = fopen(path, "r");
    if (!fi) return serr(s, LESGPU_EIO, "no restart_info.txt");
    int step = 0, binary = 0;
    if (fgets(line, sizeof line, fi) && strncmp(line, "BINARY", 6) == 0 && fgets(line, sizeof line, fi) &&
        sscanf(line, "%d", &step) == 1)
        binary = 1;
    fclose(fi);
    if (!binary) return serr(s, LESGPU_EIO, "restart_info.txt does not name a binary checkpoint");
    /* fixed mode: read the sidecar first, so a bad one leaves the solver untouched */
    les_rng rng;
    double numax = 0.0, amax = 0.0;
    double* vort = NULL;
    const int nv = s->cfg.num_vortices;
    const size_t nvd = (size_t)(nv > 0 ? nv : 0) * 7;
    if (mode == LES_RESUME_FIXED) {
        join_path(path, sizeof(path), dir, "les_resume.bin");
        FILE* fp = fopen(path, "rb");
        if (!fp) return serr(s, LESGPU_EIO, "les_resume.bin missing: the checkpoint was not written by a fixed finish");
        unsigned int magic = 0;
        int fnv = -1, ft = 0;
        vort = (double*)malloc(nvd ? nvd * sizeof(double) : sizeof(double));
        int ok = vort && fread(&magic, sizeof magic, 1, fp) == 1 && magic == LES_RESUME_MAGIC &&
                 fread(&fnv, sizeof fnv, 1, fp) == 1 && fnv == nv && fread(&ft, sizeof ft, 1, fp) == 1 &&
                 fread(&rng, sizeof rng, 1, fp) == 1 && fread(&numax, sizeof numax, 1, fp) == 1 &&
                 fread(&amax, sizeof amax, 1, fp) == 1 && (nvd == 0 || fread(vort, sizeof(double), nvd, fp) == nvd);
        fclose(fp);
        if (!ok) { free(vort); return serr(s, LESGPU_EIO, "les_resume.bin does not match this solver"); }
    }
    /* load_quick_checkpoint (:3701-3726); the run continues from the step stored in it (:4189) */
    join_path(path, sizeof(path), dir, "checkpoint.bin");
    int t = 0;
    int rc = les_solver_load_checkpoint(s, path, &t);
    if (rc) { free(vort); return rc; }
    if (s->avg_on) {                                   /* load_statistics_backup (:4190) */
        join_path(path, sizeof(path), dir, "stats_backup.bin");
        FILE* fs = fopen(path, "rb");
        if (fs) {
            fclose(fs);
            rc = les_solver_load_stats(s, path);
            if (rc) { free(vort); return rc; }
        }
    }
    if (mode == LES_RESUME_REFERENCE) {
        /* initialize_vortices (:4193) after the start-up srand(seed) (:4085) */
        les_rng_seed(&s->rng, s->cfg.seed);
        les_vortices_init(&s->rng, &s->cfg, s->vort);
        /* the start-up attribute map (:4123-4136): setting() does not run on a resume, so the
           j = 0 face keeps code 4 instead of the symmetry code 5 (and no rim code 6) */
        for (size_t c = 0; c < s->n; c++)
            if (s->attr[c] == 5 || s->attr[c] == 6) s->attr[c] = 4;
        rc = lesgpu_upload_attribute(s->ctx, s->attr);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
        /* the nu/alpha maxima stay 0, as the state upload of les_solver_load_checkpoint left them */
    } else {
        s->rng = rng;
        if (nvd) memcpy(s->vort, vort, nvd * sizeof(double));
        free(vort);
        rc = lesgpu_set_dt_inputs(s->ctx, numax, amax);
        if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    }
    s->t_loop = t;
    if (t_out) *t_out = t;
    return LESGPU_OK;
}

/* ------------------------------------------------------------------ time averages */

int les_solver_set_averaging(les_solver* s, int start_step) {
    if (!s) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "end the device loop before changing the averaging");
    int rc;
    if (start_step < 0) {
        rc = lesgpu_avg_end(s->ctx);
        s->avg_on = 0;
    } else {
        rc = lesgpu_avg_begin(s->ctx, start_step);
        s->avg_on = (rc == LESGPU_OK);
        s->avg_start = start_step;
    }
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    return LESGPU_OK;
}

static int avg_fields(les_solver* s, double** f) {
    for (int q = 0; q < 10; q++) {
        f[q] = (double*)malloc(s->n * sizeof(double));
        if (!f[q]) {
            for (int r = 0; r < q; r++) free(f[r]);
            return LESGPU_ENOMEM;
        }
    }
    return LESGPU_OK;
}

/* save_statistics_backup (:3736-3756): int time_avg_steps, then the ten sums. */
int les_solver_save_stats(les_solver* s, const char* path) {
    if (!s || !path) return LESGPU_EINVAL;
    if (!s->avg_on) return serr(s, LESGPU_ESTATE, "time averages are not enabled");
    double* f[10];
    if (avg_fields(s, f)) return serr(s, LESGPU_ENOMEM, "host buffers");
    int count = 0;
    int rc = lesgpu_avg_download(s->ctx, (double* const*)f, &count);
    if (rc == LESGPU_OK) {
        FILE* fp = fopen(path, "wb");
        if (!fp) {
            rc = serr(s, LESGPU_EIO, "cannot open stats backup for writing");
        } else {
            int ok = fwrite(&count, sizeof(int), 1, fp) == 1;
            for (int q = 0; q < 10 && ok; q++) ok = fwrite(f[q], sizeof(double), s->n, fp) == s->n;
            fclose(fp);
            if (!ok) rc = serr(s, LESGPU_EIO, "short stats backup write");
        }
    } else {
        serr(s, rc, lesgpu_last_error(s->ctx));
    }
    for (int q = 0; q < 10; q++) free(f[q]);
    return rc;
}

/* load_statistics_backup (:3758-3778). */
int les_solver_load_stats(les_solver* s, const char* path) {
    if (!s || !path) return LESGPU_EINVAL;
    if (!s->avg_on) return serr(s, LESGPU_ESTATE, "enable the time averages first");
    FILE* fp = fopen(path, "rb");
    if (!fp) return serr(s, LESGPU_EIO, "cannot open stats backup");
    double* f[10];
    if (avg_fields(s, f)) { fclose(fp); return serr(s, LESGPU_ENOMEM, "host buffers"); }
    int count = 0;
    int ok = fread(&count, sizeof(int), 1, fp) == 1 && count >= 0;
    for (int q = 0; q < 10 && ok; q++) ok = fread(f[q], sizeof(double), s->n, fp) == s->n;
    fclose(fp);
    int rc = ok ? lesgpu_avg_upload(s->ctx, (const double* const*)f, count) : LESGPU_EIO;
    for (int q = 0; q < 10; q++) free(f[q]);
    if (!ok) return serr(s, LESGPU_EIO, "truncated or invalid stats backup");
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    return LESGPU_OK;
}

/* calculate_resolved_reynolds_stresses (:3194-3217): <u'u'>, <v'v'>, <w'w'>, <u'v'>, <u'w'>,
 * <v'w'> and the mean G, from the sums and time_avg_steps (left unchanged here; the
 * reference divides G_mean in place). */
int les_solver_reynolds_stresses(les_solver* s, double* const* out, int* count) {
    if (!s || !out) return LESGPU_EINVAL;
    for (int q = 0; q < 7; q++)
        if (!out[q]) return LESGPU_EINVAL;
    if (!s->avg_on) return serr(s, LESGPU_ESTATE, "time averages are not enabled");
    double* f[10];
    if (avg_fields(s, f)) return serr(s, LESGPU_ENOMEM, "host buffers");
    int n = 0;
    int rc = lesgpu_avg_download(s->ctx, (double* const*)f, &n);
    if (rc == LESGPU_OK && n > 0) {
        for (size_t c = 0; c < s->n; c++) {
            double au = f[0][c] / n, av = f[1][c] / n, aw = f[2][c] / n;
            out[0][c] = (f[3][c] / n) - (au * au);
            out[1][c] = (f[4][c] / n) - (av * av);
            out[2][c] = (f[5][c] / n) - (aw * aw);
            out[3][c] = (f[6][c] / n) - (au * av);
            out[4][c] = (f[7][c] / n) - (au * aw);
            out[5][c] = (f[8][c] / n) - (av * aw);
            out[6][c] = f[9][c] / n;
        }
    } else if (rc == LESGPU_OK) {
        for (int q = 0; q < 7; q++) memset(out[q], 0, s->n * sizeof(double));
    }
    for (int q = 0; q < 10; q++) free(f[q]);
    if (count) *count = n;
    if (rc) return serr(s, rc, lesgpu_last_error(s->ctx));
    return LESGPU_OK;
}

/* Final output of a run (:4604-4623): the VTK file of the last step (when VTK output is on)
 * and the remaining point rows. */
int les_solver_flush(les_solver* s) {
    if (!s) return LESGPU_EINVAL;
    if (s->loop_on) return serr(s, LESGPU_ESTATE, "end the device loop first");
    int rc = write_vtk_step(s, s->t_loop);
    flush_points(s);
    if (rc == LESGPU_OK && s->ps_on && (s->out_flags & LES_OUT_PSTAT) && s->out_dir[0]) {
        char path[1200];
        join_path(path, sizeof(path), s->out_dir, "profile_stats.bin");
        rc = les_solver_pstat_write(s, path);
    }
    return rc;
}

/* ------------------------------------------------------------------ VTK */

/* output_vtk (:3473-3668): legacy ASCII structured grid, points and values in k-j-i order,
 * non-finite values written as 0.  Fields: velocity, temperature, G, the five mass
 * fractions, density, omega (never computed by the reference: 0), mu_mix, nu_mix (the
 * reference's defaults on non-fluid cells), ST_turbulent, nu_t, |grad G| (0 unless
 * lesgpu_keep_grad_g is on), the six resolved Reynolds stresses and G_mean (0 without time
 * averages).  The reference divides G_mean by time_avg_steps in place before writing it
 * (:3215), so with averages on its file carries sum/n^2; here it is sum/n. */
int les_solver_write_vtk(les_solver* s, const char* path) {
    if (!s || !path) return LESGPU_EINVAL;
    const size_t n = s->n;
    const int nf = 11 + 5 + 10;
    double* buf = (double*)malloc((size_t)nf * n * sizeof(double));
    if (!buf) return serr(s, LESGPU_ENOMEM, "host buffers");
    double* st[11];
    for (int q = 0; q < 11; q++) st[q] = buf + (size_t)q * n;
    double* mu = buf + 11 * n; double* nu = buf + 12 * n; double* ST = buf + 13 * n;
    double* nut = buf + 14 * n; double* gg = buf + 15 * n;
    double* av[10];
    for (int q = 0; q < 10; q++) av[q] = buf + (size_t)(16 + q) * n;
    int rc = lesgpu_download_state(s->ctx, (double* const*)st, 11);
    if (rc == LESGPU_OK) rc = lesgpu_get_field(s->ctx, LESGPU_F_MU_MIX, mu);
    if (rc == LESGPU_OK) rc = lesgpu_get_field(s->ctx, LESGPU_F_NU, nu);
    if (rc == LESGPU_OK) rc = lesgpu_get_field(s->ctx, LESGPU_F_ST, ST);
    if (rc == LESGPU_OK) rc = lesgpu_get_field(s->ctx, LESGPU_F_NU_T, nut);
    if (rc == LESGPU_OK && lesgpu_get_field(s->ctx, LESGPU_F_GRAD_G, gg) != LESGPU_OK) memset(gg, 0, n * sizeof(double));
    int navg = 0;
    if (rc == LESGPU_OK && s->avg_on) rc = lesgpu_avg_download(s->ctx, (double* const*)av, &navg);
    if (rc) { free(buf); return serr(s, rc, lesgpu_last_error(s->ctx)); }
    for (size_t c = 0; c < n; c++)
        if (s->attr[c] != 3) { mu[c] = 1.8e-5; nu[c] = 1.5e-5; }     /* update_nu_mix defaults (:1556-1561) */
    FILE* fp = fopen(path, "w");
    if (!fp) { free(buf); return serr(s, LESGPU_EIO, "cannot open the VTK file"); }
    char* iobuf = (char*)malloc(1 << 20);     /* per call: solvers may write from several threads */
    if (iobuf) setvbuf(fp, iobuf, _IOFBF, 1 << 20);
    const int NXv = s->nx, NYv = s->ny, NZv = s->nz;
#define VTK_LOOP for (int k = 0; k < NZv; k++) for (int j = 0; j < NYv; j++) for (int i = 0; i < NXv; i++)
#define VTK_ID ((((size_t)i * NYv) + j) * NZv + k)
#define FIN(x) (isfinite(x) ? (x) : 0.0)
    fprintf(fp, "# vtk DataFile Version 3.0\nVTK output\nASCII\nDATASET STRUCTURED_GRID\n");
    fprintf(fp, "DIMENSIONS %d %d %d\n", NXv, NYv, NZv);
    fprintf(fp, "POINTS %d float\n", NXv * NYv * NZv);
    VTK_LOOP fprintf(fp, "%.6f %.6f %.6f\n", (double)i * s->dx, (double)j * s->dy, (double)k * s->dz);
    fprintf(fp, "\nPOINT_DATA %d\n", NXv * NYv * NZv);
    fprintf(fp, "VECTORS velocity float\n");
    VTK_LOOP { size_t c = VTK_ID; fprintf(fp, "%.6f %.6f %.6f\n", FIN(st[0][c]), FIN(st[1][c]), FIN(st[2][c])); }
    static const char* names6[] = {"temperature", "G_value", "Y_C3H8", "Y_O2", "Y_N2", "Y_CO2", "Y_H2O", "density"};
    const double* f6[] = {st[3], st[4], st[6], st[7], st[8], st[9], st[10], st[5]};
    for (int q = 0; q < 8; q++) {
        fprintf(fp, "SCALARS %s float\nLOOKUP_TABLE default\n", names6[q]);
        VTK_LOOP fprintf(fp, "%.6f\n", FIN(f6[q][VTK_ID]));
    }
    fprintf(fp, "SCALARS omega float\nLOOKUP_TABLE default\n");
    VTK_LOOP fprintf(fp, "%.6e\n", 0.0);
    static const char* names_e[] = {"mu_mix", "nu_mix", "ST_turbulent", "nu_t", "grad_G_magnitude"};
    const double* fe[] = {mu, nu, ST, nut, gg};
    for (int q = 0; q < 5; q++) {
        fprintf(fp, "SCALARS %s float\nLOOKUP_TABLE default\n", names_e[q]);
        VTK_LOOP fprintf(fp, "%.6e\n", FIN(fe[q][VTK_ID]));
    }
    /* re_stress_xy = <xy> - <x><y>, 0 before any averaged step (:3586-3655) */
    static const char* rs[] = {"re_stress_uu", "re_stress_vv", "re_stress_ww", "re_stress_uv", "re_stress_uw",
                               "re_stress_vw"};
    static const int ra[6] = {0, 1, 2, 0, 0, 1}, rb[6] = {0, 1, 2, 1, 2, 2}, rp[6] = {3, 4, 5, 6, 7, 8};
    for (int q = 0; q < 6; q++) {
        fprintf(fp, "SCALARS %s float\nLOOKUP_TABLE default\n", rs[q]);
        VTK_LOOP {
            double v = 0.0;
            if (navg > 0) {
                size_t c = VTK_ID;
                double aa = av[ra[q]][c] / navg, ab = av[rb[q]][c] / navg;
                v = (av[rp[q]][c] / navg) - (aa * ab);
            }
            fprintf(fp, "%.6e\n", FIN(v));
        }
    }
    fprintf(fp, "SCALARS G_mean float\nLOOKUP_TABLE default\n");
    VTK_LOOP fprintf(fp, "%.6f\n", navg > 0 ? FIN(av[9][VTK_ID] / navg) : 0.0);
#undef VTK_LOOP
#undef VTK_ID
#undef FIN
    int bad = ferror(fp);
    fclose(fp);
    free(iobuf);
    free(buf);
    if (bad) return serr(s, LESGPU_EIO, "VTK write failed");
    return LESGPU_OK;
}

static int write_vtk_step(les_solver* s, int t) {
    if (!(s->out_flags & LES_OUT_VTK) || !s->out_dir[0]) return LESGPU_OK;
    char name[64], path[1200];
    snprintf(name, sizeof(name), "Premixed_C3H8_Air_%04d.vtk", t);
    join_path(path, sizeof(path), s->out_dir, name);
    return les_solver_write_vtk(s, path);
}
