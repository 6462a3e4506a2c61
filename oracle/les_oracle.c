/*
 * les_oracle.c -- CPU restatement of the per-timestep hot path of les_combustion_solver.c.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA solver step;
 * only the test-suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * It is never part of the product path.
 *
 * It restates, serially and with runtime grid sizes, exactly what the reference computes
 * when run with OMP_NUM_THREADS=1.  Every function cites the reference lines it follows
 * (file les_combustion_solver.c).  Expressions keep the reference's operation order so
 * that, built with the same gcc/libm and -ffp-contract=off, results are bit-identical to
 * the compiled reference (pinned by tests against oracle/_ref runs and tests/golden).
 *
 * Storage: every field is a flat double array in the reference's [i][j][k] order
 * (k fastest), index (i*NY + j)*NZ + k (les_combustion_solver.c:286).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NSP 5
#define C3H8_INDEX 0
#define O2_INDEX 1
#define N2_INDEX 2
#define CO2_INDEX 3
#define H2O_INDEX 4

/* fixed constants of the reference (les_combustion_solver.c:136-188, 2164-2166, 234-245) */
#define R_univ 8.314462
#define PATM 101325.0
#define pressure_const 101325.0
#define G_GRAVITY -9.81
#define DEFAULT_RHO_AIR 1.2
#define SMALL_NUMBER 1e-10
#define SSR_A 0.2340
#define SSR_B 0.2187
#define SSR_C 10.0
#define FILTER_WEIGHT_CENTER 50.0
#define UW2 0.0
#define UW1 0.5
#define DW1 0.5
#define MIN_T_CLIP 200.0
#define MAX_T_CLIP 3000.0
#define MIN_MU_MIX_CLIP 1e-7
#define MIN_NU_MIX_CLIP 1e-7
#define TENO_CUTOFF 1.0e-6
#define MAX_FLAME_FORCE_LIMIT 500.0
#define FLAME_RAMP_DISTANCE 0.03
#define ONE_THIRD (1.0 / 3.0)

typedef struct {
    int nx, ny, nz, num_vortices;
    int initial_flame_front_i, weno_transition_step;
    unsigned int seed;
    int flame_accel;                         /* USE_FLAME_ACCEL_MODEL */
    double lx, ly, lz;
    double inlet_radius, rim_outer_radius;
    double inlet_velocity, inlet_temperature, ambient_temperature;
    double turbulence_intensity, length_scale;
    double s_l, burnt_gas_temperature, pr_t, sc_t, d3;
    double courant, courant_diffusion;
    double cs_unburned, cs_burnt, cs_flame_boost;
    double accel_strength, accel_width, accel_center, relax;
    double nu_unburnt, rho_unburnt_approx, rho_burnt_approx, equivalence_ratio;
} orc_config;

typedef struct { double x, y, z, radius, su, sv, sw; } orc_vortex;

typedef struct {
    orc_config c;
    int NX, NY, NZ;
    size_t n;
    double DX, DY, DZ;
    /* species (les_combustion_solver.c:292-305) */
    double mw[NSP], t_mid[NSP], nasa_high[NSP][7], nasa_low[NSP][7], lam[NSP][4], eta[NSP][4];
    double dco[NSP][NSP][4];
    double inletYk[NSP], ambientYk[NSP];
    double stoich_o2, stoich_co2, stoich_h2o;
    int* attr;
    /* state */
    double *u, *v, *w, *T, *P, *rho, *G, *Y[NSP], *rhou, *rhov, *rhow;
    /* RHS intermediates */
    double *u_f, *v_f, *w_f, *T_f, *P_f, *rho_f, *G_f, *Y_f[NSP];
    double *nu, *mu_mix, *alpha, *nu_t, *S_mag, *SijSij, *div_u, *ST, *Cp_mix, *lambda_mix, *Dk[NSP];
    double *gradG_dbg;
    /* RK4 */
    double *rhou0, *rhov0, *rhow0, *T0, *G0, *Y0[NSP];
    double *ut, *vt, *wt, *Tt, *Gt, *Yt[NSP], *rhot, *rhout, *rhovt, *rhowt;
    double *k_rhou[4], *k_rhov[4], *k_rhow[4], *k_T[4], *k_G[4], *k_Y[4][NSP];
    /* SEM */
    orc_vortex* vort;
    int* inlet_attr;                          /* [NY][NZ] */
    double *u_in, *v_in, *w_in;               /* [NY][NZ] */
    int t_loop;
    double dt, max_velocity;
} orc_ctx;

#define ID(i, j, k) (((size_t)(i) * (size_t)c->NY + (size_t)(j)) * (size_t)c->NZ + (size_t)(k))

/* ------------------------------------------------------------------ property loaders */

static unsigned char* read_record(FILE* fp, int* len) {
    int n;
    if (fread(&n, sizeof(int), 1, fp) != 1 || n < 0) return NULL;
    unsigned char* b = (unsigned char*)malloc((size_t)n + 1);
    if (!b) return NULL;
    if (fread(b, 1, (size_t)n, fp) != (size_t)n) { free(b); return NULL; }
    int e;
    if (fread(&e, sizeof(int), 1, fp) != 1) { free(b); return NULL; }
    if (len) *len = n;
    return b;
}

/* les_combustion_solver.c:324-356 */
static int load_chem(orc_ctx* c, const char* path) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return 0;
    unsigned char* b;
    int mm = 0, kk = 0;
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; } free(b);
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; }
    memcpy(&mm, b + 12, 4); memcpy(&kk, b + 16, 4); free(b);
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; } free(b);
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; }
    if (kk != NSP) { free(b); fclose(fp); return 0; }
    size_t per = 16 + 4 * (size_t)mm + 8 + 8 + 4 + 24 + 2 * 56;
    for (int i = 0; i < kk; i++) {
        size_t base = 8 + (size_t)i * per;
        size_t mwo = base + 16 + 4 * (size_t)mm + 8;
        size_t tmo = mwo + 8 + 4 + 16;
        memcpy(&c->mw[i], b + mwo, 8);
        memcpy(&c->t_mid[i], b + tmo, 8);
        memcpy(c->nasa_high[i], b + tmo + 8, 56);
        memcpy(c->nasa_low[i], b + tmo + 8 + 56, 56);
    }
    free(b);
    fclose(fp);
    return 1;
}

/* les_combustion_solver.c:359-382 */
static int load_tran(orc_ctx* c, const char* path) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return 0;
    unsigned char* b;
    for (int r = 0; r < 4; r++) { b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; } free(b); }
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; }
    for (int i = 0; i < NSP; i++) memcpy(c->lam[i], b + i * 32, 32);
    free(b);
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; }
    for (int i = 0; i < NSP; i++) memcpy(c->eta[i], b + i * 32, 32);
    free(b);
    b = read_record(fp, NULL); if (!b) { fclose(fp); return 0; }
    for (int i = 0; i < NSP; i++)
        for (int j = 0; j < NSP; j++) memcpy(c->dco[i][j], b + (i * NSP + j) * 32, 32);
    free(b);
    fclose(fp);
    return 1;
}

/* ------------------------------------------------------------- property evaluations */

/* les_combustion_solver.c:385-391 */
static double property_from_fit(double temp, const double co[4]) {
    if (temp <= 0) return 0.0;
    if (co[0] == 0.0 && co[1] == 0.0 && co[2] == 0.0 && co[3] == 0.0) return 0.0;
    double lt = log(temp);
    double lp = co[0] + co[1] * lt + co[2] * pow(lt, 2) + co[3] * pow(lt, 3);
    return exp(lp);
}
/* :394-398 */
static double mu_dynamic(const orc_ctx* c, int s, double T) { return property_from_fit(T, c->eta[s]) * 0.1; }
/* :401-416 */
static double cp_per_mole(const orc_ctx* c, int s, double temp) {
    if (temp <= 0.0) temp = 1.0;
    const double* a = (temp > c->t_mid[s]) ? c->nasa_high[s] : c->nasa_low[s];
    double cpr = a[0] + a[1] * temp + a[2] * pow(temp, 2) + a[3] * pow(temp, 3) + a[4] * pow(temp, 4);
    return cpr * R_univ;
}
/* :419-428 */
static double cp_dynamic(const orc_ctx* c, int s, double T) {
    double cpm = cp_per_mole(c, s, T);
    double mwk = c->mw[s] / 1000.0;
    if (mwk < 1e-9) return 1000.0;
    return cpm / mwk;
}
/* :431-437 */
static double lambda_dynamic(const orc_ctx* c, int s, double T) { return property_from_fit(T, c->lam[s]) * 1e-5; }
/* :440-447 */
static double dkj_dynamic(const orc_ctx* c, int k, int j, double T) { return property_from_fit(T, c->dco[k][j]) * 1e-4; }

/* ------------------------------------------------------------------ glibc rand() */
/* The reference draws with glibc rand(); the oracle calls the same function. */

static double rnd01(void) { return rand() / (double)RAND_MAX; }

/* ------------------------------------------------------------------ allocation */

static double* zalloc(size_t n) { return (double*)calloc(n, sizeof(double)); }

static void orc_free_arrays(orc_ctx* c);

orc_ctx* orc_create(const orc_config* cfg, const char* chem_path, const char* tran_path) {
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    if (!c) return NULL;
    c->c = *cfg;
    c->NX = cfg->nx; c->NY = cfg->ny; c->NZ = cfg->nz;
    c->n = (size_t)c->NX * c->NY * c->NZ;
    c->DX = cfg->lx / (double)cfg->nx;
    c->DY = cfg->ly / (double)cfg->ny;
    c->DZ = cfg->lz / (double)cfg->nz;
    if (!load_chem(c, chem_path) || !load_tran(c, tran_path)) { free(c); return NULL; }
    size_t n = c->n;
    /* the reference's malloc'd grids start as fresh zero pages (les_combustion_solver.c:3853) */
    double** all[] = {&c->u, &c->v, &c->w, &c->T, &c->P, &c->rho, &c->G, &c->rhou, &c->rhov, &c->rhow,
                      &c->u_f, &c->v_f, &c->w_f, &c->T_f, &c->P_f, &c->rho_f, &c->G_f,
                      &c->nu, &c->mu_mix, &c->alpha, &c->nu_t, &c->S_mag, &c->SijSij, &c->div_u, &c->ST,
                      &c->Cp_mix, &c->lambda_mix, &c->gradG_dbg,
                      &c->rhou0, &c->rhov0, &c->rhow0, &c->T0, &c->G0,
                      &c->ut, &c->vt, &c->wt, &c->Tt, &c->Gt, &c->rhot, &c->rhout, &c->rhovt, &c->rhowt};
    for (size_t q = 0; q < sizeof(all) / sizeof(all[0]); q++) { *all[q] = zalloc(n); if (!*all[q]) { orc_free_arrays(c); free(c); return NULL; } }
    for (int s = 0; s < NSP; s++) {
        c->Y[s] = zalloc(n); c->Y_f[s] = zalloc(n); c->Dk[s] = zalloc(n);
        c->Y0[s] = zalloc(n); c->Yt[s] = zalloc(n);
        for (int r = 0; r < 4; r++) c->k_Y[r][s] = zalloc(n);
    }
    for (int r = 0; r < 4; r++) {
        c->k_rhou[r] = zalloc(n); c->k_rhov[r] = zalloc(n); c->k_rhow[r] = zalloc(n);
        c->k_T[r] = zalloc(n); c->k_G[r] = zalloc(n);
    }
    c->attr = (int*)calloc(n, sizeof(int));
    c->vort = (orc_vortex*)calloc((size_t)cfg->num_vortices > 0 ? (size_t)cfg->num_vortices : 1, sizeof(orc_vortex));
    size_t np = (size_t)c->NY * c->NZ;
    c->inlet_attr = (int*)calloc(np, sizeof(int));
    c->u_in = zalloc(np); c->v_in = zalloc(np); c->w_in = zalloc(np);

    /* inlet composition and stoichiometry (les_combustion_solver.c:4101-4120) */
    const double phi = cfg->equivalence_ratio;
    double m_f = 1.0, m_o2 = 5.0 / phi, m_n2 = m_o2 * 3.76;
    double mass_total = m_f * c->mw[C3H8_INDEX] + m_o2 * c->mw[O2_INDEX] + m_n2 * c->mw[N2_INDEX];
    c->inletYk[C3H8_INDEX] = (m_f * c->mw[C3H8_INDEX]) / mass_total;
    c->inletYk[O2_INDEX] = (m_o2 * c->mw[O2_INDEX]) / mass_total;
    c->inletYk[N2_INDEX] = (m_n2 * c->mw[N2_INDEX]) / mass_total;
    c->inletYk[CO2_INDEX] = 0.0; c->inletYk[H2O_INDEX] = 0.0;
    c->ambientYk[C3H8_INDEX] = 0.0; c->ambientYk[O2_INDEX] = 0.232; c->ambientYk[N2_INDEX] = 0.768;
    c->ambientYk[CO2_INDEX] = 0.0; c->ambientYk[H2O_INDEX] = 0.0;
    c->stoich_o2 = (5.0 * c->mw[O2_INDEX]) / c->mw[C3H8_INDEX];
    c->stoich_co2 = (3.0 * c->mw[CO2_INDEX]) / c->mw[C3H8_INDEX];
    c->stoich_h2o = (4.0 * c->mw[H2O_INDEX]) / c->mw[C3H8_INDEX];
    return c;
}

static void orc_free_arrays(orc_ctx* c) {
    double* all[] = {c->u, c->v, c->w, c->T, c->P, c->rho, c->G, c->rhou, c->rhov, c->rhow,
                     c->u_f, c->v_f, c->w_f, c->T_f, c->P_f, c->rho_f, c->G_f,
                     c->nu, c->mu_mix, c->alpha, c->nu_t, c->S_mag, c->SijSij, c->div_u, c->ST,
                     c->Cp_mix, c->lambda_mix, c->gradG_dbg, c->rhou0, c->rhov0, c->rhow0, c->T0, c->G0,
                     c->ut, c->vt, c->wt, c->Tt, c->Gt, c->rhot, c->rhout, c->rhovt, c->rhowt};
    for (size_t q = 0; q < sizeof(all) / sizeof(all[0]); q++) free(all[q]);
    for (int s = 0; s < NSP; s++) {
        free(c->Y[s]); free(c->Y_f[s]); free(c->Dk[s]); free(c->Y0[s]); free(c->Yt[s]);
        for (int r = 0; r < 4; r++) free(c->k_Y[r][s]);
    }
    for (int r = 0; r < 4; r++) { free(c->k_rhou[r]); free(c->k_rhov[r]); free(c->k_rhow[r]); free(c->k_T[r]); free(c->k_G[r]); }
    free(c->attr); free(c->vort); free(c->inlet_attr); free(c->u_in); free(c->v_in); free(c->w_in);
}

void orc_destroy(orc_ctx* c) {
    if (!c) return;
    orc_free_arrays(c);
    free(c);
}

/* ------------------------------------------------------------------ SEM inflow */

/* les_combustion_solver.c:861-897 (three printed test draws, then 7 draws per vortex) */
static void initialize_vortices(orc_ctx* c) {
    (void)rand(); (void)rand(); (void)rand();
    double u_rms = c->c.inlet_velocity * c->c.turbulence_intensity;
    double box_x = c->c.length_scale, box_y = c->c.ly, box_z = c->c.lz;
    for (int i = 0; i < c->c.num_vortices; i++) {
        double r1 = rnd01(), r2 = rnd01(), r3 = rnd01(), r4 = rnd01(), r5 = rnd01(), r6 = rnd01(), r7 = rnd01();
        orc_vortex* vt = &c->vort[i];
        vt->x = (r1 - 0.5) * box_x;
        vt->y = r2 * box_y;
        vt->z = r3 * box_z;
        double min_r = c->c.length_scale * 0.5, max_r = c->c.length_scale * 1.5;
        vt->radius = min_r + (max_r - min_r) * r4;
        vt->su = (r5 * 2.0 - 1.0) * u_rms;
        vt->sv = (r6 * 2.0 - 1.0) * u_rms;
        vt->sw = (r7 * 2.0 - 1.0) * u_rms;
    }
}

/* :900-939 */
static void update_vortices(orc_ctx* c, double dt) {
    double u_rms = c->c.inlet_velocity * c->c.turbulence_intensity;
    double box_x = c->c.length_scale;
    for (int i = 0; i < c->c.num_vortices; i++) {
        orc_vortex* vt = &c->vort[i];
        vt->x += c->c.inlet_velocity * dt;
        if (vt->x > box_x / 2.0) {
            vt->x -= box_x;
            double ry = (double)rand() / (double)RAND_MAX;
            double rz = (double)rand() / (double)RAND_MAX;
            vt->y = ry * c->c.ly;
            vt->z = rz * c->c.lz;
            double ru = (double)rand() / (double)RAND_MAX;
            double rv = (double)rand() / (double)RAND_MAX;
            double rw = (double)rand() / (double)RAND_MAX;
            vt->su = (ru * 2.0 - 1.0) * u_rms;
            vt->sv = (rv * 2.0 - 1.0) * u_rms;
            vt->sw = (rw * 2.0 - 1.0) * u_rms;
            double rr = (double)rand() / (double)RAND_MAX;
            double min_r = c->c.length_scale * 0.5, max_r = c->c.length_scale * 1.5;
            vt->radius = min_r + (max_r - min_r) * rr;
        }
    }
}

/* :943-1075 */
static void generate_inlet_sem(orc_ctx* c, double dt) {
    update_vortices(c, dt);
    const int NY = c->NY, NZ = c->NZ;
    for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) {
            size_t p = (size_t)j * NZ + k;
            c->u_in[p] = 0.0; c->v_in[p] = 0.0; c->w_in[p] = 0.0;
            if (c->inlet_attr[p] == 1) {
                double y = j * c->DY, z = k * c->DZ;
                for (int q = 0; q < c->c.num_vortices; q++) {
                    double dx = 0.0 - c->vort[q].x;
                    double dy = y - c->vort[q].y;
                    double dz = z - c->vort[q].z;
                    double dist = sqrt(dx * dx + dy * dy + dz * dz);
                    double radius = c->vort[q].radius;
                    double infl = 0.0;
                    if (dist < radius) infl = 1.0 - (dist / radius);
                    c->u_in[p] += c->vort[q].su * infl;
                    c->v_in[p] += c->vort[q].sv * infl;
                    c->w_in[p] += c->vort[q].sw * infl;
                }
            }
        }
    double tu = 0.0, tv = 0.0, tw = 0.0;
    int cnt = 0;
    for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) {
            size_t p = (size_t)j * NZ + k;
            if (c->inlet_attr[p] == 1) { tu += c->u_in[p]; tv += c->v_in[p]; tw += c->w_in[p]; cnt++; }
        }
    if (cnt > 0) {
        double au = tu / cnt, av = tv / cnt, aw = tw / cnt;
        for (size_t p = 0; p < (size_t)NY * NZ; p++)
            if (c->inlet_attr[p] == 1) { c->u_in[p] -= au; c->v_in[p] -= av; c->w_in[p] -= aw; }
    }
    double su = 0.0, sv = 0.0, sw = 0.0;
    for (size_t p = 0; p < (size_t)NY * NZ; p++)
        if (c->inlet_attr[p] == 1) {
            su += c->u_in[p] * c->u_in[p]; sv += c->v_in[p] * c->v_in[p]; sw += c->w_in[p] * c->w_in[p];
        }
    if (cnt > 0) {
        double ru = sqrt(su / cnt), rv = sqrt(sv / cnt), rw = sqrt(sw / cnt);
        double target = c->c.inlet_velocity * c->c.turbulence_intensity;
        double sc_u = (ru > SMALL_NUMBER) ? target / ru : 0.0;
        double sc_v = (rv > SMALL_NUMBER) ? target / rv : 0.0;
        double sc_w = (rw > SMALL_NUMBER) ? target / rw : 0.0;
        for (size_t p = 0; p < (size_t)NY * NZ; p++)
            if (c->inlet_attr[p] == 1) { c->u_in[p] *= sc_u; c->v_in[p] *= sc_v; c->w_in[p] *= sc_w; }
    }
}

/* ------------------------------------------------------------------ initial state */

/* les_combustion_solver.c:1135-1285 (setting) with the attribute map of :1151-1181,
 * then initialize_vortices (:4360) and the inlet mask (:4366-4367). */
void orc_init(orc_ctx* c, int start_step) {
    srand(c->c.seed);
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    double ic_y = 0.0, ic_z = c->c.lz / 2.0;
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ; k++) {
                int a;
                if (i == 0) {
                    double y = j * c->DY, z = k * c->DZ;
                    double d2 = pow(y - ic_y, 2) + pow(z - ic_z, 2);
                    if (d2 <= pow(c->c.inlet_radius, 2)) a = 1;
                    else if (d2 <= pow(c->c.rim_outer_radius, 2)) a = 6;
                    else a = 4;
                } else if (i == NX - 1) a = 2;
                else if (j == 0) a = 5;
                else if (j == NY - 1 || k == 0 || k == NZ - 1) a = 4;
                else a = 3;
                c->attr[ID(i, j, k)] = a;
            }
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ; k++) {
                size_t id = ID(i, j, k);
                c->P[id] = 0.0;
                switch (c->attr[id]) {
                    case 1:
                        c->u[id] = c->c.inlet_velocity; c->v[id] = 0.0; c->w[id] = 0.0;
                        c->T[id] = c->c.inlet_temperature; c->G[id] = 0.0;
                        for (int s = 0; s < NSP; s++) c->Y[s][id] = c->inletYk[s];
                        break;
                    case 4:
                    case 2:
                        c->u[id] = 0.0; c->v[id] = 0.0; c->w[id] = 0.0;
                        c->T[id] = c->c.ambient_temperature; c->G[id] = 0.0;
                        for (int s = 0; s < NSP; s++) c->Y[s][id] = c->ambientYk[s];
                        break;
                    case 5:
                    case 3:
                        c->u[id] = 0.0; c->v[id] = 0.0; c->w[id] = 0.0;
                        if (i <= c->c.initial_flame_front_i) {
                            c->G[id] = 1.0;
                            c->T[id] = c->c.burnt_gas_temperature;
                            double cons = c->inletYk[C3H8_INDEX];
                            c->Y[C3H8_INDEX][id] = c->inletYk[C3H8_INDEX] - cons;
                            c->Y[O2_INDEX][id] = c->inletYk[O2_INDEX] - cons * c->stoich_o2;
                            c->Y[N2_INDEX][id] = c->inletYk[N2_INDEX];
                            c->Y[CO2_INDEX][id] = c->inletYk[CO2_INDEX] + cons * c->stoich_co2;
                            c->Y[H2O_INDEX][id] = c->inletYk[H2O_INDEX] + cons * c->stoich_h2o;
                        } else {
                            c->G[id] = 0.0;
                            c->T[id] = c->c.inlet_temperature;
                            for (int s = 0; s < NSP; s++) c->Y[s][id] = c->inletYk[s];
                        }
                        break;
                    default: break;
                }
                double syw = 0.0;
                for (int s = 0; s < NSP; s++) syw += c->Y[s][id] / (c->mw[s] / 1000.0);
                if (syw > SMALL_NUMBER && c->T[id] > 1.0) {
                    double W = 1.0 / syw;
                    double Rm = R_univ / W;
                    c->rho[id] = pressure_const / (Rm * c->T[id]);
                } else {
                    c->rho[id] = DEFAULT_RHO_AIR;
                }
                c->rhou[id] = c->rho[id] * c->u[id];
                c->rhov[id] = c->rho[id] * c->v[id];
                c->rhow[id] = c->rho[id] * c->w[id];
            }
    initialize_vortices(c);
    for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) c->inlet_attr[(size_t)j * NZ + k] = (c->attr[ID(0, j, k)] == 1) ? 1 : 0;
    c->t_loop = start_step;
}

/* ------------------------------------------------------------------ RHS pieces */

/* les_combustion_solver.c:1307-1470 -- 7-point box filter on fluid cells, copy elsewhere.
 * (The uG/vG/wG outputs of the reference are never read and are not restated.) */
static void box_filter(orc_ctx* c, const double* in, double* out) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double den = 6.0 + FILTER_WEIGHT_CENTER;
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ; k++) {
                size_t id = ID(i, j, k);
                if (i >= 1 && i < NX - 1 && j >= 1 && j < NY - 1 && k >= 1 && k < NZ - 1 && c->attr[id] == 3) {
                    out[id] = (in[ID(i - 1, j, k)] + in[ID(i, j - 1, k)] + in[ID(i, j, k - 1)] +
                               FILTER_WEIGHT_CENTER * in[id] +
                               in[ID(i, j, k + 1)] + in[ID(i, j + 1, k)] + in[ID(i + 1, j, k)]) / den;
                } else {
                    out[id] = in[id];
                }
            }
}

/* :1489-1565 */
static void update_nu_mix(orc_ctx* c) {
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            double Tl = c->T_f[id];
            if (Tl <= 0) { c->nu[id] = 1.5e-5; c->mu_mix[id] = 1.8e-5; continue; }
            double X[NSP], syw = 0.0;
            for (int s = 0; s < NSP; s++) syw += c->Y_f[s][id] / (c->mw[s] / 1000.0);
            if (syw < 1e-9) { c->nu[id] = 1.5e-5; c->mu_mix[id] = 1.8e-5; continue; }
            for (int s = 0; s < NSP; s++) X[s] = (c->Y_f[s][id] / (c->mw[s] / 1000.0)) / syw;
            double mu = 0.0, muk[NSP];
            for (int s = 0; s < NSP; s++) muk[s] = mu_dynamic(c, s, Tl);
            for (int a = 0; a < NSP; a++) {
                if (X[a] < 1e-12) continue;
                double mu_i = muk[a], M_i = c->mw[a], den = 0.0;
                for (int b = 0; b < NSP; b++) {
                    if (X[b] < 1e-12) continue;
                    double mu_j = muk[b], M_j = c->mw[b];
                    double ph = pow(1.0 + pow(mu_i / mu_j, 0.5) * pow(M_j / M_i, 0.25), 2) / (sqrt(8.0) * sqrt(1.0 + M_i / M_j));
                    den += X[b] * ph;
                }
                if (den > 1e-9) mu += (X[a] * mu_i) / den;
            }
            c->mu_mix[id] = fmax(MIN_MU_MIX_CLIP, mu);
            if (c->rho_f[id] > 1e-3) c->nu[id] = c->mu_mix[id] / c->rho_f[id];
            else c->nu[id] = 1.5e-5;
            c->nu[id] = fmax(MIN_NU_MIX_CLIP, c->nu[id]);
        } else {
            c->nu[id] = 1.5e-5;
            c->mu_mix[id] = 1.8e-5;
        }
    }
}

/* :1569-1633 */
static void calculate_nu_t(orc_ctx* c) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double DX = c->DX, DY = c->DY, DZ = c->DZ, Delta = DX;
    const double* uf = c->u_f; const double* vf = c->v_f; const double* wf = c->w_f;
    for (int i = 1; i < NX - 1; i++)
        for (int j = 1; j < NY - 1; j++)
            for (int k = 1; k < NZ - 1; k++) {
                size_t id = ID(i, j, k);
                if (c->attr[id] == 3) {
                    double du_dx = (uf[ID(i + 1, j, k)] - uf[ID(i - 1, j, k)]) / (2.0 * DX);
                    double dv_dy = (vf[ID(i, j + 1, k)] - vf[ID(i, j - 1, k)]) / (2.0 * DY);
                    double dw_dz = (wf[ID(i, j, k + 1)] - wf[ID(i, j, k - 1)]) / (2.0 * DZ);
                    double du_dy = (uf[ID(i, j + 1, k)] - uf[ID(i, j - 1, k)]) / (2.0 * DY);
                    double du_dz = (uf[ID(i, j, k + 1)] - uf[ID(i, j, k - 1)]) / (2.0 * DZ);
                    double dv_dx = (vf[ID(i + 1, j, k)] - vf[ID(i - 1, j, k)]) / (2.0 * DX);
                    double dv_dz = (vf[ID(i, j, k + 1)] - vf[ID(i, j, k - 1)]) / (2.0 * DZ);
                    double dw_dx = (wf[ID(i + 1, j, k)] - wf[ID(i - 1, j, k)]) / (2.0 * DX);
                    double dw_dy = (wf[ID(i, j + 1, k)] - wf[ID(i, j - 1, k)]) / (2.0 * DY);
                    double S11 = du_dx, S22 = dv_dy, S33 = dw_dz;
                    double S12 = 0.5 * (du_dy + dv_dx), S13 = 0.5 * (du_dz + dw_dx), S23 = 0.5 * (dv_dz + dw_dy);
                    c->SijSij[id] = 2.0 * (S12 * S12 + S13 * S13 + S23 * S23) + S11 * S11 + S22 * S22 + S33 * S33;
                    c->S_mag[id] = sqrt(2.0 * c->SijSij[id]);
                    c->div_u[id] = du_dx + dv_dy + dw_dz;
                    double g = c->G_f[id];
                    if (g < 0.0) g = 0.0;
                    if (g > 1.0) g = 1.0;
                    double cs = c->c.cs_unburned + (c->c.cs_burnt - c->c.cs_unburned) * g;
                    cs += c->c.cs_flame_boost * 4.0 * g * (1.0 - g);
                    c->nu_t[id] = (cs * Delta) * (cs * Delta) * c->S_mag[id];
                } else {
                    c->SijSij[id] = 0.0; c->div_u[id] = 0.0; c->S_mag[id] = 0.0; c->nu_t[id] = 0.0;
                }
            }
}

/* :683-727 -- conservative flux with the reference's central face coefficients */
static double conv_conservative(const orc_ctx* c, int i, int j, int k, const double* phi,
                                const double* u, const double* v, const double* w, const double* rho) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double DX = c->DX, DY = c->DY, DZ = c->DZ;
    if (i < 2 || i >= NX - 2 || j < 2 || j >= NY - 2 || k < 2 || k >= NZ - 2) {
        size_t id = ID(i, j, k);
        double mf_iph = 0.5 * (rho[ID(i + 1, j, k)] + rho[id]) * 0.5 * (u[ID(i + 1, j, k)] + u[id]);
        double mf_imh = 0.5 * (rho[id] + rho[ID(i - 1, j, k)]) * 0.5 * (u[id] + u[ID(i - 1, j, k)]);
        double mf_jph = 0.5 * (rho[ID(i, j + 1, k)] + rho[id]) * 0.5 * (v[ID(i, j + 1, k)] + v[id]);
        double mf_jmh = 0.5 * (rho[id] + rho[ID(i, j - 1, k)]) * 0.5 * (v[id] + v[ID(i, j - 1, k)]);
        double mf_kph = 0.5 * (rho[ID(i, j, k + 1)] + rho[id]) * 0.5 * (w[ID(i, j, k + 1)] + w[id]);
        double mf_kmh = 0.5 * (rho[id] + rho[ID(i, j, k - 1)]) * 0.5 * (w[id] + w[ID(i, j, k - 1)]);
        double p_iph = (mf_iph > 0) ? phi[id] : phi[ID(i + 1, j, k)];
        double p_imh = (mf_imh > 0) ? phi[ID(i - 1, j, k)] : phi[id];
        double p_jph = (mf_jph > 0) ? phi[id] : phi[ID(i, j + 1, k)];
        double p_jmh = (mf_jmh > 0) ? phi[ID(i, j - 1, k)] : phi[id];
        double p_kph = (mf_kph > 0) ? phi[id] : phi[ID(i, j, k + 1)];
        double p_kmh = (mf_kmh > 0) ? phi[ID(i, j, k - 1)] : phi[id];
        return (mf_iph * p_iph - mf_imh * p_imh) / DX + (mf_jph * p_jph - mf_jmh * p_jmh) / DY + (mf_kph * p_kph - mf_kmh * p_kmh) / DZ;
    }
    size_t id = ID(i, j, k);
    double p_iph, p_imh, p_jph, p_jmh, p_kph, p_kmh;
    double u_iph = 0.5 * (u[ID(i + 1, j, k)] + u[id]); double u_imh = 0.5 * (u[id] + u[ID(i - 1, j, k)]);
    double v_jph = 0.5 * (v[ID(i, j + 1, k)] + v[id]); double v_jmh = 0.5 * (v[id] + v[ID(i, j - 1, k)]);
    double w_kph = 0.5 * (w[ID(i, j, k + 1)] + w[id]); double w_kmh = 0.5 * (w[id] + w[ID(i, j, k - 1)]);
    double r_iph = 0.5 * (rho[ID(i + 1, j, k)] + rho[id]); double r_imh = 0.5 * (rho[id] + rho[ID(i - 1, j, k)]);
    double r_jph = 0.5 * (rho[ID(i, j + 1, k)] + rho[id]); double r_jmh = 0.5 * (rho[id] + rho[ID(i, j - 1, k)]);
    double r_kph = 0.5 * (rho[ID(i, j, k + 1)] + rho[id]); double r_kmh = 0.5 * (rho[id] + rho[ID(i, j, k - 1)]);
    double mf_iph = r_iph * u_iph, mf_imh = r_imh * u_imh;
    double mf_jph = r_jph * v_jph, mf_jmh = r_jmh * v_jmh;
    double mf_kph = r_kph * w_kph, mf_kmh = r_kmh * w_kmh;
    if (u_iph >= 0.0) p_iph = (UW2 * phi[ID(i - 1, j, k)] + UW1 * phi[id] + DW1 * phi[ID(i + 1, j, k)]);
    else p_iph = (UW2 * phi[ID(i + 2, j, k)] + UW1 * phi[ID(i + 1, j, k)] + DW1 * phi[id]);
    if (u_imh >= 0.0) p_imh = (UW2 * phi[ID(i - 2, j, k)] + UW1 * phi[ID(i - 1, j, k)] + DW1 * phi[id]);
    else p_imh = (UW2 * phi[ID(i + 1, j, k)] + UW1 * phi[id] + DW1 * phi[ID(i - 1, j, k)]);
    if (v_jph >= 0.0) p_jph = (UW2 * phi[ID(i, j - 1, k)] + UW1 * phi[id] + DW1 * phi[ID(i, j + 1, k)]);
    else p_jph = (UW2 * phi[ID(i, j + 2, k)] + UW1 * phi[ID(i, j + 1, k)] + DW1 * phi[id]);
    if (v_jmh >= 0.0) p_jmh = (UW2 * phi[ID(i, j - 2, k)] + UW1 * phi[ID(i, j - 1, k)] + DW1 * phi[id]);
    else p_jmh = (UW2 * phi[ID(i, j + 1, k)] + UW1 * phi[id] + DW1 * phi[ID(i, j - 1, k)]);
    if (w_kph >= 0.0) p_kph = (UW2 * phi[ID(i, j, k - 1)] + UW1 * phi[id] + DW1 * phi[ID(i, j, k + 1)]);
    else p_kph = (UW2 * phi[ID(i, j, k + 2)] + UW1 * phi[ID(i, j, k + 1)] + DW1 * phi[id]);
    if (w_kmh >= 0.0) p_kmh = (UW2 * phi[ID(i, j, k - 2)] + UW1 * phi[ID(i, j, k - 1)] + DW1 * phi[id]);
    else p_kmh = (UW2 * phi[ID(i, j, k + 1)] + UW1 * phi[id] + DW1 * phi[ID(i, j, k - 1)]);
    return (mf_iph * p_iph - mf_imh * p_imh) / DX + (mf_jph * p_jph - mf_jmh * p_jmh) / DY + (mf_kph * p_kph - mf_kmh * p_kmh) / DZ;
}

/* :637-678 */
static double conv_nonconservative(const orc_ctx* c, int i, int j, int k, const double* phi,
                                   const double* u, const double* v, const double* w) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double DX = c->DX, DY = c->DY, DZ = c->DZ;
    size_t id = ID(i, j, k);
    if (i < 2 || i >= NX - 2 || j < 2 || j >= NY - 2 || k < 2 || k >= NZ - 2) {
        double f = 0.0;
        if (u[id] >= 0.0) f = u[id] * (phi[id] - phi[ID(i - 1, j, k)]) / DX;
        else f = u[id] * (phi[ID(i + 1, j, k)] - phi[id]) / DX;
        if (v[id] >= 0.0) f += v[id] * (phi[id] - phi[ID(i, j - 1, k)]) / DY;
        else f += v[id] * (phi[ID(i, j + 1, k)] - phi[id]) / DY;
        if (w[id] >= 0.0) f += w[id] * (phi[id] - phi[ID(i, j, k - 1)]) / DZ;
        else f += w[id] * (phi[ID(i, j, k + 1)] - phi[id]) / DZ;
        return f;
    }
    double p_iph, p_imh, p_jph, p_jmh, p_kph, p_kmh;
    if (u[id] >= 0.0) {
        p_iph = (UW2 * phi[ID(i - 1, j, k)] + UW1 * phi[id] + DW1 * phi[ID(i + 1, j, k)]);
        p_imh = (UW2 * phi[ID(i - 2, j, k)] + UW1 * phi[ID(i - 1, j, k)] + DW1 * phi[id]);
    } else {
        p_iph = (UW2 * phi[ID(i + 2, j, k)] + UW1 * phi[ID(i + 1, j, k)] + DW1 * phi[id]);
        p_imh = (UW2 * phi[ID(i + 1, j, k)] + UW1 * phi[id] + DW1 * phi[ID(i - 1, j, k)]);
    }
    if (v[id] >= 0.0) {
        p_jph = (UW2 * phi[ID(i, j - 1, k)] + UW1 * phi[id] + DW1 * phi[ID(i, j + 1, k)]);
        p_jmh = (UW2 * phi[ID(i, j - 2, k)] + UW1 * phi[ID(i, j - 1, k)] + DW1 * phi[id]);
    } else {
        p_jph = (UW2 * phi[ID(i, j + 2, k)] + UW1 * phi[ID(i, j + 1, k)] + DW1 * phi[id]);
        p_jmh = (UW2 * phi[ID(i, j + 1, k)] + UW1 * phi[id] + DW1 * phi[ID(i, j - 1, k)]);
    }
    if (w[id] >= 0.0) {
        p_kph = (UW2 * phi[ID(i, j, k - 1)] + UW1 * phi[id] + DW1 * phi[ID(i, j, k + 1)]);
        p_kmh = (UW2 * phi[ID(i, j, k - 2)] + UW1 * phi[ID(i, j, k - 1)] + DW1 * phi[id]);
    } else {
        p_kph = (UW2 * phi[ID(i, j, k + 2)] + UW1 * phi[ID(i, j, k + 1)] + DW1 * phi[id]);
        p_kmh = (UW2 * phi[ID(i, j, k + 1)] + UW1 * phi[id] + DW1 * phi[ID(i, j, k - 1)]);
    }
    double cx = u[id] * (p_iph - p_imh) / DX;
    double cy = v[id] * (p_jph - p_jmh) / DY;
    double cz = w[id] * (p_kph - p_kmh) / DZ;
    return cx + cy + cz;
}

/* :735-744 */
static void weno5_smoothness(double v1, double v2, double v3, double v4, double v5, double* is0, double* is1, double* is2) {
    *is0 = (13.0 / 12.0) * pow(v1 - 2.0 * v2 + v3, 2) + (1.0 / 4.0) * pow(v1 - 4.0 * v2 + 3.0 * v3, 2);
    *is1 = (13.0 / 12.0) * pow(v2 - 2.0 * v3 + v4, 2) + (1.0 / 4.0) * pow(v2 - v4, 2);
    *is2 = (13.0 / 12.0) * pow(v3 - 2.0 * v4 + v5, 2) + (1.0 / 4.0) * pow(3.0 * v3 - 4.0 * v4 + v5, 2);
}

/* :749-827 (the discarded intermediate "grad" values of the reference are omitted) */
static double weno5_gradient_1d(const double p[6], double dx) {
    double is0_p, is1_p, is2_p;
    weno5_smoothness(p[1], p[2], p[3], p[4], p[5], &is0_p, &is1_p, &is2_p);
    const double eps = 1.0e-6;
    const double d0_p = 3.0 / 10.0, d1_p = 6.0 / 10.0, d2_p = 1.0 / 10.0;
    double a0p = d0_p / pow(eps + is0_p, 2), a1p = d1_p / pow(eps + is1_p, 2), a2p = d2_p / pow(eps + is2_p, 2);
    double sap = a0p + a1p + a2p;
    double w0p = a0p / sap, w1p = a1p / sap, w2p = a2p / sap;
    double s0p = (2.0 * p[1] - 7.0 * p[2] + 11.0 * p[3]) / 6.0;
    double s1p = (-p[2] + 5.0 * p[3] + 2.0 * p[4]) / 6.0;
    double s2p = (2.0 * p[3] + 5.0 * p[4] - p[5]) / 6.0;
    double phi_iph = w0p * s0p + w1p * s1p + w2p * s2p;
    double is0_m, is1_m, is2_m;
    weno5_smoothness(p[0], p[1], p[2], p[3], p[4], &is0_m, &is1_m, &is2_m);
    const double d0_m = 1.0 / 10.0, d1_m = 6.0 / 10.0, d2_m = 3.0 / 10.0;
    double a0m = d0_m / pow(eps + is0_m, 2), a1m = d1_m / pow(eps + is1_m, 2), a2m = d2_m / pow(eps + is2_m, 2);
    double sam = a0m + a1m + a2m;
    double w0m = a0m / sam, w1m = a1m / sam, w2m = a2m / sam;
    double s0m = (-p[0] + 5.0 * p[1] + 2.0 * p[2]) / 6.0;
    double s1m = (2.0 * p[1] + 5.0 * p[2] - p[3]) / 6.0;
    double s2m = (11.0 * p[2] - 7.0 * p[3] + 2.0 * p[4]) / 6.0;
    double phi_imh = w0m * s0m + w1m * s1m + w2m * s2m;
    return (phi_iph - phi_imh) / dx;
}

/* :2017-2028 */
static double superbee(double r) {
    if (r <= 0.0) return 0.0;
    double t1 = fmin(2.0 * r, 1.0);
    double t2 = fmin(r, 2.0);
    return fmax(t1, t2);
}

/* MUSCL-superbee along one axis; pm2..pp2 are phi at offsets -2..+2 (:2058-2094) */
static double muscl_axis(double vel, double pm2, double pm1, double p0, double pp1, double pp2, double d) {
    if (vel >= 0.0) {
        double dup_im = pm1 - pm2, ddn_im = p0 - pm1;
        double r_im = (fabs(ddn_im) < SMALL_NUMBER) ? 1e9 : dup_im / ddn_im;
        double phi_imh = pm1 + 0.5 * superbee(r_im) * ddn_im;
        double dup_i = p0 - pm1, ddn_i = pp1 - p0;
        double r_i = (fabs(ddn_i) < SMALL_NUMBER) ? 1e9 : dup_i / ddn_i;
        double phi_iph = p0 + 0.5 * superbee(r_i) * ddn_i;
        return vel * (phi_iph - phi_imh) / d;
    } else {
        double dup_i = pp1 - p0, ddn_i = p0 - pm1;
        double r_i = (fabs(ddn_i) < SMALL_NUMBER) ? 1e9 : dup_i / ddn_i;
        double phi_imh = p0 - 0.5 * superbee(r_i) * ddn_i;
        double dup_ip = pp2 - pp1, ddn_ip = pp1 - p0;
        double r_ip = (fabs(ddn_ip) < SMALL_NUMBER) ? 1e9 : dup_ip / ddn_ip;
        double phi_iph = pp1 - 0.5 * superbee(r_ip) * ddn_ip;
        return vel * (phi_iph - phi_imh) / d;
    }
}

/* :2037-2159 */
static double conv_muscl(const orc_ctx* c, int i, int j, int k, const double* phi,
                         const double* u, const double* v, const double* w) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    size_t id = ID(i, j, k);
    if (i < 2 || i >= NX - 2 || j < 2 || j >= NY - 2 || k < 2 || k >= NZ - 2) {
        double f = 0.0;
        if (u[id] >= 0.0) f = u[id] * (phi[id] - phi[ID(i - 1, j, k)]) / c->DX;
        else f = u[id] * (phi[ID(i + 1, j, k)] - phi[id]) / c->DX;
        if (v[id] >= 0.0) f += v[id] * (phi[id] - phi[ID(i, j - 1, k)]) / c->DY;
        else f += v[id] * (phi[ID(i, j + 1, k)] - phi[id]) / c->DY;
        if (w[id] >= 0.0) f += w[id] * (phi[id] - phi[ID(i, j, k - 1)]) / c->DZ;
        else f += w[id] * (phi[ID(i, j, k + 1)] - phi[id]) / c->DZ;
        return f;
    }
    double cx = muscl_axis(u[id], phi[ID(i - 2, j, k)], phi[ID(i - 1, j, k)], phi[id], phi[ID(i + 1, j, k)], phi[ID(i + 2, j, k)], c->DX);
    double cy = muscl_axis(v[id], phi[ID(i, j - 2, k)], phi[ID(i, j - 1, k)], phi[id], phi[ID(i, j + 1, k)], phi[ID(i, j + 2, k)], c->DY);
    double cz = muscl_axis(w[id], phi[ID(i, j, k - 2)], phi[ID(i, j, k - 1)], phi[id], phi[ID(i, j, k + 1)], phi[ID(i, j, k + 2)], c->DZ);
    return cx + cy + cz;
}

/* :2190-2236 */
static double teno5_reconstruct(double v0, double v1, double v2, double v3, double v4) {
    double is0 = (13.0 / 12.0) * pow(v0 - 2.0 * v1 + v2, 2) + (1.0 / 4.0) * pow(v0 - 4.0 * v1 + 3.0 * v2, 2);
    double is1 = (13.0 / 12.0) * pow(v1 - 2.0 * v2 + v3, 2) + (1.0 / 4.0) * pow(v1 - v3, 2);
    double is2 = (13.0 / 12.0) * pow(v2 - 2.0 * v3 + v4, 2) + (1.0 / 4.0) * pow(3.0 * v2 - 4.0 * v3 + v4, 2);
    int d0 = (is0 < TENO_CUTOFF) ? 1 : 0, d1 = (is1 < TENO_CUTOFF) ? 1 : 0, d2 = (is2 < TENO_CUTOFF) ? 1 : 0;
    double p0 = (2.0 * v0 - 7.0 * v1 + 11.0 * v2) / 6.0;
    double p1 = (-v1 + 5.0 * v2 + 2.0 * v3) / 6.0;
    double p2 = (2.0 * v2 + 5.0 * v3 - v4) / 6.0;
    if (d0 + d1 + d2 == 0) {
        if (is0 <= is1 && is0 <= is2) return p0;
        else if (is1 <= is0 && is1 <= is2) return p1;
        else return p2;
    }
    const double c0 = 0.1, c1 = 0.6, c2 = 0.3;
    double w0 = d0 * c0, w1 = d1 * c1, w2 = d2 * c2;
    double ws = w0 + w1 + w2;
    if (ws < 1e-40) return p1;
    return (w0 * p0 + w1 * p1 + w2 * p2) / ws;
}

/* one axis of :2258-2295; q[0..6] = phi at offsets -3..+3 */
static double teno_axis(double vel, const double q[7], double d) {
    if (vel >= 0.0) {
        double ph = teno5_reconstruct(q[1], q[2], q[3], q[4], q[5]);
        double mh = teno5_reconstruct(q[0], q[1], q[2], q[3], q[4]);
        return vel * (ph - mh) / d;
    } else {
        double mh = teno5_reconstruct(q[5], q[4], q[3], q[2], q[1]);
        double ph = teno5_reconstruct(q[6], q[5], q[4], q[3], q[2]);
        return vel * (ph - mh) / d;
    }
}

/* :2245-2298 */
static double conv_teno(const orc_ctx* c, int i, int j, int k, const double* phi,
                        const double* u, const double* v, const double* w) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    if (i < 3 || i >= NX - 3 || j < 3 || j >= NY - 3 || k < 3 || k >= NZ - 3)
        return conv_nonconservative(c, i, j, k, phi, u, v, w);
    size_t id = ID(i, j, k);
    double q[7];
    for (int m = 0; m < 7; m++) q[m] = phi[ID(i - 3 + m, j, k)];
    double fx = teno_axis(u[id], q, c->DX);
    for (int m = 0; m < 7; m++) q[m] = phi[ID(i, j - 3 + m, k)];
    double fy = teno_axis(v[id], q, c->DY);
    for (int m = 0; m < 7; m++) q[m] = phi[ID(i, j, k - 3 + m)];
    double fz = teno_axis(w[id], q, c->DZ);
    return fx + fy + fz;
}

/* :1913-1965 */
static void calculate_ST(orc_ctx* c) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double DX = c->DX;
    const double S_L_param = c->c.s_l, nu_u = c->c.nu_unburnt, D3 = c->c.d3;
    const double tau = (c->c.rho_unburnt_approx / c->c.rho_burnt_approx) - 1.0;   /* :2701-2703 */
    for (int i = 1; i < NX - 1; ++i)
        for (int j = 1; j < NY - 1; ++j)
            for (int k = 1; k < NZ - 1; ++k) {
                size_t id = ID(i, j, k);
                if (c->attr[id] == 3) {
                    double nul = c->nu[id];
                    double num = c->SijSij[id] - (c->div_u[id] * c->div_u[id]) * ONE_THIRD;
                    double X = (pow(DX, 4.0) / (nul * nul)) * num;
                    double d_eta;
                    if (X < SMALL_NUMBER) d_eta = 1.0;
                    else {
                        double pX = pow(X, 0.75);
                        double arg = SSR_B * pX;
                        d_eta = SSR_A * pX * (arg > 1.0 ? log(arg) : 0.0);
                    }
                    double eta = DX / (d_eta + SMALL_NUMBER);
                    double dF = nu_u / (S_L_param + SMALL_NUMBER);
                    double Dce = 8.0 * eta;
                    double asf = 8.0 * exp(SSR_C * dF / (Dce + SMALL_NUMBER));
                    double base = asf * eta / DX;
                    double wr = pow(base, (2.0 - D3));
                    double te = 0.0;
                    if (tau * S_L_param > SMALL_NUMBER) te = DX * fmax(0.0, c->div_u[id]) / (tau * S_L_param);
                    double ratio = wr + te;
                    c->ST[id] = S_L_param * fmax(0.0, ratio);
                    c->ST[id] = fmax(S_L_param, c->ST[id]);
                } else {
                    c->ST[id] = S_L_param;
                }
            }
}

/* :1684-1756 */
static void update_Dk(orc_ctx* c) {
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            double Tl = c->T_f[id];
            if (Tl <= 0) { for (int s = 0; s < NSP; s++) c->Dk[s][id] = 1e-5; continue; }
            double X[NSP], syw = 0.0;
            for (int s = 0; s < NSP; s++) syw += c->Y_f[s][id] / (c->mw[s] / 1000.0);
            if (syw < 1e-9) { for (int s = 0; s < NSP; s++) c->Dk[s][id] = 1e-5; continue; }
            for (int s = 0; s < NSP; s++) X[s] = (c->Y_f[s][id] / (c->mw[s] / 1000.0)) / syw;
            for (int a = 0; a < NSP; a++) {
                double sx = 0.0;
                for (int b = 0; b < NSP; b++) {
                    if (a == b) continue;
                    if (X[b] > 1e-12) {
                        double D = dkj_dynamic(c, a, b, Tl);
                        if (D > 1e-12) sx += X[b] / D;
                    }
                }
                double Dv;
                if (fabs(1.0 - X[a]) < 1e-9) {
                    int o = (a != N2_INDEX) ? N2_INDEX : O2_INDEX;
                    Dv = dkj_dynamic(c, a, o, Tl);
                } else if (sx > 1e-12) {
                    Dv = (1.0 - X[a]) / sx;
                } else {
                    Dv = 1e-5;
                }
                double tp = pressure_const + c->P_f[id];
                if (tp > 1.0) Dv *= (PATM / tp);
                c->Dk[a][id] = fmax(1e-9, fmin(1e-2, Dv));
            }
        } else {
            for (int s = 0; s < NSP; s++) c->Dk[s][id] = 0.0;
        }
    }
}

/* :1762-1795 */
static void update_Cp_mix(orc_ctx* c) {
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            double Tl = c->T_f[id];
            if (Tl <= 0) { c->Cp_mix[id] = 1000.0; continue; }
            double cp = 0.0;
            for (int s = 0; s < NSP; s++) cp += c->Y_f[s][id] * cp_dynamic(c, s, Tl);
            c->Cp_mix[id] = fmax(100.0, cp);
        } else {
            c->Cp_mix[id] = 1000.0;
        }
    }
}

/* :1798-1881 */
static void update_lambda_alpha(orc_ctx* c) {
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            double Tl = c->T_f[id];
            if (Tl <= 0) { c->lambda_mix[id] = 0.025; c->alpha[id] = 1.8e-5; continue; }
            double X[NSP], syw = 0.0;
            for (int s = 0; s < NSP; s++) syw += c->Y_f[s][id] / (c->mw[s] / 1000.0);
            if (syw < 1e-9) { c->lambda_mix[id] = 0.025; c->alpha[id] = 1.8e-5; continue; }
            for (int s = 0; s < NSP; s++) X[s] = (c->Y_f[s][id] / (c->mw[s] / 1000.0)) / syw;
            double lm = 0.0, lk[NSP], mk[NSP];
            for (int s = 0; s < NSP; s++) { lk[s] = lambda_dynamic(c, s, Tl); mk[s] = mu_dynamic(c, s, Tl); }
            for (int a = 0; a < NSP; a++) {
                if (X[a] < 1e-12) continue;
                double li = lk[a], mi = mk[a], Mi = c->mw[a], den = 0.0;
                for (int b = 0; b < NSP; b++) {
                    if (X[b] < 1e-12) continue;
                    double mj = mk[b], Mj = c->mw[b];
                    double A = pow(1.0 + pow(mi / mj, 0.5) * pow(Mj / Mi, 0.25), 2) / (sqrt(8.0) * sqrt(1.0 + Mi / Mj));
                    den += X[b] * A;
                }
                if (den > 1e-9) lm += (X[a] * li) / den;
            }
            c->lambda_mix[id] = fmax(1e-3, lm);
            if (c->rho_f[id] > 1e-6 && c->Cp_mix[id] > 1e-6) c->alpha[id] = c->lambda_mix[id] / (c->rho_f[id] * c->Cp_mix[id]);
            else c->alpha[id] = 1.8e-5;
            c->alpha[id] = fmax(1e-7, c->alpha[id]);
        } else {
            c->lambda_mix[id] = 0.0;
            c->alpha[id] = 0.0;
        }
    }
}

/* :2494-2963 calculate_RHS; k_* are the outputs for stage r */
static void calculate_rhs(orc_ctx* c, int t_loop, const double* u_in, const double* v_in, const double* w_in,
                          const double* T_in, const double* G_in, double* const* Y_in, const double* rho_in, int r) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double DX = c->DX, DY = c->DY, DZ = c->DZ;
    double* ku = c->k_rhou[r]; double* kv = c->k_rhov[r]; double* kw = c->k_rhow[r];
    double* kT = c->k_T[r]; double* kG = c->k_G[r];

    /* 1. filter (:2520) */
    box_filter(c, u_in, c->u_f); box_filter(c, v_in, c->v_f); box_filter(c, w_in, c->w_f);
    box_filter(c, c->P, c->P_f); box_filter(c, T_in, c->T_f); box_filter(c, rho_in, c->rho_f);
    for (int s = 0; s < NSP; s++) box_filter(c, Y_in[s], c->Y_f[s]);
    box_filter(c, G_in, c->G_f);
    /* 2. properties and eddy viscosity (:2530-2531) */
    update_nu_mix(c);
    calculate_nu_t(c);
    /* 3a. dynamic reference density (:2536-2550) */
    double tm = 0.0, tv = 0.0;
    for (size_t id = 0; id < c->n; id++) {
        int a = c->attr[id];
        if (a == 1 || a == 2 || a == 3 || a == 5) { tm += c->rho_f[id] * DX * DY * DZ; tv += DX * DY * DZ; }
    }
    double rho_avg = (tv > 0) ? (tm / tv) : DEFAULT_RHO_AIR;
    const double* uf = c->u_f; const double* vf = c->v_f; const double* wf = c->w_f;
    const double* rf = c->rho_f; const double* Gf = c->G_f; const double* nut = c->nu_t;
    const double ic_z = c->c.lz / 2.0;
    /* momentum (:2552-2697) */
    for (int i = 1; i < NX - 1; i++)
        for (int j = 1; j < NY - 1; j++)
            for (int k = 1; k < NZ - 1; k++) {
                size_t id = ID(i, j, k);
                if (c->attr[id] != 3) { ku[id] = 0.0; kv[id] = 0.0; kw[id] = 0.0; continue; }
                double cu = conv_conservative(c, i, j, k, uf, uf, vf, wf, rf);
                double cv = conv_conservative(c, i, j, k, vf, uf, vf, wf, rf);
                double cw = conv_conservative(c, i, j, k, wf, uf, vf, wf, rf);
                double mu_eff = c->mu_mix[id] + rf[id] * nut[id];
                double d2u_dx2 = (uf[ID(i + 1, j, k)] - 2.0 * uf[id] + uf[ID(i - 1, j, k)]) / (DX * DX);
                double d2u_dy2 = (uf[ID(i, j + 1, k)] - 2.0 * uf[id] + uf[ID(i, j - 1, k)]) / (DY * DY);
                double d2u_dz2 = (uf[ID(i, j, k + 1)] - 2.0 * uf[id] + uf[ID(i, j, k - 1)]) / (DZ * DZ);
                double diff_u = mu_eff * (d2u_dx2 + d2u_dy2 + d2u_dz2);
                double d2v_dx2 = (vf[ID(i + 1, j, k)] - 2.0 * vf[id] + vf[ID(i - 1, j, k)]) / (DX * DX);
                double d2v_dy2 = (vf[ID(i, j + 1, k)] - 2.0 * vf[id] + vf[ID(i, j - 1, k)]) / (DY * DY);
                double d2v_dz2 = (vf[ID(i, j, k + 1)] - 2.0 * vf[id] + vf[ID(i, j, k - 1)]) / (DZ * DZ);
                double diff_v = mu_eff * (d2v_dx2 + d2v_dy2 + d2v_dz2);
                double d2w_dx2 = (wf[ID(i + 1, j, k)] - 2.0 * wf[id] + wf[ID(i - 1, j, k)]) / (DX * DX);
                double d2w_dy2 = (wf[ID(i, j + 1, k)] - 2.0 * wf[id] + wf[ID(i, j - 1, k)]) / (DY * DY);
                double d2w_dz2 = (wf[ID(i, j, k + 1)] - 2.0 * wf[id] + wf[ID(i, j, k - 1)]) / (DZ * DZ);
                double diff_w = mu_eff * (d2w_dx2 + d2w_dy2 + d2w_dz2);
                double grav = (rf[id] - rho_avg) * G_GRAVITY;
                double fx = 0.0, fy = 0.0, fz = 0.0;
                if (c->c.flame_accel) {
                    double Gl = Gf[id];
                    if (Gl > 0.01 && Gl < 0.99) {
                        double dGx = (Gf[ID(i + 1, j, k)] - Gf[ID(i - 1, j, k)]) / (2.0 * DX);
                        double dGy = (Gf[ID(i, j + 1, k)] - Gf[ID(i, j - 1, k)]) / (2.0 * DY);
                        double dGz = (Gf[ID(i, j, k + 1)] - Gf[ID(i, j, k - 1)]) / (2.0 * DZ);
                        if (dGx < 0.0) dGx = 0.0;
                        if (dGy < 0.0) dGy = 0.0;
                        double zrel = (k * DZ) - ic_z;
                        if (zrel > 0.0) { if (dGz < 0.0) dGz = 0.0; }
                        else { if (dGz > 0.0) dGz = 0.0; }
                        double diff = Gl - c->c.accel_center;
                        double window = exp(-(diff * diff) / (2.0 * c->c.accel_width * c->c.accel_width));
                        double tip_mask = 1.0;
                        double cf = c->c.accel_strength * rf[id] * window * tip_mask;
                        double wx = 0.05, wyz = 1.0;
                        fx = cf * dGx * wx; fy = cf * dGy * wyz; fz = cf * dGz * wyz;
                        double zp = k * DZ, ramp = 1.0;
                        if (zp < FLAME_RAMP_DISTANCE) ramp = zp / FLAME_RAMP_DISTANCE;
                        fx *= ramp; fy *= ramp; fz *= ramp;
                    }
                }
                if (fx > MAX_FLAME_FORCE_LIMIT) fx = MAX_FLAME_FORCE_LIMIT;
                if (fx < -MAX_FLAME_FORCE_LIMIT) fx = -MAX_FLAME_FORCE_LIMIT;
                if (fy > MAX_FLAME_FORCE_LIMIT) fy = MAX_FLAME_FORCE_LIMIT;
                if (fy < -MAX_FLAME_FORCE_LIMIT) fy = -MAX_FLAME_FORCE_LIMIT;
                if (fz > MAX_FLAME_FORCE_LIMIT) fz = MAX_FLAME_FORCE_LIMIT;
                if (fz < -MAX_FLAME_FORCE_LIMIT) fz = -MAX_FLAME_FORCE_LIMIT;
                ku[id] = -cu + diff_u + grav + fx;
                kv[id] = -cv + diff_v + fy;
                kw[id] = -cw + diff_w + fz;
            }
    /* (b) G (:2700-2825) */
    calculate_ST(c);
    for (int i = 1; i < NX - 1; i++)
        for (int j = 1; j < NY - 1; j++)
            for (int k = 1; k < NZ - 1; k++) {
                size_t id = ID(i, j, k);
                if (c->attr[id] != 3) { c->gradG_dbg[id] = 0.0; kG[id] = 0.0; continue; }
                double conv = conv_teno(c, i, j, k, Gf, uf, vf, wf);
                const double sct2 = 2.0 * c->c.sc_t;
                double g_iph = (nut[ID(i + 1, j, k)] + nut[id]) / sct2;
                double g_imh = (nut[id] + nut[ID(i - 1, j, k)]) / sct2;
                double g_jph = (nut[ID(i, j + 1, k)] + nut[id]) / sct2;
                double g_jmh = (nut[id] + nut[ID(i, j - 1, k)]) / sct2;
                double g_kph = (nut[ID(i, j, k + 1)] + nut[id]) / sct2;
                double g_kmh = (nut[id] + nut[ID(i, j, k - 1)]) / sct2;
                double sx = (g_iph * (Gf[ID(i + 1, j, k)] - Gf[id]) / DX - g_imh * (Gf[id] - Gf[ID(i - 1, j, k)]) / DX) / DX;
                double sy = (g_jph * (Gf[ID(i, j + 1, k)] - Gf[id]) / DY - g_jmh * (Gf[id] - Gf[ID(i, j - 1, k)]) / DY) / DY;
                double sz = (g_kph * (Gf[ID(i, j, k + 1)] - Gf[id]) / DZ - g_kmh * (Gf[id] - Gf[ID(i, j, k - 1)]) / DZ) / DZ;
                double sgs = sx + sy + sz;
                double gx, gy, gz;
                if (t_loop < c->c.weno_transition_step) {
                    gx = (Gf[ID(i + 1, j, k)] - Gf[ID(i - 1, j, k)]) / (2.0 * DX);
                    gy = (Gf[ID(i, j + 1, k)] - Gf[ID(i, j - 1, k)]) / (2.0 * DY);
                    gz = (Gf[ID(i, j, k + 1)] - Gf[ID(i, j, k - 1)]) / (2.0 * DZ);
                } else if (i >= 3 && i < NX - 3 && j >= 3 && j < NY - 3 && k >= 3 && k < NZ - 3) {
                    double p[6];
                    for (int m = 0; m < 6; m++) p[m] = Gf[ID(i - 2 + m, j, k)];
                    gx = weno5_gradient_1d(p, DX);
                    for (int m = 0; m < 6; m++) p[m] = Gf[ID(i, j - 2 + m, k)];
                    gy = weno5_gradient_1d(p, DY);
                    for (int m = 0; m < 6; m++) p[m] = Gf[ID(i, j, k - 2 + m)];
                    gz = weno5_gradient_1d(p, DZ);
                } else {
                    gx = (Gf[ID(i + 1, j, k)] - Gf[ID(i - 1, j, k)]) / (2.0 * DX);
                    gy = (Gf[ID(i, j + 1, k)] - Gf[ID(i, j - 1, k)]) / (2.0 * DY);
                    gz = (Gf[ID(i, j, k + 1)] - Gf[ID(i, j, k - 1)]) / (2.0 * DZ);
                }
                double gmag = sqrt(gx * gx + gy * gy + gz * gz);
                c->gradG_dbg[id] = gmag;
                double prop = c->ST[id] * gmag;
                double art = 0.0;
                if (c->c.flame_accel) {
                    double Gl = Gf[id];
                    if (Gl > 0.1 && Gl < 0.99) {
                        double diff = Gl - c->c.accel_center;
                        double window = exp(-(diff * diff) / (2.0 * c->c.accel_width * c->c.accel_width));
                        double d2x = (Gf[ID(i + 1, j, k)] - 2.0 * Gl + Gf[ID(i - 1, j, k)]) / (DX * DX);
                        double d2y = (Gf[ID(i, j + 1, k)] - 2.0 * Gl + Gf[ID(i, j - 1, k)]) / (DY * DY);
                        double d2z = (Gf[ID(i, j, k + 1)] - 2.0 * Gl + Gf[ID(i, j, k - 1)]) / (DZ * DZ);
                        /* TIP_PROTECTION_RADIUS is 0.0, so 1 - exp(-r^2/0) is exactly 1 for j >= 1 (:2806-2807) */
                        double tip_mask = 1.0;
                        double adc = 5.0 * (nut[id] + 1.0e-5) * window * tip_mask;
                        art = adc * (d2x + d2y + d2z);
                    }
                }
                kG[id] = -conv + prop + sgs + art;
            }
    /* (c) species (:2834-2904) */
    const double RELAX = c->c.relax;
    update_Dk(c);
    for (int s = 0; s < NSP; ++s) {
        double* kY = c->k_Y[r][s];
        const double* Yf = c->Y_f[s];
        for (int i = 1; i < NX - 1; i++)
            for (int j = 1; j < NY - 1; j++)
                for (int k = 1; k < NZ - 1; k++) {
                    size_t id = ID(i, j, k);
                    if (c->attr[id] != 3) { kY[id] = 0.0; continue; }
                    double conv = conv_muscl(c, i, j, k, Yf, uf, vf, wf);
                    double d2x = (Yf[ID(i + 1, j, k)] - 2.0 * Yf[id] + Yf[ID(i - 1, j, k)]) / (DX * DX);
                    double d2y = (Yf[ID(i, j + 1, k)] - 2.0 * Yf[id] + Yf[ID(i, j - 1, k)]) / (DY * DY);
                    double d2z = (Yf[ID(i, j, k + 1)] - 2.0 * Yf[id] + Yf[ID(i, j, k - 1)]) / (DZ * DZ);
                    double mol = c->Dk[s][id] * (d2x + d2y + d2z);
                    const double sct2 = 2.0 * c->c.sc_t;
                    double Dt_iph = (nut[ID(i + 1, j, k)] + nut[id]) / sct2, Dt_imh = (nut[id] + nut[ID(i - 1, j, k)]) / sct2;
                    double Dt_jph = (nut[ID(i, j + 1, k)] + nut[id]) / sct2, Dt_jmh = (nut[id] + nut[ID(i, j - 1, k)]) / sct2;
                    double Dt_kph = (nut[ID(i, j, k + 1)] + nut[id]) / sct2, Dt_kmh = (nut[id] + nut[ID(i, j, k - 1)]) / sct2;
                    double fxs = (Dt_iph * (Yf[ID(i + 1, j, k)] - Yf[id]) / DX - Dt_imh * (Yf[id] - Yf[ID(i - 1, j, k)]) / DX) / DX;
                    double fys = (Dt_jph * (Yf[ID(i, j + 1, k)] - Yf[id]) / DY - Dt_jmh * (Yf[id] - Yf[ID(i, j - 1, k)]) / DY) / DY;
                    double fzs = (Dt_kph * (Yf[ID(i, j, k + 1)] - Yf[id]) / DZ - Dt_kmh * (Yf[id] - Yf[ID(i, j, k - 1)]) / DZ) / DZ;
                    double sgs = fxs + fys + fzs;
                    double g = Gf[id];
                    if (g < 0.0) g = 0.0;
                    if (g > 1.0) g = 1.0;
                    double tgt;
                    if (s == C3H8_INDEX) tgt = c->inletYk[C3H8_INDEX] * (1.0 - g);
                    else if (s == O2_INDEX) { double cons = c->inletYk[C3H8_INDEX] * c->stoich_o2; tgt = fmax(0.0, c->inletYk[O2_INDEX] - cons * g); }
                    else if (s == CO2_INDEX) { double pr = c->inletYk[C3H8_INDEX] * c->stoich_co2; tgt = c->inletYk[CO2_INDEX] + pr * g; }
                    else if (s == H2O_INDEX) { double pr = c->inletYk[C3H8_INDEX] * c->stoich_h2o; tgt = c->inletYk[H2O_INDEX] + pr * g; }
                    else tgt = c->inletYk[N2_INDEX];
                    double nud = RELAX * (tgt - Yf[id]);
                    kY[id] = -conv + mol + sgs + nud;
                }
    }
    /* (d) temperature (:2909-2962) */
    update_Cp_mix(c);
    update_lambda_alpha(c);
    const double* Tf = c->T_f;
    for (int i = 1; i < NX - 1; i++)
        for (int j = 1; j < NY - 1; j++)
            for (int k = 1; k < NZ - 1; k++) {
                size_t id = ID(i, j, k);
                if (c->attr[id] != 3) { kT[id] = 0.0; continue; }
                double conv = conv_muscl(c, i, j, k, Tf, uf, vf, wf);
                double d2x = (Tf[ID(i + 1, j, k)] - 2.0 * Tf[id] + Tf[ID(i - 1, j, k)]) / (DX * DX);
                double d2y = (Tf[ID(i, j + 1, k)] - 2.0 * Tf[id] + Tf[ID(i, j - 1, k)]) / (DY * DY);
                double d2z = (Tf[ID(i, j, k + 1)] - 2.0 * Tf[id] + Tf[ID(i, j, k - 1)]) / (DZ * DZ);
                double mol = 0.0;
                if (rf[id] > 1e-6 && c->Cp_mix[id] > 1e-6) mol = c->lambda_mix[id] / (rf[id] * c->Cp_mix[id]) * (d2x + d2y + d2z);
                const double prt2 = 2.0 * c->c.pr_t;
                double k_iph = (nut[ID(i + 1, j, k)] + nut[id]) / prt2, k_imh = (nut[id] + nut[ID(i - 1, j, k)]) / prt2;
                double k_jph = (nut[ID(i, j + 1, k)] + nut[id]) / prt2, k_jmh = (nut[id] + nut[ID(i, j - 1, k)]) / prt2;
                double k_kph = (nut[ID(i, j, k + 1)] + nut[id]) / prt2, k_kmh = (nut[id] + nut[ID(i, j, k - 1)]) / prt2;
                double fxs = (k_iph * (Tf[ID(i + 1, j, k)] - Tf[id]) / DX - k_imh * (Tf[id] - Tf[ID(i - 1, j, k)]) / DX) / DX;
                double fys = (k_jph * (Tf[ID(i, j + 1, k)] - Tf[id]) / DY - k_jmh * (Tf[id] - Tf[ID(i, j - 1, k)]) / DY) / DY;
                double fzs = (k_kph * (Tf[ID(i, j, k + 1)] - Tf[id]) / DZ - k_kmh * (Tf[id] - Tf[ID(i, j, k - 1)]) / DZ) / DZ;
                double sgs = fxs + fys + fzs;
                double g = Gf[id];
                if (g < 0.0) g = 0.0;
                if (g > 1.0) g = 1.0;
                double Tt = c->c.inlet_temperature + g * (c->c.burnt_gas_temperature - c->c.inlet_temperature);
                double nud = RELAX * (Tt - Tf[id]);
                kT[id] = -conv + mol + sgs + nud;
            }
}

/* :1883-1910 -- note the fallback reads the global rho (q3) */
static void rho_from_eos(orc_ctx* c, const double* Tn, double* const* Yn, double* rn) {
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3 || c->attr[id] == 2) {
            double syw = 0.0;
            for (int s = 0; s < NSP; s++) syw += Yn[s][id] / (c->mw[s] / 1000.0);
            if (syw > 1e-9 && Tn[id] > 1.0) {
                double W = 1.0 / syw;
                double Rm = R_univ / W;
                rn[id] = pressure_const / (Rm * Tn[id]);
            } else {
                rn[id] = c->rho[id];
            }
        }
    }
}

/* :4432-4455 (stage combine for stage 1..3, coefficient cf = 0.5/0.5/1.0) */
static void stage_update(orc_ctx* c, int r, double cf) {
    const double dt = c->dt;
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            c->Tt[id] = c->T0[id] + cf * dt * c->k_T[r][id];
            c->Gt[id] = c->G0[id] + cf * dt * c->k_G[r][id];
            for (int s = 0; s < NSP; s++) c->Yt[s][id] = c->Y0[s][id] + cf * dt * c->k_Y[r][s][id];
            c->Tt[id] = fmax(MIN_T_CLIP, fmin(MAX_T_CLIP, c->Tt[id]));
            c->Gt[id] = fmax(0.0, fmin(1.0, c->Gt[id]));
            double sy = 0;
            for (int s = 0; s < NSP; s++) { c->Yt[s][id] = fmax(0.0, fmin(1.0, c->Yt[s][id])); sy += c->Yt[s][id]; }
            if (sy > SMALL_NUMBER) for (int s = 0; s < NSP; s++) c->Yt[s][id] /= sy;
        } else {
            c->Tt[id] = c->T0[id]; c->Gt[id] = c->G0[id];
            for (int s = 0; s < NSP; s++) c->Yt[s][id] = c->Y0[s][id];
        }
    }
    rho_from_eos(c, c->Tt, c->Yt, c->rhot);
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            c->rhout[id] = c->rhou0[id] + cf * dt * c->k_rhou[r][id];
            c->rhovt[id] = c->rhov0[id] + cf * dt * c->k_rhov[r][id];
            c->rhowt[id] = c->rhow0[id] + cf * dt * c->k_rhow[r][id];
            if (c->rhot[id] > SMALL_NUMBER) {
                c->ut[id] = c->rhout[id] / c->rhot[id]; c->vt[id] = c->rhovt[id] / c->rhot[id]; c->wt[id] = c->rhowt[id] / c->rhot[id];
            } else { c->ut[id] = 0; c->vt[id] = 0; c->wt[id] = 0; }
        } else {
            c->ut[id] = c->u[id]; c->vt[id] = c->v[id]; c->wt[id] = c->w[id];
        }
    }
}

/* :2967-3161 */
static void apply_bc(orc_ctx* c) {
    const int NX = c->NX, NY = c->NY, NZ = c->NZ;
    const double Uin = c->c.inlet_velocity, Tin = c->c.inlet_temperature, Tamb = c->c.ambient_temperature;
    double *u = c->u, *v = c->v, *w = c->w, *T = c->T, *G = c->G, *P = c->P;
    for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) {
            size_t i0 = ID(0, j, k), i1 = ID(1, j, k);
            int a0 = c->attr[i0];
            if (a0 == 1) {
                double amp = 0.10 * Uin;
                double r1 = ((double)rand() / RAND_MAX) * 2.0 - 1.0;
                double r2 = ((double)rand() / RAND_MAX) * 2.0 - 1.0;
                double r3 = ((double)rand() / RAND_MAX) * 2.0 - 1.0;
                size_t p = (size_t)j * NZ + k;
                u[i0] = fmax(0.0, Uin + c->u_in[p] + amp * r1);
                v[i0] = c->v_in[p] + amp * r2;
                w[i0] = c->w_in[p] + amp * r3;
                T[i0] = Tin; G[i0] = 0.0;
                for (int s = 0; s < NSP; s++) c->Y[s][i0] = c->inletYk[s];
            } else if (a0 == 4) {
                if (u[i1] < 0) {
                    u[i0] = 0.0; v[i0] = 0.0; w[i0] = 0.0; T[i0] = Tamb; G[i0] = 0.0;
                    for (int s = 0; s < NSP; s++) c->Y[s][i0] = c->ambientYk[s];
                } else {
                    u[i0] = u[i1]; v[i0] = v[i1]; w[i0] = w[i1]; T[i0] = T[i1]; G[i0] = G[i1];
                    for (int s = 0; s < NSP; s++) c->Y[s][i0] = c->Y[s][i1];
                }
            } else if (a0 == 6) {
                u[i0] = 0.0; v[i0] = 0.0; w[i0] = 0.0; T[i0] = T[i1]; G[i0] = G[i1];
                for (int s = 0; s < NSP; s++) c->Y[s][i0] = c->Y[s][i1];
            }
            size_t in = ID(NX - 1, j, k), im = ID(NX - 2, j, k);
            if (c->attr[in] == 2) {
                u[in] = u[im]; v[in] = v[im]; w[in] = w[im]; T[in] = T[im]; G[in] = G[im]; P[in] = P[im];
                for (int s = 0; s < NSP; s++) c->Y[s][in] = c->Y[s][im];
            }
        }
    for (int i = 1; i < NX - 1; i++) {
        for (int k = 0; k < NZ; k++) {
            size_t b = ID(i, 0, k), n1 = ID(i, 1, k);
            if (c->attr[b] == 5) {
                T[b] = T[n1]; G[b] = G[n1]; P[b] = P[n1];
                for (int s = 0; s < NSP; s++) c->Y[s][b] = c->Y[s][n1];
                u[b] = u[n1]; v[b] = 0.0; w[b] = w[n1];
            }
            size_t t = ID(i, NY - 1, k), tm = ID(i, NY - 2, k);
            if (c->attr[t] == 4) {
                if (v[tm] < 0) {
                    u[t] = 0.0; v[t] = 0.0; w[t] = 0.0; T[t] = Tamb; G[t] = 0.0;
                    for (int s = 0; s < NSP; s++) c->Y[s][t] = c->ambientYk[s];
                } else {
                    u[t] = u[tm]; v[t] = v[tm]; w[t] = w[tm]; T[t] = T[tm]; G[t] = G[tm]; P[t] = P[tm];
                    for (int s = 0; s < NSP; s++) c->Y[s][t] = c->Y[s][tm];
                }
            }
        }
        for (int j = 0; j < NY; j++) {
            size_t b = ID(i, j, 0), n1 = ID(i, j, 1);
            if (c->attr[b] == 4) {
                if (w[n1] > 0) {
                    u[b] = 0.0; v[b] = 0.0; w[b] = 0.0; T[b] = Tamb; G[b] = 0.0;
                    for (int s = 0; s < NSP; s++) c->Y[s][b] = c->ambientYk[s];
                } else {
                    u[b] = u[n1]; v[b] = v[n1]; w[b] = w[n1]; T[b] = T[n1]; G[b] = G[n1]; P[b] = P[n1];
                    for (int s = 0; s < NSP; s++) c->Y[s][b] = c->Y[s][n1];
                }
            }
            size_t t = ID(i, j, NZ - 1), tm = ID(i, j, NZ - 2);
            if (c->attr[t] == 4) {
                if (w[tm] < 0) {
                    u[t] = 0.0; v[t] = 0.0; w[t] = 0.0; T[t] = Tamb; G[t] = 0.0;
                    for (int s = 0; s < NSP; s++) c->Y[s][t] = c->ambientYk[s];
                } else {
                    u[t] = u[tm]; v[t] = v[tm]; w[t] = w[tm]; T[t] = T[tm]; G[t] = G[tm]; P[t] = P[tm];
                    for (int s = 0; s < NSP; s++) c->Y[s][t] = c->Y[s][tm];
                }
            }
        }
    }
    for (size_t id = 0; id < c->n; id++) {
        double syw = 0;
        for (int s = 0; s < NSP; ++s) syw += c->Y[s][id] / (c->mw[s] / 1000.0);
        if (syw > 1e-9 && T[id] > 1.0) c->rho[id] = pressure_const / (R_univ / (1.0 / syw) * T[id]);
        else c->rho[id] = 1.2;
        c->rhou[id] = c->rho[id] * u[id];
        c->rhov[id] = c->rho[id] * v[id];
        c->rhow[id] = c->rho[id] * w[id];
        int a = c->attr[id];
        if (a == 3 || a == 2 || a == 5) {
            double sy = 0.0;
            for (int s = 0; s < NSP; s++) sy += c->Y[s][id];
            if (sy > 1e-6) for (int s = 0; s < NSP; s++) c->Y[s][id] /= sy;
        }
    }
}

/* :1472-1485 and :4399-4411 */
static double compute_dt(orc_ctx* c) {
    double mv = 0.0;
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 1 || c->attr[id] == 3) {
            double vel = sqrt(c->u[id] * c->u[id] + c->v[id] * c->v[id] + c->w[id] * c->w[id]);
            if (vel > mv) mv = vel;
        }
    }
    c->max_velocity = mv > SMALL_NUMBER ? mv : c->c.inlet_velocity;
    double dt_conv = c->c.courant * c->DX / (c->max_velocity + SMALL_NUMBER);
    double mnu = 0.0, mal = 0.0;
    for (size_t id = 0; id < c->n; id++)
        if (c->attr[id] == 3) {
            if (c->nu[id] > mnu) mnu = c->nu[id];
            if (c->alpha[id] > mal) mal = c->alpha[id];
        }
    double dtn = c->c.courant_diffusion * (c->DX * c->DX) / (mnu + SMALL_NUMBER);
    double dta = c->c.courant_diffusion * (c->DX * c->DX) / (mal + SMALL_NUMBER);
    return fmin(dt_conv, fmin(dtn, dta));
}

/* one iteration of the time loop, :4399-4555 */
void orc_step(orc_ctx* c) {
    c->dt = compute_dt(c);
    generate_inlet_sem(c, c->dt);
    const double dt = c->dt;
    memcpy(c->rhou0, c->rhou, c->n * sizeof(double));
    memcpy(c->rhov0, c->rhov, c->n * sizeof(double));
    memcpy(c->rhow0, c->rhow, c->n * sizeof(double));
    memcpy(c->T0, c->T, c->n * sizeof(double));
    memcpy(c->G0, c->G, c->n * sizeof(double));
    for (int s = 0; s < NSP; s++) memcpy(c->Y0[s], c->Y[s], c->n * sizeof(double));
    const int t = c->t_loop;
    calculate_rhs(c, t, c->u, c->v, c->w, c->T, c->G, c->Y, c->rho, 0);
    stage_update(c, 0, 0.5);
    calculate_rhs(c, t, c->ut, c->vt, c->wt, c->Tt, c->Gt, c->Yt, c->rhot, 1);
    stage_update(c, 1, 0.5);
    calculate_rhs(c, t, c->ut, c->vt, c->wt, c->Tt, c->Gt, c->Yt, c->rhot, 2);
    stage_update(c, 2, 1.0);
    calculate_rhs(c, t, c->ut, c->vt, c->wt, c->Tt, c->Gt, c->Yt, c->rhot, 3);
    /* final update (:4517-4544) */
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            c->T[id] = c->T0[id] + (dt / 6.0) * (c->k_T[0][id] + 2.0 * c->k_T[1][id] + 2.0 * c->k_T[2][id] + c->k_T[3][id]);
            c->G[id] = c->G0[id] + (dt / 6.0) * (c->k_G[0][id] + 2.0 * c->k_G[1][id] + 2.0 * c->k_G[2][id] + c->k_G[3][id]);
            for (int s = 0; s < NSP; s++)
                c->Y[s][id] = c->Y0[s][id] + (dt / 6.0) * (c->k_Y[0][s][id] + 2.0 * c->k_Y[1][s][id] + 2.0 * c->k_Y[2][s][id] + c->k_Y[3][s][id]);
            c->T[id] = fmax(MIN_T_CLIP, fmin(MAX_T_CLIP, c->T[id]));
            c->G[id] = fmax(0.0, fmin(1.0, c->G[id]));
            double sy = 0;
            for (int s = 0; s < NSP; s++) { c->Y[s][id] = fmax(0.0, fmin(1.0, c->Y[s][id])); sy += c->Y[s][id]; }
            if (sy > SMALL_NUMBER) for (int s = 0; s < NSP; s++) c->Y[s][id] /= sy;
        }
    }
    rho_from_eos(c, c->T, c->Y, c->rho);
    for (size_t id = 0; id < c->n; id++) {
        if (c->attr[id] == 3) {
            c->rhou[id] = c->rhou0[id] + (dt / 6.0) * (c->k_rhou[0][id] + 2.0 * c->k_rhou[1][id] + 2.0 * c->k_rhou[2][id] + c->k_rhou[3][id]);
            c->rhov[id] = c->rhov0[id] + (dt / 6.0) * (c->k_rhov[0][id] + 2.0 * c->k_rhov[1][id] + 2.0 * c->k_rhov[2][id] + c->k_rhov[3][id]);
            c->rhow[id] = c->rhow0[id] + (dt / 6.0) * (c->k_rhow[0][id] + 2.0 * c->k_rhow[1][id] + 2.0 * c->k_rhow[2][id] + c->k_rhow[3][id]);
            if (c->rho[id] > SMALL_NUMBER) {
                c->u[id] = c->rhou[id] / c->rho[id]; c->v[id] = c->rhov[id] / c->rho[id]; c->w[id] = c->rhow[id] / c->rho[id];
            } else { c->u[id] = 0; c->v[id] = 0; c->w[id] = 0; }
        }
    }
    apply_bc(c);
    c->t_loop++;
}

/* stage-1 RHS at the current state without advancing it (per-kernel checks) */
void orc_rhs_only(orc_ctx* c, int t_loop) {
    calculate_rhs(c, t_loop, c->u, c->v, c->w, c->T, c->G, c->Y, c->rho, 0);
}

/* ------------------------------------------------------------------ accessors */

enum {
    ORC_U = 0, ORC_V, ORC_W, ORC_T, ORC_G, ORC_RHO, ORC_Y0, ORC_Y1, ORC_Y2, ORC_Y3, ORC_Y4,
    ORC_NU_T, ORC_S_MAG,
    /* RHS intermediates of the most recent RHS evaluation */
    ORC_U_F = 100, ORC_V_F, ORC_W_F, ORC_T_F, ORC_G_F, ORC_RHO_F, ORC_Y0_F, ORC_Y1_F, ORC_Y2_F, ORC_Y3_F, ORC_Y4_F,
    ORC_NU, ORC_MU_MIX, ORC_ST, ORC_CP, ORC_LAMBDA, ORC_ALPHA, ORC_D0, ORC_D1, ORC_D2, ORC_D3, ORC_D4,
    ORC_K_RHOU, ORC_K_RHOV, ORC_K_RHOW, ORC_K_T, ORC_K_G, ORC_K_Y0, ORC_K_Y1, ORC_K_Y2, ORC_K_Y3, ORC_K_Y4
};

static double* field_ptr(orc_ctx* c, int id) {
    switch (id) {
        case ORC_U: return c->u; case ORC_V: return c->v; case ORC_W: return c->w; case ORC_T: return c->T;
        case ORC_G: return c->G; case ORC_RHO: return c->rho;
        case ORC_NU_T: return c->nu_t; case ORC_S_MAG: return c->S_mag;
        case ORC_U_F: return c->u_f; case ORC_V_F: return c->v_f; case ORC_W_F: return c->w_f; case ORC_T_F: return c->T_f;
        case ORC_G_F: return c->G_f; case ORC_RHO_F: return c->rho_f;
        case ORC_NU: return c->nu; case ORC_MU_MIX: return c->mu_mix; case ORC_ST: return c->ST; case ORC_CP: return c->Cp_mix;
        case ORC_LAMBDA: return c->lambda_mix; case ORC_ALPHA: return c->alpha;
        case ORC_K_RHOU: return c->k_rhou[0]; case ORC_K_RHOV: return c->k_rhov[0]; case ORC_K_RHOW: return c->k_rhow[0];
        case ORC_K_T: return c->k_T[0]; case ORC_K_G: return c->k_G[0];
        default: break;
    }
    if (id >= ORC_Y0 && id <= ORC_Y4) return c->Y[id - ORC_Y0];
    if (id >= ORC_Y0_F && id <= ORC_Y4_F) return c->Y_f[id - ORC_Y0_F];
    if (id >= ORC_D0 && id <= ORC_D4) return c->Dk[id - ORC_D0];
    if (id >= ORC_K_Y0 && id <= ORC_K_Y4) return c->k_Y[0][id - ORC_K_Y0];
    return NULL;
}

int orc_get_field(orc_ctx* c, int id, double* out) {
    double* p = field_ptr(c, id);
    if (!p) return -1;
    memcpy(out, p, c->n * sizeof(double));
    return 0;
}

/* Set a state field (u,v,w,T,G,rho,Y0..4); keeps rhou = rho*u as after a checkpoint load
 * (les_combustion_solver.c:3717-3721). */
int orc_set_field(orc_ctx* c, int id, const double* in) {
    if (id < ORC_U || id > ORC_Y4) return -1;
    double* p = field_ptr(c, id);
    memcpy(p, in, c->n * sizeof(double));
    for (size_t q = 0; q < c->n; q++) {
        c->rhou[q] = c->rho[q] * c->u[q]; c->rhov[q] = c->rho[q] * c->v[q]; c->rhow[q] = c->rho[q] * c->w[q];
    }
    return 0;
}

int orc_get_attr(orc_ctx* c, int* out) { memcpy(out, c->attr, c->n * sizeof(int)); return 0; }
double orc_dt(orc_ctx* c) { return c->dt; }
int orc_t_loop(orc_ctx* c) { return c->t_loop; }
void orc_set_t_loop(orc_ctx* c, int t) { c->t_loop = t; }
double orc_max_velocity(orc_ctx* c) { return c->max_velocity; }
int orc_get_inflow(orc_ctx* c, double* out) {
    size_t np = (size_t)c->NY * c->NZ;
    memcpy(out, c->u_in, np * sizeof(double)); memcpy(out + np, c->v_in, np * sizeof(double)); memcpy(out + 2 * np, c->w_in, np * sizeof(double));
    return 0;
}
int orc_get_vortices(orc_ctx* c, double* out) {
    for (int q = 0; q < c->c.num_vortices; q++) {
        out[7 * q + 0] = c->vort[q].x; out[7 * q + 1] = c->vort[q].y; out[7 * q + 2] = c->vort[q].z;
        out[7 * q + 3] = c->vort[q].radius; out[7 * q + 4] = c->vort[q].su; out[7 * q + 5] = c->vort[q].sv; out[7 * q + 6] = c->vort[q].sw;
    }
    return c->c.num_vortices;
}
void orc_get_inlet_yk(orc_ctx* c, double* in5, double* amb5, double* stoich3) {
    for (int s = 0; s < NSP; s++) { in5[s] = c->inletYk[s]; amb5[s] = c->ambientYk[s]; }
    stoich3[0] = c->stoich_o2; stoich3[1] = c->stoich_co2; stoich3[2] = c->stoich_h2o;
}
size_t orc_sizeof_config(void) { return sizeof(orc_config); }
