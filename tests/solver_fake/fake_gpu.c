/*
 * Stand-in for the CUDA library under host/les_host.c (the lesgpu_* calls of les_gpu.h), so
 * that the host driver's own logic -- the rand() stream, the vortex bookkeeping, the dt
 * formula, checkpoint / resume files -- can be tested on a machine without a GPU.  Test
 * infrastructure, not product code.
 *
 * The "device" keeps the state on the host.  A step changes it by a deterministic function of
 * dt, t_loop, the vortex table and the inflow noise it was given, and sets the nu/alpha
 * maxima from the step index, so that a resumed run reproduces an uninterrupted one only if
 * the host restored every input the step depends on.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "les_gpu.h"

struct lesgpu_ctx {
    lesgpu_config cfg;
    size_t n;
    int* attr;
    double* f[LESGPU_NSTATE];
    double numax, alphamax;
    int have_attr, have_state;
    const double* vort;
    int nv;
    double noise0;
    int uploads_attr;
};

int lesgpu_load_species(const char* chem_path, const char* tran_path, lesgpu_species* out) {
    (void)chem_path; (void)tran_path;
    memset(out, 0, sizeof(*out));
    const double mw[LESGPU_NSP] = {44.097, 31.998, 28.014, 44.009, 18.015};
    for (int q = 0; q < LESGPU_NSP; q++) { out->mw[q] = mw[q]; out->t_mid[q] = 1000.0; }
    return LESGPU_OK;
}

int lesgpu_create(const lesgpu_config* cfg, const lesgpu_species* sp, lesgpu_ctx** out) {
    (void)sp;
    lesgpu_ctx* c = (lesgpu_ctx*)calloc(1, sizeof(lesgpu_ctx));
    if (!c) return LESGPU_ENOMEM;
    c->cfg = *cfg;
    c->n = (size_t)cfg->nx * cfg->ny * cfg->nz;
    c->attr = (int*)calloc(c->n, sizeof(int));
    for (int q = 0; q < LESGPU_NSTATE; q++) c->f[q] = (double*)calloc(c->n, sizeof(double));
    *out = c;
    return LESGPU_OK;
}

void lesgpu_destroy(lesgpu_ctx* c) {
    if (!c) return;
    free(c->attr);
    for (int q = 0; q < LESGPU_NSTATE; q++) free(c->f[q]);
    free(c);
}

const char* lesgpu_last_error(const lesgpu_ctx* c) { (void)c; return "fake"; }

int lesgpu_upload_attribute(lesgpu_ctx* c, const int* attr) {
    memcpy(c->attr, attr, c->n * sizeof(int));
    c->have_attr = 1;
    c->uploads_attr++;
    return LESGPU_OK;
}

int lesgpu_upload_state(lesgpu_ctx* c, const double* const* f, int nf) {
    if (!c->have_attr) return LESGPU_ESTATE;
    for (int q = 0; q < nf; q++) memcpy(c->f[q], f[q], c->n * sizeof(double));
    c->numax = c->alphamax = 0.0;
    c->have_state = 1;
    return LESGPU_OK;
}

int lesgpu_download_state(lesgpu_ctx* c, double* const* f, int nf) {
    for (int q = 0; q < nf; q++) memcpy(f[q], c->f[q], c->n * sizeof(double));
    return LESGPU_OK;
}

int lesgpu_get_field(lesgpu_ctx* c, int id, double* out) {
    if (id >= 0 && id < LESGPU_NSTATE) memcpy(out, c->f[id], c->n * sizeof(double));
    else memset(out, 0, c->n * sizeof(double));
    return LESGPU_OK;
}

int lesgpu_dt_inputs(lesgpu_ctx* c, double* umax, double* numax, double* alphamax) {
    double m = 0.0;
    for (size_t q = 0; q < c->n; q++)
        if (c->attr[q] == 1 || c->attr[q] == 3) {
            double u = c->f[0][q], v = c->f[1][q], w = c->f[2][q];
            m = fmax(m, sqrt(u * u + v * v + w * w));
        }
    *umax = m > 1e-10 ? m : c->cfg.inlet_velocity;
    *numax = c->numax;
    *alphamax = c->alphamax;
    return LESGPU_OK;
}

int lesgpu_set_dt_inputs(lesgpu_ctx* c, double numax, double alphamax) {
    c->numax = numax;
    c->alphamax = alphamax;
    return LESGPU_OK;
}

int lesgpu_set_inflow(lesgpu_ctx* c, const double* vort, int nv, const double* noise) {
    c->vort = vort;
    c->nv = nv;
    double s = 0.0;
    for (size_t q = 0; q < 3 * (size_t)c->cfg.ny * c->cfg.nz; q++) s += noise[q];
    c->noise0 = s;
    return LESGPU_OK;
}

/* every cell's u and T move by amounts that depend on dt, t_loop, the vortex table, the
   noise and the attribute code; the maxima follow the step index */
int lesgpu_step(lesgpu_ctx* c, double dt, int t_loop) {
    double vs = 0.0;
    for (int q = 0; q < c->nv * 7; q++) vs += c->vort[q] * (double)(q % 7 + 1);
    for (size_t q = 0; q < c->n; q++) {
        c->f[0][q] += dt * (1e-3 * vs + 1e-2 * c->noise0 + 0.1 * c->attr[q] + 1e-3 * (t_loop % 11));
        c->f[3][q] += dt * (t_loop >= 500 ? 2.0 : 1.0);
    }
    c->numax = 1.0e-2 * (1.0 + 0.01 * (t_loop % 13));   /* large enough that the diffusive dt limit binds */
    c->alphamax = 2.0e-5 * (1.0 + 0.02 * (t_loop % 5));
    return LESGPU_OK;
}

int lesgpu_sync(lesgpu_ctx* c) { (void)c; return LESGPU_OK; }

int lesgpu_probe_lines(lesgpu_ctx* c, const int* st, int n, int kline, double* out) {
    for (int q = 0; q < n; q++)
        for (int j = 0; j < c->cfg.ny; j++) {
            size_t id = ((size_t)st[q] * c->cfg.ny + j) * c->cfg.nz + kline;
            double* o = out + ((size_t)q * c->cfg.ny + j) * 6;
            o[0] = c->f[0][id]; o[1] = c->f[1][id]; o[2] = c->f[2][id]; o[3] = c->f[4][id]; o[4] = 0.0; o[5] = 0.0;
        }
    return LESGPU_OK;
}

int lesgpu_monitor(lesgpu_ctx* c, double out[6]) {
    (void)c;
    for (int q = 0; q < 6; q++) out[q] = 0.0;
    return LESGPU_OK;
}

int lesgpu_keep_grad_g(lesgpu_ctx* c, int enable) { (void)c; (void)enable; return LESGPU_OK; }

/* time averages and the device-resident loop are not part of what this stand-in covers */
int lesgpu_avg_begin(lesgpu_ctx* c, int start) { (void)c; (void)start; return LESGPU_EINVAL; }
int lesgpu_avg_end(lesgpu_ctx* c) { (void)c; return LESGPU_OK; }
int lesgpu_avg_download(lesgpu_ctx* c, double* const* f, int* count) { (void)c; (void)f; (void)count; return LESGPU_EINVAL; }
int lesgpu_avg_upload(lesgpu_ctx* c, const double* const* f, int count) { (void)c; (void)f; (void)count; return LESGPU_EINVAL; }
int lesgpu_loop_begin(lesgpu_ctx* c, const unsigned int win[31], const double* vort, int nv, int t_loop) {
    (void)c; (void)win; (void)vort; (void)nv; (void)t_loop;
    return LESGPU_EINVAL;
}
int lesgpu_loop_config(lesgpu_ctx* c, const int* st, int n, int kline, int cap) {
    (void)c; (void)st; (void)n; (void)kline; (void)cap;
    return LESGPU_EINVAL;
}
int lesgpu_run(lesgpu_ctx* c, int nsteps) { (void)c; (void)nsteps; return LESGPU_EINVAL; }
int lesgpu_loop_history(lesgpu_ctx* c, int nsteps, double* dt, double* umax, double* probes, double* monitor) {
    (void)c; (void)nsteps; (void)dt; (void)umax; (void)probes; (void)monitor;
    return LESGPU_EINVAL;
}
int lesgpu_loop_end(lesgpu_ctx* c, unsigned int win[31], double* vort, int* t_loop) {
    (void)c; (void)win; (void)vort; (void)t_loop;
    return LESGPU_EINVAL;
}

int lesgpu_pstat_begin(lesgpu_ctx* c, const double* ye, int ny, const double* grc, int ngrc, const double* gho, int ngho,
                       const double* ue, const double* ve, int npdf) {
    (void)c; (void)ye; (void)ny; (void)grc; (void)ngrc; (void)gho; (void)ngho; (void)ue; (void)ve; (void)npdf;
    return LESGPU_EINVAL;
}
int lesgpu_pstat_accumulate(lesgpu_ctx* c, int nsteps, int n_lines) { (void)c; (void)nsteps; (void)n_lines; return LESGPU_EINVAL; }
size_t lesgpu_pstat_size(const lesgpu_ctx* c) { (void)c; return 0; }
int lesgpu_pstat_layout(const lesgpu_ctx* c, int* a, int* b, int* d, int* e, double* edges, size_t* ne) {
    (void)c; (void)a; (void)b; (void)d; (void)e; (void)edges; (void)ne;
    return LESGPU_EINVAL;
}
int lesgpu_pstat_read(lesgpu_ctx* c, double* out) { (void)c; (void)out; return LESGPU_EINVAL; }

/* for the test: the attribute map the "device" holds and how often it was uploaded */
int fake_attr(const lesgpu_ctx* c, int* out) {
    memcpy(out, c->attr, c->n * sizeof(int));
    return c->uploads_attr;
}
