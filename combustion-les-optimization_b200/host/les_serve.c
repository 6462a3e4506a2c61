/*
 * les_serve.c -- a request loop that serves many LES solves on one GPU at once.
 *
 * No counterpart in the reference, which runs one solve per process.  Requests (a config,
 * a step count, optional output files) are submitted at any time.  Each scheduling round
 * (les_serve_step):
 *   1. admits queued requests in arrival order while a slot is free and the request's
 *      device memory fits the remaining HBM budget (a request that can never fit is refused
 *      at submission);
 *   2. queues up to `quantum` device-loop steps of every active request, each on its own
 *      stream as a replayed CUDA graph, so the solves overlap on the device;
 *   3. collects every active request's step history (probe / monitor rows) and retires the
 *      requests that have finished: the final state is copied to the host when results are
 *      kept, the solver is destroyed and its memory returns to the budget at once.
 * Requests that arrive while others run join at the next round (continuous batching).  A
 * request's result does not depend on what else is running: every solver has its own
 * state, rand() stream and tiles, and the device loop's results do not depend on how its
 * steps are chunked.
 */
#define _POSIX_C_SOURCE 199309L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "les_serve.h"

typedef struct serve_req {
    long long id;
    lesgpu_config cfg;
    int nsteps, done_steps;
    int state;
    int err;
    double t_submit, t_admit, t_done;
    size_t bytes;
    les_solver* sol;
    double* result;               /* 11 fields x cells, host, when results are kept */
    char out_dir[1024];
    int out_flags;
} serve_req;

typedef struct tile_entry {
    int nx, ny, nz, precision;
    int tiles[5];
    int staged;                   /* scalar pass through the staged (TMA) kernel */
} tile_entry;

struct les_serve {
    les_serve_options opt;
    size_t in_use;
    serve_req** reqs;             /* every request ever submitted, index = id */
    long long n, cap;
    long long head;               /* first request still queued or active */
    int n_active;
    long long n_done, n_failed, n_cancelled;
    double cell_steps;
    double t_first_admit, t_last_done;
    tile_entry tiles[64];
    int n_tiles;
    char err[256];
};

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int serr(les_serve* s, int code, const char* msg) {
    if (s) snprintf(s->err, sizeof(s->err), "%s", msg);
    return code;
}

size_t les_serve_request_bytes(const lesgpu_config* cfg, int quantum) {
    if (!cfg) return 0;
    const size_t planes = (size_t)cfg->ny * cfg->nz;
    size_t b = lesgpu_bytes_for_grid(cfg->nx, cfg->ny, cfg->nz, cfg->precision);
    /* device-loop session: rand() jump table (<= 6 draws per vortex + 3 per inlet cell,
     * 31 words each) and the step history (7 stations of NY rows x 6, dt, |u|max, monitor) */
    const size_t jrows = 6 * (size_t)(cfg->num_vortices > 0 ? cfg->num_vortices : 0) + 3 * planes + 31;
    b += jrows * 31 * sizeof(unsigned int);
    b += (size_t)(quantum > 0 ? quantum : 1) * (7 * (size_t)cfg->ny * 6 + 8) * sizeof(double);
    b += (size_t)(cfg->num_vortices > 0 ? cfg->num_vortices : 1) * 7 * sizeof(double) + 4096;
    return b;
}

void les_serve_default_options(les_serve_options* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->budget_bytes = (size_t)150 * 1000 * 1000 * 1000;
    o->max_slots = 64;
    o->quantum_steps = 16;
    o->keep_results = 1;
    o->autotune = 0;
    o->backfill = 0;
    o->device = 0;
}

int les_serve_create(const les_serve_options* opt, les_serve** out) {
    if (!opt || !out || opt->max_slots < 1 || opt->quantum_steps < 1 || opt->budget_bytes == 0) return LESGPU_EINVAL;
    if (!opt->chem_path[0] || !opt->tran_path[0]) return LESGPU_EINVAL;
    *out = NULL;
    les_serve* s = (les_serve*)calloc(1, sizeof(les_serve));
    if (!s) return LESGPU_ENOMEM;
    s->opt = *opt;
    s->t_first_admit = -1.0;
    *out = s;
    return LESGPU_OK;
}

static serve_req* find(les_serve* s, long long id) {
    if (!s || id < 0 || id >= s->n) return NULL;
    return s->reqs[id];
}

int les_serve_submit(les_serve* s, const lesgpu_config* cfg, int nsteps, const char* out_dir, int out_flags,
                     long long* id) {
    if (!s || !cfg || nsteps < 1 || !id) return LESGPU_EINVAL;
    *id = -1;
    if (cfg->device != s->opt.device) return serr(s, LESGPU_EINVAL, "request is for another device");
    if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 4) return serr(s, LESGPU_EINVAL, "grid too small");
    if (out_dir && strlen(out_dir) >= sizeof(((serve_req*)0)->out_dir)) return serr(s, LESGPU_EINVAL, "path too long");
    const size_t need = les_serve_request_bytes(cfg, s->opt.quantum_steps);
    if (need > s->opt.budget_bytes) return serr(s, LESGPU_ENOMEM, "request needs more device memory than the budget");
    if (s->n == s->cap) {
        long long nc = s->cap ? 2 * s->cap : 256;
        serve_req** r = (serve_req**)realloc(s->reqs, (size_t)nc * sizeof(serve_req*));
        if (!r) return serr(s, LESGPU_ENOMEM, "request table");
        s->reqs = r;
        s->cap = nc;
    }
    serve_req* q = (serve_req*)calloc(1, sizeof(serve_req));
    if (!q) return serr(s, LESGPU_ENOMEM, "request");
    q->id = s->n;
    q->cfg = *cfg;
    q->nsteps = nsteps;
    q->state = LES_REQ_QUEUED;
    q->t_submit = now_s();
    q->bytes = need;
    if (out_dir) snprintf(q->out_dir, sizeof(q->out_dir), "%s", out_dir);
    q->out_flags = out_dir ? out_flags : 0;
    s->reqs[s->n++] = q;
    *id = q->id;
    return LESGPU_OK;
}

static void retire(les_serve* s, serve_req* q, int state, int err) {
    if (q->sol) {
        les_solver_destroy(q->sol);
        q->sol = NULL;
    }
    if (q->state == LES_REQ_ACTIVE) {
        s->in_use -= q->bytes;
        s->n_active--;
    }
    q->state = state;
    q->err = err;
    q->t_done = now_s();
    if (state == LES_REQ_DONE) {
        s->n_done++;
        s->t_last_done = q->t_done;
    } else if (state == LES_REQ_CANCELLED) {
        s->n_cancelled++;
    } else {
        s->n_failed++;
    }
}

int les_serve_cancel(les_serve* s, long long id) {
    serve_req* q = find(s, id);
    if (!q) return LESGPU_EINVAL;
    if (q->state != LES_REQ_QUEUED && q->state != LES_REQ_ACTIVE) return LESGPU_ESTATE;
    /* between rounds no step of an active request is in flight (collect waited for it) */
    retire(s, q, LES_REQ_CANCELLED, 0);
    return LESGPU_OK;
}

static const tile_entry* cached_tiles(les_serve* s, const lesgpu_config* c) {
    for (int q = 0; q < s->n_tiles; q++) {
        const tile_entry* t = &s->tiles[q];
        if (t->nx == c->nx && t->ny == c->ny && t->nz == c->nz && t->precision == c->precision) return t;
    }
    return NULL;
}

static int admit(les_serve* s, serve_req* q) {
    int rc = les_solver_create(&q->cfg, s->opt.chem_path, s->opt.tran_path, 0, &q->sol);
    if (rc) return rc;
    lesgpu_ctx* ctx = les_solver_ctx(q->sol);
    if (s->opt.autotune) {
        /* one autotuning per grid shape and precision; later requests of that shape get the
           same tiles and scalar-pass form, so their results do not depend on arrival order */
        const tile_entry* t = cached_tiles(s, &q->cfg);
        if (t) {
            rc = lesgpu_set_tiles(ctx, t->tiles);
            if (rc == LESGPU_OK) rc = lesgpu_set_scalar_staging(ctx, t->staged);
        } else {
            int tl[5];
            rc = lesgpu_autotune(ctx, 3, tl, NULL);
            if (rc == LESGPU_OK && s->n_tiles < 64) {
                tile_entry* e = &s->tiles[s->n_tiles++];
                e->nx = q->cfg.nx; e->ny = q->cfg.ny; e->nz = q->cfg.nz; e->precision = q->cfg.precision;
                memcpy(e->tiles, tl, sizeof(tl));
                e->staged = lesgpu_get_scalar_staging(ctx);
            }
        }
    }
    if (rc == LESGPU_OK && q->out_dir[0]) rc = les_solver_set_outputs(q->sol, q->out_dir, q->out_flags);
    if (rc == LESGPU_OK) rc = les_solver_loop_begin(q->sol, s->opt.quantum_steps);
    if (rc) {
        les_solver_destroy(q->sol);
        q->sol = NULL;
        return rc;
    }
    q->state = LES_REQ_ACTIVE;
    q->t_admit = now_s();
    s->in_use += q->bytes;
    s->n_active++;
    if (s->t_first_admit < 0) s->t_first_admit = q->t_admit;
    return LESGPU_OK;
}

static int finish(les_serve* s, serve_req* q) {
    int rc = les_solver_loop_end(q->sol);
    if (rc == LESGPU_OK && s->opt.keep_results) {
        const size_t n = (size_t)q->cfg.nx * q->cfg.ny * q->cfg.nz;
        q->result = (double*)malloc(LESGPU_NSTATE * n * sizeof(double));
        if (!q->result) return LESGPU_ENOMEM;
        double* f[LESGPU_NSTATE];
        for (int k = 0; k < LESGPU_NSTATE; k++) f[k] = q->result + (size_t)k * n;
        rc = lesgpu_download_state(les_solver_ctx(q->sol), f, LESGPU_NSTATE);
    }
    return rc;
}

static void admit_queued(les_serve* s) {
    for (long long i = s->head; i < s->n && s->n_active < s->opt.max_slots; i++) {
        serve_req* q = s->reqs[i];
        if (q->state != LES_REQ_QUEUED) continue;
        if (s->in_use + q->bytes > s->opt.budget_bytes) {
            if (s->opt.backfill) continue;
            break;
        }
        int rc = admit(s, q);
        if (rc == LESGPU_ENOMEM && s->n_active > 0) break;   /* the device is fuller than budgeted: wait */
        if (rc) retire(s, q, LES_REQ_FAILED, rc);
    }
}

int les_serve_step(les_serve* s) {
    if (!s) return LESGPU_EINVAL;
    while (s->head < s->n && s->reqs[s->head]->state != LES_REQ_QUEUED && s->reqs[s->head]->state != LES_REQ_ACTIVE)
        s->head++;
    /* with nothing running there is nothing to overlap: admit first */
    const int admit_early = (s->n_active == 0);
    if (admit_early) admit_queued(s);
    /* 1. queue one quantum of every active request (asynchronous, one stream each) */
    int* qn = NULL;
    serve_req** act = NULL;
    int na = 0;
    const int cap_a = s->n_active;
    if (cap_a > 0) {
        qn = (int*)malloc((size_t)cap_a * sizeof(int));
        act = (serve_req**)malloc((size_t)cap_a * sizeof(serve_req*));
        if (!qn || !act) {
            free(qn);
            free(act);
            return serr(s, LESGPU_ENOMEM, "round tables");
        }
        for (long long i = s->head; i < s->n && na < cap_a; i++) {
            serve_req* q = s->reqs[i];
            if (q->state != LES_REQ_ACTIVE) continue;
            int left = q->nsteps - q->done_steps;
            int n = les_solver_next_chunk(q->sol, left);
            int rc = (n > 0) ? lesgpu_run(les_solver_ctx(q->sol), n) : LESGPU_ESTATE;
            if (rc) {
                retire(s, q, LES_REQ_FAILED, rc);
                continue;
            }
            act[na] = q;
            qn[na] = n;
            na++;
        }
    }
    /* 2. admission, in arrival order, while the quanta just queued run on the device (the
     *    host-side set-up of a new request overlaps them); new requests join next round */
    if (!admit_early) admit_queued(s);
    /* 3. collect histories and retire finished requests */
    for (int a = 0; a < na; a++) {
        serve_req* q = act[a];
        int rc = les_solver_loop_collect(q->sol, qn[a]);
        if (rc) {
            retire(s, q, LES_REQ_FAILED, rc);
            continue;
        }
        q->done_steps += qn[a];
        s->cell_steps += (double)qn[a] * (double)q->cfg.nx * q->cfg.ny * q->cfg.nz;
        if (q->done_steps >= q->nsteps) {
            rc = finish(s, q);
            retire(s, q, rc ? LES_REQ_FAILED : LES_REQ_DONE, rc);
        }
    }
    free(qn);
    free(act);
    long long pending = 0;
    for (long long i = s->head; i < s->n; i++)
        if (s->reqs[i]->state == LES_REQ_QUEUED || s->reqs[i]->state == LES_REQ_ACTIVE) pending++;
    return pending > 0x7fffffff ? 0x7fffffff : (int)pending;
}

int les_serve_info(les_serve* s, long long id, les_serve_request_info* info) {
    serve_req* q = find(s, id);
    if (!q || !info) return LESGPU_EINVAL;
    info->state = q->state;
    info->error = q->err;
    info->steps_done = q->done_steps;
    info->nsteps = q->nsteps;
    info->bytes = q->bytes;
    info->device_bytes = q->sol ? lesgpu_device_bytes(les_solver_ctx(q->sol)) : 0;
    info->t_submit = q->t_submit;
    info->t_admit = q->t_admit;
    info->t_done = q->t_done;
    info->latency_s = (q->state == LES_REQ_DONE) ? q->t_done - q->t_submit : -1.0;
    return LESGPU_OK;
}

int les_serve_result(les_serve* s, long long id, double* const* fields, int nfields) {
    serve_req* q = find(s, id);
    if (!q || !fields || nfields < 1 || nfields > LESGPU_NSTATE) return LESGPU_EINVAL;
    if (q->state != LES_REQ_DONE) return serr(s, LESGPU_ESTATE, "request has not finished");
    if (!q->result) return serr(s, LESGPU_ESTATE, "result not kept (or released)");
    const size_t n = (size_t)q->cfg.nx * q->cfg.ny * q->cfg.nz;
    for (int k = 0; k < nfields; k++)
        if (fields[k]) memcpy(fields[k], q->result + (size_t)k * n, n * sizeof(double));
    return LESGPU_OK;
}

int les_serve_release(les_serve* s, long long id) {
    serve_req* q = find(s, id);
    if (!q) return LESGPU_EINVAL;
    free(q->result);
    q->result = NULL;
    return LESGPU_OK;
}

static int cmp_double(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* q-quantile with linear interpolation between order statistics (numpy's default). */
static double quantile(const double* v, long long n, double p) {
    if (n <= 0) return -1.0;
    double h = p * (double)(n - 1);
    long long lo = (long long)h;
    if (lo >= n - 1) return v[n - 1];
    return v[lo] + (h - (double)lo) * (v[lo + 1] - v[lo]);
}

int les_serve_stats(les_serve* s, les_serve_summary* st) {
    if (!s || !st) return LESGPU_EINVAL;
    memset(st, 0, sizeof(*st));
    st->submitted = s->n;
    st->done = s->n_done;
    st->failed = s->n_failed;
    st->cancelled = s->n_cancelled;
    st->active = s->n_active;
    st->bytes_in_use = s->in_use;
    st->cell_steps = s->cell_steps;
    for (long long i = 0; i < s->n; i++)
        if (s->reqs[i]->state == LES_REQ_QUEUED) st->queued++;
    double* lat = (double*)malloc((size_t)(s->n_done > 0 ? s->n_done : 1) * sizeof(double));
    if (!lat) return LESGPU_ENOMEM;
    long long m = 0;
    for (long long i = 0; i < s->n; i++)
        if (s->reqs[i]->state == LES_REQ_DONE) lat[m++] = s->reqs[i]->t_done - s->reqs[i]->t_submit;
    qsort(lat, (size_t)m, sizeof(double), cmp_double);
    st->latency_p50_s = quantile(lat, m, 0.50);
    st->latency_p99_s = quantile(lat, m, 0.99);
    st->latency_max_s = m ? lat[m - 1] : -1.0;
    free(lat);
    st->busy_s = (s->t_first_admit >= 0 && s->t_last_done > s->t_first_admit) ? s->t_last_done - s->t_first_admit : 0.0;
    st->cell_steps_per_s = st->busy_s > 0 ? s->cell_steps / st->busy_s : 0.0;
    return LESGPU_OK;
}

const char* les_serve_last_error(const les_serve* s) { return s ? s->err : "null server"; }

void les_serve_destroy(les_serve* s) {
    if (!s) return;
    for (long long i = 0; i < s->n; i++) {
        serve_req* q = s->reqs[i];
        if (q->sol) les_solver_destroy(q->sol);
        free(q->result);
        free(q);
    }
    free(s->reqs);
    free(s);
}
