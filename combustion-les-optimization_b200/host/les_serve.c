/*
 * les_serve.c -- a request loop that serves many LES solves on one GPU at once.
 *
 * No counterpart in the reference, which runs one solve per process.  Requests (a config,
 * a step count, optional output files) are submitted at any time.  Each scheduling round
 * (les_serve_step):
 *   1. starts the requests whose set-up has finished (their first quantum is queued) and
 *      retires those whose tear-down has finished;
 *   2. admits queued requests in arrival order while a slot is free and the request's
 *      device memory fits the remaining HBM budget (a request that can never fit is refused
 *      at submission); their set-up (solver, initial state, uploads, tiles, device-loop
 *      session) runs on the server's worker threads while the device steps the others;
 *   3. collects every running request's quantum in turn (its probe / monitor rows) and
 *      queues that request's next quantum at once, each request on its own stream as a
 *      replayed CUDA graph, so the device always holds the other requests' work while the
 *      host handles one; a finished request goes to a worker, which closes its session,
 *      copies the final state to the host when results are kept and frees its device
 *      memory, after which its budget returns.
 * Requests that arrive while others run join as soon as they are set up (continuous
 * batching).  A request's result does not depend on what else is running: every solver has
 * its own state, rand() stream and tiles (one autotuning per grid shape, shared), and the
 * device loop's results do not depend on how its steps are chunked.
 */
#define _POSIX_C_SOURCE 200809L
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "les_serve.h"

/* Where a request is in its life; phases PREP and FIN belong to a set-up worker. */
enum {
    PH_NONE = 0,      /* queued, or retired: holds no budget */
    PH_PREP = 1,      /* budget reserved, handed to a worker for set-up */
    PH_READY = 2,     /* set-up done (job_rc) */
    PH_RUN = 3,       /* stepping on the device */
    PH_FIN = 4,       /* handed to a worker for loop end, result copy and release */
    PH_FINISHED = 5   /* that done (job_rc, t_done) */
};

typedef struct serve_req {
    long long id;
    lesgpu_config cfg;
    int nsteps, done_steps;
    int state;                    /* LES_REQ_* as the caller sees it */
    int err;
    double t_submit, t_admit, t_done;
    size_t bytes;
    les_solver* sol;
    double* result;               /* 11 fields x cells, host, when results are kept */
    char out_dir[1024];
    int out_flags;
    int phase;                    /* PH_*; changed under the server mutex */
    int job_rc;
    int inflight;                 /* steps queued on the device and not yet collected */
    size_t dev_bytes;             /* device bytes of the solver when it started */
    long long retry_after;        /* set-up ran out of device memory: wait until more than this
                                     many requests have ended */
    struct serve_req* next_job;
} serve_req;

typedef struct tile_entry {
    int nx, ny, nz, precision;
    int tiles[5];
    int staged;                   /* scalar pass through the staged (TMA) kernel */
    int ready;                    /* 0 being tuned, 1 filled, -1 tuning failed */
} tile_entry;

struct les_serve {
    les_serve_options opt;
    size_t in_use;                /* budget held by requests in phases PREP..FINISHED */
    serve_req** reqs;             /* every request ever submitted, index = id */
    long long n, cap;
    long long head;               /* first request still queued or active */
    int n_slots;                  /* requests holding budget */
    int n_active;                 /* requests in state LES_REQ_ACTIVE */
    long long n_done, n_failed, n_cancelled;
    double cell_steps;
    double t_first_admit, t_last_done;
    tile_entry tiles[64];
    int n_tiles;
    char err[256];
    /* set-up / tear-down workers and their job queue */
    pthread_mutex_t mu;
    pthread_cond_t cv_job, cv_done;
    pthread_t* th;
    int n_th;
    int stop;
    serve_req *jq_head, *jq_tail;
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
    /* 16 requests on the device at once keep it busy; more only share L2 and SM time among
       more solves (measured on the mixed 100-request stream: 16 slots 7.8e8 cell-steps/s,
       p50 12 s; 64 slots 6.8e8, p50 21 s) */
    o->max_slots = 16;
    o->quantum_steps = 16;
    o->keep_results = 1;
    o->autotune = 0;
    o->backfill = 0;
    o->policy = LES_SERVE_FIFO;
    o->device = 0;
    o->prep_threads = 4;
}

/* ------------------------------------------------------------------ worker jobs */

static tile_entry* find_tiles(les_serve* s, const lesgpu_config* c) {
    for (int q = 0; q < s->n_tiles; q++) {
        tile_entry* t = &s->tiles[q];
        if (t->nx == c->nx && t->ny == c->ny && t->nz == c->nz && t->precision == c->precision) return t;
    }
    return NULL;
}

/* One autotuning per grid shape and precision; later requests of that shape (also those set
   up meanwhile by other workers, which wait for it) get the same tiles and scalar-pass form,
   so a result does not depend on arrival order.  An entry is 0 while its autotune runs, 1
   once published, -1 after a failed autotune: the next request of that shape (a woken waiter
   or a later arrival) claims it and tunes again, so a failure is never cached and every
   request of the shape still ends up with the one published result. */
static int tiles_for(les_serve* s, serve_req* q, lesgpu_ctx* ctx) {
    pthread_mutex_lock(&s->mu);
    tile_entry* t = find_tiles(s, &q->cfg);
    while (t && t->ready == 0) {
        pthread_cond_wait(&s->cv_done, &s->mu);
        t = find_tiles(s, &q->cfg);
    }
    if (t && t->ready == 1) {
        tile_entry c = *t;
        pthread_mutex_unlock(&s->mu);
        int rc = lesgpu_set_tiles(ctx, c.tiles);
        if (rc == LESGPU_OK) rc = lesgpu_set_scalar_staging(ctx, c.staged);
        return rc;
    }
    tile_entry* e = NULL;
    if (t) {
        e = t;                     /* the last autotune of this shape failed: retry here */
        e->ready = 0;
    } else if (s->n_tiles < 64) {
        e = &s->tiles[s->n_tiles++];
        e->nx = q->cfg.nx; e->ny = q->cfg.ny; e->nz = q->cfg.nz; e->precision = q->cfg.precision;
        e->ready = 0;
    }
    pthread_mutex_unlock(&s->mu);
    int tl[5];
    int rc = lesgpu_autotune(ctx, 3, tl, NULL);
    if (e) {
        pthread_mutex_lock(&s->mu);
        if (rc == LESGPU_OK) {
            memcpy(e->tiles, tl, sizeof(tl));
            e->staged = lesgpu_get_scalar_staging(ctx);
            e->ready = 1;
        } else {
            e->ready = -1;
        }
        pthread_cond_broadcast(&s->cv_done);
        pthread_mutex_unlock(&s->mu);
    }
    return rc;
}

/* Set-up of an admitted request: solver (initial state, device arena), tiles, output
   files, device-loop session. */
static int job_prepare(les_serve* s, serve_req* q) {
    les_solver* sol = NULL;
    int rc = les_solver_create(&q->cfg, s->opt.chem_path, s->opt.tran_path, 0, &sol);
    if (rc) return rc;
    if (s->opt.autotune) rc = tiles_for(s, q, les_solver_ctx(sol));
    if (rc == LESGPU_OK && q->out_dir[0]) rc = les_solver_set_outputs(sol, q->out_dir, q->out_flags);
    if (rc == LESGPU_OK) rc = les_solver_loop_begin(sol, s->opt.quantum_steps);
    if (rc) {
        les_solver_destroy(sol);
        return rc;
    }
    q->sol = sol;
    return LESGPU_OK;
}

/* End of a finished request: close the loop session (files flushed, les_solver_flush), copy
   the final state to the host when results are kept, release the solver and its device memory. */
static int job_finish(les_serve* s, serve_req* q) {
    int rc = les_solver_loop_end(q->sol);
    /* the end-of-run writes (final VTK, point rows, profile_stats.bin) of the enabled outputs */
    if (rc == LESGPU_OK && q->out_dir[0]) rc = les_solver_flush(q->sol);
    if (rc == LESGPU_OK && s->opt.keep_results) {
        const size_t n = (size_t)q->cfg.nx * q->cfg.ny * q->cfg.nz;
        q->result = (double*)malloc(LESGPU_NSTATE * n * sizeof(double));
        if (!q->result) {
            rc = LESGPU_ENOMEM;
        } else {
            double* f[LESGPU_NSTATE];
            for (int k = 0; k < LESGPU_NSTATE; k++) f[k] = q->result + (size_t)k * n;
            rc = lesgpu_download_state(les_solver_ctx(q->sol), f, LESGPU_NSTATE);
        }
    }
    les_solver_destroy(q->sol);
    q->sol = NULL;
    return rc;
}

static void run_job(les_serve* s, serve_req* q, int phase) {
    int rc = (phase == PH_PREP) ? job_prepare(s, q) : job_finish(s, q);
    pthread_mutex_lock(&s->mu);
    q->job_rc = rc;
    if (phase == PH_FIN) q->t_done = now_s();
    q->phase = (phase == PH_PREP) ? PH_READY : PH_FINISHED;
    pthread_cond_broadcast(&s->cv_done);
    pthread_mutex_unlock(&s->mu);
}

static void* worker_main(void* arg) {
    les_serve* s = (les_serve*)arg;
    /* CUDA's current device is per host thread */
    lesgpu_bind_device(s->opt.device);
    pthread_mutex_lock(&s->mu);
    for (;;) {
        while (!s->stop && !s->jq_head) pthread_cond_wait(&s->cv_job, &s->mu);
        if (!s->jq_head) break;                    /* stopping with the queue drained */
        serve_req* q = s->jq_head;
        s->jq_head = q->next_job;
        if (!s->jq_head) s->jq_tail = NULL;
        q->next_job = NULL;
        const int phase = q->phase;
        pthread_mutex_unlock(&s->mu);
        run_job(s, q, phase);
        pthread_mutex_lock(&s->mu);
    }
    pthread_mutex_unlock(&s->mu);
    return NULL;
}

/* Move q into PREP or FIN and have it done: by a worker, or here when the server has none. */
static void hand_out(les_serve* s, serve_req* q, int phase) {
    pthread_mutex_lock(&s->mu);
    q->phase = phase;
    if (s->n_th > 0) {
        q->next_job = NULL;
        if (s->jq_tail) s->jq_tail->next_job = q;
        else s->jq_head = q;
        s->jq_tail = q;
        pthread_cond_signal(&s->cv_job);
        pthread_mutex_unlock(&s->mu);
        return;
    }
    pthread_mutex_unlock(&s->mu);
    run_job(s, q, phase);
}

/* ------------------------------------------------------------------ server */

int les_serve_create(const les_serve_options* opt, les_serve** out) {
    if (!opt || !out || opt->max_slots < 1 || opt->quantum_steps < 1 || opt->budget_bytes == 0) return LESGPU_EINVAL;
    if (!opt->chem_path[0] || !opt->tran_path[0]) return LESGPU_EINVAL;
    if (opt->prep_threads < 0 || opt->prep_threads > 64) return LESGPU_EINVAL;
    if (opt->policy != LES_SERVE_FIFO && opt->policy != LES_SERVE_SHORTEST) return LESGPU_EINVAL;
    *out = NULL;
    les_serve* s = (les_serve*)calloc(1, sizeof(les_serve));
    if (!s) return LESGPU_ENOMEM;
    s->opt = *opt;
    s->t_first_admit = -1.0;
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->cv_job, NULL);
    pthread_cond_init(&s->cv_done, NULL);
    if (opt->prep_threads > 0) {
        s->th = (pthread_t*)calloc((size_t)opt->prep_threads, sizeof(pthread_t));
        if (!s->th) {
            les_serve_destroy(s);
            return LESGPU_ENOMEM;
        }
        for (int t = 0; t < opt->prep_threads; t++) {
            if (pthread_create(&s->th[t], NULL, worker_main, s) != 0) break;
            s->n_th++;
        }
        if (s->n_th == 0) {
            les_serve_destroy(s);
            return LESGPU_ENOMEM;
        }
    }
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
    q->phase = PH_NONE;
    q->retry_after = -1;
    q->t_submit = now_s();
    q->bytes = need;
    if (out_dir) snprintf(q->out_dir, sizeof(q->out_dir), "%s", out_dir);
    q->out_flags = out_dir ? out_flags : 0;
    s->reqs[s->n++] = q;
    *id = q->id;
    return LESGPU_OK;
}

/* Final bookkeeping of a request no worker holds: its solver (if any) is destroyed and its
   budget returned. */
static void retire(les_serve* s, serve_req* q, int state, int err) {
    if (q->sol) {
        les_solver_destroy(q->sol);
        q->sol = NULL;
    }
    pthread_mutex_lock(&s->mu);
    if (q->phase != PH_NONE) {
        s->in_use -= q->bytes;
        s->n_slots--;
    }
    q->phase = PH_NONE;
    pthread_mutex_unlock(&s->mu);
    if (q->state == LES_REQ_ACTIVE) s->n_active--;
    q->state = state;
    q->err = err;
    if (state != LES_REQ_DONE) q->t_done = now_s();
    if (state == LES_REQ_DONE) {
        s->n_done++;
        if (q->t_done > s->t_last_done) s->t_last_done = q->t_done;
    } else if (state == LES_REQ_CANCELLED) {
        s->n_cancelled++;
    } else {
        s->n_failed++;
    }
}

static int phase_of(les_serve* s, serve_req* q) {
    pthread_mutex_lock(&s->mu);
    int p = q->phase;
    pthread_mutex_unlock(&s->mu);
    return p;
}

/* Wait until no worker holds q. */
static void wait_idle(les_serve* s, serve_req* q) {
    pthread_mutex_lock(&s->mu);
    while (q->phase == PH_PREP || q->phase == PH_FIN) pthread_cond_wait(&s->cv_done, &s->mu);
    pthread_mutex_unlock(&s->mu);
}

int les_serve_cancel(les_serve* s, long long id) {
    serve_req* q = find(s, id);
    if (!q) return LESGPU_EINVAL;
    if (q->state != LES_REQ_QUEUED && q->state != LES_REQ_ACTIVE) return LESGPU_ESTATE;
    wait_idle(s, q);
    const int ph = phase_of(s, q);
    if (ph == PH_FINISHED) return serr(s, LESGPU_ESTATE, "request has already finished");
    if (ph == PH_RUN && q->inflight > 0) {
        /* let the steps already queued end before the solver is released */
        (void)les_solver_loop_collect(q->sol, q->inflight);
        q->inflight = 0;
    }
    retire(s, q, LES_REQ_CANCELLED, 0);
    return LESGPU_OK;
}

/* Queue the next quantum of a running request. */
static void launch(les_serve* s, serve_req* q) {
    int n = les_solver_next_chunk(q->sol, q->nsteps - q->done_steps);
    int rc = (n > 0) ? lesgpu_run(les_solver_ctx(q->sol), n) : LESGPU_ESTATE;
    if (rc) {
        retire(s, q, LES_REQ_FAILED, rc);
        return;
    }
    q->inflight = n;
}

/* Requests whose worker job ended: set-up done -> running (first quantum queued at once),
   tear-down done -> done. */
static void harvest(les_serve* s) {
    for (long long i = s->head; i < s->n; i++) {
        serve_req* q = s->reqs[i];
        if (q->state != LES_REQ_QUEUED && q->state != LES_REQ_ACTIVE) continue;
        const int ph = phase_of(s, q);
        if (ph == PH_READY) {
            if (q->job_rc == LESGPU_ENOMEM && s->n_slots > 1) {
                /* the device is fuller than budgeted while other requests hold memory (set-ups
                   in progress, running or finishing solves): queue it again until another
                   request ends */
                pthread_mutex_lock(&s->mu);
                s->in_use -= q->bytes;
                s->n_slots--;
                q->phase = PH_NONE;
                pthread_mutex_unlock(&s->mu);
                q->retry_after = s->n_done + s->n_failed + s->n_cancelled;
                continue;
            }
            if (q->job_rc) {
                retire(s, q, LES_REQ_FAILED, q->job_rc);
                continue;
            }
            pthread_mutex_lock(&s->mu);
            q->phase = PH_RUN;
            pthread_mutex_unlock(&s->mu);
            q->state = LES_REQ_ACTIVE;
            q->dev_bytes = lesgpu_device_bytes(les_solver_ctx(q->sol));
            s->n_active++;
            launch(s, q);
        } else if (ph == PH_FINISHED) {
            retire(s, q, q->job_rc ? LES_REQ_FAILED : LES_REQ_DONE, q->job_rc);
        }
    }
}

/* A queued request that may be admitted now: not yet handed out, and not waiting for other
   requests to end after its set-up found the device full. */
static int admissible(const les_serve* s, const serve_req* q) {
    if (q->state != LES_REQ_QUEUED || phase_of((les_serve*)s, (serve_req*)q) != PH_NONE) return 0;
    if (q->retry_after >= 0 && s->n_done + s->n_failed + s->n_cancelled <= q->retry_after && s->n_slots > 0) return 0;
    return 1;
}

static void admit_one(les_serve* s, serve_req* q) {
    pthread_mutex_lock(&s->mu);
    s->in_use += q->bytes;
    s->n_slots++;
    pthread_mutex_unlock(&s->mu);
    q->t_admit = now_s();
    if (s->t_first_admit < 0) s->t_first_admit = q->t_admit;
    hand_out(s, q, PH_PREP);
}

/* LES_SERVE_SHORTEST: the admissible request with the least work (cells x steps) first, ties
   in arrival order; without backfill the round stops at the first one whose memory does not
   fit, with backfill the shortest that fits is taken. */
static int admit_shortest(les_serve* s) {
    int k = 0;
    while (s->n_slots < s->opt.max_slots) {
        serve_req* best = NULL;
        double best_w = 0.0;
        for (long long i = s->head; i < s->n; i++) {
            serve_req* q = s->reqs[i];
            if (!admissible(s, q)) continue;
            if (s->opt.backfill && s->in_use + q->bytes > s->opt.budget_bytes) continue;
            const double w = (double)q->cfg.nx * q->cfg.ny * q->cfg.nz * (double)q->nsteps;
            if (!best || w < best_w) { best = q; best_w = w; }
        }
        if (!best || s->in_use + best->bytes > s->opt.budget_bytes) break;
        admit_one(s, best);
        k++;
    }
    return k;
}

/* Reserve budget and a slot for queued requests in arrival order (or least work first) and
   hand them to the set-up workers.  Returns how many were handed out. */
static int admit_queued(les_serve* s) {
    if (s->opt.policy == LES_SERVE_SHORTEST) return admit_shortest(s);
    int k = 0;
    for (long long i = s->head; i < s->n && s->n_slots < s->opt.max_slots; i++) {
        serve_req* q = s->reqs[i];
        if (q->state != LES_REQ_QUEUED || phase_of(s, q) != PH_NONE) continue;
        if (q->retry_after >= 0 && s->n_done + s->n_failed + s->n_cancelled <= q->retry_after && s->n_slots > 0) {
            if (s->opt.backfill) continue;
            break;
        }
        if (s->in_use + q->bytes > s->opt.budget_bytes) {
            if (s->opt.backfill) continue;
            break;
        }
        admit_one(s, q);
        k++;
    }
    return k;
}

/* Wait for the next worker job to end, or until no job is pending. */
static void wait_any_job(les_serve* s) {
    pthread_mutex_lock(&s->mu);
    for (;;) {
        int busy = 0, ready = 0;
        for (long long i = s->head; i < s->n; i++) {
            const int p = s->reqs[i]->phase;
            if (p == PH_PREP || p == PH_FIN) busy = 1;
            if (p == PH_READY || p == PH_FINISHED) ready = 1;
        }
        if (ready || !busy) break;
        pthread_cond_wait(&s->cv_done, &s->mu);
    }
    pthread_mutex_unlock(&s->mu);
}

static int count_running(les_serve* s) {
    int r = 0;
    for (long long i = s->head; i < s->n; i++) {
        serve_req* q = s->reqs[i];
        if (q->state == LES_REQ_ACTIVE && phase_of(s, q) == PH_RUN) r++;
    }
    return r;
}

int les_serve_step(les_serve* s) {
    if (!s) return LESGPU_EINVAL;
    /* the workers create the contexts; this thread drives them on the server's device */
    if (lesgpu_bind_device(s->opt.device) != LESGPU_OK) return serr(s, LESGPU_ECUDA, "cannot select the device");
    while (s->head < s->n && s->reqs[s->head]->state != LES_REQ_QUEUED && s->reqs[s->head]->state != LES_REQ_ACTIVE)
        s->head++;
    /* 1. results of set-up / tear-down jobs; newly running requests get their first quantum */
    harvest(s);
    /* 2. admission, in arrival order; set-up runs on the workers while the device steps */
    admit_queued(s);
    if (count_running(s) == 0) {
        /* nothing on the device to overlap with: wait for every set-up in progress */
        pthread_mutex_lock(&s->mu);
        for (;;) {
            int busy = 0;
            for (long long i = s->head; i < s->n; i++)
                if (s->reqs[i]->phase == PH_PREP) busy = 1;
            if (!busy) break;
            pthread_cond_wait(&s->cv_done, &s->mu);
        }
        pthread_mutex_unlock(&s->mu);
        harvest(s);
    }
    /* 3. collect every running request's quantum in turn; the next quantum of a request is
     *    queued as soon as its last one is collected, so the device keeps the other
     *    requests' work while the host handles one */
    for (long long i = s->head; i < s->n; i++) {
        serve_req* q = s->reqs[i];
        if (q->state != LES_REQ_ACTIVE || phase_of(s, q) != PH_RUN) continue;
        if (q->inflight == 0) {
            launch(s, q);
            if (q->state != LES_REQ_ACTIVE) continue;
        }
        const int n = q->inflight;
        int rc = les_solver_loop_collect(q->sol, n);
        q->inflight = 0;
        if (rc) {
            retire(s, q, LES_REQ_FAILED, rc);
            continue;
        }
        q->done_steps += n;
        s->cell_steps += (double)n * (double)q->cfg.nx * q->cfg.ny * q->cfg.nz;
        if (q->done_steps >= q->nsteps) hand_out(s, q, PH_FIN);
        else launch(s, q);
    }
    /* 4. with nothing left on the device, wait for a worker instead of returning at once */
    if (count_running(s) == 0) {
        wait_any_job(s);
        harvest(s);
    }
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
    info->device_bytes = (q->state == LES_REQ_ACTIVE) ? q->dev_bytes : 0;
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
    pthread_mutex_lock(&s->mu);
    st->bytes_in_use = s->in_use;
    pthread_mutex_unlock(&s->mu);
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
    /* the workers end the jobs they hold or have queued, then exit */
    pthread_mutex_lock(&s->mu);
    s->stop = 1;
    pthread_cond_broadcast(&s->cv_job);
    pthread_mutex_unlock(&s->mu);
    for (int t = 0; t < s->n_th; t++) pthread_join(s->th[t], NULL);
    free(s->th);
    for (long long i = 0; i < s->n; i++) {
        serve_req* q = s->reqs[i];
        if (q->sol) les_solver_destroy(q->sol);
        free(q->result);
        free(q);
    }
    free(s->reqs);
    pthread_cond_destroy(&s->cv_job);
    pthread_cond_destroy(&s->cv_done);
    pthread_mutex_destroy(&s->mu);
    free(s);
}
