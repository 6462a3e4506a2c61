/*
 * Stand-in for the solver and device library behind host/les_serve.c, so that the serving
 * scheduler (admission by budget, worker threads, quanta, retry when the device is full,
 * cancellation) can be tested on a machine without a GPU.  Every call keeps host-side
 * bookkeeping only: "device memory" is a counter with an optional limit, set-up and stepping
 * take a little wall time, and the downloaded state encodes the request's seed, the steps it
 * ran and its tiles, so a test can check each result.  Test infrastructure, not product code.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "les_solver.h"

struct les_solver {
    lesgpu_config cfg;
    int chunk, loop_on, steps_done, inflight, staged, tiles[5];
    size_t bytes;
};

static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
static size_t g_used, g_peak, g_limit = (size_t)-1;
static long long g_creates, g_enomem, g_tunes, g_live, g_max_live, g_collect_errors;
static double g_setup_s = 0.002, g_step_ns_per_cell = 1.0;
static int g_fail_tunes;            /* the next g_fail_tunes autotunes report LESGPU_ECUDA */

void fake_fail_tunes(int n) {
    pthread_mutex_lock(&g_mu);
    g_fail_tunes = n;
    pthread_mutex_unlock(&g_mu);
}

static void nap(double s) {
    if (s <= 0) return;
    struct timespec ts;
    ts.tv_sec = (time_t)s;
    ts.tv_nsec = (long)((s - (double)ts.tv_sec) * 1e9);
    nanosleep(&ts, NULL);
}

/* limit: device bytes before set-up reports LESGPU_ENOMEM (0: none). */
void fake_configure(size_t limit, double setup_s, double step_ns_per_cell) {
    pthread_mutex_lock(&g_mu);
    g_limit = limit ? limit : (size_t)-1;
    g_setup_s = setup_s;
    g_step_ns_per_cell = step_ns_per_cell;
    g_used = g_peak = 0;
    g_creates = g_enomem = g_tunes = g_live = g_max_live = g_collect_errors = 0;
    g_fail_tunes = 0;
    pthread_mutex_unlock(&g_mu);
}

/* used, peak, creates, enomem, tunes, live, max_live, collect_errors */
void fake_stats(long long out[8]) {
    pthread_mutex_lock(&g_mu);
    out[0] = (long long)g_used; out[1] = (long long)g_peak; out[2] = g_creates; out[3] = g_enomem;
    out[4] = g_tunes; out[5] = g_live; out[6] = g_max_live; out[7] = g_collect_errors;
    pthread_mutex_unlock(&g_mu);
}

size_t lesgpu_bytes_for_grid(int nx, int ny, int nz, int precision) {
    return (size_t)nx * ny * nz * (precision == LESGPU_FP64 ? 472 : 280);
}

size_t lesgpu_device_bytes(const lesgpu_ctx* ctx) { return ctx ? ((const les_solver*)ctx)->bytes : 0; }

int lesgpu_bind_device(int device) { return device < 0 ? LESGPU_EINVAL : LESGPU_OK; }

int les_solver_create(const lesgpu_config* cfg, const char* chem, const char* tran, int start, les_solver** out) {
    (void)chem; (void)tran; (void)start;
    if (!cfg || !out) return LESGPU_EINVAL;
    *out = NULL;
    nap(g_setup_s);
    const size_t b = lesgpu_bytes_for_grid(cfg->nx, cfg->ny, cfg->nz, cfg->precision);
    pthread_mutex_lock(&g_mu);
    if (g_used + b > g_limit) {
        g_enomem++;
        pthread_mutex_unlock(&g_mu);
        return LESGPU_ENOMEM;
    }
    g_used += b;
    if (g_used > g_peak) g_peak = g_used;
    g_creates++;
    if (++g_live > g_max_live) g_max_live = g_live;
    pthread_mutex_unlock(&g_mu);
    les_solver* s = (les_solver*)calloc(1, sizeof(les_solver));
    s->cfg = *cfg;
    s->bytes = b;
    *out = s;
    return LESGPU_OK;
}

void les_solver_destroy(les_solver* s) {
    if (!s) return;
    pthread_mutex_lock(&g_mu);
    g_used -= s->bytes;
    g_live--;
    pthread_mutex_unlock(&g_mu);
    free(s);
}

lesgpu_ctx* les_solver_ctx(les_solver* s) { return (lesgpu_ctx*)s; }
int les_solver_set_outputs(les_solver* s, const char* dir, int flags) { (void)dir; (void)flags; return s ? 0 : -1; }

int les_solver_loop_begin(les_solver* s, int chunk) {
    if (!s || chunk < 1) return LESGPU_EINVAL;
    s->chunk = chunk;
    s->loop_on = 1;
    return LESGPU_OK;
}

int les_solver_flush(les_solver* s) { (void)s; return LESGPU_OK; }

int les_solver_loop_end(les_solver* s) {
    if (!s || !s->loop_on || s->inflight) return LESGPU_ESTATE;
    s->loop_on = 0;
    return LESGPU_OK;
}

int les_solver_next_chunk(const les_solver* s, int left) { return left < s->chunk ? left : s->chunk; }

int lesgpu_run(lesgpu_ctx* ctx, int n) {
    les_solver* s = (les_solver*)ctx;
    if (!s || !s->loop_on || n < 1 || s->inflight + n > s->chunk) return LESGPU_ESTATE;
    s->inflight += n;
    return LESGPU_OK;
}

int les_solver_loop_collect(les_solver* s, int n) {
    if (!s || n != s->inflight) {
        pthread_mutex_lock(&g_mu);
        g_collect_errors++;
        pthread_mutex_unlock(&g_mu);
        return LESGPU_ESTATE;
    }
    nap(1e-9 * g_step_ns_per_cell * (double)n * s->cfg.nx * s->cfg.ny * s->cfg.nz);
    s->steps_done += n;
    s->inflight = 0;
    return LESGPU_OK;
}

/* field k, cell q: seed * 1000 + steps run + k + 1e6 * tiles[0] */
int lesgpu_download_state(lesgpu_ctx* ctx, double* const* fields, int nfields) {
    les_solver* s = (les_solver*)ctx;
    if (!s || s->inflight) return LESGPU_ESTATE;
    const size_t n = (size_t)s->cfg.nx * s->cfg.ny * s->cfg.nz;
    for (int k = 0; k < nfields; k++)
        for (size_t q = 0; q < n; q++)
            fields[k][q] = (double)s->cfg.seed * 1000.0 + s->steps_done + k + 1e6 * s->tiles[0];
    return LESGPU_OK;
}

/* tiles from the grid alone, so every tuning of one shape gives the same tiles */
int lesgpu_autotune(lesgpu_ctx* ctx, int reps, int tiles_out[5], double* ms_out) {
    (void)reps; (void)ms_out;
    les_solver* s = (les_solver*)ctx;
    nap(g_setup_s);
    pthread_mutex_lock(&g_mu);
    g_tunes++;
    const int fail = g_fail_tunes > 0;
    if (fail) g_fail_tunes--;
    pthread_mutex_unlock(&g_mu);
    if (fail) return LESGPU_ECUDA;
    for (int q = 0; q < 5; q++) s->tiles[q] = s->cfg.nx % 8;
    if (tiles_out) memcpy(tiles_out, s->tiles, sizeof(s->tiles));
    return LESGPU_OK;
}

int lesgpu_set_tiles(lesgpu_ctx* ctx, const int tiles[5]) {
    memcpy(((les_solver*)ctx)->tiles, tiles, 5 * sizeof(int));
    return LESGPU_OK;
}
int lesgpu_get_scalar_staging(const lesgpu_ctx* ctx) { return ((const les_solver*)ctx)->staged; }
int lesgpu_set_scalar_staging(lesgpu_ctx* ctx, int enable) {
    ((les_solver*)ctx)->staged = enable;
    return LESGPU_OK;
}
