/*
 * les_ensemble.c -- many solver instances on one GPU advanced by one graph per step.
 *
 * The reference tunes its model constants with a Bayesian optimiser that proposes a
 * parameter set, recompiles the solver and runs one LES per trial (bayesian_optimizer.py:
 * 568-673, :703-716).  Here every proposed set is a member with its own grid, constants,
 * seed and state, and all members advance together: one step of every member is a single
 * multi-stream CUDA graph (lesgpu_group_*), so grids too small to fill the GPU alone share
 * it.  Each member keeps its own device-loop session, history and output files.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "les_solver.h"

struct les_ensemble {
    int n;
    int batched;          /* lesgpu_group_create_batched instead of lesgpu_group_create */
    int per_batch;        /* its max_per_batch */
    les_solver** members;
    char err[256];
};

static int eerr(les_ensemble* e, int code, const char* msg, int member) {
    if (e) {
        if (member >= 0)
            snprintf(e->err, sizeof(e->err), "member %d: %s", member, msg);
        else
            snprintf(e->err, sizeof(e->err), "%s", msg);
    }
    return code;
}

int les_ensemble_create(const lesgpu_config* cfgs, int n, const char* chem_path, const char* tran_path, int autotune,
                        les_ensemble** out) {
    if (!cfgs || n < 1 || !chem_path || !tran_path || !out) return LESGPU_EINVAL;
    *out = NULL;
    for (int q = 1; q < n; q++)
        if (cfgs[q].device != cfgs[0].device) return LESGPU_EINVAL;
    les_ensemble* e = (les_ensemble*)calloc(1, sizeof(les_ensemble));
    if (!e) return LESGPU_ENOMEM;
    e->members = (les_solver**)calloc((size_t)n, sizeof(les_solver*));
    if (!e->members) {
        free(e);
        return LESGPU_ENOMEM;
    }
    e->n = n;
    for (int q = 0; q < n; q++) {
        int rc = les_solver_create(&cfgs[q], chem_path, tran_path, 0, &e->members[q]);
        if (rc == LESGPU_OK && autotune) {
            /* tiles are tuned on the first member of each grid shape and precision and reused
               by the others, so members of one shape run the same kernels */
            int p = 0;
            while (p < q && !(cfgs[p].nx == cfgs[q].nx && cfgs[p].ny == cfgs[q].ny && cfgs[p].nz == cfgs[q].nz &&
                              cfgs[p].precision == cfgs[q].precision))
                p++;
            lesgpu_ctx* c = les_solver_ctx(e->members[q]);
            if (p < q) {
                int tl[5];
                lesgpu_ctx* src = les_solver_ctx(e->members[p]);
                rc = lesgpu_get_tiles(src, tl);
                if (rc == LESGPU_OK) rc = lesgpu_set_tiles(c, tl);
                if (rc == LESGPU_OK) rc = lesgpu_set_scalar_staging(c, lesgpu_get_scalar_staging(src));
            } else {
                rc = lesgpu_autotune(c, 3, NULL, NULL);
            }
        }
        if (rc) {
            les_ensemble_destroy(e);
            return rc;
        }
    }
    *out = e;
    return LESGPU_OK;
}

int les_ensemble_run(les_ensemble* e, int nsteps, int chunk) {
    if (!e || nsteps < 0) return LESGPU_EINVAL;
    if (nsteps == 0) return LESGPU_OK;
    if (chunk <= 0) chunk = 64;
    int rc = LESGPU_OK, bad = -1;
    int begun = 0;
    for (; begun < e->n && rc == LESGPU_OK; begun++) {
        rc = les_solver_loop_begin(e->members[begun], chunk);
        if (rc) { bad = begun; break; }
    }
    lesgpu_group* g = NULL;
    lesgpu_ctx** ctxs = NULL;
    if (rc == LESGPU_OK) {
        ctxs = (lesgpu_ctx**)malloc((size_t)e->n * sizeof(lesgpu_ctx*));
        if (!ctxs) rc = LESGPU_ENOMEM;
    }
    if (rc == LESGPU_OK) {
        for (int q = 0; q < e->n; q++) ctxs[q] = les_solver_ctx(e->members[q]);
        rc = e->batched ? lesgpu_group_create_batched(ctxs, e->n, e->per_batch, &g) : lesgpu_group_create(ctxs, e->n, &g);
    }
    int left = nsteps;
    while (rc == LESGPU_OK && left > 0) {
        /* the chunk every member can take: the shortest of their own schedules */
        int n = left;
        for (int q = 0; q < e->n; q++) {
            int m = les_solver_next_chunk(e->members[q], left);
            if (m < n) n = m;
        }
        if (n <= 0) { rc = LESGPU_ESTATE; break; }
        rc = lesgpu_group_run(g, n);
        for (int q = 0; q < e->n && rc == LESGPU_OK; q++) {
            rc = les_solver_loop_collect(e->members[q], n);
            if (rc) bad = q;
        }
        left -= n;
    }
    if (g) lesgpu_group_destroy(g);
    free(ctxs);
    for (int q = 0; q < begun; q++) {
        int rc2 = les_solver_loop_end(e->members[q]);
        if (rc == LESGPU_OK && rc2 != LESGPU_OK) { rc = rc2; bad = q; }
    }
    if (rc) {
        const char* msg = (bad >= 0) ? les_solver_last_error(e->members[bad]) : "ensemble run failed";
        if (bad < 0 && ctxs == NULL && e->n > 0) msg = lesgpu_last_error(les_solver_ctx(e->members[0]));
        return eerr(e, rc, msg, bad);
    }
    return LESGPU_OK;
}

int les_ensemble_set_batched(les_ensemble* e, int enable, int max_per_batch) {
    if (!e || max_per_batch < 0) return LESGPU_EINVAL;
    e->batched = enable != 0;
    e->per_batch = max_per_batch;
    return LESGPU_OK;
}

int les_ensemble_size(const les_ensemble* e) { return e ? e->n : 0; }

les_solver* les_ensemble_member(les_ensemble* e, int i) {
    if (!e || i < 0 || i >= e->n) return NULL;
    return e->members[i];
}

const char* les_ensemble_last_error(const les_ensemble* e) { return e ? e->err : "null ensemble"; }

void les_ensemble_destroy(les_ensemble* e) {
    if (!e) return;
    for (int q = 0; q < e->n; q++)
        if (e->members[q]) les_solver_destroy(e->members[q]);
    free(e->members);
    free(e);
}
