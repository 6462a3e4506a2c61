/*
 * les_serve.h -- serving loop: many LES solve requests on one GPU, admitted by an HBM
 * budget and advanced together (continuous batching).
 *
 * No counterpart in the reference, which runs one solve per process (main(),
 * les_combustion_solver.c:4016-4632).  Each request is one les_solver (les_solver.h) with
 * its own grid, model constants, seed, rand() stream and output files; its results are the
 * same as running it alone with les_solver_run_device.  One host thread calls a server;
 * the server keeps prep_threads worker threads of its own for the per-request set-up and
 * tear-down (solver creation with its initial state and uploads, the final state's copy to
 * the host, releasing device memory), so that host work overlaps the device's.
 *
 *   les_serve_submit   queue a request (refused at once if it can never fit the budget);
 *   les_serve_step     one scheduling round: admit queued requests (in arrival order, or
 *                      least work first with LES_SERVE_SHORTEST) while a slot is free and
 *                      their memory fits (their set-up goes to the
 *                      workers; with nothing running the round waits for it), start
 *                      requests whose set-up is done, and collect the step history of every
 *                      running request in turn, queueing its next quantum_steps steps (one
 *                      stream and graph per request, overlapping on the device) as soon as
 *                      the last ones are collected; finished requests go to the workers and
 *                      are retired when their final state is on the host and their device
 *                      memory returned.  Returns the number of requests still queued or
 *                      active (>= 0) or a negative LESGPU_E* code;
 *   les_serve_cancel   drop a queued or active request (waits for its steps in flight);
 *   les_serve_info / les_serve_result / les_serve_release / les_serve_stats.
 * Latency is completion time minus submission time (CLOCK_MONOTONIC); p50/p99 use linear
 * interpolation between order statistics.
 */
#ifndef LES_SERVE_H
#define LES_SERVE_H

#include <stddef.h>

#include "les_solver.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { LES_REQ_QUEUED = 0, LES_REQ_ACTIVE = 1, LES_REQ_DONE = 2, LES_REQ_CANCELLED = 3, LES_REQ_FAILED = 4 };

typedef struct les_serve_options {
    size_t budget_bytes;      /* HBM the server may hand to requests */
    int max_slots;            /* at most this many active requests */
    int quantum_steps;        /* steps per request per round */
    int keep_results;         /* copy each final state to the host (les_serve_result) */
    int autotune;             /* tiles per grid size, timed on its first request and reused */
    int backfill;             /* admit later requests that fit while the head of the queue waits */
    int device;
    char chem_path[1024];
    char tran_path[1024];
    int prep_threads;         /* host threads that set up and tear down requests (0: the
                                 thread calling les_serve_step does it) */
    int policy;               /* LES_SERVE_FIFO (arrival order) or LES_SERVE_SHORTEST (least work,
                                 cells x steps, first; ties in arrival order) */
} les_serve_options;

/* Admission order.  LES_SERVE_SHORTEST lowers the median latency of a burst of requests of
 * uneven size (the short ones no longer wait behind the long ones) at the cost of the long
 * ones, which can wait while shorter requests keep arriving. */
#define LES_SERVE_FIFO 0
#define LES_SERVE_SHORTEST 1

typedef struct les_serve_request_info {
    int state, error, steps_done, nsteps;
    size_t bytes;             /* budgeted bytes */
    size_t device_bytes;      /* device bytes of the request's solver, from its start until
                                 the request is retired (0 otherwise) */
    double t_submit, t_admit, t_done, latency_s;
} les_serve_request_info;

typedef struct les_serve_summary {
    long long submitted, queued, active, done, failed, cancelled;
    size_t bytes_in_use;
    double cell_steps;        /* cell-steps completed */
    double busy_s;            /* first admission to last completion */
    double cell_steps_per_s;
    double latency_p50_s, latency_p99_s, latency_max_s;
} les_serve_summary;

typedef struct les_serve les_serve;

void les_serve_default_options(les_serve_options* opt);
/* Device bytes the server budgets for one request (grid fields, device-loop tables). */
size_t les_serve_request_bytes(const lesgpu_config* cfg, int quantum_steps);
int les_serve_create(const les_serve_options* opt, les_serve** out);
int les_serve_submit(les_serve* s, const lesgpu_config* cfg, int nsteps, const char* out_dir, int out_flags,
                     long long* id);
int les_serve_step(les_serve* s);
int les_serve_cancel(les_serve* s, long long id);
int les_serve_info(les_serve* s, long long id, les_serve_request_info* info);
int les_serve_result(les_serve* s, long long id, double* const* fields, int nfields);
int les_serve_release(les_serve* s, long long id);
int les_serve_stats(les_serve* s, les_serve_summary* st);
const char* les_serve_last_error(const les_serve* s);
void les_serve_destroy(les_serve* s);

#ifdef __cplusplus
}
#endif

#endif /* LES_SERVE_H */
