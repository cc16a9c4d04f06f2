/*
 * op2b_serve.h -- the continuous-batching solve server: admission,
 * retirement and latency bookkeeping over a group of solves
 * (include/op2b_group.h).  No counterpart in the reference, whose apps solve
 * one mesh per process.
 *
 * Requests (a mesh, a flow condition, a stopping rule, an arrival time)
 * queue on arrival.  Each op2b_server_step:
 *   1. when nothing is running, admits queued requests;
 *   2. enqueues iters_per_step outer iterations of every running solve (one
 *      launch per loop over all of them, asynchronous);
 *   3. admits queued requests while those iterations run on the GPU: first
 *      come first served (policy 0) or least work -- cells x iteration cap
 *      -- first (policy 1), while the group's device bytes plus the
 *      request's fit the budget and, if max_active > 0, fewer than
 *      max_active solves run (a request that does not fit waits at the head
 *      of the queue; the first one is always admitted into an empty group);
 *   4. waits for the iterations, retires the solves that stopped (rms below
 *      rel_tol x the first iteration's, or the iteration cap), keeps their
 *      rms history (and final q when keep_q) and frees their device memory.
 * A solve's results do not depend on what it ran with, so an answer is the
 * same alone or in the mix.
 *
 * The group is reached through a table of functions, so the same admission
 * logic runs the GPU engine (op2b_group_ops_fill) or any stand-in with the
 * same contract (the host tests use one).  Times are seconds on the
 * server's clock: the table's `now`, or, when it is NULL, a steady clock
 * started by op2b_server_create.  Calls are from one host thread.
 */
#ifndef OP2B_SERVE_H
#define OP2B_SERVE_H

#include "op2b_group.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  void *ctx;
  /* admit a solve of request rid; returns its solve id (>= 0) or -1 */
  int (*add)(void *ctx, long long rid, const op2b_mesh *m, double mach, double alpha_deg,
             int max_iter, double rel_tol);
  int (*run)(void *ctx, int niter);                   /* enqueue niter iterations; < 0 error */
  int (*poll)(void *ctx, int *ids, int max);          /* stopped solves not reported before */
  int (*history)(void *ctx, int sid, double *rms, int max); /* returns the count */
  int (*fetch_q)(void *ctx, int sid, void *q);        /* ncell * 4 reals; < 0 error */
  int (*remove)(void *ctx, int sid);
  long long (*solve_bytes)(void *ctx, long long rid, const op2b_mesh *m, int max_iter);
  long long (*device_bytes)(void *ctx);
  double (*now)(void *ctx); /* NULL: the server's steady clock */
} op2b_group_ops;

/* The table of the GPU engine `g` (op2b_group_*); the server does not own g. */
int op2b_group_ops_fill(op2b_group g, op2b_group_ops *ops);

typedef struct op2b_server_s *op2b_server;

/* policy: 0 first come first served, 1 least work first.  keep_q: keep each
 * finished request's final q (real_bytes = 4 or 8 per real). */
op2b_server op2b_server_create(const op2b_group_ops *ops, long long budget_bytes,
                               int iters_per_step, int max_active, int policy, int keep_q,
                               int real_bytes);
void op2b_server_destroy(op2b_server s);

/* Queue request rid.  The mesh arrays are the caller's and must stay valid
 * until the request has been admitted (the group copies them then).
 * Returns 0, or -1 on bad arguments. */
int op2b_server_submit(op2b_server s, long long rid, const op2b_mesh *m, double mach,
                       double alpha_deg, int max_iter, double rel_tol, double arrival);

/* One round (admit, iterate, admit, retire); returns the number of requests
 * finished in it, or -1 (see op2b_last_error). */
int op2b_server_step(op2b_server s);

typedef struct {
  long long rid;
  int sid, iterations;
  double arrival, admitted, finished;
} op2b_served;

/* Records of finished requests not returned before, in finishing order. */
int op2b_server_done(op2b_server s, op2b_served *out, int max);
/* A finished request's rms history (returns its length) and final q (when
 * keep_q; ncell * 4 reals); kept until op2b_server_release(rid). */
int op2b_server_history(op2b_server s, long long rid, double *rms, int max);
int op2b_server_q(op2b_server s, long long rid, void *q);
void op2b_server_release(op2b_server s, long long rid);

/* Running requests: fills rids/sids (up to max), returns their count. */
int op2b_server_active(op2b_server s, long long *rids, int *sids, int max);
int op2b_server_queued(op2b_server s);
int op2b_server_peak_active(op2b_server s);
int op2b_server_idle(op2b_server s);   /* nothing queued, nothing running */
double op2b_server_now(op2b_server s); /* the server's clock */

/* Latency (finished - arrival) over every request finished so far:
 * percentiles by linear interpolation between order statistics. */
int op2b_server_latency(op2b_server s, double *p50, double *p99, double *mean, double *max);

#ifdef __cplusplus
}
#endif

#endif
