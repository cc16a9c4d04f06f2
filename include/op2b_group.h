/*
 * op2b_group.h -- many airfoil solves on one GPU: the batched and served
 * forms of the airfoil iteration.  No counterpart in the reference, whose
 * apps solve one mesh per process (airfoil/airfoil_op.cpp:112-303).
 *
 * A group holds any number of independent solves, each a mesh plus a flow
 * condition, with its datasets, maps and contribution lists resident in HBM.
 * Every loop of the outer iteration (save_soln + adt_calc, then twice
 * res_calc + bres_calc + update [+ adt_calc]) runs as one launch over a
 * whole block of active solves (all of them, or as many as keep the block's
 * intermediate values in L2): a tile table lists tiles of one solve's
 * elements, and each CTA works on one tile.  The iteration is rotated: the
 * next iteration's save_soln + adt_calc run in the second update's launch,
 * and a solve's first ones in a launch before its first iteration.  The per-element arithmetic is the plain path's
 * (same device functions, same contribution order), so a solve's flow field
 * q is bit-identical to the plain op_par_loop solve of the same mesh and
 * flow.  Each solve's rms is folded from its own tiles' partials, in tile
 * order, by the last of its CTAs to finish: it depends only on that solve, so
 * a solve's results are bit-identical whether it runs alone or with any
 * other solves.  The rms history and the stopping test live on the device:
 * no host round trip per iteration.
 *
 * A solve stops after max_iter outer iterations, or at the end of the first
 * iteration k >= 2 whose rms is below rel_tol times the rms of iteration 1
 * (rel_tol <= 0: iteration count only).  rms = sqrt(sum of del^2 over the
 * cells / ncell) of the iteration's second update, as airfoil computes it
 * (airfoil/airfoil_op.cpp:291-296).
 *
 * Calls are from one host thread.  Admission (op2b_group_add) uploads and
 * builds on a stream of its own, so it overlaps the running iterations of
 * the other solves; a solve joins at the next op2b_group_run.
 */
#ifndef OP2B_GROUP_H
#define OP2B_GROUP_H

#include "op2b_mesh.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct op2b_group_s *op2b_group;

/* Free-stream state for Mach number `mach` and angle of attack `alpha_deg`
 * (degrees), computed as airfoil/airfoil.cpp:134-149 does in the app's real
 * type, with the velocity turned by alpha: qinf = (r, r*u*cos a, r*u*sin a,
 * r*e).  alpha = 0 gives the reference's qinf exactly (the reference leaves
 * alpha out of qinf).  qinf4 points to 4 floats (fp64 = 0) or 4 doubles;
 * consts4, when not NULL, receives gam, gm1, cfl, eps in the same type. */
int op2b_flow_qinf(double mach, double alpha_deg, int fp64, void *qinf4, void *consts4);

op2b_group op2b_group_create(int fp64);
void op2b_group_destroy(op2b_group g);

/* Admit one solve: returns its id (>= 0), or -1 (see op2b_last_error).  The
 * mesh arrays are copied; the caller may free them after the call. */
int op2b_group_add(op2b_group g, const op2b_mesh *m, double mach, double alpha_deg, int max_iter,
                   double rel_tol);

/* Enqueue niter outer iterations of every active solve (solves admitted
 * since the last call join first).  Returns the number of solves in the
 * launches, or -1.  Asynchronous: it does not wait for the GPU. */
int op2b_group_run(op2b_group g, int niter);

/* Wait for the enqueued work; fills ids[0..] (up to max) with solves that
 * have stopped and were not reported before; returns their count. */
int op2b_group_poll(op2b_group g, int *ids, int max);

/* Per-solve results.  op2b_group_sync waits for all enqueued work. */
int op2b_group_sync(op2b_group g);
int op2b_group_iterations(op2b_group g, int id);
int op2b_group_history(op2b_group g, int id, double *rms, int max); /* returns count */
int op2b_group_fetch_q(op2b_group g, int id, void *q);              /* ncell*4 reals */
/* The same for a solve op2b_group_poll has reported stopped, queued while
 * the other solves iterate (into pinned memory for an overlapped copy): q is
 * valid after op2b_group_sync.  Any other solve: as op2b_group_fetch_q. */
int op2b_group_fetch_q_async(op2b_group g, int id, void *q);

/* Release a solve's device memory; it leaves the group. */
int op2b_group_remove(op2b_group g, int id);

/* Device bytes a solve of this mesh takes, and the group's total. */
long long op2b_group_solve_bytes(op2b_group g, int nnode, int ncell, int nedge, int nbedge,
                                 int max_iter);
long long op2b_group_device_bytes(op2b_group g);
int op2b_group_active(op2b_group g); /* solves in the launches (joined, not stopped) */

/* An iteration runs block by block over the solves (in id order), each
 * block's launches together, so that a block's flux values -- written
 * by one launch, read by the next -- stay in L2: a block holds up to `bytes`
 * of values (<= 0, the default: all solves in one block).  Results do not
 * depend on it. */
int op2b_group_set_block_bytes(op2b_group g, long long bytes);
/* Blocks are dealt round-robin to n streams (1..8) inside the captured
 * iteration, so independent blocks' launches overlap (one block's per-cell
 * pass beside another's flux pass).  Results do not depend on it. */
int op2b_group_set_streams(op2b_group g, int n);
/* The tiled chain: each update and the loops fused with it as ONE launch
 * over all solves, a CTA per tile of consecutive cells of one solve, the
 * flux values in shared memory (edges between tiles computed by both)
 * instead of written to and read back from device memory; update and
 * adt_calc write to second buffers of q and adt (20 bytes per cell in FP32,
 * plus the tile lists, counted by op2b_group_solve_bytes while it is on).
 * Fields are bit-identical to the two-launch form; each solve's rms is
 * folded over its own tiles, so the rms history differs from the two-launch
 * form's in the last bits and is the same alone or in any mix.  on = 0
 * (the default) or 1; returns 0.  op2b_group_tiled returns the mode. */
int op2b_group_set_tiled(op2b_group g, int on);
int op2b_group_tiled(op2b_group g);

/* Launch shape of the flux pass: edges per tile (multiple of 256, 256..8192).
 * Results do not depend on it; op2b_group_autotune picks it by timing. */
int op2b_group_set_edge_tile(op2b_group g, int edges_per_tile);
int op2b_group_edge_tile(op2b_group g);
/* Time `iters` iterations at each candidate edge tile, then at each block
 * size and stream count (one block on one stream; 96 or 48 MiB blocks on
 * one stream; 48 or 24 MiB on two; 24 MiB on three; 12 MiB on four), on the
 * current active solves, putting their state back after each trial; keeps
 * the fastest of each and returns the edge tile. */
int op2b_group_autotune(op2b_group g, int iters);
/* The same candidates, each timed on `iters` REAL iterations of the active
 * solves (their state advances; launch shapes do not change results);
 * keeps the fastest of each and returns the iterations run (11 x iters), or
 * -1.  Tuning then costs only the graph rebuilds.  Synchronises. */
int op2b_group_autotune_run(op2b_group g, int iters);

#ifdef __cplusplus
}
#endif

#endif
