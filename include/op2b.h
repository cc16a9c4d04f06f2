/*
 * op2b.h -- extensions of the B200 OP2 library beyond the reference C API.
 *
 * Nothing here is needed by the reference apps; op_lib.h alone is the
 * drop-in.  These calls choose how the loops run, expose the device stream
 * and timers to benchmark drivers, and return errors instead of exiting.
 * All have C linkage.
 */
#ifndef OP2B_H
#define OP2B_H

#include "op_lib_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* How loops with OP_INC through a map are executed.
 *  GATHER   : owner-computes.  Each target element sums its contributions
 *             in ascending (element, argument) order, which is exactly the
 *             order of the reference's sequential op_seq.h back-end, so the
 *             results are bit-identical to it.  No colouring, no atomics.
 *  COLOURED : the two-level colouring of op_plan (blocks staged in shared
 *             memory, increments applied in thread-colour order, blocks
 *             launched colour by colour).  Deterministic; summation order
 *             differs from op_seq.h, as in the reference's CUDA/OpenMP code.
 *  AUTO     : per loop, the faster of the two as measured by the tuner. */
enum { OP2B_STRATEGY_AUTO = 0, OP2B_STRATEGY_GATHER = 1, OP2B_STRATEGY_COLOURED = 2 };

/* How global OP_INC reductions (op_arg_gbl ... OP_INC) are summed.
 *  TREE : fixed-shape tree (per-thread, warp shuffle, per-block, one final
 *         block); deterministic run to run.
 *  SEQ  : element order, one addition at a time, exactly as op_seq.h does;
 *         bit-identical to the reference, at the cost of a serial pass. */
enum { OP2B_REDUCE_TREE = 0, OP2B_REDUCE_SEQ = 1 };

/* Kernel-variant knobs, used by the tuner and by experiments; returns the
 * previous value or -1.  Keys:
 *   "gather_tiled"  0: one thread per incremented element, contributions
 *                   loaded in batches (default); 1: one thread per
 *                   contribution in CTA tiles, folded in shared memory
 *   "gather_flux"   1: res_calc as two passes, each edge's flux computed once
 *                   into a buffer, then folded per cell in edge order
 *                   (default); 0: one pass, each cell recomputes its fluxes
 *   "gather_batch"  contributions whose loads are issued together per
 *                   thread in the per-element GATHER kernel (1, 2, 4)
 *   "unroll"        elements per thread in the direct loops (1, 2, 4)
 *   "fold_variant", "flux_ctas_per_sm"
 *                   launch shapes of the two-launch res_calc chain
 *   "chain_persist" 1: the res_calc chain as one persistent launch over a
 *                   dependency-ordered queue of flux and cell tiles
 *                   ("persist_et", "persist_u", "persist_lag" shape it)
 *   "chain_tiled"   1: the res_calc chain as one launch in which each CTA
 *                   computes its tile's fluxes into shared memory and
 *                   updates the tile's cells ("tile_threads" 1024 or 512
 *                   per CTA, "tile_cells" the tile size, 0 automatic)
 *   "jac_step"      1 (default): with reductions deferred, jac1's update and
 *                   the res that follows it as one launch ("jac_tile_nodes"
 *                   the tile size, 0 automatic; "jac_step_threads" 512,
 *                   1024 or 256 per CTA); 0: two launches
 *   "known_zero"    1 (default): the res_calc chain neither reads nor
 *                   rewrites res when res is known to hold zeros
 *                   (op2b_res_skips); 0: it always reads res
 * Every setting leaves the fields bit-identical. */
int op2b_set_tuning(const char *key, int value);
/* The value of a tuning knob, or `def` when it is unset. */
int op2b_get_tuning(const char *key, int def);

/* Autotuner for the launch shapes of the airfoil res_calc chain
 * (res_calc + bres_calc + update + adt_calc), the choice the reference
 * leaves to compile-time OP_PART_SIZE / OP_BLOCK_SIZE macros
 * (airfoil/res_calc_kernel.cu:181-204, common/op_lib_core.c:663-673).  Call
 * it after one outer iteration has run through the loop API.  If
 * `cache_path` (may be NULL) holds an entry for this device, real type and
 * mesh (set sizes), its knobs are applied and 1 is returned.  Otherwise
 * every candidate -- the persistent one-launch chain at several flux tile
 * sizes, cells per thread and queue lags, the tiled one-launch chain at
 * 1024 and 512 threads per CTA, and the two-launch chain with its per-cell
 * pass variants -- is timed for `iters` launches (each after an L2
 * flush) on the app's own data, which is saved first and put back after
 * each candidate; the fastest is applied, appended to the cache file, and 0
 * is returned.  All these candidates leave every field bit-identical; only
 * the order of the TREE rms sum follows the launch shape.  allow_reorder
 * != 0 also times COLOURED (the reference's colouring scheme) at part sizes
 * 64..512 with 64..512 threads per block (the run-time OP_PART_SIZE and
 * OP_BLOCK_SIZE of op_init), whose fields differ from op_seq.h's in the
 * last bits.  -1 on
 * error (no chain has run, captured graphs exist).  Synchronises. */
int op2b_autotune(const char *cache_path, int iters, int allow_reorder);

/* Renumber every set for locality of the indirect gathers (off by default).
 * Call before the first loop; the first loop call then orders the sets
 * (Cuthill-McKee on the set most maps point to, the others following through
 * the maps), stores every dataset in the new order on the device and maps in
 * the new numbering.  op_fetch_data returns data in the app's order, and
 * results are the same as without renumbering (contributions still follow
 * the app's element order); plans from op_plan_get describe the renumbered
 * sets, and TREE-mode global sums are summed in another order.  Returns 0,
 * or -1 when turning it off after it has been applied. */
int op2b_set_renumber(int on);
/* Renumber by recursive coordinate bisection (the reference's developer
 * notes propose it, doc/dev.tex:191-210) instead of Cuthill-McKee:
 * `coords` (1 to 3 float or double components per element) orders its own
 * set -- each segment of the order halved at its median along its longest
 * extent, down to single elements, coordinates compared rounded to float,
 * ties by element number -- and the other sets follow through the maps as
 * above.  Turns renumbering on; NULL returns to Cuthill-McKee.  Call before
 * the first loop.  Returns 0, or -1 (bad coordinates, or after the first
 * loop).  No reference counterpart. */
int op2b_set_renumber_coords(op_dat coords);
/* The new -> old order renumbering would give `set` (computed on the GPU from
 * the sets and maps declared so far).  Returns 1 if the set is reordered,
 * 0 if it keeps its numbering (new2old = identity), -1 on bad arguments. */
int op2b_renumber_order(op_set set, int *new2old);
/* Seconds the renumbering took at the first loop call (orders computed on
 * the GPU, maps and datasets moved), 0 before it.  No reference counterpart. */
double op2b_renumber_seconds(void);

/* Checkpointing (doc/dev.tex:1080-1087 proposes it; the reference has no
 * implementation).  op2b_checkpoint_file(path) names the checkpoint file;
 * call it after op_init, before the first loop.  If the file holds a
 * checkpoint, the run fast-forwards: loop calls do not run but return the
 * global reduction values recorded in the file, until the op_checkpoint call
 * at which it was saved, which restores every dataset (matched by name) and
 * resumes.  Returns 1 when resuming, 0 when starting fresh, -1 on error.
 * op_checkpoint() saves every dataset and every reduction value returned so
 * far (atomically: written to path.tmp, then renamed); returns 1 when saved,
 * 2 where a fast-forwarded run resumed, 0 for an earlier checkpoint passed
 * while fast-forwarding, -1 on error.  Needs reductions returned at each loop
 * call (not op2b_set_gbl_deferred). */
int op2b_checkpoint_file(const char *path);
int op_checkpoint(void);

/* op_decl_const of include/op_seq.h (the sequential API's unnamed form,
 * op_lib.h:177-182): declares the constant under the name written in `expr`,
 * the app's argument expression ("&gam" -> "gam", "qinf" -> "qinf"). */
void op2b_decl_const_named(int dim, const char *type, int size, char *dat, const char *expr);

/* Errors: EXIT (default, like the reference: print and exit) or RETURN
 * (print, remember the message, return NULL / do nothing). */
enum { OP2B_ERRORS_EXIT = 0, OP2B_ERRORS_RETURN = 1 };

int         op2b_set_strategy(int strategy);   /* returns the previous value */
int         op2b_set_reduction(int mode);      /* returns the previous value */
int         op2b_set_error_mode(int mode);     /* returns the previous value */
const char *op2b_last_error(void);             /* "" when none               */
void        op2b_clear_error(void);

/* The CUDA stream all loops are issued on (a cudaStream_t).  Setting it lets
 * a caller capture the loops into a CUDA graph or order them with its own
 * work. */
void *op2b_get_stream(void);
void  op2b_set_stream(void *stream);
/* Wait for all issued loops; returns 0 or a CUDA error code. */
int   op2b_sync(void);

/* Global reductions normally complete inside the loop call (the reference
 * semantics: the host variable holds the result on return).  With deferred
 * mode on, a loop with OP_INC/OP_MIN/OP_MAX global arguments only issues
 * device work; the results reach the host variables at the next
 * op2b_sync(), op_fetch_data() or op2b_set_gbl_deferred(0).  Deferred mode is
 * what makes an outer iteration capturable as one CUDA graph. */
int   op2b_set_gbl_deferred(int on);

/* Per-loop device time in seconds and call count, by loop name (CUDA events
 * around each loop; summed lazily).  Returns -1 if the name is unknown. */
double op2b_loop_time(char const *name, int *count);
/* Per-loop device timing for op_timing_output / op2b_loop_time: 0 off,
 * 1 sampled (default: a loop's first call and every 16th call are timed with
 * events, the total is estimated from them; each event pair costs host time
 * on every timed call), 2 every call.  Call counts are always exact.
 * Returns the old mode. */
int    op2b_set_timing(int mode);

/* CUDA graphs.  op2b_capture_begin() starts capturing the library stream;
 * the op_par_loop calls that follow are recorded, not run, with their global
 * reductions deferred; op2b_capture_end() instantiates them as one graph.
 * Plans must already exist (run the loops once before capturing).  Each
 * op2b_graph_launch() re-arms the graph's reductions: the results of the
 * latest launch reach the host variables at the next op2b_sync().  With
 * profile != 0 each loop is bracketed by event nodes so that
 * op2b_graph_loop_times() reports per-loop device time of the most recent
 * launch.  Handles are opaque; 0 / NULL means failure. */
int   op2b_capture_begin(int profile);
void *op2b_capture_end(void);
int   op2b_graph_launch(void *graph);
int   op2b_graph_nloops(void *graph);
int   op2b_graph_nkernels(void *graph);
char const *op2b_graph_loop_name(void *graph, int i);
/* seconds of each recorded loop in the last launch (waits for it) */
int   op2b_graph_loop_times(void *graph, double *seconds, int n);
void  op2b_graph_destroy(void *graph);

/* Plan validation on the device: the reference's op_plan_check plus the
 * colouring checks it lacks.  Returns the number of violations found. */
long op2b_plan_validate(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                        int ninds, int *inds);

/* Evict L2 on the library stream by reading (not writing) a buffer three
 * times its size; benchmark drivers call it between timed steps. */
int op2b_l2_flush(void);

/* Layout measurement (bench.py --mode layout): res_calc's flux pass over
 * every interior edge of the given mesh and fields, with the datasets stored
 * element-major (AoS, the library's layout) and component-major (SoA), the
 * same arithmetic in the same order.  Times `iters` launches of each (L2
 * flushed before each) into *us_aos and *us_soa (microseconds per launch).
 * Returns 0 when both wrote bit-identical flux records, 1 when they differ,
 * -1 on bad arguments or a CUDA failure.  No counterpart in the reference,
 * whose developer notes weigh the two layouts (doc/dev.tex:529-651). */
int op2b_layout_ab(int nedge, int ncell, int nnode, const int *pedge, const int *pecell,
                   const float *x, const float *q, const float *adt, float gm1, float eps,
                   int iters, double *us_aos, double *us_soa);

/* Bounded waits that ran out in the library's kernels (the persistent
 * chain's waits for the flux tiles a cell tile reads) since the last reset;
 * reset != 0 clears the count.  Every wait gives up after one second, counts
 * here and lets its kernel return, so a lost completion shows up as a
 * nonzero count (and wrong results) instead of a hung GPU; 0 in every
 * correct run.  Synchronises the library stream.  No counterpart in the
 * reference. */
unsigned op2b_wait_timeouts(int reset);

/* Launches of the tiled res_calc chain (tuning knob "chain_tiled": one
 * launch per res_calc + bres_calc + update [+ adt_calc] [+ save_soln], each
 * CTA computing its tile's fluxes into shared memory and updating the tile's
 * cells, q and adt written to second buffers that are swapped in) queued or
 * captured since the last reset; reset != 0 clears the count.  No
 * counterpart in the reference. */
unsigned long long op2b_tiled_launches(int reset);

/* Launches of the res_calc chain (res_calc + bres_calc + update, fused) that
 * neither read nor rewrote res because res held +0.0 in every element when
 * res_calc was called -- as the previous update leaves it and nothing else
 * wrote it since -- queued or captured since the last reset; reset != 0
 * clears the count.  The fold's sums start from the same +0.0 in registers,
 * so every value is the same as when res is read.  A graph captured while
 * res was known zero is set, at each launch, to read res when res may hold
 * other values then.  No counterpart in the reference. */
unsigned long long op2b_res_skips(int reset);

/* Bytes copied from host to device by dataset declarations and map uploads
 * since the last reset; reset != 0 clears the count.  A dataset declared
 * from a large (1 MiB or more) array in pageable host memory that holds only
 * zero bytes is not copied: its device buffer is cleared instead (same
 * bytes; knob "decl_zero_scan", 1 by default) and the dataset is known to
 * hold zeros.  No counterpart in the reference. */
unsigned long long op2b_h2d_bytes(int reset);

/* The airfoil update loop (q = qold - res/adt, res = 0, *rms += sum of
 * del^2) for callers that must not allocate device memory: code that cannot
 * afford cudaMalloc's device synchronisation, hosts that reserve all device
 * memory for their own pool, or latency-bound threads that cannot take a
 * first-call allocation.  No counterpart in the reference.
 * All pointers are the caller's 16-byte-aligned FP32 device arrays (qold, q,
 * res: 4 per cell; adt: 1 per cell; rms: 1 value, added to).  Nothing is
 * allocated: the reduction's scratch is a fixed 16 KB array inside the
 * library, so ncell must be at most 4,194,304 (larger sizes return -1 and run
 * nothing).  The first call on a device looks up that array's address: make
 * it before any stream capture.  All calls share the array, so calls that
 * overlap on the GPU race; calls in one stream are safe.  Misaligned or
 * null pointers return -3 before anything is launched.  The scratch address
 * is cached per device until op_exit: call op_exit before resetting a
 * device.  The call runs on the caller's `stream` (a cudaStream_t, NULL for
 * the default stream) with no ordering against the library's own stream:
 * synchronise, or pass op2b_get_stream(), when mixing it with op_par_loop
 * calls on the same data.  Returns 0, a negative code for bad arguments, or
 * a CUDA error code; asynchronous. */
int op2b_update_noalloc(int ncell, const float *qold, float *q, float *res, const float *adt,
                        float *rms, void *stream);

/* Library build string (arch, flags). */
char const *op2b_version(void);

#ifdef __cplusplus
}
#endif

#endif
