/*
 * op_lib_core.h -- OP2 core types and C entry points of the B200 library
 * (libop2b200.so).
 *
 * Drop-in for the reference's common/op_lib_core.h: every type below has the
 * reference's field order and sizes (op_lib_core.h:67-158), because apps pass
 * op_arg by value and read op_plan / op_kernel fields directly.  Functions
 * are declared with C linkage so any FFI (ctypes, cgo, JNI) can bind them.
 */
#ifndef OP_LIB_CORE_H
#define OP_LIB_CORE_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

typedef unsigned int uint;
typedef long long ll;
typedef unsigned long long ull;

#ifdef __cplusplus
extern "C" {
#endif

/* diagnostics level set by op_init (op_lib_core.h:52-61):
 * 0 none, 1 error checks, 2 plan info, 3 loop execution, 4 old plans,
 * 7 positive plan checks */
extern int OP_diags;

/* op_lib_core.h:67-69 */
typedef enum { OP_READ, OP_WRITE, OP_RW, OP_INC, OP_MIN, OP_MAX } op_access;
typedef enum { OP_ARG_GBL, OP_ARG_DAT } op_arg_type;

/* op_lib_core.h:75-80 */
typedef struct {
  int         index; /* position in the set registry */
  int         size;  /* number of elements           */
  char const *name;
} op_set_core;
typedef op_set_core *op_set;

/* op_lib_core.h:84-92; map points at the caller's array (borrowed) */
typedef struct {
  int         index;
  op_set      from, to;
  int         dim, *map;
  char const *name;
} op_map_core;
typedef op_map_core *op_map;

/* op_lib_core.h:96-105; data = caller's array (borrowed), data_d = the
 * device copy this library owns */
typedef struct {
  int         index;
  op_set      set;
  int         dim, size; /* size = dim * bytes per item */
  char       *data, *data_d;
  char const *type, *name;
} op_dat_core;
typedef op_dat_core *op_dat;

/* op_lib_core.h:107-119; passed by value to every loop */
typedef struct {
  int         index;
  op_dat      dat;
  op_map      map;
  int         dim, idx, size;
  char       *data, *data_d;
  char const *type;
  op_access   acc;
  op_arg_type argtype;
} op_arg;

/* op_lib_core.h:122-150.  From op_plan_core the arrays are host memory;
 * from op_plan_get they are device memory except ncolblk and nindirect. */
typedef struct {
  char const *name;
  op_set      set;
  int         nargs, ninds, part_size;
  op_map     *maps;
  op_dat     *dats;
  int        *idxs;
  op_access  *accs;
  int        *nthrcol;
  int        *thrcol;
  int        *offset;
  int       **ind_maps;
  int        *ind_offs;
  int        *ind_sizes;
  int        *nindirect;
  short     **loc_maps;
  int         nblocks;
  int        *nelems;
  int         ncolors;
  int        *ncolblk;
  int        *blkmap;
  int         nshared;
  float       transfer;
  float       transfer2;
  int         count;
} op_plan;

/* op_lib_core.h:152-158 */
typedef struct {
  char const *name;
  int         count;
  float       time;
  float       transfer;
  float       transfer2;
} op_kernel;

#ifndef MIN
#define MIN(a, b) ((a < b) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) ((a > b) ? (a) : (b))
#endif
#define ROUND_UP(bytes) (((bytes) + 15) & ~15)

/* ---- core entry points (common/op_lib.h:101-154) ---- */
void    op_init_core(int argc, char **argv, int diags);
op_set  op_decl_set(int size, char const *name);
op_map  op_decl_map(op_set from, op_set to, int dim, int *imap, char const *name);
op_dat  op_decl_dat_core(op_set set, int dim, char const *type, int size, char *data,
                         char const *name);
void    op_arg_check(op_set set, int m, op_arg arg, int *ninds, char const *name);
op_arg  op_arg_dat(op_dat dat, int idx, op_map map, int dim, char const *type, op_access acc);
op_arg  op_arg_gbl_core(char *data, int dim, char const *type, op_access acc);
void    op_diagnostic_output(void);
void    op_timing_output(void);
op_plan *op_plan_core(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                      int ninds, int *inds);
void    op_timers(double *cpu, double *et);
void    op_timing_realloc(int kernel);
void    op_exit_core(void);

#ifdef __cplusplus
}
#endif

#endif
