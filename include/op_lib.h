/*
 * op_lib.h -- OP2 user API of the B200 library (libop2b200.so).
 *
 * Drop-in for the reference's common/op_lib.h: the generated app mains
 * (airfoil/airfoil_op.cpp, jac1/jac_op.cpp, jac2/jac_op.cpp) include this
 * header unchanged and link against libop2b200.so instead of op_lib.cu +
 * the generated *_kernel.cu files.
 *
 * Differences from the reference header, all link-level:
 *  - every non-template function has C linkage (the reference gave C++
 *    linkage to op_init, op_decl_dat_char, op_decl_const_char, op_fetch_data,
 *    op_plan_get and op_exit), so FFIs can bind them by plain name;
 *  - the loop entry points this library implements are declared here with C
 *    linkage.  The app's own later declarations of the same functions
 *    (airfoil/airfoil_op.cpp:64-99) then inherit that linkage.  Define
 *    OP2B_NO_LOOP_DECLS to leave them out.
 */
#ifndef OP_LIB_H
#define OP_LIB_H

#include "op_lib_core.h"

#ifdef __cplusplus
/* run-time type checks (op_lib.h:45-51) */
inline int type_error(const double *, const char *type) { return strcmp(type, "double"); }
inline int type_error(const float *, const char *type) { return strcmp(type, "float"); }
inline int type_error(const int *, const char *type) { return strcmp(type, "int"); }
inline int type_error(const uint *, const char *type) { return strcmp(type, "uint"); }
inline int type_error(const ll *, const char *type) { return strcmp(type, "ll"); }
inline int type_error(const ull *, const char *type) { return strcmp(type, "ull"); }
inline int type_error(const bool *, const char *type) { return strcmp(type, "bool"); }

#ifdef OP_USER_DATATYPES
#include <OP_USER_DATATYPES>
#endif
#endif

/* zero constants (op_lib.h:65-71) */
#define ZERO_double 0.0;
#define ZERO_float 0.0f;
#define ZERO_int 0;
#define ZERO_uint 0;
#define ZERO_ll 0;
#define ZERO_ull 0;
#define ZERO_bool 0;

/* identity mapping and global identifier (op_lib.h:76-77) */
#define OP_ID (op_map) NULL
#define OP_GBL (op_map) NULL

#ifdef __cplusplus
extern "C" {
#endif

/* registries and settings (op_lib.h:83-95) */
extern int OP_diags, OP_part_size, OP_block_size;
extern int OP_set_index, OP_set_max, OP_map_index, OP_map_max, OP_dat_index, OP_dat_max,
    OP_plan_index, OP_plan_max, OP_kern_max;
extern op_set *OP_set_list;
extern op_map *OP_map_list;
extern op_dat *OP_dat_list;
extern op_plan *OP_plans;
extern op_kernel *OP_kernels;

/* CUDA-side entry points (op_lib.h:103-154; common/op_lib.cu) */
void     op_init(int argc, char **argv, int diags);
op_dat   op_decl_dat_char(op_set set, int dim, char const *type, int size, char *data,
                          char const *name);
void     op_decl_const_char(int dim, char const *type, int size, char *dat, char const *name);
void     op_fetch_data(op_dat dat);
op_plan *op_plan_get(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                     int ninds, int *inds);
void     op_exit(void);

#ifndef OP2B_NO_LOOP_DECLS
/* parallel loops of the reference apps (airfoil/airfoil_op.cpp:64-99,
 * jac1/jac_op.cpp:58-73); arguments as in those files */
void op_par_loop_save_soln(char const *, op_set, op_arg, op_arg);
void op_par_loop_adt_calc(char const *, op_set, op_arg, op_arg, op_arg, op_arg, op_arg, op_arg);
void op_par_loop_res_calc(char const *, op_set, op_arg, op_arg, op_arg, op_arg, op_arg, op_arg,
                          op_arg, op_arg);
void op_par_loop_bres_calc(char const *, op_set, op_arg, op_arg, op_arg, op_arg, op_arg, op_arg);
void op_par_loop_update(char const *, op_set, op_arg, op_arg, op_arg, op_arg, op_arg);
void op_par_loop_res(char const *, op_set, op_arg, op_arg, op_arg, op_arg);
#endif

/* generic form of every loop above: dispatch by name and argument signature */
void op2b_par_loop(char const *name, op_set set, int nargs, const op_arg *args);

#ifdef __cplusplus
}

/* templates for datasets, constants and global arguments (op_lib.h:160-190) */
template <class T>
op_dat op_decl_dat(op_set set, int dim, char const *type, T *data, char const *name) {
  if (type_error(data, type)) {
    printf("incorrect type specified for dataset \"%s\" \n", name);
    exit(1);
  }
  return op_decl_dat_char(set, dim, type, sizeof(T), (char *)data, name);
}

template <class T>
void op_decl_const2(char const *name, int dim, char const *type, T *data) {
  if (type_error(data, type)) {
    printf("incorrect type specified for constant \"%s\" \n", name);
    exit(1);
  }
  op_decl_const_char(dim, type, sizeof(T), (char *)data, name);
}

template <class T>
void op_decl_const(int dim, char const *type, T *data) {
  if (type_error(data, type)) {
    printf("incorrect type specified for constant in op_decl_const");
    exit(1);
  }
}

template <class T>
op_arg op_arg_gbl(T *data, int dim, char const *type, op_access acc) {
  if (type_error(data, type)) return op_arg_gbl_core((char *)data, dim, "error", acc);
  return op_arg_gbl_core((char *)data, dim, type, acc);
}
#endif

#endif
