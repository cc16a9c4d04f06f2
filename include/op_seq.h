/*
 * op_seq.h -- the sequential back-end's header (common/op_seq.h), for this
 * library: an app written against the un-generated OP2 API -- the template
 * op_par_loop(kernel, name, set, args...) of common/op_seq.h:26-1340 and the
 * unnamed op_decl_const(dim, type, ptr) -- compiles unchanged against this
 * header and runs its loops on the GPU.
 *
 *  - op_par_loop(kernel, name, set, arg0, ...) passes the arguments to
 *    op2b_par_loop, which matches their signature to a device loop (the
 *    same dispatch as the generated op_par_loop_<name> entry points).  The
 *    host kernel pointer is not called: there is no host fallback.
 *  - op_decl_const(dim, type, ptr) declares the constant under the name of
 *    the variable the app passes (`&gam` -> "gam", `qinf` -> "qinf"): the
 *    names the generated mains give op_decl_const2 (airfoil_op.cpp:227-233)
 *    and the device loops look up.
 *  - As with the reference's CUDA build, datasets live on the device; the
 *    app's host arrays are brought up to date by op_fetch_data (the
 *    sequential back-end's op_fetch_data is a no-op because it computes in
 *    the host arrays).
 */
#ifndef OP2B_OP_SEQ_H
#define OP2B_OP_SEQ_H

#include "op2b.h"
#include "op_lib.h"

/* the sequential back-end's pointer helper (common/op_seq.h:11-19) */
inline void op_arg_set(int n, op_arg arg, char **p_arg) {
  int n2 = arg.map == NULL ? n : arg.map->map[arg.idx + n * arg.map->dim];
  *p_arg = arg.data + n2 * arg.size;
}

template <class... K, class... A>
void op_par_loop(void (*kernel)(K *...), char const *name, op_set set, A... args) {
  static_assert(sizeof...(K) == sizeof...(A), "op_par_loop: one op_arg per kernel argument");
  (void)kernel;
  op_arg list[] = {args...};
  op2b_par_loop(name, set, (int)sizeof...(A), list);
}

/* constant named after the expression that passes it */
#undef op_decl_const
#define op_decl_const(dim, type, dat) \
  op2b_decl_const_named((dim), (type), (int)sizeof(*(dat)), (char *)(dat), #dat)

#endif
