/*
 * op2_oracle.h -- CPU restatement of the reference's op_par_loop path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the
 * checker.  The product (oplus2_matlab_b200) never links or calls it.
 *
 * What it restates (reference paths relative to the reference project):
 *   - op_plan_core, the block partition / indirect renumbering / two-level
 *     greedy colouring plan builder        common/op_lib_core.c:627-1089
 *   - the sequential op_par_loop semantics (element order, pointers straight
 *     into the global arrays)              common/op_seq.h:11-57
 *   - the airfoil user kernels             airfoil/{save_soln,adt_calc,res_calc,
 *                                          bres_calc,update}.h
 *   - the airfoil main loop and constants  airfoil/airfoil.cpp:175-258
 *   - the jac1 / jac2 user kernels         jac1/res.h, jac1/update.h,
 *                                          jac2/res.h, jac2/update.h
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the
 * reference's own seq build (oracle/Makefile), and tests check this library
 * against them bit for bit.
 */
#ifndef OP2_ORACLE_H
#define OP2_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- plan (common/op_lib_core.c:627-1089) ---------------- */

typedef struct {
  int    set_size, nargs, ninds, bsize, nblocks, ncolors, nshared;
  int   *nthrcol;    /* [nblocks]          thread colours per block          */
  int   *thrcol;     /* [set_size]         thread colour of each element     */
  int   *offset;     /* [nblocks]          first element of each block       */
  int   *nelems;     /* [nblocks]          elements per block                */
  int   *ind_offs;   /* [nblocks*ninds]    block offsets into ind_maps       */
  int   *ind_sizes;  /* [nblocks*ninds]    distinct targets per block        */
  int   *nindirect;  /* [ninds]            total length of ind_maps[m]       */
  int  **ind_maps;   /* [ninds][nindirect] sorted distinct targets per block  */
  short**loc_maps;   /* [nargs][set_size]  block-local target index, or NULL */
  int   *ncolblk;    /* [ncolors]          blocks per block colour           */
  int   *blkmap;     /* [nblocks]          blocks grouped by colour          */
  double transfer, transfer2;  /* byte models, exact sums                   */
} op2o_plan;

/* maps[m]: int32 map of arg m (NULL for direct args), map_dims[m], idxs[m],
 * to_sizes[m] (size of the target set), dat_sizes[m] (bytes per element),
 * accs[m] (op_access value: READ 0 WRITE 1 RW 2 INC 3 MIN 4 MAX 5),
 * inds[m] (indirect dataset number or -1).  Returns 0 on success. */
int  op2o_plan_core(int set_size, int part_size, int nargs, const int *const *maps,
                    const int *map_dims, const int *idxs, const int *to_sizes,
                    const int *dat_sizes, const int *accs, int ninds, const int *inds,
                    int cache_line_size, op2o_plan *out);
void op2o_plan_free(op2o_plan *p);

/* The reference's op_plan_check (common/op_lib_core.c:469-620); returns the
 * number of failed checks (0 = plan consistent). */
int  op2o_plan_check(const op2o_plan *p, const int *const *maps, const int *map_dims,
                     const int *idxs, const int *to_sizes, const int *inds);

/* Colouring validity, which op_plan_check leaves out: no two elements of one
 * block with the same thread colour, and no two blocks with the same block
 * colour, may reach one target through OP_INC args.  Returns the number of
 * conflicts found. */
long op2o_plan_check_colours(const op2o_plan *p, const int *const *maps, const int *map_dims,
                             const int *idxs, const int *to_sizes, const int *accs,
                             const int *inds);

/* ---------------- airfoil (airfoil/*.h, airfoil/airfoil.cpp) ---------------- */

/* Constants as the app computes them (airfoil/airfoil.cpp:175-199):
 * out = {gam, gm1, cfl, eps, mach, alpha, qinf[0..3]}.  The _f64 form is
 * the mechanical float->double variant (literals stay float). */
void op2o_airfoil_consts_f32(float out[10]);
void op2o_airfoil_consts_f64(double out[10]);

void op2o_save_soln_f32(int ncell, const float *q, float *qold);
void op2o_adt_calc_f32(int ncell, const int *pcell, const float *x, const float *q, float *adt,
                       const float *consts);
void op2o_res_calc_f32(int nedge, const int *pedge, const int *pecell, const float *x,
                       const float *q, const float *adt, float *res, const float *consts);
void op2o_bres_calc_f32(int nbedge, const int *pbedge, const int *pbecell, const float *x,
                        const float *q, const float *adt, float *res, const int *bound,
                        const float *consts);
void op2o_update_f32(int ncell, const float *qold, float *q, float *res, const float *adt,
                     float *rms);
/* niter outer iterations of airfoil/airfoil.cpp:203-258 on the given state;
 * rms_hist[iter-1] = the printed sqrt(rms/ncell). */
void op2o_airfoil_f32(int ncell, int nedge, int nbedge, const int *pcell, const int *pedge,
                      const int *pecell, const int *pbedge, const int *pbecell, const int *bound,
                      const float *x, float *q, float *qold, float *adt, float *res,
                      const float *consts, int niter, float *rms_hist);

void op2o_save_soln_f64(int ncell, const double *q, double *qold);
void op2o_adt_calc_f64(int ncell, const int *pcell, const double *x, const double *q,
                       double *adt, const double *consts);
void op2o_res_calc_f64(int nedge, const int *pedge, const int *pecell, const double *x,
                       const double *q, const double *adt, double *res, const double *consts);
void op2o_bres_calc_f64(int nbedge, const int *pbedge, const int *pbecell, const double *x,
                        const double *q, const double *adt, double *res, const int *bound,
                        const double *consts);
void op2o_update_f64(int ncell, const double *qold, double *q, double *res, const double *adt,
                     double *rms);
void op2o_airfoil_f64(int ncell, int nedge, int nbedge, const int *pcell, const int *pedge,
                      const int *pecell, const int *pbedge, const int *pbecell, const int *bound,
                      const double *x, double *q, double *qold, double *adt, double *res,
                      const double *consts, int niter, double *rms_hist);

/* ---------------- jac1 / jac2 (jac1/res.h, jac1/update.h, jac2/res.h, jac2/update.h) ---------------- */

/* jac1: A[nedge], u/du/r[nnode] floats; pp = edge->node map (dim 2). */
void op2o_jac1_res(int nedge, const int *pp, const float *A, const float *u, float *du,
                   float beta);
void op2o_jac1_update(int nnode, const float *r, float *du, float *u, float *u_sum,
                      float *u_max, float alpha);
/* jac2: A[nedge][3] double, u[nnode][2], du[nnode][3], r[nnode][2] floats. */
void op2o_jac2_res(int nedge, const int *pp, const double *A, const float *u, float *du,
                   float beta);
void op2o_jac2_update(int nnode, const float *r, float *du, float *u, float *u_sum,
                      float *u_max, float alpha);

#ifdef __cplusplus
}
#endif

#endif
