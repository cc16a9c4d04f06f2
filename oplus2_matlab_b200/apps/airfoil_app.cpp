// airfoil_app.cpp -- the airfoil application over the OP2 C API, as a
// callable function: what a user's main program does (airfoil/airfoil_op.cpp:
// 112-303), timed end to end.  Built into libop2b200_apps.so; the benchmark
// calls it for the end-to-end number (host arrays in, host results out).
//
// It declares sets, maps and datasets from the caller's host arrays (the
// device copies are made here), sets the constants the way the reference app
// computes them, runs niter outer iterations of
//   save_soln; 2 x (adt_calc, res_calc, bres_calc, update -> rms on the host)
// and fetches q back into the caller's array.

#include <math.h>
#include <stdint.h>
#include <time.h>

#include <cuda_runtime.h>

#include "op2b.h"
#include "op2b_group.h"
#include "op2b_mesh.h"
#include "op_lib.h"

extern "C" {
typedef struct {
  double t_declare;  // op_init + declarations (host -> device copies)
  double t_iterate;  // niter outer iterations (plans built in the first)
  double t_fetch;    // op_fetch_data of q
  double t_total;
  long long h2d_bytes, d2h_bytes;
} op2b_app_timing;

int op2b_airfoil_app(const op2b_mesh *m, int fp64, int niter, void *q, double *rms_hist,
                     int strategy, op2b_app_timing *t);
// the same solve at another flow condition (Mach number, alpha in degrees)
int op2b_airfoil_app_flow(const op2b_mesh *m, int fp64, int niter, double mach, double alpha_deg,
                          void *q, double *rms_hist, int strategy, op2b_app_timing *t);
// with the sets renumbered (1: Cuthill-McKee, 2: coordinate bisection)
int op2b_airfoil_app_renumbered(const op2b_mesh *m, int fp64, int niter, void *q,
                                double *rms_hist, int strategy, int renumber,
                                op2b_app_timing *t);
}

static double now() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

template <class T>
static int run(const op2b_mesh *m, int niter, double mach_d, double alpha_deg, T *q,
               double *rms_hist, op2b_app_timing *tm, int renumber = 0) {
  const char *tn = sizeof(T) == 8 ? "double" : "float";
  double t0 = now();
  // airfoil/airfoil.cpp:134-149: the constants and the free stream, with the
  // flow condition as parameters (op2b_flow_qinf; Mach 0.4, alpha 0 is the
  // reference's own)
  T qinf[4], c4[4];
  op2b_flow_qinf(mach_d, alpha_deg, sizeof(T) == 8, qinf, c4);
  T gam = c4[0], gm1 = c4[1], cfl = c4[2], eps = c4[3];
  T mach = (T)(float)mach_d, alpha = (T)((float)alpha_deg * (atanf(1.0f) / 45.0f));
  const int nc = m->ncell;
  // qold, adt, res start as the app starts them: zero
  T *qold = (T *)calloc((size_t)nc * 4, sizeof(T));
  T *adt = (T *)calloc((size_t)nc, sizeof(T));
  T *res = (T *)calloc((size_t)nc * 4, sizeof(T));
  T *x = (T *)(sizeof(T) == 8 ? (void *)m->x64 : (void *)m->x32);

  op_init(0, nullptr, 0);
  const unsigned long long h2d0 = op2b_h2d_bytes(0);
  op_set nodes = op_decl_set(m->nnode, "nodes");
  op_set edges = op_decl_set(m->nedge, "edges");
  op_set bedges = op_decl_set(m->nbedge, "bedges");
  op_set cells = op_decl_set(m->ncell, "cells");
  op_map pedge = op_decl_map(edges, nodes, 2, m->edge, "pedge");
  op_map pecell = op_decl_map(edges, cells, 2, m->ecell, "pecell");
  op_map pbedge = op_decl_map(bedges, nodes, 2, m->bedge, "pbedge");
  op_map pbecell = op_decl_map(bedges, cells, 1, m->becell, "pbecell");
  op_map pcell = op_decl_map(cells, nodes, 4, m->cell, "pcell");
  op_dat p_bound = op_decl_dat(bedges, 1, "int", m->bound, "p_bound");
  op_dat p_x = op_decl_dat(nodes, 2, tn, x, "p_x");
  op_dat p_q = op_decl_dat(cells, 4, tn, q, "p_q");
  op_dat p_qold = op_decl_dat(cells, 4, tn, qold, "p_qold");
  op_dat p_adt = op_decl_dat(cells, 1, tn, adt, "p_adt");
  op_dat p_res = op_decl_dat(cells, 4, tn, res, "p_res");
  op_decl_const2("gam", 1, tn, &gam);
  op_decl_const2("gm1", 1, tn, &gm1);
  op_decl_const2("cfl", 1, tn, &cfl);
  op_decl_const2("eps", 1, tn, &eps);
  op_decl_const2("mach", 1, tn, &mach);
  op_decl_const2("alpha", 1, tn, &alpha);
  op_decl_const2("qinf", 4, tn, qinf);
  if (renumber == 1) op2b_set_renumber(1);
  if (renumber == 2) op2b_set_renumber_coords(p_x);
  op2b_sync();
  double t1 = now();

  T rms = 0;
  for (int iter = 1; iter <= niter; iter++) {
    op_par_loop_save_soln("save_soln", cells, op_arg_dat(p_q, -1, OP_ID, 4, tn, OP_READ),
                          op_arg_dat(p_qold, -1, OP_ID, 4, tn, OP_WRITE));
    for (int k = 0; k < 2; k++) {
      op_par_loop_adt_calc("adt_calc", cells, op_arg_dat(p_x, 0, pcell, 2, tn, OP_READ),
                           op_arg_dat(p_x, 1, pcell, 2, tn, OP_READ),
                           op_arg_dat(p_x, 2, pcell, 2, tn, OP_READ),
                           op_arg_dat(p_x, 3, pcell, 2, tn, OP_READ),
                           op_arg_dat(p_q, -1, OP_ID, 4, tn, OP_READ),
                           op_arg_dat(p_adt, -1, OP_ID, 1, tn, OP_WRITE));
      op_par_loop_res_calc("res_calc", edges, op_arg_dat(p_x, 0, pedge, 2, tn, OP_READ),
                           op_arg_dat(p_x, 1, pedge, 2, tn, OP_READ),
                           op_arg_dat(p_q, 0, pecell, 4, tn, OP_READ),
                           op_arg_dat(p_q, 1, pecell, 4, tn, OP_READ),
                           op_arg_dat(p_adt, 0, pecell, 1, tn, OP_READ),
                           op_arg_dat(p_adt, 1, pecell, 1, tn, OP_READ),
                           op_arg_dat(p_res, 0, pecell, 4, tn, OP_INC),
                           op_arg_dat(p_res, 1, pecell, 4, tn, OP_INC));
      op_par_loop_bres_calc("bres_calc", bedges, op_arg_dat(p_x, 0, pbedge, 2, tn, OP_READ),
                            op_arg_dat(p_x, 1, pbedge, 2, tn, OP_READ),
                            op_arg_dat(p_q, 0, pbecell, 4, tn, OP_READ),
                            op_arg_dat(p_adt, 0, pbecell, 1, tn, OP_READ),
                            op_arg_dat(p_res, 0, pbecell, 4, tn, OP_INC),
                            op_arg_dat(p_bound, -1, OP_ID, 1, "int", OP_READ));
      rms = 0;
      op_par_loop_update("update", cells, op_arg_dat(p_qold, -1, OP_ID, 4, tn, OP_READ),
                         op_arg_dat(p_q, -1, OP_ID, 4, tn, OP_WRITE),
                         op_arg_dat(p_res, -1, OP_ID, 4, tn, OP_RW),
                         op_arg_dat(p_adt, -1, OP_ID, 1, tn, OP_READ),
                         op_arg_gbl(&rms, 1, tn, OP_INC));
    }
    rms = sqrt(rms / (T)nc);
    if (rms_hist) rms_hist[iter - 1] = (double)rms;
  }
  op2b_sync();
  double t2 = now();
  op_fetch_data(p_q);
  double t3 = now();
  const long long h2d = (long long)(op2b_h2d_bytes(0) - h2d0);
  int err = op2b_last_error()[0] != 0;
  op_exit();
  free(qold);
  free(adt);
  free(res);

  if (tm) {
    tm->t_declare = t1 - t0;
    tm->t_iterate = t2 - t1;
    tm->t_fetch = t3 - t2;
    tm->t_total = t3 - t0;
    long long sz = sizeof(T);
    // what the library copied (zero-filled arrays are cleared on the
    // device instead of copied)
    tm->h2d_bytes = h2d;
    tm->d2h_bytes = sz * 4LL * nc + sz * 2LL * niter;
  }
  return err;
}

extern "C" int op2b_airfoil_app(const op2b_mesh *m, int fp64, int niter, void *q, double *rms_hist,
                                int strategy, op2b_app_timing *t) {
  op2b_set_strategy(strategy);
  return fp64 ? run<double>(m, niter, 0.4, 0.0, (double *)q, rms_hist, t)
              : run<float>(m, niter, 0.4, 0.0, (float *)q, rms_hist, t);
}

extern "C" int op2b_airfoil_app_flow(const op2b_mesh *m, int fp64, int niter, double mach,
                                     double alpha_deg, void *q, double *rms_hist, int strategy,
                                     op2b_app_timing *t) {
  op2b_set_strategy(strategy);
  return fp64 ? run<double>(m, niter, mach, alpha_deg, (double *)q, rms_hist, t)
              : run<float>(m, niter, mach, alpha_deg, (float *)q, rms_hist, t);
}

// the same solve with the sets renumbered for locality at the first loop
// (renumber 1: Cuthill-McKee, 2: recursive coordinate bisection of the node
// coordinates); the ordering is timed with the iterations
extern "C" int op2b_airfoil_app_renumbered(const op2b_mesh *m, int fp64, int niter, void *q,
                                           double *rms_hist, int strategy, int renumber,
                                           op2b_app_timing *t) {
  if (renumber < 0 || renumber > 2) return -1;
  op2b_set_strategy(strategy);
  return fp64 ? run<double>(m, niter, 0.4, 0.0, (double *)q, rms_hist, t, renumber)
              : run<float>(m, niter, 0.4, 0.0, (float *)q, rms_hist, t, renumber);
}
