// jac_app.cpp -- the jac1 application over the OP2 C API, as a callable
// function: what the reference's generated main does (jac1/jac_op.cpp:143-190)
// with the grid passed in, timed end to end.  Built into
// libop2b200_apps.so; the benchmark calls it for jac1's end-to-end number
// (host arrays in, u out, u_max and u_sum returned to the host after every
// update as the reference's loop prints them).

#include <math.h>
#include <stdlib.h>
#include <time.h>

#include "op2b.h"
#include "op_lib.h"

extern "C" {
typedef struct {
  double t_declare;  // op_init + declarations (host -> device copies)
  double t_iterate;  // niter iterations (plans built in the first)
  double t_fetch;    // op_fetch_data of u
  double t_total;
  long long h2d_bytes, d2h_bytes;
} op2b_app_timing;

int op2b_jac1_app(int nnode, int nedge, const int *pp, const float *A, const float *r,
                  int niter, float *u, double *u_max_hist, double *u_rms_hist,
                  op2b_app_timing *t);
}

static double now() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

extern "C" int op2b_jac1_app(int nnode, int nedge, const int *pp, const float *A, const float *r,
                             int niter, float *u, double *u_max_hist, double *u_rms_hist,
                             op2b_app_timing *tm) {
  if (nnode <= 0 || nedge <= 0 || !pp || !A || !r || !u || niter < 0) return -1;
  const double t0 = now();
  // u and du start at zero (jac1/jac_op.cpp:110-113); u is the caller's array
  float *du = (float *)calloc((size_t)nnode, sizeof(float));
  for (int n = 0; n < nnode; n++) u[n] = 0.0f;

  op_init(0, nullptr, 0);
  const unsigned long long h2d0 = op2b_h2d_bytes(0);
  op_set nodes = op_decl_set(nnode, "nodes");
  op_set edges = op_decl_set(nedge, "edges");
  op_map ppedge = op_decl_map(edges, nodes, 2, (int *)pp, "ppedge");
  op_dat p_A = op_decl_dat(edges, 1, "float", (float *)A, "p_A");
  op_dat p_r = op_decl_dat(nodes, 1, "float", (float *)r, "p_r");
  op_dat p_u = op_decl_dat(nodes, 1, "float", u, "p_u");
  op_dat p_du = op_decl_dat(nodes, 1, "float", du, "p_du");
  float alpha = 1.0f;
  op_decl_const2("alpha", 1, "float", &alpha);
  op2b_sync();
  const double t1 = now();

  // jac1/jac_op.cpp:166-183
  float u_sum, u_max, beta = 1.0f;
  for (int iter = 0; iter < niter; iter++) {
    op_par_loop_res("res", edges, op_arg_dat(p_A, -1, OP_ID, 1, "float", OP_READ),
                    op_arg_dat(p_u, 1, ppedge, 1, "float", OP_READ),
                    op_arg_dat(p_du, 0, ppedge, 1, "float", OP_INC),
                    op_arg_gbl(&beta, 1, "float", OP_READ));
    u_sum = 0.0f;
    u_max = 0.0f;
    op_par_loop_update("update", nodes, op_arg_dat(p_r, -1, OP_ID, 1, "float", OP_READ),
                       op_arg_dat(p_du, -1, OP_ID, 1, "float", OP_RW),
                       op_arg_dat(p_u, -1, OP_ID, 1, "float", OP_INC),
                       op_arg_gbl(&u_sum, 1, "float", OP_INC),
                       op_arg_gbl(&u_max, 1, "float", OP_MAX));
    if (u_max_hist) u_max_hist[iter] = (double)u_max;
    if (u_rms_hist) u_rms_hist[iter] = (double)sqrtf(u_sum / (float)nnode);
  }
  op2b_sync();
  const double t2 = now();
  op_fetch_data(p_u);
  const double t3 = now();
  const long long h2d = (long long)(op2b_h2d_bytes(0) - h2d0);
  const int err = op2b_last_error()[0] != 0;
  op_exit();
  free(du);
  if (tm) {
    tm->t_declare = t1 - t0;
    tm->t_iterate = t2 - t1;
    tm->t_fetch = t3 - t2;
    tm->t_total = t3 - t0;
    tm->h2d_bytes = h2d;  // what the library copied
    tm->d2h_bytes = 4LL * nnode + 8LL * niter;
  }
  return err;
}
