/*
 * op2_oracle.c -- CPU restatement of the reference's op_par_loop path.
 * TEST INFRASTRUCTURE ONLY (see op2_oracle.h): the checker, never the product.
 *
 * Build: oracle/Makefile (target "port"), plain C99 with -ffp-contract=off so
 * no multiply-add is contracted, as in the reference's own x86 builds.
 */
#define _DEFAULT_SOURCE
#include "op2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

enum { ACC_READ = 0, ACC_WRITE = 1, ACC_RW = 2, ACC_INC = 3 };

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* ------------------------------------------------------------------------ */
/* op_plan_core restated (common/op_lib_core.c:627-1089).  Same block        */
/* partition, same sorted/deduplicated indirect lists, same greedy thread    */
/* and block colouring in passes of 32 colours, same colour-grouped blkmap.  */
/* ------------------------------------------------------------------------ */

static int first_arg_of(int m, int nargs, const int *inds) {
  for (int a = 0; a < nargs; a++)
    if (inds[a] == m) return a;
  return -1;
}

int op2o_plan_core(int set_size, int part_size, int nargs, const int *const *maps,
                   const int *map_dims, const int *idxs, const int *to_sizes,
                   const int *dat_sizes, const int *accs, int ninds, const int *inds,
                   int cache_line_size, op2o_plan *P) {
  memset(P, 0, sizeof(*P));
  if (set_size <= 0 || nargs <= 0) return 1;

  /* block size from the 48 KB shared-memory budget (op_lib_core.c:663-673) */
  int maxbytes = 0;
  for (int m = 0; m < nargs; m++)
    if (inds[m] >= 0) maxbytes += dat_sizes[m];
  int bsize = part_size;
  if (bsize == 0) bsize = maxbytes > 0 ? (48 * 1024 / (64 * maxbytes)) * 64 : 512;
  if (bsize <= 0) return 2;
  int nblocks = (set_size - 1) / bsize + 1;

  P->set_size = set_size; P->nargs = nargs; P->ninds = ninds;
  P->bsize = bsize; P->nblocks = nblocks;
  P->nthrcol = malloc(sizeof(int) * nblocks);
  P->thrcol = malloc(sizeof(int) * set_size);
  P->offset = malloc(sizeof(int) * nblocks);
  P->nelems = malloc(sizeof(int) * nblocks);
  P->ind_offs = malloc(sizeof(int) * (size_t)nblocks * (ninds ? ninds : 1));
  P->ind_sizes = malloc(sizeof(int) * (size_t)nblocks * (ninds ? ninds : 1));
  P->nindirect = calloc(ninds ? ninds : 1, sizeof(int));
  P->ind_maps = calloc(ninds ? ninds : 1, sizeof(int *));
  P->loc_maps = calloc(nargs, sizeof(short *));
  P->blkmap = malloc(sizeof(int) * nblocks);

  unsigned **work = calloc(ninds ? ninds : 1, sizeof(unsigned *));
  for (int m = 0; m < ninds; m++) {
    int count = 0;
    for (int a = 0; a < nargs; a++) count += (inds[a] == m);
    P->ind_maps[m] = malloc(sizeof(int) * (size_t)count * set_size);
    work[m] = malloc(sizeof(unsigned) * (size_t)to_sizes[first_arg_of(m, nargs, inds)]);
  }
  for (int a = 0; a < nargs; a++)
    if (inds[a] >= 0) P->loc_maps[a] = malloc(sizeof(short) * set_size);

#define TGT(a, e) (maps[a][idxs[a] + (size_t)(e) * map_dims[a]])

  int *buf = malloc(sizeof(int) * (size_t)nargs * bsize);
  for (int b = 0; b < nblocks; b++) {
    int e0 = b * bsize, bs = set_size - e0 < bsize ? set_size - e0 : bsize;
    P->offset[b] = e0;
    P->nelems[b] = bs;

    for (int m = 0; m < ninds; m++) {
      int ne = 0;
      for (int a = 0; a < nargs; a++)
        if (inds[a] == m)
          for (int e = e0; e < e0 + bs; e++) buf[ne++] = TGT(a, e);
      qsort(buf, ne, sizeof(int), cmp_int);
      int nu = 0;
      for (int p = 0; p < ne; p++)
        if (p == 0 || buf[p] != buf[nu - 1]) buf[nu++] = buf[p];
      for (int u = 0; u < nu; u++) {
        P->ind_maps[m][P->nindirect[m]++] = buf[u];
        work[m][buf[u]] = (unsigned)u; /* inverse map: target -> local index */
      }
      for (int a = 0; a < nargs; a++)
        if (inds[a] == m)
          for (int e = e0; e < e0 + bs; e++) P->loc_maps[a][e] = (short)work[m][TGT(a, e)];
      P->ind_offs[m + b * ninds] = b == 0 ? 0 : P->ind_offs[m + (b - 1) * ninds] +
                                                     P->ind_sizes[m + (b - 1) * ninds];
      P->ind_sizes[m + b * ninds] = P->nindirect[m] - P->ind_offs[m + b * ninds];
    }

    /* greedy thread colouring in element order, 32 colours per pass */
    for (int e = e0; e < e0 + bs; e++) P->thrcol[e] = -1;
    int base = 0, ncol = 0, again = 1;
    while (again) {
      again = 0;
      for (int a = 0; a < nargs; a++)
        if (inds[a] >= 0)
          for (int e = e0; e < e0 + bs; e++) work[inds[a]][TGT(a, e)] = 0;
      for (int e = e0; e < e0 + bs; e++) {
        if (P->thrcol[e] != -1) continue;
        unsigned mask = 0;
        for (int a = 0; a < nargs; a++)
          if (inds[a] >= 0 && accs[a] == ACC_INC) mask |= work[inds[a]][TGT(a, e)];
        int c = ffs((int)~mask) - 1;
        if (c == -1) { again = 1; continue; }
        P->thrcol[e] = base + c;
        if (base + c + 1 > ncol) ncol = base + c + 1;
        for (int a = 0; a < nargs; a++)
          if (inds[a] >= 0 && accs[a] == ACC_INC) work[inds[a]][TGT(a, e)] |= 1u << c;
      }
      base += 32;
    }
    P->nthrcol[b] = ncol;
  }

  /* greedy block colouring in block order, 32 colours per pass */
  int *blk_col = malloc(sizeof(int) * nblocks);
  for (int b = 0; b < nblocks; b++) blk_col[b] = -1;
  int base = 0, ncolors = 0, again = 1;
  while (again) {
    again = 0;
    for (int a = 0; a < nargs; a++)
      if (inds[a] >= 0) memset(work[inds[a]], 0, sizeof(unsigned) * (size_t)to_sizes[a]);
    for (int b = 0; b < nblocks; b++) {
      if (blk_col[b] != -1) continue;
      int e0 = P->offset[b], bs = P->nelems[b];
      unsigned mask = 0;
      for (int a = 0; a < nargs; a++)
        if (inds[a] >= 0 && accs[a] == ACC_INC)
          for (int e = e0; e < e0 + bs; e++) mask |= work[inds[a]][TGT(a, e)];
      int c = ffs((int)~mask) - 1;
      if (c == -1) { again = 1; continue; }
      blk_col[b] = base + c;
      if (base + c + 1 > ncolors) ncolors = base + c + 1;
      for (int a = 0; a < nargs; a++)
        if (inds[a] >= 0 && accs[a] == ACC_INC)
          for (int e = e0; e < e0 + bs; e++) work[inds[a]][TGT(a, e)] |= 1u << c;
    }
    base += 32;
  }
  P->ncolors = ncolors;

  /* blocks grouped by colour, block order kept within a colour */
  P->ncolblk = calloc(ncolors ? ncolors : 1, sizeof(int));
  for (int b = 0; b < nblocks; b++) P->ncolblk[blk_col[b]]++;
  int *start = calloc(ncolors ? ncolors : 1, sizeof(int));
  for (int c = 1; c < ncolors; c++) start[c] = start[c - 1] + P->ncolblk[c - 1];
  for (int b = 0; b < nblocks; b++) P->blkmap[start[blk_col[b]]++] = b;
  free(start);
  free(blk_col);

  /* shared memory: largest per-block sum of 16-byte-rounded staging areas */
  P->nshared = 0;
  for (int b = 0; b < nblocks; b++) {
    int nbytes = 0;
    for (int m = 0; m < ninds; m++) {
      int a = first_arg_of(m, nargs, inds);
      nbytes += (P->ind_sizes[m + b * ninds] * dat_sizes[a] + 15) & ~15;
    }
    if (nbytes > P->nshared) P->nshared = nbytes;
  }

  /* byte models "transfer" (bytes used) and "transfer2" (whole cache lines),
   * op_lib_core.c:989-1056, summed exactly */
  double t1 = 0.0, t2 = 0.0;
  const double cls = (double)cache_line_size;
  for (int b = 0; b < nblocks; b++) {
    for (int a = 0; a < nargs; a++) {
      if (inds[a] < 0) {
        double fac = accs[a] == ACC_READ ? 1.0 : 2.0;
        if (dat_sizes[a] > 0) {
          t1 += fac * P->nelems[b] * dat_sizes[a];
          t2 += fac * P->nelems[b] * dat_sizes[a];
        }
      } else {
        t1 += (double)P->nelems[b] * sizeof(short);
        t2 += (double)P->nelems[b] * sizeof(short);
      }
    }
    for (int m = 0; m < ninds; m++) {
      int a = first_arg_of(m, nargs, inds);
      int sz = dat_sizes[a];
      double fac = accs[a] == ACC_READ ? 1.0 : 2.0;
      t1 += fac * P->ind_sizes[m + b * ninds] * sz;
      int u0 = P->ind_offs[m + b * ninds], u1 = u0 + P->ind_sizes[m + b * ninds];
      long l_old = -1;
      for (int u = u0; u < u1; u++) {
        long t = P->ind_maps[m][u];
        long l_new = (t * sz) / cache_line_size;
        if (l_new > l_old) t2 += fac * cls;
        l_old = l_new;
        l_new = ((t + 1) * sz - 1) / cache_line_size;
        t2 += fac * (double)(l_new - l_old) * cls;
        l_old = l_new;
      }
      fac = accs[a] == ACC_RW ? 2.0 : 1.0;
      t1 += fac * P->ind_sizes[m + b * ninds] * (double)sizeof(int);
      t2 += fac * P->ind_sizes[m + b * ninds] * (double)sizeof(int);
    }
  }
  P->transfer = t1;
  P->transfer2 = t2;

  free(buf);
  for (int m = 0; m < ninds; m++) free(work[m]);
  free(work);
#undef TGT
  return 0;
}

void op2o_plan_free(op2o_plan *P) {
  if (!P) return;
  for (int m = 0; m < P->ninds; m++) free(P->ind_maps ? P->ind_maps[m] : NULL);
  for (int a = 0; a < P->nargs; a++) free(P->loc_maps ? P->loc_maps[a] : NULL);
  free(P->nthrcol); free(P->thrcol); free(P->offset); free(P->nelems);
  free(P->ind_offs); free(P->ind_sizes); free(P->nindirect); free(P->ind_maps);
  free(P->loc_maps); free(P->ncolblk); free(P->blkmap);
  memset(P, 0, sizeof(*P));
}

/* op_plan_check restated (common/op_lib_core.c:469-620) */
int op2o_plan_check(const op2o_plan *P, const int *const *maps, const int *map_dims,
                    const int *idxs, const int *to_sizes, const int *inds) {
  int fails = 0, nblock = 0, nelem = 0;
  for (int c = 0; c < P->ncolors; c++) nblock += P->ncolblk[c];
  for (int n = 0; n < nblock; n++) nelem += P->nelems[n];
  fails += (nelem != P->set_size);

  int err = 0, tot = 0;
  for (int n = 0; n < nblock; n++) { err += (P->offset[n] != tot); tot += P->nelems[n]; }
  fails += (err != 0);

  int *seen = calloc(nblock > 0 ? (size_t)nblock : 1, sizeof(int));
  err = 0;
  for (int n = 0; n < nblock; n++) {
    int b = P->blkmap[n];
    if (b < 0 || b >= nblock || seen[b]++) err++;
  }
  free(seen);
  fails += (err != 0);

  err = 0;
  for (int m = 0; m < P->ninds; m++) {
    tot = 0;
    for (int n = 0; n < nblock; n++) {
      err += (P->ind_offs[m + n * P->ninds] != tot);
      tot += P->ind_sizes[m + n * P->ninds];
    }
  }
  fails += (err != 0);

  err = 0;
  for (int m = 0; m < P->ninds; m++) {
    int a = first_arg_of(m, P->nargs, inds);
    tot = 0;
    for (int n = 0; n < nblock; n++) {
      int last = -1;
      for (int u = tot; u < tot + P->ind_sizes[m + n * P->ninds]; u++) {
        err += (P->ind_maps[m][u] <= last);
        last = P->ind_maps[m][u];
      }
      err += (last >= to_sizes[a]);
      tot += P->ind_sizes[m + n * P->ninds];
    }
  }
  fails += (err != 0);

  err = 0;
  for (int a = 0; a < P->nargs; a++) {
    if (!maps[a] || inds[a] < 0) continue;
    int m = inds[a];
    tot = 0;
    for (int n = 0; n < nblock; n++) {
      for (int e = tot; e < tot + P->nelems[n]; e++) {
        int loc = P->loc_maps[a][e];
        int glob = P->ind_maps[m][loc + P->ind_offs[m + n * P->ninds]];
        err += (glob != maps[a][idxs[a] + (size_t)e * map_dims[a]]);
      }
      tot += P->nelems[n];
    }
  }
  fails += (err != 0);
  return fails;
}

long op2o_plan_check_colours(const op2o_plan *P, const int *const *maps, const int *map_dims,
                             const int *idxs, const int *to_sizes, const int *accs,
                             const int *inds) {
  long conflicts = 0;
  int ninds = P->ninds;
  long **tag = calloc(ninds ? ninds : 1, sizeof(long *));
  int **own = calloc(ninds ? ninds : 1, sizeof(int *));
  for (int m = 0; m < ninds; m++) {
    int a = first_arg_of(m, P->nargs, inds);
    tag[m] = malloc(sizeof(long) * (size_t)to_sizes[a]);
    own[m] = malloc(sizeof(int) * (size_t)to_sizes[a]);
    for (int t = 0; t < to_sizes[a]; t++) tag[m][t] = -1;
  }
  /* thread colours: within each block and colour, an INC target is reached
   * by one element at most */
  for (int b = 0; b < P->nblocks; b++) {
    int e0 = P->offset[b], bs = P->nelems[b];
    for (int c = 0; c < P->nthrcol[b]; c++) {
      long key = (long)b * 100000 + c;
      for (int e = e0; e < e0 + bs; e++) {
        if (P->thrcol[e] != c) continue;
        for (int a = 0; a < P->nargs; a++) {
          if (inds[a] < 0 || accs[a] != ACC_INC) continue;
          int m = inds[a], t = maps[a][idxs[a] + (size_t)e * map_dims[a]];
          if (tag[m][t] == key && own[m][t] != e) conflicts++;
          tag[m][t] = key;
          own[m][t] = e;
        }
      }
    }
    for (int e = e0; e < e0 + bs; e++)
      if (P->thrcol[e] < 0 || P->thrcol[e] >= P->nthrcol[b]) conflicts++;
  }
  /* block colours: within each colour, an INC target is reached by one
   * block at most */
  for (int m = 0; m < ninds; m++) {
    int a = first_arg_of(m, P->nargs, inds);
    for (int t = 0; t < to_sizes[a]; t++) tag[m][t] = -1;
  }
  int pos = 0;
  for (int c = 0; c < P->ncolors; c++) {
    long key = -2 - c;
    for (int k = 0; k < P->ncolblk[c]; k++, pos++) {
      int b = P->blkmap[pos];
      for (int e = P->offset[b]; e < P->offset[b] + P->nelems[b]; e++)
        for (int a = 0; a < P->nargs; a++) {
          if (inds[a] < 0 || accs[a] != ACC_INC) continue;
          int m = inds[a], t = maps[a][idxs[a] + (size_t)e * map_dims[a]];
          if (tag[m][t] == key && own[m][t] != b) conflicts++;
          tag[m][t] = key;
          own[m][t] = b;
        }
    }
  }
  for (int m = 0; m < ninds; m++) { free(tag[m]); free(own[m]); }
  free(tag);
  free(own);
  return conflicts;
}

/* ------------------------------------------------------------------------ */
/* airfoil: user kernels (airfoil/res_calc.h and siblings) and the app's outer loop             */
/* (airfoil/airfoil.cpp:175-258), stated once for REAL = float / double.    */
/* Expression trees follow the reference term for term: no reassociation.  */
/* ------------------------------------------------------------------------ */

void op2o_airfoil_consts_f32(float out[10]) {
  float gam = 1.4f, gm1 = gam - 1.0f, cfl = 0.9f, eps = 0.05f;
  float mach = 0.4f, alpha = 3.0f * atanf(1.0f) / 45.0f, p = 1.0f, r = 1.0f;
  float u = sqrtf(gam * p / r) * mach;
  float e = p / (r * gm1) + 0.5f * u * u;
  out[0] = gam; out[1] = gm1; out[2] = cfl; out[3] = eps; out[4] = mach; out[5] = alpha;
  out[6] = r; out[7] = r * u; out[8] = 0.0f; out[9] = r * e;
}

/* the float->double variant keeps the float literals (airfoil.cpp:175-186) */
void op2o_airfoil_consts_f64(double out[10]) {
  double gam = 1.4f, gm1 = gam - 1.0f, cfl = 0.9f, eps = 0.05f;
  double mach = 0.4f, alpha = 3.0f * atanf(1.0f) / 45.0f, p = 1.0f, r = 1.0f;
  double u = sqrt(gam * p / r) * mach;
  double e = p / (r * gm1) + 0.5f * u * u;
  out[0] = gam; out[1] = gm1; out[2] = cfl; out[3] = eps; out[4] = mach; out[5] = alpha;
  out[6] = r; out[7] = r * u; out[8] = 0.0f; out[9] = r * e;
}

#define AIRFOIL_ORACLE(SUF, REAL, SQRT, FABS)                                                   \
  static void k_adt_##SUF(const REAL *x1, const REAL *x2, const REAL *x3, const REAL *x4,        \
                          const REAL *q, REAL *adt, const REAL *K) {                             \
    REAL gam = K[0], gm1 = K[1], cfl = K[2];                                                     \
    REAL dx, dy, ri, u, v, c;                                                                    \
    ri = 1.0f / q[0];                                                                            \
    u = ri * q[1];                                                                               \
    v = ri * q[2];                                                                               \
    c = SQRT(gam * gm1 * (ri * q[3] - 0.5f * (u * u + v * v)));                                  \
    dx = x2[0] - x1[0]; dy = x2[1] - x1[1];                                                      \
    *adt = FABS(u * dy - v * dx) + c * SQRT(dx * dx + dy * dy);                                  \
    dx = x3[0] - x2[0]; dy = x3[1] - x2[1];                                                      \
    *adt += FABS(u * dy - v * dx) + c * SQRT(dx * dx + dy * dy);                                 \
    dx = x4[0] - x3[0]; dy = x4[1] - x3[1];                                                      \
    *adt += FABS(u * dy - v * dx) + c * SQRT(dx * dx + dy * dy);                                 \
    dx = x1[0] - x4[0]; dy = x1[1] - x4[1];                                                      \
    *adt += FABS(u * dy - v * dx) + c * SQRT(dx * dx + dy * dy);                                 \
    *adt = (*adt) / cfl;                                                                         \
  }                                                                                              \
  static void k_res_##SUF(const REAL *x1, const REAL *x2, const REAL *q1, const REAL *q2,        \
                          const REAL *adt1, const REAL *adt2, REAL *res1, REAL *res2,            \
                          const REAL *K) {                                                       \
    REAL gm1 = K[1], eps = K[3];                                                                 \
    REAL dx, dy, mu, ri, p1, vol1, p2, vol2, f;                                                  \
    dx = x1[0] - x2[0];                                                                          \
    dy = x1[1] - x2[1];                                                                          \
    ri = 1.0f / q1[0];                                                                           \
    p1 = gm1 * (q1[3] - 0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));                            \
    vol1 = ri * (q1[1] * dy - q1[2] * dx);                                                       \
    ri = 1.0f / q2[0];                                                                           \
    p2 = gm1 * (q2[3] - 0.5f * ri * (q2[1] * q2[1] + q2[2] * q2[2]));                            \
    vol2 = ri * (q2[1] * dy - q2[2] * dx);                                                       \
    mu = 0.5f * ((*adt1) + (*adt2)) * eps;                                                       \
    f = 0.5f * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]);                             \
    res1[0] += f; res2[0] -= f;                                                                  \
    f = 0.5f * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) + mu * (q1[1] - q2[1]);         \
    res1[1] += f; res2[1] -= f;                                                                  \
    f = 0.5f * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) + mu * (q1[2] - q2[2]);         \
    res1[2] += f; res2[2] -= f;                                                                  \
    f = 0.5f * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) + mu * (q1[3] - q2[3]);               \
    res1[3] += f; res2[3] -= f;                                                                  \
  }                                                                                              \
  static void k_bres_##SUF(const REAL *x1, const REAL *x2, const REAL *q1, const REAL *adt1,     \
                           REAL *res1, const int *bound, const REAL *K) {                        \
    REAL gm1 = K[1], eps = K[3];                                                                 \
    const REAL *qinf = K + 6;                                                                    \
    REAL dx, dy, mu, ri, p1, vol1, p2, vol2, f;                                                  \
    dx = x1[0] - x2[0];                                                                          \
    dy = x1[1] - x2[1];                                                                          \
    ri = 1.0f / q1[0];                                                                           \
    p1 = gm1 * (q1[3] - 0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));                            \
    if (*bound == 1) {                                                                           \
      res1[1] += +p1 * dy;                                                                       \
      res1[2] += -p1 * dx;                                                                       \
    } else {                                                                                     \
      vol1 = ri * (q1[1] * dy - q1[2] * dx);                                                     \
      ri = 1.0f / qinf[0];                                                                       \
      p2 = gm1 * (qinf[3] - 0.5f * ri * (qinf[1] * qinf[1] + qinf[2] * qinf[2]));                \
      vol2 = ri * (qinf[1] * dy - qinf[2] * dx);                                                 \
      mu = (*adt1) * eps;                                                                        \
      f = 0.5f * (vol1 * q1[0] + vol2 * qinf[0]) + mu * (q1[0] - qinf[0]);                       \
      res1[0] += f;                                                                              \
      f = 0.5f * (vol1 * q1[1] + p1 * dy + vol2 * qinf[1] + p2 * dy) + mu * (q1[1] - qinf[1]);   \
      res1[1] += f;                                                                              \
      f = 0.5f * (vol1 * q1[2] - p1 * dx + vol2 * qinf[2] - p2 * dx) + mu * (q1[2] - qinf[2]);   \
      res1[2] += f;                                                                              \
      f = 0.5f * (vol1 * (q1[3] + p1) + vol2 * (qinf[3] + p2)) + mu * (q1[3] - qinf[3]);         \
      res1[3] += f;                                                                              \
    }                                                                                            \
  }                                                                                              \
  static void k_update_##SUF(const REAL *qold, REAL *q, REAL *res, const REAL *adt, REAL *rms) { \
    REAL del, adti;                                                                              \
    adti = 1.0f / (*adt);                                                                        \
    for (int n = 0; n < 4; n++) {                                                                \
      del = adti * res[n];                                                                       \
      q[n] = qold[n] - del;                                                                      \
      res[n] = 0.0f;                                                                             \
      *rms += del * del;                                                                         \
    }                                                                                            \
  }                                                                                              \
  void op2o_save_soln_##SUF(int ncell, const REAL *q, REAL *qold) {                             \
    for (int c = 0; c < ncell; c++)                                                              \
      for (int n = 0; n < 4; n++) qold[4 * (size_t)c + n] = q[4 * (size_t)c + n];                \
  }                                                                                              \
  void op2o_adt_calc_##SUF(int ncell, const int *pcell, const REAL *x, const REAL *q, REAL *adt, \
                           const REAL *K) {                                                      \
    for (int c = 0; c < ncell; c++) {                                                            \
      const int *pc = pcell + 4 * (size_t)c;                                                     \
      k_adt_##SUF(x + 2 * (size_t)pc[0], x + 2 * (size_t)pc[1], x + 2 * (size_t)pc[2],           \
                  x + 2 * (size_t)pc[3], q + 4 * (size_t)c, adt + c, K);                         \
    }                                                                                            \
  }                                                                                              \
  void op2o_res_calc_##SUF(int nedge, const int *pedge, const int *pecell, const REAL *x,       \
                           const REAL *q, const REAL *adt, REAL *res, const REAL *K) {           \
    for (int e = 0; e < nedge; e++) {                                                            \
      int n1 = pedge[2 * (size_t)e], n2 = pedge[2 * (size_t)e + 1];                              \
      int c1 = pecell[2 * (size_t)e], c2 = pecell[2 * (size_t)e + 1];                            \
      k_res_##SUF(x + 2 * (size_t)n1, x + 2 * (size_t)n2, q + 4 * (size_t)c1,                    \
                  q + 4 * (size_t)c2, adt + c1, adt + c2, res + 4 * (size_t)c1,                  \
                  res + 4 * (size_t)c2, K);                                                      \
    }                                                                                            \
  }                                                                                              \
  void op2o_bres_calc_##SUF(int nbedge, const int *pbedge, const int *pbecell, const REAL *x,   \
                            const REAL *q, const REAL *adt, REAL *res, const int *bound,         \
                            const REAL *K) {                                                     \
    for (int e = 0; e < nbedge; e++) {                                                           \
      int n1 = pbedge[2 * (size_t)e], n2 = pbedge[2 * (size_t)e + 1], c1 = pbecell[e];           \
      k_bres_##SUF(x + 2 * (size_t)n1, x + 2 * (size_t)n2, q + 4 * (size_t)c1, adt + c1,         \
                   res + 4 * (size_t)c1, bound + e, K);                                          \
    }                                                                                            \
  }                                                                                              \
  void op2o_update_##SUF(int ncell, const REAL *qold, REAL *q, REAL *res, const REAL *adt,      \
                         REAL *rms) {                                                            \
    for (int c = 0; c < ncell; c++)                                                              \
      k_update_##SUF(qold + 4 * (size_t)c, q + 4 * (size_t)c, res + 4 * (size_t)c, adt + c,      \
                     rms);                                                                       \
  }                                                                                              \
  void op2o_airfoil_##SUF(int ncell, int nedge, int nbedge, const int *pcell, const int *pedge, \
                          const int *pecell, const int *pbedge, const int *pbecell,              \
                          const int *bound, const REAL *x, REAL *q, REAL *qold, REAL *adt,       \
                          REAL *res, const REAL *K, int niter, REAL *rms_hist) {                 \
    for (int iter = 1; iter <= niter; iter++) {                                                  \
      REAL rms = 0.0f;                                                                           \
      op2o_save_soln_##SUF(ncell, q, qold);                                                      \
      for (int k = 0; k < 2; k++) {                                                              \
        op2o_adt_calc_##SUF(ncell, pcell, x, q, adt, K);                                         \
        op2o_res_calc_##SUF(nedge, pedge, pecell, x, q, adt, res, K);                            \
        op2o_bres_calc_##SUF(nbedge, pbedge, pbecell, x, q, adt, res, bound, K);                 \
        rms = 0.0f;                                                                              \
        op2o_update_##SUF(ncell, qold, q, res, adt, &rms);                                       \
      }                                                                                          \
      rms = SQRT(rms / (REAL)ncell);                                                             \
      if (rms_hist) rms_hist[iter - 1] = rms;                                                    \
    }                                                                                            \
  }

AIRFOIL_ORACLE(f32, float, sqrtf, fabsf)
AIRFOIL_ORACLE(f64, double, sqrt, fabs)

/* ------------------------------------------------------------------------ */
/* jac1 / jac2 (jac1/res.h, jac1/update.h, jac2 likewise; loops of jac1/jac.cpp:147-163) */
/* ------------------------------------------------------------------------ */

void op2o_jac1_res(int nedge, const int *pp, const float *A, const float *u, float *du,
                   float beta) {
  for (int e = 0; e < nedge; e++) {
    float *d = du + pp[2 * (size_t)e];
    *d += beta * A[e] * u[pp[2 * (size_t)e + 1]];
  }
}

void op2o_jac1_update(int nnode, const float *r, float *du, float *u, float *u_sum,
                      float *u_max, float alpha) {
  for (int n = 0; n < nnode; n++) {
    u[n] += du[n] + alpha * r[n];
    du[n] = 0.0f;
    *u_sum += u[n] * u[n];
    *u_max = (*u_max > u[n]) ? *u_max : u[n];
  }
}

void op2o_jac2_res(int nedge, const int *pp, const double *A, const float *u, float *du,
                   float beta) {
  for (int e = 0; e < nedge; e++) {
    float *d = du + 3 * (size_t)pp[2 * (size_t)e];
    *d += (double)beta * A[3 * (size_t)e] * (double)u[2 * (size_t)pp[2 * (size_t)e + 1]];
  }
}

void op2o_jac2_update(int nnode, const float *r, float *du, float *u, float *u_sum,
                      float *u_max, float alpha) {
  for (int n = 0; n < nnode; n++) {
    float *un = u + 2 * (size_t)n, *dn = du + 3 * (size_t)n;
    *un += *dn + alpha * r[2 * (size_t)n];
    *dn = 0.0f;
    *u_sum += (*un) * (*un);
    *u_max = (*u_max > *un) ? *u_max : *un;
  }
}
