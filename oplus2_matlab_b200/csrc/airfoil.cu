// airfoil.cu -- the five parallel loops of the airfoil app, as hand-written
// sm_100a kernels (FP32 and FP64), replacing the generated
// airfoil/{save_soln,adt_calc,res_calc,bres_calc,update}_kernel.cu.
//
// The user-kernel arithmetic (airfoil/*.h) is restated term for term in the
// reference's evaluation order; the library is compiled with -fmad=false and
// IEEE division / square root, so every per-element value is bit-identical
// to the reference's x86 build.
//
// Indirect loops with OP_INC (res_calc, bres_calc) have two executions:
//  GATHER   one thread per incremented cell walks that cell's contributions
//           in ascending (edge, argument) order -- op_seq.h's order -- and
//           writes the cell once: bit-identical to the sequential reference,
//           no colouring, no atomics, one launch.
//  COLOURED the reference's two-level scheme on the device plan: a CTA per
//           block stages x, q, adt of its distinct targets in shared memory,
//           applies increments in thread-colour order, and adds its block
//           increment to res once; block colours are separate launches.

#include <string.h>

#include <algorithm>
#include <type_traits>

#include "airfoil_math.cuh"
#include "tile_chain.cuh"
#include "launch.cuh"
#include "loops.h"
#include "reduce.cuh"
#include "tma.cuh"

namespace op2b {

__device__ __forceinline__ int at(const IdxMap &m, int e) {
  return m.map ? __ldg(m.map + m.idx + (size_t)e * m.dim) : e;
}

// ------------------------------------------------------------- kernels ----

// Two map entries of one element.  When both args use one map of dim 2 with
// idx 0 and 1 (pedge, pecell, pbedge) this is a single 8-byte load.
__device__ __forceinline__ void at2(const IdxMap &a, const IdxMap &b, int e, int &i, int &j) {
  if (a.map && a.map == b.map && a.dim == 2 && a.idx == 0 && b.idx == 1) {
    int2 v = __ldg(reinterpret_cast<const int2 *>(a.map) + e);
    i = v.x;
    j = v.y;
  } else {
    i = at(a, e);
    j = at(b, e);
  }
}

// save_soln: qold = q, U elements per thread issued before any store
template <class T, int U>
__global__ void k_save_soln(int n, const T *__restrict__ q, T *__restrict__ qold) {
  pdl_wait();
  pdl_trigger();
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += stride * U) {
    T v[U][4];
#pragma unroll
    for (int u = 0; u < U; u++) {
      int c = base + u * stride;
      if (c < n) ld4(q + 4 * (size_t)c, v[u]);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      int c = base + u * stride;
      if (c < n) st4(qold + 4 * (size_t)c, v[u]);
    }
  }
}

// adt_calc: direct over cells, x gathered through pcell (one 16-byte load
// of the 4 node indices when the four args share a dim-4 map in order)
template <class T, int U>
__global__ void k_adt_calc(int n, IdxMap m0, IdxMap m1, IdxMap m2, IdxMap m3, IdxMap mq,
                           const T *__restrict__ x0, const T *__restrict__ x1,
                           const T *__restrict__ x2, const T *__restrict__ x3,
                           const T *__restrict__ q, T *__restrict__ adt, AirConsts<T> K) {
  const bool quad = m0.map && m0.map == m1.map && m0.map == m2.map && m0.map == m3.map &&
                    m0.dim == 4 && m0.idx == 0 && m1.idx == 1 && m2.idx == 2 && m3.idx == 3;
  const int stride = gridDim.x * blockDim.x;
  int nd[U][4];
  auto nodes = [&](int base) {
#pragma unroll
    for (int u = 0; u < U; u++) {  // node indices of U cells
      const int c = base + u * stride;
      if (c >= n) continue;
      if (quad) {
        int4 v = __ldg(reinterpret_cast<const int4 *>(m0.map) + c);
        nd[u][0] = v.x; nd[u][1] = v.y; nd[u][2] = v.z; nd[u][3] = v.w;
      } else {
        nd[u][0] = at(m0, c); nd[u][1] = at(m1, c); nd[u][2] = at(m2, c); nd[u][3] = at(m3, c);
      }
    }
  };
  const int base0 = blockIdx.x * blockDim.x + threadIdx.x;
  nodes(base0);  // map entries: read-only, fetched before the wait
  pdl_wait();
  pdl_trigger();
  for (int base = base0; base < n; base += stride * U) {
    if (base != base0) nodes(base);
    T xs[U][4][2], qq[U][4];
#pragma unroll
    for (int u = 0; u < U; u++) {  // then every gather of the U cells
      const int c = base + u * stride;
      if (c >= n) continue;
      ld4(q + 4 * (size_t)at(mq, c), qq[u]);
      ld2(x0 + 2 * (size_t)nd[u][0], xs[u][0]);
      ld2(x1 + 2 * (size_t)nd[u][1], xs[u][1]);
      ld2(x2 + 2 * (size_t)nd[u][2], xs[u][2]);
      ld2(x3 + 2 * (size_t)nd[u][3], xs[u][3]);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int c = base + u * stride;
      if (c < n) adt[c] = adt_calc(xs[u][0], xs[u][1], xs[u][2], xs[u][3], qq[u], K);
    }
  }
}

// res_calc, GATHER, contribution-parallel: CTA b owns the cells whose first
// contribution lies in [kTile*b, kTile*(b+1)).  Each thread computes the
// flux of one (edge, side) contribution into shared memory (negated for the
// second cell of the edge); then one thread per owned cell folds its
// contributions in ascending order -- op_seq.h's order -- onto res.
constexpr int kTileExtra = 64;  // contributions past the tile end (max row - 1)

template <class T>
__global__ void __launch_bounds__(kTile) k_res_calc_tiled(
    const int *__restrict__ tile_first, const int *__restrict__ active,
    const int *__restrict__ row, const int *__restrict__ keys, IdxMap mx1, IdxMap mx2,
    IdxMap mq1, IdxMap mq2, IdxMap ma1, IdxMap ma2, const T *__restrict__ xa,
    const T *__restrict__ xb, const T *__restrict__ qa, const T *__restrict__ qb,
    const T *__restrict__ adta, const T *__restrict__ adtb, T *__restrict__ res, T gm1, T eps) {
  __shared__ __align__(16) T fl[(kTile + kTileExtra) * 4];
  const int t0 = tile_first[blockIdx.x], t1 = tile_first[blockIdx.x + 1];
  if (t0 == t1) return;
  const int e0 = row[t0], e1 = row[t1];
  const int j = threadIdx.x;
  const bool owner = j < t1 - t0;
  int c = 0, k0 = 0, k1 = 0;
  T r[4];
  if (owner) {  // start the owner's reads early
    c = active ? active[t0 + j] : t0 + j;
    k0 = row[t0 + j];
    k1 = row[t0 + j + 1];
    ldw4(res + 4 * (size_t)c, r);
  }
  const bool same_cells = mq1.map == ma1.map && mq1.idx == ma1.idx && mq2.map == ma2.map &&
                          mq2.idx == ma2.idx && mq1.dim == ma1.dim && mq2.dim == ma2.dim;
  for (int i = e0 + j; i < e1; i += kTile) {
    const int key = __ldg(keys + i);
    const int e = key >> 1;
    int n1, n2, c1, c2, a1, a2;
    at2(mx1, mx2, e, n1, n2);
    at2(mq1, mq2, e, c1, c2);
    if (same_cells) {
      a1 = c1;
      a2 = c2;
    } else {
      at2(ma1, ma2, e, a1, a2);
    }
    T p[2], s[2], q1[4], q2[4], f[4];
    ld4(qa + 4 * (size_t)c1, q1);
    ld4(qb + 4 * (size_t)c2, q2);
    ld2(xa + 2 * (size_t)n1, p);
    ld2(xb + 2 * (size_t)n2, s);
    const T ad1 = __ldg(adta + a1), ad2 = __ldg(adtb + a2);
    res_flux(p, s, q1, q2, ad1, ad2, gm1, eps, f);
    if (key & 1) {
      f[0] = -f[0]; f[1] = -f[1]; f[2] = -f[2]; f[3] = -f[3];
    }
    st4(fl + 4 * (i - e0), f);
  }
  __syncthreads();
  if (owner) {
    for (int k = k0; k < k1; k++) {
      const T *g = fl + 4 * (k - e0);
      r[0] += g[0]; r[1] += g[1]; r[2] += g[2]; r[3] += g[3];
    }
    st4(res + 4 * (size_t)c, r);
  }
}

// res_calc, GATHER: one thread per incremented cell
template <class T, int BATCH>
__global__ void k_res_calc_gather(int nrows, const int *__restrict__ active,
                                  const int *__restrict__ row, const int *__restrict__ keys,
                                  IdxMap mx1, IdxMap mx2, IdxMap mq1, IdxMap mq2, IdxMap ma1,
                                  IdxMap ma2, const T *__restrict__ xa, const T *__restrict__ xb,
                                  const T *__restrict__ qa, const T *__restrict__ qb,
                                  const T *__restrict__ adta, const T *__restrict__ adtb,
                                  T *__restrict__ res, T gm1, T eps) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows) return;
  int c = active ? active[t] : t;
  T r[4];
  ldw4(res + 4 * (size_t)c, r);
  const int k1 = row[t + 1];
  const bool same_cells = mq1.map == ma1.map && mq1.idx == ma1.idx && mq2.map == ma2.map &&
                          mq2.idx == ma2.idx && mq1.dim == ma1.dim && mq2.dim == ma2.dim;
  // contributions in batches of B: every load of a batch is issued before
  // any flux is computed (B = 1: one edge at a time, fewest registers --
  // the fastest on the 720k airfoil mesh; B = 4: one chain of dependent
  // loads per cell instead of per edge, at the cost of occupancy)
  constexpr int B = BATCH;
  for (int kb = row[t]; kb < k1; kb += B) {
    int key[B], n1[B], n2[B], c1[B], c2[B], a1[B], a2[B];
#pragma unroll
    for (int b = 0; b < B; b++) key[b] = kb + b < k1 ? __ldg(keys + kb + b) : -2;
#pragma unroll
    for (int b = 0; b < B; b++) {
      if (key[b] < 0) continue;
      const int e = key[b] >> 1;
      at2(mx1, mx2, e, n1[b], n2[b]);
      at2(mq1, mq2, e, c1[b], c2[b]);
      if (same_cells) {
        a1[b] = c1[b];
        a2[b] = c2[b];
      } else {
        at2(ma1, ma2, e, a1[b], a2[b]);
      }
    }
    T p[B][2], s[B][2], q1[B][4], q2[B][4], d1[B], d2[B];
#pragma unroll
    for (int b = 0; b < B; b++) {
      if (key[b] < 0) continue;
      ld4(qa + 4 * (size_t)c1[b], q1[b]);
      ld4(qb + 4 * (size_t)c2[b], q2[b]);
      ld2(xa + 2 * (size_t)n1[b], p[b]);
      ld2(xb + 2 * (size_t)n2[b], s[b]);
      d1[b] = __ldg(adta + a1[b]);
      d2[b] = __ldg(adtb + a2[b]);
    }
#pragma unroll
    for (int b = 0; b < B; b++) {  // ascending order: op_seq.h's order
      if (key[b] < 0) continue;
      T f[4];
      res_flux(p[b], s[b], q1[b], q2[b], d1[b], d2[b], gm1, eps, f);
      if ((key[b] & 1) == 0) {
        r[0] += f[0]; r[1] += f[1]; r[2] += f[2]; r[3] += f[3];
      } else {
        r[0] -= f[0]; r[1] -= f[1]; r[2] -= f[2]; r[3] -= f[3];
      }
    }
  }
  st4(res + 4 * (size_t)c, r);
}

// res_calc, GATHER in two passes.  Pass 1, one thread per edge in edge
// order (coalesced map reads): the flux f of airfoil/res_calc.h, computed
// once, into flux[e].  Pass 2, one thread per cell: fold +f (first cell of
// the edge) or -f (second cell) in ascending edge order onto res -- the
// order of op_seq.h, so still bit-identical.  The flux buffer (16 B per
// edge in FP32) is written and re-read while it sits in L2.
template <class T>
__global__ void k_res_flux(int nedge, IdxMap mx1, IdxMap mx2, IdxMap mq1, IdxMap mq2,
                           IdxMap ma1, IdxMap ma2, const T *__restrict__ xa,
                           const T *__restrict__ xb, const T *__restrict__ qa,
                           const T *__restrict__ qb, const T *__restrict__ adta,
                           const T *__restrict__ adtb, T *__restrict__ flux, T gm1, T eps) {
  const bool same_cells = mq1.map == ma1.map && mq1.idx == ma1.idx && mq2.map == ma2.map &&
                          mq2.idx == ma2.idx && mq1.dim == ma1.dim && mq2.dim == ma2.dim;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nedge; e += gridDim.x * blockDim.x) {
    int n1, n2, c1, c2, a1, a2;
    at2(mx1, mx2, e, n1, n2);
    at2(mq1, mq2, e, c1, c2);
    if (same_cells) {
      a1 = c1;
      a2 = c2;
    } else {
      at2(ma1, ma2, e, a1, a2);
    }
    T p[2], s[2], q1[4], q2[4], f[4];
    ld4(qa + 4 * (size_t)c1, q1);
    ld4(qb + 4 * (size_t)c2, q2);
    ld2(xa + 2 * (size_t)n1, p);
    ld2(xb + 2 * (size_t)n2, s);
    const T d1 = __ldg(adta + a1), d2 = __ldg(adtb + a2);
    res_flux(p, s, q1, q2, d1, d2, gm1, eps, f);
    st4(flux + 4 * (size_t)e, f);
  }
}

template <class T>
__global__ void k_res_fold(int nrows, const int *__restrict__ active, const int *__restrict__ row,
                           const int *__restrict__ keys, const T *__restrict__ flux,
                           T *__restrict__ res) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows) return;
  const int c = active ? active[t] : t;
  T r[4];
  ldw4(res + 4 * (size_t)c, r);
  const int k1 = row[t + 1];
  constexpr int B = 4;  // keys, then fluxes, of up to B contributions in flight
  for (int kb = row[t]; kb < k1; kb += B) {
    int key[B];
    T f[B][4];
#pragma unroll
    for (int b = 0; b < B; b++) key[b] = kb + b < k1 ? __ldg(keys + kb + b) : -1;
#pragma unroll
    for (int b = 0; b < B; b++)
      if (key[b] >= 0) ld4(flux + 4 * (size_t)(key[b] >> 1), f[b]);
#pragma unroll
    for (int b = 0; b < B; b++) {
      if (key[b] < 0) continue;
      if ((key[b] & 1) == 0) {
        r[0] += f[b][0]; r[1] += f[b][1]; r[2] += f[b][2]; r[3] += f[b][3];
      } else {
        r[0] -= f[b][0]; r[1] -= f[b][1]; r[2] -= f[b][2]; r[3] -= f[b][3];
      }
    }
  }
  st4(res + 4 * (size_t)c, r);
}

// ------------------------------------------------- list-ordered res_calc --
// res_calc (and bres_calc after it) in two passes over fixed-width
// contribution lists (SlotPlan).  Pass 1, one thread per edge in edge order
// (coalesced map reads and stores): the flux f of airfoil/res_calc.h,
// computed once, into v[e]; one thread per boundary edge: the increment
// bres_calc adds to its cell, into v[nedge + b].  Pass 2, a direct loop over
// cells: one load of the cell's list, then its values added in list order
// (negated for the second cell of an edge) onto res -- the order of
// op_seq.h running res_calc then bres_calc, so bit-identical.  v is written
// and re-read while it sits in L2.

template <class T>
struct ResEdges {  // res_calc's arguments (airfoil/airfoil_op.cpp:259-267)
  int n;
  IdxMap x1, x2, q1, q2, a1, a2;
  const T *xa, *xb, *qa, *qb, *adta, *adtb;
};
template <class T>
struct BresEdges {  // bres_calc's arguments (airfoil/airfoil_op.cpp:269-276)
  int n;  // 0: no bres_calc in this pass
  IdxMap x1, x2, q, a, bound;
  const T *xa, *xb, *q_d, *adt;
  const int *bound_d;
};

__device__ __forceinline__ bool same_map(const IdxMap &a, const IdxMap &b) {
  return a.map == b.map && a.idx == b.idx && a.dim == b.dim;
}

// PIPE: fetch the next edge's map entries while this edge gathers (more
// registers: MINB 6 CTAs per SM instead of 8)
template <class T, bool PIPE, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_res_flux_list(ResEdges<T> E, BresEdges<T> B, T *__restrict__ v, AirConsts<T> K) {
  const bool same_a = same_map(E.q1, E.a1) && same_map(E.q2, E.a2);
  const int total = E.n + B.n;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  // map entries of this thread's first edge: read-only, fetched before the
  // previous kernel has finished
  // map entries of an edge (read-only): the first edge's are fetched before
  // the previous kernel has finished, the next edge's while this one gathers
  int m[6] = {0, 0, 0, 0, 0, 0}, mn[6] = {0, 0, 0, 0, 0, 0};
  auto edge_maps = [&](int e, int (&o)[6]) {
    if (e >= E.n) return;
    at2(E.x1, E.x2, e, o[0], o[1]);
    at2(E.q1, E.q2, e, o[2], o[3]);
    if (same_a) {
      o[4] = o[2]; o[5] = o[3];
    } else {
      at2(E.a1, E.a2, e, o[4], o[5]);
    }
  };
  edge_maps(i0, m);
  pdl_wait();
  pdl_trigger();
  const int stride = gridDim.x * blockDim.x;
  for (int i = i0; i < total; i += stride) {
    T f[4];
    if (i < E.n) {
      T p[2], s[2], q1[4], q2[4];
      ld4(E.qa + 4 * (size_t)m[2], q1);
      ld4(E.qb + 4 * (size_t)m[3], q2);
      ld2(E.xa + 2 * (size_t)m[0], p);
      ld2(E.xb + 2 * (size_t)m[1], s);
      const T d1 = __ldg(E.adta + m[4]), d2 = __ldg(E.adtb + m[5]);
      if (PIPE) {
        edge_maps(i + stride, mn);
#pragma unroll
        for (int j = 0; j < 6; j++) m[j] = mn[j];
      }
      res_flux(p, s, q1, q2, d1, d2, K.gm1, K.eps, f);
      if (!PIPE) edge_maps(i + stride, m);
    } else {
      const int b = i - E.n;
      int m1, m2;
      at2(B.x1, B.x2, b, m1, m2);
      T p[2], s[2], q1[4];
      ld2(B.xa + 2 * (size_t)m1, p);
      ld2(B.xb + 2 * (size_t)m2, s);
      ld4(B.q_d + 4 * (size_t)at(B.q, b), q1);
      const T b1 = __ldg(B.adt + at(B.a, b));
      bres_contrib(p, s, q1, b1, __ldg(B.bound_d + at(B.bound, b)), K, f);
    }
    st4(v + 4 * (size_t)i, f);
  }
}

// The same pass for the shape res_calc always has in the airfoil app: both
// x arguments through one dim-2 map (pedge, idx 0 and 1), q and adt through
// another (pecell), one dataset each -- one 8-byte load per map, 32-bit
// index arithmetic (map values are checked against the target set's size
// at op_decl_map; the host takes this path only for sets below 2^30).
template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4)
    k_res_flux_pair(int ne, const int2 *__restrict__ pedge, const int2 *__restrict__ pecell,
                    const T *__restrict__ x, const T *__restrict__ q,
                    const T *__restrict__ adt, BresEdges<T> B, T *__restrict__ v,
                    AirConsts<T> K) {
  const unsigned total = (unsigned)ne + (unsigned)B.n, n_e = (unsigned)ne;
  const unsigned i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned stride = gridDim.x * blockDim.x;
  int2 nn = make_int2(0, 0), cc = make_int2(0, 0);
  if (i0 < n_e) {  // map entries: read-only, fetched before the wait
    nn = __ldg(pedge + i0);
    cc = __ldg(pecell + i0);
  }
  pdl_wait();
  pdl_trigger();
  for (unsigned i = i0; i < total; i += stride) {
    T f[4];
    if (i < n_e) {
      T p[2], s[2], q1[4], q2[4];
      ld4(q + 4u * (unsigned)cc.x, q1);
      ld4(q + 4u * (unsigned)cc.y, q2);
      ld2(x + 2u * (unsigned)nn.x, p);
      ld2(x + 2u * (unsigned)nn.y, s);
      const T d1 = __ldg(adt + (unsigned)cc.x), d2 = __ldg(adt + (unsigned)cc.y);
      if (i + stride < n_e) {
        nn = __ldg(pedge + i + stride);
        cc = __ldg(pecell + i + stride);
      }
      res_flux(p, s, q1, q2, d1, d2, K.gm1, K.eps, f);
    } else {
      const int b = (int)(i - n_e);
      int m1, m2;
      at2(B.x1, B.x2, b, m1, m2);
      T p[2], s[2], q1[4];
      ld2(B.xa + 2 * (size_t)m1, p);
      ld2(B.xb + 2 * (size_t)m2, s);
      ld4(B.q_d + 4 * (size_t)at(B.q, b), q1);
      const T b1 = __ldg(B.adt + at(B.a, b));
      bres_contrib(p, s, q1, b1, __ldg(B.bound_d + at(B.bound, b)), K, f);
    }
    st4(v + 4u * i, f);
  }
}

// r += the listed values of cell c, in list order
template <class T>
__device__ __forceinline__ void fold_list(const int *__restrict__ ell, int W,
                                          const T *__restrict__ v, int c, T r[4]) {
  for (int j0 = 0; j0 < W; j0 += 4) {
    int k[4];
    if (W - j0 >= 4 && ((W & 3) == 0)) {
      const int4 kk = __ldg(reinterpret_cast<const int4 *>(ell + (size_t)c * W + j0));
      k[0] = kk.x; k[1] = kk.y; k[2] = kk.z; k[3] = kk.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) k[j] = j0 + j < W ? __ldg(ell + (size_t)c * W + j0 + j) : -1;
    }
    T f[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (k[j] >= 0) ld4(v + 4 * (size_t)(k[j] >> 1), f[j]);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (k[j] < 0) continue;
      if (k[j] & 1) {
        r[0] -= f[j][0]; r[1] -= f[j][1]; r[2] -= f[j][2]; r[3] -= f[j][3];
      } else {
        r[0] += f[j][0]; r[1] += f[j][1]; r[2] += f[j][2]; r[3] += f[j][3];
      }
    }
  }
}

template <class T>
__global__ void k_res_fold_list(int n, const int *__restrict__ ell, int W,
                                const T *__restrict__ v, T *__restrict__ res) {
  pdl_wait();
  pdl_trigger();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    T r[4];
    ldw4(res + 4 * (size_t)c, r);
    fold_list(ell, W, v, c, r);
    st4(res + 4 * (size_t)c, r);
  }
}

// the fold followed by update (airfoil/update.h:1-12) on the same cell and,
// with ADT, adt_calc on the new q (airfoil/adt_calc.h); update's del^2 go
// to the tree reduction, or to seq (element order) for the serial fold
struct CellNodes {  // adt_calc's four x arguments through pcell
  IdxMap m0, m1, m2, m3;
};
// U cells per thread: every index load of the U cells, then every data
// load, then the arithmetic, so up to U cells' gathers are in flight at
// once; MINB is the launch-bounds occupancy target (register cap).  SAVE:
// save_soln follows update (the next outer iteration's first loop), so the
// new q is also stored to qsave -- usually qold itself, which update read at
// the same cell first, hence the plain (coherent) load of qold.  adt_out,
// when not null, receives adt_calc's values instead of adt (update still
// reads adt): the loops run ahead of their calls into spare buffers.  NORES:
// res is known to hold +0.0 everywhere, so the sums start from +0.0 and res
// is neither read nor rewritten
template <class T, bool ADT, int U, int MINB, bool SAVE = false, bool NORES = false>
__global__ void __launch_bounds__(256, MINB)
    k_fold_update(int n, const int *__restrict__ ell, int W, const T *__restrict__ vals,
                  const T *qold, T *__restrict__ q, T *__restrict__ res,
                  T *__restrict__ adt, CellNodes N, const T *__restrict__ x0,
                  const T *__restrict__ x1, const T *__restrict__ x2, const T *__restrict__ x3,
                  AirConsts<T> K, T *seq, RedSlot<T> slot, unsigned *ticket, T *qsave,
                  T *adt_out) {
  const bool quad = N.m0.map && N.m0.map == N.m1.map && N.m0.map == N.m2.map &&
                    N.m0.map == N.m3.map && N.m0.dim == 4 && N.m0.idx == 0 && N.m1.idx == 1 &&
                    N.m2.idx == 2 && N.m3.idx == 3;
  const int stride = gridDim.x * blockDim.x;
  T rms = T(0);
  // list heads and node indices of U cells: plan and map data (read-only),
  // fetched one pass ahead so they arrive while the current pass gathers
  int nd[U][4], k[U][4], ndn[U][4], kn[U][4];
  auto indices = [&](int base, int (&kk)[U][4], int (&nn)[U][4]) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int c = base + u * stride;
      if (c >= n) continue;
      list_head(ell, W, c, kk[u]);
      if (ADT) {
        if (quad) {
          int4 v = __ldg(reinterpret_cast<const int4 *>(N.m0.map) + c);
          nn[u][0] = v.x; nn[u][1] = v.y; nn[u][2] = v.z; nn[u][3] = v.w;
        } else {
          nn[u][0] = at(N.m0, c); nn[u][1] = at(N.m1, c);
          nn[u][2] = at(N.m2, c); nn[u][3] = at(N.m3, c);
        }
      }
    }
  };
  const int base0 = blockIdx.x * blockDim.x + threadIdx.x;
  // the cells' own streams and node coordinates (res, qold, adt, x): the
  // flux pass this kernel follows does not write them, and the launches
  // that did had completed before the flux pass could let this kernel
  // start, so the first pass fetches them before the wait too; only the
  // flux values wait
  T r[U][4], qo[U][4], ad[U], xs[U][4][2];
  auto streams = [&](int base) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int c = base + u * stride;
      if (c >= n) continue;
      if (!NORES) ldw4(res + 4 * (size_t)c, r[u]);
      else r[u][0] = r[u][1] = r[u][2] = r[u][3] = T(0);
      if (SAVE) ldw4(qold + 4 * (size_t)c, qo[u]);
      else ld4(qold + 4 * (size_t)c, qo[u]);
      ad[u] = adt[c];
      if (ADT) {
        ld2(x0 + 2 * (size_t)nd[u][0], xs[u][0]);
        ld2(x1 + 2 * (size_t)nd[u][1], xs[u][1]);
        ld2(x2 + 2 * (size_t)nd[u][2], xs[u][2]);
        ld2(x3 + 2 * (size_t)nd[u][3], xs[u][3]);
      }
    }
  };
  indices(base0, k, nd);  // before the previous kernel has finished
  streams(base0);
  pdl_wait();
  pdl_trigger();
  for (int base = base0; base < n; base += stride * U) {
    T f[U][4][4];
    if (base != base0) streams(base);
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int c = base + u * stride;
      if (c >= n) continue;
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (k[u][j] >= 0) ld4(vals + 4 * (size_t)(k[u][j] >> 1), f[u][j]);
    }
    indices(base + stride * U, kn, ndn);
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int c = base + u * stride;
      if (c >= n) continue;
#pragma unroll
      for (int j = 0; j < 4; j++) add_listed(r[u], k[u][j], f[u][j]);
      for (int j = 4; j < W; j++) {  // lists longer than 4
        const int kk = __ldg(ell + (size_t)c * W + j);
        T g[4];
        ld4(vals + 4 * (size_t)(kk >> 1), g);
        add_listed(r[u], kk, g);
      }
      // airfoil/update.h:1-12
      T adti = rcp(ad[u]);
      T qn[4], sq[4];
      for (int d = 0; d < 4; d++) {
        T del = adti * r[u][d];
        qn[d] = qo[u][d] - del;
        sq[d] = del * del;
        rms += sq[d];
      }
      st4(q + 4 * (size_t)c, qn);
      if (SAVE) st4(qsave + 4 * (size_t)c, qn);  // airfoil/save_soln.h:1-3
      const T z[4] = {T(0), T(0), T(0), T(0)};
      if (!NORES) st4(res + 4 * (size_t)c, z);
      if (seq) st4(seq + 4 * (size_t)c, sq);
      if (ADT) (adt_out ? adt_out : adt)[c] = adt_calc(xs[u][0], xs[u][1], xs[u][2], xs[u][3], qn, K);
    }
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        k[u][j] = kn[u][j];
        nd[u][j] = ndn[u][j];
      }
  }
  if (seq) return;
  const T v[1] = {rms}, id[1] = {T(0)};
  RedSlot<T> sl[1] = {slot};
  grid_finish<T, OpSum, OpSum, 1>(v, id, OpSum(), OpSum(), sl, ticket);
}

// One cell per thread, with the cell's own streams (res, qold, adt) fetched
// a cell ahead together with its list and node indices: the next cell's
// DRAM loads are in flight while this cell's gathers return and its
// arithmetic runs, so a pass waits on the (mostly L2) gathers alone.  The
// arithmetic and its order are k_fold_update's.  Reading the next cell's
// res/qold/adt before this cell's stores is safe: every cell belongs to one
// thread.
template <class T, bool ADT, int MINB, bool SAVE, bool NORES = false>
__global__ void __launch_bounds__(256, MINB)
    k_fold_update_pf(int n, const int *__restrict__ ell, int W, const T *__restrict__ vals,
                     const T *qold, T *__restrict__ q, T *__restrict__ res, T *__restrict__ adt,
                     CellNodes N, const T *__restrict__ x0, const T *__restrict__ x1,
                     const T *__restrict__ x2, const T *__restrict__ x3, AirConsts<T> K, T *seq,
                     RedSlot<T> slot, unsigned *ticket, T *qsave, T *adt_out) {
  const bool quad = N.m0.map && N.m0.map == N.m1.map && N.m0.map == N.m2.map &&
                    N.m0.map == N.m3.map && N.m0.dim == 4 && N.m0.idx == 0 && N.m1.idx == 1 &&
                    N.m2.idx == 2 && N.m3.idx == 3;
  const int stride = gridDim.x * blockDim.x;
  T rms = T(0);
  auto indices = [&](int c, int (&kk)[4], int (&nn)[4]) {
    list_head(ell, W, c, kk);
    if (ADT) {
      if (quad) {
        int4 v = __ldg(reinterpret_cast<const int4 *>(N.m0.map) + c);
        nn[0] = v.x; nn[1] = v.y; nn[2] = v.z; nn[3] = v.w;
      } else {
        nn[0] = at(N.m0, c); nn[1] = at(N.m1, c); nn[2] = at(N.m2, c); nn[3] = at(N.m3, c);
      }
    }
  };
  auto streams = [&](int c, T (&r)[4], T (&qo)[4], T &ad) {
    if (!NORES) ldw4(res + 4 * (size_t)c, r);
    else r[0] = r[1] = r[2] = r[3] = T(0);
    if (SAVE) ldw4(qold + 4 * (size_t)c, qo);
    else ld4(qold + 4 * (size_t)c, qo);
    ad = adt[c];
  };
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int k[4] = {-1, -1, -1, -1}, nd[4] = {0, 0, 0, 0};
  if (c < n) indices(c, k, nd);  // before the previous kernel has finished
  pdl_wait();
  pdl_trigger();
  T r[4], qo[4], ad = T(1);
  if (c < n) streams(c, r, qo, ad);
  for (; c < n; c += stride) {
    T f[4][4], xs[4][2];
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (k[j] >= 0) ld4(vals + 4 * (size_t)(k[j] >> 1), f[j]);
    if (ADT) {
      ld2(x0 + 2 * (size_t)nd[0], xs[0]);
      ld2(x1 + 2 * (size_t)nd[1], xs[1]);
      ld2(x2 + 2 * (size_t)nd[2], xs[2]);
      ld2(x3 + 2 * (size_t)nd[3], xs[3]);
    }
    const int cn = c + stride;
    int kn[4] = {-1, -1, -1, -1}, ndn[4] = {0, 0, 0, 0};
    T rn[4], qon[4], adn = T(1);
    if (cn < n) {
      indices(cn, kn, ndn);
      streams(cn, rn, qon, adn);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) add_listed(r, k[j], f[j]);
    for (int j = 4; j < W; j++) {  // lists longer than 4
      const int kk = __ldg(ell + (size_t)c * W + j);
      T g[4];
      ld4(vals + 4 * (size_t)(kk >> 1), g);
      add_listed(r, kk, g);
    }
    // airfoil/update.h:1-12
    T adti = rcp(ad);
    T qn[4], sq[4];
    for (int d = 0; d < 4; d++) {
      T del = adti * r[d];
      qn[d] = qo[d] - del;
      sq[d] = del * del;
      rms += sq[d];
    }
    st4(q + 4 * (size_t)c, qn);
    if (SAVE) st4(qsave + 4 * (size_t)c, qn);  // airfoil/save_soln.h:1-3
    const T z[4] = {T(0), T(0), T(0), T(0)};
    if (!NORES) st4(res + 4 * (size_t)c, z);
    if (seq) st4(seq + 4 * (size_t)c, sq);
    if (ADT) (adt_out ? adt_out : adt)[c] = adt_calc(xs[0], xs[1], xs[2], xs[3], qn, K);
    if (cn < n) {
#pragma unroll
      for (int j = 0; j < 4; j++) {
        k[j] = kn[j];
        nd[j] = ndn[j];
        r[j] = rn[j];
        qo[j] = qon[j];
      }
      ad = adn;
    }
  }
  if (seq) return;
  const T v[1] = {rms}, id[1] = {T(0)};
  RedSlot<T> sl[1] = {slot};
  grid_finish<T, OpSum, OpSum, 1>(v, id, OpSum(), OpSum(), sl, ticket);
}

// --------------------------------------------- persistent res_calc chain ----
// res_calc + bres_calc + update [+ adt_calc] [+ save_soln] as ONE persistent
// launch over a static queue of work items: flux tiles (ET consecutive
// entries of the flux index space -- res_calc's edges, then bres_calc's
// boundary edges) and cell tiles (CT consecutive cells: ordered fold of the
// cells' lists, update, adt_calc, save_soln).  Each CTA takes the next item
// with an atomic counter, so issue-bound flux tiles and latency-bound cell
// tiles run side by side on every SM instead of one pass after the other.
//
// A cell tile may start only when the flux tiles its lists read (at most
// kChainMaxDeps distinct ones, listed per cell tile at plan time) are done.
// The queue places each cell tile `lag` flux tiles after the last of them.
// A flux tile publishes completion with an epoch-tagged flag (block barrier,
// then a release store by one thread); a CTA about to fold checks its tile's
// flags with one warp, one flag per lane (acquire loads, in parallel), and
// a block barrier passes the result on.  Items are taken in queue
// order and a cell tile waits only on items taken before it, which belong
// to CTAs that are running (or hold them next, behind an item that waits on
// still earlier ones): the waits always end.  They are bounded all the same
// (one second, then counted in op2b_wait_timeouts and skipped).
//
// The same dependency covers the chain's write-after-read hazards: a flux
// tile reads q and adt of the cells of its edges, and every such edge is in
// those cells' lists, so no cell's q or adt is overwritten before the last
// flux value that reads it has been computed.  Values written by other CTAs
// of this launch are read through L2 (ld.global.cg).
//
// The arithmetic and its order per cell and per edge are those of
// k_res_flux_pair and k_fold_update: q, res, adt, qold are bit-identical.
// The rms: each cell tile's partial (its threads' sums, block tree) goes to
// partials[tile]; the last CTA folds them in tile order.
struct ChainSchedDev {
  const int *queue;    // [nitems]: >= 0 flux tile, < 0 cell tile -(t + 1)
  const int *dep_off;  // [ncell_tiles + 1]: a cell tile's flux tiles are
  const int *deps;     //   deps[dep_off[t], dep_off[t+1]) (distinct, <= 64)
  unsigned *flags;     // [nflux_tiles]: epoch of the last launch that wrote it
  unsigned *ctl;       // next item, (unused), finish ticket, epoch
  void *partials;      // [ncell_tiles] rms partials (8-byte slots)
  int nitems, nflux, ncellt, et, ct;
};
constexpr int kChainMaxDeps = 64;  // flux tiles one cell tile may wait for

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// L2-coherent vector loads of values written by other CTAs of this launch
__device__ __forceinline__ void ld4cg(const float *p, float v[4]) {
  float4 t = __ldcg(reinterpret_cast<const float4 *>(p));
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ld4cg(const double *p, double v[4]) {
  double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
  double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <class T, bool ADT, bool SAVE, int U>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    k_chain_persist(ChainSchedDev S, int ne, const int2 *__restrict__ pedge,
                    const int2 *__restrict__ pecell, const T *__restrict__ x,
                    const T *__restrict__ qf, const T *__restrict__ adtf, BresEdges<T> B,
                    T *vals, int n, const int *__restrict__ ell, int W, const T *qold, T *q,
                    T *res, const T *adt, CellNodes N, const T *__restrict__ x0,
                    const T *__restrict__ x1, const T *__restrict__ x2,
                    const T *__restrict__ x3, AirConsts<T> K, T *seq, T *result, T *qsave,
                    T *adt_out) {
  __shared__ int s_item[2];
  __shared__ T ws[32];
  __shared__ bool last;
  const int tid = threadIdx.x;
  pdl_wait();
  pdl_trigger();
  const unsigned ep = ld_acquire(S.ctl + 3) + 1u;
  T *partials = reinterpret_cast<T *>(S.partials);
  const unsigned total = (unsigned)ne + (unsigned)B.n;
  if (tid == 0) s_item[0] = (int)atomicAdd(S.ctl, 1u);
  __syncthreads();
  for (int par = 0;; par ^= 1) {
    const int it = s_item[par];
    if (it >= S.nitems) break;
    if (tid == 0) s_item[par ^ 1] = (int)atomicAdd(S.ctl, 1u);  // in flight meanwhile
    const int code = __ldg(S.queue + it);
    if (code >= 0) {  // ------------------------------------- flux tile
      const unsigned e0 = (unsigned)code * (unsigned)S.et;
      const unsigned e1 = min(total, e0 + (unsigned)S.et);
      for (unsigned i = e0 + tid; i < e1; i += 256) {
        T f[4];
        if (i < (unsigned)ne) {
          const int2 nn = __ldg(pedge + i), cc = __ldg(pecell + i);
          T p[2], s2[2], q1[4], q2[4];
          ld4(qf + 4u * (unsigned)cc.x, q1);
          ld4(qf + 4u * (unsigned)cc.y, q2);
          ld2(x + 2u * (unsigned)nn.x, p);
          ld2(x + 2u * (unsigned)nn.y, s2);
          const T d1 = __ldg(adtf + (unsigned)cc.x), d2 = __ldg(adtf + (unsigned)cc.y);
          res_flux(p, s2, q1, q2, d1, d2, K.gm1, K.eps, f);
        } else {
          const int b = (int)(i - (unsigned)ne);
          int m1, m2;
          at2(B.x1, B.x2, b, m1, m2);
          T p[2], s2[2], q1[4];
          ld2(B.xa + 2 * (size_t)m1, p);
          ld2(B.xb + 2 * (size_t)m2, s2);
          ld4(B.q_d + 4 * (size_t)at(B.q, b), q1);
          const T b1 = __ldg(B.adt + at(B.a, b));
          bres_contrib(p, s2, q1, b1, __ldg(B.bound_d + at(B.bound, b)), K, f);
        }
        st4(vals + 4u * i, f);
      }
      __syncthreads();  // the tile's values are written
      if (tid == 0) st_release(S.flags + code, ep);
    } else {  // ---------------------------------------------- cell tile
      const int t = -code - 1;
      if (tid < 32) {  // one warp checks the tile's flux tiles, a flag per lane
        const int d0 = __ldg(S.dep_off + t), d1 = __ldg(S.dep_off + t + 1);
        const int ja = d0 + tid < d1 ? __ldg(S.deps + d0 + tid) : -1;
        const int jb = d0 + tid + 32 < d1 ? __ldg(S.deps + d0 + tid + 32) : -1;
        bool da = ja < 0 || ld_acquire(S.flags + ja) == ep;
        bool db = jb < 0 || ld_acquire(S.flags + jb) == ep;
        if (!__all_sync(0xffffffffu, da && db)) {
          const unsigned long long t0 = global_ns();
          for (;;) {
            __nanosleep(100);
            if (!da) da = ld_acquire(S.flags + ja) == ep;
            if (!db) db = ld_acquire(S.flags + jb) == ep;
            if (__all_sync(0xffffffffu, da && db)) break;
            if (global_ns() - t0 > kWaitLimitNs) {  // give up: counted, results wrong
              if (tid == 0) atomicAdd(&g_wait_timeouts, 1u);
              break;
            }
          }
        }
      }
      __syncthreads();
      T rms = T(0);
      const int c0 = t * S.ct;
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int c = c0 + u * 256 + tid;
        if (c >= n || u * 256 >= S.ct) continue;
        int k[4];
        list_head(ell, W, c, k);
        int nd[4] = {0, 0, 0, 0};
        if (ADT) {
          const int4 v = __ldg(reinterpret_cast<const int4 *>(N.m0.map) + c);
          nd[0] = v.x; nd[1] = v.y; nd[2] = v.z; nd[3] = v.w;
        }
        T r[4], qo[4], f[4][4], xs[4][2];
        ldw4(res + 4 * (size_t)c, r);
        if (SAVE) ldw4(qold + 4 * (size_t)c, qo);
        else ld4(qold + 4 * (size_t)c, qo);
        const T ad = adt[c];
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (k[j] >= 0) ld4cg(vals + 4 * (size_t)(k[j] >> 1), f[j]);
        if (ADT) {
          ld2(x0 + 2 * (size_t)nd[0], xs[0]);
          ld2(x1 + 2 * (size_t)nd[1], xs[1]);
          ld2(x2 + 2 * (size_t)nd[2], xs[2]);
          ld2(x3 + 2 * (size_t)nd[3], xs[3]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) add_listed(r, k[j], f[j]);
        for (int j = 4; j < W; j++) {  // lists longer than 4
          const int kk = __ldg(ell + (size_t)c * W + j);
          T g[4];
          ld4cg(vals + 4 * (size_t)(kk >> 1), g);
          add_listed(r, kk, g);
        }
        // airfoil/update.h:1-12
        T adti = rcp(ad);
        T qn[4], sq[4];
        for (int d = 0; d < 4; d++) {
          T del = adti * r[d];
          qn[d] = qo[d] - del;
          sq[d] = del * del;
          rms += sq[d];
        }
        st4(q + 4 * (size_t)c, qn);
        if (SAVE) st4(qsave + 4 * (size_t)c, qn);  // airfoil/save_soln.h:1-3
        const T z[4] = {T(0), T(0), T(0), T(0)};
        st4(res + 4 * (size_t)c, z);
        if (seq) st4(seq + 4 * (size_t)c, sq);
        if (ADT) adt_out[c] = adt_calc(xs[0], xs[1], xs[2], xs[3], qn, K);
      }
      const T b = block_fold(rms, T(0), OpSum(), ws);
      if (tid == 0) partials[t] = b;
    }
    __syncthreads();  // s_item[par ^ 1] is set; everyone has read s_item[par]
  }
  // the last CTA to finish folds the cell tiles' partials in tile order and
  // re-arms the queue for the next launch
  if (tid == 0) {
    __threadfence();
    last = atomicAdd(S.ctl + 2, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  T xsum = T(0);
  for (int k = tid; k < S.ncellt; k += 256) xsum += __ldcg(partials + k);
  xsum = block_fold(xsum, T(0), OpSum(), ws);
  if (tid == 0) {
    if (!seq) *result = xsum;
    S.ctl[0] = 0u;
    S.ctl[2] = 0u;
    __threadfence();
    st_release(S.ctl + 3, ep);
  }
}


template <class T>
__global__ void k_fill(T *p, size_t n, T v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// bres_calc, GATHER: one thread per cell that has boundary edges
template <class T>
__global__ void k_bres_calc_gather(int nrows, const int *__restrict__ active,
                                   const int *__restrict__ row, const int *__restrict__ keys,
                                   IdxMap mx1, IdxMap mx2, IdxMap mq, IdxMap ma, IdxMap mb,
                                   const T *__restrict__ xa, const T *__restrict__ xb,
                                   const T *__restrict__ q, const T *__restrict__ adt,
                                   const int *__restrict__ bound, T *__restrict__ res,
                                   AirConsts<T> K) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows) return;
  int c = active ? active[t] : t;
  T r[4];
  ldw4(res + 4 * (size_t)c, r);
  int k1 = row[t + 1];
  for (int k = row[t]; k < k1; k++) {
    int e = __ldg(keys + k);
    T p[2], s[2], q1[4];
    ld2(xa + 2 * (size_t)at(mx1, e), p);
    ld2(xb + 2 * (size_t)at(mx2, e), s);
    ld4(q + 4 * (size_t)at(mq, e), q1);
    T a1 = __ldg(adt + at(ma, e));
    bres_apply(p, s, q1, a1, __ldg(bound + at(mb, e)), K, r);
  }
  st4(res + 4 * (size_t)c, r);
}

// The plan arrays one coloured launch needs
struct PlanView {
  const int *blkmap, *offset, *nelems, *nthrcol, *thrcol, *ind_offs, *ind_sizes;
  const int *ind_maps[4];
  const short *loc_maps[8];
  int ninds;
};

// res_calc, COLOURED (inds {0,0,1,1,2,2,3,3}: x, q, adt read; res incremented)
template <class T>
__global__ void k_res_calc_coloured(PlanView P, int block_offset, const T *__restrict__ x,
                                    const T *__restrict__ q, const T *__restrict__ adt,
                                    T *__restrict__ res, T gm1, T eps) {
  extern __shared__ __align__(16) char smem[];
  const int b = P.blkmap[blockIdx.x + block_offset];
  const int nelem = P.nelems[b], off = P.offset[b], ncol = P.nthrcol[b];
  int sz[4], io[4];
  for (int m = 0; m < 4; m++) {
    sz[m] = P.ind_sizes[m + b * 4];
    io[m] = P.ind_offs[m + b * 4];
  }
  T *xs = (T *)smem;
  T *qs = (T *)(smem + ROUND_UP(sz[0] * 2 * (int)sizeof(T)));
  T *as = (T *)((char *)qs + ROUND_UP(sz[1] * 4 * (int)sizeof(T)));
  T *rs = (T *)((char *)as + ROUND_UP(sz[2] * (int)sizeof(T)));
  for (int u = threadIdx.x; u < sz[0]; u += blockDim.x) {
    T v[2];
    ld2(x + 2 * (size_t)P.ind_maps[0][io[0] + u], v);
    xs[2 * u] = v[0]; xs[2 * u + 1] = v[1];
  }
  for (int u = threadIdx.x; u < sz[1]; u += blockDim.x) {
    T v[4];
    ld4(q + 4 * (size_t)P.ind_maps[1][io[1] + u], v);
    st4(qs + 4 * u, v);
  }
  for (int u = threadIdx.x; u < sz[2]; u += blockDim.x) as[u] = __ldg(adt + P.ind_maps[2][io[2] + u]);
  for (int u = threadIdx.x; u < sz[3] * 4; u += blockDim.x) rs[u] = T(0);
  __syncthreads();
  const int nelems2 = blockDim.x * (1 + (nelem - 1) / blockDim.x);
  for (int n = threadIdx.x; n < nelems2; n += blockDim.x) {
    int col2 = -1;
    T l6[4], l7[4];
    int m6 = 0, m7 = 0;
    if (n < nelem) {
      const int e = n + off;
      T f[4];
      res_flux(xs + 2 * P.loc_maps[0][e], xs + 2 * P.loc_maps[1][e], qs + 4 * P.loc_maps[2][e],
               qs + 4 * P.loc_maps[3][e], as[P.loc_maps[4][e]], as[P.loc_maps[5][e]], gm1, eps, f);
      for (int d = 0; d < 4; d++) {
        l6[d] = T(0) + f[d];
        l7[d] = T(0) - f[d];
      }
      m6 = P.loc_maps[6][e];
      m7 = P.loc_maps[7][e];
      col2 = P.thrcol[e];
    }
    for (int col = 0; col < ncol; col++) {
      if (col2 == col) {
        for (int d = 0; d < 4; d++) rs[d + m6 * 4] += l6[d];
        for (int d = 0; d < 4; d++) rs[d + m7 * 4] += l7[d];
      }
      __syncthreads();
    }
  }
  for (int u = threadIdx.x; u < sz[3]; u += blockDim.x) {
    T *dst = res + 4 * (size_t)P.ind_maps[3][io[3] + u];
    T v[4];
    ldw4(dst, v);
    for (int d = 0; d < 4; d++) v[d] += rs[4 * u + d];
    st4(dst, v);
  }
}

// bres_calc, COLOURED (inds {0,0,1,2,3,-1}; bound is direct)
template <class T>
__global__ void k_bres_calc_coloured(PlanView P, int block_offset, const T *__restrict__ x,
                                     const T *__restrict__ q, const T *__restrict__ adt,
                                     const int *__restrict__ bound, T *__restrict__ res,
                                     AirConsts<T> K) {
  extern __shared__ __align__(16) char smem[];
  const int b = P.blkmap[blockIdx.x + block_offset];
  const int nelem = P.nelems[b], off = P.offset[b], ncol = P.nthrcol[b];
  int sz[4], io[4];
  for (int m = 0; m < 4; m++) {
    sz[m] = P.ind_sizes[m + b * 4];
    io[m] = P.ind_offs[m + b * 4];
  }
  T *xs = (T *)smem;
  T *qs = (T *)(smem + ROUND_UP(sz[0] * 2 * (int)sizeof(T)));
  T *as = (T *)((char *)qs + ROUND_UP(sz[1] * 4 * (int)sizeof(T)));
  T *rs = (T *)((char *)as + ROUND_UP(sz[2] * (int)sizeof(T)));
  for (int u = threadIdx.x; u < sz[0]; u += blockDim.x) {
    T v[2];
    ld2(x + 2 * (size_t)P.ind_maps[0][io[0] + u], v);
    xs[2 * u] = v[0]; xs[2 * u + 1] = v[1];
  }
  for (int u = threadIdx.x; u < sz[1]; u += blockDim.x) {
    T v[4];
    ld4(q + 4 * (size_t)P.ind_maps[1][io[1] + u], v);
    st4(qs + 4 * u, v);
  }
  for (int u = threadIdx.x; u < sz[2]; u += blockDim.x) as[u] = __ldg(adt + P.ind_maps[2][io[2] + u]);
  for (int u = threadIdx.x; u < sz[3] * 4; u += blockDim.x) rs[u] = T(0);
  __syncthreads();
  const int nelems2 = blockDim.x * (1 + (nelem - 1) / blockDim.x);
  for (int n = threadIdx.x; n < nelems2; n += blockDim.x) {
    int col2 = -1, m4 = 0;
    T l4[4] = {T(0), T(0), T(0), T(0)};
    if (n < nelem) {
      const int e = n + off;
      bres_apply(xs + 2 * P.loc_maps[0][e], xs + 2 * P.loc_maps[1][e], qs + 4 * P.loc_maps[2][e],
                 as[P.loc_maps[3][e]], __ldg(bound + e), K, l4);
      m4 = P.loc_maps[4][e];
      col2 = P.thrcol[e];
    }
    for (int col = 0; col < ncol; col++) {
      if (col2 == col)
        for (int d = 0; d < 4; d++) rs[d + m4 * 4] += l4[d];
      __syncthreads();
    }
  }
  for (int u = threadIdx.x; u < sz[3]; u += blockDim.x) {
    T *dst = res + 4 * (size_t)P.ind_maps[3][io[3] + u];
    T v[4];
    ldw4(dst, v);
    for (int d = 0; d < 4; d++) v[d] += rs[4 * u + d];
    st4(dst, v);
  }
}

// update: q = qold - res/adt, res = 0, rms += del^2 (airfoil/update.h:1-12).
// SEQ != nullptr: store each del^2 in element order for the serial fold.
template <class T, int U>
__global__ void k_update(int n, const T *__restrict__ qold, T *__restrict__ q,
                         T *__restrict__ res, const T *__restrict__ adt, T *seq,
                         RedSlot<T> slot, unsigned *ticket) {
  pdl_wait();
  pdl_trigger();
  T rms = T(0);
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += stride * U) {
    T qo[U][4], r[U][4], ad[U];
#pragma unroll
    for (int u = 0; u < U; u++) {  // all loads of the U cells first
      int c = base + u * stride;
      if (c < n) {
        ld4(qold + 4 * (size_t)c, qo[u]);
        ldw4(res + 4 * (size_t)c, r[u]);
        ad[u] = __ldg(adt + c);
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      int c = base + u * stride;
      if (c >= n) continue;
      T adti = rcp(ad[u]);
      T qn[4], sq[4];
      for (int d = 0; d < 4; d++) {
        T del = adti * r[u][d];
        qn[d] = qo[u][d] - del;
        sq[d] = del * del;
        rms += sq[d];
      }
      st4(q + 4 * (size_t)c, qn);
      const T z[4] = {T(0), T(0), T(0), T(0)};
      st4(res + 4 * (size_t)c, z);
      if (seq) st4(seq + 4 * (size_t)c, sq);
    }
  }
  if (seq) return;
  const T v[1] = {rms}, id[1] = {T(0)};
  RedSlot<T> sl[1] = {slot};
  grid_finish<T, OpSum, OpSum, 1>(v, id, OpSum(), OpSum(), sl, ticket);
}

// ------------------------------------------------------------ host side ---

template <class T>
static AirConsts<T> air_consts_lookup();

// the constants by name, looked up again only when a constant was declared
template <class T>
static AirConsts<T> air_consts() {
  static AirConsts<T> cached;
  static unsigned version = ~0u;
  if (version != rt().consts_version) {
    cached = air_consts_lookup<T>();
    if (error_pending()) return cached;
    version = rt().consts_version;
  }
  return cached;
}

template <class T>
static AirConsts<T> air_consts_lookup() {
  AirConsts<T> K;
  memset(&K, 0, sizeof K);
  T v[4];
  auto get = [&](const char *nm, int dim) -> bool {
    int got = sizeof(T) == 4 ? const_get_f32(nm, (float *)v, dim) : const_get_f64(nm, (double *)v, dim);
    if (got < dim) {
      fail(-1, "op2b error -- constant \"%s\" (dim %d) not declared with op_decl_const2\n", nm, dim);
      return false;
    }
    return true;
  };
  if (get("gam", 1)) K.gam = v[0];
  if (get("gm1", 1)) K.gm1 = v[0];
  if (get("cfl", 1)) K.cfl = v[0];
  if (get("eps", 1)) K.eps = v[0];
  if (get("qinf", 4))
    for (int i = 0; i < 4; i++) K.qinf[i] = v[i];
  return K;
}

static bool is_double(const op_arg &a) { return a.dat && strcmp(a.dat->type, "double") == 0; }

static int grid_for(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  long long cap = (long long)rt().num_sms * 16;
  if (g < 1) g = 1;
  return (int)(g < cap ? g : cap);
}

// direct loops: U elements per thread, at most 8 CTAs of 256 per SM (full
// occupancy), so one pass covers the 720k-cell set
constexpr int kUnroll = 4;
static int unroll() {
  int u = tuning("unroll", kUnroll);
  return u == 1 || u == 2 ? u : 4;
}
static int grid_direct(long long n, int U) {
  long long g = (n + 256LL * U - 1) / (256LL * U);
  long long cap = (long long)rt().num_sms * tuning("direct_ctas_per_sm", 8);
  if (g < 1) g = 1;
  return (int)(g < cap ? g : cap);
}

static PlanView plan_view(const DevPlan &p) {
  PlanView v;
  memset(&v, 0, sizeof v);
  v.blkmap = p.d_blkmap; v.offset = p.d_offset; v.nelems = p.d_nelems; v.nthrcol = p.d_nthrcol;
  v.thrcol = p.d_thrcol; v.ind_offs = p.d_ind_offs; v.ind_sizes = p.d_ind_sizes;
  v.ninds = p.ninds;
  for (int m = 0; m < p.ninds && m < 4; m++) v.ind_maps[m] = p.d_ind_maps[m];
  for (int a = 0; a < p.nargs && a < 8; a++) v.loc_maps[a] = p.d_loc_maps[a];
  return v;
}

template <class T>
static void save_soln_t(char const *name, op_set set, const op_arg *args) {
  LoopScope ls(name, compulsory_bytes(set, 2, args), 0);
  int n = set->size;
  const int U = unroll();
  const T *q = (const T *)args[0].dat->data_d;
  T *qold = (T *)args[1].dat->data_d;
  cudaStream_t s = rt().stream;
  if (U == 1) launch_pdl(k_save_soln<T, 1>, grid_direct(n, 1), 256, 0, s, n, q, qold);
  else if (U == 2) launch_pdl(k_save_soln<T, 2>, grid_direct(n, 2), 256, 0, s, n, q, qold);
  else launch_pdl(k_save_soln<T, 4>, grid_direct(n, 4), 256, 0, s, n, q, qold);
}
void run_save_soln(char const *name, op_set set, const op_arg *args) {
  if (is_double(args[0])) save_soln_t<double>(name, set, args);
  else save_soln_t<float>(name, set, args);
}

template <class T>
static void adt_calc_t(char const *name, op_set set, const op_arg *args) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return;
  LoopScope ls(name, compulsory_bytes(set, 6, args), 0);
  int n = set->size;
  const int U = tuning("adt_unroll", 1) >= 2 ? 2 : 1;
  auto launch = [&](auto kernel, int u) {
    launch_pdl(kernel, grid_direct(n, u), 256, 0, rt().stream, n, idx_map(args[0]),
               idx_map(args[1]), idx_map(args[2]), idx_map(args[3]), idx_map(args[4]),
               (const T *)args[0].dat->data_d, (const T *)args[1].dat->data_d,
               (const T *)args[2].dat->data_d, (const T *)args[3].dat->data_d,
               (const T *)args[4].dat->data_d, (T *)args[5].dat->data_d, K);
  };
  if (U == 2) launch(k_adt_calc<T, 2>, 2);
  else launch(k_adt_calc<T, 1>, 1);
}
void run_adt_calc(char const *name, op_set set, const op_arg *args) {
  if (is_double(args[0])) adt_calc_t<double>(name, set, args);
  else adt_calc_t<float>(name, set, args);
}

static const int kResInds[8] = {0, 0, 1, 1, 2, 2, 3, 3};
static const int kBresInds[6] = {0, 0, 1, 2, 3, -1};

template <class T>
static void res_calc_t(char const *name, op_set set, const op_arg *args) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return;
  cudaStream_t s = rt().stream;
  if (effective_strategy(name) == OP2B_STRATEGY_COLOURED) {
    int part = OP_part_size;
    DevPlan *p = get_plan(name, set, part, 8, args, 4, kResInds);
    if (!p) return;
    LoopScope ls(name, p->transfer, p->transfer2);
    PlanView v = plan_view(*p);
    int nthread = OP_block_size > 0 ? OP_block_size : 512;
    if (p->nshared > 48 * 1024)
      OP2B_CUDA(cudaFuncSetAttribute(k_res_calc_coloured<T>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, p->nshared));
    for (int c = 0, off = 0; c < p->ncolors; off += p->ncolblk[c], c++)
      if (p->ncolblk[c] > 0)
        k_res_calc_coloured<T><<<p->ncolblk[c], nthread, p->nshared, s>>>(
            v, off, (const T *)args[0].dat->data_d, (const T *)args[2].dat->data_d,
            (const T *)args[4].dat->data_d, (T *)args[6].dat->data_d, K.gm1, K.eps);
    return;
  }
  GatherPlan *g = get_gather_plan(set, args, {6, 7});
  if (!g) return;
  if (tuning("gather_flux", 1) && tuning("gather_slots", 1) &&
      run_res_chain(name, set, args, nullptr, nullptr, nullptr, nullptr, nullptr))
    return;
  LoopScope ls(name, compulsory_bytes(set, 8, args), 0);
  if (g->nactive == 0) return;
  if (tuning("gather_flux", 1)) {
    // two passes: each edge's flux once, then the ordered per-cell fold
    const int ne = set->size;
    const size_t need = sizeof(T) * 4 * (size_t)ne;
    if (g->contrib_bytes < need) {
      dev_free(g->d_contrib);
      g->d_contrib = dev_alloc(need);
      g->contrib_bytes = g->d_contrib ? need : 0;
      if (!g->d_contrib) return;
    }
    T *flux = (T *)g->d_contrib;
    k_res_flux<T><<<grid_for(ne, 256), 256, 0, s>>>(
        ne, idx_map(args[0]), idx_map(args[1]), idx_map(args[2]), idx_map(args[3]),
        idx_map(args[4]), idx_map(args[5]), (const T *)args[0].dat->data_d,
        (const T *)args[1].dat->data_d, (const T *)args[2].dat->data_d,
        (const T *)args[3].dat->data_d, (const T *)args[4].dat->data_d,
        (const T *)args[5].dat->data_d, flux, K.gm1, K.eps);
    k_res_fold<T><<<(g->nactive + 255) / 256, 256, 0, s>>>(g->nactive, g->d_active, g->d_row,
                                                          g->d_keys, flux,
                                                          (T *)args[6].dat->data_d);
    return;
  }
  if (tuning("gather_tiled", 0) && g->max_row - 1 <= kTileExtra && g->ntiles > 0) {
    k_res_calc_tiled<T><<<g->ntiles, kTile, 0, s>>>(
        g->d_tile_first, g->d_active, g->d_row, g->d_keys, idx_map(args[0]), idx_map(args[1]),
        idx_map(args[2]), idx_map(args[3]), idx_map(args[4]), idx_map(args[5]),
        (const T *)args[0].dat->data_d, (const T *)args[1].dat->data_d,
        (const T *)args[2].dat->data_d, (const T *)args[3].dat->data_d,
        (const T *)args[4].dat->data_d, (const T *)args[5].dat->data_d, (T *)args[6].dat->data_d,
        K.gm1, K.eps);
    return;
  }
  // one thread per cell (default)
  auto launch = [&](auto kernel) {
    kernel<<<(g->nactive + 255) / 256, 256, 0, s>>>(
        g->nactive, g->d_active, g->d_row, g->d_keys, idx_map(args[0]), idx_map(args[1]),
        idx_map(args[2]), idx_map(args[3]), idx_map(args[4]), idx_map(args[5]),
        (const T *)args[0].dat->data_d, (const T *)args[1].dat->data_d,
        (const T *)args[2].dat->data_d, (const T *)args[3].dat->data_d,
        (const T *)args[4].dat->data_d, (const T *)args[5].dat->data_d,
        (T *)args[6].dat->data_d, K.gm1, K.eps);
  };
  if (tuning("gather_batch", 1) >= 4) launch(k_res_calc_gather<T, 4>);
  else if (tuning("gather_batch", 1) >= 2) launch(k_res_calc_gather<T, 2>);
  else launch(k_res_calc_gather<T, 1>);
}
void run_res_calc(char const *name, op_set set, const op_arg *args) {
  if (is_double(args[0])) res_calc_t<double>(name, set, args);
  else res_calc_t<float>(name, set, args);
}

template <class T>
static void bres_calc_t(char const *name, op_set set, const op_arg *args) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return;
  cudaStream_t s = rt().stream;
  if (effective_strategy(name) == OP2B_STRATEGY_COLOURED) {
    DevPlan *p = get_plan(name, set, OP_part_size, 6, args, 4, kBresInds);
    if (!p) return;
    LoopScope ls(name, p->transfer, p->transfer2);
    PlanView v = plan_view(*p);
    int nthread = OP_block_size > 0 ? OP_block_size : 512;
    if (p->nshared > 48 * 1024)
      OP2B_CUDA(cudaFuncSetAttribute(k_bres_calc_coloured<T>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, p->nshared));
    for (int c = 0, off = 0; c < p->ncolors; off += p->ncolblk[c], c++)
      if (p->ncolblk[c] > 0)
        k_bres_calc_coloured<T><<<p->ncolblk[c], nthread, p->nshared, s>>>(
            v, off, (const T *)args[0].dat->data_d, (const T *)args[2].dat->data_d,
            (const T *)args[3].dat->data_d, (const int *)args[5].dat->data_d,
            (T *)args[4].dat->data_d, K);
    return;
  }
  GatherPlan *g = get_gather_plan(set, args, {4});
  if (!g) return;
  LoopScope ls(name, compulsory_bytes(set, 6, args), 0);
  if (g->nactive == 0) return;
  k_bres_calc_gather<T><<<(g->nactive + 255) / 256, 256, 0, s>>>(
      g->nactive, g->d_active, g->d_row, g->d_keys, idx_map(args[0]), idx_map(args[1]),
      idx_map(args[2]), idx_map(args[3]), idx_map(args[5]), (const T *)args[0].dat->data_d,
      (const T *)args[1].dat->data_d, (const T *)args[2].dat->data_d,
      (const T *)args[3].dat->data_d, (const int *)args[5].dat->data_d, (T *)args[4].dat->data_d,
      K);
}
void run_bres_calc(char const *name, op_set set, const op_arg *args) {
  if (is_double(args[0])) bres_calc_t<double>(name, set, args);
  else bres_calc_t<float>(name, set, args);
}

template <class T>
static void update_t(char const *name, op_set set, const op_arg *args) {
  cudaStream_t s = rt().stream;
  const int n = set->size;
  const bool seq = rt().reduction == OP2B_REDUCE_SEQ;
  int slot = red_new_slot();
  T *result = (T *)red_slot_ptr(slot);
  {
    LoopScope ls(name, compulsory_bytes(set, 5, args), 0);
    T *seqbuf = seq ? (T *)red_seq_buffer(sizeof(T) * 4 * (size_t)n) : nullptr;
    const int threads = 256, U = unroll();
    // fewer, fuller CTAs than the other direct loops: fewer partials for the
    // last block to fold (measured best at 4 per SM); <= kMaxRedBlocks and
    // fixed by n and U, so the sum is reproducible
    long long gw = (n + 256LL * U - 1) / (256LL * U);
    long long gcap = (long long)rt().num_sms * tuning("update_ctas_per_sm", 4);
    const int grid = (int)std::max(1LL, std::min(gw, std::min(gcap, (long long)kMaxRedBlocks)));
    RedSlot<T> rslot{(T *)red_partials(0), result};
    const T *qold = (const T *)args[0].dat->data_d, *adt = (const T *)args[3].dat->data_d;
    T *q = (T *)args[1].dat->data_d, *res = (T *)args[2].dat->data_d;
    auto launch = [&](auto kernel) {
      launch_pdl(kernel, grid, threads, 0, s, n, qold, q, res, adt, seqbuf, rslot, red_ticket());
    };
    if (U == 1) launch(k_update<T, 1>);
    else if (U == 2) launch(k_update<T, 2>);
    else launch(k_update<T, 4>);
    if (seq) {
      T init = *(const T *)args[4].data;
      k_seq_sum<T><<<1, 32, 0, s>>>(seqbuf, 4LL * n, init, result, perm_old2new_dev(set), 4);
    }
  }
  red_finish({GblRequest{args[4].data, slot, OP_INC, sizeof(T) == 8 ? GBL_F64 : GBL_F32, seq}});
}
void run_airfoil_update(char const *name, op_set set, const op_arg *args) {
  if (is_double(args[0])) update_t<double>(name, set, args);
  else update_t<float>(name, set, args);
}

// ------------------------------------------------------- fused loop pairs --
// Two consecutive op_par_loop calls run as one kernel when the second only
// reads what the first leaves unchanged, or reads it at the same element
// (loops.cpp decides; these are the kernels).  The arithmetic of each loop
// and the order of every increment are unchanged, so results are identical
// to running the two loops one after the other.

// save_soln then adt_calc over the same cells: q is read once
template <class T>
__global__ void k_save_adt(int n, const T *__restrict__ q, T *__restrict__ qold, IdxMap m0,
                           IdxMap m1, IdxMap m2, IdxMap m3, const T *__restrict__ x0,
                           const T *__restrict__ x1, const T *__restrict__ x2,
                           const T *__restrict__ x3, const T *__restrict__ q2,
                           T *__restrict__ adt, AirConsts<T> K) {
  const bool quad = m0.map && m0.map == m1.map && m0.map == m2.map && m0.map == m3.map &&
                    m0.dim == 4 && m0.idx == 0 && m1.idx == 1 && m2.idx == 2 && m3.idx == 3;
  int nd[4];
  auto nodes = [&](int c) {
    if (quad) {
      int4 v = __ldg(reinterpret_cast<const int4 *>(m0.map) + c);
      nd[0] = v.x; nd[1] = v.y; nd[2] = v.z; nd[3] = v.w;
    } else {
      nd[0] = at(m0, c); nd[1] = at(m1, c); nd[2] = at(m2, c); nd[3] = at(m3, c);
    }
  };
  const int c0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (c0 < n) nodes(c0);  // map entries: read-only, fetched early
  pdl_wait();
  pdl_trigger();
  for (int c = c0; c < n; c += gridDim.x * blockDim.x) {
    if (c != c0) nodes(c);
    T qq[4], qa[4], a[2], b[2], d[2], e[2];
    ld4(q + 4 * (size_t)c, qq);
    if (q2 != q) ld4(q2 + 4 * (size_t)c, qa);
    ld2(x0 + 2 * (size_t)nd[0], a);
    ld2(x1 + 2 * (size_t)nd[1], b);
    ld2(x2 + 2 * (size_t)nd[2], d);
    ld2(x3 + 2 * (size_t)nd[3], e);
    st4(qold + 4 * (size_t)c, qq);
    adt[c] = adt_calc(a, b, d, e, q2 != q ? qa : qq, K);
  }
}

// update then adt_calc over the same cells: adt_calc reads the q this
// thread has just written and overwrites the adt it has just read
template <class T>
__global__ void k_update_adt(int n, const T *__restrict__ qold, T *__restrict__ q,
                             T *__restrict__ res, T *__restrict__ adt, IdxMap m0, IdxMap m1,
                             IdxMap m2, IdxMap m3, const T *__restrict__ x0,
                             const T *__restrict__ x1, const T *__restrict__ x2,
                             const T *__restrict__ x3, AirConsts<T> K, RedSlot<T> slot,
                             unsigned *ticket) {
  const bool quad = m0.map && m0.map == m1.map && m0.map == m2.map && m0.map == m3.map &&
                    m0.dim == 4 && m0.idx == 0 && m1.idx == 1 && m2.idx == 2 && m3.idx == 3;
  pdl_wait();
  pdl_trigger();
  T rms = T(0);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    int nd[4];
    if (quad) {
      int4 v = __ldg(reinterpret_cast<const int4 *>(m0.map) + c);
      nd[0] = v.x; nd[1] = v.y; nd[2] = v.z; nd[3] = v.w;
    } else {
      nd[0] = at(m0, c); nd[1] = at(m1, c); nd[2] = at(m2, c); nd[3] = at(m3, c);
    }
    T qo[4], r[4], a[2], b[2], d[2], e[2];
    ld4(qold + 4 * (size_t)c, qo);
    ldw4(res + 4 * (size_t)c, r);
    const T ad = adt[c];
    ld2(x0 + 2 * (size_t)nd[0], a);
    ld2(x1 + 2 * (size_t)nd[1], b);
    ld2(x2 + 2 * (size_t)nd[2], d);
    ld2(x3 + 2 * (size_t)nd[3], e);
    // airfoil/update.h:1-12
    T adti = rcp(ad);
    T qn[4];
    for (int k = 0; k < 4; k++) {
      T del = adti * r[k];
      qn[k] = qo[k] - del;
      rms += del * del;
    }
    st4(q + 4 * (size_t)c, qn);
    const T z[4] = {T(0), T(0), T(0), T(0)};
    st4(res + 4 * (size_t)c, z);
    // airfoil/adt_calc.h on the new q
    adt[c] = adt_calc(a, b, d, e, qn, K);
  }
  const T v[1] = {rms}, id[1] = {T(0)};
  RedSlot<T> sl[1] = {slot};
  grid_finish<T, OpSum, OpSum, 1>(v, id, OpSum(), OpSum(), sl, ticket);
}

// res_calc's ordered fold followed by bres_calc's contributions to the same
// cell, in bedge order: the per-cell order of running the two loops in turn
template <class T>
__global__ void k_res_fold_bres(int nrows, const int *__restrict__ row,
                                const int *__restrict__ keys, const T *__restrict__ flux,
                                const int *__restrict__ brow, const int *__restrict__ bkeys,
                                IdxMap bx1, IdxMap bx2, IdxMap bq, IdxMap ba, IdxMap bb,
                                const T *__restrict__ xa, const T *__restrict__ xb,
                                const T *__restrict__ q, const T *__restrict__ adt,
                                const int *__restrict__ bound, T *__restrict__ res,
                                AirConsts<T> K) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nrows) return;
  T r[4];
  ldw4(res + 4 * (size_t)c, r);
  const int k1 = row[c + 1];
  constexpr int B = 4;
  for (int kb = row[c]; kb < k1; kb += B) {
    int key[B];
    T f[B][4];
#pragma unroll
    for (int b = 0; b < B; b++) key[b] = kb + b < k1 ? __ldg(keys + kb + b) : -1;
#pragma unroll
    for (int b = 0; b < B; b++)
      if (key[b] >= 0) ld4(flux + 4 * (size_t)(key[b] >> 1), f[b]);
#pragma unroll
    for (int b = 0; b < B; b++) {
      if (key[b] < 0) continue;
      if ((key[b] & 1) == 0) {
        r[0] += f[b][0]; r[1] += f[b][1]; r[2] += f[b][2]; r[3] += f[b][3];
      } else {
        r[0] -= f[b][0]; r[1] -= f[b][1]; r[2] -= f[b][2]; r[3] -= f[b][3];
      }
    }
  }
  const int j1 = brow[c + 1];
  for (int j = brow[c]; j < j1; j++) {
    const int e = __ldg(bkeys + j);
    T p[2], s[2], q1[4];
    ld2(xa + 2 * (size_t)at(bx1, e), p);
    ld2(xb + 2 * (size_t)at(bx2, e), s);
    ld4(q + 4 * (size_t)at(bq, e), q1);
    bres_apply(p, s, q1, __ldg(adt + at(ba, e)), __ldg(bound + at(bb, e)), K, r);
  }
  st4(res + 4 * (size_t)c, r);
}

// brow[c] = first bres contribution of cell c = row_b[lower_bound(active_b, c)]
__global__ void k_bres_rows(int ncell, const int *__restrict__ active_b, int nactive_b,
                            const int *__restrict__ row_b, int *brow) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncell; c += gridDim.x * blockDim.x) {
    int lo = 0, hi = nactive_b;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (active_b[mid] < c) lo = mid + 1; else hi = mid;
    }
    brow[c] = row_b[lo];
  }
}

template <class T>
static bool save_adt_t(op_set set, const op_arg *sa, const op_arg *aa) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return true;
  LoopScope ls("save_soln+adt_calc", compulsory_bytes(set, 2, sa) + compulsory_bytes(set, 6, aa), 0);
  const int n = set->size;
  launch_pdl(k_save_adt<T>, grid_for(n, 256), 256, 0, rt().stream, n,
             (const T *)sa[0].dat->data_d, (T *)sa[1].dat->data_d, idx_map(aa[0]), idx_map(aa[1]),
             idx_map(aa[2]), idx_map(aa[3]), (const T *)aa[0].dat->data_d,
             (const T *)aa[1].dat->data_d, (const T *)aa[2].dat->data_d,
             (const T *)aa[3].dat->data_d, (const T *)aa[4].dat->data_d, (T *)aa[5].dat->data_d,
             K);
  return true;
}

bool run_save_adt(op_set set, const op_arg *sa, const op_arg *aa) {
  return is_double(sa[0]) ? save_adt_t<double>(set, sa, aa) : save_adt_t<float>(set, sa, aa);
}

template <class T>
static bool update_adt_t(op_set set, const op_arg *ua, const op_arg *aa) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return true;
  cudaStream_t s = rt().stream;
  const int n = set->size;
  int slot = red_new_slot();
  T *result = (T *)red_slot_ptr(slot);
  {
    LoopScope ls("update+adt_calc", compulsory_bytes(set, 5, ua) + compulsory_bytes(set, 6, aa), 0);
    long long gw = (n + 255LL) / 256;
    long long gcap = (long long)rt().num_sms * tuning("update_ctas_per_sm", 4);
    const int grid = (int)std::max(1LL, std::min(gw, std::min(gcap, (long long)kMaxRedBlocks)));
    RedSlot<T> rslot{(T *)red_partials(0), result};
    launch_pdl(k_update_adt<T>, grid, 256, 0, s, n, (const T *)ua[0].dat->data_d,
               (T *)ua[1].dat->data_d, (T *)ua[2].dat->data_d, (T *)ua[3].dat->data_d,
               idx_map(aa[0]), idx_map(aa[1]), idx_map(aa[2]), idx_map(aa[3]),
               (const T *)aa[0].dat->data_d, (const T *)aa[1].dat->data_d,
               (const T *)aa[2].dat->data_d, (const T *)aa[3].dat->data_d, K, rslot,
               red_ticket());
  }
  red_finish({GblRequest{ua[4].data, slot, OP_INC, sizeof(T) == 8 ? GBL_F64 : GBL_F32, false}});
  return true;
}

bool run_update_adt(op_set set, const op_arg *ua, const op_arg *aa) {
  return is_double(ua[0]) ? update_adt_t<double>(set, ua, aa) : update_adt_t<float>(set, ua, aa);
}

// fused res_calc + bres_calc needs the bres contributions indexed by cell
struct BresRows {
  const GatherPlan *res = nullptr, *bres = nullptr;
  int *d_brow = nullptr;
};
static std::vector<BresRows> g_bres_rows;

void release_fused_plans() {
  for (auto &b : g_bres_rows) dev_free(b.d_brow);
  g_bres_rows.clear();
}

template <class T>
static bool res_bres_t(op_set rset, const op_arg *ra, op_set bset, const op_arg *ba) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return true;
  cudaStream_t s = rt().stream;
  GatherPlan *g = get_gather_plan(rset, ra, {6, 7});
  GatherPlan *gb = get_gather_plan(bset, ba, {4});
  if (!g || !gb) return true;
  // only when every cell is a res_calc target, so the fold covers bres's cells
  if (g->d_active || g->nactive != ra[6].dat->set->size) return false;
  const BresRows *br = nullptr;
  for (auto &b : g_bres_rows)
    if (b.res == g && b.bres == gb) br = &b;
  if (!br) {
    BresRows b{g, gb, (int *)dev_alloc(sizeof(int) * ((size_t)g->nactive + 1))};
    if (!b.d_brow) return true;
    if (gb->d_active)
      k_bres_rows<<<grid_for(g->nactive + 1, 256), 256, 0, s>>>(g->nactive, gb->d_active,
                                                                gb->nactive, gb->d_row, b.d_brow);
    else
      OP2B_CUDA(cudaMemcpyAsync(b.d_brow, gb->d_row, sizeof(int) * ((size_t)g->nactive + 1),
                                cudaMemcpyDeviceToDevice, s));
    g_bres_rows.push_back(b);
    br = &g_bres_rows.back();
  }
  const int ne = rset->size;
  const size_t need = sizeof(T) * 4 * (size_t)ne;
  if (g->contrib_bytes < need) {
    dev_free(g->d_contrib);
    g->d_contrib = dev_alloc(need);
    g->contrib_bytes = g->d_contrib ? need : 0;
    if (!g->d_contrib) return true;
  }
  T *flux = (T *)g->d_contrib;
  LoopScope ls("res_calc+bres_calc",
               compulsory_bytes(rset, 8, ra) + compulsory_bytes(bset, 6, ba), 0);
  k_res_flux<T><<<grid_for(ne, 256), 256, 0, s>>>(
      ne, idx_map(ra[0]), idx_map(ra[1]), idx_map(ra[2]), idx_map(ra[3]), idx_map(ra[4]),
      idx_map(ra[5]), (const T *)ra[0].dat->data_d, (const T *)ra[1].dat->data_d,
      (const T *)ra[2].dat->data_d, (const T *)ra[3].dat->data_d, (const T *)ra[4].dat->data_d,
      (const T *)ra[5].dat->data_d, flux, K.gm1, K.eps);
  k_res_fold_bres<T><<<(g->nactive + 255) / 256, 256, 0, s>>>(
      g->nactive, g->d_row, g->d_keys, flux, br->d_brow, gb->d_keys, idx_map(ba[0]),
      idx_map(ba[1]), idx_map(ba[2]), idx_map(ba[3]), idx_map(ba[5]),
      (const T *)ba[0].dat->data_d, (const T *)ba[1].dat->data_d, (const T *)ba[2].dat->data_d,
      (const T *)ba[3].dat->data_d, (const int *)ba[5].dat->data_d, (T *)ra[6].dat->data_d, K);
  return true;
}

bool run_res_bres(op_set rset, const op_arg *ra, op_set bset, const op_arg *ba) {
  if (tuning("gather_slots", 1) &&
      run_res_chain(nullptr, rset, ra, bset, ba, nullptr, nullptr, nullptr))
    return true;
  return is_double(ra[0]) ? res_bres_t<double>(rset, ra, bset, ba)
                          : res_bres_t<float>(rset, ra, bset, ba);
}

// the flux pass of res_calc (and bres_calc's values when B.n > 0) into vals
template <class T>
static void launch_flux(const op_arg *ra, const ResEdges<T> &E, const BresEdges<T> &B, T *vals,
                        size_t nval, const AirConsts<T> &K, cudaStream_t s) {
  const long long nflux = (long long)E.n + B.n;
  // flux_ctas_per_sm = 0: one edge per thread (many short CTAs balance the
  // SMs); n > 0: at most n CTAs per SM, grid-stride (default 16 in FP32,
  // 8 in FP64: measured 24.7 -> 23.3 us for the FP64 pass at 720k cells)
  const int per_sm = tuning("flux_ctas_per_sm", sizeof(T) == 8 ? 8 : 16);
  long long fg = (nflux + 255) / 256;
  if (per_sm > 0) fg = std::min(fg, (long long)rt().num_sms * per_sm);
  const unsigned fgrid = (unsigned)std::max(1LL, fg);
  auto pair = [](const op_arg &a, const op_arg &b) {
    return a.map && a.map == b.map && a.map->dim == 2 && a.idx == 0 && b.idx == 1;
  };
  const bool shape = pair(ra[0], ra[1]) && pair(ra[2], ra[3]) && pair(ra[4], ra[5]) &&
                     ra[2].map == ra[4].map && ra[0].dat == ra[1].dat && ra[2].dat == ra[3].dat &&
                     ra[4].dat == ra[5].dat && (long long)nval < (1LL << 30) &&
                     (long long)ra[2].dat->set->size < (1LL << 30) &&
                     (long long)ra[0].dat->set->size < (1LL << 30);
  if (shape && tuning("flux_pair", 1))
    launch_pdl(k_res_flux_pair<T>, fgrid, 256, 0, s, E.n,
               reinterpret_cast<const int2 *>(map_dev(ra[0].map)),
               reinterpret_cast<const int2 *>(map_dev(ra[2].map)), E.xa, E.qa, E.adta, B, vals, K);
  else if (tuning("flux_pipe", 0))
    launch_pdl(k_res_flux_list<T, true, sizeof(T) == 4 ? 6 : 3>, fgrid, 256, 0, s, E, B, vals, K);
  else
    launch_pdl(k_res_flux_list<T, false, sizeof(T) == 4 ? 8 : 4>, fgrid, 256, 0, s, E, B, vals, K);
}

// the persistent chain's queue for a slot plan (host side of ChainSchedDev)
struct ChainSched {
  int et = 0, ct = 0, lag = 0;
  ChainSchedDev dev;
};

void release_chain_sched(SlotPlan *sp) {
  if (!sp->chain) return;
  ChainSchedDev &d = sp->chain->dev;
  dev_free((void *)d.queue);
  dev_free((void *)d.dep_off);
  dev_free((void *)d.deps);
  dev_free(d.flags);
  dev_free(d.ctl);
  dev_free(d.partials);
  delete sp->chain;
  sp->chain = nullptr;
}

// Build (once per slot plan and tile shape) the work queue: flux tiles in
// order, each cell tile `lag` flux tiles after the last flux tile its lists
// read, and each cell tile's distinct flux tiles.  Reads the lists back to
// the host, so it runs on a loop's first call, before any capture; nullptr
// when it cannot be built or some cell tile reads more than kChainMaxDeps
// flux tiles (a numbering without locality: the caller then uses the
// two-launch chain).
static ChainSched *chain_sched(SlotPlan *sp, int et, int ct, int lag) {
  if (sp->chain && sp->chain->et == et && sp->chain->ct == ct && sp->chain->lag == lag)
    return sp->chain;
  if (sp->chain_unsuited) return nullptr;
  if (live_graphs() > 0 && sp->chain) return sp->chain;  // keep what captured graphs use
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  OP2B_CUDA(cudaStreamIsCapturing(rt().stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) return sp->chain;
  release_chain_sched(sp);
  cudaStream_t s = rt().stream;
  const int nvals = sp->na + sp->nb, ncell = sp->ntarget, W = sp->width;
  const int nflux = (nvals + et - 1) / et, ncellt = (ncell + ct - 1) / ct;
  if (nflux < 1 || ncellt < 1) return nullptr;
  std::vector<int> ell((size_t)ncell * W);
  OP2B_CUDA(cudaMemcpyAsync(ell.data(), sp->d_ell, sizeof(int) * ell.size(),
                            cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  std::vector<int> dep_off(ncellt + 1, 0), deps, last(ncellt, -1), tiles;
  for (int t = 0; t < ncellt; t++) {
    tiles.clear();
    const int c1 = std::min(ncell, (t + 1) * ct);
    for (size_t e = (size_t)t * ct * W; e < (size_t)c1 * W; e++) {
      const int v = ell[e] >> 1;
      if (v < nvals) tiles.push_back(v / et);
    }
    std::sort(tiles.begin(), tiles.end());
    tiles.erase(std::unique(tiles.begin(), tiles.end()), tiles.end());
    if ((int)tiles.size() > kChainMaxDeps) {
      sp->chain_unsuited = true;
      return nullptr;
    }
    deps.insert(deps.end(), tiles.begin(), tiles.end());
    dep_off[t + 1] = (int)deps.size();
    if (!tiles.empty()) last[t] = tiles.back();
  }
  // cell tiles by the flux tile after which they are queued (stable)
  std::vector<std::vector<int>> after(nflux);
  for (int t = 0; t < ncellt; t++)
    after[std::min(nflux - 1, std::max(last[t], 0) + lag)].push_back(t);
  std::vector<int> queue;
  queue.reserve((size_t)nflux + ncellt);
  for (int j = 0; j < nflux; j++) {
    queue.push_back(j);
    for (int t : after[j]) queue.push_back(-(t + 1));
  }
  ChainSched *cs = new ChainSched();
  cs->et = et;
  cs->ct = ct;
  cs->lag = lag;
  ChainSchedDev &d = cs->dev;
  d.nitems = (int)queue.size();
  d.nflux = nflux;
  d.ncellt = ncellt;
  d.et = et;
  d.ct = ct;
  int *d_queue = (int *)dev_alloc(sizeof(int) * queue.size());
  int *d_off = (int *)dev_alloc(sizeof(int) * dep_off.size());
  int *d_deps = (int *)dev_alloc(sizeof(int) * std::max<size_t>(1, deps.size()));
  d.queue = d_queue;
  d.dep_off = d_off;
  d.deps = d_deps;
  d.flags = (unsigned *)dev_alloc(sizeof(unsigned) * (size_t)nflux);
  d.ctl = (unsigned *)dev_alloc(4 * sizeof(unsigned));
  d.partials = dev_alloc(8 * (size_t)ncellt);
  sp->chain = cs;
  if (!d_queue || !d_off || !d_deps || !d.flags || !d.ctl || !d.partials) {
    release_chain_sched(sp);
    return nullptr;
  }
  OP2B_CUDA(cudaMemcpyAsync(d_queue, queue.data(), sizeof(int) * queue.size(),
                            cudaMemcpyHostToDevice, s));
  OP2B_CUDA(cudaMemcpyAsync(d_off, dep_off.data(), sizeof(int) * dep_off.size(),
                            cudaMemcpyHostToDevice, s));
  if (!deps.empty())
    OP2B_CUDA(cudaMemcpyAsync(d_deps, deps.data(), sizeof(int) * deps.size(),
                              cudaMemcpyHostToDevice, s));
  OP2B_CUDA(cudaMemsetAsync(d.flags, 0, sizeof(unsigned) * (size_t)nflux, s));
  OP2B_CUDA(cudaMemsetAsync(d.ctl, 0, 4 * sizeof(unsigned), s));
  OP2B_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return cs;
}

// res_calc's arguments in the airfoil shape: both x through one dim-2 map
// (idx 0, 1), q and adt through another, one dataset each, sizes that keep
// 32-bit index arithmetic
static bool flux_pair_shape(const op_arg *ra, size_t nval) {
  auto pair = [](const op_arg &a, const op_arg &b) {
    return a.map && a.map == b.map && a.map->dim == 2 && a.idx == 0 && b.idx == 1;
  };
  return pair(ra[0], ra[1]) && pair(ra[2], ra[3]) && pair(ra[4], ra[5]) &&
         ra[2].map == ra[4].map && ra[0].dat == ra[1].dat && ra[2].dat == ra[3].dat &&
         ra[4].dat == ra[5].dat && (long long)nval < (1LL << 30) &&
         (long long)ra[2].dat->set->size < (1LL << 30) &&
         (long long)ra[0].dat->set->size < (1LL << 30);
}

// the plans and value buffer of a res_calc (+ bres_calc) chain; nullptr
// when the mesh does not suit slots; *err when a plan failed
template <class T>
static SlotPlan *chain_plans(op_set rset, const op_arg *ra, op_set bset, const op_arg *ba,
                             bool *err) {
  *err = false;
  GatherPlan *g = get_gather_plan(rset, ra, {6, 7});
  GatherPlan *gb = ba ? get_gather_plan(bset, ba, {4}) : nullptr;
  if (!g || (ba && !gb)) {
    *err = true;
    return nullptr;
  }
  SlotPlan *sp = get_slot_plan(g, gb);
  if (!sp) return nullptr;
  const size_t nval = (size_t)sp->na + sp->nb + 1;
  const size_t need = sizeof(T) * 4 * nval;
  if (sp->buf_bytes < need) {
    dev_free(sp->d_buf);
    sp->d_buf = dev_alloc(need);
    sp->buf_bytes = sp->d_buf ? need : 0;
    if (!sp->d_buf) {
      *err = true;
      return nullptr;
    }
    // the padding entry, never written by the flux pass: -0.0
    k_fill<T><<<1, 32, 0, rt().stream>>>((T *)sp->d_buf + 4 * (nval - 1), 4, T(-0.0));
  }
  return sp;
}

template <class T>
static ResEdges<T> res_edges(op_set rset, const op_arg *ra) {
  return ResEdges<T>{rset->size, idx_map(ra[0]), idx_map(ra[1]), idx_map(ra[2]), idx_map(ra[3]),
                     idx_map(ra[4]), idx_map(ra[5]), (const T *)ra[0].dat->data_d,
                     (const T *)ra[1].dat->data_d, (const T *)ra[2].dat->data_d,
                     (const T *)ra[3].dat->data_d, (const T *)ra[4].dat->data_d,
                     (const T *)ra[5].dat->data_d};
}

template <class T>
static BresEdges<T> bres_edges(op_set bset, const op_arg *ba) {
  BresEdges<T> B;
  memset(&B, 0, sizeof B);
  if (ba)
    B = BresEdges<T>{bset->size, idx_map(ba[0]), idx_map(ba[1]), idx_map(ba[2]),
                     idx_map(ba[3]), idx_map(ba[5]), (const T *)ba[0].dat->data_d,
                     (const T *)ba[1].dat->data_d, (const T *)ba[2].dat->data_d,
                     (const T *)ba[3].dat->data_d, (const int *)ba[5].dat->data_d};
  return B;
}

// The flux pass of a res_calc + bres_calc chain that has not been called
// yet, with adt read from adt_now (a spare buffer about to become adt's):
// the values the chain's per-cell pass will fold, if the calls come as
// expected (the caller checks that before skipping its own flux pass)
template <class T>
static bool res_flux_ahead_t(op_set rset, const op_arg *ra, op_set bset, const op_arg *ba,
                             op_dat adt, const void *adt_now) {
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return false;
  bool err = false;
  SlotPlan *sp = chain_plans<T>(rset, ra, bset, ba, &err);
  if (!sp || err) return false;
  ResEdges<T> E = res_edges<T>(rset, ra);
  BresEdges<T> B = bres_edges<T>(bset, ba);
  if (ra[4].dat == adt) E.adta = (const T *)adt_now;
  if (ra[5].dat == adt) E.adtb = (const T *)adt_now;
  if (ba && ba[3].dat == adt) B.adt = (const T *)adt_now;
  launch_flux<T>(ra, E, B, (T *)sp->d_buf, (size_t)sp->na + sp->nb + 1, K, rt().stream);
  return true;
}

bool run_res_flux_ahead(op_set rset, const op_arg *ra, op_set bset, const op_arg *ba, op_dat adt,
                        const void *adt_now) {
  return is_double(ra[0]) ? res_flux_ahead_t<double>(rset, ra, bset, ba, adt, adt_now)
                          : res_flux_ahead_t<float>(rset, ra, bset, ba, adt, adt_now);
}

// res_calc [+ bres_calc [+ update [+ adt_calc]]] over contribution lists:
// the flux pass, then one per-cell pass that folds the cell's list and, when
// update follows, applies it (and adt_calc) to the cell before storing
// res_calc + bres_calc + update [+ adt_calc] [+ save_soln] as one persistent
// launch (k_chain_persist); false when the shapes do not suit it (the
// caller then runs the flux pass and the per-cell pass)
template <class T>
static bool persist_chain(const std::string &name, SlotPlan *sp, const op_arg *ra,
                          const ResEdges<T> &E, const BresEdges<T> &B, const op_arg *ua,
                          const op_arg *aa, const op_arg *sa, void *adt_out, void *save_out,
                          const AirConsts<T> &K, bool seq, int rslot_id, cudaStream_t s) {
  const size_t nval = (size_t)sp->na + sp->nb + 1;
  if (!tuning("chain_persist", 0) || !flux_pair_shape(ra, nval)) return false;
  if (aa && !(aa[0].map && aa[0].map == aa[1].map && aa[0].map == aa[2].map &&
              aa[0].map == aa[3].map && aa[0].map->dim == 4 && aa[0].idx == 0 &&
              aa[1].idx == 1 && aa[2].idx == 2 && aa[3].idx == 3))
    return false;
  const int U = tuning("persist_u", 1) == 2 ? 2 : 1;
  const int et = std::max(256, tuning("persist_et", 1024));
  const bool adt_calc_on = aa != nullptr, save_on = sa != nullptr;
  const void *kp;
  if (save_on)
    kp = U == 2 ? (const void *)k_chain_persist<T, true, true, 2>
                : (const void *)k_chain_persist<T, true, true, 1>;
  else if (adt_calc_on)
    kp = U == 2 ? (const void *)k_chain_persist<T, true, false, 2>
                : (const void *)k_chain_persist<T, true, false, 1>;
  else
    kp = U == 2 ? (const void *)k_chain_persist<T, false, false, 2>
                : (const void *)k_chain_persist<T, false, false, 1>;
  const int grid = std::max(1, resident_ctas(kp, 256) * rt().num_sms);
  const int lag_knob = tuning("persist_lag", -1);
  const int lag = lag_knob >= 0 ? lag_knob : grid;
  ChainSched *cs = chain_sched(sp, et, 256 * U, lag);
  if (!cs) return false;
  const int ncell = sp->ntarget;
  T *seqbuf = seq ? (T *)red_seq_buffer(sizeof(T) * 4 * (size_t)ncell) : nullptr;
  T *result = (T *)red_slot_ptr(rslot_id);
  const T *qold = (const T *)ua[0].dat->data_d;
  T *q = (T *)ua[1].dat->data_d, *adt = (T *)ua[3].dat->data_d, *res = (T *)ua[2].dat->data_d;
  CellNodes N;
  memset(&N, 0, sizeof N);
  const T *xs[4] = {nullptr, nullptr, nullptr, nullptr};
  if (aa) {
    N = CellNodes{idx_map(aa[0]), idx_map(aa[1]), idx_map(aa[2]), idx_map(aa[3])};
    for (int i = 0; i < 4; i++) xs[i] = (const T *)aa[i].dat->data_d;
  }
  T *qsave = sa ? (T *)(save_out ? save_out : sa[1].dat->data_d) : nullptr;
  T *adt_to = aa ? (T *)(adt_out ? adt_out : adt) : nullptr;
  const int2 *pedge = reinterpret_cast<const int2 *>(map_dev(ra[0].map));
  const int2 *pecell = reinterpret_cast<const int2 *>(map_dev(ra[2].map));
  {
    PhaseScope ph(name + ":persist");
    auto go = [&](auto kernel) {
      launch_pdl(kernel, grid, 256, 0, s, cs->dev, E.n, pedge, pecell, E.xa, E.qa, E.adta, B,
                 (T *)sp->d_buf, ncell, (const int *)sp->d_ell, sp->width, qold, q, res,
                 (const T *)adt, N, xs[0], xs[1], xs[2], xs[3], K, seqbuf, result, qsave, adt_to);
    };
    if (save_on) {
      if (U == 2) go(k_chain_persist<T, true, true, 2>);
      else go(k_chain_persist<T, true, true, 1>);
    } else if (adt_calc_on) {
      if (U == 2) go(k_chain_persist<T, true, false, 2>);
      else go(k_chain_persist<T, true, false, 1>);
    } else {
      if (U == 2) go(k_chain_persist<T, false, false, 2>);
      else go(k_chain_persist<T, false, false, 1>);
    }
  }
  if (seq) {
    T init = *(const T *)ua[4].data;
    k_seq_sum<T><<<1, 32, 0, s>>>(seqbuf, 4LL * ncell, init, result,
                                  perm_old2new_dev(ra[6].dat->set), 4);
  }
  return true;
}

// ------------------------------------------------ tiled res_calc chain ----
// res_calc + bres_calc + update [+ adt_calc] [+ save_soln] as ONE launch
// with no wait between CTAs: the cells are cut into tiles of consecutive
// cells, and a CTA takes a whole tile.  It computes the flux of every edge
// and boundary edge in its cells' lists into shared memory (an edge whose
// two cells lie in different tiles is computed by both tiles, with the same
// arithmetic, so both get the same value), then folds each cell's list from
// there in list order, applies update and adt_calc to the cell, and stores.
// The flux reads q and adt of cells of other tiles, which those tiles update
// in the same launch: update writes the new q, and adt_calc the new adt,
// into a second buffer of each dataset, which becomes the dataset's when
// the launch has been queued (the old one becomes the second buffer).
// Nothing else changes: each cell's fold, update and adt_calc are those of
// k_fold_update, each flux that of k_res_flux_pair, so q, res, adt and qold
// are bit-identical; only the order of the TREE rms sum follows the grid.
//
// The tile plan (per slot plan, built on the device): every list entry gives
// the key (tile << 32 | flux index); the sorted, de-duplicated keys are each
// tile's flux list in ascending flux order (toff: where each tile's run
// starts), and each cell's list is rewritten as (slot in its tile's run << 1
// | side).
struct TilePlan {
  int want = 0;  // the tile size asked for (tl.ct is smaller when that did not fit)
  TileLists tl;
};

static void free_tile_plan(TilePlan *tp) {
  if (!tp) return;
  free_tile_lists(&tp->tl, rt().stream);
  delete tp;
}

void release_tile_plan(SlotPlan *sp) {
  free_tile_plan(sp->tile);
  sp->tile = nullptr;
}

__global__ void k_tile_keys(const int *__restrict__ ell, int W, int ncell, int ct, long long m,
                            unsigned long long *key) {
  const long long n = (long long)ncell * W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned long long k = ~0ull;
    if (i < n) {
      const int e = ell[i];
      if (e >= 0) k = ((unsigned long long)(unsigned)((int)(i / W) / ct) << 32) | (unsigned)(e >> 1);
    }
    key[i] = k;
  }
}

// 1 at the first of each run of equal (valid) keys
__global__ void k_tile_first(const unsigned long long *__restrict__ key, int n, int *flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flag[i] = key[i] != ~0ull && (i == 0 || key[i] != key[i - 1]);
}

// the distinct keys' flux indices in order; toff[t] = position of tile t's
// first key for every tile after the previous key's tile (toff holds the
// total beforehand, for tiles past the last key)
__global__ void k_tile_place(const unsigned long long *__restrict__ key,
                             const int *__restrict__ flag, const int *__restrict__ pos, int n,
                             int *tflux, int *toff) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const int p = pos[i], t = (int)(key[i] >> 32);
    tflux[p] = (int)(unsigned)(key[i] & 0xffffffffull);
    const int prev = i == 0 ? -1 : (int)(key[i - 1] >> 32);
    for (int u = prev + 1; u <= t; u++) toff[u] = p;
  }
}

// toff[0..ntile] = the number of distinct keys (pos and flag of the last key)
__global__ void k_tile_total(const int *__restrict__ flag, const int *__restrict__ pos, int n,
                             int ntile, int *toff) {
  const int total = pos[n - 1] + flag[n - 1];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntile; t += gridDim.x * blockDim.x)
    toff[t] = total;
}

// *out = the longest tile run (one CTA)
__global__ void k_tile_longest(const int *__restrict__ toff, int ntile, int *out) {
  __shared__ int best;
  if (threadIdx.x == 0) best = 0;
  __syncthreads();
  int m = 0;
  for (int t = threadIdx.x; t < ntile; t += blockDim.x) m = max(m, toff[t + 1] - toff[t]);
  atomicMax(&best, m);
  __syncthreads();
  if (threadIdx.x == 0) *out = best;
}

// each list entry as its slot in the tile's flux run (binary search)
__global__ void k_tile_lists(const int *__restrict__ ell, int W, int ncell, int ct,
                             const int *__restrict__ toff, const int *__restrict__ tflux,
                             int *tell) {
  const long long n = (long long)ncell * W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int e = ell[i];
    if (e < 0) {
      tell[i] = -1;
      continue;
    }
    const int t = (int)(i / W) / ct, f = e >> 1;
    int lo = toff[t], hi = toff[t + 1];
    const int base = lo;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (tflux[mid] < f) lo = mid + 1;
      else hi = mid;
    }
    tell[i] = ((lo - base) << 1) | (e & 1);
  }
}

// Tile lists for tiles of ct consecutive cells over the contribution lists
// ell (ncell x W entries, (index << 1 | side)): device arrays from the pool,
// allocated and built on stream s, which this synchronises (it reads the
// tile offsets back for the largest tile).  False when they cannot be built.
bool build_tile_lists(const int *ell, int ncell, int W, int ct, cudaStream_t s, TileLists *out) {
  *out = TileLists();
  const long long n = (long long)ncell * W;
  if (ncell < 1 || W < 1 || ct < 1 || n >= (1LL << 31)) return false;
  const int ntile = (ncell + ct - 1) / ct;
  long long m = 1;
  while (m < n) m <<= 1;
  unsigned long long *key = nullptr;
  int *flag = nullptr, *pos = nullptr;
  TileLists tl;
  tl.ct = ct;
  tl.ntile = ntile;
  bool ok = pool_malloc_async((void **)&key, sizeof(unsigned long long) * m, s) == cudaSuccess &&
            pool_malloc_async((void **)&flag, sizeof(int) * n, s) == cudaSuccess &&
            pool_malloc_async((void **)&pos, sizeof(int) * n, s) == cudaSuccess &&
            pool_malloc_async((void **)&tl.toff, sizeof(int) * (ntile + 1), s) == cudaSuccess &&
            pool_malloc_async((void **)&tl.tell, sizeof(int) * n, s) == cudaSuccess;
  if (!ok) cudaGetLastError();
  const int g = rt().num_sms * 8;
  std::vector<int> toff(ntile + 1);
  if (ok) {
    k_tile_keys<<<g, 256, 0, s>>>(ell, W, ncell, ct, m, key);
    ok = sort_keys_u64(key, m, s);
  }
  if (ok) {
    k_tile_first<<<g, 256, 0, s>>>(key, (int)n, flag);
    const long long total = exclusive_scan(flag, pos, (int)n, s);
    ok = total < (1LL << 30) &&
         pool_malloc_async((void **)&tl.tflux, sizeof(int) * std::max(1LL, total), s) ==
             cudaSuccess;
    if (ok) {
      std::fill(toff.begin(), toff.end(), (int)total);
      OP2B_CUDA(cudaMemcpyAsync(tl.toff, toff.data(), sizeof(int) * (ntile + 1),
                                cudaMemcpyHostToDevice, s));
      k_tile_place<<<g, 256, 0, s>>>(key, flag, pos, (int)n, tl.tflux, tl.toff);
      k_tile_lists<<<g, 256, 0, s>>>(ell, W, ncell, ct, tl.toff, tl.tflux, tl.tell);
      OP2B_CUDA(cudaMemcpyAsync(toff.data(), tl.toff, sizeof(int) * (ntile + 1),
                                cudaMemcpyDeviceToHost, s));
    } else {
      cudaGetLastError();
    }
  }
  for (void *p : {(void *)key, (void *)flag, (void *)pos})
    if (p) cudaFreeAsync(p, s);
  OP2B_CUDA(cudaStreamSynchronize(s));
  if (ok && !error_pending()) {
    for (int t = 0; t < ntile; t++) tl.maxcnt = std::max(tl.maxcnt, toff[t + 1] - toff[t]);
    *out = tl;
    return true;
  }
  free_tile_lists(&tl, s);
  return false;
}

// The same lists queued on stream s with no host wait: the flux runs get
// room for every list entry, and the longest run is left in tl->d_longest
// (read it with tile_lists_longest once s has run them).  False when the
// memory cannot be had.
bool build_tile_lists_async(const int *ell, int ncell, int W, int ct, cudaStream_t s,
                            TileLists *out) {
  *out = TileLists();
  const long long n = (long long)ncell * W;
  if (ncell < 1 || W < 1 || ct < 1 || n >= (1LL << 30)) return false;
  const int ntile = (ncell + ct - 1) / ct;
  long long m = 1;
  while (m < n) m <<= 1;
  unsigned long long *key = nullptr;
  int *flag = nullptr, *pos = nullptr;
  TileLists tl;
  tl.ct = ct;
  tl.ntile = ntile;
  tl.maxcnt = -1;  // in d_longest
  bool ok = pool_malloc_async((void **)&key, sizeof(unsigned long long) * m, s) == cudaSuccess &&
            pool_malloc_async((void **)&flag, sizeof(int) * n, s) == cudaSuccess &&
            pool_malloc_async((void **)&pos, sizeof(int) * n, s) == cudaSuccess &&
            pool_malloc_async((void **)&tl.toff, sizeof(int) * (ntile + 1), s) == cudaSuccess &&
            pool_malloc_async((void **)&tl.tell, sizeof(int) * n, s) == cudaSuccess &&
            pool_malloc_async((void **)&tl.tflux, sizeof(int) * n, s) == cudaSuccess &&
            pool_malloc_async((void **)&tl.d_longest, sizeof(int), s) == cudaSuccess;
  if (!ok) cudaGetLastError();
  const int g = rt().num_sms * 8;
  if (ok) {
    k_tile_keys<<<g, 256, 0, s>>>(ell, W, ncell, ct, m, key);
    ok = sort_keys_u64(key, m, s);
  }
  if (ok) {
    k_tile_first<<<g, 256, 0, s>>>(key, (int)n, flag);
    exclusive_scan_nosync(flag, pos, (int)n, s);
    k_tile_total<<<std::max(1, (ntile + 256) / 256), 256, 0, s>>>(flag, pos, (int)n, ntile, tl.toff);
    k_tile_place<<<g, 256, 0, s>>>(key, flag, pos, (int)n, tl.tflux, tl.toff);
    k_tile_lists<<<g, 256, 0, s>>>(ell, W, ncell, ct, tl.toff, tl.tflux, tl.tell);
    k_tile_longest<<<1, 1024, 0, s>>>(tl.toff, ntile, tl.d_longest);
  }
  for (void *p : {(void *)key, (void *)flag, (void *)pos})
    if (p) cudaFreeAsync(p, s);
  if (ok && !error_pending()) {
    *out = tl;
    return true;
  }
  free_tile_lists(&tl, s);
  return false;
}

// the longest run of lists built by build_tile_lists_async (waits for s)
int tile_lists_longest(TileLists *tl, cudaStream_t s) {
  if (tl->maxcnt < 0 && tl->d_longest) {
    int v = 0;
    OP2B_CUDA(cudaMemcpyAsync(&v, tl->d_longest, sizeof(int), cudaMemcpyDeviceToHost, s));
    OP2B_CUDA(cudaStreamSynchronize(s));
    tl->maxcnt = v;
  }
  return tl->maxcnt;
}

void free_tile_lists(TileLists *tl, cudaStream_t s) {
  for (void *p : {(void *)tl->toff, (void *)tl->tflux, (void *)tl->tell, (void *)tl->d_longest})
    if (p) cudaFreeAsync(p, s);
  *tl = TileLists();
}

// the plain path's tile plan for tiles of ct cells; nullptr when it cannot
// be built (synchronises: a loop's first call, never inside a capture)
static TilePlan *build_tile_plan(const SlotPlan *sp, int ct) {
  TilePlan *tp = new TilePlan();
  if (build_tile_lists((const int *)sp->d_ell, sp->ntarget, sp->width, ct, rt().stream, &tp->tl))
    return tp;
  delete tp;
  return nullptr;
}

struct TileView {
  int ct, ntile, W;
  const int *toff, *tflux, *tell;
};

template <class T, bool ADT, bool SAVE, int BS>
__global__ void __launch_bounds__(BS, 1024 / BS)
    k_chain_tiled(TileView P, int ne, const int2 *__restrict__ pedge,
                  const int2 *__restrict__ pecell, const T *__restrict__ x,
                  const T *__restrict__ q, const T *__restrict__ adt, BresEdges<T> B, int ncell,
                  const T *qold, T *__restrict__ qout, T *__restrict__ res,
                  const int4 *__restrict__ pcell, const T *__restrict__ xc, AirConsts<T> K,
                  T *seq, RedSlot<T> slot, unsigned *ticket, T *qsave, T *__restrict__ adt_out) {
  extern __shared__ __align__(16) unsigned char tile_smem[];
  T *fv = reinterpret_cast<T *>(tile_smem);  // [maxcnt][4]
  T rms = T(0);
  auto bres = [&](int b, T (&r)[4]) {
    int m1, m2;
    at2(B.x1, B.x2, b, m1, m2);
    T p[2], sx[2], q1[4];
    ld2(B.xa + 2 * (size_t)m1, p);
    ld2(B.xb + 2 * (size_t)m2, sx);
    ld4(B.q_d + 4 * (size_t)at(B.q, b), q1);
    bres_contrib(p, sx, q1, __ldg(B.adt + at(B.a, b)), __ldg(B.bound_d + at(B.bound, b)), K, r);
  };
  for (int t = blockIdx.x; t < P.ntile; t += gridDim.x) {
    const int beg = __ldg(P.toff + t), cnt = __ldg(P.toff + t + 1) - beg;
    // plan data, so the first tile's indices are staged before the previous
    // kernel has finished
    tile_stage<T, BS>(P.tflux, beg, cnt, fv);
    if (t == (int)blockIdx.x) {
      pdl_wait();
      pdl_trigger();
    }
    __syncthreads();
    tile_fluxes<T, BS>(cnt, (unsigned)ne, (unsigned)B.n, pedge, pecell, x, q, adt, K, fv, bres);
    __syncthreads();
    rms += tile_cells<T, ADT, SAVE, BS>(t * P.ct, min(ncell, (t + 1) * P.ct), P.tell, P.W, pcell,
                                        xc, qold, adt, qout, res, qsave, adt_out, seq, K, fv);
    __syncthreads();  // the next tile reuses the shared values
  }
  if (seq) return;
  const T v[1] = {rms}, id[1] = {T(0)};
  RedSlot<T> sl[1] = {slot};
  grid_finish<T, OpSum, OpSum, 1>(v, id, OpSum(), OpSum(), sl, ticket);
}

// The second buffers of datasets the tiled chain writes (by dataset index),
// and the swaps made while a graph is being captured (a graph must leave
// each dataset in the buffer it found it in: an odd count is undone at the
// end of the capture by a copy inside the graph).
static std::vector<void *> g_alt;
static std::vector<int> g_alt_flips;
static unsigned long long g_tiled_launches = 0;  // tiled chain launches queued or captured
static unsigned long long g_res_skips = 0;  // chain launches that skipped reading res

void *alt_of(op_dat d) {
  if (g_alt.size() <= (size_t)d->index) g_alt.resize(d->index + 1, nullptr);
  if (!g_alt[d->index]) g_alt[d->index] = dev_alloc((size_t)d->size * d->set->size);
  return g_alt[d->index];
}

void flip(op_dat d, bool capturing) {
  std::swap(d->data_d, reinterpret_cast<char *&>(g_alt[d->index]));
  if (capturing) {
    if (g_alt_flips.size() <= (size_t)d->index) g_alt_flips.resize(d->index + 1, 0);
    g_alt_flips[d->index]++;
  }
}

void tile_capture_begin() { g_alt_flips.clear(); }

void tile_capture_end() {  // still capturing: the copies become graph nodes
  for (size_t i = 0; i < g_alt_flips.size(); i++) {
    if (!(g_alt_flips[i] & 1)) continue;
    op_dat d = OP_dat_list[i];
    OP2B_CUDA(cudaMemcpyAsync(g_alt[i], d->data_d, (size_t)d->size * d->set->size,
                              cudaMemcpyDeviceToDevice, rt().stream));
    std::swap(d->data_d, reinterpret_cast<char *&>(g_alt[i]));
  }
  g_alt_flips.clear();
}

void release_tile_alts() {
  for (void *p : g_alt) dev_free(p);
  g_alt.clear();
  g_alt_flips.clear();
}

// res_calc + bres_calc + update [+ adt_calc] [+ save_soln] as one tiled
// launch; false when it does not apply (the caller runs the two passes)
// a kernel just launched skipped reading d, known zero; inside a capture,
// when the zeros come from before it, the graph records the kernel
// (read_kernel, read_grid: the kernel and grid that read d instead, or
// nullptr when the kernel itself reads d when given its buffer)
static void zero_entry(op_dat d, int arg, int nparams, const void *read_kernel = nullptr,
                       int read_grid = 0) {
  g_res_skips++;
  if (known_zero_from_before_capture(d))
    capture_zero_entry(d, arg, nparams, d->data_d, read_kernel, read_grid);
}

template <class T>
static bool tiled_chain(const std::string &name, SlotPlan *sp, const op_arg *ra,
                        const op_arg *ba, const ResEdges<T> &E, const BresEdges<T> &B,
                        const op_arg *ua, const op_arg *aa, const op_arg *sa, void *adt_out,
                        void *save_out, const AirConsts<T> &K, bool seq, int rslot_id,
                        cudaStream_t s, bool skip_res) {
  const size_t nval = (size_t)sp->na + sp->nb + 1;
  if (!tuning("chain_tiled", 0) || !flux_pair_shape(ra, nval) || sp->tile_unsuited) return false;
  // CTAs of 1024 threads (one per SM) or 512 (two per SM, each on its own tile)
  const int threads = tuning("tile_threads", 1024) == 512 ? 512 : 1024;
  const int per_sm = 1024 / threads;
  op_dat q = ua[1].dat, adt = ua[3].dat;
  // the flux reads q and adt -- the datasets update and adt_calc write, into
  // second buffers -- and must read nothing else the cell phase writes
  // (res in place, save_soln's output)
  if (ra[2].dat != q || ra[4].dat != adt || ra[0].dat == q || ra[0].dat == adt) return false;
  if (aa && !(aa[0].map && aa[0].map == aa[1].map && aa[0].map == aa[2].map &&
              aa[0].map == aa[3].map && aa[0].map->dim == 4 && aa[0].idx == 0 &&
              aa[1].idx == 1 && aa[2].idx == 2 && aa[3].idx == 3 && aa[0].dat == aa[1].dat &&
              aa[0].dat == aa[2].dat && aa[0].dat == aa[3].dat && aa[5].dat == adt &&
              aa[4].dat == q))
    return false;
  {
    const op_dat written[2] = {ua[2].dat, sa && !save_out ? sa[1].dat : nullptr};
    std::vector<op_dat> read = {ra[0].dat, q, adt};
    if (aa) read.push_back(aa[0].dat);
    if (ba)
      for (int i : {0, 1, 2, 3, 5}) read.push_back(ba[i].dat);
    for (op_dat r : read)
      if (r == written[0] || (written[1] && r == written[1])) return false;
    if (written[1] && (written[1] == q || written[1] == adt)) return false;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  OP2B_CUDA(cudaStreamIsCapturing(s, &cap));
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  // a graph holds the buffers it was captured with: no swaps between launches
  if (!capturing && live_graphs() > 0) return false;
  const int ncell = sp->ntarget;
  const size_t static_smem = 1024,
               budget = (size_t)rt().smem_optin / per_sm - static_smem;
  // tile size: the knob, else one tile per resident CTA; shrunk until a
  // tile's fluxes fit the CTA's shared memory
  const long long ctas = (long long)rt().num_sms * per_sm;
  const int want = tuning("tile_cells", 0) > 0
                       ? tuning("tile_cells", 0)
                       : (int)std::max(64LL, (ncell + ctas - 1) / ctas);
  if (!sp->tile || sp->tile->want != want ||
      (size_t)sp->tile->tl.maxcnt * 4 * sizeof(T) > budget) {
    if (capturing) return false;  // plans are built before a capture
    release_tile_plan(sp);
    for (int ct = want;; ct = ct * 3 / 4) {
      if (ct < 16) {
        sp->tile_unsuited = true;
        return false;
      }
      TilePlan *tp = build_tile_plan(sp, ct);
      if (!tp) {
        sp->tile_unsuited = true;
        return false;
      }
      if ((size_t)tp->tl.maxcnt * 4 * sizeof(T) <= budget) {
        tp->want = want;
        sp->tile = tp;
        break;
      }
      free_tile_plan(tp);
    }
  }
  TilePlan *tp = sp->tile;
  const size_t smem = (size_t)tp->tl.maxcnt * 4 * sizeof(T);
  void *qout = alt_of(q);
  void *adt_to = nullptr;
  bool flip_adt = false;
  if (aa) {
    adt_to = adt_out;
    if (!adt_to) {
      adt_to = alt_of(adt);
      flip_adt = true;
    }
  }
  if (!qout || (aa && !adt_to) || error_pending()) return false;
  const void *kp =
      threads == 512
          ? (sa ? (const void *)k_chain_tiled<T, true, true, 512>
                : aa ? (const void *)k_chain_tiled<T, true, false, 512>
                     : (const void *)k_chain_tiled<T, false, false, 512>)
          : (sa ? (const void *)k_chain_tiled<T, true, true, 1024>
                : aa ? (const void *)k_chain_tiled<T, true, false, 1024>
                     : (const void *)k_chain_tiled<T, false, false, 1024>);
  static size_t sized[2][2][3] = {};
  size_t &have = sized[sizeof(T) == 8][threads == 512][sa ? 2 : aa ? 1 : 0];
  if (smem > have) {
    OP2B_CUDA(cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    have = smem;
  }
  T *seqbuf = seq ? (T *)red_seq_buffer(sizeof(T) * 4 * (size_t)ncell) : nullptr;
  T *result = (T *)red_slot_ptr(rslot_id);
  RedSlot<T> rslot{(T *)red_partials(0), result};
  const int grid = std::min(tp->tl.ntile, std::min(kMaxRedBlocks, rt().num_sms * per_sm));
  TileView P{tp->tl.ct, tp->tl.ntile, sp->width, tp->tl.toff, tp->tl.tflux, tp->tl.tell};
  const T *xc = aa ? (const T *)aa[0].dat->data_d : nullptr;
  const int4 *pcell = aa ? reinterpret_cast<const int4 *>(map_dev(aa[0].map)) : nullptr;
  T *qsave = sa ? (T *)(save_out ? save_out : sa[1].dat->data_d) : nullptr;
  {
    PhaseScope ph(name + ":tiled");
    auto go = [&](auto kernel) {
      launch_pdl(kernel, grid, threads, smem, s, P, E.n,
                 reinterpret_cast<const int2 *>(map_dev(ra[0].map)),
                 reinterpret_cast<const int2 *>(map_dev(ra[2].map)), E.xa, E.qa, E.adta, B,
                 ncell, (const T *)ua[0].dat->data_d, (T *)qout,
                 skip_res ? (T *)nullptr : (T *)ua[2].dat->data_d, pcell, xc, K, seqbuf, rslot,
                 red_ticket(), qsave, (T *)adt_to);
      if (skip_res) zero_entry(ua[2].dat, 11, kernel_nparams(kernel));
    };
    if (threads == 512) {
      if (sa) go(k_chain_tiled<T, true, true, 512>);
      else if (aa) go(k_chain_tiled<T, true, false, 512>);
      else go(k_chain_tiled<T, false, false, 512>);
    } else {
      if (sa) go(k_chain_tiled<T, true, true, 1024>);
      else if (aa) go(k_chain_tiled<T, true, false, 1024>);
      else go(k_chain_tiled<T, false, false, 1024>);
    }
  }
  if (error_pending()) return true;
  g_tiled_launches++;
  flip(q, capturing);
  if (flip_adt) flip(adt, capturing);
  if (seq) {
    T init = *(const T *)ua[4].data;
    k_seq_sum<T><<<1, 32, 0, s>>>(seqbuf, 4LL * ncell, init, result,
                                  perm_old2new_dev(ra[6].dat->set), 4);
  }
  return true;
}

template <class T>
static bool res_chain_t(char const *loop_name, op_set rset, const op_arg *ra, op_set bset,
                        const op_arg *ba, const op_arg *ua, const op_arg *aa, const op_arg *sa,
                        void *adt_out, void *save_out, bool flux_done,
                        std::vector<GblRequest> *held, bool res_zero) {
  // save_soln rides on the one-cell-per-thread fold + update + adt_calc forms
  const int fvar = tuning("fold_variant", 0);
  if (sa && (!ua || !aa || (fvar != 0 && fvar != 4 && fvar != 5))) return false;
  AirConsts<T> K = air_consts<T>();
  if (error_pending()) return true;
  cudaStream_t s = rt().stream;
  bool err = false;
  SlotPlan *sp = chain_plans<T>(rset, ra, bset, ba, &err);
  if (err) return true;
  if (!sp) return false;
  const int W = sp->width, ncell = sp->ntarget;
  const size_t nval = (size_t)sp->na + sp->nb + 1;
  T *vals = (T *)sp->d_buf;

  std::string name = loop_name ? loop_name : "res_calc";
  double bytes = compulsory_bytes(rset, 8, ra);
  if (ba) name += "+bres_calc", bytes += compulsory_bytes(bset, 6, ba);
  if (ua) name += "+update", bytes += compulsory_bytes(ra[6].dat->set, 5, ua);
  if (sa) name += "+save_soln", bytes += compulsory_bytes(ra[6].dat->set, 2, sa);
  if (aa) name += "+adt_calc", bytes += compulsory_bytes(ra[6].dat->set, 6, aa);
  const bool seq = ua && rt().reduction == OP2B_REDUCE_SEQ;
  // res held +0.0 everywhere when res_calc was called: the fold's sums start
  // from +0.0 in registers, and res is neither read nor rewritten
  const bool skip_res = res_zero && ua && ua[2].dat == ra[6].dat && tuning("known_zero", 1);
  int rslot_id = ua ? red_new_slot() : -1;
  {
    LoopScope ls(name.c_str(), bytes, 0);
    ResEdges<T> E = res_edges<T>(rset, ra);
    BresEdges<T> B = bres_edges<T>(bset, ba);
    if (ua && !flux_done && ua[2].dat == ra[6].dat &&
        tiled_chain<T>(name, sp, ra, ba, E, B, ua, aa, sa, adt_out, save_out, K, seq, rslot_id,
                       s, skip_res))
      goto chained;
    if (ua && !flux_done && ua[2].dat == ra[6].dat &&
        persist_chain<T>(name, sp, ra, E, B, ua, aa, sa, adt_out, save_out, K, seq, rslot_id, s))
      goto chained;
    if (!flux_done) {
      PhaseScope ph(name + ":flux");
      launch_flux<T>(ra, E, B, vals, nval, K, s);
    }
    {
    PhaseScope ph(name + ":fold");
    T *res = (T *)ra[6].dat->data_d;
    if (!ua) {
      launch_pdl(k_res_fold_list<T>, grid_for(ncell, 256), 256, 0, s, ncell,
                 (const int *)sp->d_ell, W, (const T *)vals, res);
    } else {
      T *seqbuf = seq ? (T *)red_seq_buffer(sizeof(T) * 4 * (size_t)ncell) : nullptr;
      // one wave of grid-stride CTAs: as many as the kernel keeps resident
      // on every SM at once (fewer, longer CTAs beat one cell per thread --
      // each CTA ends with a block reduction and a ticket -- and a second
      // wave of CTAs starting late leaves SMs idle at the end: measured
      // 25.6 -> 21.3 us for the fold + update + adt_calc at 720k cells).
      // The grid depends only on ncell and the kernel, so sums reproduce.
      // Knob > 0: that many CTAs per SM; 0: one cell per thread
      const long long gw = (ncell + 255LL) / 256;
      const int per_sm = aa ? tuning("fold_adt_ctas_per_sm", -1) : tuning("fold_ctas_per_sm", -1);
      auto grid_of = [&](const void *kernel) {
        long long per = per_sm;
        if (per < 0) per = resident_ctas(kernel, 256);
        long long gcap = per > 0 ? (long long)rt().num_sms * per : (long long)kMaxRedBlocks;
        return (int)std::max(1LL, std::min(gw, std::min(gcap, (long long)kMaxRedBlocks)));
      };
      T *result = (T *)red_slot_ptr(rslot_id);
      RedSlot<T> rslot{(T *)red_partials(0), result};
      const T *qold = (const T *)ua[0].dat->data_d;
      T *q = (T *)ua[1].dat->data_d, *adt = (T *)ua[3].dat->data_d;
      CellNodes N;
      memset(&N, 0, sizeof N);
      const T *xs[4] = {nullptr, nullptr, nullptr, nullptr};
      if (aa) {
        N = CellNodes{idx_map(aa[0]), idx_map(aa[1]), idx_map(aa[2]), idx_map(aa[3])};
        for (int i = 0; i < 4; i++) xs[i] = (const T *)aa[i].dat->data_d;
      }
      // fold_variant: 0 one cell per thread at >= 5 CTAs per SM (4 with
      // adt_calc; FP64 2), measured best; 1 the same at >= 6; 2 two cells
      // per thread; 3 two cells at >= 3 CTAs per SM; 4 one cell per thread
      // at >= 4 (3 with adt_calc; FP64 3); 5 one cell per thread, the
      // cell's own streams fetched a cell ahead
      T *qsave = sa ? (T *)(save_out ? save_out : sa[1].dat->data_d) : nullptr;
      T *adt_to = aa ? (T *)adt_out : nullptr;
      // kr reads res; ks, the same kernel for res known zero, neither reads
      // nor rewrites it (no branch per cell).  A graph captured with ks
      // also records kr, for launches at which res may not be zero
      auto launch = [&](auto kr, auto ks) {
        const bool skip = skip_res;
        auto kernel = skip ? ks : kr;
        launch_pdl(kernel, grid_of((const void *)kernel), 256, 0, s, ncell,
                   (const int *)sp->d_ell, W, (const T *)vals,
                   qold, q, skip ? (T *)nullptr : res, adt, N, xs[0], xs[1], xs[2], xs[3],
                   K, seqbuf, rslot, red_ticket(), qsave, adt_to);
        if (skip)
          zero_entry(ra[6].dat, 6, kernel_nparams(kernel), (const void *)kr,
                     grid_of((const void *)kr));
      };
      const int fv = fvar;
#define OP2B_FOLD(...) launch(k_fold_update<__VA_ARGS__>, k_fold_update<__VA_ARGS__, true>)
#define OP2B_FOLD_PF(...) launch(k_fold_update_pf<__VA_ARGS__>, k_fold_update_pf<__VA_ARGS__, true>)
      if (sa) {
        if (fv == 4) OP2B_FOLD(T, true, 1, 3, true);
        else if (fv == 5) OP2B_FOLD_PF(T, true, sizeof(T) == 4 ? 3 : 2, true);
        else OP2B_FOLD(T, true, 1, sizeof(T) == 4 ? 4 : 2, true);
      } else if (aa) {
        if (fv == 1) OP2B_FOLD(T, true, 1, 6, false);
        else if (fv == 2) OP2B_FOLD(T, true, 2, 1, false);
        else if (fv == 3) OP2B_FOLD(T, true, 2, 3, false);
        else if (fv == 4) OP2B_FOLD(T, true, 1, 3, false);
        else if (fv == 5) OP2B_FOLD_PF(T, true, sizeof(T) == 4 ? 3 : 2, false);
        else OP2B_FOLD(T, true, 1, sizeof(T) == 4 ? 4 : 2, false);
      } else {
        if (fv == 1) OP2B_FOLD(T, false, 1, 6, false);
        else if (fv == 2) OP2B_FOLD(T, false, 2, 1, false);
        else if (fv == 3) OP2B_FOLD(T, false, 2, 3, false);
        else if (fv == 4) OP2B_FOLD(T, false, 1, sizeof(T) == 4 ? 4 : 3, false);
        else if (fv == 5) OP2B_FOLD_PF(T, false, sizeof(T) == 4 ? 4 : 2, false);
        else OP2B_FOLD(T, false, 1, sizeof(T) == 4 ? 5 : 2, false);
      }
#undef OP2B_FOLD
#undef OP2B_FOLD_PF
      if (seq) {
        T init = *(const T *)ua[4].data;
        k_seq_sum<T><<<1, 32, 0, s>>>(seqbuf, 4LL * ncell, init, result,
                                  perm_old2new_dev(ra[6].dat->set), 4);
      }
    }
    }
  chained:;
  }
  // every update zeroes res, whichever form ran
  if (ua && ua[2].dat == ra[6].dat && !error_pending()) dat_set_known_zero(ra[6].dat, true);
  if (ua) {
    GblRequest rq{ua[4].data, rslot_id, OP_INC, sizeof(T) == 8 ? GBL_F64 : GBL_F32, seq};
    if (held) held->push_back(rq);  // the caller delivers it
    else red_finish({rq});
  }
  return true;
}

unsigned wait_timeouts(bool reset) {
  unsigned v = 0;
  if (!rt().cuda_ready) return 0;
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  OP2B_CUDA(cudaMemcpyFromSymbol(&v, g_wait_timeouts, sizeof v));
  if (reset) {
    const unsigned z = 0;
    OP2B_CUDA(cudaMemcpyToSymbol(g_wait_timeouts, &z, sizeof z));
  }
  return v;
}

bool run_res_chain(char const *name, op_set rset, const op_arg *ra, op_set bset,
                   const op_arg *ba, const op_arg *ua, const op_arg *aa, const op_arg *sa,
                   void *adt_out, void *save_out, bool flux_done,
                   std::vector<GblRequest> *held, bool res_zero) {
  return is_double(ra[0]) ? res_chain_t<double>(name, rset, ra, bset, ba, ua, aa, sa, adt_out,
                                                save_out, flux_done, held, res_zero)
                          : res_chain_t<float>(name, rset, ra, bset, ba, ua, aa, sa, adt_out,
                                               save_out, flux_done, held, res_zero);
}

}  // namespace op2b

extern "C" unsigned op2b_wait_timeouts(int reset) { return op2b::wait_timeouts(reset != 0); }

extern "C" unsigned long long op2b_res_skips(int reset) {
  const unsigned long long n = op2b::g_res_skips;
  if (reset) op2b::g_res_skips = 0;
  return n;
}

extern "C" unsigned long long op2b_tiled_launches(int reset) {
  const unsigned long long n = op2b::g_tiled_launches;
  if (reset) op2b::g_tiled_launches = 0;
  return n;
}
