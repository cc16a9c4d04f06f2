// group.cu -- many airfoil solves on one GPU (op2b_group.h): the batched and
// served forms of the airfoil iteration.
//
// Each solve keeps its own datasets, maps and contribution lists in HBM (one
// stream-ordered allocation per solve).  One outer iteration of every active
// solve is four launches, the plain path's fused chains with the iteration
// rotated so that save_soln + adt_calc ride on the last update:
//   k_grp_flux          res_calc flux + bres_calc values  (edge tiles)
//   k_grp_fold<0>       fold + update + adt_calc          (cell tiles)
//   k_grp_flux
//   k_grp_fold<2>       fold + update + rms, then the next iteration's
//                       save_soln + adt_calc              (cell tiles)
// A solve's first save_soln + adt_calc (k_grp_save_adt) is a launch of its
// own before its first iteration.  With the "group_rotate" knob at 0 the
// iteration is k_grp_save_adt, flux, fold<0>, flux, fold<1> (no save).
// A tile is a run of one solve's elements; a launch's grid is its tile table,
// so one launch covers many solves, whatever their sizes: a block of solves
// whose intermediate flux values fit L2 together (Group::rebuild).  The device
// functions are the plain path's (airfoil_math.cuh) and the contribution
// lists have the plain path's order, so q is bit-identical to the plain
// solve.  The first update's rms is not computed: the reference app zeroes it
// before the second update (airfoil/airfoil_op.cpp:283-290).
//
// The second update's rms: every cell tile of a solve writes one partial
// (its threads' sums, folded in a fixed tree); the last CTA of the solve to
// finish (a per-solve ticket) folds the solve's partials in tile order,
// stores sqrt(sum / ncell) in the solve's history, advances its iteration
// count and applies the stopping test.  Tiles are fixed by the solve's own
// cell count (kCellTile), so the rms does not depend on the other solves.
// A stopped solve's CTAs return at once; the host drops it from the tile
// tables at the next op2b_group_run after a poll.

#include <math.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "airfoil_math.cuh"
#include "internal.h"
#include "launch.cuh"
#include "op2b_group.h"
#include "reduce.cuh"
#include "tile_chain.cuh"

namespace op2b {
namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 4;
constexpr int kCellTile = kThreads * kCellsPerThread;  // fixes the rms fold order
constexpr int kMaxWidth = 8;                           // longest contribution list

template <class T>
struct SolveDev {  // device view of one solve; written by the host only
  const T *x;
  T *q, *qold, *adt, *vals, *partials, *hist;
  const int *pedge, *pecell, *pbedge, *pbecell, *bound, *pcell, *ell;
  int ncell, nedge, nbedge, W, ntiles, pad;
  T qinf[4];
  // the tiled chain: second buffers of q and adt, and the tile lists
  T *q2, *adt2;
  const int *toff, *tflux, *tell;
  int tct, tntile;
};

struct SolveState {  // written by the kernels
  int active, iter, max_iter;
  unsigned ticket;
  double rms1, tol;
};

struct Tile {
  int solve, start, count, local;
};

__device__ __forceinline__ bool solve_active(const SolveState *st, int s) {
  return *reinterpret_cast<const volatile int *>(&st[s].active) != 0;
}

template <class T>
__device__ __forceinline__ AirConsts<T> with_qinf(AirConsts<T> K, const SolveDev<T> *d) {
#pragma unroll
  for (int i = 0; i < 4; i++) K.qinf[i] = d->qinf[i];
  return K;
}

// The end of an iteration's second update: this CTA's rms partial (its
// threads' sums, block tree) into the solve's slot for the tile; the
// solve's last CTA folds the ntiles partials in tile order, records
// rms = sqrt(sum / ncell) (airfoil/airfoil_op.cpp:291) and applies the
// stopping test (iteration cap, or rms below tol x the first iteration's)
template <class T>
__device__ __forceinline__ void end_of_iteration(const SolveDev<T> *d, SolveState *st,
                                                 const Tile &t, T rms, int ntiles) {
  __shared__ T ws[32];
  __shared__ bool last;
  const T b = block_fold(rms, T(0), OpSum(), ws);
  if (threadIdx.x == 0) {  // the writer fences its partial, then takes a ticket
    d->partials[t.local] = b;
    __threadfence();
    last = atomicAdd(&st[t.solve].ticket, 1u) == (unsigned)(ntiles - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  T sum = T(0);
  for (int p = threadIdx.x; p < ntiles; p += blockDim.x) sum += __ldcg(d->partials + p);
  sum = block_fold(sum, T(0), OpSum(), ws);
  if (threadIdx.x == 0) {
    SolveState &s = st[t.solve];
    const T r = sqrt(sum / (T)d->ncell);
    const int it = s.iter;
    d->hist[it] = r;
    const int done = it + 1;
    if (done == 1) s.rms1 = (double)r;
    const bool stop =
        done >= s.max_iter || (done >= 2 && s.tol > 0.0 && (double)r < s.tol * s.rms1);
    s.iter = done;
    if (stop) s.active = 0;
    s.ticket = 0u;
  }
}

// save_soln + adt_calc over one tile of one solve's cells (a thread's cells
// one after another, the next cell's nodes fetched while this one computes)
template <class T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 6 : 4)
    k_grp_save_adt(const Tile *__restrict__ tiles, const SolveDev<T> *__restrict__ sd,
                   const SolveState *st, AirConsts<T> K) {
  const Tile t = tiles[blockIdx.x];
  const SolveDev<T> *d = sd + t.solve;
  const int4 *pcell = reinterpret_cast<const int4 *>(d->pcell);
  int4 nd = make_int4(0, 0, 0, 0);
  if ((int)threadIdx.x < t.count) nd = __ldg(pcell + t.start + threadIdx.x);  // read-only
  pdl_wait();
  pdl_trigger();
  if (!solve_active(st, t.solve)) return;
  const T *x = d->x, *q = d->q;
  T *qold = d->qold, *adt = d->adt;
#pragma unroll 1
  for (int i = threadIdx.x; i < t.count; i += kThreads) {
    const int c = t.start + i;
    T qq[4], a[2], b[2], e[2], f[2];
    ld4(q + 4 * (size_t)c, qq);
    ld2(x + 2 * (size_t)nd.x, a);
    ld2(x + 2 * (size_t)nd.y, b);
    ld2(x + 2 * (size_t)nd.z, e);
    ld2(x + 2 * (size_t)nd.w, f);
    if (i + kThreads < t.count) nd = __ldg(pcell + c + kThreads);
    st4(qold + 4 * (size_t)c, qq);
    adt[c] = adt_calc(a, b, e, f, qq, K);
  }
}

// res_calc's flux per edge and bres_calc's increment per boundary edge, over
// one tile of one solve's values (edges first, then boundary edges)
template <class T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 8 : 4)
    k_grp_flux(const Tile *__restrict__ tiles, const SolveDev<T> *__restrict__ sd,
               const SolveState *st, AirConsts<T> K0) {
  const Tile t = tiles[blockIdx.x];
  const SolveDev<T> *d = sd + t.solve;
  const int ne = d->nedge;
  const int2 *pedge = reinterpret_cast<const int2 *>(d->pedge);
  const int2 *pecell = reinterpret_cast<const int2 *>(d->pecell);
  const int i0 = t.start + threadIdx.x, end = t.start + t.count;
  int2 nn = make_int2(0, 0), cc = make_int2(0, 0);
  if (i0 < end && i0 < ne) {  // map entries: read-only
    nn = __ldg(pedge + i0);
    cc = __ldg(pecell + i0);
  }
  pdl_wait();
  pdl_trigger();
  if (!solve_active(st, t.solve)) return;
  const AirConsts<T> K = with_qinf(K0, d);
  const T *x = d->x, *q = d->q, *adt = d->adt;
  T *v = d->vals;
  for (int i = i0; i < end; i += kThreads) {
    T f[4];
    if (i < ne) {
      if (i != i0) {
        nn = __ldg(pedge + i);
        cc = __ldg(pecell + i);
      }
      T p[2], s[2], q1[4], q2[4];
      ld4(q + 4 * (size_t)cc.x, q1);
      ld4(q + 4 * (size_t)cc.y, q2);
      ld2(x + 2 * (size_t)nn.x, p);
      ld2(x + 2 * (size_t)nn.y, s);
      const T d1 = __ldg(adt + cc.x), d2 = __ldg(adt + cc.y);
      res_flux(p, s, q1, q2, d1, d2, K.gm1, K.eps, f);
    } else {
      const int b = i - ne;
      const int2 bn = __ldg(reinterpret_cast<const int2 *>(d->pbedge) + b);
      const int c = __ldg(d->pbecell + b);
      T p[2], s[2], q1[4];
      ld2(x + 2 * (size_t)bn.x, p);
      ld2(x + 2 * (size_t)bn.y, s);
      ld4(q + 4 * (size_t)c, q1);
      bres_contrib(p, s, q1, __ldg(adt + c), __ldg(d->bound + b), K, f);
    }
    st4(v + 4 * (size_t)i, f);
  }
}

// the cell pass: fold each cell's listed values onto res in list order, then
// update (airfoil/update.h:1-12).  A solve's res is +0.0 on every cell when
// each fold starts (zero at admission, zeroed by every update, written by
// nothing else), so the fold starts its sums from +0.0 in registers and the
// group keeps no res array: the same values as reading it, 32 bytes per cell
// less traffic per update.  MODE 0 (the iteration's first update):
// then adt_calc on the new q, no rms.  MODE 1 (its second): the rms partial,
// and the solve's last CTA ends the iteration.  MODE 2: MODE 1 plus the next
// iteration's save_soln and adt_calc on the new q (qold = q, then adt), so
// that iteration starts at its res_calc; update reads qold at the cell
// before the copy overwrites it, hence the coherent load
template <class T, int MODE>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? (MODE == 1 ? 4 : 3) : 2)
    k_grp_fold(const Tile *__restrict__ tiles, const SolveDev<T> *__restrict__ sd,
               SolveState *st, AirConsts<T> K) {
  constexpr bool FIRST = MODE == 0, ADT = MODE != 1, SAVE = MODE == 2;
  const Tile t = tiles[blockIdx.x];
  const SolveDev<T> *d = sd + t.solve;
  const int W = d->W;
  const int *ell = d->ell;
  const int4 *pcell = reinterpret_cast<const int4 *>(d->pcell);
  // a thread's cells one after another; the next cell's list head and nodes
  // (read-only) are fetched while this cell gathers
  int k[4];
  int4 nd = make_int4(0, 0, 0, 0);
  if ((int)threadIdx.x < t.count) {
    list_head(ell, W, t.start + threadIdx.x, k);
    if (ADT) nd = __ldg(pcell + t.start + threadIdx.x);
  }
  pdl_wait();
  pdl_trigger();
  const bool live = solve_active(st, t.solve);  // the same for the whole CTA
  if (!live) return;
  const T *x = d->x, *qold = d->qold, *vals = d->vals;
  T *q = d->q, *adt = d->adt;
  T rms = T(0);
#pragma unroll 1
  for (int i = threadIdx.x; i < t.count; i += kThreads) {
    const int c = t.start + i;
    T r[4] = {T(0), T(0), T(0), T(0)}, qo[4], f[4][4], xs[4][2];
    if (SAVE) ldw4(qold + 4 * (size_t)c, qo);
    else ld4(qold + 4 * (size_t)c, qo);
    const T ad = adt[c];
#pragma unroll
    for (int m = 0; m < 4; m++)
      if (k[m] >= 0) ld4(vals + 4 * (size_t)(k[m] >> 1), f[m]);
    if (ADT) {
      ld2(x + 2 * (size_t)nd.x, xs[0]);
      ld2(x + 2 * (size_t)nd.y, xs[1]);
      ld2(x + 2 * (size_t)nd.z, xs[2]);
      ld2(x + 2 * (size_t)nd.w, xs[3]);
    }
    int kc[4] = {k[0], k[1], k[2], k[3]};
    if (i + kThreads < t.count) {
      list_head(ell, W, c + kThreads, k);
      if (ADT) nd = __ldg(pcell + c + kThreads);
    }
#pragma unroll
    for (int m = 0; m < 4; m++) add_listed(r, kc[m], f[m]);
    for (int m = 4; m < W; m++) {  // lists longer than 4
      const int kk = __ldg(ell + (size_t)c * W + m);
      T g[4];
      ld4(vals + 4 * (size_t)(kk >> 1), g);
      add_listed(r, kk, g);
    }
    const T adti = rcp(ad);
    T qn[4];
    for (int m = 0; m < 4; m++) {
      const T del = adti * r[m];
      qn[m] = qo[m] - del;
      rms += del * del;
    }
    st4(q + 4 * (size_t)c, qn);
    if (SAVE) st4(d->qold + 4 * (size_t)c, qn);  // airfoil/save_soln.h:1-3
    if (ADT) adt[c] = adt_calc(xs[0], xs[1], xs[2], xs[3], qn, K);
  }
  if (FIRST) return;
  end_of_iteration(d, st, t, rms, d->ntiles);
}

// The tiled chain over one tile of one solve's cells per CTA
// (tile_chain.cuh): res_calc + bres_calc + update [+ adt_calc] [+ save_soln]
// in one launch over all solves, the flux values in shared memory instead of
// a DRAM round trip.  The fluxes read q and adt of cells in other tiles of
// the same solve, so update and adt_calc write to the other buffer: PAR 0
// reads (q, adt) and writes (q2, adt2), PAR 1 the reverse.  An iteration is
// two chains (PAR 0, then PAR 1), so (q, adt) hold the state between
// iterations.  MODE as in k_grp_fold; the rms partials are per tile of this
// tiling (tntile of them), so the rms's summation tree differs from the
// two-launch form's while every field is bit-identical to it.
template <class T, int MODE, int PAR>
__global__ void __launch_bounds__(1024, 1)
    k_grp_chain_tiled(const Tile *__restrict__ tiles, const SolveDev<T> *__restrict__ sd,
                      SolveState *st, AirConsts<T> K0) {
  constexpr bool FIRST = MODE == 0, ADT = MODE != 1, SAVE = MODE == 2;
  extern __shared__ __align__(16) unsigned char grp_tile_smem[];
  T *fv = reinterpret_cast<T *>(grp_tile_smem);
  const Tile t = tiles[blockIdx.x];
  const SolveDev<T> *d = sd + t.solve;
  const int beg = __ldg(d->toff + t.local), cnt = __ldg(d->toff + t.local + 1) - beg;
  tile_stage<T, 1024>(d->tflux, beg, cnt, fv);  // plan data: before the wait
  pdl_wait();
  pdl_trigger();
  if (!solve_active(st, t.solve)) return;  // the same for the whole CTA
  const AirConsts<T> K = with_qinf(K0, d);
  const T *x = d->x;
  const T *qin = PAR ? d->q2 : d->q, *ain = PAR ? d->adt2 : d->adt;
  T *qout = PAR ? d->q : d->q2, *aout = PAR ? d->adt : d->adt2;
  const int2 *pbedge = reinterpret_cast<const int2 *>(d->pbedge);
  auto bres = [&](int b, T (&r)[4]) {
    const int2 bn = __ldg(pbedge + b);
    const int c = __ldg(d->pbecell + b);
    T p[2], sx[2], q1[4];
    ld2(x + 2 * (size_t)bn.x, p);
    ld2(x + 2 * (size_t)bn.y, sx);
    ld4(qin + 4 * (size_t)c, q1);
    bres_contrib(p, sx, q1, __ldg(ain + c), __ldg(d->bound + b), K, r);
  };
  __syncthreads();
  tile_fluxes<T, 1024>(cnt, (unsigned)d->nedge, (unsigned)d->nbedge,
                       reinterpret_cast<const int2 *>(d->pedge),
                       reinterpret_cast<const int2 *>(d->pecell), x, qin, ain, K, fv, bres);
  __syncthreads();
  const T rms = tile_cells<T, ADT, SAVE, 1024>(
      t.start, t.start + t.count, d->tell, d->W, reinterpret_cast<const int4 *>(d->pcell), x,
      d->qold, ain, qout, nullptr, d->qold, aout, nullptr, K, fv);
  if (FIRST) return;
  end_of_iteration(d, st, t, rms, d->tntile);
}

// ------------------------------------------------ contribution lists ------
// The plain path's list order, built per solve: res_calc's (edge << 1 |
// side) ascending, then bres_calc's ((nedge + b) << 1) ascending, padded with
// (nedge + nbedge) << 1 -- one sort of the cell's entries gives exactly this.

__global__ void k_gl_count(int ne, int nb, const int *pecell, const int *pbecell, int *cnt) {
  const int n = 2 * ne + nb;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(cnt + (i < 2 * ne ? pecell[i] : pbecell[i - 2 * ne]), 1);
}

__global__ void k_gl_max(const int *v, int n, int *out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_gl_pad(int ncell, int W, int pad, int *ell) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)ncell * W;
       i += (size_t)gridDim.x * blockDim.x)
    ell[i] = pad;
}

__global__ void k_gl_place(int ne, int nb, const int *pecell, const int *pbecell, int W,
                           int *cursor, int *ell) {
  const int n = 2 * ne + nb;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i < 2 * ne ? pecell[i] : pbecell[i - 2 * ne];
    const int key = i < 2 * ne ? i : (ne + (i - 2 * ne)) << 1;
    const int pos = atomicAdd(cursor + c, 1);
    if (pos < W) ell[(size_t)c * W + pos] = key;
  }
}

__global__ void k_gl_sort(int ncell, int W, int *ell) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    int v[kMaxWidth];
    for (int j = 0; j < W; j++) v[j] = ell[(size_t)c * W + j];
    for (int j = 1; j < W; j++) {  // insertion sort, W <= 8
      const int x = v[j];
      int m = j - 1;
      while (m >= 0 && v[m] > x) {
        v[m + 1] = v[m];
        m--;
      }
      v[m + 1] = x;
    }
    for (int j = 0; j < W; j++) ell[(size_t)c * W + j] = v[j];
  }
}

// q = qinf on every cell; the padding value -0.0
template <class T>
__global__ void k_gl_init(int ncell, T *q, T *vals_pad, T q0, T q1, T q2, T q3) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const T v[4] = {q0, q1, q2, q3};
    st4(q + 4 * (size_t)c, v);
  }
  if (blockIdx.x == 0 && threadIdx.x < 4) vals_pad[threadIdx.x] = T(-0.0);
}

// ---------------------------------------------------------------- host ----

template <class T>
void flow_state(double mach_d, double alpha_deg, T qinf[4], T c[4]);

// airfoil/airfoil.cpp:134-149 in float, alpha added to the velocity
template <>
void flow_state<float>(double mach_d, double alpha_deg, float qinf[4], float c[4]) {
  float gam = 1.4f, gm1 = gam - 1.0f, cfl = 0.9f, eps = 0.05f;
  float mach = (float)mach_d;
  float p = 1.0f, r = 1.0f;
  float u = sqrtf(gam * p / r) * mach;
  float e = p / (r * gm1) + 0.5f * u * u;
  qinf[0] = r;
  qinf[3] = r * e;
  if (alpha_deg == 0.0) {
    qinf[1] = r * u;
    qinf[2] = 0.0f;
  } else {
    float a = (float)alpha_deg * (atanf(1.0f) / 45.0f);
    qinf[1] = r * u * cosf(a);
    qinf[2] = r * u * sinf(a);
  }
  c[0] = gam; c[1] = gm1; c[2] = cfl; c[3] = eps;
}

// the float->double variant of the same lines (float literals kept)
template <>
void flow_state<double>(double mach_d, double alpha_deg, double qinf[4], double c[4]) {
  double gam = 1.4f, gm1 = gam - 1.0f, cfl = 0.9f, eps = 0.05f;
  // the reference's float literals are kept in its FP64 variant (0.4f), so
  // Mach and alpha enter rounded to float
  double mach = (double)(float)mach_d;
  double p = 1.0f, r = 1.0f;
  double u = sqrt(gam * p / r) * mach;
  double e = p / (r * gm1) + 0.5f * u * u;
  qinf[0] = r;
  qinf[3] = r * e;
  if (alpha_deg == 0.0) {
    qinf[1] = r * u;
    qinf[2] = 0.0f;
  } else {
    double a = (double)(float)alpha_deg * (atan(1.0) / 45.0);
    qinf[1] = r * u * cos(a);
    qinf[2] = r * u * sin(a);
  }
  c[0] = gam; c[1] = gm1; c[2] = cfl; c[3] = eps;
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

struct GroupBase {
  virtual ~GroupBase() {}
  virtual int add(const op2b_mesh *m, double mach, double alpha, int max_iter, double tol) = 0;
  virtual int run(int niter) = 0;
  virtual int poll(int *ids, int max) = 0;
  virtual int sync() = 0;
  virtual int iterations(int id) = 0;
  virtual int history(int id, double *out, int max) = 0;
  virtual int fetch_q(int id, void *q) = 0;
  virtual int fetch_q_async(int id, void *q) = 0;
  virtual int remove(int id) = 0;
  virtual long long solve_bytes(int nn, int nc, int ne, int nb, int max_iter) = 0;
  virtual long long device_bytes() = 0;
  virtual int active() = 0;
  virtual int set_edge_tile(int e) = 0;
  virtual int set_block_bytes(long long bytes) = 0;
  virtual int set_streams(int n) = 0;
  virtual int set_tiled(int on) = 0;
  virtual int tiled_mode() = 0;
  virtual int edge_tile() = 0;
  virtual int autotune(int iters) = 0;
  virtual int autotune_run(int iters) = 0;
};

template <class T>
struct Group : GroupBase {
  struct Solve {
    int nnode = 0, ncell = 0, nedge = 0, nbedge = 0, max_iter = 0;
    double tol = 0;
    void *block = nullptr;
    int *ell = nullptr;
    size_t bytes = 0;
    cudaEvent_t ready = nullptr;
    bool joined = false, removed = false, done = false, reported = false;
    // its qold and adt hold the next iteration's save_soln + adt_calc (done
    // by the previous iteration's last launch, or by the priming launch)
    bool primed = false;
    long long join_epoch = 0;  // the first state mirror that includes this solve
    SolveDev<T> dev;
    cudaEvent_t fetched = nullptr;  // after an asynchronous copy of q out
    cudaStream_t tl_stream = nullptr;  // where the tile lists were queued
    // the tiled chain's second buffers of q and adt, and tile lists
    void *tbuf = nullptr;
    TileLists tl;
    size_t tbytes = 0;
  };

  cudaStream_t cs = nullptr, us = nullptr;  // iterations; admission
  // further streams of the captured iteration: blocks of solves are dealt
  // round-robin to `nstreams` streams (cs first), so independent blocks'
  // passes overlap (one block's latency-bound per-cell pass beside
  // another's flux pass); fork and join are events inside the capture
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;  // [0] fork, [1..] joins
  int nstreams = 1;
  std::vector<Solve> solves;
  SolveDev<T> *d_sd = nullptr;
  SolveState *d_st = nullptr;
  SolveState *h_st = nullptr;  // pinned mirror, filled after each run
  int cap = 0;
  Tile *d_ct = nullptr, *d_et = nullptr, *d_pt = nullptr;
  size_t ct_cap = 0, et_cap = 0, pt_cap = 0;
  int nct = 0, net = 0, npt = 0, nactive = 0;
  // rotated iteration: res_calc ... update, update + the next iteration's
  // save_soln + adt_calc -- four launches; a solve's very first save_soln +
  // adt_calc is a priming launch of its own (pt: the unprimed solves' tiles)
  bool rotate = true;
  // the tiled chain (op2b_group_set_tiled): one launch per update, each CTA
  // one tile of one solve, its flux values in shared memory
  bool tiled = false;
  long long graph_cells = 0, stopped_cells = 0;  // cells in the captured iteration; stopped since
  Tile *d_tt = nullptr;
  size_t tt_cap = 0;
  int ntt = 0;
  size_t tsmem = 0, tsmem_set = 0;
  int etile = 2048;
  bool changed = true;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t mirror_ev = nullptr;
  bool mirror_pending = false;
  long long mirror_epoch = 0;  // state mirrors issued (run) so far
  AirConsts<T> K;
  bool ok = false;

  Group() {
    ensure_cuda();
    if (error_pending()) return;
    OP2B_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    OP2B_CUDA(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking));
    OP2B_CUDA(cudaEventCreateWithFlags(&mirror_ev, cudaEventDisableTiming));
    T q[4], c[4];
    flow_state<T>(0.4, 0.0, q, c);
    memset(&K, 0, sizeof K);
    K.gam = c[0]; K.gm1 = c[1]; K.cfl = c[2]; K.eps = c[3];
    ok = !error_pending();
  }

  ~Group() override {
    if (cs) cudaStreamSynchronize(cs);
    if (us) cudaStreamSynchronize(us);
    for (auto &s : solves) release(s);
    if (exec) cudaGraphExecDestroy(exec);
    cudaFree(d_sd);
    cudaFree(d_st);
    cudaFree(d_ct);
    cudaFree(d_et);
    cudaFree(d_pt);
    cudaFree(d_tt);
    if (h_st) cudaFreeHost(h_st);
    if (mirror_ev) cudaEventDestroy(mirror_ev);
    if (cs) cudaStreamDestroy(cs);
    if (us) cudaStreamDestroy(us);
    for (cudaStream_t x : side) cudaStreamDestroy(x);
    for (cudaEvent_t e : side_ev) cudaEventDestroy(e);
  }

  void release(Solve &s) {
    if (s.removed) return;
    if (s.fetched) {  // an asynchronous copy of q out reads the solve's memory
      OP2B_CUDA(cudaStreamWaitEvent(s.joined ? cs : us, s.fetched, 0));
      cudaEventDestroy(s.fetched);
      s.fetched = nullptr;
    }
    if (s.block) cudaFreeAsync(s.block, s.joined ? cs : us);
    if (s.ell) cudaFreeAsync(s.ell, s.joined ? cs : us);
    if (s.tbuf) cudaFreeAsync(s.tbuf, s.joined ? cs : us);
    free_tile_lists(&s.tl, s.joined ? cs : us);
    s.tbuf = nullptr;
    if (s.ready) cudaEventDestroy(s.ready);
    s.block = nullptr;
    s.ell = nullptr;
    s.ready = nullptr;
    s.removed = true;
  }

  static size_t layout(int nn, int nc, int ne, int nb, int max_iter, size_t off[16]) {
    const int ntiles = (nc + kCellTile - 1) / kCellTile;
    const size_t sz[16] = {sizeof(T) * 2 * (size_t)nn,                 // x
                           sizeof(T) * 4 * (size_t)nc,                 // q
                           sizeof(T) * 4 * (size_t)nc,                 // qold
                           sizeof(T) * (size_t)nc,                     // adt
                           0,                                          // (res: none)
                           sizeof(T) * 4 * ((size_t)ne + nb + 1),      // vals
                           sizeof(T) * (size_t)std::max(ntiles, 1),    // partials
                           sizeof(T) * (size_t)std::max(max_iter, 1),  // hist
                           sizeof(int) * 2 * (size_t)ne,               // pedge
                           sizeof(int) * 2 * (size_t)ne,               // pecell
                           sizeof(int) * 2 * (size_t)std::max(nb, 1),  // pbedge
                           sizeof(int) * (size_t)std::max(nb, 1),      // pbecell
                           sizeof(int) * (size_t)std::max(nb, 1),      // bound
                           sizeof(int) * 4 * (size_t)nc,               // pcell
                           sizeof(int) * ((size_t)nc + 1),             // list counts (build)
                           0};
    size_t tot = 0;
    for (int i = 0; i < 16; i++) {
      off[i] = tot;
      tot += align256(sz[i]);
    }
    return tot;
  }

  // the tiled chain's extra bytes of a solve: q2 and adt2, the rewritten
  // lists (width about 4) and the tiles' flux indices (the edges, a share
  // of them twice, and the boundary edges)
  static size_t tiled_bytes(int nc, int ne, int nb) {
    return align256(sizeof(T) * 5 * (size_t)nc) + align256(sizeof(int) * 4 * (size_t)nc) +
           align256(sizeof(int) * (size_t)((ne + nb) * 5LL / 4 + 1024));
  }

  long long solve_bytes(int nn, int nc, int ne, int nb, int max_iter) override {
    size_t off[16];
    return (long long)(layout(nn, nc, ne, nb, max_iter, off) +
                       align256(sizeof(int) * 4 * (size_t)nc) +
                       (tiled ? tiled_bytes(nc, ne, nb) : 0));
  }

  // The tiled chain's lists of a solve, queued on stream st with no host
  // wait (tiles of 4096 cells in FP32, 2048 in FP64); whether the longest
  // tile's values fit a CTA's shared memory is checked at the next rebuild
  // (fit_tiled), which makes smaller tiles if not.
  bool ensure_tiled(Solve &s, cudaStream_t st) {
    if (s.tbuf) return true;
    void *buf = nullptr;
    if (pool_malloc_async(&buf, sizeof(T) * 5 * (size_t)s.ncell, st) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    TileLists tl;
    const int ct = std::max(kCellTile, sizeof(T) == 4 ? 4096 : 2048);
    if (!build_tile_lists_async(s.ell, s.ncell, s.dev.W, ct, st, &tl)) {
      cudaFreeAsync(buf, st);
      return false;
    }
    s.tbuf = buf;
    s.tl_stream = st;
    set_tiled_view(s, tl);
    s.tbytes = align256(sizeof(T) * 5 * (size_t)s.ncell) +
               align256(sizeof(int) * (size_t)s.dev.W * s.ncell) * 2;
    s.bytes += s.tbytes;
    SolveDev<T> &d = s.dev;
    d.q2 = (T *)buf;
    d.adt2 = (T *)buf + 4 * (size_t)s.ncell;
    return true;
  }

  void set_tiled_view(Solve &s, const TileLists &tl) {
    s.tl = tl;
    s.dev.toff = tl.toff;
    s.dev.tflux = tl.tflux;
    s.dev.tell = tl.tell;
    s.dev.tct = tl.ct;
    s.dev.tntile = tl.ntile;
  }

  // true when the solve's longest tile fits shared memory, after making
  // smaller tiles (at least the rms tile) if it did not; the solve's view
  // on the device is refreshed then
  bool fit_tiled(int id) {
    Solve &s = solves[id];
    const size_t budget = (size_t)rt().smem_optin - 2048;
    if ((size_t)tile_lists_longest(&s.tl, s.tl_stream) * 4 * sizeof(T) <= budget) return true;
    for (int ct = s.tl.ct * 3 / 4; ct >= kCellTile; ct = ct * 3 / 4) {
      TileLists tl;
      if (!build_tile_lists(s.ell, s.ncell, s.dev.W, ct, cs, &tl)) return false;
      if ((size_t)tl.maxcnt * 4 * sizeof(T) <= budget) {
        free_tile_lists(&s.tl, cs);
        set_tiled_view(s, tl);
        OP2B_CUDA(cudaMemcpyAsync(d_sd + id, &s.dev, sizeof(SolveDev<T>), cudaMemcpyHostToDevice,
                                  cs));
        return true;
      }
      free_tile_lists(&tl, cs);
    }
    return false;
  }

  int add(const op2b_mesh *m, double mach, double alpha, int max_iter, double tol) override {
    if (!ok || !m || m->ncell <= 0 || m->nedge <= 0 || m->nnode <= 0 || m->nbedge < 0 ||
        max_iter <= 0) {
      fail(-1, "op2b_group_add error -- bad mesh or max_iter\n");
      return -1;
    }
    if ((long long)m->nedge + m->nbedge + 1 >= (1LL << 30)) {
      fail(-1, "op2b_group_add error -- mesh too large for 32-bit value lists\n");
      return -1;
    }
    Solve s;
    s.nnode = m->nnode; s.ncell = m->ncell; s.nedge = m->nedge; s.nbedge = m->nbedge;
    s.max_iter = max_iter;
    s.tol = tol;
    size_t off[16];
    const size_t tot = layout(s.nnode, s.ncell, s.nedge, s.nbedge, max_iter, off);
    if (pool_malloc_async(&s.block, tot, us) != cudaSuccess) {
      cudaGetLastError();
      fail(-1, "op2b_group_add error -- out of device memory (%zu bytes)\n", tot);
      return -1;
    }
    s.bytes = tot;
    char *b = (char *)s.block;
    SolveDev<T> &d = s.dev;
    memset(&d, 0, sizeof d);
    d.x = (const T *)(b + off[0]);
    d.q = (T *)(b + off[1]); d.qold = (T *)(b + off[2]); d.adt = (T *)(b + off[3]);
    d.vals = (T *)(b + off[5]); d.partials = (T *)(b + off[6]);
    d.hist = (T *)(b + off[7]);
    d.pedge = (const int *)(b + off[8]); d.pecell = (const int *)(b + off[9]);
    d.pbedge = (const int *)(b + off[10]); d.pbecell = (const int *)(b + off[11]);
    d.bound = (const int *)(b + off[12]); d.pcell = (const int *)(b + off[13]);
    int *cnt = (int *)(b + off[14]);
    d.ncell = s.ncell; d.nedge = s.nedge; d.nbedge = s.nbedge;
    d.ntiles = (s.ncell + kCellTile - 1) / kCellTile;
    T c4[4];
    flow_state<T>(mach, alpha, d.qinf, c4);
    const T *xh = (const T *)(sizeof(T) == 8 ? (const void *)m->x64 : (const void *)m->x32);
    auto up = [&](const void *dst, const void *src, size_t n) {
      if (n) OP2B_CUDA(cudaMemcpyAsync((void *)dst, src, n, cudaMemcpyHostToDevice, us));
    };
    up(d.x, xh, sizeof(T) * 2 * (size_t)s.nnode);
    up(d.pedge, m->edge, sizeof(int) * 2 * (size_t)s.nedge);
    up(d.pecell, m->ecell, sizeof(int) * 2 * (size_t)s.nedge);
    up(d.pbedge, m->bedge, sizeof(int) * 2 * (size_t)s.nbedge);
    up(d.pbecell, m->becell, sizeof(int) * (size_t)s.nbedge);
    up(d.bound, m->bound, sizeof(int) * (size_t)s.nbedge);
    up(d.pcell, m->cell, sizeof(int) * 4 * (size_t)s.ncell);
    // contribution lists: count, width, place, sort
    const int grid = rt().num_sms * 4;
    OP2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)s.ncell + 1), us));
    k_gl_count<<<grid, 256, 0, us>>>(s.nedge, s.nbedge, d.pecell, d.pbecell, cnt);
    k_gl_max<<<grid, 256, 0, us>>>(cnt, s.ncell, cnt + s.ncell);
    int W = 0;
    OP2B_CUDA(cudaMemcpyAsync(&W, cnt + s.ncell, sizeof(int), cudaMemcpyDeviceToHost, us));
    OP2B_CUDA(cudaStreamSynchronize(us));
    if (W < 1 || W > kMaxWidth) {
      cudaFreeAsync(s.block, us);
      fail(-1, "op2b_group_add error -- a cell has %d contributions (at most %d)\n", W,
           kMaxWidth);
      return -1;
    }
    d.W = W;
    if (pool_malloc_async((void **)&s.ell, sizeof(int) * W * (size_t)s.ncell, us) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeAsync(s.block, us);
      fail(-1, "op2b_group_add error -- out of device memory\n");
      return -1;
    }
    s.bytes += align256(sizeof(int) * W * (size_t)s.ncell);
    d.ell = s.ell;
    k_gl_pad<<<grid, 256, 0, us>>>(s.ncell, W, (s.nedge + s.nbedge) << 1, s.ell);
    OP2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)s.ncell, us));
    k_gl_place<<<grid, 256, 0, us>>>(s.nedge, s.nbedge, d.pecell, d.pbecell, W, cnt, s.ell);
    k_gl_sort<<<grid, 256, 0, us>>>(s.ncell, W, s.ell);
    OP2B_CUDA(cudaMemsetAsync(d.qold, 0, sizeof(T) * 4 * (size_t)s.ncell, us));
    OP2B_CUDA(cudaMemsetAsync(d.adt, 0, sizeof(T) * (size_t)s.ncell, us));
    k_gl_init<T><<<grid, 256, 0, us>>>(s.ncell, d.q, d.vals + 4 * ((size_t)s.nedge + s.nbedge),
                                       d.qinf[0], d.qinf[1], d.qinf[2], d.qinf[3]);
    if (tiled && !ensure_tiled(s, us)) {
      cudaFreeAsync(s.ell, us);
      cudaFreeAsync(s.block, us);
      fail(-1, "op2b_group_add error -- out of device memory for the tiled chain\n");
      return -1;
    }
    OP2B_CUDA(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
    OP2B_CUDA(cudaEventRecord(s.ready, us));
    if (error_pending()) return -1;
    solves.push_back(s);
    return (int)solves.size() - 1;
  }

  // device arrays of solve views and states, at least n entries
  void reserve(int n) {
    if (n <= cap) return;
    int nc = std::max(64, cap);
    while (nc < n) nc *= 2;
    SolveDev<T> *sd = nullptr;
    SolveState *st = nullptr, *hs = nullptr;
    OP2B_CUDA(pool_malloc_async((void **)&sd, sizeof(SolveDev<T>) * nc, cs));
    OP2B_CUDA(pool_malloc_async((void **)&st, sizeof(SolveState) * nc, cs));
    OP2B_CUDA(cudaMallocHost((void **)&hs, sizeof(SolveState) * nc));
    OP2B_CUDA(cudaMemsetAsync(st, 0, sizeof(SolveState) * nc, cs));
    if (cap) {
      OP2B_CUDA(cudaMemcpyAsync(sd, d_sd, sizeof(SolveDev<T>) * cap, cudaMemcpyDeviceToDevice, cs));
      OP2B_CUDA(cudaMemcpyAsync(st, d_st, sizeof(SolveState) * cap, cudaMemcpyDeviceToDevice, cs));
      OP2B_CUDA(cudaFreeAsync(d_sd, cs));
      OP2B_CUDA(cudaFreeAsync(d_st, cs));
    }
    if (h_st) {
      OP2B_CUDA(cudaStreamSynchronize(cs));  // the mirror may be the target of a copy
      memcpy(hs, h_st, sizeof(SolveState) * cap);
      cudaFreeHost(h_st);
    } else {
      memset(hs, 0, sizeof(SolveState) * nc);
    }
    d_sd = sd;
    d_st = st;
    h_st = hs;
    cap = nc;
    changed = true;
  }

  void upload_tiles(Tile *&dptr, size_t &dcap, const std::vector<Tile> &h) {
    const size_t need = std::max<size_t>(h.size(), 1);
    if (need > dcap) {
      if (dptr) OP2B_CUDA(cudaFreeAsync(dptr, cs));
      OP2B_CUDA(pool_malloc_async((void **)&dptr, sizeof(Tile) * need, cs));
      dcap = need;
    }
    if (!h.empty())
      OP2B_CUDA(cudaMemcpyAsync(dptr, h.data(), sizeof(Tile) * h.size(), cudaMemcpyHostToDevice, cs));
  }

  // Solves are independent, so an iteration may run block by block: each
  // block of solves takes its five launches while its flux values (16 B per
  // edge in FP32) are still in L2, instead of five launches over all solves
  // whose values go out to DRAM and back.  A block holds solves in id order
  // up to block_bytes of values (a larger solve makes a block of its own).
  struct Block {
    int ct0, nct, et0, net, tt0, ntt;
  };
  std::vector<Block> blocks;
  // default one block: measured on 64 solves (12M cells), blocks of 24, 48
  // and 96 MiB of values took 1.42, 1.27 and 1.15 ms per iteration against
  // 1.01 ms for one block (the launches' ramps and tails cost more than the
  // DRAM round trip of the values); the autotuner tries them all
  size_t block_bytes = ~(size_t)0;

  void rebuild() {
    std::vector<Tile> ct, et, pt, tt;
    blocks.clear();
    nactive = 0;
    graph_cells = stopped_cells = 0;
    rotate = tuning("group_rotate", 1) != 0;
    size_t in_block = 0;
    tsmem = 0;
    if (tiled)  // tile lists of solves that joined before the tiled chain was chosen
      for (int id = 0; id < (int)solves.size(); id++) {
        Solve &s = solves[id];
        if (!s.joined || s.removed || s.done || s.tbuf) continue;
        if (!ensure_tiled(s, cs)) {
          tiled = false;  // this solve cannot: the whole group takes the two launches
          break;
        }
        OP2B_CUDA(cudaMemcpyAsync(d_sd + id, &s.dev, sizeof(SolveDev<T>), cudaMemcpyHostToDevice,
                                  cs));
      }
    if (tiled)
      for (int id = 0; id < (int)solves.size() && tiled; id++) {
        const Solve &s = solves[id];
        if (s.joined && !s.removed && !s.done && !fit_tiled(id)) tiled = false;
      }
    for (int id = 0; id < (int)solves.size(); id++) {
      const Solve &s = solves[id];
      if (!s.joined || s.removed || s.done) continue;
      nactive++;
      graph_cells += s.ncell;
      if (rotate && !s.primed)
        for (int a = 0, l = 0; a < s.ncell; a += kCellTile, l++)
          pt.push_back(Tile{id, a, std::min(kCellTile, s.ncell - a), l});
      const int nv = s.nedge + s.nbedge;
      const size_t vbytes = sizeof(T) * 4 * (size_t)nv;
      if (blocks.empty() || (in_block > 0 && in_block + vbytes > block_bytes)) {
        blocks.push_back(Block{(int)ct.size(), 0, (int)et.size(), 0, (int)tt.size(), 0});
        in_block = 0;
      }
      in_block += vbytes;
      for (int a = 0, l = 0; a < s.ncell; a += kCellTile, l++)
        ct.push_back(Tile{id, a, std::min(kCellTile, s.ncell - a), l});
      for (int a = 0, l = 0; a < nv; a += etile, l++)
        et.push_back(Tile{id, a, std::min(etile, nv - a), l});
      if (tiled) {
        for (int a = 0, l = 0; a < s.ncell; a += s.tl.ct, l++)
          tt.push_back(Tile{id, a, std::min(s.tl.ct, s.ncell - a), l});
        tsmem = std::max(tsmem, (size_t)s.tl.maxcnt * 4 * sizeof(T));
      }
      blocks.back().nct = (int)ct.size() - blocks.back().ct0;
      blocks.back().net = (int)et.size() - blocks.back().et0;
      blocks.back().ntt = (int)tt.size() - blocks.back().tt0;
    }
    upload_tiles(d_ct, ct_cap, ct);
    upload_tiles(d_et, et_cap, et);
    upload_tiles(d_pt, pt_cap, pt);
    upload_tiles(d_tt, tt_cap, tt);
    nct = (int)ct.size();
    net = (int)et.size();
    npt = (int)pt.size();
    ntt = (int)tt.size();
    if (tiled && tsmem > tsmem_set) {
      for (const void *k : {(const void *)k_grp_chain_tiled<T, 0, 0>,
                            (const void *)k_grp_chain_tiled<T, 1, 1>,
                            (const void *)k_grp_chain_tiled<T, 2, 1>})
        OP2B_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem));
      tsmem_set = tsmem;
    }
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    if (nactive == 0) return;
    cudaGraph_t graph = nullptr;
    const int K = std::max(1, std::min(nstreams, (int)blocks.size()));
    while ((int)side.size() < K - 1) {  // created outside the capture
      cudaStream_t x;
      OP2B_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
      side.push_back(x);
    }
    while ((int)side_ev.size() < K) {
      cudaEvent_t e;
      OP2B_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      side_ev.push_back(e);
    }
    OP2B_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    if (K > 1) {
      OP2B_CUDA(cudaEventRecord(side_ev[0], cs));
      for (int k = 1; k < K; k++) OP2B_CUDA(cudaStreamWaitEvent(side[k - 1], side_ev[0], 0));
    }
    for (size_t i = 0; i < blocks.size(); i++)
      iteration(blocks[i], i % K == 0 ? cs : side[i % K - 1]);
    if (K > 1)
      for (int k = 1; k < K; k++) {
        OP2B_CUDA(cudaEventRecord(side_ev[k], side[k - 1]));
        OP2B_CUDA(cudaStreamWaitEvent(cs, side_ev[k], 0));
      }
    OP2B_CUDA(cudaStreamEndCapture(cs, &graph));
    if (graph) {
      OP2B_CUDA(cudaGraphInstantiate(&exec, graph, 0));
      cudaGraphDestroy(graph);
    }
    changed = false;
  }

  void iteration(const Block &b, cudaStream_t cs) {
    const Tile *ct = d_ct + b.ct0, *et = d_et + b.et0;
    if (!rotate)
      launch_pdl(k_grp_save_adt<T>, b.nct, kThreads, 0, cs, ct, (const SolveDev<T> *)d_sd,
                 (const SolveState *)d_st, K);
    if (tiled) {  // (q, adt) -> (q2, adt2) -> (q, adt)
      const Tile *tt = d_tt + b.tt0;
      launch_pdl(k_grp_chain_tiled<T, 0, 0>, b.ntt, 1024, tsmem, cs, tt,
                 (const SolveDev<T> *)d_sd, d_st, K);
      if (rotate)
        launch_pdl(k_grp_chain_tiled<T, 2, 1>, b.ntt, 1024, tsmem, cs, tt,
                   (const SolveDev<T> *)d_sd, d_st, K);
      else
        launch_pdl(k_grp_chain_tiled<T, 1, 1>, b.ntt, 1024, tsmem, cs, tt,
                   (const SolveDev<T> *)d_sd, d_st, K);
      return;
    }
    launch_pdl(k_grp_flux<T>, b.net, kThreads, 0, cs, et, (const SolveDev<T> *)d_sd,
               (const SolveState *)d_st, K);
    launch_pdl(k_grp_fold<T, 0>, b.nct, kThreads, 0, cs, ct, (const SolveDev<T> *)d_sd, d_st, K);
    launch_pdl(k_grp_flux<T>, b.net, kThreads, 0, cs, et, (const SolveDev<T> *)d_sd,
               (const SolveState *)d_st, K);
    if (rotate)
      launch_pdl(k_grp_fold<T, 2>, b.nct, kThreads, 0, cs, ct, (const SolveDev<T> *)d_sd, d_st,
                 K);
    else
      launch_pdl(k_grp_fold<T, 1>, b.nct, kThreads, 0, cs, ct, (const SolveDev<T> *)d_sd, d_st,
                 K);
  }

  // save_soln + adt_calc of the solves that have not had them yet (rotated
  // iteration only), before their first iteration
  void prime() {
    if (!rotate || npt == 0) return;
    launch_pdl(k_grp_save_adt<T>, npt, kThreads, 0, cs, (const Tile *)d_pt,
               (const SolveDev<T> *)d_sd, (const SolveState *)d_st, K);
    for (auto &s : solves)
      if (s.joined && !s.removed && !s.done) s.primed = true;
    npt = 0;
  }

  int join_pending() {
    int joined = 0;
    for (int id = 0; id < (int)solves.size(); id++) {
      Solve &s = solves[id];
      if (s.joined || s.removed) continue;
      reserve(id + 1);
      OP2B_CUDA(cudaStreamWaitEvent(cs, s.ready, 0));
      SolveState st0;
      memset(&st0, 0, sizeof st0);
      st0.active = 1;
      st0.max_iter = s.max_iter;
      st0.tol = s.tol;
      OP2B_CUDA(cudaMemcpyAsync(d_sd + id, &s.dev, sizeof(SolveDev<T>), cudaMemcpyHostToDevice, cs));
      OP2B_CUDA(cudaMemcpyAsync(d_st + id, &st0, sizeof(SolveState), cudaMemcpyHostToDevice, cs));
      s.join_epoch = mirror_epoch + 1;
      s.joined = true;
      joined++;
    }
    if (joined) changed = true;
    return joined;
  }

  int run(int niter) override {
    if (!ok || niter < 0) return -1;
    if (!solves.empty()) reserve((int)solves.size());  // the state mirror covers every id
    join_pending();
    if (error_pending()) return -1;
    if (changed) rebuild();
    if (error_pending()) return -1;
    if (exec && niter > 0) prime();
    if (exec)
      for (int i = 0; i < niter; i++) OP2B_CUDA(cudaGraphLaunch(exec, cs));
    if ((int)solves.size() > 0 && cap > 0) {
      OP2B_CUDA(cudaMemcpyAsync(h_st, d_st, sizeof(SolveState) * solves.size(),
                                cudaMemcpyDeviceToHost, cs));
      OP2B_CUDA(cudaEventRecord(mirror_ev, cs));
      mirror_pending = true;
      mirror_epoch++;
    }
    return error_pending() ? -1 : nactive;
  }

  int sync() override {
    if (!ok) return -1;
    OP2B_CUDA(cudaStreamSynchronize(cs));
    OP2B_CUDA(cudaStreamSynchronize(us));
    mirror_pending = false;
    return error_pending() ? -1 : 0;
  }

  int poll(int *ids, int max) override {
    if (!ok) return -1;
    if (mirror_pending) {
      OP2B_CUDA(cudaEventSynchronize(mirror_ev));
      mirror_pending = false;
    }
    int n = 0;
    for (int id = 0; id < (int)solves.size(); id++) {
      Solve &s = solves[id];
      if (!s.joined || s.removed || s.reported || s.join_epoch > mirror_epoch || h_st[id].active)
        continue;
      if (!s.done) {
        s.done = true;
        // a stopped solve's CTAs return at once, so the captured iteration is
        // rebuilt without it only when the stopped cells are a quarter of
        // those it holds (knob group_lazy_retire 0: at every stop)
        stopped_cells += s.ncell;
        if (!tuning("group_lazy_retire", 1) || 4 * stopped_cells > graph_cells) changed = true;
      }
      if (n < max && ids) {
        ids[n++] = id;
        s.reported = true;
      }
    }
    return error_pending() ? -1 : n;
  }

  Solve *get(int id) {
    if (id < 0 || id >= (int)solves.size() || solves[id].removed) {
      fail(-1, "op2b_group error -- no solve %d\n", id);
      return nullptr;
    }
    return &solves[id];
  }

  int iterations(int id) override {
    Solve *s = get(id);
    if (!s) return -1;
    if (!s->joined) return 0;
    sync();
    SolveState st;
    OP2B_CUDA(cudaMemcpy(&st, d_st + id, sizeof st, cudaMemcpyDeviceToHost));
    return st.iter;
  }

  int history(int id, double *out, int max) override {
    Solve *s = get(id);
    if (!s) return -1;
    int n = iterations(id);
    if (n <= 0) return n;
    n = std::min(n, max);
    std::vector<T> h(n);
    OP2B_CUDA(cudaMemcpy(h.data(), s->dev.hist, sizeof(T) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) out[i] = (double)h[i];
    return error_pending() ? -1 : n;
  }

  int fetch_q(int id, void *q) override {
    Solve *s = get(id);
    if (!s) return -1;
    sync();
    OP2B_CUDA(cudaMemcpy(q, s->dev.q, sizeof(T) * 4 * (size_t)s->ncell, cudaMemcpyDeviceToHost));
    return error_pending() ? -1 : 0;
  }

  // q of a solve that poll has reported stopped: its device q is final (the
  // launches after its stop return before writing it), so the copy is
  // queued on the admission stream while the other solves iterate; q is
  // valid after op2b_group_sync.  Other solves: the synchronous fetch_q.
  int fetch_q_async(int id, void *q) override {
    Solve *s = get(id);
    if (!s) return -1;
    if (!s->done || !s->reported) return fetch_q(id, q);
    OP2B_CUDA(cudaMemcpyAsync(q, s->dev.q, sizeof(T) * 4 * (size_t)s->ncell,
                              cudaMemcpyDeviceToHost, us));
    if (!s->fetched) OP2B_CUDA(cudaEventCreateWithFlags(&s->fetched, cudaEventDisableTiming));
    OP2B_CUDA(cudaEventRecord(s->fetched, us));
    return error_pending() ? -1 : 0;
  }

  int remove(int id) override {
    Solve *s = get(id);
    if (!s) return -1;
    release(*s);
    changed = true;
    return error_pending() ? -1 : 0;
  }

  long long device_bytes() override {
    long long b = 0;
    for (auto &s : solves)
      if (!s.removed) b += (long long)s.bytes;
    return b + (long long)cap * (sizeof(SolveDev<T>) + sizeof(SolveState)) +
           (long long)(ct_cap + et_cap + tt_cap) * sizeof(Tile);
  }

  int active() override {  // joined and not stopped (stopped ones may still be in the graph)
    int n = 0;
    for (const auto &s : solves) n += s.joined && !s.removed && !s.done;
    return n;
  }

  int set_block_bytes(long long bytes) override {
    const size_t b = bytes <= 0 ? ~(size_t)0 : (size_t)bytes;  // <= 0: one block
    if (b != block_bytes) changed = true;
    block_bytes = b;
    return 0;
  }

  int set_tiled(int on) override {
    if ((on != 0) != tiled) changed = true;
    tiled = on != 0;
    return 0;
  }
  int tiled_mode() override { return tiled ? 1 : 0; }

  int set_streams(int n) override {
    if (n < 1 || n > 8) {
      fail(-1, "op2b_group error -- %d streams: 1 to 8\n", n);
      return -1;
    }
    if (n != nstreams) changed = true;
    nstreams = n;
    return 0;
  }

  int set_edge_tile(int e) override {
    if (e < kThreads || e > 8192 || e % kThreads) {
      fail(-1, "op2b_group error -- edge tile %d: a multiple of %d in [%d, 8192]\n", e, kThreads,
           kThreads);
      return -1;
    }
    if (e != etile) changed = true;
    etile = e;
    return 0;
  }
  int edge_tile() override { return etile; }

  // time each candidate edge tile on the active solves, restoring their
  // state after each trial (the tile does not change results)
  int autotune(int iters) override {
    if (!ok) return -1;
    join_pending();
    if (changed) rebuild();
    if (nactive == 0 || iters <= 0) return etile;
    prime();  // before the snapshot: trials start from primed solves
    // snapshot of everything an iteration writes
    std::vector<std::pair<void *, size_t>> regions;
    for (auto &s : solves) {
      if (!s.joined || s.removed || s.done) continue;
      regions.push_back({s.dev.q, sizeof(T) * 4 * (size_t)s.ncell});
      regions.push_back({s.dev.qold, sizeof(T) * 4 * (size_t)s.ncell});
      regions.push_back({s.dev.adt, sizeof(T) * (size_t)s.ncell});
    }
    regions.push_back({d_st, sizeof(SolveState) * (size_t)solves.size()});
    size_t tot = 0;
    for (auto &r : regions) tot += align256(r.second);
    void *snap = nullptr;
    if (pool_malloc_async(&snap, tot, cs) != cudaSuccess) {
      cudaGetLastError();
      return etile;  // no room to snapshot: keep the current tile
    }
    auto copy = [&](bool save) {
      size_t o = 0;
      for (auto &r : regions) {
        char *sp = (char *)snap + o;
        OP2B_CUDA(cudaMemcpyAsync(save ? sp : r.first, save ? r.first : sp, r.second,
                                  cudaMemcpyDeviceToDevice, cs));
        o += align256(r.second);
      }
    };
    copy(true);
    cudaEvent_t e0, e1;
    OP2B_CUDA(cudaEventCreate(&e0));
    OP2B_CUDA(cudaEventCreate(&e1));
    auto trial = [&]() {
      rebuild();
      OP2B_CUDA(cudaGraphLaunch(exec, cs));  // warm
      OP2B_CUDA(cudaEventRecord(e0, cs));
      for (int i = 0; i < iters; i++) OP2B_CUDA(cudaGraphLaunch(exec, cs));
      OP2B_CUDA(cudaEventRecord(e1, cs));
      OP2B_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      OP2B_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      copy(false);
      return ms;
    };
    const int cands[] = {512, 1024, 2048, 4096, 8192};
    int best = etile;
    float best_ms = 1e30f;
    for (int c : cands) {
      etile = c;
      const float ms = trial();
      if (ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    etile = best;
    // blocks of solves (bytes of flux values per block) x streams they are
    // dealt to; one block on one stream is the plain form
    const std::pair<size_t, int> blk[] = {{~(size_t)0, 1}, {96u << 20, 1}, {48u << 20, 1},
                                          {48u << 20, 2}, {24u << 20, 2}, {24u << 20, 3},
                                          {12u << 20, 4}};
    std::pair<size_t, int> best_blk{block_bytes, nstreams};
    best_ms = 1e30f;
    for (const auto &bb : blk) {
      block_bytes = bb.first;
      nstreams = bb.second;
      const float ms = trial();
      if (ms < best_ms) {
        best_ms = ms;
        best_blk = bb;
      }
    }
    block_bytes = best_blk.first;
    nstreams = best_blk.second;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    OP2B_CUDA(cudaFreeAsync(snap, cs));
    rebuild();
    OP2B_CUDA(cudaStreamSynchronize(cs));
    return error_pending() ? -1 : best;
  }

  // The same candidates timed on real iterations: each candidate runs
  // `iters` iterations of the active solves, which count (nothing is put
  // back).  The candidates' graphs are built while the previous candidates'
  // iterations run (one synchronisation at the end; a graph is destroyed
  // only then), so tuning costs little beyond the iterations themselves.
  // Launch shapes do not change results, so a solve ends bit-identical to
  // an untuned run of the same length.  Returns the iterations run (every
  // active solve advanced by that many, or stopped).
  int autotune_run(int iters) override {
    if (!ok || iters < 1) return -1;
    join_pending();
    if (changed) rebuild();
    if (nactive == 0) return 0;
    prime();
    struct Trial {
      int etile;
      size_t block_bytes;
      int nstreams;
      cudaEvent_t e0 = nullptr, e1 = nullptr;
    };
    std::vector<Trial> trials;
    for (int c : {512, 1024, 2048, 4096, 8192}) trials.push_back(Trial{c, ~(size_t)0, 1});
    const std::pair<size_t, int> blk[] = {{96u << 20, 1}, {48u << 20, 1}, {48u << 20, 2},
                                          {24u << 20, 2}, {24u << 20, 3}, {12u << 20, 4}};
    for (const auto &bb : blk) trials.push_back(Trial{-1, bb.first, bb.second});
    std::vector<cudaGraphExec_t> retired;  // destroyed after the final synchronisation
    int ran = 0;
    auto enqueue = [&](Trial &t) {
      if (exec) {
        retired.push_back(exec);
        exec = nullptr;
      }
      rebuild();
      OP2B_CUDA(cudaEventCreate(&t.e0));
      OP2B_CUDA(cudaEventCreate(&t.e1));
      OP2B_CUDA(cudaEventRecord(t.e0, cs));
      if (exec)
        for (int i = 0; i < iters; i++) OP2B_CUDA(cudaGraphLaunch(exec, cs));
      OP2B_CUDA(cudaEventRecord(t.e1, cs));
      ran += iters;
    };
    auto elapsed = [&](Trial &t) {
      float ms = 1e30f;
      OP2B_CUDA(cudaEventSynchronize(t.e1));
      if (cudaEventElapsedTime(&ms, t.e0, t.e1) != cudaSuccess) ms = 1e30f;
      cudaEventDestroy(t.e0);
      cudaEventDestroy(t.e1);
      return ms;
    };
    // edge tiles (one block, one stream), then blocks x streams at the best tile
    for (int k = 0; k < 5; k++) {
      etile = trials[k].etile;
      block_bytes = ~(size_t)0;
      nstreams = 1;
      enqueue(trials[k]);
    }
    int best = 0;
    float best_ms = 1e30f;
    for (int k = 0; k < 5; k++) {
      const float ms = elapsed(trials[k]);
      if (ms < best_ms) {
        best_ms = ms;
        best = k;
      }
    }
    etile = trials[best].etile;
    std::pair<size_t, int> best_blk{~(size_t)0, 1};
    for (size_t k = 5; k < trials.size(); k++) {
      block_bytes = trials[k].block_bytes;
      nstreams = trials[k].nstreams;
      enqueue(trials[k]);
    }
    for (size_t k = 5; k < trials.size(); k++) {
      const float ms = elapsed(trials[k]);
      if (ms < best_ms) {
        best_ms = ms;
        best_blk = {trials[k].block_bytes, trials[k].nstreams};
      }
    }
    block_bytes = best_blk.first;
    nstreams = best_blk.second;
    if (exec) {
      retired.push_back(exec);
      exec = nullptr;
    }
    rebuild();
    OP2B_CUDA(cudaStreamSynchronize(cs));
    for (cudaGraphExec_t e : retired) cudaGraphExecDestroy(e);
    return error_pending() ? -1 : ran;
  }
};

}  // namespace
}  // namespace op2b

using namespace op2b;

struct op2b_group_s {
  std::unique_ptr<GroupBase> impl;
};

extern "C" {

int op2b_flow_qinf(double mach, double alpha_deg, int fp64, void *qinf4, void *consts4) {
  if (!qinf4) return -1;
  if (fp64) {
    double q[4], c[4];
    flow_state<double>(mach, alpha_deg, q, c);
    memcpy(qinf4, q, sizeof q);
    if (consts4) memcpy(consts4, c, sizeof c);
  } else {
    float q[4], c[4];
    flow_state<float>(mach, alpha_deg, q, c);
    memcpy(qinf4, q, sizeof q);
    if (consts4) memcpy(consts4, c, sizeof c);
  }
  return 0;
}

op2b_group op2b_group_create(int fp64) {
  op2b_group g = new op2b_group_s;
  if (fp64) g->impl.reset(new Group<double>());
  else g->impl.reset(new Group<float>());
  if (error_pending()) {
    delete g;
    return nullptr;
  }
  return g;
}

void op2b_group_destroy(op2b_group g) { delete g; }

#define GROUP_CALL(expr) \
  do {                   \
    if (!g) return -1;   \
    return g->impl->expr; \
  } while (0)

int op2b_group_add(op2b_group g, const op2b_mesh *m, double mach, double alpha_deg, int max_iter,
                   double rel_tol) {
  GROUP_CALL(add(m, mach, alpha_deg, max_iter, rel_tol));
}
int op2b_group_run(op2b_group g, int niter) { GROUP_CALL(run(niter)); }
int op2b_group_poll(op2b_group g, int *ids, int max) { GROUP_CALL(poll(ids, max)); }
int op2b_group_sync(op2b_group g) { GROUP_CALL(sync()); }
int op2b_group_iterations(op2b_group g, int id) { GROUP_CALL(iterations(id)); }
int op2b_group_history(op2b_group g, int id, double *rms, int max) {
  GROUP_CALL(history(id, rms, max));
}
int op2b_group_fetch_q(op2b_group g, int id, void *q) { GROUP_CALL(fetch_q(id, q)); }
int op2b_group_fetch_q_async(op2b_group g, int id, void *q) { GROUP_CALL(fetch_q_async(id, q)); }
int op2b_group_remove(op2b_group g, int id) { GROUP_CALL(remove(id)); }
long long op2b_group_solve_bytes(op2b_group g, int nnode, int ncell, int nedge, int nbedge,
                                 int max_iter) {
  GROUP_CALL(solve_bytes(nnode, ncell, nedge, nbedge, max_iter));
}
long long op2b_group_device_bytes(op2b_group g) { GROUP_CALL(device_bytes()); }
int op2b_group_active(op2b_group g) { GROUP_CALL(active()); }
int op2b_group_set_edge_tile(op2b_group g, int e) { GROUP_CALL(set_edge_tile(e)); }
int op2b_group_set_block_bytes(op2b_group g, long long bytes) {
  GROUP_CALL(set_block_bytes(bytes));
}
int op2b_group_edge_tile(op2b_group g) { GROUP_CALL(edge_tile()); }
int op2b_group_set_streams(op2b_group g, int n) { GROUP_CALL(set_streams(n)); }
int op2b_group_set_tiled(op2b_group g, int on) { GROUP_CALL(set_tiled(on)); }
int op2b_group_tiled(op2b_group g) { GROUP_CALL(tiled_mode()); }
int op2b_group_autotune(op2b_group g, int iters) { GROUP_CALL(autotune(iters)); }
int op2b_group_autotune_run(op2b_group g, int iters) { GROUP_CALL(autotune_run(iters)); }

}  // extern "C"
