// jac.cu -- the two loops of the jac1 / jac2 Jacobi apps as sm_100a kernels,
// replacing the generated jac*/res_kernel.cu and jac*/update_kernel.cu.
//
//   res    (jac1/res.h:1-3)    du[p0] += beta * A * u[p1], p = edge->node map
//   update (jac1/update.h:1-6) u += du + alpha*r; du = 0;
//                              u_sum += u*u; u_max = MAX(u_max, u)
// jac2 stores A as double[3], u as float[2], du as float[3], r as float[2]
// and uses component 0 only (jac2/res.h, jac2/update.h); beta * A * u is
// evaluated in double there, and so it is here.

#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "launch.cuh"
#include "loops.h"
#include "reduce.cuh"

namespace op2b {

__device__ __forceinline__ int jat(const IdxMap &m, int e) {
  return m.map ? __ldg(m.map + m.idx + (size_t)e * m.dim) : e;
}

// V = 1: A float[1], u float[1], du float[1];  V = 2: A double[3], u float[2], du float[3]
template <int V>
struct JacLayout;
template <>
struct JacLayout<1> {
  typedef float AT;
  static constexpr int A = 1, U = 1, DU = 1, R = 1;
};
template <>
struct JacLayout<2> {
  typedef double AT;
  static constexpr int A = 3, U = 2, DU = 3, R = 2;
};

// du += beta * A * u, with jac2's double product
template <int V>
__device__ __forceinline__ float jac_inc(float du, float beta, typename JacLayout<V>::AT a, float u) {
  if (V == 1) return du + beta * (float)a * u;
  return (float)((double)du + (double)beta * (double)a * (double)u);
}

// res, GATHER: one thread per node with incoming contributions; du_out is du
// itself, or a spare buffer when the loop runs ahead of its call
template <int V>
__global__ void k_jac_res_gather(int nrows, const int *__restrict__ active,
                                 const int *__restrict__ row, const int *__restrict__ keys,
                                 IdxMap mA, IdxMap mu,
                                 const typename JacLayout<V>::AT *__restrict__ A,
                                 const float *__restrict__ u, const float *du, float beta,
                                 float *du_out) {
  typedef JacLayout<V> L;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n = 0, k0 = 0, k1 = 0;
  if (t < nrows) {  // plan arrays: read-only, fetched before the wait
    n = active ? active[t] : t;
    k0 = row[t];
    k1 = row[t + 1];
  }
  pdl_wait();
  pdl_trigger();
  if (t >= nrows) return;
  float d = du[(size_t)n * L::DU];
  for (int k = k0; k < k1; k++) {
    int e = __ldg(keys + k);
    typename L::AT a = __ldg(A + (size_t)jat(mA, e) * L::A);
    float uu = __ldg(u + (size_t)jat(mu, e) * L::U);
    d = jac_inc<V>(d, beta, a, uu);
  }
  du_out[(size_t)n * L::DU] = d;
}

// res, GATHER over precomputed (edge, u element) pairs per contribution:
// row -> pair -> (A, u) instead of row -> key -> map entry -> u
template <int V>
__global__ void k_jac_res_pairs(int nrows, const int *__restrict__ active,
                                const int *__restrict__ row, const int2 *__restrict__ pairs,
                                const typename JacLayout<V>::AT *__restrict__ A,
                                const float *__restrict__ u, const float *du, float beta,
                                float *du_out) {
  typedef JacLayout<V> L;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n = 0, k0 = 0, k1 = 0;
  if (t < nrows) {  // plan arrays: read-only, fetched before the wait
    n = active ? active[t] : t;
    k0 = row[t];
    k1 = row[t + 1];
  }
  pdl_wait();
  pdl_trigger();
  if (t >= nrows) return;
  float d = du[(size_t)n * L::DU];
  for (int k = k0; k < k1; k++) {
    const int2 p = __ldg(pairs + k);
    typename L::AT a = __ldg(A + (size_t)p.x * L::A);
    float uu = __ldg(u + (size_t)p.y * L::U);
    d = jac_inc<V>(d, beta, a, uu);
  }
  du_out[(size_t)n * L::DU] = d;
}

// pairs[k] = (A element, u element) of gather key k (slot 0 of the group)
__global__ void k_jac_pairs(long long nkeys, const int *__restrict__ keys, IdxMap mA, IdxMap mu,
                            int2 *pairs) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nkeys;
       k += (long long)gridDim.x * blockDim.x) {
    const int e = keys[k];
    pairs[k] = make_int2(jat(mA, e), jat(mu, e));
  }
}

struct JacPlanView {
  const int *blkmap, *offset, *nelems, *nthrcol, *thrcol, *ind_offs, *ind_sizes;
  const int *ind_u, *ind_du;
  const short *loc_u, *loc_du;
};

// res, COLOURED (inds {-1, 0, 1, -1}: u read, du incremented)
template <int V>
__global__ void k_jac_res_coloured(JacPlanView P, int block_offset, IdxMap mA,
                                   const typename JacLayout<V>::AT *__restrict__ A,
                                   const float *__restrict__ u, float *__restrict__ du,
                                   float beta) {
  typedef JacLayout<V> L;
  extern __shared__ __align__(16) char smem[];
  const int b = P.blkmap[blockIdx.x + block_offset];
  const int nelem = P.nelems[b], off = P.offset[b], ncol = P.nthrcol[b];
  const int su = P.ind_sizes[0 + b * 2], sd = P.ind_sizes[1 + b * 2];
  const int ou = P.ind_offs[0 + b * 2], od = P.ind_offs[1 + b * 2];
  float *us = (float *)smem;
  float *ds = (float *)(smem + ROUND_UP(su * L::U * (int)sizeof(float)));
  for (int i = threadIdx.x; i < su * L::U; i += blockDim.x)
    us[i] = u[(size_t)P.ind_u[ou + i / L::U] * L::U + i % L::U];
  for (int i = threadIdx.x; i < sd * L::DU; i += blockDim.x) ds[i] = 0.0f;
  __syncthreads();
  const int nelems2 = blockDim.x * (1 + (nelem - 1) / blockDim.x);
  for (int n = threadIdx.x; n < nelems2; n += blockDim.x) {
    int col2 = -1, md = 0;
    float l[L::DU];
    for (int j = 0; j < L::DU; j++) l[j] = 0.0f;
    if (n < nelem) {
      const int e = n + off;
      typename L::AT a = __ldg(A + (size_t)jat(mA, e) * L::A);
      l[0] = jac_inc<V>(l[0], beta, a, us[P.loc_u[e] * L::U]);
      md = P.loc_du[e];
      col2 = P.thrcol[e];
    }
    for (int col = 0; col < ncol; col++) {
      if (col2 == col)
        for (int j = 0; j < L::DU; j++) ds[j + md * L::DU] += l[j];
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < sd * L::DU; i += blockDim.x)
    du[(size_t)P.ind_du[od + i / L::DU] * L::DU + i % L::DU] += ds[i];
}

// update (direct): SEQ != nullptr stores u*u in element order for the serial
// fold; the maximum is order independent and always folded as a tree
template <int V>
__global__ void k_jac_update(int n, const float *__restrict__ r, float *__restrict__ du,
                             float *__restrict__ u, float alpha, float *seq,
                             RedSlot<float> s_sum, RedSlot<float> s_max, unsigned *ticket) {
  typedef JacLayout<V> L;
  pdl_wait();
  pdl_trigger();
  float sum = 0.0f, mx = -INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float *up = u + (size_t)i * L::U;
    float *dp = du + (size_t)i * L::DU;
    float uu = *up + (*dp + alpha * __ldg(r + (size_t)i * L::R));
    *up = uu;
    *dp = 0.0f;
    float sq = uu * uu;
    sum += sq;
    mx = (mx > uu) ? mx : uu;
    if (seq) seq[i] = sq;
  }
  const float v[2] = {sum, mx}, id[2] = {0.0f, -INFINITY};
  RedSlot<float> sl[2] = {s_sum, s_max};
  grid_finish<float, OpSum, OpMax, 2>(v, id, OpSum(), OpMax(), sl, ticket);
}

static const int kJacResInds[4] = {-1, 0, 1, -1};

// the pair arrays, by gather plan and the A / u maps they were made for
struct JacPairs {
  const GatherPlan *g;
  op_map mA, mu;
  int iA, iu;
  int2 *d;
};
static std::vector<JacPairs> g_jac_pairs;

static int2 *jac_pairs(const GatherPlan *g, const op_arg *args, cudaStream_t s) {
  if (!tuning("jac_pairs", 1)) return nullptr;
  for (auto &p : g_jac_pairs)
    if (p.g == g && p.mA == args[0].map && p.mu == args[1].map && p.iA == args[0].idx &&
        p.iu == args[1].idx)
      return p.d;
  JacPairs p{g, args[0].map, args[1].map, args[0].idx, args[1].idx, nullptr};
  p.d = (int2 *)dev_alloc(sizeof(int2) * (size_t)std::max(1LL, g->nkeys));
  if (!p.d) return nullptr;
  if (g->nkeys)
    k_jac_pairs<<<rt().num_sms * 8, 256, 0, s>>>(g->nkeys, g->d_keys, idx_map(args[0]),
                                                 idx_map(args[1]), p.d);
  g_jac_pairs.push_back(p);
  return p.d;
}

void release_jac_pairs() {
  for (auto &p : g_jac_pairs) dev_free(p.d);
  g_jac_pairs.clear();
}

// du_out: nullptr (in place) or a spare buffer of du's size, written for
// every node (the loop run ahead: GATHER only, every node a target)
template <int V>
static bool jac_res_t(char const *name, op_set set, const op_arg *args, float *du_out) {
  typedef JacLayout<V> L;
  cudaStream_t s = rt().stream;
  const float beta = *(const float *)args[3].data;  // gbl OP_READ, passed by value
  if (du_out && (V != 1 || effective_strategy(name) == OP2B_STRATEGY_COLOURED)) return false;
  if (effective_strategy(name) == OP2B_STRATEGY_COLOURED) {
    DevPlan *p = get_plan(name, set, OP_part_size, 4, args, 2, kJacResInds);
    if (!p) return false;
    LoopScope ls(name, p->transfer, p->transfer2);
    JacPlanView v;
    v.blkmap = p->d_blkmap; v.offset = p->d_offset; v.nelems = p->d_nelems;
    v.nthrcol = p->d_nthrcol; v.thrcol = p->d_thrcol; v.ind_offs = p->d_ind_offs;
    v.ind_sizes = p->d_ind_sizes; v.ind_u = p->d_ind_maps[0]; v.ind_du = p->d_ind_maps[1];
    v.loc_u = p->d_loc_maps[1]; v.loc_du = p->d_loc_maps[2];
    int nthread = OP_block_size > 0 ? OP_block_size : 512;
    if (p->nshared > 48 * 1024)
      OP2B_CUDA(cudaFuncSetAttribute(k_jac_res_coloured<V>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, p->nshared));
    for (int c = 0, off = 0; c < p->ncolors; off += p->ncolblk[c], c++)
      if (p->ncolblk[c] > 0)
        k_jac_res_coloured<V><<<p->ncolblk[c], nthread, p->nshared, s>>>(
            v, off, idx_map(args[0]), (const typename L::AT *)args[0].dat->data_d,
            (const float *)args[1].dat->data_d, (float *)args[2].dat->data_d, beta);
    return true;
  }
  GatherPlan *g = get_gather_plan(set, args, {2});
  if (!g) return false;
  if (du_out && g->nactive != args[2].dat->set->size) return false;
  LoopScope ls(name, compulsory_bytes(set, 4, args), 0);
  if (g->nactive == 0) return true;
  float *du = (float *)args[2].dat->data_d;
  float *dst = du_out ? du_out : du;
  // (edge, u element) per contribution, built once per plan and map pair
  int2 *pairs = jac_pairs(g, args, s);
  if (pairs)
    launch_pdl(k_jac_res_pairs<V>, (unsigned)((g->nactive + 255) / 256), 256, 0, s, g->nactive,
               (const int *)g->d_active, (const int *)g->d_row, (const int2 *)pairs,
               (const typename L::AT *)args[0].dat->data_d, (const float *)args[1].dat->data_d,
               (const float *)du, beta, dst);
  else
    launch_pdl(k_jac_res_gather<V>, (unsigned)((g->nactive + 255) / 256), 256, 0, s, g->nactive,
               (const int *)g->d_active, (const int *)g->d_row, (const int *)g->d_keys,
               idx_map(args[0]), idx_map(args[1]), (const typename L::AT *)args[0].dat->data_d,
               (const float *)args[1].dat->data_d, (const float *)du, beta, dst);
  return true;
}

void run_jac_res(char const *name, op_set set, const op_arg *args, int variant) {
  if (variant == 2) jac_res_t<2>(name, set, args, nullptr);
  else jac_res_t<1>(name, set, args, nullptr);
}

bool run_jac_res_ahead(char const *name, op_set set, const op_arg *args, int variant,
                       void *du_out) {
  return variant == 1 && jac_res_t<1>(name, set, args, (float *)du_out);
}

bool can_run_jac_res_ahead(char const *name, op_set set, const op_arg *args, int variant) {
  if (variant != 1 || effective_strategy(name) == OP2B_STRATEGY_COLOURED) return false;
  GatherPlan *g = get_gather_plan(set, args, {2});
  return g && g->nactive == args[2].dat->set->size;
}

template <int V>
static void jac_update_t(char const *name, op_set set, const op_arg *args,
                         std::vector<GblRequest> *held) {
  cudaStream_t s = rt().stream;
  float alpha = 0.f;
  if (const_get_f32("alpha", &alpha, 1) < 1) {
    fail(-1, "op2b error -- constant \"alpha\" not declared with op_decl_const2\n");
    return;
  }
  const int n = set->size;
  const bool seq = rt().reduction == OP2B_REDUCE_SEQ;
  int slot_sum = red_new_slot(), slot_max = red_new_slot();
  float *r_sum = (float *)red_slot_ptr(slot_sum), *r_max = (float *)red_slot_ptr(slot_max);
  {
    LoopScope ls(name, compulsory_bytes(set, 5, args), 0);
    float *seqbuf = seq ? (float *)red_seq_buffer(sizeof(float) * (size_t)n) : nullptr;
    const int threads = 256, grid = red_grid(n, threads);
    RedSlot<float> ss{(float *)red_partials(0), r_sum}, sm{(float *)red_partials(1), r_max};
    launch_pdl(k_jac_update<V>, grid, threads, 0, s, n, (const float *)args[0].dat->data_d,
               (float *)args[1].dat->data_d, (float *)args[2].dat->data_d, alpha, seqbuf, ss, sm,
               red_ticket());
    if (seq)
      k_seq_sum<float><<<1, 32, 0, s>>>(seqbuf, n, *(const float *)args[3].data, r_sum,
                                        perm_old2new_dev(set), 1);
  }
  std::vector<GblRequest> rq{GblRequest{args[3].data, slot_sum, OP_INC, GBL_F32, seq},
                             GblRequest{args[4].data, slot_max, OP_MAX, GBL_F32, false}};
  if (held) held->insert(held->end(), rq.begin(), rq.end());  // the caller delivers them
  else red_finish(rq);
}

void run_jac_update(char const *name, op_set set, const op_arg *args, int variant,
                    std::vector<GblRequest> *held) {
  if (variant == 2) jac_update_t<2>(name, set, args, held);
  else jac_update_t<1>(name, set, args, held);
}

// ------------------------------------------------- fused jac1 step ------
// update (iteration k) and the res that follows it (iteration k + 1) as ONE
// launch.  The nodes are cut into tiles of consecutive nodes, and a CTA takes
// a tile.  Phase 1: u after update, u + (du + alpha*r), of every node the
// tile's res contributions read (its own nodes and the neighbours across the
// tile's edges: recomputed by each tile that reads them, with the same
// arithmetic) into shared memory.  Phase 2, per node of the tile: update's
// new u (to the second buffer of u, with the sum and max reductions) and
// res's new du, 0 + beta*A*u' over its contributions in op_seq.h's order (to
// the second buffer of du: update leaves du zero, and res adds to that).
// Other tiles read this tile's old u and du, hence the second buffers, which
// become the datasets' after the launch.  Per element the arithmetic is that
// of k_jac_update and k_jac_res_pairs, so u and du are bit-identical to the
// two launches; only the TREE order of u_sum follows the tiles.

// ELL of the res contributions from the gather plan (every node a target):
// entry j of node i is its j-th (A element, u element) pair, as
// (u element << 1) and the A element, or -1 past the node's count
__global__ void k_jac_ell(int n, int W, const int *__restrict__ row,
                          const int2 *__restrict__ pairs, int *ell_u, int *ell_a) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)n * W;
       i += (long long)gridDim.x * blockDim.x) {
    const int node = (int)(i / W), j = (int)(i % W);
    const int k = row[node] + j;
    if (k < row[node + 1]) {
      const int2 p = pairs[k];
      ell_u[i] = p.y << 1;
      ell_a[i] = p.x;
    } else {
      ell_u[i] = -1;
      ell_a[i] = 0;
    }
  }
}

constexpr int kJacStepW = 8;  // the longest contribution list the fused step takes

template <int BS>
__global__ void __launch_bounds__(BS)
    k_jac_step(int n, int ntile, int ct, int W, const int *__restrict__ toff,
               const int *__restrict__ tflux, const int *__restrict__ tell,
               const int *__restrict__ ell_a, const float *__restrict__ A,
               const float *__restrict__ r, const float *__restrict__ du,
               const float *__restrict__ u, float alpha, float beta, float *__restrict__ u_out,
               float *__restrict__ du_out, float *seq, RedSlot<float> s_sum,
               RedSlot<float> s_max, unsigned *ticket) {
  extern __shared__ float us[];
  constexpr int QA = 4;  // phase-1 elements per thread per pass, loads issued together
  float sum = 0.0f, mx = -INFINITY;
  bool waited = false;
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int beg = __ldg(toff + t), cnt = __ldg(toff + t + 1) - beg;
    // plan data (read-only, before the wait on the first tile): this
    // thread's first phase-1 indices
    int j[QA];
#pragma unroll
    for (int q = 0; q < QA; q++) {
      const int i = threadIdx.x + q * BS;
      j[q] = i < cnt ? __ldg(tflux + beg + i) : -1;
    }
    if (!waited) {
      pdl_wait();
      pdl_trigger();
      waited = true;
    }
    // phase 1: u after update of every node the tile's res reads
    for (int i0 = threadIdx.x; i0 < cnt; i0 += QA * BS) {
      float uu[QA], dd[QA], rr[QA];
#pragma unroll
      for (int q = 0; q < QA; q++)
        if (j[q] >= 0) {
          uu[q] = u[j[q]];
          dd[q] = du[j[q]];
          rr[q] = __ldg(r + j[q]);
        }
      int jn[QA];
#pragma unroll
      for (int q = 0; q < QA; q++) {
        const int i = i0 + (QA + q) * BS;
        jn[q] = i < cnt ? __ldg(tflux + beg + i) : -1;
      }
#pragma unroll
      for (int q = 0; q < QA; q++)
        if (j[q] >= 0) us[i0 + q * BS] = uu[q] + (dd[q] + alpha * rr[q]);  // jac1/update.h:2
#pragma unroll
      for (int q = 0; q < QA; q++) j[q] = jn[q];
    }
    __syncthreads();
    // phase 2: each node's update and res; its own streams and list entries
    // first, then the A values they point to
    const int c1 = min(n, (t + 1) * ct);
    for (int c = t * ct + threadIdx.x; c < c1; c += BS) {
      const float u0 = u[c], d0 = du[c], r0 = __ldg(r + c);
      int kk[kJacStepW], ka[kJacStepW];
#pragma unroll
      for (int m = 0; m < kJacStepW; m++) {
        kk[m] = m < W ? __ldg(tell + (size_t)c * W + m) : -1;
        ka[m] = m < W ? __ldg(ell_a + (size_t)c * W + m) : 0;
      }
      float av[kJacStepW];
#pragma unroll
      for (int m = 0; m < kJacStepW; m++) av[m] = kk[m] >= 0 ? __ldg(A + ka[m]) : 0.0f;
      const float uu = u0 + (d0 + alpha * r0);
      u_out[c] = uu;
      const float sq = uu * uu;
      sum += sq;
      mx = (mx > uu) ? mx : uu;
      if (seq) seq[c] = sq;
      float d = 0.0f;  // update's du = 0, then res adds in list order
#pragma unroll
      for (int m = 0; m < kJacStepW; m++)
        if (kk[m] >= 0) d = jac_inc<1>(d, beta, av[m], us[kk[m] >> 1]);
      du_out[c] = d;
    }
    __syncthreads();  // the next tile reuses the shared u
  }
  if (!waited) {
    pdl_wait();
    pdl_trigger();
  }
  const float v[2] = {sum, mx}, id[2] = {0.0f, -INFINITY};
  RedSlot<float> sl[2] = {s_sum, s_max};
  grid_finish<float, OpSum, OpMax, 2>(v, id, OpSum(), OpMax(), sl, ticket);
}

// the step's plan, by gather plan and the maps of the pairs
struct JacStep {
  const GatherPlan *g;
  op_map mA, mu;
  int iA, iu, ct;
  int W = 0;
  int *ell_a = nullptr;
  TileLists tl;
};
static std::vector<JacStep> g_jac_steps;

void release_jac_steps() {
  for (auto &p : g_jac_steps) {
    if (p.ell_a) cudaFreeAsync(p.ell_a, rt().stream);
    free_tile_lists(&p.tl, rt().stream);
  }
  g_jac_steps.clear();
}

static JacStep *jac_step_plan(const GatherPlan *g, const op_arg *ra, int2 *pairs, int ct,
                              cudaStream_t s) {
  for (auto &p : g_jac_steps)
    if (p.g == g && p.mA == ra[0].map && p.mu == ra[1].map && p.iA == ra[0].idx &&
        p.iu == ra[1].idx && p.ct == ct)
      return &p;
  const int n = g->ntarget, W = g->max_row;
  if (W < 1 || W > kJacStepW || (long long)n * W >= (1LL << 31)) return nullptr;
  JacStep p{g, ra[0].map, ra[1].map, ra[0].idx, ra[1].idx, ct};
  p.W = W;
  int *ell_u = nullptr;
  if (pool_malloc_async((void **)&ell_u, sizeof(int) * (size_t)n * W, s) != cudaSuccess ||
      pool_malloc_async((void **)&p.ell_a, sizeof(int) * (size_t)n * W, s) != cudaSuccess) {
    cudaGetLastError();
    if (ell_u) cudaFreeAsync(ell_u, s);
    if (p.ell_a) cudaFreeAsync(p.ell_a, s);
    return nullptr;
  }
  k_jac_ell<<<rt().num_sms * 8, 256, 0, s>>>(n, W, g->d_row, pairs, ell_u, p.ell_a);
  const bool ok = build_tile_lists(ell_u, n, W, ct, s, &p.tl);
  cudaFreeAsync(ell_u, s);
  if (!ok) {
    cudaFreeAsync(p.ell_a, s);
    return nullptr;
  }
  g_jac_steps.push_back(p);
  return &g_jac_steps.back();
}

// jac1's update `ua` (r, du, u, u_sum, u_max) followed by its res `ra`
// (A, u through the map, du incremented through the map, beta) as one
// launch; false when the shapes do not suit it (the caller runs both)
bool run_jac_step(char const *uname, op_set uset, const op_arg *ua, char const *rname,
                  op_set rset, const op_arg *ra) {
  if (!tuning("jac_step", 1) || effective_strategy(rname) == OP2B_STRATEGY_COLOURED) return false;
  op_dat r = ua[0].dat, du = ua[1].dat, u = ua[2].dat;
  if (ra[1].dat != u || ra[2].dat != du || ra[0].dat == u || ra[0].dat == du ||
      r == u || r == du || !ra[1].map || !ra[2].map || ra[0].map)
    return false;
  cudaStream_t s = rt().stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  OP2B_CUDA(cudaStreamIsCapturing(s, &cap));
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (!capturing && live_graphs() > 0) return false;  // graphs hold the buffers they captured
  GatherPlan *g = get_gather_plan(rset, ra, {2});
  if (!g || g->nactive != uset->size || g->d_active || uset != du->set) return false;
  int2 *pairs = jac_pairs(g, ra, s);
  if (!pairs) return false;
  const int n = uset->size;
  // threads per CTA (knob jac_step_threads: 512, 1024 or 256) and nodes per
  // tile (knob jac_tile_nodes; 0: one tile per resident CTA -- two CTAs of
  // 512 per SM at the kernel's 63 registers -- so that every SM gets the
  // same share)
  const int BS = tuning("jac_step_threads", 512) == 1024 ? 1024
                 : tuning("jac_step_threads", 512) == 256 ? 256 : 512;
  const long long slots = (long long)rt().num_sms * std::max(1, 1024 / BS);
  const int ct = tuning("jac_tile_nodes", 0) > 0
                     ? std::max(64, tuning("jac_tile_nodes", 0))
                     : (int)std::max(64LL, (n + slots - 1) / slots);
  JacStep *p = nullptr;
  for (auto &q : g_jac_steps)
    if (q.g == g && q.mA == ra[0].map && q.mu == ra[1].map && q.iA == ra[0].idx &&
        q.iu == ra[1].idx && q.ct == ct)
      p = &q;
  if (!p) {
    if (capturing) return false;  // plans are built before a capture
    p = jac_step_plan(g, ra, pairs, ct, s);
    if (!p) return false;
  }
  const size_t smem = sizeof(float) * (size_t)std::max(1, p->tl.maxcnt);
  if (smem > (size_t)rt().smem_optin - 1024) return false;
  float alpha = 0.f;
  if (const_get_f32("alpha", &alpha, 1) < 1) return false;
  const float beta = *(const float *)ra[3].data;
  float *u_out = (float *)alt_of(u), *du_out = (float *)alt_of(du);
  if (!u_out || !du_out || error_pending()) return false;
  auto kern = BS == 1024 ? k_jac_step<1024> : BS == 256 ? k_jac_step<256> : k_jac_step<512>;
  static size_t sized[3] = {0, 0, 0};
  size_t &have = sized[BS == 1024 ? 2 : BS == 256 ? 0 : 1];
  if (smem > 48 * 1024 && smem > have) {
    OP2B_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    have = smem;
  }
  const bool seq = rt().reduction == OP2B_REDUCE_SEQ;
  int slot_sum = red_new_slot(), slot_max = red_new_slot();
  float *r_sum = (float *)red_slot_ptr(slot_sum), *r_max = (float *)red_slot_ptr(slot_max);
  {
    std::string name = std::string(uname) + "+" + rname;
    LoopScope ls(name.c_str(),
                 compulsory_bytes(uset, 5, ua) + compulsory_bytes(rset, 4, ra), 0);
    float *seqbuf = seq ? (float *)red_seq_buffer(sizeof(float) * (size_t)n) : nullptr;
    const int grid = std::min(p->tl.ntile, kMaxRedBlocks);
    RedSlot<float> ss{(float *)red_partials(0), r_sum}, sm{(float *)red_partials(1), r_max};
    launch_pdl(kern, grid, BS, smem, s, n, p->tl.ntile, p->tl.ct, p->W,
               (const int *)p->tl.toff, (const int *)p->tl.tflux, (const int *)p->tl.tell,
               (const int *)p->ell_a, (const float *)ra[0].dat->data_d,
               (const float *)r->data_d, (const float *)du->data_d, (const float *)u->data_d,
               alpha, beta, u_out, du_out, seqbuf, ss, sm, red_ticket());
    if (seq)
      k_seq_sum<float><<<1, 32, 0, s>>>(seqbuf, n, *(const float *)ua[3].data, r_sum,
                                        perm_old2new_dev(uset), 1);
  }
  if (error_pending()) return true;
  flip(u, capturing);
  flip(du, capturing);
  red_finish({GblRequest{ua[3].data, slot_sum, OP_INC, GBL_F32, seq},
              GblRequest{ua[4].data, slot_max, OP_MAX, GBL_F32, false}});
  return true;
}

}  // namespace op2b
