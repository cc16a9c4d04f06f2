// renumber.cu -- optional renumbering of every set for locality of the
// indirect gathers (op2b_set_renumber).
//
// A mesh whose numbering is scrambled turns each gather into a random
// access.  When renumbering is on, the first loop call orders every set,
// all of it computed on the GPU:
//  - with coordinates given (op2b_set_renumber_coords), the anchor set is
//    the coordinates' set, ordered by recursive coordinate bisection
//    (rcb_order below);
//  - otherwise the anchor set is the one most maps point to (ties: the larger);
//    elements that share a row of a map of dim >= 2 onto it are neighbours
//    (a CSR graph built by count, scan and fill kernels), and a
//    level-synchronous breadth-first walk from a least-connected element of
//    each connected component gives its order (Cuthill-McKee): each level is
//    found in one parallel expansion of the previous one and ordered by the
//    smallest new index among an element's parents, ties by old index (a
//    counting sort by parent, then a sort within each parent's bucket), so
//    the order is deterministic whatever the threads' timing;
//  - every set with a map onto an ordered set follows: its elements sorted
//    by the smallest new index they point to (ties by old index);
//  - a set only pointed to by an ordered set takes the order in which the
//    ordered set's rows first reach it (unreached elements last, in order);
//  - anything left keeps its numbering.
// The host only decides which set follows which and reads one count per
// level of the walk.
// Each dataset is then stored permuted on the device (element i of the new
// order is element P[i] of the app's), each map's device copy is rewritten
// on the device with its rows in the new order of its from-set and its
// values in the new numbering of its to-set, and op_fetch_data puts the
// app's order back.
//
// Results do not change: per-element arithmetic is the same, and the
// owner-computes plans order each target's contributions by the APP's
// element numbers (get_gather_plan sorts by original keys), which is still
// op_seq.h's order.  Global sums in TREE mode are summed in another order
// (as with any launch shape); plans returned by op_plan_get describe the
// renumbered sets.

#include <limits.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "internal.h"
#include "plan.h"

namespace op2b {

namespace {

struct SetPerm {
  std::vector<int> P;                  // new -> old (host copy, for op2b_renumber_order)
  int *d_P = nullptr, *d_Q = nullptr;  // new -> old, old -> new
};

std::vector<SetPerm> g_perm;  // by set index; empty P: not permuted
bool g_enabled = false, g_applied = false, g_computed = false;
op_dat g_rcb = nullptr;  // coordinates: order by bisection instead of Cuthill-McKee
double g_order_seconds = 0.0;  // the last order computation, GPU work included

bool permuted(int set_index) {
  return set_index < (int)g_perm.size() && g_perm[set_index].d_P;
}

// ----------------------------------------------------------- kernels ----

#define GRID_STRIDE(i, n)                                                     \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); \
       i += (long long)gridDim.x * blockDim.x)

__global__ void k_fill_int(int *p, long long n, int v) {
  GRID_STRIDE(i, n) p[i] = v;
}

// every entry of a map row is a neighbour of the dim - 1 others
__global__ void k_degree(const int *__restrict__ map, long long rows, int dim, int *deg) {
  GRID_STRIDE(e, rows * dim) atomicAdd(deg + map[e], dim - 1);
}

__global__ void k_adjacency(const int *__restrict__ map, long long rows, int dim,
                            const int *__restrict__ off, int *cur, int *adj) {
  GRID_STRIDE(e, rows * dim) {
    const long long r = e / dim;
    const int a = (int)(e % dim), v = map[e];
    for (int b = 0; b < dim; b++)
      if (b != a) adj[off[v] + atomicAdd(cur + v, 1)] = map[r * dim + b];
  }
}

// least (degree, index) among the elements not yet placed
__global__ void k_seed(const int *__restrict__ level, const int *__restrict__ deg, long long n,
                       unsigned long long *best) {
  unsigned long long mine = ~0ull;
  GRID_STRIDE(v, n) if (level[v] < 0) {
    const unsigned long long k = ((unsigned long long)(unsigned)deg[v] << 32) | (unsigned)v;
    mine = k < mine ? k : mine;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_down_sync(0xffffffffu, mine, o);
    mine = x < mine ? x : mine;
  }
  if ((threadIdx.x & 31) == 0 && mine != ~0ull) atomicMin(best, mine);
}

__global__ void k_seed_place(const unsigned long long *best, int *order, int pos, int *level) {
  const int v = (int)(*best & 0xffffffffull);
  order[pos] = v;
  level[v] = 0;
}

// one breadth-first level: the neighbours of order[fs, fe) not yet reached
// join level L + 1 (appended to next, unordered); each records the smallest
// position of a parent (pkey) for the ordering of the level
__global__ void k_expand(const int *__restrict__ order, int fs, int fe,
                         const int *__restrict__ off, const int *__restrict__ adj, int *level,
                         int L, int *pkey, int *next, int *count) {
  GRID_STRIDE(t, (long long)(fe - fs)) {
    const int p = fs + (int)t, v = order[p];
    for (int j = off[v]; j < off[v + 1]; j++) {
      const int w = adj[j];
      const int old = atomicCAS(level + w, -1, L + 1);
      if (old == -1) next[atomicAdd(count, 1)] = w;
      if (old == -1 || old == L + 1) atomicMin(pkey + w, p);
    }
  }
}

// bucket key of each listed element: its parent's position minus base
__global__ void k_level_keys(const int *__restrict__ items, int n, const int *__restrict__ pkey,
                             int base, int *bkey) {
  GRID_STRIDE(i, (long long)n) bkey[i] = pkey[items[i]] - base;
}

// bucket key of element e of a set with a map onto an ordered set: the
// smallest new index it points to
__global__ void k_row_min_key(const int *__restrict__ map, long long rows, int dim,
                              const int *__restrict__ Q, int *bkey) {
  GRID_STRIDE(r, rows) {
    int m = INT_MAX;
    for (int a = 0; a < dim; a++) m = min(m, Q[map[r * dim + a]]);
    bkey[r] = m;
  }
}

// first slot (new row x dim + column) of an ordered set's map that reaches
// each element of the to-set
__global__ void k_reach_key(const int *__restrict__ map, long long rows, int dim,
                            const int *__restrict__ Qfrom, int *rkey) {
  GRID_STRIDE(e, rows * dim) {
    const long long r = e / dim;
    atomicMin(rkey + map[e], Qfrom[r] * dim + (int)(e % dim));
  }
}

// unreached elements go last, in their old order: key after every slot
__global__ void k_reach_finish(int *rkey, long long n, long long slots) {
  GRID_STRIDE(v, n) if (rkey[v] == INT_MAX) rkey[v] = (int)(slots + v);
}

__global__ void k_bucket_count(const int *__restrict__ bkey, int n, int *cnt) {
  GRID_STRIDE(i, (long long)n) atomicAdd(cnt + bkey[i], 1);
}

__global__ void k_bucket_place(const int *__restrict__ items, const int *__restrict__ bkey, int n,
                               const int *__restrict__ boff, int *cur, int *out) {
  GRID_STRIDE(i, (long long)n) {
    const int b = bkey[i];
    out[boff[b] + atomicAdd(cur + b, 1)] = items ? items[i] : (int)i;
  }
}

// each bucket's elements by index (buckets hold a few elements: the
// neighbours of one parent, the rows whose smallest target is one element)
__global__ void k_bucket_sort(int *out, const int *__restrict__ boff, int nb, int n) {
  GRID_STRIDE(b, (long long)nb) {
    const int lo = boff[b], hi = b + 1 < nb ? boff[b + 1] : n;
    for (int i = lo + 1; i < hi; i++) {
      const int x = out[i];
      int j = i - 1;
      while (j >= lo && out[j] > x) {
        out[j + 1] = out[j];
        j--;
      }
      out[j + 1] = x;
    }
  }
}

// The whole walk in one CTA, without host round trips: each level is
// expanded by all threads (atomics on level and pkey, which are read back
// through L2 since L1 does not see atomics), then sorted by (parent
// position, index) with a bitonic sort in shared memory.  status: 0 done,
// 1 a level wider than kBfsCtaMax (the caller falls back to the
// multi-launch walk).
constexpr int kBfsCtaMax = 8192;
__global__ void __launch_bounds__(1024)
    k_bfs_cta(int n, const int *__restrict__ off, const int *__restrict__ adj,
              const int *__restrict__ deg, int *level, int *pkey, int *order, int *next,
              int *status) {
  extern __shared__ unsigned long long keys[];  // kBfsCtaMax
  __shared__ int s_cnt;
  __shared__ unsigned long long s_best;
  const int tid = threadIdx.x, nt = blockDim.x;
  int placed = 0;
  while (placed < n) {  // one connected component per pass
    if (tid == 0) s_best = ~0ull;
    __syncthreads();
    unsigned long long mine = ~0ull;
    for (int v = tid; v < n; v += nt)
      if (__ldcg(level + v) < 0) {
        const unsigned long long k = ((unsigned long long)(unsigned)deg[v] << 32) | (unsigned)v;
        mine = k < mine ? k : mine;
      }
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long x = __shfl_down_sync(0xffffffffu, mine, o);
      mine = x < mine ? x : mine;
    }
    if ((tid & 31) == 0) atomicMin(&s_best, mine);
    __syncthreads();
    if (tid == 0) {
      const int v = (int)(s_best & 0xffffffffull);
      order[placed] = v;
      atomicExch(level + v, 0);
    }
    int fs = placed, fe = placed + 1, L = 0;
    __syncthreads();
    for (;;) {
      if (tid == 0) s_cnt = 0;
      __syncthreads();
      for (int p = fs + tid; p < fe; p += nt) {
        const int v = order[p];
        for (int j = off[v]; j < off[v + 1]; j++) {
          const int w = adj[j];
          const int old = atomicCAS(level + w, -1, L + 1);
          if (old == -1) {
            const int slot = atomicAdd(&s_cnt, 1);
            if (slot < kBfsCtaMax) next[slot] = w;
          }
          if (old == -1 || old == L + 1) atomicMin(pkey + w, p);
        }
      }
      __syncthreads();
      const int c = s_cnt;
      if (c == 0) break;
      if (c > kBfsCtaMax || fe + c > n) {
        if (tid == 0) *status = 1;
        return;
      }
      int m = 1;
      while (m < c) m <<= 1;
      for (int i = tid; i < m; i += nt)
        keys[i] = i < c ? ((unsigned long long)(unsigned)__ldcg(pkey + next[i]) << 32) |
                              (unsigned)next[i]
                        : ~0ull;
      __syncthreads();
      for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = tid; i < m; i += nt) {
            const int ixj = i ^ j;
            if (ixj > i) {
              const unsigned long long a = keys[i], b = keys[ixj];
              if ((a > b) == ((i & k) == 0)) {
                keys[i] = b;
                keys[ixj] = a;
              }
            }
          }
          __syncthreads();
        }
      for (int i = tid; i < c; i += nt) order[fe + i] = (int)(keys[i] & 0xffffffffull);
      __syncthreads();
      fs = fe;
      fe += c;
      L++;
    }
    placed = fe;
    __syncthreads();
  }
  if (tid == 0) *status = 0;
}

__global__ void k_inverse(const int *__restrict__ P, long long n, int *Q) {
  GRID_STRIDE(i, n) Q[P[i]] = (int)i;
}

// out[i * dim + a] = Qto[in[Pfrom[i] * dim + a]] (either permutation optional)
__global__ void k_renumber_map(const int *__restrict__ in, long long rows, int dim,
                               const int *__restrict__ Pfrom, const int *__restrict__ Qto,
                               int *out) {
  GRID_STRIDE(e, rows * dim) {
    const long long i = e / dim;
    const int a = (int)(e % dim);
    const long long src = Pfrom ? Pfrom[i] : i;
    const int v = in[src * dim + a];
    out[e] = Qto ? Qto[v] : v;
  }
}

// ------------------------------------- recursive coordinate bisection ----

// unsigned key with the order of the float f (-0 before +0)
__device__ __forceinline__ unsigned float_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// component a of every element's coordinates, rounded to float, into cf,
// and the sort keys (coordinate key, element) padded with ~0 up to m
template <class T>
__global__ void k_rcb_keys(const T *__restrict__ xyz, long long n, int dim, int a, long long m,
                           float *cf, unsigned long long *key) {
  GRID_STRIDE(i, m) {
    if (i < n) {
      const float f = (float)xyz[i * dim + a];
      cf[i] = f;
      key[i] = ((unsigned long long)float_key(f) << 32) | (unsigned)i;
    } else {
      key[i] = ~0ull;
    }
  }
}

// Bitonic sort of 64-bit keys in chunks of c (a power of two <= kSortChunk)
// in shared memory: with k = 0 every chunk is sorted (stages 2..c, each
// chunk ascending or descending by its place in the whole array); with
// k > c the steps j = c/2 .. 1 of stage k, after k_bitonic_step has done
// the steps j >= c that cross chunks.
constexpr int kSortChunk = 2048;
__global__ void __launch_bounds__(1024)
    k_bitonic_chunk(unsigned long long *a, int c, long long k) {
  __shared__ unsigned long long s[kSortChunk];
  const long long base = (long long)blockIdx.x * c;
  for (int i = threadIdx.x; i < c; i += blockDim.x) s[i] = a[base + i];
  __syncthreads();
  const long long k0 = k ? k : 2, k1 = k ? k : c;
  for (long long kk = k0; kk <= k1; kk <<= 1)
    for (int j = (int)(kk < c ? kk : c) >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < c / 2; t += blockDim.x) {
        const int i = 2 * j * (t / j) + t % j, l = i + j;
        const bool up = ((base + i) & kk) == 0;
        const unsigned long long x = s[i], y = s[l];
        if ((x > y) == up) {
          s[i] = y;
          s[l] = x;
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < c; i += blockDim.x) a[base + i] = s[i];
}

// one step (stage k, distance j) of the bitonic sort over the whole array
__global__ void k_bitonic_step(unsigned long long *a, long long m, long long k, long long j) {
  GRID_STRIDE(t, m / 2) {
    const long long i = 2 * j * (t / j) + t % j, l = i + j;
    const bool up = (i & k) == 0;
    const unsigned long long x = a[i], y = a[l];
    if ((x > y) == up) {
      a[i] = y;
      a[l] = x;
    }
  }
}

__global__ void k_rcb_list(const unsigned long long *__restrict__ key, int n, int *La) {
  GRID_STRIDE(p, (long long)n) La[p] = (int)(unsigned)(key[p] & 0xffffffffull);
}

// The lists L (one per axis, n positions each) hold the same elements in
// every segment [lo, hi); list a orders a segment by coordinate a.  Each
// segment of two or more is halved at mid = lo + (hi - lo) / 2 along the
// axis of its largest extent (last minus first coordinate in that axis'
// list; ties: the lower axis): the elements at positions >= mid of that
// axis' list take side 1, the rest side 0.  Every element gets its side
// from exactly one position.
__global__ void k_rcb_side(const int *__restrict__ L, const float *__restrict__ cf, int n, int dim,
                           const int *__restrict__ seg_lo, const int *__restrict__ seg_hi,
                           int *side) {
  GRID_STRIDE(p, (long long)n) {
    const int lo = seg_lo[p], hi = seg_hi[p];
    if (hi - lo < 2) {
      side[L[p]] = 0;
      continue;
    }
    int ax = 0;
    float best = 0.0f;
    for (int a = 0; a < dim; a++) {
      const int *La = L + (size_t)a * n;
      const float *ca = cf + (size_t)a * n;
      const float e = ca[La[hi - 1]] - ca[La[lo]];
      if (a == 0 || e > best) {
        best = e;
        ax = a;
      }
    }
    side[L[(size_t)ax * n + p]] = (int)p >= lo + (hi - lo) / 2;
  }
}

__global__ void k_rcb_flags(const int *__restrict__ La, const int *__restrict__ side, int n,
                            int *f) {
  GRID_STRIDE(p, (long long)n) f[p] = side[La[p]];
}

// stable partition of list a within each halved segment: side 0 to
// [lo, mid), side 1 to [mid, hi), each in its list order (S: exclusive scan
// of the flags f)
__global__ void k_rcb_scatter(const int *__restrict__ La, const int *__restrict__ f,
                              const int *__restrict__ S, int n, const int *__restrict__ seg_lo,
                              const int *__restrict__ seg_hi, int *out) {
  GRID_STRIDE(p, (long long)n) {
    const int lo = seg_lo[p], hi = seg_hi[p];
    int q = (int)p;
    if (hi - lo >= 2) {
      const int mid = lo + (hi - lo) / 2, ones = S[p] - S[lo];
      q = f[p] ? mid + ones : (int)p - ones;
      if (q < lo || q >= hi) continue;  // cannot happen: every list holds the segment's elements
    }
    out[q] = La[p];
  }
}

__global__ void k_rcb_halve(int n, int *seg_lo, int *seg_hi) {
  GRID_STRIDE(p, (long long)n) {
    const int lo = seg_lo[p], hi = seg_hi[p];
    if (hi - lo >= 2) {
      const int mid = lo + (hi - lo) / 2;
      if ((int)p < mid) seg_hi[p] = mid;
      else seg_lo[p] = mid;
    }
  }
}

#undef GRID_STRIDE

// --------------------------------------------------------- host driver ----

int grid_for_n(long long n) {
  return (int)std::max(1LL, std::min((n + 255) / 256, (long long)rt().num_sms * 8));
}

struct DevInts {  // scoped device scratch
  int *p = nullptr;
  explicit DevInts(long long n) { p = (int *)dev_alloc(sizeof(int) * (size_t)std::max(1LL, n)); }
  ~DevInts() { dev_free(p); }
  DevInts(const DevInts &) = delete;
  DevInts &operator=(const DevInts &) = delete;
};

// items (0..n-1 when null) ordered by (bkey, item) into out; bkey in [0, nb)
bool bucket_sort(const int *items, const int *bkey, int n, long long nb, int *out) {
  if (n <= 0) return true;
  if (nb <= 0 || nb >= INT_MAX) return false;
  cudaStream_t s = rt().stream;
  DevInts cnt(nb), off(nb), cur(nb);
  if (!cnt.p || !off.p || !cur.p) return false;
  OP2B_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (size_t)nb, s));
  OP2B_CUDA(cudaMemsetAsync(cur.p, 0, sizeof(int) * (size_t)nb, s));
  k_bucket_count<<<grid_for_n(n), 256, 0, s>>>(bkey, n, cnt.p);
  exclusive_scan(cnt.p, off.p, (int)nb, s);
  k_bucket_place<<<grid_for_n(n), 256, 0, s>>>(items, bkey, n, off.p, cur.p, out);
  k_bucket_sort<<<grid_for_n(nb), 256, 0, s>>>(out, off.p, (int)nb, n);
  return !error_pending();
}

// the order d_P (new -> old, device, owned by the set's entry from now on)
// of set s: its inverse and a host copy
void set_perm(op_set s, int *d_P) {
  if ((int)g_perm.size() <= s->index) g_perm.resize(s->index + 1);
  SetPerm &sp = g_perm[s->index];
  dev_free(sp.d_P);
  dev_free(sp.d_Q);
  sp.d_P = d_P;
  sp.d_Q = (int *)dev_alloc(sizeof(int) * (size_t)std::max(1, s->size));
  sp.P.assign(s->size, 0);
  if (!sp.d_Q) return;
  k_inverse<<<grid_for_n(s->size), 256, 0, rt().stream>>>(d_P, s->size, sp.d_Q);
  OP2B_CUDA(cudaMemcpyAsync(sp.P.data(), d_P, sizeof(int) * (size_t)s->size,
                            cudaMemcpyDeviceToHost, rt().stream));
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
}

// Cuthill-McKee order of the anchor set's neighbour graph, on the device
int *anchor_order(op_set s) {
  cudaStream_t st = rt().stream;
  const int n = s->size;
  std::vector<op_map> onto;
  for (int k = 0; k < OP_map_index; k++) {
    op_map m = OP_map_list[k];
    if (m->to == s && m->dim >= 2) onto.push_back(m);
  }
  DevInts deg(n), off(n + 1), cur(n), level(n), pkey(n), next(n), bkey(n), count(1);
  int *order = (int *)dev_alloc(sizeof(int) * (size_t)std::max(1, n));
  unsigned long long *best = (unsigned long long *)dev_alloc(sizeof(unsigned long long));
  auto fail_out = [&]() {
    dev_free(order);
    dev_free(best);
    return (int *)nullptr;
  };
  if (!order || !best || !deg.p || !off.p || !cur.p || !level.p || !pkey.p || !next.p ||
      !bkey.p || !count.p)
    return fail_out();
  OP2B_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(int) * (size_t)n, st));
  for (op_map m : onto)
    k_degree<<<grid_for_n((long long)m->from->size * m->dim), 256, 0, st>>>(
        map_dev(m), m->from->size, m->dim, deg.p);
  const long long nnz = exclusive_scan(deg.p, off.p, n, st);
  if (nnz >= INT_MAX) return fail_out();
  const int nnz_i = (int)nnz;
  OP2B_CUDA(cudaMemcpyAsync(off.p + n, &nnz_i, sizeof(int), cudaMemcpyHostToDevice, st));
  DevInts adj(nnz);
  if (!adj.p) return fail_out();
  OP2B_CUDA(cudaMemsetAsync(cur.p, 0, sizeof(int) * (size_t)n, st));
  for (op_map m : onto)
    k_adjacency<<<grid_for_n((long long)m->from->size * m->dim), 256, 0, st>>>(
        map_dev(m), m->from->size, m->dim, off.p, cur.p, adj.p);
  k_fill_int<<<grid_for_n(n), 256, 0, st>>>(level.p, n, -1);
  k_fill_int<<<grid_for_n(n), 256, 0, st>>>(pkey.p, n, INT_MAX);
  {  // the whole walk in one CTA; levels wider than kBfsCtaMax fall back below
    const size_t smem = sizeof(unsigned long long) * kBfsCtaMax;
    static bool sized = false;
    if (!sized) {
      OP2B_CUDA(cudaFuncSetAttribute(k_bfs_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
      sized = true;
    }
    int status = 2;
    OP2B_CUDA(cudaMemsetAsync(count.p, 0xff, sizeof(int), st));
    k_bfs_cta<<<1, 1024, smem, st>>>(n, off.p, adj.p, deg.p, level.p, pkey.p, order, next.p,
                                     count.p);
    OP2B_CUDA(cudaMemcpyAsync(&status, count.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    OP2B_CUDA(cudaStreamSynchronize(st));
    if (error_pending()) return fail_out();
    if (status == 0) {
      dev_free(best);
      return order;
    }
    k_fill_int<<<grid_for_n(n), 256, 0, st>>>(level.p, n, -1);
    k_fill_int<<<grid_for_n(n), 256, 0, st>>>(pkey.p, n, INT_MAX);
  }
  int placed = 0;
  while (placed < n) {  // one connected component per pass
    OP2B_CUDA(cudaMemsetAsync(best, 0xff, sizeof(unsigned long long), st));
    k_seed<<<grid_for_n(n), 256, 0, st>>>(level.p, deg.p, n, best);
    k_seed_place<<<1, 1, 0, st>>>(best, order, placed, level.p);
    int fs = placed, fe = placed + 1, L = 0;
    for (;;) {
      OP2B_CUDA(cudaMemsetAsync(count.p, 0, sizeof(int), st));
      k_expand<<<grid_for_n(fe - fs), 256, 0, st>>>(order, fs, fe, off.p, adj.p, level.p, L,
                                                    pkey.p, next.p, count.p);
      int c = 0;
      OP2B_CUDA(cudaMemcpyAsync(&c, count.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      OP2B_CUDA(cudaStreamSynchronize(st));
      if (error_pending()) return fail_out();
      if (c <= 0 || fe + c > n) break;
      k_level_keys<<<grid_for_n(c), 256, 0, st>>>(next.p, c, pkey.p, fs, bkey.p);
      if (!bucket_sort(next.p, bkey.p, c, fe - fs, order + fe)) return fail_out();
      fs = fe;
      fe += c;
      L++;
    }
    placed = fe;
  }
  dev_free(best);
  return order;
}

// sorts the m 64-bit keys at a (m a power of two) ascending
bool bitonic_sort(unsigned long long *a, long long m, cudaStream_t st) {
  if (m < 2) return true;
  const int c = (int)std::min<long long>(kSortChunk, m);
  const int threads = std::min(1024, c / 2);
  const unsigned chunks = (unsigned)(m / c);
  k_bitonic_chunk<<<chunks, threads, 0, st>>>(a, c, 0);
  for (long long k = 2LL * c; k <= m; k <<= 1) {
    for (long long j = k >> 1; j >= c; j >>= 1)
      k_bitonic_step<<<grid_for_n(m / 2), 256, 0, st>>>(a, m, k, j);
    k_bitonic_chunk<<<chunks, threads, 0, st>>>(a, c, k);
  }
  return !error_pending();
}

// Recursive coordinate bisection of the coordinates' set (the reference's
// developer notes propose it for renumbering, doc/dev.tex:191-210): every
// segment of the order -- at first the whole set -- is halved at its median
// along the axis of its largest extent, the lower half first, until every
// segment holds one element.  Coordinates are compared rounded to float,
// ties by element number; each axis is sorted once (bitonic), and each
// level is a stable partition of every axis' list by the halves (one scan
// per axis), so the order is deterministic.
int *rcb_order(op_dat xyz) {
  cudaStream_t st = rt().stream;
  const int n = xyz->set->size, dim = xyz->dim;
  const bool dbl = strcmp(xyz->type, "double") == 0;
  long long m = 1;
  while (m < n) m <<= 1;
  DevInts L((long long)dim * n), L2((long long)dim * n), lo(n), hi(n), side(n), f(n), S(n);
  float *cf = (float *)dev_alloc(sizeof(float) * (size_t)dim * std::max(1, n));
  unsigned long long *key = (unsigned long long *)dev_alloc(sizeof(unsigned long long) * (size_t)m);
  int *order = (int *)dev_alloc(sizeof(int) * (size_t)std::max(1, n));
  bool ok = cf && key && order && L.p && L2.p && lo.p && hi.p && side.p && f.p && S.p;
  for (int a = 0; ok && a < dim; a++) {
    if (dbl)
      k_rcb_keys<double><<<grid_for_n(m), 256, 0, st>>>((const double *)xyz->data_d, n, dim, a,
                                                          m, cf + (size_t)a * n, key);
    else
      k_rcb_keys<float><<<grid_for_n(m), 256, 0, st>>>((const float *)xyz->data_d, n, dim, a, m,
                                                         cf + (size_t)a * n, key);
    ok = bitonic_sort(key, m, st);
    k_rcb_list<<<grid_for_n(n), 256, 0, st>>>(key, n, L.p + (size_t)a * n);
  }
  if (ok) {
    k_fill_int<<<grid_for_n(n), 256, 0, st>>>(lo.p, n, 0);
    k_fill_int<<<grid_for_n(n), 256, 0, st>>>(hi.p, n, n);
  }
  int *cur = L.p, *nxt = L2.p;
  for (long long longest = n; ok && longest >= 2; longest = (longest + 1) / 2) {
    k_rcb_side<<<grid_for_n(n), 256, 0, st>>>(cur, cf, n, dim, lo.p, hi.p, side.p);
    for (int a = 0; a < dim; a++) {
      const int *La = cur + (size_t)a * n;
      k_rcb_flags<<<grid_for_n(n), 256, 0, st>>>(La, side.p, n, f.p);
      exclusive_scan(f.p, S.p, n, st);
      k_rcb_scatter<<<grid_for_n(n), 256, 0, st>>>(La, f.p, S.p, n, lo.p, hi.p,
                                                   nxt + (size_t)a * n);
    }
    k_rcb_halve<<<grid_for_n(n), 256, 0, st>>>(n, lo.p, hi.p);
    std::swap(cur, nxt);
    ok = !error_pending();
  }
  if (ok)
    OP2B_CUDA(cudaMemcpyAsync(order, cur, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
  OP2B_CUDA(cudaStreamSynchronize(st));  // the scratch is freed on return
  dev_free(cf);
  dev_free(key);
  if (!ok || error_pending()) {
    dev_free(order);
    return nullptr;
  }
  return order;
}

void compute_orders() {
  for (auto &sp : g_perm) {
    dev_free(sp.d_P);
    dev_free(sp.d_Q);
  }
  g_perm.clear();
  g_perm.resize(OP_set_index);
  g_computed = true;
  if (OP_set_index == 0) return;
  ensure_cuda();
  cudaStream_t st = rt().stream;
  // anchor: the coordinates' set under coordinate bisection; else most
  // maps onto it, then the larger
  op_set anchor = nullptr;
  int best = -1;
  if (g_rcb) {
    if (g_rcb->set->size == 0) return;
    int *P = rcb_order(g_rcb);
    if (!P) return;
    set_perm(g_rcb->set, P);
    anchor = g_rcb->set;
  }
  for (int k = 0; k < OP_set_index && !anchor; k++) {
    op_set s = OP_set_list[k];
    int score = 0;
    for (int j = 0; j < OP_map_index; j++)
      if (OP_map_list[j]->to == s && OP_map_list[j]->dim >= 2) score++;
    if (score > best || (score == best && anchor && s->size > anchor->size)) {
      best = score;
      anchor = s;
    }
  }
  if (!g_rcb) {
    if (best <= 0 || anchor->size == 0) return;  // no map with shared rows: nothing to gain
    int *P = anchor_order(anchor);
    if (!P) return;
    set_perm(anchor, P);
  }
  bool progress = true;
  while (progress) {
    progress = false;
    for (int k = 0; k < OP_set_index; k++) {
      op_set s = OP_set_list[k];
      if (permuted(s->index) || s->size == 0) continue;
      // a map from s onto an ordered set
      op_map via = nullptr;
      for (int j = 0; j < OP_map_index && !via; j++) {
        op_map m = OP_map_list[j];
        if (m->from == s && m->dim >= 1 && permuted(m->to->index)) via = m;
      }
      if (via) {
        DevInts key(s->size);
        int *dP = (int *)dev_alloc(sizeof(int) * (size_t)s->size);
        if (!key.p || !dP) return;
        k_row_min_key<<<grid_for_n(s->size), 256, 0, st>>>(map_dev(via), s->size, via->dim,
                                                           g_perm[via->to->index].d_Q, key.p);
        if (!bucket_sort(nullptr, key.p, s->size, via->to->size, dP)) {
          dev_free(dP);
          return;
        }
        set_perm(s, dP);
        progress = true;
        continue;
      }
      // a map from an ordered set onto s
      for (int j = 0; j < OP_map_index; j++) {
        op_map m = OP_map_list[j];
        if (m->to != s || m->dim < 1 || !permuted(m->from->index)) continue;
        const long long slots = (long long)m->from->size * m->dim;
        DevInts key(s->size);
        int *dP = (int *)dev_alloc(sizeof(int) * (size_t)s->size);
        if (!key.p || !dP || slots + s->size >= INT_MAX) {
          dev_free(dP);
          return;
        }
        k_fill_int<<<grid_for_n(s->size), 256, 0, st>>>(key.p, s->size, INT_MAX);
        k_reach_key<<<grid_for_n(slots), 256, 0, st>>>(map_dev(m), m->from->size, m->dim,
                                                       g_perm[m->from->index].d_Q, key.p);
        k_reach_finish<<<grid_for_n(s->size), 256, 0, st>>>(key.p, s->size, slots);
        if (!bucket_sort(nullptr, key.p, s->size, slots + s->size, dP)) {
          dev_free(dP);
          return;
        }
        set_perm(s, dP);
        progress = true;
        break;
      }
    }
  }
}

// out[i] = in[P[i]] (forward) or out[P[i]] = in[i] (back), w words per element
__global__ void k_permute(const unsigned *__restrict__ in, unsigned *__restrict__ out,
                          const int *__restrict__ P, long long n, int w, int back) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * w;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / w;
    const int c = (int)(t % w);
    const long long p = P[i];
    if (back) out[p * w + c] = in[i * w + c];
    else out[i * w + c] = in[p * w + c];
  }
}

__global__ void k_permute_bytes(const unsigned char *__restrict__ in, unsigned char *__restrict__ out,
                                const int *__restrict__ P, long long n, int w, int back) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * w;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / w;
    const int c = (int)(t % w);
    const long long p = P[i];
    if (back) out[p * w + c] = in[i * w + c];
    else out[i * w + c] = in[p * w + c];
  }
}

void permute_launch(const void *in, void *out, const int *dP, long long n, int size, int back) {
  cudaStream_t s = rt().stream;
  const int grid = rt().num_sms * 8;
  if (size % 4 == 0)
    k_permute<<<grid, 256, 0, s>>>((const unsigned *)in, (unsigned *)out, dP, n, size / 4, back);
  else
    k_permute_bytes<<<grid, 256, 0, s>>>((const unsigned char *)in, (unsigned char *)out, dP, n,
                                         size, back);
}

}  // namespace

bool renumber_enabled() { return g_enabled; }

bool sort_keys_u64(unsigned long long *a, long long m, cudaStream_t s) {
  return bitonic_sort(a, m, s);
}

// the set's device permutation (new -> old / old -> new), or nullptr
const int *perm_new2old_dev(op_set s) {
  return s && permuted(s->index) && g_applied ? g_perm[s->index].d_P : nullptr;
}
const int *perm_old2new_dev(op_set s) {
  return s && permuted(s->index) && g_applied ? g_perm[s->index].d_Q : nullptr;
}

// store a dataset of a renumbered set in the new order (in place)
void permute_dat_in_place(op_dat d) {
  if (!d || !d->data_d || !perm_new2old_dev(d->set)) return;
  const size_t bytes = (size_t)d->size * d->set->size;
  void *tmp = dev_alloc(bytes);
  if (!tmp) return;
  permute_launch(d->data_d, tmp, perm_new2old_dev(d->set), d->set->size, d->size, 0);
  OP2B_CUDA(cudaMemcpyAsync(d->data_d, tmp, bytes, cudaMemcpyDeviceToDevice, rt().stream));
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  dev_free(tmp);
}

// device data of `d` in the app's order into host memory
bool fetch_unpermuted(op_dat d, void *host) {
  if (!d || !perm_new2old_dev(d->set)) return false;
  const size_t bytes = (size_t)d->size * d->set->size;
  void *tmp = dev_alloc(bytes);
  if (!tmp) return true;
  permute_launch(d->data_d, tmp, perm_new2old_dev(d->set), d->set->size, d->size, 1);
  OP2B_CUDA(cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, rt().stream));
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  dev_free(tmp);
  return true;
}

// rewrite a map's device copy (uploaded in the app's numbering) for the
// renumbered sets: rows in the from-set's new order, values in the to-set's
// new numbering; false when neither set is renumbered
bool renumber_map_device(op_map m, int *d_map) {
  if (!g_applied) return false;
  const bool pf = permuted(m->from->index), pt = permuted(m->to->index);
  if (!pf && !pt) return false;
  const long long n = (long long)m->from->size * m->dim;
  if (n == 0) return true;
  DevInts tmp(n);
  if (!tmp.p) return true;
  cudaStream_t st = rt().stream;
  OP2B_CUDA(cudaMemcpyAsync(tmp.p, d_map, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
  k_renumber_map<<<grid_for_n(n), 256, 0, st>>>(tmp.p, m->from->size, m->dim,
                                                 pf ? g_perm[m->from->index].d_P : nullptr,
                                                 pt ? g_perm[m->to->index].d_Q : nullptr, d_map);
  OP2B_CUDA(cudaStreamSynchronize(st));  // tmp is freed on return
  return true;
}

void release_plans_and_maps();  // device.cu

// called by the first loop call: order the sets, move the data
void renumber_apply() {
  if (!g_enabled || g_applied) return;
  const auto t0 = std::chrono::steady_clock::now();
  compute_orders();  // from the sets and maps declared by now
  g_applied = true;
  release_plans_and_maps();  // device copies of maps and plans follow the new order
  for (int k = 0; k < OP_dat_index; k++) permute_dat_in_place(OP_dat_list[k]);
  known_zero_forget();
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  g_order_seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void renumber_reset() {
  for (auto &sp : g_perm) {
    dev_free(sp.d_P);
    dev_free(sp.d_Q);
  }
  g_perm.clear();
  g_applied = g_computed = false;
  g_enabled = false;
  g_rcb = nullptr;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_set_renumber(int on) {
  if (g_applied && !on) {
    fail(-1, "op2b error -- renumbering cannot be turned off after the first loop\n");
    return -1;
  }
  g_enabled = on != 0;
  return 0;
}

int op2b_set_renumber_coords(op_dat coords) {
  if (g_applied) {
    fail(-1, "op2b error -- the renumbering order cannot change after the first loop\n");
    return -1;
  }
  if (coords && (coords->dim < 1 || coords->dim > 3 || !coords->data_d ||
                 (strcmp(coords->type, "float") != 0 && strcmp(coords->type, "double") != 0))) {
    fail(-1, "op2b error -- coordinates for bisection must be 1 to 3 float or double "
             "components\n");
    return -1;
  }
  g_rcb = coords;
  g_computed = false;
  if (coords) g_enabled = true;
  return 0;
}

int op2b_renumber_order(op_set set, int *new2old) {
  if (!set || !new2old) return -1;
  if (!g_applied) compute_orders();
  if (permuted(set->index) && (int)g_perm[set->index].P.size() == set->size) {
    std::copy(g_perm[set->index].P.begin(), g_perm[set->index].P.end(), new2old);
    return 1;
  }
  for (int i = 0; i < set->size; i++) new2old[i] = i;
  return 0;
}

}  // extern "C"

extern "C" double op2b_renumber_seconds(void) { return op2b::g_order_seconds; }
