// plan.cu -- execution plans built on the device.
//
// 1. The reference's op_plan (common/op_lib_core.c:627-1089), reproduced
//    array for array: contiguous blocks, per-block sorted distinct indirect
//    targets (ind_maps) with short block-local indices (loc_maps), greedy
//    thread colouring in element order and greedy block colouring in block
//    order, both in passes of 32 colours, and blkmap grouped by colour.  The
//    O(N log N) part (gather, sort, dedupe, inverse) runs one CTA per block
//    and indirect dataset; the thread colouring runs one CTA per block; the
//    block colouring is the reference's sequential greedy over blocks, run by
//    one CTA that ORs each block's target masks in parallel.  All of it is
//    integer work with one exact answer, so the result equals op_plan_core.
// 2. A validator for any plan: the reference's op_plan_check
//    (op_lib_core.c:469-620) plus the colouring checks it leaves out.
// 3. The owner-computes ("gather") plan used by the GATHER strategy: per
//    incremented element, its contributions in ascending (element, slot)
//    order, i.e. the order in which op_seq.h applies them.

#include <limits.h>

#include <algorithm>
#include <cstring>

#include "plan.h"

namespace op2b {

constexpr int kMaxArgs = 24;

struct ArgMaps {
  const int *map[kMaxArgs];
  int dim[kMaxArgs];
  int idx[kMaxArgs];
};

struct PlanParams {
  ArgMaps am;
  int nargs, ninds, set_size, bsize, nblocks, cls;
  int ind_first[kMaxArgs];  // first position in ind_args of ind m
  int ind_k[kMaxArgs];      // number of args of ind m
  int ind_args[kMaxArgs];   // args grouped by ind, in argument order
  int ind_P[kMaxArgs];      // sort size (power of two >= k*bsize)
  int ind_size[kMaxArgs];   // dat bytes per element for ind m
  int ind_dim[kMaxArgs];    // dat dim for ind m
  int arg_ind[kMaxArgs];    // ind of arg a, or -1
  long long tmp_off[kMaxArgs];
  // OP_INC slots (thread / block colouring): arg and its ind
  int ninc;
  int inc_arg[kMaxArgs];
  int inc_ind[kMaxArgs];
  int inc_mbase[kMaxArgs];  // per INC slot: offset of its ind's masks in smem
  int mask_words;           // total mask words per block in smem
};

__device__ __forceinline__ int map_at(const ArgMaps &am, int a, int e) {
  return am.map[a][am.idx[a] + (size_t)e * am.dim[a]];
}

// block-wide exclusive scan of one int per thread (blockDim.x <= 1024)
__device__ int block_excl_scan(int v, int *total) {
  __shared__ int warp_sums[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  if (warp == 0) {
    int w = lane < nw ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_sums[lane] = w;  // inclusive
  }
  __syncthreads();
  int excl = x - v + (warp > 0 ? warp_sums[warp - 1] : 0);
  if (total) *total = warp_sums[nw - 1];
  __syncthreads();
  return excl;
}

__device__ void bitonic_sort(int *s, int P) {
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          int a = s[i], b = s[ixj];
          bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
}

// one CTA per (block b, indirect dataset m): gather the targets of all args
// of m over the block's elements, sort, deduplicate
// (common/op_lib_core.c:781-803)
__global__ void k_block_unique(PlanParams pp, int *ind_sizes, int *tmp) {
  extern __shared__ int s[];
  const int b = blockIdx.x, m = blockIdx.y;
  const int e0 = b * pp.bsize;
  const int bs = min(pp.bsize, pp.set_size - e0);
  const int k = pp.ind_k[m];
  const int K = k * bs;
  int P = 1;
  while (P < K) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    int v = INT_MAX;
    if (i < K) {
      int a = pp.ind_args[pp.ind_first[m] + i / bs];
      v = map_at(pp.am, a, e0 + i % bs);
    }
    s[i] = v;
  }
  __syncthreads();
  bitonic_sort(s, P);
  int *out = tmp + pp.tmp_off[m] + (long long)b * k * pp.bsize;
  int base = 0;
  for (int r = 0; r < K; r += blockDim.x) {
    int i = r + threadIdx.x;
    int f = (i < K) && (i == 0 || s[i] != s[i - 1]);
    int tot;
    int pos = block_excl_scan(f, &tot);
    if (f) out[base + pos] = s[i];
    base += tot;
  }
  if (threadIdx.x == 0) ind_sizes[m + b * pp.ninds] = base;
}

// exclusive scan of ind_sizes over blocks, per indirect dataset
// (common/op_lib_core.c:822-834)
__global__ void k_scan_blocks(int nblocks, int ninds, const int *ind_sizes, int *ind_offs,
                              int *nindirect) {
  const int m = blockIdx.x;
  int run = 0;
  for (int c = 0; c < nblocks; c += blockDim.x) {
    int b = c + threadIdx.x;
    int v = b < nblocks ? ind_sizes[m + b * ninds] : 0;
    int tot;
    int x = block_excl_scan(v, &tot);
    if (b < nblocks) ind_offs[m + b * ninds] = run + x;
    run += tot;
  }
  if (threadIdx.x == 0) nindirect[m] = run;
}

struct IndOut {
  int *ind_maps[kMaxArgs];
  short *loc_maps[kMaxArgs];
};

// place the block's distinct targets in ind_maps, renumber each arg's targets
// to block-local indices (common/op_lib_core.c:807-820), and count the cache
// lines the reference's byte model charges (common/op_lib_core.c:1010-1040)
__global__ void k_block_locmaps(PlanParams pp, IndOut io, const int *ind_sizes,
                                const int *ind_offs, const int *tmp, long long *lines,
                                long long *lines3) {
  extern __shared__ int list[];
  const int b = blockIdx.x, m = blockIdx.y;
  const int e0 = b * pp.bsize;
  const int bs = min(pp.bsize, pp.set_size - e0);
  const int k = pp.ind_k[m];
  const int nu = ind_sizes[m + b * pp.ninds];
  const int off = ind_offs[m + b * pp.ninds];
  const int *src = tmp + pp.tmp_off[m] + (long long)b * k * pp.bsize;
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    int t = src[u];
    list[u] = t;
    io.ind_maps[m][off + u] = t;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < k * bs; i += blockDim.x) {
    int a = pp.ind_args[pp.ind_first[m] + i / bs];
    int e = e0 + i % bs;
    int v = map_at(pp.am, a, e);
    int lo = 0, hi = nu;  // lower_bound
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (list[mid] < v) lo = mid + 1; else hi = mid;
    }
    io.loc_maps[a][e] = (short)lo;
  }
  // cache lines: element u starts a new line unless its first line is the
  // previous element's last line
  const long long sz = pp.ind_size[m], cls = pp.cls, cls3 = (long long)pp.ind_dim[m] * pp.cls;
  long long my = 0, my3 = 0;
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    long long t = list[u];
    long long a = (t * sz) / cls, z = ((t + 1) * sz - 1) / cls;
    long long prev = u > 0 ? (((long long)list[u - 1] + 1) * sz - 1) / cls : -1;
    my += (a > prev ? 1 : 0) + (z - a);
    long long a3 = (t * sz) / cls3, z3 = ((t + 1) * sz - 1) / cls3;
    long long prev3 = u > 0 ? (((long long)list[u - 1] + 1) * sz - 1) / cls3 : -1;
    my3 += (a3 > prev3 ? 1 : 0) + (z3 - a3);
  }
  for (int o = 16; o > 0; o >>= 1) {
    my += __shfl_down_sync(0xffffffffu, my, o);
    my3 += __shfl_down_sync(0xffffffffu, my3, o);
  }
  __shared__ long long red[2][32];
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = my;
    red[1][threadIdx.x >> 5] = my3;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0, s3 = 0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) {
      s += red[0][w];
      s3 += red[1][w];
    }
    lines[m + b * pp.ninds] = s;
    lines3[m + b * pp.ninds] = s3;
  }
}

// greedy thread colouring of one block in element order, 32 colours per
// pass (common/op_lib_core.c:839-880).  The loop is sequential by definition;
// one thread runs it on block-local masks in shared memory.
__global__ void k_thread_colour(PlanParams pp, IndOut io, const int *ind_sizes, int *thrcol,
                                int *nthrcol) {
  extern __shared__ unsigned smem[];
  const int b = blockIdx.x;
  const int e0 = b * pp.bsize;
  const int bs = min(pp.bsize, pp.set_size - e0);
  unsigned *masks = smem;
  unsigned short *locs = (unsigned short *)(smem + pp.mask_words);
  int *col = (int *)(smem + pp.mask_words + (pp.ninc * pp.bsize + 1) / 2);
  for (int i = threadIdx.x; i < pp.ninc * bs; i += blockDim.x) {
    int sl = i / bs, e = i % bs;
    locs[sl * bs + e] = (unsigned short)io.loc_maps[pp.inc_arg[sl]][e0 + e];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int e = 0; e < bs; e++) col[e] = -1;
    int base = 0, ncol = 0, again = 1;
    while (again) {
      again = 0;
      for (int sl = 0; sl < pp.ninc; sl++) {
        int nu = ind_sizes[pp.inc_ind[sl] + b * pp.ninds];
        for (int u = 0; u < nu; u++) masks[pp.inc_mbase[sl] + u] = 0u;
      }
      for (int e = 0; e < bs; e++) {
        if (col[e] != -1) continue;
        unsigned mask = 0;
        for (int sl = 0; sl < pp.ninc; sl++) mask |= masks[pp.inc_mbase[sl] + locs[sl * bs + e]];
        int c = __ffs(~mask) - 1;
        if (c < 0) {
          again = 1;
          continue;
        }
        col[e] = base + c;
        ncol = max(ncol, base + c + 1);
        for (int sl = 0; sl < pp.ninc; sl++) masks[pp.inc_mbase[sl] + locs[sl * bs + e]] |= 1u << c;
      }
      base += 32;
    }
    nthrcol[b] = ncol;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < bs; e += blockDim.x) thrcol[e0 + e] = col[e];
}

struct IncWork {
  unsigned *work[kMaxArgs];  // per INC slot: mask array of its ind (aliases allowed)
  int wsize[kMaxArgs];
};

// greedy block colouring in block order, 32 colours per pass, then blocks
// grouped by colour (common/op_lib_core.c:892-965).  One CTA: blocks are
// visited in order as the reference does; each block's target masks are
// ORed and set by all threads in parallel.
__global__ void k_block_colour(PlanParams pp, IncWork iw, int nwork, unsigned *const *work_arrays,
                               const int *work_sizes, int *blk_col, int *blkmap, int *ncolblk,
                               int *ncolors_out) {
  __shared__ unsigned s_mask[32];
  __shared__ int s_again, s_col;
  const int tid = threadIdx.x;
  for (int b = tid; b < pp.nblocks; b += blockDim.x) blk_col[b] = -1;
  int base = 0, ncolors = 0;
  if (tid == 0) s_again = 1;
  __syncthreads();
  while (s_again) {
    __syncthreads();
    if (tid == 0) s_again = 0;
    for (int w = 0; w < nwork; w++)
      for (int t = tid; t < work_sizes[w]; t += blockDim.x) work_arrays[w][t] = 0u;
    __syncthreads();
    for (int b = 0; b < pp.nblocks; b++) {
      if (blk_col[b] != -1) continue;
      const int e0 = b * pp.bsize;
      const int bs = min(pp.bsize, pp.set_size - e0);
      unsigned mask = 0;
      for (int i = tid; i < pp.ninc * bs; i += blockDim.x) {
        int sl = i / bs;
        int t = map_at(pp.am, pp.inc_arg[sl], e0 + i % bs);
        mask |= iw.work[sl][t];
      }
      mask = __reduce_or_sync(0xffffffffu, mask);
      if ((tid & 31) == 0) s_mask[tid >> 5] = mask;
      __syncthreads();
      if (tid == 0) {
        unsigned mm = 0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) mm |= s_mask[w];
        int c = __ffs(~mm) - 1;
        s_col = c;
        if (c < 0) s_again = 1;
        else blk_col[b] = base + c;
      }
      __syncthreads();
      int c = s_col;
      if (c >= 0) {
        ncolors = max(ncolors, base + c + 1);
        for (int i = tid; i < pp.ninc * bs; i += blockDim.x) {
          int sl = i / bs;
          int t = map_at(pp.am, pp.inc_arg[sl], e0 + i % bs);
          atomicOr(&iw.work[sl][t], 1u << c);
        }
      }
      __syncthreads();
    }
    base += 32;
    __syncthreads();
  }
  // blocks of each colour in block order (counting sort, stable)
  int start = 0;
  for (int c = 0; c < ncolors; c++) {
    for (int r = 0; r < pp.nblocks; r += blockDim.x) {
      int b = r + tid;
      int f = (b < pp.nblocks) && blk_col[b] == c;
      int tot;
      int pos = block_excl_scan(f, &tot);
      if (f) blkmap[start + pos] = b;
      start += tot;
      if (tid == 0) ncolblk[c] += tot;
    }
  }
  if (tid == 0) *ncolors_out = ncolors;
}

// ----------------------------------------------------------- validation --

__global__ void k_check_locmaps(PlanParams pp, IndOut io, const int *ind_sizes,
                                const int *ind_offs, unsigned long long *err) {
  long long n = (long long)pp.nargs * pp.set_size;
  unsigned long long bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int a = (int)(i / pp.set_size), e = (int)(i % pp.set_size);
    int m = pp.arg_ind[a];
    if (io.loc_maps[a] == nullptr || m < 0) continue;
    int b = e / pp.bsize;
    int loc = io.loc_maps[a][e];
    if (loc < 0 || loc >= ind_sizes[m + b * pp.ninds]) {
      bad++;
      continue;
    }
    int g = io.ind_maps[m][ind_offs[m + b * pp.ninds] + loc];
    bad += (g != map_at(pp.am, a, e));
  }
  if (bad) atomicAdd(err, bad);
}

__global__ void k_check_indmaps(PlanParams pp, IndOut io, const int *ind_sizes,
                                const int *ind_offs, const int *to_sizes,
                                unsigned long long *err) {
  const int b = blockIdx.x, m = blockIdx.y;
  const int nu = ind_sizes[m + b * pp.ninds], off = ind_offs[m + b * pp.ninds];
  unsigned long long bad = 0;
  if (threadIdx.x == 0 && b > 0)
    bad += (off != ind_offs[m + (b - 1) * pp.ninds] + ind_sizes[m + (b - 1) * pp.ninds]);
  if (threadIdx.x == 0 && b == 0) bad += (off != 0);
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    int t = io.ind_maps[m][off + u];
    if (u > 0) bad += (t <= io.ind_maps[m][off + u - 1]);
    bad += (t < 0 || t >= to_sizes[m]);
  }
  if (bad) atomicAdd(err, bad);
}

// no two elements of one block with the same thread colour touch one
// OP_INC target
__global__ void k_check_thread_colours(PlanParams pp, IndOut io, const int *ind_sizes,
                                       const int *thrcol, const int *nthrcol,
                                       unsigned long long *err) {
  extern __shared__ int own[];
  const int b = blockIdx.x;
  const int e0 = b * pp.bsize;
  const int bs = min(pp.bsize, pp.set_size - e0);
  const int nc = nthrcol[b];
  unsigned long long bad = 0;
  for (int e = threadIdx.x; e < bs; e += blockDim.x) {
    int c = thrcol[e0 + e];
    bad += (c < 0 || c >= nc);
  }
  for (int c = 0; c < nc; c++) {
    for (int w = threadIdx.x; w < pp.mask_words; w += blockDim.x) own[w] = -1;
    __syncthreads();
    for (int e = threadIdx.x; e < bs; e += blockDim.x) {
      if (thrcol[e0 + e] != c) continue;
      for (int sl = 0; sl < pp.ninc; sl++) {
        int loc = io.loc_maps[pp.inc_arg[sl]][e0 + e];
        int old = atomicCAS(&own[pp.inc_mbase[sl] + loc], -1, e);
        bad += (old != -1 && old != e);
      }
    }
    __syncthreads();
  }
  if (bad) atomicAdd(err, bad);
}

// no two blocks of the same block colour touch one OP_INC target
__global__ void k_check_block_colours(PlanParams pp, IncWork iw, const int *blkmap, int first,
                                      int nblk, unsigned long long *err) {
  unsigned long long bad = 0;
  for (int k = blockIdx.x; k < nblk; k += gridDim.x) {
    int b = blkmap[first + k];
    int e0 = b * pp.bsize, bs = min(pp.bsize, pp.set_size - e0);
    for (int i = threadIdx.x; i < pp.ninc * bs; i += blockDim.x) {
      int sl = i / bs;
      int t = map_at(pp.am, pp.inc_arg[sl], e0 + i % bs);
      int old = atomicCAS((int *)&iw.work[sl][t], -1, b);
      bad += (old != -1 && old != b);
    }
  }
  if (bad) atomicAdd(err, bad);
}

__global__ void k_check_blocks(PlanParams pp, const int *blkmap, const int *offset,
                               const int *nelems, int *seen, unsigned long long *err) {
  unsigned long long bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < pp.nblocks;
       i += gridDim.x * blockDim.x) {
    int b = blkmap[i];
    if (b < 0 || b >= pp.nblocks) bad++;
    else if (atomicAdd(&seen[b], 1) != 0) bad++;
    bad += (offset[i] != i * pp.bsize);
    bad += (nelems[i] != min(pp.bsize, pp.set_size - i * pp.bsize));
  }
  if (bad) atomicAdd(err, bad);
}

// ------------------------------------------------------------------ scan --

__global__ void k_scan_chunks(const int *in, int *out, int n, int *sums, int chunk) {
  int c0 = blockIdx.x * chunk;
  int run = 0;
  for (int r = 0; r < chunk; r += blockDim.x) {
    int i = c0 + r + threadIdx.x;
    int v = (i < n && r + threadIdx.x < chunk) ? in[i] : 0;
    int tot;
    int x = block_excl_scan(v, &tot);
    if (i < n && r + threadIdx.x < chunk) out[i] = run + x;
    run += tot;
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = run;
}

__global__ void k_scan_add(int *out, int n, const int *offs, int chunk) {
  int add = offs[blockIdx.x];
  int c0 = blockIdx.x * chunk;
  for (int r = threadIdx.x; r < chunk; r += blockDim.x) {
    int i = c0 + r;
    if (i < n) out[i] += add;
  }
}

void exclusive_scan_nosync(const int *d_in, int *d_out, int n, cudaStream_t s) {
  const int chunk = 8192;
  const int nch = (n + chunk - 1) / chunk;
  if (n <= 0) return;
  int *sums = nullptr;
  OP2B_CUDA(pool_malloc_async((void **)&sums, sizeof(int) * (nch + 1), s));
  k_scan_chunks<<<nch, 1024, 0, s>>>(d_in, d_out, n, sums, chunk);
  if (nch > 1) {
    exclusive_scan_nosync(sums, sums, nch, s);
    k_scan_add<<<nch, 1024, 0, s>>>(d_out, n, sums, chunk);
  }
  OP2B_CUDA(cudaFreeAsync(sums, s));
}

long long exclusive_scan(const int *d_in, int *d_out, int n, cudaStream_t s) {
  const int chunk = 8192;
  int nch = (n + chunk - 1) / chunk;
  if (n <= 0) return 0;
  int *sums = nullptr;
  OP2B_CUDA(pool_malloc_async((void **)&sums, sizeof(int) * (nch + 1), s));
  k_scan_chunks<<<nch, 1024, 0, s>>>(d_in, d_out, n, sums, chunk);
  if (nch > 1) {
    exclusive_scan(sums, sums, nch, s);
    k_scan_add<<<nch, 1024, 0, s>>>(d_out, n, sums, chunk);
  }
  // total = last exclusive value + last input
  int last_out = 0, last_in = 0;
  OP2B_CUDA(cudaMemcpyAsync(&last_out, d_out + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaMemcpyAsync(&last_in, d_in + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaFreeAsync(sums, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  return (long long)last_out + last_in;
}

// ------------------------------------------------------------- builders --

static std::vector<std::unique_ptr<DevPlan>> g_plans;
static std::vector<std::unique_ptr<GatherPlan>> g_gather;

static bool fill_params(PlanParams &pp, const DevPlan &p, std::vector<int> &to_sizes) {
  memset(&pp, 0, sizeof pp);
  if (p.nargs > kMaxArgs || p.ninds > kMaxArgs) return false;
  pp.nargs = p.nargs;
  pp.ninds = p.ninds;
  pp.set_size = p.set->size;
  pp.bsize = p.bsize;
  pp.nblocks = p.nblocks;
  pp.cls = OP_cache_line_size > 0 ? OP_cache_line_size : 128;
  for (int a = 0; a < p.nargs; a++) {
    pp.arg_ind[a] = p.inds[a];
    if (p.maps[a]) {
      pp.am.map[a] = map_dev(p.maps[a]);
      pp.am.dim[a] = p.maps[a]->dim;
      pp.am.idx[a] = p.idxs[a];
    }
  }
  int pos = 0;
  to_sizes.assign(p.ninds, 0);
  for (int m = 0; m < p.ninds; m++) {
    pp.ind_first[m] = pos;
    for (int a = 0; a < p.nargs; a++)
      if (p.inds[a] == m) {
        if (!p.maps[a]) return false;
        pp.ind_args[pos++] = a;
        if (pp.ind_k[m] == 0) {
          pp.ind_size[m] = p.dats[a]->size;
          pp.ind_dim[m] = p.dats[a]->dim;
          to_sizes[m] = p.maps[a]->to->size;
        }
        pp.ind_k[m]++;
      }
    if (pp.ind_k[m] == 0) return false;
  }
  long long off = 0;
  for (int m = 0; m < p.ninds; m++) {
    pp.tmp_off[m] = off;
    off += (long long)pp.ind_k[m] * p.bsize * p.nblocks;
    int P = 1;
    while (P < pp.ind_k[m] * p.bsize) P <<= 1;
    pp.ind_P[m] = P;
  }
  // INC slots and their mask areas (one area per distinct ind)
  int mbase_of_ind[kMaxArgs];
  for (int m = 0; m < kMaxArgs; m++) mbase_of_ind[m] = -1;
  int words = 0;
  for (int a = 0; a < p.nargs; a++)
    if (p.inds[a] >= 0 && p.accs[a] == OP_INC) {
      int m = p.inds[a];
      if (mbase_of_ind[m] < 0) {
        mbase_of_ind[m] = words;
        words += pp.ind_k[m] * p.bsize;
      }
      pp.inc_arg[pp.ninc] = a;
      pp.inc_ind[pp.ninc] = m;
      pp.inc_mbase[pp.ninc] = mbase_of_ind[m];
      pp.ninc++;
    }
  pp.mask_words = words;
  return true;
}

static size_t smem_optin() {
  static int v = -1;
  if (v < 0) {
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, rt().device);
    if (v <= 0) v = 48 * 1024;
  }
  return (size_t)v;
}

// allow a kernel the largest dynamic shared memory the device offers, less
// what the kernel declares statically
template <class K>
static size_t allow_smem(K kernel) {
  cudaFuncAttributes fa;
  OP2B_CUDA(cudaFuncGetAttributes(&fa, kernel));
  size_t dyn = smem_optin() - fa.sharedSizeBytes;
  OP2B_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  return dyn;
}

static void build_plan(DevPlan &p) {
  Runtime &R = rt();
  cudaStream_t s = R.stream;
  const int n = p.set->size;
  // block size from the reference's 48 KB shared-memory budget
  // (common/op_lib_core.c:663-673)
  int maxbytes = 0;
  for (int a = 0; a < p.nargs; a++)
    if (p.inds[a] >= 0) maxbytes += p.dats[a]->size;
  p.bsize = p.part_size;
  if (p.bsize == 0) p.bsize = maxbytes > 0 ? (48 * 1024 / (64 * maxbytes)) * 64 : 512;
  if (p.bsize <= 0) {
    fail(-1, "op_plan error -- invalid block size for kernel %s\n", p.name.c_str());
    return;
  }
  p.nblocks = (n - 1) / p.bsize + 1;

  PlanParams pp;
  std::vector<int> to_sizes;
  if (!fill_params(pp, p, to_sizes)) {
    fail(-1, "op_plan error -- unsupported argument layout for kernel %s\n", p.name.c_str());
    return;
  }
  const size_t optin = smem_optin() - 1024;  // headroom for static shared memory
  for (int m = 0; m < p.ninds; m++)
    if ((size_t)pp.ind_P[m] * sizeof(int) > optin || pp.ind_k[m] * p.bsize > 32767) {
      fail(-1,
           "op_plan error -- block size %d too large for kernel %s (block-local indices "
           "are 16-bit and each block's targets are sorted in shared memory)\n",
           p.bsize, p.name.c_str());
      return;
    }

  const int nb = p.nblocks, ni = p.ninds;
  p.d_nthrcol = (int *)dev_alloc(sizeof(int) * nb);
  p.d_thrcol = (int *)dev_alloc(sizeof(int) * (size_t)n);
  p.d_offset = (int *)dev_alloc(sizeof(int) * nb);
  p.d_nelems = (int *)dev_alloc(sizeof(int) * nb);
  p.d_ind_offs = (int *)dev_alloc(sizeof(int) * (size_t)nb * (ni ? ni : 1));
  p.d_ind_sizes = (int *)dev_alloc(sizeof(int) * (size_t)nb * (ni ? ni : 1));
  p.d_blkmap = (int *)dev_alloc(sizeof(int) * nb);
  p.d_ind_maps.assign(ni, nullptr);
  p.d_loc_maps.assign(p.nargs, nullptr);
  for (int a = 0; a < p.nargs; a++)
    if (p.inds[a] >= 0) p.d_loc_maps[a] = (short *)dev_alloc(sizeof(short) * (size_t)n);

  // offsets and sizes of the contiguous blocks (common/op_lib_core.c:768-773)
  std::vector<int> off(nb), nel(nb);
  for (int b = 0; b < nb; b++) {
    off[b] = b * p.bsize;
    nel[b] = std::min(p.bsize, n - b * p.bsize);
  }
  OP2B_CUDA(cudaMemcpyAsync(p.d_offset, off.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
  OP2B_CUDA(cudaMemcpyAsync(p.d_nelems, nel.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));

  long long tmp_total = 0;
  for (int m = 0; m < ni; m++) tmp_total += (long long)pp.ind_k[m] * p.bsize * nb;
  int *tmp = nullptr, *d_nind = nullptr;
  long long *d_lines = nullptr, *d_lines3 = nullptr;
  OP2B_CUDA(pool_malloc_async((void **)&tmp, sizeof(int) * (tmp_total ? tmp_total : 1), s));
  OP2B_CUDA(pool_malloc_async((void **)&d_nind, sizeof(int) * (ni ? ni : 1), s));
  OP2B_CUDA(pool_malloc_async((void **)&d_lines, sizeof(long long) * nb * (ni ? ni : 1), s));
  OP2B_CUDA(pool_malloc_async((void **)&d_lines3, sizeof(long long) * nb * (ni ? ni : 1), s));

  IndOut io;
  memset(&io, 0, sizeof io);
  for (int a = 0; a < p.nargs; a++) io.loc_maps[a] = p.d_loc_maps[a];

  p.nindirect.assign(ni, 0);
  if (ni > 0) {
    int maxP = 0;
    for (int m = 0; m < ni; m++) maxP = std::max(maxP, pp.ind_P[m]);
    size_t sm = sizeof(int) * (size_t)maxP;
    allow_smem(k_block_unique);
    k_block_unique<<<dim3(nb, ni), 1024, sm, s>>>(pp, p.d_ind_sizes, tmp);
    k_scan_blocks<<<ni, 1024, 0, s>>>(nb, ni, p.d_ind_sizes, p.d_ind_offs, d_nind);
    OP2B_CUDA(cudaMemcpyAsync(p.nindirect.data(), d_nind, sizeof(int) * ni,
                              cudaMemcpyDeviceToHost, s));
    OP2B_CUDA(cudaStreamSynchronize(s));
    for (int m = 0; m < ni; m++) {
      p.d_ind_maps[m] = (int *)dev_alloc(sizeof(int) * (size_t)std::max(1, p.nindirect[m]));
      io.ind_maps[m] = p.d_ind_maps[m];
    }
    int maxk = 0;
    for (int m = 0; m < ni; m++) maxk = std::max(maxk, pp.ind_k[m]);
    size_t sm2 = sizeof(int) * (size_t)maxk * p.bsize;
    allow_smem(k_block_locmaps);
    k_block_locmaps<<<dim3(nb, ni), 512, sm2, s>>>(pp, io, p.d_ind_sizes, p.d_ind_offs, tmp,
                                                   d_lines, d_lines3);
  }

  // thread colouring
  size_t sm3 = sizeof(unsigned) * pp.mask_words + sizeof(unsigned short) * (pp.ninc * p.bsize + 2) +
               sizeof(int) * p.bsize;
  if (sm3 > optin) {
    fail(-1, "op_plan error -- block size %d too large to colour kernel %s\n", p.bsize,
         p.name.c_str());
    return;
  }
  allow_smem(k_thread_colour);
  k_thread_colour<<<nb, 128, sm3, s>>>(pp, io, p.d_ind_sizes, p.d_thrcol, p.d_nthrcol);

  // block colouring: one mask array per distinct INC ind
  IncWork iw;
  memset(&iw, 0, sizeof iw);
  std::vector<unsigned *> warr;
  std::vector<int> wsz;
  std::vector<int> ind_w(kMaxArgs, -1);
  for (int sl = 0; sl < pp.ninc; sl++) {
    int m = pp.inc_ind[sl];
    if (ind_w[m] < 0) {
      unsigned *w = nullptr;
      OP2B_CUDA(pool_malloc_async((void **)&w, sizeof(unsigned) * (size_t)to_sizes[m], s));
      ind_w[m] = (int)warr.size();
      warr.push_back(w);
      wsz.push_back(to_sizes[m]);
    }
    iw.work[sl] = warr[ind_w[m]];
    iw.wsize[sl] = to_sizes[m];
  }
  unsigned **d_warr = nullptr;
  int *d_wsz = nullptr, *d_blkcol = nullptr, *d_ncolblk = nullptr, *d_ncolors = nullptr;
  int nw = (int)warr.size();
  OP2B_CUDA(pool_malloc_async((void **)&d_warr, sizeof(unsigned *) * (nw ? nw : 1), s));
  OP2B_CUDA(pool_malloc_async((void **)&d_wsz, sizeof(int) * (nw ? nw : 1), s));
  OP2B_CUDA(pool_malloc_async((void **)&d_blkcol, sizeof(int) * nb, s));
  OP2B_CUDA(pool_malloc_async((void **)&d_ncolblk, sizeof(int) * nb, s));
  OP2B_CUDA(pool_malloc_async((void **)&d_ncolors, sizeof(int), s));
  if (nw) {
    OP2B_CUDA(cudaMemcpyAsync(d_warr, warr.data(), sizeof(unsigned *) * nw, cudaMemcpyHostToDevice, s));
    OP2B_CUDA(cudaMemcpyAsync(d_wsz, wsz.data(), sizeof(int) * nw, cudaMemcpyHostToDevice, s));
  }
  OP2B_CUDA(cudaMemsetAsync(d_ncolblk, 0, sizeof(int) * nb, s));
  k_block_colour<<<1, 1024, 0, s>>>(pp, iw, nw, d_warr, d_wsz, d_blkcol, p.d_blkmap, d_ncolblk,
                                    d_ncolors);

  // back to the host: the small per-block tables for nshared and the byte
  // models, the colour counts for the launch loop
  std::vector<int> ind_sizes((size_t)nb * ni);
  std::vector<long long> lines((size_t)nb * ni), lines3((size_t)nb * ni);
  int ncolors = 0;
  p.nthrcol_h.assign(nb, 0);
  if (ni) {
    OP2B_CUDA(cudaMemcpyAsync(ind_sizes.data(), p.d_ind_sizes, sizeof(int) * nb * ni,
                              cudaMemcpyDeviceToHost, s));
    OP2B_CUDA(cudaMemcpyAsync(lines.data(), d_lines, sizeof(long long) * nb * ni,
                              cudaMemcpyDeviceToHost, s));
    OP2B_CUDA(cudaMemcpyAsync(lines3.data(), d_lines3, sizeof(long long) * nb * ni,
                              cudaMemcpyDeviceToHost, s));
  }
  OP2B_CUDA(cudaMemcpyAsync(p.nthrcol_h.data(), p.d_nthrcol, sizeof(int) * nb,
                            cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaMemcpyAsync(&ncolors, d_ncolors, sizeof(int), cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  p.ncolors = ncolors;
  p.ncolblk.assign(std::max(1, ncolors), 0);
  OP2B_CUDA(cudaMemcpy(p.ncolblk.data(), d_ncolblk, sizeof(int) * std::max(1, ncolors),
                       cudaMemcpyDeviceToHost));
  p.colstart.assign(ncolors + 1, 0);
  for (int c = 0; c < ncolors; c++) p.colstart[c + 1] = p.colstart[c] + p.ncolblk[c];

  for (void *w : warr) OP2B_CUDA(cudaFreeAsync(w, s));
  OP2B_CUDA(cudaFreeAsync(d_warr, s));
  OP2B_CUDA(cudaFreeAsync(d_wsz, s));
  OP2B_CUDA(cudaFreeAsync(d_blkcol, s));
  OP2B_CUDA(cudaFreeAsync(d_ncolblk, s));
  OP2B_CUDA(cudaFreeAsync(d_ncolors, s));
  OP2B_CUDA(cudaFreeAsync(tmp, s));
  OP2B_CUDA(cudaFreeAsync(d_nind, s));
  OP2B_CUDA(cudaFreeAsync(d_lines, s));
  OP2B_CUDA(cudaFreeAsync(d_lines3, s));

  // shared memory requirement (common/op_lib_core.c:972-985)
  p.nshared = 0;
  double total_shared = 0;
  for (int b = 0; b < nb; b++) {
    int nbytes = 0;
    for (int m = 0; m < ni; m++) nbytes += ROUND_UP(ind_sizes[m + (size_t)b * ni] * pp.ind_size[m]);
    p.nshared = std::max(p.nshared, nbytes);
    total_shared += nbytes;
  }
  // byte models (common/op_lib_core.c:989-1056), exact integer sums
  double t1 = 0, t2 = 0, t3 = 0;
  const double cls = pp.cls;
  for (int b = 0; b < nb; b++) {
    for (int a = 0; a < p.nargs; a++) {
      if (p.inds[a] < 0) {
        double fac = p.accs[a] == OP_READ ? 1.0 : 2.0;
        if (p.dats[a]) {
          double v = fac * nel[b] * p.dats[a]->size;
          t1 += v; t2 += v; t3 += v;
        }
      } else {
        double v = (double)nel[b] * sizeof(short);
        t1 += v; t2 += v; t3 += v;
      }
    }
    for (int m = 0; m < ni; m++) {
      int a = pp.ind_args[pp.ind_first[m]];
      double fac = p.accs[a] == OP_READ ? 1.0 : 2.0;
      double isz = ind_sizes[m + (size_t)b * ni];
      t1 += fac * isz * pp.ind_size[m];
      t2 += fac * (double)lines[m + (size_t)b * ni] * cls;
      t3 += fac * (double)lines3[m + (size_t)b * ni] * pp.ind_dim[m] * cls;
      double fac2 = p.accs[a] == OP_RW ? 2.0 : 1.0;
      t1 += fac2 * isz * sizeof(int);
      t2 += fac2 * isz * sizeof(int);
      t3 += fac2 * isz * sizeof(int);
    }
  }
  p.transfer = t1;
  p.transfer2 = t2;
  p.transfer3 = t3;
  long long tc = 0;
  for (int b = 0; b < nb; b++) {
    tc += p.nthrcol_h[b];
    p.max_thread_colours = std::max(p.max_thread_colours, p.nthrcol_h[b]);
  }
  p.avg_thread_colours = (float)tc / nb;

  if (OP_diags > 1) {
    printf(" number of blocks       = %d \n", nb);
    printf(" number of block colors = %d \n", p.ncolors);
    printf(" maximum block size     = %d \n", p.bsize);
    printf(" average thread colors  = %.2f \n", p.avg_thread_colours);
    printf(" shared memory required = %.2f KB \n", p.nshared / 1024.0f);
    printf(" average data reuse     = %.2f \n", maxbytes * (n / total_shared));
    printf(" data transfer (used)   = %.2f MB \n", p.transfer / (1024.0f * 1024.0f));
    printf(" data transfer (total)  = %.2f MB \n", p.transfer2 / (1024.0f * 1024.0f));
    printf(" SoA/AoS transfer ratio = %.2f \n\n", p.transfer3 / p.transfer2);
  }
}

static void fill_pub(DevPlan &p) {
  op_plan &o = p.pub;
  memset(&o, 0, sizeof o);
  o.name = p.name.c_str();
  o.set = p.set;
  o.nargs = p.nargs;
  o.ninds = p.ninds;
  o.part_size = p.part_size;
  o.maps = p.maps.data();
  o.dats = p.dats.data();
  o.idxs = p.idxs.data();
  o.accs = p.accs.data();
  o.nthrcol = p.d_nthrcol;
  o.thrcol = p.d_thrcol;
  o.offset = p.d_offset;
  p.pub_ind_maps = p.d_ind_maps;
  p.pub_loc_maps = p.d_loc_maps;
  o.ind_maps = p.pub_ind_maps.data();
  o.ind_offs = p.d_ind_offs;
  o.ind_sizes = p.d_ind_sizes;
  o.nindirect = p.nindirect.data();
  o.loc_maps = p.pub_loc_maps.data();
  o.nblocks = p.nblocks;
  o.nelems = p.d_nelems;
  o.ncolors = p.ncolors;
  o.ncolblk = p.ncolblk.data();
  o.blkmap = p.d_blkmap;
  o.nshared = p.nshared;
  o.transfer = (float)p.transfer;
  o.transfer2 = (float)p.transfer2;
  o.count = p.count;
}

DevPlan *get_plan(char const *name, op_set set, int part_size, int nargs, const op_arg *args,
                  int ninds, const int *inds) {
  // cache lookup (common/op_lib_core.c:632-659)
  for (auto &up : g_plans) {
    DevPlan &p = *up;
    if (p.name != name || p.set != set || p.nargs != nargs || p.ninds != ninds ||
        p.part_size != part_size)
      continue;
    bool match = true;
    for (int m = 0; m < nargs && match; m++)
      match = args[m].dat == p.dats[m] && args[m].map == p.maps[m] && args[m].idx == p.idxs[m] &&
              args[m].acc == p.accs[m];
    if (match) {
      if (OP_diags > 3) printf(" old execution plan #%d\n", (int)(&up - &g_plans[0]));
      p.count++;
      p.pub.count = p.count;
      return &p;
    }
  }
  if (OP_diags > 1) printf(" new execution plan #%d for kernel %s\n", (int)g_plans.size(), name);
  std::unique_ptr<DevPlan> up(new DevPlan());
  DevPlan &p = *up;
  p.name = name;
  p.set = set;
  p.part_size = part_size;
  p.nargs = nargs;
  p.ninds = ninds;
  for (int m = 0; m < nargs; m++) {
    p.dats.push_back(args[m].dat);
    p.maps.push_back(args[m].map);
    p.idxs.push_back(args[m].idx);
    p.accs.push_back(args[m].acc);
    p.inds.push_back(inds[m]);
  }
  p.count = 1;
  ensure_cuda();
  build_plan(p);
  if (error_pending()) return nullptr;
  fill_pub(p);
  g_plans.push_back(std::move(up));
  OP_plan_index = (int)g_plans.size();
  return g_plans.back().get();
}

long validate_plan(const DevPlan &p) {
  Runtime &R = rt();
  cudaStream_t s = R.stream;
  PlanParams pp;
  std::vector<int> to_sizes;
  if (!fill_params(pp, p, to_sizes)) return 1;
  unsigned long long *err = nullptr;
  int *d_to = nullptr, *seen = nullptr;
  OP2B_CUDA(pool_malloc_async((void **)&err, sizeof(unsigned long long), s));
  OP2B_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned long long), s));
  OP2B_CUDA(pool_malloc_async((void **)&d_to, sizeof(int) * (p.ninds ? p.ninds : 1), s));
  if (p.ninds)
    OP2B_CUDA(cudaMemcpyAsync(d_to, to_sizes.data(), sizeof(int) * p.ninds,
                              cudaMemcpyHostToDevice, s));
  OP2B_CUDA(pool_malloc_async((void **)&seen, sizeof(int) * p.nblocks, s));
  OP2B_CUDA(cudaMemsetAsync(seen, 0, sizeof(int) * p.nblocks, s));
  IndOut io;
  memset(&io, 0, sizeof io);
  for (int m = 0; m < p.ninds; m++) io.ind_maps[m] = p.d_ind_maps[m];
  for (int a = 0; a < p.nargs; a++) io.loc_maps[a] = p.d_loc_maps[a];

  k_check_blocks<<<64, 256, 0, s>>>(pp, p.d_blkmap, p.d_offset, p.d_nelems, seen, err);
  if (p.ninds) {
    k_check_indmaps<<<dim3(p.nblocks, p.ninds), 256, 0, s>>>(pp, io, p.d_ind_sizes,
                                                             p.d_ind_offs, d_to, err);
    k_check_locmaps<<<592, 256, 0, s>>>(pp, io, p.d_ind_sizes, p.d_ind_offs, err);
  }
  size_t sm = sizeof(int) * (pp.mask_words ? pp.mask_words : 1);
  allow_smem(k_check_thread_colours);
  k_check_thread_colours<<<p.nblocks, 256, sm, s>>>(pp, io, p.d_ind_sizes, p.d_thrcol,
                                                    p.d_nthrcol, err);
  // block colours: one pass per colour over its blocks, owner arrays reset
  IncWork iw;
  memset(&iw, 0, sizeof iw);
  std::vector<unsigned *> owners;
  std::vector<int> ind_w(kMaxArgs, -1), osz;
  for (int sl = 0; sl < pp.ninc; sl++) {
    int m = pp.inc_ind[sl];
    if (ind_w[m] < 0) {
      unsigned *w = nullptr;
      OP2B_CUDA(pool_malloc_async((void **)&w, sizeof(int) * (size_t)to_sizes[m], s));
      ind_w[m] = (int)owners.size();
      owners.push_back(w);
      osz.push_back(to_sizes[m]);
    }
    iw.work[sl] = owners[ind_w[m]];
  }
  for (int c = 0; c < p.ncolors; c++) {
    for (size_t w = 0; w < owners.size(); w++)
      OP2B_CUDA(cudaMemsetAsync(owners[w], 0xff, sizeof(int) * (size_t)osz[w], s));
    if (pp.ninc && p.ncolblk[c] > 0)
      k_check_block_colours<<<std::min(p.ncolblk[c], 4096), 256, 0, s>>>(
          pp, iw, p.d_blkmap, p.colstart[c], p.ncolblk[c], err);
  }
  unsigned long long h = 0;
  OP2B_CUDA(cudaMemcpyAsync(&h, err, sizeof h, cudaMemcpyDeviceToHost, s));
  for (unsigned *w : owners) OP2B_CUDA(cudaFreeAsync(w, s));
  OP2B_CUDA(cudaFreeAsync(err, s));
  OP2B_CUDA(cudaFreeAsync(d_to, s));
  OP2B_CUDA(cudaFreeAsync(seen, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  // block count / colour count consistency (common/op_lib_core.c:476-492)
  long nblock = 0;
  for (int c = 0; c < p.ncolors; c++) nblock += p.ncolblk[c];
  if (nblock != p.nblocks) h++;
  return (long)h;
}

// ------------------------------------------------------------ gather plan --

struct SlotMaps {
  const int *map[kMaxArgs];
  int dim[kMaxArgs];
  int idx[kMaxArgs];
};

__global__ void k_gather_count(SlotMaps sm, int nslots, int n, int *cnt) {
  long long tot = (long long)n * nslots;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    int e = (int)(i / nslots), sl = (int)(i % nslots);
    int t = sm.map[sl][sm.idx[sl] + (size_t)e * sm.dim[sl]];
    atomicAdd(&cnt[t], 1);
  }
}

__global__ void k_flags(const int *cnt, int n, int *flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flags[i] = cnt[i] > 0;
}

__global__ void k_compact_active(const int *cnt, const int *pos, int n, int *active,
                                 int *acnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (cnt[i] > 0) {
      active[pos[i]] = i;
      acnt[pos[i]] = cnt[i];
    }
}

__global__ void k_gather_scatter(SlotMaps sm, int nslots, int n, const int *slot_of_target,
                                 int *cursor, int *keys) {
  long long tot = (long long)n * nslots;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    int e = (int)(i / nslots), sl = (int)(i % nslots);
    int t = sm.map[sl][sm.idx[sl] + (size_t)e * sm.dim[sl]];
    int r = slot_of_target ? slot_of_target[t] : t;
    int p = atomicAdd(&cursor[r], 1);
    keys[p] = (int)i;  // i == e * nslots + sl
  }
}

// rows are short on meshes; insertion-sort each row, one thread per row,
// and leave rows longer than 64 to the CTA sorter below
__global__ void k_sort_rows(const int *row, int nrows, int *keys, int *long_rows, int *nlong,
                            int *maxlen) {
  int mx = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
    int a = row[r], b = row[r + 1];
    mx = max(mx, b - a);
    if (b - a > 64) {
      long_rows[atomicAdd(nlong, 1)] = r;
      continue;
    }
    for (int i = a + 1; i < b; i++) {
      int v = keys[i], j = i - 1;
      while (j >= a && keys[j] > v) {
        keys[j + 1] = keys[j];
        j--;
      }
      keys[j + 1] = v;
    }
  }
  mx = __reduce_max_sync(0xffffffffu, mx);
  if ((threadIdx.x & 31) == 0 && mx > 0) atomicMax(maxlen, mx);
}

// tile_first[b] = first row r with row[r] >= kTile * b (lower bound), for
// b = 0..ntiles; row has nrows + 1 non-decreasing entries
__global__ void k_tile_first(const int *row, int nrows, int ntiles, int *tile_first) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= ntiles; b += gridDim.x * blockDim.x) {
    long long want = (long long)kTile * b;
    int lo = 0, hi = nrows;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (row[mid] < want) lo = mid + 1; else hi = mid;
    }
    tile_first[b] = b == ntiles ? nrows : lo;
  }
}

__global__ void k_sort_long_rows(const int *row, const int *long_rows, int *keys) {
  extern __shared__ int s[];
  int r = long_rows[blockIdx.x];
  int a = row[r], len = row[r + 1] - a;
  int P = 1;
  while (P < len) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < len ? keys[a + i] : INT_MAX;
  __syncthreads();
  bitonic_sort(s, P);
  for (int i = threadIdx.x; i < len; i += blockDim.x) keys[a + i] = s[i];
}

// key = element * nslots + slot -> perm[element] * nslots + slot
__global__ void k_keys_through(int *keys, long long n, int nslots, const int *perm) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = keys[i];
    keys[i] = perm[k / nslots] * nslots + k % nslots;
  }
}

GatherPlan *get_gather_plan(op_set set, const op_arg *args, const std::vector<int> &slots) {
  for (auto &up : g_gather) {
    GatherPlan &g = *up;
    if (g.set != set || g.nslots != (int)slots.size() || g.dat != args[slots[0]].dat) continue;
    bool match = true;
    for (int k = 0; k < g.nslots && match; k++)
      match = g.maps[k] == args[slots[k]].map && g.idxs[k] == args[slots[k]].idx;
    if (match) return &g;
  }
  Runtime &R = rt();
  cudaStream_t s = R.stream;
  std::unique_ptr<GatherPlan> up(new GatherPlan());
  GatherPlan &g = *up;
  g.set = set;
  g.dat = args[slots[0]].dat;
  g.nslots = (int)slots.size();
  g.ntarget = g.dat->set->size;
  SlotMaps sm;
  memset(&sm, 0, sizeof sm);
  if (g.nslots > kMaxArgs) {
    fail(-1, "op2b error -- too many OP_INC arguments on one dataset\n");
    return nullptr;
  }
  for (int k = 0; k < g.nslots; k++) {
    const op_arg &a = args[slots[k]];
    g.maps.push_back(a.map);
    g.idxs.push_back(a.idx);
    sm.map[k] = map_dev(a.map);
    sm.dim[k] = a.map->dim;
    sm.idx[k] = a.idx;
  }
  const int n = set->size, T = g.ntarget;
  const long long nkeys = (long long)n * g.nslots;
  if (nkeys > INT_MAX) {
    fail(-1, "op2b error -- loop too large for 32-bit gather keys\n");
    return nullptr;
  }
  int *cnt = nullptr, *flags = nullptr, *pos = nullptr, *acnt = nullptr;
  OP2B_CUDA(pool_malloc_async((void **)&cnt, sizeof(int) * T, s));
  OP2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * T, s));
  const int grid = R.num_sms * 8;
  k_gather_count<<<grid, 256, 0, s>>>(sm, g.nslots, n, cnt);
  OP2B_CUDA(pool_malloc_async((void **)&flags, sizeof(int) * T, s));
  OP2B_CUDA(pool_malloc_async((void **)&pos, sizeof(int) * T, s));
  k_flags<<<grid, 256, 0, s>>>(cnt, T, flags);
  g.nactive = (int)exclusive_scan(flags, pos, T, s);
  int *rowcnt = cnt;
  const int *slot_of_target = nullptr;
  if (g.nactive < T) {
    g.d_active = (int *)dev_alloc(sizeof(int) * std::max(1, g.nactive));
    OP2B_CUDA(pool_malloc_async((void **)&acnt, sizeof(int) * std::max(1, g.nactive), s));
    k_compact_active<<<grid, 256, 0, s>>>(cnt, pos, T, g.d_active, acnt);
    rowcnt = acnt;
    slot_of_target = pos;
  }
  g.d_row = (int *)dev_alloc(sizeof(int) * ((size_t)g.nactive + 1));
  g.d_keys = (int *)dev_alloc(sizeof(int) * (size_t)std::max(1LL, nkeys));
  long long total = g.nactive ? exclusive_scan(rowcnt, g.d_row, g.nactive, s) : 0;
  int tot32 = (int)total;
  OP2B_CUDA(cudaMemcpyAsync(g.d_row + g.nactive, &tot32, sizeof(int), cudaMemcpyHostToDevice, s));
  int *cursor = nullptr, *long_rows = nullptr, *nlong = nullptr, *maxlen = nullptr;
  OP2B_CUDA(pool_malloc_async((void **)&cursor, sizeof(int) * ((size_t)g.nactive + 1), s));
  OP2B_CUDA(cudaMemcpyAsync(cursor, g.d_row, sizeof(int) * ((size_t)g.nactive + 1),
                            cudaMemcpyDeviceToDevice, s));
  k_gather_scatter<<<grid, 256, 0, s>>>(sm, g.nslots, n, slot_of_target, cursor, g.d_keys);
  // renumbered loop set: order each row by the app's element numbers (the
  // order of op_seq.h), then turn the keys back into device numbers below
  const int *to_orig = perm_new2old_dev(set), *to_dev = perm_old2new_dev(set);
  if (to_orig && nkeys)
    k_keys_through<<<grid, 256, 0, s>>>(g.d_keys, nkeys, g.nslots, to_orig);
  OP2B_CUDA(pool_malloc_async((void **)&long_rows, sizeof(int) * std::max(1, g.nactive), s));
  OP2B_CUDA(pool_malloc_async((void **)&nlong, sizeof(int) * 2, s));
  maxlen = nlong + 1;
  OP2B_CUDA(cudaMemsetAsync(nlong, 0, sizeof(int) * 2, s));
  k_sort_rows<<<grid, 256, 0, s>>>(g.d_row, g.nactive, g.d_keys, long_rows, nlong, maxlen);
  int h[2] = {0, 0};
  OP2B_CUDA(cudaMemcpyAsync(h, nlong, sizeof h, cudaMemcpyDeviceToHost, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  g.max_row = h[1];
  g.nkeys = total;
  g.ntiles = (int)((total + kTile - 1) / kTile);
  g.d_tile_first = (int *)dev_alloc(sizeof(int) * ((size_t)g.ntiles + 1));
  k_tile_first<<<(g.ntiles + 256) / 256, 256, 0, s>>>(g.d_row, g.nactive, g.ntiles, g.d_tile_first);
  if (h[0] > 0) {
    int P = 1;
    while (P < g.max_row) P <<= 1;
    if ((size_t)P * sizeof(int) > smem_optin()) {
      fail(-1, "op2b error -- a target has %d contributions, too many to order on chip\n",
           g.max_row);
      return nullptr;
    }
    allow_smem(k_sort_long_rows);
    k_sort_long_rows<<<h[0], 1024, sizeof(int) * P, s>>>(g.d_row, long_rows, g.d_keys);
  }
  if (to_dev && nkeys) k_keys_through<<<grid, 256, 0, s>>>(g.d_keys, nkeys, g.nslots, to_dev);
  OP2B_CUDA(cudaFreeAsync(cnt, s));
  OP2B_CUDA(cudaFreeAsync(flags, s));
  OP2B_CUDA(cudaFreeAsync(pos, s));
  if (acnt) OP2B_CUDA(cudaFreeAsync(acnt, s));
  OP2B_CUDA(cudaFreeAsync(cursor, s));
  OP2B_CUDA(cudaFreeAsync(long_rows, s));
  OP2B_CUDA(cudaFreeAsync(nlong, s));
  OP2B_CUDA(cudaStreamSynchronize(s));
  g_gather.push_back(std::move(up));
  return g_gather.back().get();
}

// ------------------------------------------------------------- slot plan --

// contributions per target of plan a (cnt = row length) and then of b
__global__ void k_ell_count(int nrows, const int *active, const int *row, int *cnt) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nrows; t += gridDim.x * blockDim.x)
    cnt[active ? active[t] : t] += row[t + 1] - row[t];
}

// write plan a's entries (its CSR keys are already edge << 1 | slot), or
// plan b's ((na + key) << 1) after a's; cnt is the fill level per target
__global__ void k_ell_fill(int nrows, const int *active, const int *row, const int *keys,
                           int width, int offset, int shift, int *cnt, int *ell) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nrows; t += gridDim.x * blockDim.x) {
    const int c = active ? active[t] : t;
    const int k0 = row[t], k1 = row[t + 1], base = cnt[c];
    for (int k = k0; k < k1; k++)
      ell[(size_t)c * width + base + (k - k0)] = (offset + keys[k]) << shift;
    cnt[c] = base + k1 - k0;
  }
}

__global__ void k_max_int(const int *v, int n, int *out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_fill_int(int *p, size_t n, int v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

static std::vector<std::unique_ptr<SlotPlan>> g_slot_plans;

SlotPlan *get_slot_plan(const GatherPlan *a, const GatherPlan *b) {
  for (auto &up : g_slot_plans)
    if (up->a == a && up->b == b) return up->width > 0 ? up.get() : nullptr;
  std::unique_ptr<SlotPlan> up(new SlotPlan());
  SlotPlan &p = *up;
  p.a = a;
  p.b = b;
  p.ntarget = a->ntarget;
  p.na = a->set->size;
  p.nb = b ? b->set->size : 0;
  const bool shape = a->nslots == 2 && (!b || (b->nslots == 1 && b->ntarget == a->ntarget)) &&
                     (long long)p.na + p.nb + 1 < (1LL << 30);
  if (shape && a->nactive > 0) {
    cudaStream_t s = rt().stream;
    const int grid = rt().num_sms * 8;
    int *cnt = nullptr;
    OP2B_CUDA(pool_malloc_async((void **)&cnt, sizeof(int) * ((size_t)p.ntarget + 1), s));
    int *mx = cnt + p.ntarget;
    OP2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)p.ntarget + 1), s));
    k_ell_count<<<grid, 256, 0, s>>>(a->nactive, a->d_active, a->d_row, cnt);
    if (b && b->nactive) k_ell_count<<<grid, 256, 0, s>>>(b->nactive, b->d_active, b->d_row, cnt);
    k_max_int<<<grid, 256, 0, s>>>(cnt, p.ntarget, mx);
    int w = 0;
    OP2B_CUDA(cudaMemcpyAsync(&w, mx, sizeof(int), cudaMemcpyDeviceToHost, s));
    OP2B_CUDA(cudaStreamSynchronize(s));
    const long long nkeys = a->nkeys + (b ? b->nkeys : 0);
    if (w >= 1 && w <= kMaxSlotWidth && (long long)w * p.ntarget <= 2 * nkeys + p.ntarget) {
      p.width = w;
      const size_t n = (size_t)w * p.ntarget;
      p.d_ell = (int *)dev_alloc(sizeof(int) * n);
      if (!p.d_ell) {
        p.width = 0;
      } else {
        k_fill_int<<<grid, 256, 0, s>>>(p.d_ell, n, (p.na + p.nb) << 1);
        OP2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)p.ntarget, s));
        k_ell_fill<<<grid, 256, 0, s>>>(a->nactive, a->d_active, a->d_row, a->d_keys, w, 0, 0,
                                        cnt, p.d_ell);
        if (b && b->nactive)
          k_ell_fill<<<grid, 256, 0, s>>>(b->nactive, b->d_active, b->d_row, b->d_keys, w, p.na,
                                          1, cnt, p.d_ell);
      }
    }
    OP2B_CUDA(cudaFreeAsync(cnt, s));
    OP2B_CUDA(cudaStreamSynchronize(s));
  }
  g_slot_plans.push_back(std::move(up));
  SlotPlan *r = g_slot_plans.back().get();
  return r->width > 0 ? r : nullptr;
}

}  // namespace op2b

using namespace op2b;

void op2b_release_plans() {
  for (auto &up : g_slot_plans) {
    release_chain_sched(up.get());
    release_tile_plan(up.get());
    dev_free(up->d_ell);
    dev_free(up->d_buf);
  }
  g_slot_plans.clear();
  for (auto &up : g_plans) {
    DevPlan &p = *up;
    dev_free(p.d_nthrcol); dev_free(p.d_thrcol); dev_free(p.d_offset); dev_free(p.d_nelems);
    dev_free(p.d_ind_offs); dev_free(p.d_ind_sizes); dev_free(p.d_blkmap);
    for (int *q : p.d_ind_maps) dev_free(q);
    for (short *q : p.d_loc_maps) dev_free(q);
  }
  g_plans.clear();
  for (auto &up : g_gather) {
    dev_free(up->d_row); dev_free(up->d_keys); dev_free(up->d_active);
    dev_free(up->d_tile_first);
    dev_free(up->d_contrib);
  }
  g_gather.clear();
  extern void op2b_release_host_plans();
  op2b_release_host_plans();
  OP_plan_index = 0;
}

// host copies made by op_plan_core
static std::vector<op_plan *> g_host_plans;

void op2b_release_host_plans() {
  for (op_plan *o : g_host_plans) {
    for (int m = 0; m < o->ninds; m++) free(o->ind_maps[m]);
    for (int a = 0; a < o->nargs; a++) free(o->loc_maps[a]);
    free(o->ind_maps); free(o->loc_maps); free(o->nthrcol); free(o->thrcol); free(o->offset);
    free(o->ind_offs); free(o->ind_sizes); free(o->nindirect); free(o->nelems);
    free(o->ncolblk); free(o->blkmap);
    delete o;
  }
  g_host_plans.clear();
}

extern "C" {

op_plan *op_plan_get(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                     int ninds, int *inds) {
  DevPlan *p = get_plan(name, set, part_size, nargs, args, ninds, inds);
  return p ? &p->pub : nullptr;
}

// common/op_lib_core.c:627: the same plan, with every array in host memory
op_plan *op_plan_core(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                      int ninds, int *inds) {
  DevPlan *p = get_plan(name, set, part_size, nargs, args, ninds, inds);
  if (!p) return nullptr;
  for (op_plan *o : g_host_plans)
    if (o->name == p->pub.name && o->set == set && o->part_size == part_size &&
        o->dats == p->pub.dats) {
      o->count = p->count;
      return o;
    }
  cudaStream_t s = rt().stream;
  op_plan *o = new op_plan(p->pub);
  const int nb = p->nblocks, n = set->size, ni = p->ninds;
  auto d2h = [&](const void *d, size_t bytes) {
    void *h = malloc(bytes ? bytes : 1);
    if (bytes) OP2B_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
    return h;
  };
  o->nthrcol = (int *)d2h(p->d_nthrcol, sizeof(int) * nb);
  o->thrcol = (int *)d2h(p->d_thrcol, sizeof(int) * (size_t)n);
  o->offset = (int *)d2h(p->d_offset, sizeof(int) * nb);
  o->nelems = (int *)d2h(p->d_nelems, sizeof(int) * nb);
  o->ind_offs = (int *)d2h(p->d_ind_offs, sizeof(int) * (size_t)nb * ni);
  o->ind_sizes = (int *)d2h(p->d_ind_sizes, sizeof(int) * (size_t)nb * ni);
  o->blkmap = (int *)d2h(p->d_blkmap, sizeof(int) * nb);
  o->ind_maps = (int **)calloc(ni ? ni : 1, sizeof(int *));
  for (int m = 0; m < ni; m++)
    o->ind_maps[m] = (int *)d2h(p->d_ind_maps[m], sizeof(int) * (size_t)p->nindirect[m]);
  o->loc_maps = (short **)calloc(p->nargs, sizeof(short *));
  for (int a = 0; a < p->nargs; a++)
    if (p->d_loc_maps[a]) o->loc_maps[a] = (short *)d2h(p->d_loc_maps[a], sizeof(short) * (size_t)n);
  o->nindirect = (int *)malloc(sizeof(int) * (size_t)(ni > 0 ? ni : 1));
  for (int m = 0; m < ni; m++) o->nindirect[m] = p->nindirect[m];
  o->ncolblk = (int *)malloc(sizeof(int) * std::max(1, p->ncolors));
  for (int c = 0; c < p->ncolors; c++) o->ncolblk[c] = p->ncolblk[c];
  OP2B_CUDA(cudaStreamSynchronize(s));
  g_host_plans.push_back(o);
  return o;
}

long op2b_plan_validate(char const *name, op_set set, int part_size, int nargs, op_arg *args,
                        int ninds, int *inds) {
  DevPlan *p = get_plan(name, set, part_size, nargs, args, ninds, inds);
  if (!p) return -1;
  return validate_plan(*p);
}

}  // extern "C"
