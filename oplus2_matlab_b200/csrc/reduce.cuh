// reduce.cuh -- device side of global reductions (op_arg_gbl with OP_INC /
// OP_MIN / OP_MAX).
//
// The reference reduces with a shared-memory tree whose last 32 steps rely on
// warp-synchronous execution (common/op_lib.cu:268-332), a pattern that is
// undefined under independent thread scheduling (sm_70 and later), then sums
// 200 block partials on the host.  Here:
//   TREE: each thread folds its elements in ascending order, lanes combine with
//         __shfl_down_sync in a fixed pattern, warps through shared memory,
//         blocks write a partial, and the last block to finish (atomic ticket)
//         folds the partials in index order.  The grid is a function of the
//         set size only, so results are bit-reproducible run to run.
//   SEQ:  the loop writes each contribution to a scratch array in element
//         order and one warp folds them one addition at a time from the
//         caller's initial value -- the order of op_seq.h, bit for bit.
#pragma once

#include <cuda_runtime.h>

namespace op2b {

struct OpSum {
  template <class T>
  __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};
// MAX(a, b) of common/op_lib_core.h:167 with a = running value
struct OpMax {
  template <class T>
  __device__ __forceinline__ T operator()(T a, T b) const { return (a > b) ? a : b; }
};
struct OpMin {
  template <class T>
  __device__ __forceinline__ T operator()(T a, T b) const { return (a < b) ? a : b; }
};

template <class T, class Op>
__device__ __forceinline__ T warp_fold(T v, Op op) {
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Block fold; result valid in thread 0.  Uses `ws` (>= 32 entries).
template <class T, class Op>
__device__ __forceinline__ T block_fold(T v, T identity, Op op, T *ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_fold(v, op);
  __syncthreads();
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < nw ? ws[lane] : identity;
    v = warp_fold(v, op);
  }
  return v;
}

// Per-call device storage of one reduction: block partials and the result.
template <class T>
struct RedSlot {
  T *partials;         // [gridDim.x]
  T *result;           // final value (no host seed applied)
};

// Finish up to two reductions of one kernel: write block partials, and let
// the last block fold them in index order.  `ticket` must be 0 on entry and
// is reset to 0 by the last block.
template <class T, class Op0, class Op1, int N>
__device__ __forceinline__ void grid_finish(const T (&v)[N], const T (&identity)[N], Op0 op0,
                                            Op1 op1, RedSlot<T> (&slot)[N], unsigned *ticket) {
  __shared__ T ws[32];
  __shared__ bool last;
#pragma unroll
  for (int i = 0; i < N; i++) {
    T b = i == 0 ? block_fold(v[i], identity[i], op0, ws) : block_fold(v[i], identity[i], op1, ws);
    if (threadIdx.x == 0) slot[i].partials[blockIdx.x] = b;
  }
  // thread 0 wrote the partials: it alone fences them before taking a ticket
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int i = 0; i < N; i++) {
    T x = identity[i];
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
      T p = __ldcg(slot[i].partials + k);
      x = i == 0 ? op0(x, p) : op1(x, p);
    }
    x = i == 0 ? block_fold(x, identity[i], op0, ws) : block_fold(x, identity[i], op1, ws);
    if (threadIdx.x == 0) *slot[i].result = x;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// SEQ mode: out = (((init + v[0]) + v[1]) + ...) + v[n-1], in order.  One
// warp: the lanes stage 32-element tiles in shared memory (double buffered),
// lane 0 folds them.
template <class T>
__global__ void k_seq_sum(const T *__restrict__ v, long long n, T init, T *out,
                          const int *__restrict__ order = nullptr, int w = 1) {
  __shared__ T tile[2][1024];
  const int lane = threadIdx.x;
  T acc = init;
  long long base = 0;
  int buf = 0;
  // value j of the sum: v[j], or, for a renumbered set, component j % w of
  // the element the app numbers j / w, stored at order[j / w]
  auto at = [&](long long j) {
    return order ? v[(long long)w * order[j / w] + j % w] : v[j];
  };
  for (int i = lane; i < 1024; i += 32) tile[0][i] = (i < n) ? at(i) : T(0);
  __syncwarp();
  while (base < n) {
    long long next = base + 1024;
    for (int i = lane; i < 1024; i += 32) {
      long long j = next + i;
      tile[buf ^ 1][i] = (j < n) ? at(j) : T(0);
    }
    if (lane == 0) {
      long long m = n - base < 1024 ? n - base : 1024;
      for (int i = 0; i < m; i++) acc = acc + tile[buf][i];
    }
    __syncwarp();
    buf ^= 1;
    base = next;
  }
  if (lane == 0) *out = acc;
}

}  // namespace op2b
