// noalloc.cu -- the airfoil update loop for callers that cannot allocate.
//
// op_par_loop_update needs scratch memory for its rms reduction (one partial
// sum per block, a completion ticket, a result slot), which the library
// allocates on first use.  Some callers cannot allow that:
//  - code that must not call cudaMalloc while other work is in flight,
//    because cudaMalloc can synchronise the device and stall it;
//  - hosts that hand all device memory to their own pool up front and
//    forbid any other allocation;
//  - real-time or latency-bound threads where a first-call allocation is
//    an unbounded pause.
// For them, op2b_update_noalloc runs the same update on arrays the caller
// owns.  Its scratch is the fixed array below, compiled into the library;
// every GPU that loads the library holds it (16 KB) until the process exits.
//
// Limits and rules (also in include/op2b.h):
//  - ncell <= 4096 * 1024 = 4,194,304 (one partial sum per 1024 cells);
//    larger sets are rejected with an error and nothing runs;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  The address is cached per device until
//    op_exit; a caller that resets a device (cudaDeviceReset) must call
//    op_exit first, so that the next call looks the address up again;
//  - qold, q and res are read and written as 16-byte vectors, so they must
//    be 16-byte aligned (adt and rms 4-byte); misaligned pointers are
//    rejected before anything is launched;
//  - all calls share the one array: calls that overlap on the GPU (on
//    different streams, or from different threads) race and give wrong
//    sums.  Calls in one stream are ordered and safe.
// No cudaMalloc, cudaFree or other allocating routine is called here.

#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "reduce.cuh"

namespace {

constexpr int kNoAllocCellsPerBlock = 1024;  // 256 threads x 4 cells
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kNoAllocMaxCells = kNoAllocCellsPerBlock * kNoAllocMaxBlocks;

// partial sums [0, kNoAllocMaxBlocks), then the ticket (as unsigned bits)
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocMaxBlocks + 64];

// q = qold - res/adt, res = 0, rms += del^2 (airfoil/update.h:1-12), one
// pass of 4 cells per thread; the block partials go to `partials`, the last
// block adds their fold to *rms
__global__ void __launch_bounds__(256) k_update_noalloc(int n, const float *__restrict__ qold,
                                                         float *__restrict__ q,
                                                         float *__restrict__ res,
                                                         const float *__restrict__ adt,
                                                         float *rms, float *partials,
                                                         unsigned *ticket) {
  float sum = 0.0f;
  const int stride = gridDim.x * blockDim.x;
  const int base = blockIdx.x * blockDim.x + threadIdx.x;
  float qo[4][4], r[4][4], ad[4];
#pragma unroll
  for (int u = 0; u < 4; u++) {
    int c = base + u * stride;
    if (c < n) {
      float4 a = __ldg(reinterpret_cast<const float4 *>(qold) + c);
      float4 b = reinterpret_cast<const float4 *>(res)[c];
      qo[u][0] = a.x; qo[u][1] = a.y; qo[u][2] = a.z; qo[u][3] = a.w;
      r[u][0] = b.x; r[u][1] = b.y; r[u][2] = b.z; r[u][3] = b.w;
      ad[u] = __ldg(adt + c);
    }
  }
#pragma unroll
  for (int u = 0; u < 4; u++) {
    int c = base + u * stride;
    if (c >= n) continue;
    float adti = __frcp_rn(ad[u]);  // IEEE 1/x, as 1.0f/x on x86
    float qn[4];
    for (int d = 0; d < 4; d++) {
      float del = adti * r[u][d];
      qn[d] = qo[u][d] - del;
      sum += del * del;
    }
    reinterpret_cast<float4 *>(q)[c] = make_float4(qn[0], qn[1], qn[2], qn[3]);
    reinterpret_cast<float4 *>(res)[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  __shared__ float ws[32];
  __shared__ bool last;
  float b = op2b::block_fold(sum, 0.0f, op2b::OpSum(), ws);
  if (threadIdx.x == 0) {  // the writer fences its partial, then takes a ticket
    partials[blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  float x = 0.0f;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) x += __ldcg(partials + k);
  x = op2b::block_fold(x, 0.0f, op2b::OpSum(), ws);
  if (threadIdx.x == 0) {
    *rms = *rms + x;  // OP_INC: added to the value already there
    *ticket = 0u;
  }
}

// device address of g_noalloc_scratch, looked up once per device
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kNoAllocMaxDevices];

}  // namespace

namespace op2b {
// op_exit: forget the cached addresses (a device reset after op_exit
// invalidates them; the next call looks them up again)
void noalloc_reset() {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto &a : g_addr) a = nullptr;
}
}  // namespace op2b

extern "C" int op2b_update_noalloc(int ncell, const float *qold, float *q, float *res,
                                   const float *adt, float *rms, void *stream) {
  if (ncell < 0 || ncell > kNoAllocMaxCells) {
    fprintf(stderr,
            "op2b_update_noalloc error: %d cells is outside 0..%d, the most its fixed "
            "scratch can reduce; nothing was run\n",
            ncell, kNoAllocMaxCells);
    return -1;
  }
  if (ncell > 0 && (!qold || !q || !res || !adt || !rms)) {
    fprintf(stderr, "op2b_update_noalloc error: null device pointer argument\n");
    return -3;
  }
  if (ncell > 0 && ((((uintptr_t)qold | (uintptr_t)q | (uintptr_t)res) & 15) ||
                    (((uintptr_t)adt | (uintptr_t)rms) & 3))) {
    fprintf(stderr,
            "op2b_update_noalloc error: qold, q and res must be 16-byte aligned and adt, rms "
            "4-byte aligned; nothing was run\n");
    return -3;
  }
  if (ncell == 0) return 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    fprintf(stderr,
            "op2b_update_noalloc error: device %d is beyond the %d devices whose scratch "
            "address it caches; nothing was run\n",
            dev, kNoAllocMaxDevices);
    return -2;
  }
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      e = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_addr[dev] = nullptr;
        fprintf(stderr, "op2b_update_noalloc error: cannot find the scratch array: %s\n",
                cudaGetErrorString(e));
        return -2;
      }
    }
    base = g_addr[dev];
  }
  float *partials = (float *)base;
  unsigned *ticket = (unsigned *)((float *)base + kNoAllocMaxBlocks);
  cudaStream_t s = (cudaStream_t)stream;
  // the array keeps the last call's contents: the ticket must start at zero
  e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return (int)e;
  const int grid = (ncell + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock;
  k_update_noalloc<<<grid, 256, 0, s>>>(ncell, qold, q, res, adt, rms, partials, ticket);
  return (int)cudaGetLastError();
}
