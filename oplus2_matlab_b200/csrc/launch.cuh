// launch.cuh -- kernel launches with programmatic dependent launch (PDL).
//
// Consecutive loops are dependent kernels on one stream.  Launched with
// the programmatic-serialization attribute, a kernel's CTAs may start while
// the previous kernel's last CTAs still run; the kernel then
//   1. loads only data no kernel writes (op_map arrays and the library's own
//      plan arrays, fixed once built) -- the first hop of its gathers,
//   2. executes griddepcontrol.wait, which returns once the previous grid
//      has completed and its memory operations are visible -- every thread
//      runs it before it reads or writes any dataset or reduction scratch,
//   3. executes griddepcontrol.launch_dependents, so the next kernel's CTAs
//      may take the SM slots this grid frees.
// A kernel triggers only after its own wait, so when the next kernel starts
// every kernel before this one has completed.  Without the attribute (the
// "pdl" tuning knob at 0), or after a kernel that never triggers, both
// instructions are no-ops and ordering is the stream's usual one.
#pragma once

#include <cuda_runtime.h>

#include <unordered_map>
#include <utility>

#include "internal.h"

namespace op2b {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// number of parameters of a kernel
template <class... KArgs>
constexpr int kernel_nparams(void (*)(KArgs...)) {
  return (int)sizeof...(KArgs);
}

// kernel<<<grid, block, smem, s>>>(args...), with PDL unless "pdl" is 0;
// only for kernels that call pdl_wait() before touching any dataset
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem,
                       cudaStream_t s, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = tuning("pdl", 1) ? 1 : 0;
  OP2B_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

// CTAs of `threads` threads (no dynamic shared memory) that one SM keeps
// resident at once for `kernel`: the size of one wave of a grid-stride
// grid is that times the SM count.  Cached per kernel (the host-side query
// costs microseconds; a loop call should not pay it each time).
inline int resident_ctas(const void *kernel, int threads, size_t smem = 0) {
  static std::unordered_map<const void *, int> cache;
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess ||
      n < 1)
    n = 1;
  cache.emplace(kernel, n);
  return n;
}

}  // namespace op2b
