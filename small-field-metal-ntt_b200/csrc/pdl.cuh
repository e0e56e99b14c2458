// pdl.cuh -- programmatic dependent launch between consecutive passes.
//
// A pass launched with launch_pdl may be scheduled while the previous kernel
// on its stream is still running; its threads first let their own dependents
// launch, then wait (griddepcontrol.wait) until every prerequisite grid has
// completed and its writes are visible, before touching global memory.  The
// launch gap between passes disappears; the ordering of their memory effects
// is that of a plain stream.  A kernel launched without the attribute (or
// after a non-kernel operation) passes the wait at once.
//
// Used for tiny grids only (pdl_fits): there the launch gap is most of a
// pass's time.  An early-launched grid is placed on whatever SM slots are free
// while the previous pass still runs; measured on B200, partial grids then
// end up packed onto part of the GPU and full persistent grids of the
// four-step BabyBear passes run slower, so larger grids launch plainly.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

namespace sfntt {

// First statement of every kernel launched with launch_pdl.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// PDL for a grid of `ctas` CTAs.
inline bool pdl_fits(uint64_t ctas) { return ctas <= 16; }

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl,
                              Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
#ifdef SFNTT_NO_PDL  // plain stream ordering (for comparisons)
  cfg.numAttrs = 0;
#else
  cfg.numAttrs = pdl ? 1 : 0;
#endif
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace sfntt
