// Instantiates the persistent TMA passes for M31, inv direction.
#include "tma_launch.cuh"

namespace sfntt {
Status run_tma_pass_m31_inv(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s) {
  return run_tma_pass_impl<M31, false>(ctx, r, s);
}
}  // namespace sfntt
