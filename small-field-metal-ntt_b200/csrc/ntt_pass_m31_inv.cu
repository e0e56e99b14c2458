// Instantiates the tile-engine passes for M31, inv direction.
#include "ntt_launch.cuh"

namespace sfntt {
Status run_pass_m31_inv(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  return run_pass_impl<M31, false>(ctx, req, s);
}
}  // namespace sfntt
