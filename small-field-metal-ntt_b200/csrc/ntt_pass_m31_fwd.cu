// Instantiates the tile-engine passes for M31, fwd direction.
#include "ntt_launch.cuh"

namespace sfntt {
Status run_pass_m31_fwd(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  return run_pass_impl<M31, true>(ctx, req, s);
}
}  // namespace sfntt
