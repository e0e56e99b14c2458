// Instantiates the tile-engine passes for BabyBear, fwd direction.
#include "ntt_launch.cuh"

namespace sfntt {
Status run_pass_bb_fwd(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  return run_pass_impl<BabyBear, true>(ctx, req, s);
}
}  // namespace sfntt
