// Instantiates the tile-engine passes for BabyBear, inv direction.
#include "ntt_launch.cuh"

namespace sfntt {
Status run_pass_bb_inv(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  return run_pass_impl<BabyBear, false>(ctx, req, s);
}
}  // namespace sfntt
