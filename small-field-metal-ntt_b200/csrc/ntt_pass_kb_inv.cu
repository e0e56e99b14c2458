// Instantiates the tile-engine passes for KoalaBear, inv direction.
#include "ntt_launch.cuh"

namespace sfntt {
Status run_pass_kb_inv(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  return run_pass_impl<KoalaBear, false>(ctx, req, s);
}
}  // namespace sfntt
