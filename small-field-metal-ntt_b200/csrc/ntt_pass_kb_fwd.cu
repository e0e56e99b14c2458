// Instantiates the tile-engine passes for KoalaBear, fwd direction.
#include "ntt_launch.cuh"

namespace sfntt {
Status run_pass_kb_fwd(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  return run_pass_impl<KoalaBear, true>(ctx, req, s);
}
}  // namespace sfntt
