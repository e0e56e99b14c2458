// Instantiates the persistent TMA passes for KoalaBear, fwd direction.
#include "tma_launch.cuh"

namespace sfntt {
Status run_tma_pass_kb_fwd(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s) {
  return run_tma_pass_impl<KoalaBear, true>(ctx, r, s);
}
}  // namespace sfntt
