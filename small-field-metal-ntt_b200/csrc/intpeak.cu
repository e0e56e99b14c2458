// intpeak.cu -- measured integer ceilings of this GPU for the NTT arithmetic.
//
// The NTT kernels are bound by 32-bit integer issue, not by HBM or tensor
// cores, so the bench reports a second roofline against what the SMs can do
// with register-resident data: the same butterflies the passes execute (GS on
// canonical values, lazy CT, Shoup multiplication), with no memory traffic at
// all.  Each thread keeps 16 independent values and a few twiddles in
// registers; results are folded into one word per thread so nothing is dead.
#include <algorithm>

#include "context.hpp"
#include "field.cuh"
#include "ntt_pass.cuh"

namespace sfntt {
namespace {

template <bool GS>
__global__ void __launch_bounds__(256) butterfly_peak_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
  uint32_t v[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) v[m] = (seed * (threadIdx.x + 1u) + 977u * m) % BabyBear::P;
  uint2 w[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const uint32_t x = (seed ^ (0x9E3779B9u * (l + 1) + blockIdx.x)) % BabyBear::P;
    w[l] = make_uint2(x, (uint32_t)(((uint64_t)x << 32) / BabyBear::P));
  }
  for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 3; j >= 0; --j) {
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        if (m & (1 << j)) continue;
        butterfly<BabyBear, GS>(v[m], v[m | (1 << j)], w[j]);
      }
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int m = 0; m < 16; ++m) acc ^= v[m];
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace
}  // namespace sfntt

extern "C" int sfntt_butterfly_peak(sfntt_ctx* ctx, int gs, double* butterflies_per_s) {
  using namespace sfntt;
  if (!ctx || !butterflies_per_s) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  auto run = [&]() -> Status {
    const uint32_t blocks = (uint32_t)ctx->sm_count * 8;  // 2048 threads per SM
    const uint32_t threads = 256;
    SFNTT_TRY(ctx->buf_aux.reserve((size_t)blocks * threads * 4));
    uint32_t* out = ctx->buf_aux.as<uint32_t>();
    const uint32_t iters = 4096;
    auto launch = [&](uint32_t it) {
      if (gs) butterfly_peak_kernel<true><<<blocks, threads, 0, ctx->stream>>>(out, it, 12345u);
      else butterfly_peak_kernel<false><<<blocks, threads, 0, ctx->stream>>>(out, it, 12345u);
    };
    launch(64);  // warm-up
    SFNTT_TRY(launch_check(ctx, "butterfly_peak"));
    SFNTT_CU(cudaEventRecord(ctx->ev_start, ctx->stream));
    launch(iters);
    SFNTT_TRY(launch_check(ctx, "butterfly_peak"));
    SFNTT_CU(cudaEventRecord(ctx->ev_stop, ctx->stream));
    SFNTT_CU(cudaEventSynchronize(ctx->ev_stop));
    float ms = 0.f;
    SFNTT_CU(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
    const double bf = (double)blocks * threads * iters * 32.0;  // 4 layers x 8 butterflies
    *butterflies_per_s = bf / (ms * 1e-3);
    return {};
  };
  Status s = run();
  cudaSetDevice(prev);
  ctx->last_error = s.ok() ? std::string() : s.msg;
  return s.code;
}
