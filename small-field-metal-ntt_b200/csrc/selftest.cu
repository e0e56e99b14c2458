// selftest.cu -- exercises the bounded device-side wait without a fault.
//
// Every mbarrier wait of the tile kernels gives up after a time limit, sets
// the context's error flag and lets the kernel return, so a copy that never
// lands surfaces as SFNTT_TIMEOUT instead of a hung GPU.  This entry point
// runs that same wait (tma::mbar_wait) on a barrier that nothing arrives on
// (arrive = 0) or that gets its one arrival (arrive = 1), with a short limit,
// so tests can check the whole path: the flag, the status, and a context that
// still works afterwards.
#include <algorithm>

#include "context.hpp"
#include "tma.cuh"

namespace sfntt {
namespace {

__global__ void __launch_bounds__(64) bounded_wait_kernel(int* err, uint64_t timeout_ns, int arrive) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tma::mbar_init(&bar, 1);
    tma::fence_mbar_init();
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0) tma::mbar_arrive(&bar);
  const bool ok = tma::mbar_wait(&bar, 0, timeout_ns);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicExch(err, 1);
}

}  // namespace
}  // namespace sfntt

extern "C" int sfntt_selftest_bounded_wait(sfntt_ctx* ctx, uint64_t timeout_ns, int arrive) {
  using namespace sfntt;
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  auto run = [&]() -> Status {
    const uint64_t limit = std::min<uint64_t>(std::max<uint64_t>(timeout_ns, 1000), 1000000000ull);  // <= 1 s
    launch_begin(ctx, ctx->stream);
    bounded_wait_kernel<<<1, 64, 0, ctx->stream>>>(ctx->err.as<int>(), limit, arrive ? 1 : 0);
    SFNTT_TRY(launch_check(ctx, "selftest_bounded_wait", ctx->stream));
    SFNTT_CU(cudaStreamSynchronize(ctx->stream));
    return {};
  };
  Status s = run();
  cudaSetDevice(prev);
  ctx->last_error = s.ok() ? std::string() : s.msg;
  if (!s.ok()) return s.code;
  return sfntt_check_device_error(ctx);
}
