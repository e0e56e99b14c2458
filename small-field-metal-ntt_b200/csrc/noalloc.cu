// noalloc.cu -- an NTT entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they run an NTT: code
// that executes while an allocator is locked down (a prover whose memory pool
// is sized once at start-up and must not grow), code inside host callbacks or
// in processes where device allocation is forbidden after initialisation, or
// embedders that account for every device byte themselves.  The library's
// other paths allocate lazily (context staging buffers, the Stockham variant's
// ping-pong buffer), so this entry point gives them the out-of-place Stockham
// transform (variant V3) with its ping-pong partner in a fixed, file-scope
// device array instead.
//
// Contract:
//   * the scratch array holds kNoAllocMaxWords words (4 MiB); every GPU that
//     loads the library keeps it until the process exits;
//   * batch << log_n must not exceed kNoAllocMaxWords (SFNTT_INVALID_SIZE);
//   * the context's twiddle tables for (field, log_n) must already be resident
//     (sfntt_prepare); the call never builds them (SFNTT_INVALID_ARGUMENT);
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it until the
//     process exits: make that first call before any stream capture, and do
//     not reset the device (cudaDeviceReset) while the library is loaded;
//   * every call shares the one array and leaves its last contents there; each
//     layer writes every word of its destination before any is read, so nothing
//     needs clearing, but calls whose work overlaps on the GPU (different
//     streams, no ordering between them) race on the array.
#include <mutex>

#include "context.hpp"
#include "host_field.hpp"

namespace sfntt {

constexpr size_t kNoAllocMaxWords = size_t(1) << 20;

// Device-side scratch.  In host code this name is only a stand-in for the
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxWords];

Status stockham_layer_dev(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* in, uint32_t* out,
                          const uint2* tw, uint32_t log_n, uint32_t L, uint32_t batch, uint32_t scale_w,
                          cudaStream_t s);

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
uint32_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which is current).
Status scratch_address(int device, uint32_t** out) {
  if (device < 0 || device >= kMaxDevices) return {SFNTT_DEVICE_NOT_FOUND, "device index out of range"};
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return {map_cuda_error(e), std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e)};
    }
    g_scratch_ptr[device] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_ptr[device];
  return {};
}

// Cached twiddles only: never generates (generation allocates).
Status resident_twiddles(sfntt_ctx* ctx, int field, bool inverse, uint32_t log_n, const uint2** tw) {
  const int d = inverse ? 1 : 0;
  if (is_monty(field)) {
    const int k = monty_slot(field);
    if (ctx->monty_tw[k][d].p && ctx->monty_log[k][d] >= log_n) {
      *tw = ctx->monty_tw[k][d].as<uint2>();
      return {};
    }
  } else {
    auto it = ctx->m31_tw[d].find(log_n);
    if (it != ctx->m31_tw[d].end()) {
      *tw = it->second.as<uint2>();
      return {};
    }
  }
  return {SFNTT_INVALID_ARGUMENT, "twiddles for this size are not resident: call sfntt_prepare first"};
}

}  // namespace
}  // namespace sfntt

extern "C" int sfntt_stockham_noalloc(sfntt_ctx* ctx, int field, int inverse, uint32_t* d_data, uint32_t log_n,
                                      uint32_t batch, void* stream) {
  using namespace sfntt;
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != ctx->device) cudaSetDevice(ctx->device);
  auto run = [&]() -> Status {
    if (!valid_field(field)) return {SFNTT_INVALID_ARGUMENT, "unknown field"};
    if ((is_monty(field) && log_n > host::monty_field(field).two_adicity) || (field == SFNTT_M31 && log_n > 30))
      return {SFNTT_INVALID_SIZE, "log_n exceeds the field's maximum"};
    const uint64_t words = (uint64_t)batch << log_n;
    if (words > kNoAllocMaxWords)
      return {SFNTT_INVALID_SIZE, "batch << log_n = " + std::to_string(words) + " exceeds the no-allocation scratch of " +
                                      std::to_string(kNoAllocMaxWords) + " words"};
    if (log_n == 0 || batch == 0) return {};
    if (!d_data) return {SFNTT_INVALID_ARGUMENT, "null buffer"};
    uint32_t* scratch = nullptr;
    SFNTT_TRY(scratch_address(ctx->device, &scratch));
    const uint2* tw = nullptr;
    SFNTT_TRY(resident_twiddles(ctx, field, inverse != 0, log_n, &tw));
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t scale = inverse ? inv_n_of(field, log_n) : 0u;
    uint32_t* bufs[2] = {d_data, scratch};
    int cur = 0;
    for (uint32_t i = 0; i < log_n; ++i) {
      const uint32_t L = inverse ? i : log_n - 1 - i;
      SFNTT_TRY(stockham_layer_dev(ctx, field, inverse != 0, bufs[cur], bufs[cur ^ 1], tw, log_n, L, batch,
                                   (inverse && i + 1 == log_n) ? scale : 0u, s));
      cur ^= 1;
    }
    if (cur != 0) SFNTT_CU(cudaMemcpyAsync(d_data, scratch, words * 4, cudaMemcpyDeviceToDevice, s));
    return {};
  };
  Status st = run();
  if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  ctx->last_error = st.ok() ? std::string() : st.msg;
  return st.code;
}
