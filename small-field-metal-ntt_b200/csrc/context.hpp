// context.hpp -- internal state behind an sfntt_ctx: device, stream, the
// device-resident twiddle / multiplier caches and the staging buffers used by
// the host-memory entry points.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/sfntt.h"

namespace sfntt {

// Error carried from a failing step to the C ABI.
struct Status {
  int code = SFNTT_OK;
  std::string msg;
  bool ok() const { return code == SFNTT_OK; }
};

inline int map_cuda_error(cudaError_t e) {
  switch (e) {
    case cudaSuccess: return SFNTT_OK;
    case cudaErrorMemoryAllocation: return SFNTT_ALLOC_FAILED;
    case cudaErrorNoDevice:
    case cudaErrorInvalidDevice:
    case cudaErrorInsufficientDriver: return SFNTT_DEVICE_NOT_FOUND;
    case cudaErrorNoKernelImageForDevice:
    case cudaErrorInvalidDeviceFunction:
    case cudaErrorInvalidKernelImage: return SFNTT_KERNEL_LOAD;
    default: return SFNTT_GPU_EXECUTION;
  }
}

#define SFNTT_CU(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return ::sfntt::Status{::sfntt::map_cuda_error(e_),                              \
                             std::string(#call) + ": " + cudaGetErrorString(e_)};      \
  } while (0)

#define SFNTT_TRY(expr)                  \
  do {                                   \
    ::sfntt::Status s_ = (expr);         \
    if (!s_.ok()) return s_;             \
  } while (0)

// Device buffer owned by a context (grow-only).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  Status reserve(size_t want) {
    if (want <= bytes) return {};
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return {SFNTT_ALLOC_FAILED, "cudaMalloc(" + std::to_string(want) + " bytes) failed"};
    }
    bytes = want;
    return {};
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace sfntt

#ifndef SFNTT_NTT_PLAIN_DEFAULT
#define SFNTT_NTT_PLAIN_DEFAULT true
#endif
#ifndef SFNTT_LDE_PLAIN_DEFAULT
#define SFNTT_LDE_PLAIN_DEFAULT false
#endif

struct sfntt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;         // host-memory calls run here
  cudaStream_t copy_streams[2] = {};     // H2D / D2H lanes of the pipelined LDE
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::recursive_mutex mu;
  std::string last_error;
  int sm_count = 0;
  std::atomic<uint64_t> launches{0};

  // Twiddle tables: BabyBear / KoalaBear per-layer Shoup pairs (layer s at
  // 2^s - 1), shared by every n <= 2^monty_log[field slot][dir]; M31 per log_n
  // (layer l at n - n/2^l).
  sfntt::DevBuf monty_tw[2][2];
  uint32_t monty_log[2][2] = {{0, 0}, {0, 0}};
  std::map<uint32_t, sfntt::DevBuf> m31_tw[2];
  // canonic-coset circle FFT twiddles (same layout as m31_tw)
  std::map<uint32_t, sfntt::DevBuf> m31c_tw[2];
  // LDE multiplier and twist tables keyed by (field, log_n, added_bits, shift, kind)
  std::map<std::tuple<int, uint32_t, uint32_t, uint32_t, int>, sfntt::DevBuf> lde_tabs;

  // staging for host-memory calls
  sfntt::DevBuf buf_in, buf_out, buf_aux;
  // base-field planes of CM31 transforms (ext.cu)
  sfntt::DevBuf buf_ext;
  // device int set by a kernel whose bounded wait ran out (SFNTT_TIMEOUT)
  sfntt::DevBuf err;
  // route every pass through the first (non-TMA) tile engine (tests / A-B)
  bool no_tma = false;
  // single-launch cluster NTT for columns of 2^13 .. 2^16 points off (A-B)
  bool no_cluster = false;
  // BabyBear strided passes: plain sub-transforms + four-step twists applied by
  // neighbouring passes (true) or per-position twiddles (false); separately
  // for plain NTTs and the fused LDE.
  bool ntt_plain = SFNTT_NTT_PLAIN_DEFAULT;
  bool lde_plain = SFNTT_LDE_PLAIN_DEFAULT;
  // Tuning knobs (autotuned plans): layer ranges above 12 layers split as a
  // 12-layer contiguous pass plus the rest (instead of 8-layer strided passes
  // plus the rest); persistent TMA passes launched with at most this many CTAs
  // per SM (0: the kernel's own residency).
  bool split_c12 = false;
  int tma_ctas = 0;
  // contiguous 8- and 12-layer TMA passes run their two CTA halves as
  // independent pipelines (half tiles, own barriers); off: whole tiles
  bool c_halves = true;
  // persistent batches: items of at most this many tiles (2^13 input words)
  // join the work-list phases; larger items fill the GPU on their own and run
  // per item beside them.  -1: 16 tiles per SM; 0: no limit.
  int64_t worklist_max_tiles = -1;
  // autotuned plans: "field/log_n/columns/added_bits" -> sfntt_plan
  std::map<std::string, int> tuned;

  // Opt-in per-kernel timing (sfntt_kernel_timing): an event pair around every
  // launch, resolved and aggregated by name in sfntt_kernel_times.
  struct TimedLaunch { std::string name; uint64_t bytes; cudaEvent_t start, stop; };
  bool timing = false;
  std::vector<TimedLaunch> timed;
  cudaEvent_t pending_start = nullptr;
};

namespace sfntt {

// Montgomery-form fields (BabyBear, KoalaBear) share every kernel family;
// monty_slot indexes their per-field caches.
inline bool is_monty(int field) { return field == SFNTT_BABYBEAR || field == SFNTT_KOALABEAR; }
inline bool valid_field(int field) { return field == SFNTT_M31 || is_monty(field); }
inline int monty_slot(int field) { return field == SFNTT_KOALABEAR ? 1 : 0; }
// log_n + added_bits <= max_log, without the 32-bit sum wrapping for huge inputs.
inline bool ext_fits(uint32_t log_n, uint32_t added_bits, uint32_t max_log) {
  return log_n <= max_log && added_bits <= max_log && log_n + added_bits <= max_log;
}

// Table accessors (twiddles.cu).  All generate on a miss (allocating) and
// refuse to do so while `stream` is capturing.  `field` is BabyBear or
// KoalaBear for the monty_* tables.
Status monty_twiddles(sfntt_ctx* ctx, int field, bool inverse, uint32_t log_n, cudaStream_t stream,
                      const uint2** out);
Status m31_twiddles(sfntt_ctx* ctx, bool inverse, uint32_t log_n, cudaStream_t stream, const uint2** out);
Status m31_circle_twiddles(sfntt_ctx* ctx, bool inverse, uint32_t log_n, cudaStream_t stream, const uint2** out);
// kind 0: fused LDE multipliers M_q[i] = n^-1 (shift g^{rev(q)})^i, q < 2^added, i < n
// kind 1: plain shift powers shift^i, i < n_ext (unfused path)
// kind 2: kind 0 in the TMA expansion's tile order (log_n >= 13): entry
//         q n + (chunk 2^13 + e 32 + u) is M_q[chunk 32 + u + e 2^(log_n - 8)]
Status monty_lde_table(sfntt_ctx* ctx, int field, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty,
                       int kind, cudaStream_t stream, const uint2** out);

// Tables of the natural-order coset LDE (n >= 2^13): multipliers M_r[p] =
// n^-1 (shift g_ext^r)^rev(p) (r < 2^added_bits, p < n; within each 2^13-word
// tile, position 16 t + m is stored at m * 512 + t) and the n-point forward
// DIT twiddles laid out for columns of 2^added_bits interleaved cosets.
Status monty_natural_tables(sfntt_ctx* ctx, int field, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty,
                            cudaStream_t stream, const uint2** mul, const uint2** coset_tw);

// Twist of a strided BabyBear / KoalaBear pass over layers [lo, lo + P),
// indexed by column position mod 2^(lo+P) (cached like the LDE tables).
// compact: one word per entry, the Shoup companion w' (w = mulhi(w', p) + 1),
// for twists spanning 2^22 positions or more (the pair table would be 32 MiB+).
Status monty_twist_table(sfntt_ctx* ctx, int field, uint32_t lo, uint32_t P, bool inverse, cudaStream_t stream,
                         const uint2** out, bool compact = false);
inline bool twist_compact_for(uint32_t lo, uint32_t P) { return lo + P >= 22; }

// Kernel drivers (ntt.cu / lde.cu / elementwise.cu)
Status ntt_dev(sfntt_ctx* ctx, int field, int variant, bool inverse, uint32_t* d_data, uint32_t log_n,
               uint32_t batch, cudaStream_t stream);
// Layers [a, b) of a 2^log_n network on `batch` columns (first pass in -> out,
// later passes in place); scale_w != 0 multiplies the final outputs.
// edge_twist (BabyBear / KoalaBear, TMA engine only): a four-step twist applied to the
// inputs of a forward range or the outputs of an inverse range, indexed by
// column position & edge_mask -- the boundary with an adjacent strided pass
// run by another kernel.
// Layer split of a TMA range [a, b) (ntt.cu): passes lo[i], cnt[i]; 0 = none.
int tma_split(uint32_t a, uint32_t b, uint32_t lo[4], uint32_t cnt[4], bool c12_first, uint32_t cmax);
Status layers_dev(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* in, uint32_t* out, uint64_t in_stride,
                  uint64_t out_stride, uint32_t log_n, uint32_t batch, uint32_t a, uint32_t b, uint32_t scale_w,
                  const uint2* tw, cudaStream_t stream, const uint2* edge_twist = nullptr,
                  uint32_t edge_mask = 0);
// One-launch NTT of 2^13 .. 2^16-point columns on a thread-block cluster
// (cluster_ntt.cu), in place on dense columns; fits: shape, alignment and at
// most one wave of CTAs.
bool cluster_ntt_fits(const sfntt_ctx* ctx, uint32_t log_n, uint32_t batch, const void* d);
Status cluster_ntt_dev(sfntt_ctx* ctx, int field, bool inverse, uint32_t* d, uint32_t log_n, uint32_t batch,
                       const uint2* tw, uint32_t scale_w, cudaStream_t stream);
Status ntt_dev_oop(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* d_in, uint32_t* d_out,
                   uint64_t in_stride, uint64_t out_stride, uint32_t log_n, uint32_t batch, bool normalize,
                   cudaStream_t stream);
// Coset LDE over BabyBear or KoalaBear (lde.cu).
Status monty_lde_dev(sfntt_ctx* ctx, int field, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n,
                     uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode, cudaStream_t stream);
// canonic = false: the reference-network composition inverse(odds(log_n)) ->
// zero-pad -> forward(odds(log_n + added)); true: the canonic-coset circle LDE
// (same network, canonic circle-FFT twiddles).
Status m31_lde_dev(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                   uint32_t added_bits, cudaStream_t stream, bool canonic = false);
// Canonic-coset circle FFT (evaluate) / inverse (interpolate, times n^-1), in place.
Status circle_ntt_dev(sfntt_ctx* ctx, bool inverse, uint32_t* d, uint32_t log_n, uint32_t batch, cudaStream_t stream);
// n^-1 mod p, canonical (ntt.cu).
uint32_t inv_n_of(int field, uint32_t log_n);
// Row-order / row-major permutations of SoA batches (layout.cu); bitrev_cols_dev
// permutes each column's rows with separate column strides (in place if in == out).
Status bitrev_cols_dev(sfntt_ctx* ctx, const uint32_t* in, uint64_t in_stride, uint32_t* out, uint64_t out_stride,
                       uint32_t log_n, uint32_t batch, cudaStream_t s);
Status layout_dev(sfntt_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t log_n, uint32_t batch, int flags,
                  cudaStream_t s);
// One LDE / blow-up work item (batch.cu): run under its plan, or make its tables resident.
Status run_item(sfntt_ctx* ctx, const sfntt_lde_item& it, cudaStream_t s);
Status prepare_item(sfntt_ctx* ctx, const sfntt_lde_item& it, cudaStream_t s);
// CM31 = M31[i]/(i^2+1), interleaved (re, im) pairs (ext.cu).
Status cm31_scratch(sfntt_ctx* ctx, uint32_t log_n, uint32_t batch, cudaStream_t s, uint32_t** out);
Status cm31_ntt_dev(sfntt_ctx* ctx, bool inverse, uint32_t* d_pairs, uint32_t log_n, uint32_t batch, cudaStream_t s);
Status cm31_mul_dev(sfntt_ctx* ctx, const uint32_t* a, const uint32_t* b, uint32_t* out, size_t n, cudaStream_t s);
Status pointwise_mul_dev(sfntt_ctx* ctx, int field, const uint32_t* a, const uint32_t* b, uint32_t* out,
                         size_t n, cudaStream_t stream);
Status monty_convert_dev(sfntt_ctx* ctx, int field, bool to_monty, uint32_t* d, size_t n, cudaStream_t stream);
Status scale_dev(sfntt_ctx* ctx, int field, uint32_t* d, uint64_t n, uint32_t w_canonical, cudaStream_t stream);
Status zero_pad_dev(sfntt_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t log_n, uint32_t batch,
                    uint32_t added_bits, cudaStream_t stream);
Status mul_table_dev(sfntt_ctx* ctx, int field, uint32_t* d, uint32_t log_n_ext, uint32_t batch, const uint2* tab,
                     cudaStream_t stream);

inline void count_launch(sfntt_ctx* ctx, uint64_t n = 1) { ctx->launches.fetch_add(n, std::memory_order_relaxed); }

// Call right before a kernel launch on stream s (records the start event when
// per-kernel timing is on).
inline void launch_begin(sfntt_ctx* ctx, cudaStream_t s) {
  if (!ctx->timing) return;
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) == cudaSuccess && cudaEventRecord(e, s) == cudaSuccess) ctx->pending_start = e;
}

// Call right after the launch: checks the launch, counts it and, when timing
// is on, closes the event pair under `what` with its algorithmic HBM bytes.
inline Status launch_check(sfntt_ctx* ctx, const char* what, cudaStream_t s = nullptr, uint64_t bytes = 0) {
  count_launch(ctx);
  cudaError_t e = cudaGetLastError();
  if (ctx->timing && ctx->pending_start) {
    cudaEvent_t stop = nullptr;
    if (cudaEventCreate(&stop) == cudaSuccess && cudaEventRecord(stop, s) == cudaSuccess)
      ctx->timed.push_back({what, bytes, ctx->pending_start, stop});
    ctx->pending_start = nullptr;
  }
  if (e != cudaSuccess) return {map_cuda_error(e), std::string(what) + ": " + cudaGetErrorString(e)};
  return {};
}

// Raises a kernel's dynamic shared-memory limit once per device (the
// attribute stays with the function on that device); `done` is a static owned
// by the caller's launch function, one per kernel instantiation.
template <class Kernel>
inline Status smem_limit_once(Kernel kern, int bytes, int device, std::atomic<uint64_t>& done) {
  const uint64_t bit = 1ull << (device & 63);
  if (done.load(std::memory_order_acquire) & bit) return {};
  SFNTT_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.fetch_or(bit, std::memory_order_release);
  return {};
}

inline bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return st != cudaStreamCaptureStatusNone;
}

}  // namespace sfntt
