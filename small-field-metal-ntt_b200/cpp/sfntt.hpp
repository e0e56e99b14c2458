// sfntt.hpp -- C++ host mirror of the reference's NTT / LDE API over the C ABI.
//
// The reference is a Rust crate; its hot-path surface is the NttBackend<F>
// trait (src/ntt/mod.rs:26-49) with one backend type per algorithm variant
// and field (src/ntt/m31/*, src/ntt/babybear/*), the NttError enum
// (src/ntt/mod.rs:52-69) and CosetLdeBatch / LdeResult (src/lde/mod.rs:15-107).
// This header mirrors that surface for C++ callers: the same type names
// (Metal* names are aliases of the Cuda* ones), the same argument meaning
// (in-place slices, SoA columns data[col * n + row], Montgomery BabyBear,
// canonical M31, bit-reversed forward output), and NttError as an exception
// carrying the variant and its payload.  Everything runs through
// include/sfntt.h (link with -lsfntt); there is no CPU fallback.
//
// Beyond the reference: device-pointer calls, uneven batches in one CUDA-graph
// launch (LdeBatch / Graph), and the continuous-batching request server.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

#include "../../include/sfntt.h"

namespace sfntt {

// Field element types: #[repr(transparent)] u32 newtypes in the reference
// (M31(pub u32), src/field/m31.rs:10; BabyBear(pub u32), src/field/babybear.rs:12).
struct M31 {
  uint32_t v;
  static constexpr int kField = SFNTT_M31;
};
struct BabyBear {
  uint32_t v;  // Montgomery form
  static constexpr int kField = SFNTT_BABYBEAR;
};
// KoalaBear (p = 2^31 - 2^24 + 1): planned in the reference (README.md:20), no
// type there; Montgomery form like BabyBear.
struct KoalaBear {
  uint32_t v;  // Montgomery form
  static constexpr int kField = SFNTT_KOALABEAR;
};
static_assert(sizeof(M31) == 4 && sizeof(BabyBear) == 4 && sizeof(KoalaBear) == 4, "field elements are one u32");

enum class Variant : int { Best = SFNTT_BEST, CtDitR2 = 1, CtGsR2 = 2, StockhamR2 = 3, CtGsR4 = 4 };

// NttError (src/ntt/mod.rs:52-69).  size() is the InvalidSize payload (the
// offending length) or the requested bytes of BufferAllocFailed.
class NttError : public std::runtime_error {
 public:
  enum class Kind : int {
    InvalidSize = SFNTT_INVALID_SIZE,
    DeviceNotFound = SFNTT_DEVICE_NOT_FOUND,
    BufferAllocFailed = SFNTT_ALLOC_FAILED,
    ShaderCompileError = SFNTT_KERNEL_LOAD,
    GpuExecutionError = SFNTT_GPU_EXECUTION,
    CorrectnessMismatch = SFNTT_MISMATCH,
    Unsupported = SFNTT_UNSUPPORTED,  // the reference panics (V1 inverse is todo!())
    Timeout = SFNTT_TIMEOUT,
    InvalidArgument = SFNTT_INVALID_ARGUMENT,
  };
  NttError(Kind kind, const std::string& what, size_t size = 0)
      : std::runtime_error(what), kind_(kind), size_(size) {}
  Kind kind() const { return kind_; }
  size_t size() const { return size_; }

 private:
  Kind kind_;
  size_t size_;
};

namespace detail {

inline void check(const sfntt_ctx* ctx, int status, size_t size = 0) {
  if (status == SFNTT_OK) return;
  std::string what = sfntt_status_string(status);
  const char* detail = ctx ? sfntt_last_error(ctx) : nullptr;
  if (detail && *detail) what += std::string(": ") + detail;
  if (status == SFNTT_INVALID_SIZE) what = "Invalid NTT size: " + std::to_string(size) + " (" + what + ")";
  throw NttError(static_cast<NttError::Kind>(status), what, size);
}

template <class F>
uint32_t* words(std::span<F> s) {
  return s.empty() ? nullptr : reinterpret_cast<uint32_t*>(s.data());
}
template <class F>
const uint32_t* words(std::span<const F> s) {
  return s.empty() ? nullptr : reinterpret_cast<const uint32_t*>(s.data());
}

}  // namespace detail

// MetalContext (src/gpu.rs:26-64): one device, its stream, cached twiddle
// tables and staging buffers.  Copies share the same context.
class Context {
 public:
  explicit Context(int device = 0) {
    sfntt_ctx* h = nullptr;
    detail::check(nullptr, sfntt_ctx_create(device, &h));
    ctx_ = std::shared_ptr<sfntt_ctx>(h, sfntt_ctx_destroy);
  }
  sfntt_ctx* handle() const { return ctx_.get(); }
  // MetalContext::device_info (src/gpu.rs:132-150)
  std::string device_info() const {
    char buf[256] = {};
    detail::check(handle(), sfntt_device_info(handle(), buf, sizeof buf));
    return buf;
  }
  void prepare(int field, uint32_t log_n) const { detail::check(handle(), sfntt_prepare(handle(), field, log_n)); }
  void prepare_lde(int field, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty = 0) const {
    detail::check(handle(), sfntt_prepare_lde(handle(), field, log_n, added_bits, shift_monty));
  }
  uint64_t launch_count() const { return sfntt_launch_count(handle()); }
  // Device-side waits are bounded; after asynchronous _dev work, synchronise
  // the stream and call this to turn a timed-out wait into NttError::Timeout.
  void check_device_error() const { detail::check(handle(), sfntt_check_device_error(handle())); }

 private:
  std::shared_ptr<sfntt_ctx> ctx_;
};

// trait NttBackend<F: Field> (src/ntt/mod.rs:26-49).
template <class F>
class NttBackend {
 public:
  virtual ~NttBackend() = default;
  virtual std::string_view name() const = 0;
  // Coefficients -> evaluations (bit-reversed order), in place.  The twiddles
  // are ignored, as by every reference backend (src/ntt/mod.rs:33-36).
  virtual void forward_ntt(std::span<F> data, std::span<const F> twiddles = {}) const = 0;
  // Bit-reversed evaluations -> coefficients (times n^-1), in place.
  virtual void inverse_ntt(std::span<F> data, std::span<const F> twiddles = {}) const = 0;
  virtual void pointwise_mul(std::span<const F> a, std::span<const F> b, std::span<F> out) const = 0;
};

// One backend type per (field, variant): the reference's Metal* structs.
template <class F, Variant V>
class CudaBackend final : public NttBackend<F> {
 public:
  explicit CudaBackend(Context ctx = Context()) : ctx_(std::move(ctx)) {}
  // Same shape as the reference's `new(shader_dir)`: kernels are compiled
  // ahead of time for sm_100a, so the directory is not used.
  static CudaBackend create(const std::string& /*shader_dir*/ = {}, int device = 0) {
    return CudaBackend(Context(device));
  }

  std::string_view name() const override { return kName; }

  void forward_ntt(std::span<F> data, std::span<const F> = {}) const override {
    detail::check(ctx_.handle(), sfntt_forward(ctx_.handle(), F::kField, (int)V, detail::words(data), data.size(),
                                               nullptr),
                  data.size());
  }
  void inverse_ntt(std::span<F> data, std::span<const F> = {}) const override {
    detail::check(ctx_.handle(), sfntt_inverse(ctx_.handle(), F::kField, (int)V, detail::words(data), data.size(),
                                               nullptr),
                  data.size());
  }
  void pointwise_mul(std::span<const F> a, std::span<const F> b, std::span<F> out) const override {
    detail::check(ctx_.handle(),
                  sfntt_pointwise_mul(ctx_.handle(), F::kField, detail::words(a), a.size(), detail::words(b),
                                      b.size(), detail::words(out), out.size()),
                  a.size());
  }

  // forward_ntt_gpu / inverse_ntt_gpu(input, log_n) -> (Vec<u32>, ns)
  // (src/ntt/babybear/metal_ct_gs_r4.rs:87-172, src/ntt/m31/metal_ct_gs_r4.rs:61-99)
  std::pair<std::vector<uint32_t>, uint64_t> forward_ntt_gpu(std::span<const uint32_t> input, uint32_t log_n) const {
    return gpu(sfntt_forward_gpu, input, log_n);
  }
  std::pair<std::vector<uint32_t>, uint64_t> inverse_ntt_gpu(std::span<const uint32_t> input, uint32_t log_n) const {
    return gpu(sfntt_inverse_gpu, input, log_n);
  }
  // BbBatchNtt::forward_ntt_batch_gpu / inverse_ntt_batch_gpu (src/ntt/babybear/batch.rs:76-180)
  std::pair<std::vector<uint32_t>, uint64_t> forward_ntt_batch_gpu(std::span<const uint32_t> input, uint32_t log_n,
                                                                   uint32_t batch) const {
    return batched(sfntt_forward_batch, input, log_n, batch);
  }
  std::pair<std::vector<uint32_t>, uint64_t> inverse_ntt_batch_gpu(std::span<const uint32_t> input, uint32_t log_n,
                                                                   uint32_t batch) const {
    return batched(sfntt_inverse_batch, input, log_n, batch);
  }
  // Device-pointer twins: asynchronous on `stream` (a cudaStream_t).
  void forward_dev(uint32_t* d_data, uint32_t log_n, uint32_t batch = 1, void* stream = nullptr) const {
    detail::check(ctx_.handle(), sfntt_forward_dev(ctx_.handle(), F::kField, (int)V, d_data, log_n, batch, stream),
                  (size_t)batch << log_n);
  }
  void inverse_dev(uint32_t* d_data, uint32_t log_n, uint32_t batch = 1, void* stream = nullptr) const {
    detail::check(ctx_.handle(), sfntt_inverse_dev(ctx_.handle(), F::kField, (int)V, d_data, log_n, batch, stream),
                  (size_t)batch << log_n);
  }
  const Context& ctx() const { return ctx_; }

 private:
  static constexpr std::string_view name_of() {
    constexpr bool bb = F::kField == SFNTT_BABYBEAR, kb = F::kField == SFNTT_KOALABEAR;
    switch (V) {
      case Variant::CtDitR2: return bb ? "bb-cuda-ct-dit-r2" : kb ? "kb-cuda-ct-dit-r2" : "cuda-ct-dit-r2";
      case Variant::CtGsR2: return bb ? "bb-cuda-r2" : kb ? "kb-cuda-r2" : "cuda-ct-gs-r2";
      case Variant::StockhamR2: return bb ? "bb-cuda-stockham-r2" : kb ? "kb-cuda-stockham-r2" : "cuda-stockham-r2";
      case Variant::CtGsR4: return bb ? "bb-cuda-ct-gs-r4" : kb ? "kb-cuda-ct-gs-r4" : "cuda-ct-gs-r4";
      default: return bb ? "bb-cuda" : kb ? "kb-cuda" : "cuda";
    }
  }
  static constexpr std::string_view kName = name_of();

  template <class Fn>
  std::pair<std::vector<uint32_t>, uint64_t> gpu(Fn fn, std::span<const uint32_t> input, uint32_t log_n) const {
    std::vector<uint32_t> out(input.size());
    uint64_t ns = 0;
    detail::check(ctx_.handle(),
                  fn(ctx_.handle(), F::kField, (int)V, input.data(), input.size(), log_n, out.data(), &ns),
                  input.size());
    return {std::move(out), ns};
  }
  template <class Fn>
  std::pair<std::vector<uint32_t>, uint64_t> batched(Fn fn, std::span<const uint32_t> input, uint32_t log_n,
                                                     uint32_t batch) const {
    std::vector<uint32_t> out(input.size());
    uint64_t ns = 0;
    detail::check(ctx_.handle(), fn(ctx_.handle(), F::kField, input.data(), input.size(), log_n, batch, out.data(), &ns),
                  input.size());
    return {std::move(out), ns};
  }

  Context ctx_;
};

// M31 Circle NTT (DCCT) backends (src/ntt/m31/*).
using CudaCtDitR2 = CudaBackend<M31, Variant::CtDitR2>;       // V1, forward only
using CudaCtGsR2 = CudaBackend<M31, Variant::CtGsR2>;         // V2
using CudaStockhamR2 = CudaBackend<M31, Variant::StockhamR2>; // V3
using CudaCtGsR4 = CudaBackend<M31, Variant::CtGsR4>;         // V4
// BabyBear backends (src/ntt/babybear/*).
using BbCudaCtDitR2 = CudaBackend<BabyBear, Variant::CtDitR2>;
using BbBatchNtt = CudaBackend<BabyBear, Variant::CtGsR2>;
using BbCudaStockhamR2 = CudaBackend<BabyBear, Variant::StockhamR2>;
using BbCudaCtGsR4 = CudaBackend<BabyBear, Variant::CtGsR4>;
// KoalaBear backends: the BabyBear variants over KoalaBear.
using KbCudaCtDitR2 = CudaBackend<KoalaBear, Variant::CtDitR2>;
using KbBatchNtt = CudaBackend<KoalaBear, Variant::CtGsR2>;
using KbCudaStockhamR2 = CudaBackend<KoalaBear, Variant::StockhamR2>;
using KbCudaCtGsR4 = CudaBackend<KoalaBear, Variant::CtGsR4>;
// The reference's type names (src/ntt/m31/*, src/ntt/babybear/*, src/ntt/metal_r2.rs:337-340).
using MetalCtDitR2 = CudaCtDitR2;
using MetalCtGsR2 = CudaCtGsR2;
using MetalStockhamR2 = CudaStockhamR2;
using MetalCtGsR4 = CudaCtGsR4;
using BbMetalCtDitR2 = BbCudaCtDitR2;
using BbMetalR2 = BbBatchNtt;
using BbMetalStockhamR2 = BbCudaStockhamR2;
using BbMetalCtGsR4 = BbCudaCtGsR4;

// LdeResult (src/lde/mod.rs:20-25): SoA data[col * n_ext + row], device time.
struct LdeResult {
  std::vector<uint32_t> data;
  uint64_t total_ns = 0;
};

// CosetLdeBatch (src/lde/mod.rs:15-107): iDFT -> x n^-1 -> zero-pad ->
// x shift^i -> DFT over batch_size BabyBear columns (KbCosetLdeBatch: the
// same over KoalaBear).
// natural = true: natural-order input evaluations and output rows (Plonky3's
// coset_lde_batch convention) instead of the reference's bit-reversed ones.
template <class F>
class BasicCosetLdeBatch {
 public:
  explicit BasicCosetLdeBatch(Context ctx = Context(), bool fused = true, bool natural = false)
      : ctx_(std::move(ctx)),
        mode_((fused ? SFNTT_LDE_FUSED : SFNTT_LDE_UNFUSED) | (natural ? SFNTT_LDE_NATURAL : 0)) {}
  static BasicCosetLdeBatch create(const std::string& /*shader_dir*/ = {}, int device = 0) {
    return BasicCosetLdeBatch(Context(device));
  }
  // shift_monty = 0: the reference shift two_adic_generator(log_n + added_bits + 1).
  LdeResult execute(std::span<const uint32_t> input, size_t log_n, size_t batch_size, size_t added_bits,
                    uint32_t shift_monty = 0) const {
    LdeResult r;
    r.data.resize(batch_size << (log_n + added_bits));
    detail::check(ctx_.handle(),
                  sfntt_coset_lde(ctx_.handle(), F::kField, input.data(), input.size(), (uint32_t)log_n,
                                  (uint32_t)batch_size, (uint32_t)added_bits, shift_monty, mode_, r.data.data(),
                                  &r.total_ns),
                  input.size());
    return r;
  }
  void execute_dev(const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch_size, uint32_t added_bits,
                   uint32_t shift_monty = 0, void* stream = nullptr) const {
    detail::check(ctx_.handle(),
                  sfntt_coset_lde_dev(ctx_.handle(), F::kField, d_in, d_out, log_n, batch_size, added_bits,
                                      shift_monty, mode_, stream),
                  (size_t)batch_size << log_n);
  }
  std::string device_info() const { return ctx_.device_info(); }

 private:
  Context ctx_;
  int mode_;
};
using CosetLdeBatch = BasicCosetLdeBatch<BabyBear>;
using KbCosetLdeBatch = BasicCosetLdeBatch<KoalaBear>;

// M31 blow-up: inverse on odds(log n) -> zero-pad -> forward on
// odds(log n + added_bits).  No reference counterpart; that composition of
// reference functions.
class M31Lde {
 public:
  explicit M31Lde(Context ctx = Context()) : ctx_(std::move(ctx)) {}
  LdeResult execute(std::span<const uint32_t> input, size_t log_n, size_t batch_size, size_t added_bits) const {
    LdeResult r;
    r.data.resize(batch_size << (log_n + added_bits));
    detail::check(ctx_.handle(),
                  sfntt_m31_lde(ctx_.handle(), input.data(), input.size(), (uint32_t)log_n, (uint32_t)batch_size,
                                (uint32_t)added_bits, r.data.data(), &r.total_ns),
                  input.size());
    return r;
  }
  void execute_dev(const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch_size, uint32_t added_bits,
                   void* stream = nullptr) const {
    detail::check(ctx_.handle(), sfntt_m31_lde_dev(ctx_.handle(), d_in, d_out, log_n, batch_size, added_bits, stream),
                  (size_t)batch_size << log_n);
  }

 private:
  Context ctx_;
};

// Canonic-coset circle FFT and circle LDE over M31 (no reference counterpart):
// the M31 network with circle-FFT twiddles on odds(log n) ordered half coset
// then conjugates, values bit-reversed; the LDE interpolates, zero-pads the
// coefficients and evaluates on odds(log n + added_bits).
class CircleLde {
 public:
  explicit CircleLde(Context ctx = Context()) : ctx_(std::move(ctx)) {}
  // inverse = false evaluates coefficients, true interpolates (times n^-1); returns (out, device ns)
  std::pair<std::vector<uint32_t>, uint64_t> ntt(std::span<const uint32_t> in, uint32_t log_n, uint32_t batch,
                                                 bool inverse) const {
    std::vector<uint32_t> out(in.size());
    uint64_t ns = 0;
    detail::check(ctx_.handle(),
                  sfntt_circle_ntt(ctx_.handle(), inverse ? 1 : 0, in.data(), in.size(), log_n, batch, out.data(), &ns),
                  in.size());
    return {std::move(out), ns};
  }
  LdeResult execute(std::span<const uint32_t> input, size_t log_n, size_t batch_size, size_t added_bits) const {
    LdeResult r;
    r.data.resize(log_n + added_bits <= 40 ? batch_size << (log_n + added_bits) : 0);
    detail::check(ctx_.handle(),
                  sfntt_circle_lde(ctx_.handle(), input.data(), input.size(), (uint32_t)log_n, (uint32_t)batch_size,
                                   (uint32_t)added_bits, r.data.data(), &r.total_ns),
                  input.size());
    return r;
  }

 private:
  Context ctx_;
};

// Circle NTT over CM31 = M31[i]/(i^2+1) columns of interleaved (re, im) pairs
// (the M31 transform of each coordinate; no reference counterpart).
class Cm31Ntt {
 public:
  explicit Cm31Ntt(Context ctx = Context()) : ctx_(std::move(ctx)) {}
  // len(pairs) = 2 * (batch << log_n) words; returns (out, device ns)
  std::pair<std::vector<uint32_t>, uint64_t> ntt(std::span<const uint32_t> pairs, uint32_t log_n, uint32_t batch,
                                                 bool inverse) const {
    std::vector<uint32_t> out(pairs.size());
    uint64_t ns = 0;
    detail::check(ctx_.handle(),
                  sfntt_cm31_ntt(ctx_.handle(), inverse ? 1 : 0, pairs.data(), pairs.size(), log_n, batch, out.data(),
                                 &ns),
                  pairs.size());
    return {std::move(out), ns};
  }

 private:
  Context ctx_;
};

// ---- output layout ------------------------------------------------------------
// Row order / row-major form of a SoA batch: SFNTT_LAYOUT_NATURAL (bit-reversed
// rows -> natural), SFNTT_LAYOUT_ROW_MAJOR (out[row * batch + col], the
// Merkle-commitment input).  Returns (out, device ns).
inline std::pair<std::vector<uint32_t>, uint64_t> layout(const Context& ctx, std::span<const uint32_t> in,
                                                         uint32_t log_n, uint32_t batch, int flags) {
  std::vector<uint32_t> out(in.size());
  uint64_t ns = 0;
  detail::check(ctx.handle(), sfntt_layout(ctx.handle(), in.data(), in.size(), log_n, batch, flags, out.data(), &ns),
                in.size());
  return {std::move(out), ns};
}
inline void layout_dev(const Context& ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                       int flags, void* stream = nullptr) {
  detail::check(ctx.handle(), sfntt_layout_dev(ctx.handle(), d_in, d_out, log_n, batch, flags, stream),
                (size_t)batch << log_n);
}

// ---- uneven batches in one graph launch -----------------------------------
enum class Plan : int { Auto = SFNTT_PLAN_AUTO, Tma = SFNTT_PLAN_TMA, TmaFourStep = SFNTT_PLAN_TMA_FOUR_STEP,
                        Tile = SFNTT_PLAN_TILE };

inline sfntt_lde_item lde_item(int field, uint32_t log_n, uint32_t batch, uint32_t added_bits, const uint32_t* d_in,
                               uint32_t* d_out, Plan plan = Plan::Auto, uint32_t shift_monty = 0) {
  return sfntt_lde_item{field, log_n, batch, added_bits, shift_monty, d_in, d_out, (int)plan};
}

// An instantiated CUDA graph of a whole batch; launch() is one launch.
class Graph {
 public:
  Graph(Context ctx, sfntt_graph* g) : ctx_(std::move(ctx)), g_(g, sfntt_graph_destroy) {}
  void launch(void* stream = nullptr) const { detail::check(ctx_.handle(), sfntt_graph_launch(g_.get(), stream)); }
  uint64_t kernel_count() const { return sfntt_graph_kernel_count(g_.get()); }

 private:
  Context ctx_;
  std::unique_ptr<sfntt_graph, void (*)(sfntt_graph*)> g_;
};

class LdeBatch {
 public:
  LdeBatch(Context ctx, std::vector<sfntt_lde_item> items) : ctx_(std::move(ctx)), items_(std::move(items)) {}
  void prepare() const { detail::check(ctx_.handle(), sfntt_batch_prepare(ctx_.handle(), items_.data(), items_.size())); }
  // The plain per-polynomial loop on `stream`.
  void run(void* stream = nullptr) const {
    detail::check(ctx_.handle(), sfntt_batch_run(ctx_.handle(), items_.data(), items_.size(), stream));
  }
  void autotune(int reps = 2) const {
    detail::check(ctx_.handle(), sfntt_autotune(ctx_.handle(), items_.data(), items_.size(), reps));
  }
  Plan plan_of(size_t i) const { return static_cast<Plan>(sfntt_tune_lookup(ctx_.handle(), &items_.at(i))); }
  Graph graph(int lanes = 8) const {
    sfntt_graph* g = nullptr;
    detail::check(ctx_.handle(), sfntt_batch_graph_create(ctx_.handle(), items_.data(), items_.size(), lanes, &g));
    return Graph(ctx_, g);
  }

 private:
  Context ctx_;
  std::vector<sfntt_lde_item> items_;
};

// ---- serving ----------------------------------------------------------------
// Continuous-batching server (sfntt_server_*): `slots` streams and one device
// arena of `budget_bytes`; requests are admitted in order as slots and arena
// space free up.  Driven from one thread.
class Server {
 public:
  Server(Context ctx, size_t budget_bytes, int slots = 8) : ctx_(std::move(ctx)), s_(nullptr, sfntt_server_destroy) {
    sfntt_server* s = nullptr;
    detail::check(ctx_.handle(), sfntt_server_create(ctx_.handle(), budget_bytes, slots, &s));
    s_.reset(s);
  }
  // Input on the device at req.d_in; the output lives in the arena until release.
  uint64_t submit(const sfntt_lde_item& req) {
    uint64_t t = 0;
    detail::check(ctx_.handle(), sfntt_server_submit(s_.get(), &req, &t));
    return t;
  }
  // Input copied from h_in, output copied to h_out before the ticket completes.
  uint64_t submit_host(const sfntt_lde_item& req, std::span<const uint32_t> h_in, std::span<uint32_t> h_out) {
    if (h_in.size() != ((size_t)req.batch << req.log_n) || h_out.size() != ((size_t)req.batch << (req.log_n + req.added_bits)))
      throw NttError(NttError::Kind::InvalidSize, "host buffers do not match the request", h_in.size());
    uint64_t t = 0;
    detail::check(ctx_.handle(), sfntt_server_submit_host(s_.get(), &req, h_in.data(), h_out.data(), &t));
    return t;
  }
  // Retire finished requests and admit queued ones; returns finished tickets.
  std::vector<uint64_t> poll(size_t cap = 256) {
    std::vector<uint64_t> done(cap);
    size_t n = 0;
    detail::check(ctx_.handle(), sfntt_server_poll(s_.get(), done.data(), done.size(), &n));
    done.resize(n);
    return done;
  }
  uint32_t* result(uint64_t ticket) const {
    uint32_t* p = nullptr;
    detail::check(ctx_.handle(), sfntt_server_result(s_.get(), ticket, &p));
    return p;
  }
  void release(uint64_t ticket) { detail::check(ctx_.handle(), sfntt_server_release(s_.get(), ticket)); }
  size_t pending() const { return sfntt_server_pending(s_.get()); }

 private:
  Context ctx_;
  std::unique_ptr<sfntt_server, void (*)(sfntt_server*)> s_;
};

// Replays a trace (sorted arrival times in seconds); slots = 1 is the plain
// sequential per-request loop.  Returns (latency per request, makespan).
inline std::pair<std::vector<double>, double> serve_trace(const Context& ctx, const std::vector<sfntt_lde_item>& reqs,
                                                          const std::vector<double>& arrival_s, int slots,
                                                          size_t budget_bytes) {
  std::vector<double> lat(reqs.size());
  double makespan = 0;
  detail::check(ctx.handle(), sfntt_serve_trace(ctx.handle(), reqs.data(), nullptr, nullptr, arrival_s.data(),
                                                reqs.size(), slots, budget_bytes, lat.data(), &makespan));
  return {std::move(lat), makespan};
}

}  // namespace sfntt
