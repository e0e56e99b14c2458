// capi.cu -- the extern "C" boundary (include/sfntt.h): argument checks with
// the reference's error semantics, host <-> device staging, timing, and the
// column-chunk pipelined host-memory coset LDE.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "context.hpp"
#include "host_field.hpp"

using sfntt::Status;

namespace {

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// A kernel whose bounded wait ran out raised the context's device flag.
Status device_flag(sfntt_ctx* ctx) {
  int v = 0;
  SFNTT_CU(cudaMemcpy(&v, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (v) {
    cudaMemset(ctx->err.p, 0, sizeof(int));
    return {SFNTT_TIMEOUT, "a device-side wait timed out (TMA tile never arrived)"};
  }
  return {};
}

int finish(sfntt_ctx* ctx, const Status& s) {
  if (ctx) ctx->last_error = s.ok() ? std::string() : s.msg;
  return s.code;
}

bool is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; }
uint32_t ilog2(size_t n) { uint32_t l = 0; while (((size_t)1 << l) < n) ++l; return l; }

// Internal LDE mode of M31 host calls: the canonic-coset circle LDE.
constexpr int kCircleLde = 1 << 8;

Status check_field(int field) {
  if (!sfntt::valid_field(field)) return {SFNTT_INVALID_ARGUMENT, "unknown field"};
  return {};
}

Status check_log(int field, uint32_t log_n) {
  if (sfntt::is_monty(field) && log_n > sfntt::host::monty_field(field).two_adicity) {
    const sfntt::host::MontyField& f = sfntt::host::monty_field(field);
    return {SFNTT_INVALID_SIZE, std::string(f.name) + " log_n exceeds two-adicity " + std::to_string(f.two_adicity)};
  }
  if (field == SFNTT_M31 && log_n > 30) return {SFNTT_INVALID_SIZE, "M31 log_n > 30"};  // metal_ct_gs_r4.rs:70-72
  return {};
}

Status elapsed_ns(sfntt_ctx* ctx, uint64_t* ns) {
  if (!ns) return {};
  float ms = 0.f;
  SFNTT_CU(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  *ns = (uint64_t)((double)ms * 1e6);
  return {};
}

// Copy in, transform, copy out (batch columns of 2^log_n, in place on device).
Status run_host_ntt(sfntt_ctx* ctx, int field, int variant, bool inverse, const uint32_t* in, uint32_t* out,
                    uint32_t log_n, uint32_t batch, uint64_t* ns) {
  const size_t bytes = ((size_t)batch << log_n) * sizeof(uint32_t);
  SFNTT_TRY(ctx->buf_in.reserve(bytes));
  uint32_t* d = ctx->buf_in.as<uint32_t>();
  SFNTT_CU(cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
  SFNTT_CU(cudaEventRecord(ctx->ev_start, ctx->stream));
  SFNTT_TRY(sfntt::ntt_dev(ctx, field, variant, inverse, d, log_n, batch, ctx->stream));
  SFNTT_CU(cudaEventRecord(ctx->ev_stop, ctx->stream));
  SFNTT_CU(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  SFNTT_CU(cudaStreamSynchronize(ctx->stream));
  SFNTT_TRY(device_flag(ctx));
  return elapsed_ns(ctx, ns);
}

int api_ntt_inplace(sfntt_ctx* ctx, int field, int variant, bool inverse, uint32_t* data, size_t len, uint64_t* ns) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  if (ns) *ns = 0;
  Status s = check_field(field);
  if (s.ok() && !is_pow2(len)) s = {SFNTT_INVALID_SIZE, "size " + std::to_string(len) + " is not a power of two"};
  if (s.ok() && !data) s = {SFNTT_INVALID_ARGUMENT, "null data"};
  if (s.ok() && variant == SFNTT_V1_CT_DIT_R2 && inverse && len > 1)
    s = {SFNTT_UNSUPPORTED, "V1 (CT-DIT r2) has no inverse, as in the reference (todo!())"};
  if (s.ok() && len > 1) {
    const uint32_t log_n = ilog2(len);
    s = check_log(field, log_n);
    if (s.ok()) s = run_host_ntt(ctx, field, variant, inverse, data, data, log_n, 1, ns);
  }
  return finish(ctx, s);
}

int api_ntt_gpu(sfntt_ctx* ctx, int field, int variant, bool inverse, const uint32_t* in, size_t len, uint32_t log_n,
                uint32_t batch, uint32_t* out, uint64_t* ns) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  if (ns) *ns = 0;
  Status s = check_field(field);
  if (s.ok()) s = check_log(field, log_n);
  if (s.ok() && (log_n >= 40 || len != ((size_t)batch << log_n)))
    s = {SFNTT_INVALID_SIZE, "input length " + std::to_string(len) + " != batch << log_n"};
  if (s.ok() && variant == SFNTT_V1_CT_DIT_R2 && inverse && log_n > 0)
    s = {SFNTT_UNSUPPORTED, "V1 (CT-DIT r2) has no inverse, as in the reference (todo!())"};
  if (s.ok() && len && (!in || !out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok() && len) {
    if (log_n == 0) {
      if (out != in) std::memmove(out, in, len * sizeof(uint32_t));
    } else {
      s = run_host_ntt(ctx, field, variant, inverse, in, out, log_n, batch, ns);
    }
  }
  return finish(ctx, s);
}

// Host-memory LDE: columns are processed in chunks on two buffer slots so
// that the upload of chunk i+1 and the download of chunk i-1 overlap the
// compute of chunk i.  The download (2^added_bits times the upload) is the
// bottleneck; chunks grow from an eighth of the slot, doubling, so each
// upload ends before the previous chunk's download and the download stream
// starts early and stays busy.
Status run_host_lde(sfntt_ctx* ctx, int field, const uint32_t* in, uint32_t* out, uint32_t log_n, uint32_t batch,
                    uint32_t added_bits, uint32_t shift_monty, int mode, uint64_t* ns) {
  const uint32_t log_ext = log_n + added_bits;
  const size_t n = (size_t)1 << log_n, n_ext = (size_t)1 << log_ext;
  const size_t per_col = (n + n_ext) * sizeof(uint32_t);
  const size_t target = (size_t)192 << 20;  // bytes per slot
  uint32_t chunk = (uint32_t)std::max<size_t>(1, std::min<size_t>(batch, target / per_col));
  std::vector<uint32_t> starts;  // first column of each chunk
  for (uint32_t c0 = 0, size = std::max<uint32_t>(1, chunk / 8); c0 < batch; c0 += size, size = std::min(2 * size, chunk))
    starts.push_back(c0);
  const uint32_t nchunks = (uint32_t)starts.size();
  SFNTT_TRY(ctx->buf_in.reserve(2 * (size_t)chunk * n * sizeof(uint32_t)));
  SFNTT_TRY(ctx->buf_out.reserve(2 * (size_t)chunk * n_ext * sizeof(uint32_t)));
  uint32_t* din[2] = {ctx->buf_in.as<uint32_t>(), ctx->buf_in.as<uint32_t>() + (size_t)chunk * n};
  uint32_t* dout[2] = {ctx->buf_out.as<uint32_t>(), ctx->buf_out.as<uint32_t>() + (size_t)chunk * n_ext};

  std::vector<cudaEvent_t> evs;
  auto mk = [&](cudaEvent_t* e, unsigned flags) -> Status {
    SFNTT_CU(cudaEventCreateWithFlags(e, flags));
    evs.push_back(*e);
    return {};
  };
  struct Slot { cudaEvent_t uploaded, computed, downloaded; bool used = false; } slot[2];
  std::vector<cudaEvent_t> t0(nchunks), t1(nchunks);
  Status st;
  for (int i = 0; i < 2 && st.ok(); ++i) {
    st = mk(&slot[i].uploaded, cudaEventDisableTiming);
    if (st.ok()) st = mk(&slot[i].computed, cudaEventDisableTiming);
    if (st.ok()) st = mk(&slot[i].downloaded, cudaEventDisableTiming);
  }
  for (uint32_t c = 0; c < nchunks && st.ok(); ++c) {
    st = mk(&t0[c], cudaEventDefault);
    if (st.ok()) st = mk(&t1[c], cudaEventDefault);
  }
  cudaStream_t up = ctx->copy_streams[0], down = ctx->copy_streams[1], comp = ctx->stream;
  for (uint32_t c = 0; c < nchunks && st.ok(); ++c) {
    const int k = c & 1;
    const uint32_t c0 = starts[c];
    const uint32_t cols = (c + 1 < nchunks ? starts[c + 1] : batch) - c0;
    auto step = [&]() -> Status {
      if (slot[k].used) {
        SFNTT_CU(cudaStreamWaitEvent(up, slot[k].computed, 0));     // input slot free
        SFNTT_CU(cudaStreamWaitEvent(comp, slot[k].downloaded, 0)); // output slot free
      }
      SFNTT_CU(cudaMemcpyAsync(din[k], in + (size_t)c0 * n, (size_t)cols * n * 4, cudaMemcpyHostToDevice, up));
      SFNTT_CU(cudaEventRecord(slot[k].uploaded, up));
      SFNTT_CU(cudaStreamWaitEvent(comp, slot[k].uploaded, 0));
      SFNTT_CU(cudaEventRecord(t0[c], comp));
      if (sfntt::is_monty(field))
        SFNTT_TRY(sfntt::monty_lde_dev(ctx, field, din[k], dout[k], log_n, cols, added_bits, shift_monty, mode, comp));
      else
        SFNTT_TRY(sfntt::m31_lde_dev(ctx, din[k], dout[k], log_n, cols, added_bits, comp, mode == kCircleLde));
      SFNTT_CU(cudaEventRecord(t1[c], comp));
      SFNTT_CU(cudaEventRecord(slot[k].computed, comp));
      SFNTT_CU(cudaStreamWaitEvent(down, slot[k].computed, 0));
      SFNTT_CU(cudaMemcpyAsync(out + (size_t)c0 * n_ext, dout[k], (size_t)cols * n_ext * 4, cudaMemcpyDeviceToHost,
                               down));
      SFNTT_CU(cudaEventRecord(slot[k].downloaded, down));
      slot[k].used = true;
      return {};
    };
    st = step();
  }
  cudaError_t e1 = cudaStreamSynchronize(down), e2 = cudaStreamSynchronize(comp), e3 = cudaStreamSynchronize(up);
  if (st.ok() && (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)) {
    cudaError_t e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
    st = {sfntt::map_cuda_error(e), std::string("LDE pipeline: ") + cudaGetErrorString(e)};
  }
  if (st.ok()) st = device_flag(ctx);
  if (st.ok() && ns) {
    double total = 0;
    for (uint32_t c = 0; c < nchunks; ++c) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, t0[c], t1[c]) == cudaSuccess) total += ms;
    }
    *ns = (uint64_t)(total * 1e6);
  }
  for (cudaEvent_t e : evs) cudaEventDestroy(e);
  return st;
}

int api_lde(sfntt_ctx* ctx, int field, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
            uint32_t added_bits, uint32_t shift_monty, int mode, uint32_t* out, uint64_t* ns) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  if (ns) *ns = 0;
  Status s;
  const uint32_t log_ext = log_n + added_bits;
  s = check_field(field);
  if (s.ok() && !sfntt::ext_fits(log_n, added_bits, 30)) s = {SFNTT_INVALID_SIZE, "log_n + added_bits too large"};
  if (s.ok() && sfntt::is_monty(field) && log_ext + 1 > sfntt::host::monty_field(field).two_adicity)
    s = {SFNTT_INVALID_SIZE,
         "log_n + added_bits must be <= " + std::to_string(sfntt::host::monty_field(field).two_adicity - 1)};
  if (field == SFNTT_M31 && log_ext > 30) s = {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= 30"};
  if (s.ok() && len != ((size_t)batch << log_n))  // src/lde/mod.rs:54-56
    s = {SFNTT_INVALID_SIZE, "input length " + std::to_string(len) + " != batch << log_n"};
  if (s.ok() && (field == SFNTT_M31 ? (mode != 0 && mode != kCircleLde) : (mode & ~(SFNTT_LDE_UNFUSED | SFNTT_LDE_NATURAL))))
    s = {SFNTT_INVALID_ARGUMENT, "unknown mode"};
  if (s.ok() && len && (!in || !out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok() && len) s = run_host_lde(ctx, field, in, out, log_n, batch, added_bits, shift_monty, mode, ns);
  return finish(ctx, s);
}

}  // namespace

extern "C" {

int sfntt_ctx_create(int device, sfntt_ctx** out) {
  if (!out) return SFNTT_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return SFNTT_DEVICE_NOT_FOUND;
  }
  if (device < 0 || device >= count) return SFNTT_DEVICE_NOT_FOUND;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return SFNTT_DEVICE_NOT_FOUND;
  if (prop.major != 10 || prop.minor != 0) return SFNTT_KERNEL_LOAD;  // built for sm_100a only
  DeviceGuard dg(device);
  auto* ctx = new sfntt_ctx();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  if (const char* e = std::getenv("SFNTT_NO_TMA")) ctx->no_tma = e[0] == '1';
  if (const char* e = std::getenv("SFNTT_NO_CLUSTER")) ctx->no_cluster = e[0] == '1';
  if (const char* e = std::getenv("SFNTT_HALVES")) ctx->c_halves = e[0] != '0';
  if (const char* e = std::getenv("SFNTT_LDE_PLAIN")) ctx->lde_plain = e[0] == '1';
  if (const char* e = std::getenv("SFNTT_WORKLIST_TILES")) ctx->worklist_max_tiles = std::strtoll(e, nullptr, 10);
  if (const char* e = std::getenv("SFNTT_SPLIT_C12")) ctx->split_c12 = e[0] == '1';
  bool ok = ctx->err.reserve(sizeof(int)).ok() && cudaMemset(ctx->err.p, 0, sizeof(int)) == cudaSuccess &&
            cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&ctx->copy_streams[0], cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&ctx->copy_streams[1], cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&ctx->ev_start) == cudaSuccess && cudaEventCreate(&ctx->ev_stop) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    sfntt_ctx_destroy(ctx);
    return SFNTT_GPU_EXECUTION;
  }
  *out = ctx;
  return SFNTT_OK;
}

void sfntt_ctx_destroy(sfntt_ctx* ctx) {
  if (!ctx) return;
  {
    DeviceGuard dg(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& f : ctx->monty_tw)
      for (auto& b : f) b.release();
    for (auto& m : ctx->m31_tw)
      for (auto& kv : m) kv.second.release();
    for (auto& m : ctx->m31c_tw)
      for (auto& kv : m) kv.second.release();
    for (auto& kv : ctx->lde_tabs) kv.second.release();
    ctx->buf_in.release();
    ctx->buf_out.release();
    ctx->buf_aux.release();
    ctx->buf_ext.release();
    if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
    if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
    for (cudaStream_t s : ctx->copy_streams)
      if (s) cudaStreamDestroy(s);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
}

const char* sfntt_status_string(int status) {
  switch (status) {
    case SFNTT_OK: return "ok";
    case SFNTT_INVALID_SIZE: return "invalid size";
    case SFNTT_DEVICE_NOT_FOUND: return "device not found";
    case SFNTT_ALLOC_FAILED: return "buffer allocation failed";
    case SFNTT_KERNEL_LOAD: return "kernel image not loadable on this device";
    case SFNTT_GPU_EXECUTION: return "GPU execution error";
    case SFNTT_MISMATCH: return "correctness mismatch";
    case SFNTT_UNSUPPORTED: return "unsupported operation";
    case SFNTT_TIMEOUT: return "timeout";
    case SFNTT_INVALID_ARGUMENT: return "invalid argument";
    default: return "unknown status";
  }
}

const char* sfntt_last_error(const sfntt_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int sfntt_device_info(sfntt_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return SFNTT_INVALID_ARGUMENT;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return SFNTT_DEVICE_NOT_FOUND;
  std::snprintf(buf, len, "%s, %d SMs, sm_%d%d, %.1f GiB", prop.name, prop.multiProcessorCount, prop.major,
                prop.minor, (double)prop.totalGlobalMem / (1ull << 30));
  return SFNTT_OK;
}

int sfntt_forward(sfntt_ctx* ctx, int field, int variant, uint32_t* data, size_t len, uint64_t* gpu_ns) {
  return api_ntt_inplace(ctx, field, variant, false, data, len, gpu_ns);
}

int sfntt_inverse(sfntt_ctx* ctx, int field, int variant, uint32_t* data, size_t len, uint64_t* gpu_ns) {
  return api_ntt_inplace(ctx, field, variant, true, data, len, gpu_ns);
}

int sfntt_pointwise_mul(sfntt_ctx* ctx, int field, const uint32_t* a, size_t len_a, const uint32_t* b, size_t len_b,
                        uint32_t* out, size_t len_out) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = check_field(field);
  if (s.ok() && (len_a != len_b || len_a != len_out))  // cpu_reference.rs pointwise_mul
    s = {SFNTT_INVALID_SIZE, "length mismatch " + std::to_string(len_a)};
  if (s.ok() && len_a && (!a || !b || !out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok() && len_a) {
    const size_t bytes = len_a * sizeof(uint32_t);
    auto run = [&]() -> Status {
      SFNTT_TRY(ctx->buf_in.reserve(2 * bytes));
      uint32_t* da = ctx->buf_in.as<uint32_t>();
      uint32_t* db = da + len_a;
      SFNTT_CU(cudaMemcpyAsync(da, a, bytes, cudaMemcpyHostToDevice, ctx->stream));
      SFNTT_CU(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, ctx->stream));
      SFNTT_TRY(sfntt::pointwise_mul_dev(ctx, field, da, db, da, len_a, ctx->stream));
      SFNTT_CU(cudaMemcpyAsync(out, da, bytes, cudaMemcpyDeviceToHost, ctx->stream));
      SFNTT_CU(cudaStreamSynchronize(ctx->stream));
      return {};
    };
    s = run();
  }
  return finish(ctx, s);
}

int sfntt_forward_gpu(sfntt_ctx* ctx, int field, int variant, const uint32_t* in, size_t len, uint32_t log_n,
                      uint32_t* out, uint64_t* gpu_ns) {
  return api_ntt_gpu(ctx, field, variant, false, in, len, log_n, 1, out, gpu_ns);
}

int sfntt_inverse_gpu(sfntt_ctx* ctx, int field, int variant, const uint32_t* in, size_t len, uint32_t log_n,
                      uint32_t* out, uint64_t* gpu_ns) {
  return api_ntt_gpu(ctx, field, variant, true, in, len, log_n, 1, out, gpu_ns);
}

int sfntt_forward_batch(sfntt_ctx* ctx, int field, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                        uint32_t* out, uint64_t* gpu_ns) {
  return api_ntt_gpu(ctx, field, SFNTT_BEST, false, in, len, log_n, batch, out, gpu_ns);
}

int sfntt_inverse_batch(sfntt_ctx* ctx, int field, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                        uint32_t* out, uint64_t* gpu_ns) {
  return api_ntt_gpu(ctx, field, SFNTT_BEST, true, in, len, log_n, batch, out, gpu_ns);
}

int sfntt_bb_coset_lde(sfntt_ctx* ctx, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                       uint32_t added_bits, uint32_t shift_monty, int mode, uint32_t* out, uint64_t* gpu_ns) {
  return api_lde(ctx, SFNTT_BABYBEAR, in, len, log_n, batch, added_bits, shift_monty, mode, out, gpu_ns);
}

int sfntt_coset_lde(sfntt_ctx* ctx, int field, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                    uint32_t added_bits, uint32_t shift_monty, int mode, uint32_t* out, uint64_t* gpu_ns) {
  if (field == SFNTT_M31) return finish(ctx, {SFNTT_INVALID_ARGUMENT, "coset LDE needs BabyBear or KoalaBear"});
  return api_lde(ctx, field, in, len, log_n, batch, added_bits, shift_monty, mode, out, gpu_ns);
}

int sfntt_m31_lde(sfntt_ctx* ctx, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                  uint32_t added_bits, uint32_t* out, uint64_t* gpu_ns) {
  return api_lde(ctx, SFNTT_M31, in, len, log_n, batch, added_bits, 0, SFNTT_LDE_FUSED, out, gpu_ns);
}

int sfntt_circle_lde(sfntt_ctx* ctx, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                     uint32_t added_bits, uint32_t* out, uint64_t* gpu_ns) {
  return api_lde(ctx, SFNTT_M31, in, len, log_n, batch, added_bits, 0, kCircleLde, out, gpu_ns);
}

int sfntt_circle_lde_dev(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                         uint32_t added_bits, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s;
  if (batch && (!d_in || !d_out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok()) s = sfntt::m31_lde_dev(ctx, d_in, d_out, log_n, batch, added_bits, (cudaStream_t)stream, true);
  return finish(ctx, s);
}

int sfntt_circle_ntt_dev(sfntt_ctx* ctx, int inverse, uint32_t* d_data, uint32_t log_n, uint32_t batch,
                         void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::circle_ntt_dev(ctx, inverse != 0, d_data, log_n, batch, (cudaStream_t)stream));
}

int sfntt_circle_ntt(sfntt_ctx* ctx, int inverse, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                     uint32_t* out, uint64_t* gpu_ns) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  if (gpu_ns) *gpu_ns = 0;
  Status s = check_log(SFNTT_M31, log_n);
  if (s.ok() && len != ((size_t)batch << log_n))
    s = {SFNTT_INVALID_SIZE, "input length " + std::to_string(len) + " != batch << log_n"};
  if (s.ok() && len && (!in || !out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok() && len) {
    s = [&]() -> Status {
      const size_t bytes = len * sizeof(uint32_t);
      SFNTT_TRY(ctx->buf_in.reserve(bytes));
      uint32_t* d = ctx->buf_in.as<uint32_t>();
      SFNTT_CU(cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
      SFNTT_CU(cudaEventRecord(ctx->ev_start, ctx->stream));
      SFNTT_TRY(sfntt::circle_ntt_dev(ctx, inverse != 0, d, log_n, batch, ctx->stream));
      SFNTT_CU(cudaEventRecord(ctx->ev_stop, ctx->stream));
      SFNTT_CU(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
      SFNTT_CU(cudaStreamSynchronize(ctx->stream));
      SFNTT_TRY(device_flag(ctx));
      return elapsed_ns(ctx, gpu_ns);
    }();
  }
  return finish(ctx, s);
}

int sfntt_prepare_circle(sfntt_ctx* ctx, uint32_t log_n, uint32_t added_bits) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = sfntt::ext_fits(log_n, added_bits, 30) ? check_log(SFNTT_M31, log_n + added_bits)
                                                    : Status{SFNTT_INVALID_SIZE, "log_n + added_bits too large"};
  const uint2* tw;
  for (uint32_t k : {log_n, log_n + added_bits})
    for (int inv = 0; inv < 2 && s.ok() && k > 0; ++inv) s = sfntt::m31_circle_twiddles(ctx, inv, k, ctx->stream, &tw);
  return finish(ctx, s);
}

int sfntt_prepare(sfntt_ctx* ctx, int field, uint32_t log_n) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = check_field(field);
  if (s.ok()) s = check_log(field, log_n);
  if (s.ok() && log_n > 0) {
    const uint2* tw;
    for (int inv = 0; inv < 2 && s.ok(); ++inv)
      s = sfntt::is_monty(field) ? sfntt::monty_twiddles(ctx, field, inv, log_n, ctx->stream, &tw)
                                 : sfntt::m31_twiddles(ctx, inv, log_n, ctx->stream, &tw);
  }
  return finish(ctx, s);
}

int sfntt_prepare_lde(sfntt_ctx* ctx, int field, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = check_field(field);
  if (s.ok() && !sfntt::ext_fits(log_n, added_bits, 30)) s = {SFNTT_INVALID_SIZE, "log_n + added_bits too large"};
  if (s.ok()) s = check_log(field, log_n + added_bits + (sfntt::is_monty(field) ? 1 : 0));
  if (s.ok()) {
    const uint2* tw;
    if (sfntt::is_monty(field)) {
      cudaStream_t st = ctx->stream;
      if (log_n) s = sfntt::monty_twiddles(ctx, field, true, log_n, st, &tw);
      if (s.ok()) s = sfntt::monty_twiddles(ctx, field, false, log_n + added_bits, st, &tw);
      if (s.ok() && added_bits <= 4) s = sfntt::monty_lde_table(ctx, field, log_n, added_bits, shift_monty, 0, st, &tw);
      if (s.ok() && added_bits <= 4 && log_n >= 13)
        s = sfntt::monty_lde_table(ctx, field, log_n, added_bits, shift_monty, 2, st, &tw);
      if (s.ok()) s = sfntt::monty_lde_table(ctx, field, log_n, added_bits, shift_monty, 1, st, &tw);
      // the natural-order 2x route's tables (its scratch depends on the batch and is reserved on first use)
      if (s.ok() && added_bits == 1 && log_n >= 13 && log_n <= 20) {
        const uint2* mul;
        s = sfntt::monty_natural_tables(ctx, field, log_n, 1, shift_monty, st, &mul, &tw);
      }
    } else {
      if (log_n) s = sfntt::m31_twiddles(ctx, true, log_n, ctx->stream, &tw);
      if (s.ok() && log_n) s = sfntt::m31_twiddles(ctx, false, log_n + added_bits, ctx->stream, &tw);
    }
  }
  return finish(ctx, s);
}

int sfntt_forward_dev(sfntt_ctx* ctx, int field, int variant, uint32_t* d_data, uint32_t log_n, uint32_t batch,
                      void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = check_field(field);
  if (s.ok()) s = check_log(field, log_n);
  if (s.ok() && batch && !d_data) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok()) s = sfntt::ntt_dev(ctx, field, variant, false, d_data, log_n, batch, (cudaStream_t)stream);
  return finish(ctx, s);
}

int sfntt_inverse_dev(sfntt_ctx* ctx, int field, int variant, uint32_t* d_data, uint32_t log_n, uint32_t batch,
                      void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = check_field(field);
  if (s.ok()) s = check_log(field, log_n);
  if (s.ok() && batch && !d_data) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok()) s = sfntt::ntt_dev(ctx, field, variant, true, d_data, log_n, batch, (cudaStream_t)stream);
  return finish(ctx, s);
}

int sfntt_bb_coset_lde_dev(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                           uint32_t added_bits, uint32_t shift_monty, int mode, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s;
  if (batch && (!d_in || !d_out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok())
    s = sfntt::monty_lde_dev(ctx, SFNTT_BABYBEAR, d_in, d_out, log_n, batch, added_bits, shift_monty, mode,
                             (cudaStream_t)stream);
  return finish(ctx, s);
}

int sfntt_coset_lde_dev(sfntt_ctx* ctx, int field, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n,
                        uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s;
  if (batch && (!d_in || !d_out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok())
    s = sfntt::monty_lde_dev(ctx, field, d_in, d_out, log_n, batch, added_bits, shift_monty, mode,
                             (cudaStream_t)stream);
  return finish(ctx, s);
}

int sfntt_m31_lde_dev(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                      uint32_t added_bits, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s;
  if (batch && (!d_in || !d_out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok()) s = sfntt::m31_lde_dev(ctx, d_in, d_out, log_n, batch, added_bits, (cudaStream_t)stream);
  return finish(ctx, s);
}

int sfntt_layout_dev(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch, int flags,
                     void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::layout_dev(ctx, d_in, d_out, log_n, batch, flags, (cudaStream_t)stream));
}

int sfntt_layout(sfntt_ctx* ctx, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch, int flags,
                 uint32_t* out, uint64_t* ns) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  if (ns) *ns = 0;
  Status s;
  if (log_n >= 40 || len != ((size_t)batch << log_n))
    s = {SFNTT_INVALID_SIZE, "input length " + std::to_string(len) + " != batch << log_n"};
  if (s.ok() && len && (!in || !out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok() && len) {
    s = [&]() -> Status {
      const size_t bytes = len * sizeof(uint32_t);
      SFNTT_TRY(ctx->buf_in.reserve(bytes));
      SFNTT_TRY(ctx->buf_out.reserve(bytes));
      uint32_t* din = ctx->buf_in.as<uint32_t>();
      uint32_t* dout = ctx->buf_out.as<uint32_t>();
      SFNTT_CU(cudaMemcpyAsync(din, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
      SFNTT_CU(cudaEventRecord(ctx->ev_start, ctx->stream));
      SFNTT_TRY(sfntt::layout_dev(ctx, din, dout, log_n, batch, flags, ctx->stream));
      SFNTT_CU(cudaEventRecord(ctx->ev_stop, ctx->stream));
      SFNTT_CU(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
      SFNTT_CU(cudaStreamSynchronize(ctx->stream));
      return elapsed_ns(ctx, ns);
    }();
  }
  return finish(ctx, s);
}

int sfntt_bb_to_monty_dev(sfntt_ctx* ctx, uint32_t* d, size_t len, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::monty_convert_dev(ctx, SFNTT_BABYBEAR, true, d, len, (cudaStream_t)stream));
}

int sfntt_bb_from_monty_dev(sfntt_ctx* ctx, uint32_t* d, size_t len, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::monty_convert_dev(ctx, SFNTT_BABYBEAR, false, d, len, (cudaStream_t)stream));
}

int sfntt_to_monty_dev(sfntt_ctx* ctx, int field, uint32_t* d, size_t len, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::monty_convert_dev(ctx, field, true, d, len, (cudaStream_t)stream));
}

int sfntt_from_monty_dev(sfntt_ctx* ctx, int field, uint32_t* d, size_t len, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::monty_convert_dev(ctx, field, false, d, len, (cudaStream_t)stream));
}

int sfntt_cm31_prepare(sfntt_ctx* ctx, uint32_t log_n, uint32_t batch) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  Status s = check_log(SFNTT_M31, log_n);
  if (s.ok() && log_n > 0) {
    const uint2* tw;
    for (int inv = 0; inv < 2 && s.ok(); ++inv) s = sfntt::m31_twiddles(ctx, inv, log_n, ctx->stream, &tw);
    uint32_t* scratch = nullptr;
    if (s.ok()) s = sfntt::cm31_scratch(ctx, log_n, batch, ctx->stream, &scratch);
  }
  return finish(ctx, s);
}

int sfntt_cm31_ntt_dev(sfntt_ctx* ctx, int inverse, uint32_t* d_pairs, uint32_t log_n, uint32_t batch, void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::cm31_ntt_dev(ctx, inverse != 0, d_pairs, log_n, batch, (cudaStream_t)stream));
}

int sfntt_cm31_ntt(sfntt_ctx* ctx, int inverse, const uint32_t* in, size_t len, uint32_t log_n, uint32_t batch,
                   uint32_t* out, uint64_t* gpu_ns) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  if (gpu_ns) *gpu_ns = 0;
  Status s = check_log(SFNTT_M31, log_n);
  if (s.ok() && len != ((size_t)batch << log_n) * 2)
    s = {SFNTT_INVALID_SIZE, "input length " + std::to_string(len) + " != 2 * (batch << log_n)"};
  if (s.ok() && len && (!in || !out)) s = {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (s.ok() && len) {
    s = [&]() -> Status {
      const size_t bytes = len * sizeof(uint32_t);
      SFNTT_TRY(ctx->buf_in.reserve(bytes));
      uint32_t* d = ctx->buf_in.as<uint32_t>();
      SFNTT_CU(cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
      SFNTT_CU(cudaEventRecord(ctx->ev_start, ctx->stream));
      SFNTT_TRY(sfntt::cm31_ntt_dev(ctx, inverse != 0, d, log_n, batch, ctx->stream));
      SFNTT_CU(cudaEventRecord(ctx->ev_stop, ctx->stream));
      SFNTT_CU(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
      SFNTT_CU(cudaStreamSynchronize(ctx->stream));
      SFNTT_TRY(device_flag(ctx));
      return elapsed_ns(ctx, gpu_ns);
    }();
  }
  return finish(ctx, s);
}

int sfntt_cm31_mul_dev(sfntt_ctx* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_out, size_t n,
                       void* stream) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, sfntt::cm31_mul_dev(ctx, d_a, d_b, d_out, n, (cudaStream_t)stream));
}

int sfntt_host_alloc(sfntt_ctx* ctx, size_t bytes, void** out) {
  if (!ctx || !out) return SFNTT_INVALID_ARGUMENT;
  DeviceGuard dg(ctx->device);
  cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return SFNTT_ALLOC_FAILED;
  }
  return SFNTT_OK;
}

int sfntt_host_free(sfntt_ctx* ctx, void* p) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  DeviceGuard dg(ctx->device);
  return cudaFreeHost(p) == cudaSuccess ? SFNTT_OK : SFNTT_INVALID_ARGUMENT;
}

uint64_t sfntt_launch_count(const sfntt_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

int sfntt_check_device_error(sfntt_ctx* ctx) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  return finish(ctx, device_flag(ctx));
}

int sfntt_kernel_timing(sfntt_ctx* ctx, int enable) {
  if (!ctx) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  for (auto& t : ctx->timed) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  ctx->timed.clear();
  ctx->timing = enable != 0;
  return SFNTT_OK;
}

int sfntt_kernel_times(sfntt_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  DeviceGuard dg(ctx->device);
  struct Agg { uint64_t launches = 0; double ms = 0; uint64_t bytes = 0; };
  std::map<std::string, Agg> agg;
  for (auto& t : ctx->timed) {
    if (cudaEventSynchronize(t.stop) != cudaSuccess) return finish(ctx, {SFNTT_GPU_EXECUTION, "event sync"});
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t.start, t.stop);
    Agg& a = agg[t.name];
    a.launches++;
    a.ms += ms;
    a.bytes += t.bytes;
  }
  std::string out;
  for (auto& kv : agg) {
    char line[256];
    std::snprintf(line, sizeof line, "%s %llu %.6f %llu\n", kv.first.c_str(), (unsigned long long)kv.second.launches,
                  kv.second.ms, (unsigned long long)kv.second.bytes);
    out += line;
  }
  if (out.size() + 1 > len) return finish(ctx, {SFNTT_INVALID_ARGUMENT, "buffer too small"});
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return SFNTT_OK;
}

}  // extern "C"
