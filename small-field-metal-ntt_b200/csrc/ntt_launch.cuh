// ntt_launch.cuh -- host-side dispatch of one tile-engine pass to the
// matching template instantiation.  Included by the four per-(field,
// direction) instantiation files so they compile in parallel.
#pragma once
#include <string>

#include "context.hpp"
#include "ntt_pass.cuh"

namespace sfntt {

// Tile sizes: contiguous passes use 2^13-point tiles (2^LT whole groups,
// possibly spanning columns) or a single group when the batch is too ragged;
// strided passes use 8 consecutive low positions (32-byte rows) x 2^P points.
constexpr int kCTileBits = 13;
__host__ __device__ constexpr int s_lt(int P) { return P <= 11 ? 3 : 14 - P; }

struct PassRequest {
  PassArgs args;
  int P;            // layers in this pass
  bool contiguous;  // Kind::C (args.lo == 0) or Kind::S
  uint32_t batch;
};

// Kernel label for timing / profiles, e.g. "bb_fwd_pass_S10".
template <class F, bool DESC, Kind KD, int P>
const char* pass_name() {
  static const std::string n = std::string(F::kTag) + "_" + (DESC ? "fwd" : "inv") +
                               "_pass_" + (KD == Kind::C ? "C" : "S") + std::to_string(P);
  return n.c_str();
}

template <class F, bool DESC, Kind KD, int P, int LT>
Status launch_pass(sfntt_ctx* ctx, const PassArgs& a, uint32_t tiles, cudaStream_t s) {
  constexpr int CB = P + LT;
  constexpr int R = CB < 4 ? CB : 4;
  using PS = Pass<F, DESC, KD, P, LT, R>;
  constexpr int smem = PS::SMEM_WORDS * 4;
  auto kern = pass_kernel<F, DESC, KD, P, LT, R>;
  static std::atomic<uint64_t> smem_done{0};
  if (smem > 48 * 1024) SFNTT_TRY(smem_limit_once(kern, smem, ctx->device, smem_done));
  launch_begin(ctx, s);
  SFNTT_CU(launch_pdl(kern, tiles, PS::NT, smem, s, pdl_fits(tiles), a));
  const uint64_t bytes = (uint64_t)tiles << (CB + 3);  // every point read once and written once
  return launch_check(ctx, pass_name<F, DESC, KD, P>(), s, bytes);
}

inline int ctz32(uint32_t x) { return x ? __builtin_ctz(x) : 31; }

#define SFNTT_PASS_CASE(PP)                                                                         \
  case PP:                                                                                          \
    if (req.contiguous) {                                                                           \
      if (full) return launch_pass<F, DESC, Kind::C, PP, kCTileBits - PP>(ctx, a, tiles_full, s);  \
      return launch_pass<F, DESC, Kind::C, PP, 0>(ctx, a, tiles_single, s);                        \
    }                                                                                               \
    return launch_pass<F, DESC, Kind::S, PP, s_lt(PP)>(ctx, a, tiles_s, s);

template <class F, bool DESC>
Status run_pass_impl(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s) {
  PassArgs a = req.args;
  a.batch = req.batch;
  const int P = req.P;
  if (P < 1 || P > 12) return {SFNTT_INVALID_ARGUMENT, "pass must own 1..12 layers"};
  const uint32_t log_n = a.log_n;
  // Kind::C: full 2^13-point tiles need 2^13 | batch * n
  const bool full = (int)log_n + ctz32(req.batch) >= kCTileBits;
  const uint64_t total = (uint64_t)req.batch << log_n;
  const uint32_t tiles_full = (uint32_t)(total >> kCTileBits);
  const uint32_t tiles_single = (uint32_t)(total >> P);
  uint32_t tiles_s = 0;
  if (!req.contiguous) {
    const int lt = s_lt(P);
    if ((int)a.lo < lt || a.lo + P > log_n) return {SFNTT_INVALID_ARGUMENT, "strided pass geometry"};
    a.log_tiles_per_col = log_n - P - lt;
    tiles_s = req.batch << a.log_tiles_per_col;
  } else if (a.lo != 0) {
    return {SFNTT_INVALID_ARGUMENT, "contiguous pass must start at layer 0"};
  }
  switch (P) {
    SFNTT_PASS_CASE(1) SFNTT_PASS_CASE(2) SFNTT_PASS_CASE(3) SFNTT_PASS_CASE(4)
    SFNTT_PASS_CASE(5) SFNTT_PASS_CASE(6) SFNTT_PASS_CASE(7) SFNTT_PASS_CASE(8)
    SFNTT_PASS_CASE(9) SFNTT_PASS_CASE(10) SFNTT_PASS_CASE(11) SFNTT_PASS_CASE(12)
    default: break;
  }
  return {SFNTT_INVALID_ARGUMENT, "unsupported pass size"};
}

#undef SFNTT_PASS_CASE

// One entry per (field, direction); defined in ntt_pass_*.cu.
Status run_pass_bb_fwd(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s);
Status run_pass_bb_inv(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s);
Status run_pass_kb_fwd(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s);
Status run_pass_kb_inv(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s);
Status run_pass_m31_fwd(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s);
Status run_pass_m31_inv(sfntt_ctx* ctx, const PassRequest& req, cudaStream_t s);

inline Status run_pass_field(sfntt_ctx* ctx, int field, bool desc, const PassRequest& r, cudaStream_t s) {
  if (field == SFNTT_BABYBEAR) return desc ? run_pass_bb_fwd(ctx, r, s) : run_pass_bb_inv(ctx, r, s);
  if (field == SFNTT_KOALABEAR) return desc ? run_pass_kb_fwd(ctx, r, s) : run_pass_kb_inv(ctx, r, s);
  return desc ? run_pass_m31_fwd(ctx, r, s) : run_pass_m31_inv(ctx, r, s);
}

}  // namespace sfntt
