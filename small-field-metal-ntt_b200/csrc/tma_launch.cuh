// tma_launch.cuh -- host side of the persistent TMA tile engine: tensor-map
// encoding, shape checks and dispatch to the template instantiations.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <string>

#include "context.hpp"
#include "tile_tma.cuh"

namespace sfntt {

struct TmaRequest {
  const uint32_t* in;
  uint32_t* out;
  uint64_t in_stride, out_stride;  // column strides in words
  const uint2* tw;
  uint32_t log_n, lo;
  int P;
  bool contiguous;
  uint32_t batch;
  uint32_t scale_w;  // canonical multiplier for the outputs; 0 = none
  const uint2* twist = nullptr;  // BabyBear four-step twist at the boundary
  uint32_t twist_mask = 0;
  bool twist_compact = false;    // the twist table holds Shoup companions only (TmaArgs::twist_compact)
  bool plain = false;            // BabyBear strided pass: plain sub-transform (twist by neighbours)
  // per-position twiddles staged in shared memory, one CTA per SM walking the
  // columns (BabyBear 8-layer strided or M31 contiguous passes, n >= 2^13)
  bool lstage = false;
};

// Resolved once through the runtime (no link-time dependency on libcuda).
// swizzle128: 128-byte swizzle of the box in shared memory (16-byte chunk j of
// 128-byte row r lands at chunk j ^ (r & 7); the buffer is 1024-byte aligned).
Status tensor_map_encode(CUtensorMap* map, const void* base, uint32_t rank, const cuuint64_t* dims,
                         const cuuint64_t* strides_bytes, const cuuint32_t* box, bool swizzle128 = false);

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Can a pass of this shape run on the TMA engine?  Contiguous passes over
// columns shorter than a tile need dense columns (stride n) whose batch fills
// whole tiles.
inline bool tma_pass_ok(const TmaRequest& r) {
  if (!aligned16(r.in) || !aligned16(r.out) || (r.in_stride & 3) || (r.out_stride & 3)) return false;
  const uint64_t n = 1ull << r.log_n;
  if (r.contiguous) {
    if (r.P < 5 || r.P > 14 || r.lo != 0) return false;
    if (n >= kTileWords) return true;
    return r.in_stride == n && r.out_stride == n && ((uint64_t)r.batch * n) % kTileWords == 0;
  }
  return r.P >= 1 && r.P <= 8 && r.lo >= 5 && r.lo + r.P <= r.log_n;
}

// Contiguous tiles of a P-layer pass.  Row order (c_row_perm(P) false):
// box_rows 128-byte rows per copy (a whole 2^13-word tile, or half of one for
// passes that run independent halves).  Row-permuted: a half tile per copy,
// its rows in the order [r0 r1][r3 ..][r2] of the row index r (dims: 32
// words, rows r0..r1, rows r3 and up, row r2, column), whatever box_rows says.
inline Status encode_c_map(CUtensorMap* m, const uint32_t* base, uint32_t log_n, uint64_t stride, uint32_t batch,
                           int P, uint32_t box_rows = kTileWords / 32) {
  const uint64_t n = 1ull << log_n;
  // rows per column and the column stride (dense columns shorter than a tile
  // are one long column)
  const uint64_t rows = n >= kTileWords ? n / 32 : (uint64_t)batch * n / 32;
  const uint64_t cols = n >= kTileWords ? batch : 1;
  const uint64_t col_bytes = n >= kTileWords ? stride * 4 : (uint64_t)batch * n * 4;
  if (c_row_perm(P)) {
    // half a tile per copy: 2^(tile bits - 1) words; 14-layer passes have 2^14-word tiles
    const uint32_t half_words = (P > (int)kTileBits ? (1u << P) : kTileWords) / 2;
    const cuuint64_t dims[5] = {32, 4, rows / 8, 2, cols};
    const cuuint64_t strides[4] = {128, 1024, 512, col_bytes};
    const cuuint32_t box[5] = {32, 4, half_words / 256, 2, 1};
    return tensor_map_encode(m, base, 5, dims, strides, box, kSwizzleC);
  }
  const cuuint64_t dims[3] = {32, rows, cols};
  const cuuint64_t strides[2] = {128, col_bytes};
  const cuuint32_t box[3] = {32, box_rows, 1};
  return tensor_map_encode(m, base, 3, dims, strides, box, kSwizzleC);
}

// column viewed as [hb][e][lchunk][u]: u 32 words, lchunk 2^lo/32, e 2^P (stride 2^lo), hb
inline Status encode_s_map(CUtensorMap* m, const uint32_t* base, uint32_t lo, int P, uint64_t hb_count,
                           uint64_t hb_stride, uint64_t stride, uint32_t batch) {
  const cuuint64_t dims[5] = {32, (1ull << lo) / 32, 1ull << P, hb_count, batch};
  const cuuint64_t strides[4] = {128, (1ull << lo) * 4, hb_stride * 4, stride * 4};
  const cuuint32_t box[5] = {32, 1, (cuuint32_t)(1u << P), 1, 1};
  return tensor_map_encode(m, base, 5, dims, strides, box);
}

template <class F, bool DESC, Kind KD, int P, bool PLAIN, bool TW, bool LSTAGE>
const char* tma_pass_name() {
  static const std::string nm = std::string(F::kTag) + "_" + (DESC ? "fwd" : "inv") +
                                "_tma_" + (KD == Kind::C ? "C" : "S") + std::to_string(P) + (PLAIN ? "p" : "") +
                                (TW ? "t" : "") + (LSTAGE ? "c" : "");
  return nm.c_str();
}

template <class F, bool DESC, Kind KD, int P, bool PLAIN, bool TW, bool LSTAGE = false, bool HALVES = false>
Status launch_tma_pass(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s) {
  using T = TPass<F, DESC, KD, P, PLAIN, TW, LSTAGE, HALVES>;
  const uint64_t n = 1ull << r.log_n;
  CUtensorMap min, mout;
  TmaArgs a{};
  a.tw = r.tw;
  a.log_n = r.log_n;
  a.lo = r.lo;
  a.batch = r.batch;
  a.err = ctx->err.as<int>();
  a.scale = r.scale_w ? 1u : 0u;
  a.scale_w = r.scale_w;
  a.scale_ws = (uint32_t)(((uint64_t)r.scale_w << 32) / F::P);
  a.twist = r.twist;
  a.twist_mask = r.twist_mask;
  a.twist_compact = r.twist_compact ? 1u : 0u;
  if constexpr (KD == Kind::C) {
    const uint32_t rows = HALVES ? T::HROWS : T::TWORDS / 32;
    SFNTT_TRY(encode_c_map(&min, r.in, r.log_n, r.in_stride, r.batch, P, rows));
    SFNTT_TRY(encode_c_map(&mout, r.out, r.log_n, r.out_stride, r.batch, P, rows));
    a.spans = n < T::TWORDS;
    a.log_tpc = a.spans ? 0u : r.log_n - T::CB;
    // every M31 table with n >= 2^13 carries its first-round copy from entry n on
    if constexpr (T::kRound0Copy) a.tw0 = a.spans ? nullptr : r.tw + n;
    a.ntiles = (uint32_t)(((uint64_t)r.batch * n) >> T::CB);
  } else {
    const uint64_t hb = n >> (r.lo + P);
    SFNTT_TRY(encode_s_map(&min, r.in, r.lo, P, hb, 1ull << (r.lo + P), r.in_stride, r.batch));
    SFNTT_TRY(encode_s_map(&mout, r.out, r.lo, P, hb, 1ull << (r.lo + P), r.out_stride, r.batch));
    a.ntiles = (uint32_t)(((uint64_t)r.batch * n) >> (P + 5));
  }
  constexpr int smem = T::kSmemBytes;
  auto kern = tma_pass_kernel<F, DESC, KD, P, PLAIN, TW, LSTAGE, HALVES>;
  static std::atomic<uint64_t> smem_done{0};
  SFNTT_TRY(smem_limit_once(kern, smem, ctx->device, smem_done));
  const uint32_t ctas = ctx->tma_ctas > 0 ? std::min<uint32_t>((uint32_t)ctx->tma_ctas, T::kCtasPerSm) : T::kCtasPerSm;
  const uint32_t grid = std::min<uint32_t>(a.ntiles, ctas * (uint32_t)ctx->sm_count);
  launch_begin(ctx, s);
  SFNTT_CU(launch_pdl(kern, grid, T::NT, smem, s, pdl_fits(grid), min, mout, a));
  return launch_check(ctx, tma_pass_name<F, DESC, KD, P, PLAIN, TW, LSTAGE>(), s,
                      ((uint64_t)r.batch << r.log_n) * 8u);
}

// BabyBear and KoalaBear instantiate the twist / plain variants; M31 never needs them.
#define SFNTT_TMA_C(PP)                                                                          \
  case PP:                                                                                       \
    if constexpr (F::kMontgomery) {                                                              \
      if (r.twist) {                                                                             \
        if constexpr (TPass<F, DESC, Kind::C, PP, false, true>::halves_ok())                     \
          if (ctx->c_halves) return launch_tma_pass<F, DESC, Kind::C, PP, false, true, false, true>(ctx, r, s); \
        return launch_tma_pass<F, DESC, Kind::C, PP, false, true>(ctx, r, s);                    \
      }                                                                                          \
    } else {                                                                                     \
      if (r.lstage && r.log_n >= kTileBits)                                                      \
        return launch_tma_pass<F, DESC, Kind::C, PP, false, false, true>(ctx, r, s);             \
    }                                                                                            \
    if constexpr (TPass<F, DESC, Kind::C, PP, false, false>::halves_ok())                        \
      if (ctx->c_halves) return launch_tma_pass<F, DESC, Kind::C, PP, false, false, false, true>(ctx, r, s); \
    return launch_tma_pass<F, DESC, Kind::C, PP, false, false>(ctx, r, s);
#define SFNTT_TMA_S(PP)                                                                          \
  case PP:                                                                                       \
    if constexpr (F::kMontgomery) {                                                              \
      if (r.plain && r.twist) return launch_tma_pass<F, DESC, Kind::S, PP, true, true>(ctx, r, s); \
      if (r.plain) return launch_tma_pass<F, DESC, Kind::S, PP, true, false>(ctx, r, s);         \
      if (r.twist) return launch_tma_pass<F, DESC, Kind::S, PP, false, true>(ctx, r, s);         \
      if constexpr (PP == 8) {                                                                   \
        if (r.lstage) return launch_tma_pass<F, DESC, Kind::S, PP, false, false, true>(ctx, r, s); \
      }                                                                                          \
    }                                                                                            \
    return launch_tma_pass<F, DESC, Kind::S, PP, false, false>(ctx, r, s);

template <class F, bool DESC>
Status run_tma_pass_impl(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s) {
  if (!tma_pass_ok(r)) return {SFNTT_INVALID_ARGUMENT, "pass shape not supported by the TMA engine"};
  if (!F::kMontgomery && (r.twist || r.plain)) return {SFNTT_INVALID_ARGUMENT, "M31 passes take no twist"};
  if (r.contiguous) {
    switch (r.P) {
      SFNTT_TMA_C(5) SFNTT_TMA_C(6) SFNTT_TMA_C(7) SFNTT_TMA_C(8)
      SFNTT_TMA_C(9) SFNTT_TMA_C(10) SFNTT_TMA_C(11) SFNTT_TMA_C(12) SFNTT_TMA_C(13)
      SFNTT_TMA_C(14)
      default: break;
    }
  } else {
    switch (r.P) {
      SFNTT_TMA_S(1) SFNTT_TMA_S(2) SFNTT_TMA_S(3) SFNTT_TMA_S(4)
      SFNTT_TMA_S(5) SFNTT_TMA_S(6) SFNTT_TMA_S(7) SFNTT_TMA_S(8)
      default: break;
    }
  }
  return {SFNTT_INVALID_ARGUMENT, "unsupported TMA pass size"};
}
#undef SFNTT_TMA_C
#undef SFNTT_TMA_S

Status run_tma_pass_bb_fwd(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s);
Status run_tma_pass_bb_inv(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s);
Status run_tma_pass_kb_fwd(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s);
Status run_tma_pass_kb_inv(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s);
Status run_tma_pass_m31_fwd(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s);
Status run_tma_pass_m31_inv(sfntt_ctx* ctx, const TmaRequest& r, cudaStream_t s);

inline Status run_tma_pass_field(sfntt_ctx* ctx, int field, bool desc, const TmaRequest& r, cudaStream_t s) {
  if (field == SFNTT_BABYBEAR) return desc ? run_tma_pass_bb_fwd(ctx, r, s) : run_tma_pass_bb_inv(ctx, r, s);
  if (field == SFNTT_KOALABEAR) return desc ? run_tma_pass_kb_fwd(ctx, r, s) : run_tma_pass_kb_inv(ctx, r, s);
  return desc ? run_tma_pass_m31_fwd(ctx, r, s) : run_tma_pass_m31_inv(ctx, r, s);
}

}  // namespace sfntt
