// lde.cu -- batched coset low-degree extension (src/lde/mod.rs:43-107).
//
// Reference pipeline per column: iDFT (size n) -> x n^-1 -> zero-pad to
// n_ext = n 2^b -> x shift^i -> forward DFT (size n_ext), output bit-reversed.
//
// Fused form (three kernels for n > 2^12, one below):
//   I1  inverse layers [0, lo) of every column, input -> output buffer
//   X   one tile kernel per group of 2^P points: inverse layers [lo, log_n),
//       then for each of the 2^b output blocks q: multiply by
//         M_q[i] = n^-1 * shift^i * g_ext^(i * rev_b(q)),
//       which is the normalisation, the coset shift and the top b layers of the
//       zero-padded DIF (whose upper inputs are zero, so each of those layers
//       reduces to "copy, and copy times twiddle"), then forward layers
//       [lo, log_n) of block q, stored to output rows [q n, (q+1) n)
//   F3  forward layers [0, lo) of the n_ext-point network, in place
// Every HBM byte of the input is read once and every output byte is written
// twice (X and F3), against the reference's separate iDFT / normalize+pad+
// shift / DFT passes.
//
// Unfused form ("plain"): iDFT -> normalize -> zero-pad -> coset shift -> DFT,
// one kernel (family) each, as in the reference's never-dispatched
// bb_zero_pad_batch / bb_coset_shift_batch (shaders/babybear/bb_ntt_r2.metal:379-415).
//
// M31 blow-up: iDFT (normalised) -> replicate into the 2^b blocks (the CT
// butterflies of the top b layers see a zero upper half, so they only copy)
// -> forward layers [0, log_n) of the n_ext network.
#include <algorithm>
#include <string>

#include "context.hpp"
#include "field.cuh"
#include "host_field.hpp"
#include "ntt_launch.cuh"
#include "tma_launch.cuh"

namespace sfntt {

namespace {

struct ExpandArgs {
  PassArgs inv;        // geometry + inverse twiddles (in: source, out: destination)
  const uint2* tw_fwd;
  const uint2* mul;    // M_q table, q * n + i
  uint32_t log_q;      // added bits
};

template <class F, Kind KD, int P, int LT>
struct Expand {
  static constexpr int CB = P + LT;
  static constexpr int R = CB < 4 ? CB : 4;
  using Inv = Pass<F, false, KD, P, LT, R>;
  using Fwd = Pass<F, true, KD, P, LT, R>;
  static constexpr int K = Inv::K;
  static constexpr int E = Inv::E;
  static constexpr int NT = Inv::NT;
  static constexpr int SMEM_WORDS = Inv::SMEM_WORDS;

  __device__ static __forceinline__ uint32_t pos_of(const TileGeo& g, uint32_t c, const PassArgs& a) {
    if constexpr (KD == Kind::S) return g.pos_base | Inv::map_pos(c, a.lo);
    else return g.spans ? ((g.v0 + c) & ((1u << a.log_n) - 1u)) : (g.pos_base + c);
  }

  __device__ static __forceinline__ uint32_t* out_ptr(const TileGeo& g, uint32_t c, const PassArgs& a) {
    if constexpr (KD == Kind::C) {
      if (g.spans) return a.out + (uint64_t)((g.v0 + c) >> a.log_n) * a.out_stride;
    }
    return g.out;
  }

  __device__ static void run(const ExpandArgs& ea) {
    extern __shared__ uint32_t sm[];
    const uint32_t tid = threadIdx.x;
    const PassArgs& ai = ea.inv;
    PassArgs af = ea.inv;
    af.tw = ea.tw_fwd;
    const TileGeo g = Inv::geometry(ai);
    uint32_t x[E];
    Inv::template load_global<0>(x, g, ai, tid);
    Inv::template rounds_from<0>(sm, x, g, ai, tid);  // ends in round K-1's layout, values in [0, 2p)

    using M = RM<KD, P, LT, R, K - 1>;
    using M0 = RM<KD, P, LT, R, 0>;
    const uint32_t ct = M::ctid(tid);
    const uint32_t ct0 = M0::ctid(tid);
    const uint32_t n = 1u << ai.log_n;
    const uint32_t nq = 1u << ea.log_q;
    for (uint32_t q = 0; q < nq; ++q) {
      uint32_t v[E];
      const uint2* mq = ea.mul + (uint64_t)q * n;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const uint2 w = __ldg(&mq[pos_of(g, ct | M::cm(m), ai)]);
        v[m] = mul_shoup<F>(x[m], w.x, w.y);
      }
      __syncthreads();  // the previous block's last shared-memory reads are done
      Fwd::template rounds_from<0>(sm, v, g, af, tid);  // forward starts in round K-1's layout
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const uint32_t c = ct0 | M0::cm(m);
        out_ptr(g, c, ai)[(uint64_t)q * n + pos_of(g, c, ai)] = v[m];
      }
    }
  }
};

template <class F, Kind KD, int P, int LT>
__global__ void __launch_bounds__(Expand<F, KD, P, LT>::NT) expand_kernel(ExpandArgs ea) {
  Expand<F, KD, P, LT>::run(ea);
}

template <class F, Kind KD, int P, int LT>
Status launch_expand(sfntt_ctx* ctx, const ExpandArgs& ea, uint32_t tiles, cudaStream_t s) {
  using X = Expand<F, KD, P, LT>;
  constexpr int smem = X::SMEM_WORDS * 4;
  auto kern = expand_kernel<F, KD, P, LT>;
  static std::atomic<uint64_t> smem_done{0};
  if (smem > 48 * 1024) SFNTT_TRY(smem_limit_once(kern, smem, ctx->device, smem_done));
  launch_begin(ctx, s);
  kern<<<tiles, X::NT, smem, s>>>(ea);
  // reads 2^CB points per tile, writes 2^(CB + added_bits)
  const uint64_t bytes = ((uint64_t)tiles << (X::CB + 2)) * (1u + (1u << ea.log_q));
  static const std::string name = std::string(F::kTag) + "_lde_expand_" + (KD == Kind::C ? "C" : "S") + std::to_string(P);
  return launch_check(ctx, name.c_str(), s, bytes);
}

// Expand tiles: 2^13 points for both kinds (strided: 8 low positions).
__host__ __device__ constexpr int x_lt_s(int P) { return P <= 10 ? 3 : 13 - P; }

#define SFNTT_X_CASE(PP)                                                                       \
  case PP:                                                                                     \
    if (contiguous) {                                                                          \
      if (full) return launch_expand<F, Kind::C, PP, kCTileBits - PP>(ctx, ea, tiles_full, s); \
      return launch_expand<F, Kind::C, PP, 0>(ctx, ea, tiles_single, s);                       \
    }                                                                                          \
    return launch_expand<F, Kind::S, PP, x_lt_s(PP)>(ctx, ea, tiles_s, s);

template <class F>
Status run_expand(sfntt_ctx* ctx, ExpandArgs ea, int P, uint32_t batch, cudaStream_t s) {
  const bool contiguous = ea.inv.lo == 0;
  const uint32_t log_n = ea.inv.log_n;
  ea.inv.batch = batch;
  const bool full = (int)log_n + ctz32(batch) >= kCTileBits;
  const uint64_t total = (uint64_t)batch << log_n;
  const uint32_t tiles_full = (uint32_t)(total >> kCTileBits);
  const uint32_t tiles_single = (uint32_t)(total >> P);
  uint32_t tiles_s = 0;
  if (!contiguous) {
    const int lt = x_lt_s(P);
    if ((int)ea.inv.lo < lt || ea.inv.lo + P != log_n) return {SFNTT_INVALID_ARGUMENT, "expand geometry"};
    ea.inv.log_tiles_per_col = log_n - P - lt;
    tiles_s = batch << ea.inv.log_tiles_per_col;
  }
  switch (P) {
    SFNTT_X_CASE(1) SFNTT_X_CASE(2) SFNTT_X_CASE(3) SFNTT_X_CASE(4) SFNTT_X_CASE(5) SFNTT_X_CASE(6)
    SFNTT_X_CASE(7) SFNTT_X_CASE(8) SFNTT_X_CASE(9) SFNTT_X_CASE(10) SFNTT_X_CASE(11) SFNTT_X_CASE(12)
    default: break;
  }
  return {SFNTT_INVALID_ARGUMENT, "unsupported expand size"};
}
#undef SFNTT_X_CASE

// out[c n_ext + q n + r] = out[c n_ext + r] for q in [1, 2^b)
__global__ void replicate_kernel(uint32_t* d, uint32_t log_n, uint32_t log_ext, uint64_t total) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = i >> log_n;
    const uint32_t r = (uint32_t)(i & ((1ull << log_n) - 1ull));
    const uint32_t v = d[(c << log_ext) + r];
    for (uint32_t q = 1; q < (1u << (log_ext - log_n)); ++q) d[(c << log_ext) + ((uint64_t)q << log_n) + r] = v;
  }
}

// mul: BabyBear / KoalaBear multiplier table M_q; scale_w: M31's n^-1 (canonical).
template <class F, int P, bool PLAIN, bool LSTAGE = false>
Status launch_tma_expand(sfntt_ctx* ctx, const uint32_t* src, uint64_t src_stride, uint32_t* d_out, uint32_t log_n,
                         uint32_t batch, uint32_t added_bits, const uint2* tw_inv, const uint2* tw_fwd,
                         const uint2* mul, cudaStream_t s, uint32_t scale_w = 0) {
  using X = TExpand<F, P, PLAIN, LSTAGE>;
  const uint32_t lo = log_n - P;
  const uint64_t n = 1ull << log_n, n_ext = n << added_bits;
  CUtensorMap min, mout;
  SFNTT_TRY(encode_s_map(&min, src, lo, P, 1, n, src_stride, batch));
  SFNTT_TRY(encode_s_map(&mout, d_out, lo, P, 1ull << added_bits, n, n_ext, batch));
  TmaArgs a{};
  a.tw = tw_inv;
  a.tw_fwd = tw_fwd;
  a.mul = mul;
  a.log_n = log_n;
  a.lo = lo;
  a.batch = batch;
  a.log_q = added_bits;
  a.err = ctx->err.as<int>();
  a.ntiles = (uint32_t)(((uint64_t)batch * n) >> (P + 5));
  a.scale_w = scale_w;
  a.scale_ws = (uint32_t)(((uint64_t)scale_w << 32) / F::P);
  constexpr int smem = 3 * (int)X::TBYTES + 16 + 16 * (int)X::TW_ENTRIES + 1024;
  auto kern = tma_expand_kernel<F, P, PLAIN, LSTAGE>;
  static std::atomic<uint64_t> smem_done{0};
  SFNTT_TRY(smem_limit_once(kern, smem, ctx->device, smem_done));
  const uint32_t ctas =
      ctx->tma_ctas > 0 ? std::min<uint32_t>((uint32_t)ctx->tma_ctas, (uint32_t)X::kCtasPerSm) : (uint32_t)X::kCtasPerSm;
  const uint32_t grid = std::min<uint32_t>(a.ntiles, ctas * (uint32_t)ctx->sm_count);
  launch_begin(ctx, s);
  SFNTT_CU(launch_pdl(kern, grid, X::NT, smem, s, pdl_fits(grid), min, mout, a));
  static const std::string name =
      std::string(F::kTag) + "_lde_expand_tma_S" + std::to_string(P) + (PLAIN ? "p" : "") +
      (LSTAGE ? "c" : "");
  return launch_check(ctx, name.c_str(), s, ((uint64_t)batch * n) * 4u * (1u + (1u << added_bits)));
}

// The natural-order expansion (TExpandC): src holds the inverse layers
// [12, log_n) of every column (stride n); d_out receives the 2x extension with
// the DIT layers [0, 12) of both interleaved cosets done.
template <class F>
Status launch_tma_expand_c(sfntt_ctx* ctx, const uint32_t* src, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                           const uint2* tw_inv, const uint2* tw_fwd, const uint2* mul, cudaStream_t s) {
  using X = TExpandC<F>;
  const uint64_t n = 1ull << log_n;
  CUtensorMap min, mout;
  SFNTT_TRY(encode_c_map(&min, src, log_n, n, batch, 12));
  SFNTT_TRY(encode_c_map(&mout, d_out, log_n + 1, 2 * n, batch, 12));
  TmaArgs a{};
  a.tw = tw_inv;
  a.tw_fwd = tw_fwd;
  a.mul = mul;
  a.log_n = log_n;
  a.lo = 0;
  a.batch = batch;
  a.log_q = 1;
  a.err = ctx->err.as<int>();
  a.spans = 0;
  a.log_tpc = log_n - kTileBits;
  a.ntiles = (uint32_t)(((uint64_t)batch * n) >> kTileBits);
  constexpr int smem = 4 * (int)X::TBYTES + 16 + 16 * (int)X::TW_ENTRIES + 1024;
  auto kern = tma_expand_c_kernel<F>;
  static std::atomic<uint64_t> smem_done{0};
  SFNTT_TRY(smem_limit_once(kern, smem, ctx->device, smem_done));
  const uint32_t grid = std::min<uint32_t>(a.ntiles, (uint32_t)ctx->sm_count);
  launch_begin(ctx, s);
  SFNTT_CU(launch_pdl(kern, grid, X::NT, smem, s, pdl_fits(grid), min, mout, a));
  static const std::string name = std::string(F::kTag) + "_lde_expand_tma_C12n";
  return launch_check(ctx, name.c_str(), s, ((uint64_t)batch * n) * 4u * 3u);
}

}  // namespace

namespace {

// Natural-order 2x LDE without bit-reversal passes (BabyBear / KoalaBear,
// 2^13 <= n <= 2^20): SI -- the inverse GS-DIF layers [12, log_n) on the
// natural-order input (strided pass, inverse table) into scratch; XC --
// TExpandC (inverse layers [0, 12), coset multipliers, forward DIT layers
// [0, 12) per coset, cosets interleaved); SF -- the forward CT-DIT layers
// [12, log_n) of every coset on the interleaved extended column (strided pass,
// coset twiddle table).  *done stays false (nothing launched) when the shape
// or the state does not allow it: during a capture, it needs its scratch and
// tables already resident.
template <class F>
Status monty_lde_natural2x(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                           uint32_t shift_monty, cudaStream_t s, bool* done) {
  constexpr int field = F::kId;
  *done = false;
  if (ctx->no_tma || log_n < 13 || log_n > 20 || batch == 0 || !aligned16(d_in) || !aligned16(d_out)) return {};
  const uint64_t n = 1ull << log_n;
  const size_t bytes = (size_t)(n * batch) * sizeof(uint32_t);
  if (ctx->buf_aux.bytes < bytes) {
    if (capturing(s)) return {};  // no allocation during capture: the bit-reversal route needs no scratch
    SFNTT_TRY(ctx->buf_aux.reserve(bytes));
  }
  const uint2 *itw = nullptr, *ftw = nullptr, *mul = nullptr, *ctw = nullptr;
  Status st = monty_twiddles(ctx, field, true, log_n, s, &itw);
  if (st.ok()) st = monty_twiddles(ctx, field, false, log_n, s, &ftw);
  if (st.ok()) st = monty_natural_tables(ctx, field, log_n, 1, shift_monty, s, &mul, &ctw);
  if (!st.ok()) {
    if (capturing(s)) return {};  // tables not resident before the capture: the bit-reversal route
    return st;
  }
  uint32_t* mid = ctx->buf_aux.as<uint32_t>();
  TmaRequest si{};
  si.in = d_in; si.out = mid; si.in_stride = n; si.out_stride = n; si.tw = itw;
  si.log_n = log_n; si.lo = 12; si.P = (int)log_n - 12; si.contiguous = false; si.batch = batch;
  // a chunk's twiddles are staged once for its `batch` tiles (one per column)
  si.lstage = batch >= 8;
  SFNTT_TRY(run_tma_pass_field(ctx, field, true, si, s));
  SFNTT_TRY(launch_tma_expand_c<F>(ctx, mid, d_out, log_n, batch, itw, ftw, mul, s));
  TmaRequest sf{};
  sf.in = d_out; sf.out = d_out; sf.in_stride = 2 * n; sf.out_stride = 2 * n; sf.tw = ctw;
  sf.log_n = log_n + 1; sf.lo = 13; sf.P = (int)log_n - 12; sf.contiguous = false; sf.batch = batch;
  sf.lstage = batch >= 8;
  SFNTT_TRY(run_tma_pass_field(ctx, field, false, sf, s));
  *done = true;
  return {};
}

// Input columns at stride in_stride (n, or n_ext when they already sit in the
// output columns); output bit-reversed rows.  F is BabyBear or KoalaBear.
template <class F>
Status monty_lde_rows(sfntt_ctx* ctx, const uint32_t* d_in, uint64_t in_stride, uint32_t* d_out, uint32_t log_n,
                      uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode, cudaStream_t s) {
  constexpr int field = F::kId;
  const host::MontyField& mf = host::monty_field(field);
  if (!ext_fits(log_n, added_bits, mf.two_adicity - 1))
    return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= " + std::to_string(mf.two_adicity - 1)};
  const uint32_t log_ext = log_n + added_bits;
  if (batch == 0) return {};
  const uint64_t n = 1ull << log_n, n_ext = 1ull << log_ext;
  const bool fused = mode == SFNTT_LDE_FUSED && log_n >= 1 && log_n <= 24 && added_bits <= 4;
  if (fused) {
    const uint2 *tw_inv = nullptr, *tw_fwd = nullptr, *mul = nullptr;
    SFNTT_TRY(monty_twiddles(ctx, field, true, log_n, s, &tw_inv));
    SFNTT_TRY(monty_twiddles(ctx, field, false, log_ext, s, &tw_fwd));
    const bool tma_ok = !ctx->no_tma && log_n >= 13 && aligned16(d_in) && aligned16(d_out);
    // the TMA expansion reads its multipliers in tile order (kind 2)
    SFNTT_TRY(monty_lde_table(ctx, field, log_n, added_bits, shift_monty, tma_ok ? 2 : 0, s, &mul));
    if (tma_ok) {
      // I1: inverse layers [0, lo) into the output buffer, ending with the
      // four-step pre-twist of the expand's sub-iDFT; X: the persistent TMA
      // expand on 8-layer strided tiles (plain sub-transforms); F3: forward
      // layers [0, lo) of the n_ext network, starting with the expand's
      // post-twist (the same for every output block, so indexed mod n).
      const uint32_t lo = log_n - 8;
      const uint2 *tw_i = nullptr, *tw_f = nullptr;
      const bool plain = ctx->lde_plain;
      if (plain) {
        SFNTT_TRY(monty_twist_table(ctx, field, lo, 8, true, s, &tw_i));
        SFNTT_TRY(monty_twist_table(ctx, field, lo, 8, false, s, &tw_f));
      }
      const uint32_t mask = (uint32_t)(n - 1);
      SFNTT_TRY(layers_dev(ctx, field, true, d_in, d_out, in_stride, n_ext, log_n, batch, 0, lo, 0u, tw_inv, s, tw_i,
                           mask));
      if (plain)
        SFNTT_TRY((launch_tma_expand<F, 8, true>(ctx, d_out, n_ext, d_out, log_n, batch, added_bits, tw_inv, tw_fwd,
                                                 mul, s)));
      else if (batch >= 16)  // the chunk's twiddles are reused across >= 16 columns
        SFNTT_TRY((launch_tma_expand<F, 8, false, true>(ctx, d_out, n_ext, d_out, log_n, batch, added_bits, tw_inv,
                                                        tw_fwd, mul, s)));
      else
        SFNTT_TRY((launch_tma_expand<F, 8, false>(ctx, d_out, n_ext, d_out, log_n, batch, added_bits, tw_inv, tw_fwd,
                                                  mul, s)));
      SFNTT_TRY(layers_dev(ctx, field, false, d_out, d_out, n_ext, n_ext, log_ext, batch, 0, lo, 0u, tw_fwd, s, tw_f,
                           mask));
      return {};
    }
    const uint32_t lo = log_n <= 12 ? 0u : (log_n + 1) / 2;
    const int P = (int)(log_n - lo);
    if (lo > 0) {  // I1: inverse layers [0, lo) into the output buffer
      PassRequest r{};
      r.args.in = d_in; r.args.out = d_out; r.args.tw = tw_inv;
      r.args.in_stride = in_stride; r.args.out_stride = n_ext;
      r.args.log_n = log_n; r.args.lo = 0; r.P = (int)lo; r.contiguous = true; r.batch = batch;
      SFNTT_TRY(run_pass_field(ctx, field, false, r, s));
    }
    ExpandArgs ea{};
    ea.inv.in = lo > 0 ? d_out : d_in;
    ea.inv.out = d_out;
    ea.inv.tw = tw_inv;
    ea.inv.in_stride = lo > 0 ? n_ext : in_stride;
    ea.inv.out_stride = n_ext;
    ea.inv.log_n = log_n;
    ea.inv.lo = lo;
    ea.tw_fwd = tw_fwd;
    ea.mul = mul;
    ea.log_q = added_bits;
    SFNTT_TRY(run_expand<F>(ctx, ea, P, batch, s));
    if (lo > 0) {  // F3: forward layers [0, lo) of the n_ext network
      PassRequest r{};
      r.args.in = d_out; r.args.out = d_out; r.args.tw = tw_fwd;
      r.args.in_stride = n_ext; r.args.out_stride = n_ext;
      r.args.log_n = log_ext; r.args.lo = 0; r.P = (int)lo; r.contiguous = true; r.batch = batch;
      SFNTT_TRY(run_pass_field(ctx, field, true, r, s));
    }
    return {};
  }
  // unfused: iDFT (no normalize) into scratch, normalize, zero-pad, shift, DFT
  const size_t bytes = (size_t)(n * batch) * sizeof(uint32_t);
  if (capturing(s) && ctx->buf_aux.bytes < bytes) return {SFNTT_INVALID_ARGUMENT, "LDE scratch not prepared"};
  SFNTT_TRY(ctx->buf_aux.reserve(bytes));
  uint32_t* coeffs = ctx->buf_aux.as<uint32_t>();
  if (log_n > 0) {
    SFNTT_TRY(ntt_dev_oop(ctx, field, true, d_in, coeffs, in_stride, n, log_n, batch, false, s));
    SFNTT_TRY(scale_dev(ctx, field, coeffs, n * batch, host::invmod((uint32_t)n, mf.p), s));
  } else {
    SFNTT_CU(cudaMemcpy2DAsync(coeffs, 4, d_in, in_stride * 4, 4, batch, cudaMemcpyDeviceToDevice, s));
  }
  SFNTT_TRY(zero_pad_dev(ctx, coeffs, d_out, log_n, batch, added_bits, s));
  const uint2* shift_tab = nullptr;
  SFNTT_TRY(monty_lde_table(ctx, field, log_n, added_bits, shift_monty, 1, s, &shift_tab));
  SFNTT_TRY(mul_table_dev(ctx, field, d_out, log_ext, batch, shift_tab, s));
  if (log_ext > 0) SFNTT_TRY(ntt_dev(ctx, field, SFNTT_V4_CT_GS_R4, false, d_out, log_ext, batch, s));
  return {};
}

}  // namespace

// The reference's convention: input evaluations and output rows in
// bit-reversed order.  SFNTT_LDE_NATURAL (Plonky3's coset_lde_batch):
// natural-order input and output; the input columns are bit-reversed into the
// output columns, the LDE runs there in place, and the output columns are
// bit-reversed in place.
Status monty_lde_dev(sfntt_ctx* ctx, int field, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n,
                     uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode, cudaStream_t s) {
  if (!is_monty(field)) return {SFNTT_INVALID_ARGUMENT, "coset LDE needs BabyBear or KoalaBear"};
  if (mode & ~(SFNTT_LDE_UNFUSED | SFNTT_LDE_NATURAL)) return {SFNTT_INVALID_ARGUMENT, "unknown LDE mode"};
  const int form = mode & SFNTT_LDE_UNFUSED;
  return with_monty(field, [&](auto fld) -> Status {
    using F = decltype(fld);
    if (!(mode & SFNTT_LDE_NATURAL))
      return monty_lde_rows<F>(ctx, d_in, 1ull << log_n, d_out, log_n, batch, added_bits, shift_monty, form, s);
    const host::MontyField& mf = host::monty_field(field);
    if (!ext_fits(log_n, added_bits, mf.two_adicity - 1))
      return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= " + std::to_string(mf.two_adicity - 1)};
    const uint32_t log_ext = log_n + added_bits;
    if (batch == 0) return {};
    if (form == SFNTT_LDE_FUSED && added_bits == 1) {
      bool done = false;
      SFNTT_TRY(monty_lde_natural2x<F>(ctx, d_in, d_out, log_n, batch, shift_monty, s, &done));
      if (done) return {};
    }
    const uint64_t n_ext = 1ull << log_ext;
    SFNTT_TRY(bitrev_cols_dev(ctx, d_in, 1ull << log_n, d_out, n_ext, log_n, batch, s));
    SFNTT_TRY(monty_lde_rows<F>(ctx, d_out, n_ext, d_out, log_n, batch, added_bits, shift_monty, form, s));
    return bitrev_cols_dev(ctx, d_out, n_ext, d_out, n_ext, log_ext, batch, s);
  });
}

Status m31_lde_dev(sfntt_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, uint32_t batch,
                   uint32_t added_bits, cudaStream_t s, bool canonic) {
  if (!ext_fits(log_n, added_bits, 30)) return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= 30"};
  const uint32_t log_ext = log_n + added_bits;
  if (batch == 0) return {};
  const uint64_t n = 1ull << log_n, n_ext = 1ull << log_ext;
  auto twiddles = [&](bool inverse, uint32_t k, const uint2** tw) {
    return canonic ? m31_circle_twiddles(ctx, inverse, k, s, tw) : m31_twiddles(ctx, inverse, k, s, tw);
  };
  const uint2 *tw_inv = nullptr, *tw_fwd = nullptr;
  if (log_n > 0) {  // log n = 0: the copy and the replication need no twiddles
    SFNTT_TRY(twiddles(true, log_n, &tw_inv));
    SFNTT_TRY(twiddles(false, log_ext, &tw_fwd));
  }
  if (!ctx->no_tma && log_n >= 13 && added_bits <= 4 && aligned16(d_in) && aligned16(d_out)) {
    // I1: inverse layers [0, lo) into the output columns; X: inverse layers
    // [lo, log_n), n^-1, and per output block forward layers [lo, log_n) of
    // the extended network; F3: forward layers [0, lo) of the extended network.
    const uint32_t lo = log_n - 8;
    SFNTT_TRY(layers_dev(ctx, SFNTT_M31, true, d_in, d_out, n, n_ext, log_n, batch, 0, lo, 0u, tw_inv, s));
    SFNTT_TRY((launch_tma_expand<M31, 8, false>(ctx, d_out, n_ext, d_out, log_n, batch, added_bits, tw_inv, tw_fwd,
                                                nullptr, s, inv_n_of(SFNTT_M31, log_n))));
    return layers_dev(ctx, SFNTT_M31, false, d_out, d_out, n_ext, n_ext, log_ext, batch, 0, lo, 0u, tw_fwd, s);
  }
  if (log_n > 0) {
    SFNTT_TRY(layers_dev(ctx, SFNTT_M31, true, d_in, d_out, n, n_ext, log_n, batch, 0, log_n, inv_n_of(SFNTT_M31, log_n),
                         tw_inv, s));
  } else {
    SFNTT_CU(cudaMemcpy2DAsync(d_out, n_ext * 4, d_in, 4, 4, batch, cudaMemcpyDeviceToDevice, s));
  }
  if (added_bits > 0) {
    const uint64_t total = (uint64_t)batch << log_n;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((total + 255) / 256, (uint64_t)ctx->sm_count * 16);
    launch_begin(ctx, s);
    replicate_kernel<<<grid ? grid : 1, 256, 0, s>>>(d_out, log_n, log_ext, total);
    SFNTT_TRY(launch_check(ctx, "m31_replicate", s, total * 4u * (1u + (1u << added_bits) - 1u)));
  }
  if (log_n > 0)
    SFNTT_TRY(layers_dev(ctx, SFNTT_M31, false, d_out, d_out, n_ext, n_ext, log_ext, batch, 0, log_n, 0u, tw_fwd, s));
  return {};
}

Status circle_ntt_dev(sfntt_ctx* ctx, bool inverse, uint32_t* d, uint32_t log_n, uint32_t batch, cudaStream_t s) {
  if (log_n > 30) return {SFNTT_INVALID_SIZE, "M31 log_n > 30"};
  if (log_n == 0 || batch == 0) return {};
  if (!d) return {SFNTT_INVALID_ARGUMENT, "null buffer"};
  const uint2* tw = nullptr;
  SFNTT_TRY(m31_circle_twiddles(ctx, inverse, log_n, s, &tw));
  const uint64_t n = 1ull << log_n;
  return layers_dev(ctx, SFNTT_M31, inverse, d, d, n, n, log_n, batch, 0, log_n,
                    inverse ? inv_n_of(SFNTT_M31, log_n) : 0u, tw, s);
}

}  // namespace sfntt
