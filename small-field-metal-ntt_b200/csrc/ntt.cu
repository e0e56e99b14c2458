// ntt.cu -- transform planning (which layers go to which pass), the V1-V3
// algorithm variants of the reference shootout, and the small elementwise
// kernels (normalize, zero-pad, coset shift, pointwise product, Montgomery
// conversion).
#include <algorithm>

#include "context.hpp"
#include "field.cuh"
#include "host_field.hpp"
#include "ntt_launch.cuh"
#include "tma_launch.cuh"

namespace sfntt {

// TMA plan for layers [0, b): one contiguous pass, then strided passes of at
// most 8 layers.  Default: the strided passes take 8 layers each and the
// contiguous pass the rest, 5..cmax layers (cmax 14 for the Montgomery fields:
// b = 13, 14, 21, 22 then need one pass fewer than with at most 12; for M31
// where its contiguous passes stage their per-block twiddles, 13 elsewhere:
// reading them from L2 -- twice the tile -- the 14-layer pass was slower than
// 6 + 8 layers).  c12_first (a tuning knob, for b > 12): the
// contiguous pass takes 12 layers and the strided passes share the rest as
// evenly as possible (b = 14: 12 + 2 instead of 6 + 8).
int tma_split(uint32_t a, uint32_t b, uint32_t lo[4], uint32_t cnt[4], bool c12_first, uint32_t cmax) {
  if (a != 0) return 0;
  if (c12_first && b > 12) {
    const uint32_t s = (b - 12 + 7) / 8;
    if (s > 3) return 0;
    const uint32_t rest = b - 12;
    lo[0] = 0;
    cnt[0] = 12;
    uint32_t at = 12;
    for (uint32_t i = 1; i <= s; ++i) {
      cnt[i] = rest / s + ((i - 1) < rest % s ? 1u : 0u);
      lo[i] = at;
      at += cnt[i];
    }
    return (int)(1 + s);
  }
  const uint32_t s = b > cmax ? (b - cmax + 7) / 8 : 0;
  const uint32_t c = b - 8 * s;
  if (c < 5 || c > cmax || s > 3) return 0;
  lo[0] = 0;
  cnt[0] = c;
  for (uint32_t i = 1; i <= s; ++i) { lo[i] = c + 8 * (i - 1); cnt[i] = 8; }
  return (int)(1 + s);
}

// Split layers [a, b) into passes of at most 12 layers, as even as possible,
// the lowest pass taking the remainder.  Returns the number of passes.
static int split_layers(uint32_t a, uint32_t b, uint32_t lo[4], uint32_t cnt[4]) {
  const uint32_t total = b - a;
  const int k = (int)((total + 11) / 12);
  for (int i = 0; i < k; ++i) cnt[i] = total / k + ((uint32_t)i < total % k ? 1u : 0u);
  uint32_t s = a;
  for (int i = 0; i < k; ++i) { lo[i] = s; s += cnt[i]; }
  return k;
}

static Status get_tw(sfntt_ctx* ctx, int field, bool inverse, uint32_t log_n, cudaStream_t s, const uint2** tw) {
  if (is_monty(field)) return monty_twiddles(ctx, field, inverse, log_n, s, tw);
  return m31_twiddles(ctx, inverse, log_n, s, tw);
}

static uint32_t inv_n_canonical(int field, uint32_t log_n) {
  const uint32_t p = host::field_p(field);
  return host::invmod(host::powmod(2, log_n, p), p);
}

// Runs layers [a, b) of the 2^log_n-point network (forward: descending, CT/GS
// per field; inverse: ascending) on `batch` columns.  The first pass reads
// `in`, later passes work in place on `out`.  scale_w != 0 multiplies every
// output of the last pass by the canonical constant scale_w.
Status layers_dev(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* in, uint32_t* out, uint64_t in_stride,
                  uint64_t out_stride, uint32_t log_n, uint32_t batch, uint32_t a, uint32_t b, uint32_t scale_w,
                  const uint2* tw, cudaStream_t s, const uint2* edge_twist, uint32_t edge_mask) {
  uint32_t lo[4], cnt[4];
  if (!ctx->no_tma) {
    // M31 takes the 14-layer pass only where it stages its per-block twiddles (16 or more columns)
    const uint32_t cmax = (is_monty(field) || (log_n >= 13 && batch >= 16)) ? 14u : 13u;
    const int kt = tma_split(a, b, lo, cnt, ctx->split_c12, cmax);
    TmaRequest req[4];
    bool ok = kt > 0;
    for (int i = 0; i < kt && ok; ++i) {
      const int pi = inverse ? i : (kt - 1 - i);
      TmaRequest& r = req[i];
      r.in = (i == 0) ? in : out;
      r.out = out;
      r.in_stride = (i == 0) ? in_stride : out_stride;
      r.out_stride = out_stride;
      r.tw = tw;
      r.log_n = log_n;
      r.lo = lo[pi];
      r.P = (int)cnt[pi];
      r.contiguous = lo[pi] == 0;
      r.batch = batch;
      r.scale_w = (i == kt - 1) ? scale_w : 0u;
      // M31 contiguous passes over many columns: a tile's per-block twiddles
      // (twice its own size in L2 reads) are staged once for all its columns
      r.lstage = !is_monty(field) && r.contiguous && log_n >= 13 && batch >= 16;
      ok = tma_pass_ok(r);
    }
    if (ok && is_monty(field)) {
      // Strided passes either use per-position twiddles (self-contained) or,
      // when `plain`, run plain sub-transforms whose four-step twist is applied
      // by a neighbour: forward -> the next pass at its load, inverse -> the
      // previous pass at its store.  The edge twist of the whole range goes to
      // its first (forward) / last (inverse) pass.
      const bool plain = ctx->ntt_plain;
      for (int i = 0; i < kt; ++i) {
        const int pi = inverse ? i : (kt - 1 - i);
        req[i].plain = plain && !req[i].contiguous;
        if ((!inverse && i == 0) || (inverse && i == kt - 1)) {
          req[i].twist = edge_twist;
          req[i].twist_mask = edge_mask;
          continue;
        }
        if (!plain) continue;
        const int nb = pi + 1;  // the strided chunk just above pi
        req[i].twist_compact = twist_compact_for(lo[nb], cnt[nb]);
        SFNTT_TRY(monty_twist_table(ctx, field, lo[nb], cnt[nb], inverse, s, &req[i].twist, req[i].twist_compact));
        req[i].twist_mask = (1u << (lo[nb] + cnt[nb])) - 1u;
      }
    }
    if (ok) {
      for (int i = 0; i < kt; ++i) SFNTT_TRY(run_tma_pass_field(ctx, field, !inverse, req[i], s));
      return {};
    }
  }
  if (edge_twist) return {SFNTT_INVALID_ARGUMENT, "a boundary twist needs the TMA engine"};
  const int k = split_layers(a, b, lo, cnt);
  const uint32_t p = host::field_p(field);
  for (int i = 0; i < k; ++i) {
    const int pi = inverse ? i : (k - 1 - i);  // forward runs the high layers first
    PassRequest r{};
    r.args.in = (i == 0) ? in : out;
    r.args.out = out;
    r.args.tw = tw;
    r.args.in_stride = (i == 0) ? in_stride : out_stride;
    r.args.out_stride = out_stride;
    r.args.log_n = log_n;
    r.args.lo = lo[pi];
    r.args.scale = (i == k - 1 && scale_w) ? 1 : 0;
    r.args.scale_w = scale_w;
    r.args.scale_ws = host::shoup(scale_w, p);
    r.P = (int)cnt[pi];
    r.contiguous = (lo[pi] == 0);
    r.batch = batch;
    SFNTT_TRY(run_pass_field(ctx, field, !inverse, r, s));
  }
  return {};
}

// ---------------------------------------------------------------- V1 / V3 ---
// One radix-2 layer over all columns: the per-layer dispatch of the
// reference's V1 (src/ntt/*/metal_ct_dit_r2.rs) and, out of place, V3
// (src/ntt/*/metal_stockham_r2.rs).  Same butterflies, same twiddles.
// V1 and V2 run it in place (in == out), so in and out may alias: each thread
// reads both points of its pair before it writes them, and no two threads
// share a point.
template <class F, bool DESC>
__global__ void layer_kernel(const uint32_t* in, uint32_t* out, const uint2* __restrict__ tw,
                             uint32_t log_n, uint32_t L, uint64_t pairs, uint32_t scale, uint32_t sw, uint32_t sws) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= pairs) return;
  const uint32_t half_pairs_log = log_n - 1;
  const uint64_t col = t >> half_pairs_log;
  const uint32_t k = (uint32_t)(t & ((1ull << half_pairs_log) - 1ull));
  const uint32_t j = k & ((1u << L) - 1u);
  const uint32_t blk = k >> L;
  const uint32_t i0 = (blk << (L + 1)) + j;
  const uint32_t i1 = i0 + (1u << L);
  const uint64_t base = col << log_n;
  uint32_t a = in[base + i0], b = in[base + i1];
  uint2 w;
  if constexpr (F::kMontgomery) w = tw[((1u << L) - 1u) + j];
  else w = tw[((1u << log_n) - (1u << (log_n - L))) + blk];
  if constexpr (F::kMontgomery == DESC) {  // GS
    const uint32_t s = add_mod<F>(a, b);
    b = mul_shoup<F>(a - b + F::P, w.x, w.y);
    a = s;
  } else {  // CT, canonical in and out
    const uint32_t x = mul_shoup<F>(b, w.x, w.y);
    b = sub_mod<F>(a, x);
    a = add_mod<F>(a, x);
  }
  if (scale) {
    a = mul_shoup<F>(a, sw, sws);
    b = mul_shoup<F>(b, sw, sws);
  }
  out[base + i0] = a;
  out[base + i1] = b;
}

template <class F, bool DESC>
static Status launch_layer(sfntt_ctx* ctx, const uint32_t* in, uint32_t* out, const uint2* tw, uint32_t log_n,
                           uint32_t L, uint32_t batch, uint32_t scale_w, cudaStream_t s) {
  const uint64_t pairs = (uint64_t)batch << (log_n - 1);
  const uint32_t blocks = (uint32_t)((pairs + 255) / 256);
  launch_begin(ctx, s);
  layer_kernel<F, DESC><<<blocks, 256, 0, s>>>(in, out, tw, log_n, L, pairs, scale_w ? 1u : 0u, scale_w,
                                                 host::shoup(scale_w, F::P));
  static const std::string name = std::string(F::kTag) + "_layer";
  return launch_check(ctx, name.c_str(), s, pairs * 16u);
}

static Status layer(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* in, uint32_t* out, const uint2* tw,
                    uint32_t log_n, uint32_t L, uint32_t batch, uint32_t scale_w, cudaStream_t s) {
  return with_field(field, [&](auto fld) {
    using F = decltype(fld);
    return inverse ? launch_layer<F, false>(ctx, in, out, tw, log_n, L, batch, scale_w, s)
                   : launch_layer<F, true>(ctx, in, out, tw, log_n, L, batch, scale_w, s);
  });
}

// ----------------------------------------------------------------- driver ---
Status ntt_dev(sfntt_ctx* ctx, int field, int variant, bool inverse, uint32_t* d, uint32_t log_n, uint32_t batch,
               cudaStream_t s) {
  if (!valid_field(field)) return {SFNTT_INVALID_ARGUMENT, "unknown field"};
  if (variant < SFNTT_BEST || variant > SFNTT_V4_CT_GS_R4) return {SFNTT_INVALID_ARGUMENT, "unknown variant"};
  if (is_monty(field) && log_n > host::monty_field(field).two_adicity)
    return {SFNTT_INVALID_SIZE, "log_n > " + std::to_string(host::monty_field(field).two_adicity)};
  if (field == SFNTT_M31 && log_n > 30) return {SFNTT_INVALID_SIZE, "log_n > 30"};
  if (log_n >= 32 || ((uint64_t)batch << log_n) >= (1ull << 40)) return {SFNTT_INVALID_SIZE, "too large"};
  if (variant == SFNTT_V1_CT_DIT_R2 && inverse)
    return {SFNTT_UNSUPPORTED, "V1 (CT-DIT r2) has no inverse, as in the reference (todo!())"};
  if (log_n == 0 || batch == 0) return {};
  const uint2* tw = nullptr;
  SFNTT_TRY(get_tw(ctx, field, inverse, log_n, s, &tw));
  const uint32_t scale = inverse ? inv_n_canonical(field, log_n) : 0u;
  const uint64_t stride = 1ull << log_n;
  switch (variant) {
    case SFNTT_V1_CT_DIT_R2: {
      for (int L = (int)log_n - 1; L >= 0; --L)
        SFNTT_TRY(layer(ctx, field, false, d, d, tw, log_n, (uint32_t)L, batch, 0, s));
      return {};
    }
    case SFNTT_V2_CT_GS_R2: {
      // large strides one layer per kernel, then the low layers in one tile pass
      const uint32_t tile = std::min<uint32_t>(log_n, 12);
      if (!inverse) {
        for (int L = (int)log_n - 1; L >= (int)tile; --L)
          SFNTT_TRY(layer(ctx, field, false, d, d, tw, log_n, (uint32_t)L, batch, 0, s));
        return layers_dev(ctx, field, false, d, d, stride, stride, log_n, batch, 0, tile, 0, tw, s);
      }
      SFNTT_TRY(layers_dev(ctx, field, true, d, d, stride, stride, log_n, batch, 0, tile,
                           tile == log_n ? scale : 0u, tw, s));
      for (uint32_t L = tile; L < log_n; ++L)
        SFNTT_TRY(layer(ctx, field, true, d, d, tw, log_n, L, batch, L + 1 == log_n ? scale : 0u, s));
      return {};
    }
    case SFNTT_V3_STOCKHAM_R2: {
      // out-of-place ping-pong between the caller's buffer and a scratch buffer
      const size_t bytes = ((size_t)batch << log_n) * sizeof(uint32_t);
      if (capturing(s) && ctx->buf_aux.bytes < bytes)
        return {SFNTT_INVALID_ARGUMENT, "V3 scratch not prepared before capture"};
      SFNTT_TRY(ctx->buf_aux.reserve(bytes));
      uint32_t* bufs[2] = {d, ctx->buf_aux.as<uint32_t>()};
      int cur = 0;
      for (uint32_t i = 0; i < log_n; ++i) {
        const uint32_t L = inverse ? i : log_n - 1 - i;
        SFNTT_TRY(layer(ctx, field, inverse, bufs[cur], bufs[cur ^ 1], tw, log_n, L, batch,
                        (inverse && i + 1 == log_n) ? scale : 0u, s));
        cur ^= 1;
      }
      if (cur != 0) SFNTT_CU(cudaMemcpyAsync(d, bufs[1], bytes, cudaMemcpyDeviceToDevice, s));
      return {};
    }
    default:
      // 2^13 .. 2^16 points in at most one wave of CTAs: one cluster launch
      // instead of two passes
      if (!ctx->no_tma && cluster_ntt_fits(ctx, log_n, batch, d))
        return cluster_ntt_dev(ctx, field, inverse, d, log_n, batch, tw, scale, s);
      return layers_dev(ctx, field, inverse, d, d, stride, stride, log_n, batch, 0, log_n, scale, tw, s);
  }
}

Status ntt_dev_oop(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* in, uint32_t* out, uint64_t in_stride,
                   uint64_t out_stride, uint32_t log_n, uint32_t batch, bool normalize, cudaStream_t s) {
  if (log_n == 0 || batch == 0) return {SFNTT_INVALID_ARGUMENT, "empty transform"};
  const uint2* tw = nullptr;
  SFNTT_TRY(get_tw(ctx, field, inverse, log_n, s, &tw));
  const uint32_t scale = (inverse && normalize) ? inv_n_canonical(field, log_n) : 0u;
  return layers_dev(ctx, field, inverse, in, out, in_stride, out_stride, log_n, batch, 0, log_n, scale, tw, s);
}

// One radix-2 layer between two device buffers, for entry points that
// bring their own ping-pong partner (see noalloc.cu).
Status stockham_layer_dev(sfntt_ctx* ctx, int field, bool inverse, const uint32_t* in, uint32_t* out,
                          const uint2* tw, uint32_t log_n, uint32_t L, uint32_t batch, uint32_t scale_w,
                          cudaStream_t s) {
  return layer(ctx, field, inverse, in, out, tw, log_n, L, batch, scale_w, s);
}

uint32_t inv_n_of(int field, uint32_t log_n) { return inv_n_canonical(field, log_n); }

// Layers [a, b) of a forward / inverse network, in place; used by the M31
// blow-up whose zero-padded top layers are a plain replication.
Status ntt_layers_dev(sfntt_ctx* ctx, int field, bool inverse, uint32_t* d, uint64_t stride, uint32_t log_n,
                      uint32_t batch, uint32_t a, uint32_t b, cudaStream_t s) {
  const uint2* tw = nullptr;
  SFNTT_TRY(get_tw(ctx, field, inverse, log_n, s, &tw));
  return layers_dev(ctx, field, inverse, d, d, stride, stride, log_n, batch, a, b, 0u, tw, s);
}

// ------------------------------------------------------------ elementwise ---
namespace {

template <class F>
__global__ void scale_kernel(uint32_t* d, uint64_t n, uint32_t w, uint32_t ws) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    d[i] = mul_shoup<F>(d[i], w, ws);
}

template <class F>
__global__ void pointwise_kernel(const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = mul_var<F>(a[i], b[i]);
}

template <class F>
__global__ void monty_kernel(uint32_t* d, uint64_t n, int to) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    d[i] = to ? mul_var<F>(d[i], F::R2) : mul_var<F>(d[i], 1u);
}

// out[c * n_ext + r] = r < n ? in[c * n + r] : 0   (bb_zero_pad_batch, shaders/babybear/bb_ntt_r2.metal:379-398)
__global__ void zero_pad_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t log_n,
                                uint32_t log_ext, uint64_t total) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = i >> log_ext;
    const uint32_t r = (uint32_t)(i & ((1ull << log_ext) - 1ull));
    out[i] = (r < (1u << log_n)) ? in[(c << log_n) + r] : 0u;
  }
}

// d[c * n_ext + i] *= tab[i]   (bb_coset_shift_batch, shaders/babybear/bb_ntt_r2.metal:402-415)
template <class F>
__global__ void mul_table_kernel(uint32_t* d, uint32_t log_ext, uint64_t total, const uint2* __restrict__ tab) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 w = tab[i & ((1ull << log_ext) - 1ull)];
    d[i] = mul_shoup<F>(d[i], w.x, w.y);
  }
}

uint32_t grid_for(sfntt_ctx* ctx, uint64_t n) {
  const uint64_t want = (n + 255) / 256;
  const uint64_t cap = (uint64_t)ctx->sm_count * 16;
  return (uint32_t)std::max<uint64_t>(1, std::min(want, cap));
}

}  // namespace

Status scale_dev(sfntt_ctx* ctx, int field, uint32_t* d, uint64_t n, uint32_t w, cudaStream_t s) {
  launch_begin(ctx, s);
  with_field(field, [&](auto fld) {
    using F = decltype(fld);
    scale_kernel<F><<<grid_for(ctx, n), 256, 0, s>>>(d, n, w, host::shoup(w, F::P));
    return 0;
  });
  return launch_check(ctx, "scale", s, n * 8u);
}

Status pointwise_mul_dev(sfntt_ctx* ctx, int field, const uint32_t* a, const uint32_t* b, uint32_t* out, size_t n,
                         cudaStream_t s) {
  if (n == 0) return {};
  launch_begin(ctx, s);
  with_field(field, [&](auto fld) {
    pointwise_kernel<decltype(fld)><<<grid_for(ctx, n), 256, 0, s>>>(a, b, out, n);
    return 0;
  });
  return launch_check(ctx, "pointwise_mul", s, (uint64_t)n * 12u);
}

Status monty_convert_dev(sfntt_ctx* ctx, int field, bool to, uint32_t* d, size_t n, cudaStream_t s) {
  if (!is_monty(field)) return {SFNTT_INVALID_ARGUMENT, "Montgomery conversion needs BabyBear or KoalaBear"};
  if (n == 0) return {};
  launch_begin(ctx, s);
  with_monty(field, [&](auto fld) {
    monty_kernel<decltype(fld)><<<grid_for(ctx, n), 256, 0, s>>>(d, n, to ? 1 : 0);
    return 0;
  });
  return launch_check(ctx, to ? "to_monty" : "from_monty", s, (uint64_t)n * 8u);
}

Status zero_pad_dev(sfntt_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t log_n, uint32_t batch,
                    uint32_t added_bits, cudaStream_t s) {
  const uint64_t total = (uint64_t)batch << (log_n + added_bits);
  launch_begin(ctx, s);
  zero_pad_kernel<<<grid_for(ctx, total), 256, 0, s>>>(in, out, log_n, log_n + added_bits, total);
  return launch_check(ctx, "bb_zero_pad", s, total * 4u + ((uint64_t)batch << log_n) * 4u);
}

Status mul_table_dev(sfntt_ctx* ctx, int field, uint32_t* d, uint32_t log_ext, uint32_t batch, const uint2* tab,
                     cudaStream_t s) {
  const uint64_t total = (uint64_t)batch << log_ext;
  launch_begin(ctx, s);
  with_monty(field, [&](auto fld) {
    mul_table_kernel<decltype(fld)><<<grid_for(ctx, total), 256, 0, s>>>(d, log_ext, total, tab);
    return 0;
  });
  return launch_check(ctx, "coset_shift", s, total * 8u);
}

}  // namespace sfntt
