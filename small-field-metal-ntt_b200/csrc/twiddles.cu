// twiddles.cu -- device-resident twiddle and multiplier tables, generated on
// the GPU once per (field, size) and cached in the context.
//
// BabyBear layer s holds g_{s+1}^j, j < 2^s, with g_k = two_adic_generator(k)
// (src/field/babybear.rs:83-97); the inverse table holds g_{s+1}^-j
// (src/ntt/babybear/twiddles.rs:13-19).  The tables for all s are nested, so
// one table up to the largest log n serves every smaller size.
//
// M31 layer l holds the x coordinate (y on the last layer) of the l-times
// doubled Coset::odds(log n) at bit-reversed positions; the inverse table holds
// their field inverses (src/ntt/m31/twiddles.rs:19-68).
//
// Entries are stored as Shoup pairs (w, floor(w 2^32 / p)) with w canonical.
#include <vector>

#include "context.hpp"
#include "field.cuh"
#include "host_field.hpp"

namespace sfntt {
namespace {

struct BbGens { uint32_t g[28]; };  // Montgomery-form generator per layer (index s: g_{s+1}^(+-1))

__global__ void bb_twiddle_kernel(uint2* tab, uint32_t count, BbGens gens) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t s = 31u - __clz(t + 1u);
  const uint32_t j = t + 1u - (1u << s);
  const uint32_t w = to_canonical(BabyBear{}, pow_var<BabyBear>(gens.g[s], j));
  tab[t] = make_uint2(w, shoup_of<BabyBear>(w));
}

struct M31Layers {
  uint32_t ix[31], iy[31], sx[31], sy[31];  // initial point and step of each doubled coset
};

__device__ __forceinline__ void cadd_dev(uint32_t ax, uint32_t ay, uint32_t bx, uint32_t by, uint32_t& rx,
                                         uint32_t& ry) {
  const uint32_t xx = mul_var<M31>(ax, bx), yy = mul_var<M31>(ay, by);
  const uint32_t xy = mul_var<M31>(ax, by), yx = mul_var<M31>(ay, bx);
  rx = sub_mod<M31>(xx, yy);
  ry = add_mod<M31>(xy, yx);
}

__global__ void m31_twiddle_kernel(uint2* tab, uint32_t log_n, M31Layers L, int inverse) {
  const uint32_t n = 1u << log_n;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n - 1u) return;
  // layer l occupies [n - n/2^l, n - n/2^(l+1)), so n - 1 - t (>= 1) has its
  // top bit at position log_n - 1 - l
  const uint32_t top = 31u - __clz(n - 1u - t);
  const uint32_t layer = log_n - 1u - top;
  const uint32_t start = n - (n >> layer);
  const uint32_t i = t - start;
  const uint32_t ls = log_n - layer;                   // coset log size at this layer
  const uint32_t k = (ls > 1u) ? (__brev(i) >> (32u - (ls - 1u))) : 0u;  // bit_reverse_idx(i, ls - 1)
  // point = initial + step * k   (double-and-add, src/field/circle.rs:63-74)
  uint32_t rx = 1u, ry = 0u, bx = L.sx[layer], by = L.sy[layer];
  uint32_t kk = k;
  while (kk) {
    if (kk & 1u) cadd_dev(rx, ry, bx, by, rx, ry);
    cadd_dev(bx, by, bx, by, bx, by);
    kk >>= 1;
  }
  cadd_dev(L.ix[layer], L.iy[layer], rx, ry, rx, ry);
  uint32_t w = (layer == log_n - 1u) ? ry : rx;
  if (inverse) w = pow_var<M31>(w, M31::P - 2u);
  tab[t] = make_uint2(w, shoup_of<M31>(w));
}

struct LdeBases { uint32_t b[16]; };

// kind 0: tab[q*n + i] = n^-1 * base_q^i ; kind 1: tab[i] = base_0^i
__global__ void bb_power_table_kernel(uint2* tab, uint32_t log_len, uint32_t count, LdeBases bases,
                                      uint32_t scale_monty) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t q = t >> log_len;
  const uint32_t i = t & ((1u << log_len) - 1u);
  uint32_t w = pow_var<BabyBear>(bases.b[q], i);
  w = mul_var<BabyBear>(w, scale_monty);
  w = to_canonical(BabyBear{}, w);
  tab[t] = make_uint2(w, shoup_of<BabyBear>(w));
}

// Four-step twist of a strided pass over layers [lo, lo + P) (span N =
// 2^(lo+P)): tab[pos] = g_N^(+-(pos mod 2^lo) * rev_P(pos >> lo)).  The
// reference's per-position DIF layers equal the plain 2^P-point sub-DIF
// followed by this factor, and its DIT layers equal the plain sub-DIT applied
// to inputs multiplied by the inverse factor.
__global__ void bb_twist_kernel(uint2* tab, uint32_t lo, uint32_t P, uint32_t g_monty) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (1u << (lo + P))) return;
  const uint32_t l = t & ((1u << lo) - 1u);
  const uint32_t e = t >> lo;
  const uint32_t re = __brev(e) >> (32u - P);
  uint32_t w = pow_var<BabyBear>(g_monty, l * re);
  w = to_canonical(BabyBear{}, w);
  tab[t] = make_uint2(w, shoup_of<BabyBear>(w));
}

Status sync_after_build(sfntt_ctx* ctx, cudaStream_t stream, const char* what) {
  SFNTT_TRY(launch_check(ctx, what));
  SFNTT_CU(cudaStreamSynchronize(stream));
  return {};
}

}  // namespace

Status bb_twiddles(sfntt_ctx* ctx, bool inverse, uint32_t log_n, cudaStream_t stream, const uint2** out) {
  const int d = inverse ? 1 : 0;
  if (log_n > host::BB_TWO_ADICITY) return {SFNTT_INVALID_SIZE, "BabyBear log_n exceeds two-adicity 27"};
  if (ctx->bb_log[d] < log_n || ctx->bb_tw[d].p == nullptr) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "twiddle table not prepared before capture"};
    const uint32_t want = log_n < 12 ? 12 : log_n;  // small sizes share one 4 Ki table
    const uint32_t count = (1u << want) - 1u;
    SFNTT_TRY(ctx->bb_tw[d].reserve((size_t)count * sizeof(uint2)));
    BbGens g{};
    for (uint32_t s = 0; s < 27; ++s) {
      uint32_t gen = host::bb_two_adic_generator(s + 1);
      if (inverse) gen = host::invmod(gen, host::BB_P);
      g.g[s] = host::bb_to_monty(gen);
    }
    bb_twiddle_kernel<<<(count + 255) / 256, 256, 0, stream>>>(ctx->bb_tw[d].as<uint2>(), count, g);
    SFNTT_TRY(sync_after_build(ctx, stream, "bb_twiddle_kernel"));
    ctx->bb_log[d] = want;
  }
  *out = ctx->bb_tw[d].as<uint2>();
  return {};
}

Status m31_twiddles(sfntt_ctx* ctx, bool inverse, uint32_t log_n, cudaStream_t stream, const uint2** out) {
  const int d = inverse ? 1 : 0;
  if (log_n == 0 || log_n > 30) return {SFNTT_INVALID_SIZE, "M31 log_n must be in [1, 30]"};
  auto it = ctx->m31_tw[d].find(log_n);
  if (it == ctx->m31_tw[d].end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "twiddle table not prepared before capture"};
    DevBuf buf;
    const uint32_t count = (1u << log_n) - 1u;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    M31Layers L{};
    // layer l: odds(log_n) doubled l times -> initial = G_{log_n+1-l}, step = G_{log_n-l}
    for (uint32_t l = 0; l < log_n; ++l) {
      const host::CPoint ini = host::subgroup_gen(log_n + 1 - l);
      const host::CPoint st = host::subgroup_gen(log_n - l);
      L.ix[l] = ini.x; L.iy[l] = ini.y; L.sx[l] = st.x; L.sy[l] = st.y;
    }
    m31_twiddle_kernel<<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), log_n, L, inverse ? 1 : 0);
    Status s = sync_after_build(ctx, stream, "m31_twiddle_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->m31_tw[d].emplace(log_n, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

Status bb_lde_table(sfntt_ctx* ctx, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty, int kind,
                    cudaStream_t stream, const uint2** out) {
  const uint32_t log_ext = log_n + added_bits;
  if (log_ext + 1 > host::BB_TWO_ADICITY) return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= 26"};
  if (kind == 0 && added_bits > 4) return {SFNTT_INVALID_ARGUMENT, "fused LDE supports added_bits <= 4"};
  const auto key = std::make_tuple(log_n, added_bits, shift_monty, kind);
  auto it = ctx->lde_tabs.find(key);
  if (it == ctx->lde_tabs.end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "LDE table not prepared before capture"};
    const uint32_t shift = shift_monty ? host::bb_from_monty(shift_monty) : host::bb_two_adic_generator(log_ext + 1);
    LdeBases B{};
    uint32_t log_len, count, scale;
    if (kind == 0) {
      // quarter q of the zero-padded DIF gets g_ext^{i * rev(q)} from its top
      // added_bits layers; fold it with the shift and n^-1 into one multiplier
      const uint32_t g_ext = host::bb_two_adic_generator(log_ext);
      for (uint32_t q = 0; q < (1u << added_bits); ++q) {
        uint32_t rq = 0;
        for (uint32_t bit = 0; bit < added_bits; ++bit) rq |= ((q >> bit) & 1u) << (added_bits - 1 - bit);
        B.b[q] = host::bb_to_monty(host::mulmod(shift, host::powmod(g_ext, rq, host::BB_P), host::BB_P));
      }
      log_len = log_n;
      count = 1u << log_ext;
      scale = host::bb_to_monty(host::invmod(1u << log_n, host::BB_P));
    } else {
      B.b[0] = host::bb_to_monty(shift);
      log_len = log_ext;
      count = 1u << log_ext;
      scale = host::bb_to_monty(1);
    }
    DevBuf buf;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    bb_power_table_kernel<<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), log_len, count, B, scale);
    Status s = sync_after_build(ctx, stream, "bb_power_table_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->lde_tabs.emplace(key, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

}  // namespace sfntt

namespace sfntt {

Status bb_twist_table(sfntt_ctx* ctx, uint32_t lo, uint32_t P, bool inverse, cudaStream_t stream, const uint2** out) {
  if (lo + P > host::BB_TWO_ADICITY || P == 0 || P > 8) return {SFNTT_INVALID_ARGUMENT, "twist span"};
  const auto key = std::make_tuple(lo, P, inverse ? 1u : 0u, 2);
  auto it = ctx->lde_tabs.find(key);
  if (it == ctx->lde_tabs.end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "twist table not prepared before capture"};
    uint32_t g = host::bb_two_adic_generator(lo + P);
    if (inverse) g = host::invmod(g, host::BB_P);
    const uint32_t count = 1u << (lo + P);
    DevBuf buf;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    bb_twist_kernel<<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), lo, P, host::bb_to_monty(g));
    Status s = sync_after_build(ctx, stream, "bb_twist_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->lde_tabs.emplace(key, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

}  // namespace sfntt
