// twiddles.cu -- device-resident twiddle and multiplier tables, generated on
// the GPU once per (field, size) and cached in the context.
//
// BabyBear layer s holds g_{s+1}^j, j < 2^s, with g_k = two_adic_generator(k)
// (src/field/babybear.rs:83-97); the inverse table holds g_{s+1}^-j
// (src/ntt/babybear/twiddles.rs:13-19).  The tables for all s are nested, so
// one table up to the largest log n serves every smaller size.  KoalaBear
// tables are built the same way from its own two_adic_generator.
//
// M31 layer l holds the x coordinate (y on the last layer) of the l-times
// doubled Coset::odds(log n) at bit-reversed positions; the inverse table holds
// their field inverses (src/ntt/m31/twiddles.rs:19-68).
//
// Entries are stored as Shoup pairs (w, floor(w 2^32 / p)) with w canonical.
#include <string>
#include <vector>

#include "context.hpp"
#include "field.cuh"
#include "host_field.hpp"

namespace sfntt {
namespace {

struct MontyGens { uint32_t g[28]; };  // Montgomery-form generator per layer (index s: g_{s+1}^(+-1))

template <class F>
__global__ void monty_twiddle_kernel(uint2* tab, uint32_t count, MontyGens gens) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t s = 31u - __clz(t + 1u);
  const uint32_t j = t + 1u - (1u << s);
  const uint32_t w = to_canonical(F{}, pow_var<F>(gens.g[s], j));
  tab[t] = make_uint2(w, shoup_of<F>(w));
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

// Canonic-coset circle FFT (Stwo-style; not in the reference): layer L,
// block b holds y (L = 0) or x (L >= 1) of m G_{2^(k+1)} with
// m = (1 + 4 bitrev_{k-1-L}(b)) 2^max(L-1, 0), i.e. of the half-coset point
// h_i = (1 + 4i) G_{2^(k+1)} doubled L - 1 times.
__global__ void circle_twiddle_kernel(uint2* tab, uint32_t log_n, uint32_t gx, uint32_t gy, int inverse) {
  const uint32_t n = 1u << log_n;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n - 1u) return;
  const uint32_t top = 31u - __clz(n - 1u - t);
  const uint32_t layer = log_n - 1u - top;
  const uint32_t b = t - (n - (n >> layer));
  const uint32_t bits = log_n - 1u - layer;
  const uint32_t i = bits ? (__brev(b) >> (32u - bits)) : 0u;
  const uint64_t mask = (2ull << log_n) - 1ull;  // m mod 2^(k+1)
  uint64_t m = ((uint64_t)(1u + 4u * i) << (layer ? layer - 1u : 0u)) & mask;
  uint32_t rx = 1u, ry = 0u, bx = gx, by = gy;
  while (m) {
    if (m & 1u) cadd_dev(rx, ry, bx, by, rx, ry);
    cadd_dev(bx, by, bx, by, bx, by);
    m >>= 1;
  }
  uint32_t w = layer == 0u ? ry : rx;
  if (inverse) w = pow_var<M31>(w, M31::P - 2u);
  tab[t] = make_uint2(w, shoup_of<M31>(w));
}

// M31 tables with n >= 2^13 carry, from entry n on, a copy of layers 0..3
// in the order the first round of a contiguous 2^13-word tile reads them:
// thread t owns tile words 16 t .. 16 t + 15, so its layer-L twiddles are the
// 2^(3-L) consecutive entries from ((tile base + 16 t) >> (L+1)).  Per tile,
// 7680 pairs: layer 0 as [pair k < 4][t] 128-bit words, layer 1 [k < 2][t],
// layer 2 [t], layer 3 [t] single pairs, so each load of the round is one
// contiguous run across the CTA.
constexpr uint32_t kRound0Pairs = 7680;

__global__ void round0_permute_kernel(uint2* tab, uint32_t log_n) {
  const uint32_t n = 1u << log_n;
  const uint32_t total = (n >> 13) * kRound0Pairs;
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const uint32_t T = idx / kRound0Pairs, w = idx - T * kRound0Pairs;
  uint32_t L, t, o;
  if (w < 4096) { L = 0; t = (w & 1023u) >> 1; o = 2 * (w >> 10) + (w & 1u); }
  else if (w < 6144) { L = 1; t = ((w - 4096) & 1023u) >> 1; o = 2 * ((w - 4096) >> 10) + (w & 1u); }
  else if (w < 7168) { L = 2; t = (w - 6144) >> 1; o = w & 1u; }
  else { L = 3; t = w - 7168; o = 0; }
  const uint32_t src = (n - (n >> L)) + ((T * 8192u + 16u * t) >> (L + 1)) + o;
  tab[n + idx] = tab[src];
}

struct LdeBases { uint32_t b[16]; };

// kind 0: tab[q*n + i] = n^-1 * base_q^i ; kind 1: tab[i] = base_0^i ;
// kind 2 (tile_lo = log n - 8 > 0): kind 0's entries in the order of the TMA
// expansion's strided tiles -- entry q*n + (chunk 2^13 + e 32 + u) holds
// position i = chunk 32 + u + e 2^tile_lo -- so a thread's multipliers sit at
// compile-time offsets from one base.
template <class F>
__global__ void power_table_kernel(uint2* tab, uint32_t log_len, uint32_t count, LdeBases bases,
                                   uint32_t scale_monty, uint32_t tile_lo) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t q = t >> log_len;
  uint32_t i = t & ((1u << log_len) - 1u);
  if (tile_lo) i = ((i >> 13) << 5) + (i & 31u) + (((i >> 5) & 255u) << tile_lo);
  uint32_t w = pow_var<F>(bases.b[q], i);
  w = mul_var<F>(w, scale_monty);
  w = to_canonical(F{}, w);
  tab[t] = make_uint2(w, shoup_of<F>(w));
}

// Four-step twist of a strided pass over layers [lo, lo + P) (span N =
// 2^(lo+P)): tab[pos] = g_N^(+-(pos mod 2^lo) * rev_P(pos >> lo)).  The
// reference's per-position DIF layers equal the plain 2^P-point sub-DIF
// followed by this factor, and its DIT layers equal the plain sub-DIT applied
// to inputs multiplied by the inverse factor.
template <class F>
__global__ void twist_kernel(uint2* tab, uint32_t lo, uint32_t P, uint32_t g_monty, int compact) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (1u << (lo + P))) return;
  const uint32_t l = t & ((1u << lo) - 1u);
  const uint32_t e = t >> lo;
  const uint32_t re = __brev(e) >> (32u - P);
  uint32_t w = pow_var<F>(g_monty, l * re);
  w = to_canonical(F{}, w);
  if (compact) reinterpret_cast<uint32_t*>(tab)[t] = shoup_of<F>(w);  // w = mulhi(w', p) + 1
  else tab[t] = make_uint2(w, shoup_of<F>(w));
}

// Natural-order LDE multipliers M_r[i] = n^-1 base_r^rev(i), stored in the
// order a contiguous 2^13-word tile's 512 threads read them in the first
// round (thread t's slot m is word 16 t + m of the tile): entry m * 512 + t
// of each tile, so one slot's load is a coalesced run across the CTA.
template <class F>
__global__ void natural_mul_kernel(uint2* tab, uint32_t log_n, uint32_t count, LdeBases bases,
                                   uint32_t scale_monty) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= count) return;
  const uint32_t r = o >> log_n;
  const uint32_t local = o & ((1u << log_n) - 1u);
  const uint32_t w = local & 8191u;
  const uint32_t i = (local & ~8191u) | ((w & 511u) << 4) | (w >> 9);
  uint32_t v = pow_var<F>(bases.b[r], __brev(i) >> (32u - log_n));
  v = to_canonical(F{}, mul_var<F>(v, scale_monty));
  tab[o] = make_uint2(v, shoup_of<F>(v));
}

// Forward twiddles of the n-point DIT, laid out as an extended table for
// columns that interleave 2^b cosets (word p 2^b + r): layer L (offset
// 2^L - 1) holds tab[L][j] = g_{L+1-b}^(j >> b) for L >= b, so the strided
// pass's per-position lookup tab[L][pos mod 2^L] of the extended column finds
// layer L - b's twiddle of coset position pos >> b.
template <class F>
__global__ void coset_twiddle_kernel(uint2* tab, uint32_t count, uint32_t b, MontyGens gens) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t L = 31u - __clz(t + 1u);
  const uint32_t j = t + 1u - (1u << L);
  uint32_t w = 0;
  if (L >= b) w = to_canonical(F{}, pow_var<F>(gens.g[L - b], j >> b));
  tab[t] = make_uint2(w, shoup_of<F>(w));
}

size_t m31_table_bytes(uint32_t log_n) {
  const size_t n = (size_t)1 << log_n;
  return (log_n >= 13 ? n + (n >> 13) * kRound0Pairs : n - 1) * sizeof(uint2);
}

void add_round0_copy(uint2* tab, uint32_t log_n, cudaStream_t stream) {
  if (log_n < 13) return;
  const uint32_t total = ((1u << log_n) >> 13) * kRound0Pairs;
  round0_permute_kernel<<<(total + 255) / 256, 256, 0, stream>>>(tab, log_n);
}

Status sync_after_build(sfntt_ctx* ctx, cudaStream_t stream, const char* what) {
  SFNTT_TRY(launch_check(ctx, what));
  SFNTT_CU(cudaStreamSynchronize(stream));
  return {};
}

}  // namespace

Status monty_twiddles(sfntt_ctx* ctx, int field, bool inverse, uint32_t log_n, cudaStream_t stream,
                      const uint2** out) {
  const host::MontyField& f = host::monty_field(field);
  const int d = inverse ? 1 : 0, k = monty_slot(field);
  if (log_n > f.two_adicity)
    return {SFNTT_INVALID_SIZE, std::string(f.name) + " log_n exceeds two-adicity " + std::to_string(f.two_adicity)};
  DevBuf& buf = ctx->monty_tw[k][d];
  if (ctx->monty_log[k][d] < log_n || buf.p == nullptr) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "twiddle table not prepared before capture"};
    const uint32_t want = log_n < 12 ? 12 : log_n;  // small sizes share one 4 Ki table
    const uint32_t count = (1u << want) - 1u;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    MontyGens g{};
    for (uint32_t s = 0; s < f.two_adicity; ++s) {
      uint32_t gen = host::two_adic_generator(f, s + 1);
      if (inverse) gen = host::invmod(gen, f.p);
      g.g[s] = host::to_monty(f, gen);
    }
    with_monty(field, [&](auto fld) {
      using F = decltype(fld);
      monty_twiddle_kernel<F><<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), count, g);
      return 0;
    });
    SFNTT_TRY(sync_after_build(ctx, stream, "monty_twiddle_kernel"));
    ctx->monty_log[k][d] = want;
  }
  *out = buf.as<uint2>();
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
    SFNTT_TRY(buf.reserve(m31_table_bytes(log_n)));
    M31Layers L{};
    // layer l: odds(log_n) doubled l times -> initial = G_{log_n+1-l}, step = G_{log_n-l}
    for (uint32_t l = 0; l < log_n; ++l) {
      const host::CPoint ini = host::subgroup_gen(log_n + 1 - l);
      const host::CPoint st = host::subgroup_gen(log_n - l);
      L.ix[l] = ini.x; L.iy[l] = ini.y; L.sx[l] = st.x; L.sy[l] = st.y;
    }
    m31_twiddle_kernel<<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), log_n, L, inverse ? 1 : 0);
    add_round0_copy(buf.as<uint2>(), log_n, stream);
    Status s = sync_after_build(ctx, stream, "m31_twiddle_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->m31_tw[d].emplace(log_n, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

Status m31_circle_twiddles(sfntt_ctx* ctx, bool inverse, uint32_t log_n, cudaStream_t stream, const uint2** out) {
  const int d = inverse ? 1 : 0;
  if (log_n == 0 || log_n > 30) return {SFNTT_INVALID_SIZE, "M31 log_n must be in [1, 30]"};
  auto it = ctx->m31c_tw[d].find(log_n);
  if (it == ctx->m31c_tw[d].end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "twiddle table not prepared before capture"};
    DevBuf buf;
    const uint32_t count = (1u << log_n) - 1u;
    SFNTT_TRY(buf.reserve(m31_table_bytes(log_n)));
    const host::CPoint g = host::subgroup_gen(log_n + 1);
    circle_twiddle_kernel<<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), log_n, g.x, g.y, inverse ? 1 : 0);
    add_round0_copy(buf.as<uint2>(), log_n, stream);
    Status s = sync_after_build(ctx, stream, "circle_twiddle_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->m31c_tw[d].emplace(log_n, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

Status monty_natural_tables(sfntt_ctx* ctx, int field, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty,
                            cudaStream_t stream, const uint2** mul, const uint2** coset_tw) {
  const host::MontyField& f = host::monty_field(field);
  if (!ext_fits(log_n, added_bits, f.two_adicity - 1) || added_bits > 4 || log_n < 13)
    return {SFNTT_INVALID_SIZE, "natural-order LDE tables: 2^13 <= n and log_n + added_bits within the field"};
  const uint32_t log_ext = log_n + added_bits;
  const auto kmul = std::make_tuple(monty_slot(field), log_n, added_bits, shift_monty, 3);
  const auto ktw = std::make_tuple(monty_slot(field), log_n, added_bits, 0u, 4);
  auto im = ctx->lde_tabs.find(kmul);
  if (im == ctx->lde_tabs.end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "LDE table not prepared before capture"};
    // coset r of the natural-order output: M_r[p] = n^-1 (shift g_ext^r)^rev(p)
    const uint32_t shift = shift_monty ? host::from_monty(f, shift_monty) : host::two_adic_generator(f, log_ext + 1);
    const uint32_t g_ext = host::two_adic_generator(f, log_ext);
    LdeBases B{};
    for (uint32_t r = 0; r < (1u << added_bits); ++r)
      B.b[r] = host::to_monty(f, host::mulmod(shift, host::powmod(g_ext, r, f.p), f.p));
    const uint32_t count = 1u << log_ext;
    const uint32_t scale = host::to_monty(f, host::invmod(1u << log_n, f.p));
    DevBuf buf;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    with_monty(field, [&](auto fld) {
      natural_mul_kernel<decltype(fld)><<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), log_n, count, B,
                                                                                scale);
      return 0;
    });
    Status s = sync_after_build(ctx, stream, "natural_mul_kernel");
    if (!s.ok()) { buf.release(); return s; }
    im = ctx->lde_tabs.emplace(kmul, buf).first;
  }
  auto it = ctx->lde_tabs.find(ktw);
  if (it == ctx->lde_tabs.end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "LDE table not prepared before capture"};
    MontyGens g{};
    for (uint32_t l = 0; l < f.two_adicity; ++l) g.g[l] = host::to_monty(f, host::two_adic_generator(f, l + 1));
    const uint32_t count = (1u << log_ext) - 1u;
    DevBuf buf;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    with_monty(field, [&](auto fld) {
      coset_twiddle_kernel<decltype(fld)><<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), count,
                                                                                  added_bits, g);
      return 0;
    });
    Status s = sync_after_build(ctx, stream, "coset_twiddle_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->lde_tabs.emplace(ktw, buf).first;
  }
  *mul = im->second.as<uint2>();
  *coset_tw = it->second.as<uint2>();
  return {};
}

Status monty_lde_table(sfntt_ctx* ctx, int field, uint32_t log_n, uint32_t added_bits, uint32_t shift_monty,
                       int kind, cudaStream_t stream, const uint2** out) {
  const host::MontyField& f = host::monty_field(field);
  if (!ext_fits(log_n, added_bits, f.two_adicity - 1))
    return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= " + std::to_string(f.two_adicity - 1)};
  const uint32_t log_ext = log_n + added_bits;
  if (kind != 1 && added_bits > 4) return {SFNTT_INVALID_ARGUMENT, "fused LDE supports added_bits <= 4"};
  const auto key = std::make_tuple(monty_slot(field), log_n, added_bits, shift_monty, kind);
  auto it = ctx->lde_tabs.find(key);
  if (it == ctx->lde_tabs.end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "LDE table not prepared before capture"};
    const uint32_t shift = shift_monty ? host::from_monty(f, shift_monty) : host::two_adic_generator(f, log_ext + 1);
    LdeBases B{};
    uint32_t log_len, count, scale;
    if (kind == 2 && log_n < 13) return {SFNTT_INVALID_ARGUMENT, "tile-ordered multipliers need log_n >= 13"};
    if (kind == 0 || kind == 2) {
      // quarter q of the zero-padded DIF gets g_ext^{i * rev(q)} from its top
      // added_bits layers; fold it with the shift and n^-1 into one multiplier
      const uint32_t g_ext = host::two_adic_generator(f, log_ext);
      for (uint32_t q = 0; q < (1u << added_bits); ++q) {
        uint32_t rq = 0;
        for (uint32_t bit = 0; bit < added_bits; ++bit) rq |= ((q >> bit) & 1u) << (added_bits - 1 - bit);
        B.b[q] = host::to_monty(f, host::mulmod(shift, host::powmod(g_ext, rq, f.p), f.p));
      }
      log_len = log_n;
      count = 1u << log_ext;
      scale = host::to_monty(f, host::invmod(1u << log_n, f.p));
    } else {
      B.b[0] = host::to_monty(f, shift);
      log_len = log_ext;
      count = 1u << log_ext;
      scale = host::to_monty(f, 1);
    }
    DevBuf buf;
    SFNTT_TRY(buf.reserve((size_t)count * sizeof(uint2)));
    with_monty(field, [&](auto fld) {
      using F = decltype(fld);
      power_table_kernel<F><<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), log_len, count, B, scale,
                                                                       kind == 2 ? log_n - 8 : 0u);
      return 0;
    });
    Status s = sync_after_build(ctx, stream, "power_table_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->lde_tabs.emplace(key, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

}  // namespace sfntt

namespace sfntt {

Status monty_twist_table(sfntt_ctx* ctx, int field, uint32_t lo, uint32_t P, bool inverse, cudaStream_t stream,
                         const uint2** out, bool compact) {
  const host::MontyField& f = host::monty_field(field);
  if (lo + P > f.two_adicity || P == 0 || P > 8) return {SFNTT_INVALID_ARGUMENT, "twist span"};
  const auto key = std::make_tuple(monty_slot(field), lo, P, inverse ? 1u : 0u, compact ? 5 : 2);
  auto it = ctx->lde_tabs.find(key);
  if (it == ctx->lde_tabs.end()) {
    if (capturing(stream)) return {SFNTT_INVALID_ARGUMENT, "twist table not prepared before capture"};
    uint32_t g = host::two_adic_generator(f, lo + P);
    if (inverse) g = host::invmod(g, f.p);
    const uint32_t count = 1u << (lo + P);
    DevBuf buf;
    SFNTT_TRY(buf.reserve((size_t)count * (compact ? sizeof(uint32_t) : sizeof(uint2))));
    with_monty(field, [&](auto fld) {
      using F = decltype(fld);
      twist_kernel<F><<<(count + 255) / 256, 256, 0, stream>>>(buf.as<uint2>(), lo, P, host::to_monty(f, g),
                                                                 compact ? 1 : 0);
      return 0;
    });
    Status s = sync_after_build(ctx, stream, "twist_kernel");
    if (!s.ok()) { buf.release(); return s; }
    it = ctx->lde_tabs.emplace(key, buf).first;
  }
  *out = it->second.as<uint2>();
  return {};
}

}  // namespace sfntt
