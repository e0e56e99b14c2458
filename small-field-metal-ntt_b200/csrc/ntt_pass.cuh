// ntt_pass.cuh -- the shared-memory tile engine behind every NTT pass.
//
// A radix-2 NTT network over n = 2^log_n points is split into passes; a pass
// owns the butterfly layers [lo, lo + P).  Elements that interact inside those
// layers differ only in index bits [lo, lo + P): a "group" of 2^P points with
// stride 2^lo.  One CTA loads a tile of 2^(P+LT) points (2^LT groups), runs the
// P layers in rounds of at most R layers, and writes the tile back:
//
//   * a round keeps 2^R points per thread in registers and performs r <= R
//     layers of butterflies on them (radix-2^r in registers);
//   * between rounds the tile is exchanged through shared memory;
//   * the first round reads global memory and the last one writes it, so each
//     pass touches HBM exactly once per point in each direction.
//
// Two tile kinds:
//   Kind::C (lo == 0)  -- contiguous blocks of 2^P points; the tile is 2^LT
//                         consecutive blocks (c = e | u << P, memory order).
//   Kind::S (lo > 0)   -- 2^LT consecutive low positions of 2^P-point groups
//                         (c = u | e << LT); every row of 2^LT words is one
//                         contiguous segment in HBM.
//
// The networks are the reference's exactly (same layer order, same twiddle per
// butterfly), so every intermediate value matches the reference CPU code:
//   BabyBear forward  : GS-DIF, layers descending, twiddle tw[L][pos mod 2^L]
//                       (src/ntt/babybear/cpu_reference.rs:45-60)
//   BabyBear inverse  : CT-DIT, layers ascending, same indexing
//                       (src/ntt/babybear/cpu_reference.rs:80-95)
//   M31 forward       : CT, layers descending, twiddle tw[L][pos >> (L+1)]
//                       (src/ntt/m31/cpu_reference.rs:61-74)
//   M31 inverse       : GS, layers ascending, per-block twiddle
//                       (src/ntt/m31/cpu_reference.rs:93-107)
// GS butterflies run on canonical values (9 integer ops); CT butterflies carry
// values lazily in [0, 2p) (9 ops) and are reduced when the pass stores.
#pragma once
#include <cstdint>

#include "field.cuh"
#include "pdl.cuh"

namespace sfntt {

enum class Kind : int { C = 0, S = 1 };

// Rounds: P layers split into K = ceil(P / R) rounds, the first P % K rounds
// one layer longer.  Round k covers group bits [b(k), b(k) + r(k)).
template <int P, int R>
struct Plan {
  static constexpr int K = (P + R - 1) / R;
  __host__ __device__ static constexpr int r(int k) { return P / K + ((k < P % K) ? 1 : 0); }
  __host__ __device__ static constexpr int b(int k) {
    int s = 0;
    for (int i = 0; i < k; ++i) s += r(i);
    return s;
  }
};

// Which tile bit (c-bit) each register slot bit (m-bit) and each thread-id bit
// maps to in round k.  m-bits [0, r) are the round's layers; m-bits [r, R) are
// "filler" bits taken from the highest free tile bits; thread-id bits take the
// remaining tile bits from the bottom up, so consecutive lanes touch
// consecutive words whenever possible.
struct RoundMap {
  int mpos[8];
  int ngrp;              // thread-id bits grouped by equal (c-bit - tid-bit) shift
  uint32_t gmask[16];
  int gshift[16];
};

// Filler bits: the tile bits of round k's slot bits r .. R-1 (i = 0, 1, ...),
// -1 = the highest free tile bits.  A search over the choices (against each
// round's thread map and the shared-memory bank model) looked for fillers that
// keep the thread bits two consecutive rounds share on the same thread-id bits
// -- so the exchange groups the warps instead of taking the whole CTA -- with
// no more bank conflicts.  Kept where it measured faster:
//   11 layers (rounds 4, 4, 3):            - | - | c11   CTA -> 2 groups; tile bit 12
//     then stays on thread bit 8 in every round: independent halves (2^19 x 64
//     forward + inverse 298 -> 292 us, 2^19 x 128 LDE 0.820 -> 0.804 ms)
//   14 layers (4, 4, 3, 3; 2^14-word tiles): - | - | c11 | c7   CTA + 8 groups
//     -> 4 + 4 groups (2^22 x 64 LDE 3.81 -> 3.77 ms)
// Dropped: 9 layers, c7 | c8 | c2 (both exchanges warp-local) made the twisted
// 9-layer pass 6 % slower -- its lanes then span tile bits 0, 1, 3, 4, 5 and the
// twist's global loads twice the sectors; 5 layers (CTA -> warp): no change.
template <Kind KD, int P, int LT, int R>
__host__ __device__ constexpr int filler_hint(int k, int i) {
  if (KD != Kind::C || R != 4 || i != 0) return -1;
  if (P == 14 && LT == 0) return k == 2 ? 11 : k == 3 ? 7 : -1;
  if (P == 11 && LT == 2) return k == 2 ? 11 : -1;
  return -1;
}

template <Kind KD, int P, int LT, int R>
__host__ __device__ constexpr RoundMap make_map(int k) {
  constexpr int CB = P + LT;
  constexpr int EOFF = (KD == Kind::S) ? LT : 0;
  RoundMap m{};
  const int r = Plan<P, R>::r(k);
  const int b = Plan<P, R>::b(k);
  bool used[32] = {};
  for (int j = 0; j < r; ++j) {
    m.mpos[j] = EOFF + b + j;
    used[EOFF + b + j] = true;
  }
  int f = r;
  for (int i = 0; f < R; ++i) {
    const int c = filler_hint<KD, P, LT, R>(k, i);
    if (c < 0 || used[c]) break;
    m.mpos[f++] = c;
    used[c] = true;
  }
  for (int c = CB - 1; c >= 0 && f < R; --c) {
    if (!used[c]) {
      m.mpos[f++] = c;
      used[c] = true;
    }
  }
  int t = 0;
  m.ngrp = 0;
  for (int c = 0; c < CB; ++c) {
    if (used[c]) continue;
    const int sh = c - t;
    if (m.ngrp == 0 || m.gshift[m.ngrp - 1] != sh) {
      m.gshift[m.ngrp] = sh;
      m.gmask[m.ngrp] = 0;
      ++m.ngrp;
    }
    m.gmask[m.ngrp - 1] |= 1u << t;
    ++t;
  }
  return m;
}

template <Kind KD, int P, int LT, int R, int k>
struct RM {
  // Tile bits of register slot m (a compile-time constant once loops unroll).
  __device__ static constexpr uint32_t cm(int m) {
    constexpr RoundMap map = make_map<KD, P, LT, R>(k);
    uint32_t c = 0;
    for (int j = 0; j < R; ++j)
      if ((m >> j) & 1) c |= 1u << map.mpos[j];
    return c;
  }
  __device__ static __forceinline__ uint32_t ctid(uint32_t tid) {
    constexpr RoundMap map = make_map<KD, P, LT, R>(k);
    uint32_t c = 0;
#pragma unroll
    for (int g = 0; g < map.ngrp; ++g) c |= (tid & map.gmask[g]) << map.gshift[g];
    return c;
  }
};

// Padded shared-memory index: one spare word every 32 keeps strided round
// accesses (stride <= 32 words) free of bank conflicts.
__device__ __forceinline__ uint32_t sidx(uint32_t c) { return c + (c >> 5); }

struct PassArgs {
  const uint32_t* in;
  uint32_t* out;
  const uint2* tw;      // layer-concatenated Shoup pairs (w, floor(w 2^32 / p))
  uint64_t in_stride;   // column strides, in elements
  uint64_t out_stride;
  uint32_t log_n;       // transform size
  uint32_t lo;          // first global layer of the pass
  uint32_t log_tiles_per_col;  // Kind::S only
  uint32_t batch;       // Kind::S: tiles are numbered column-fastest so that the
                        // CTAs running at the same time share twiddle rows
  uint32_t scale_w;     // if scale: multiply every output by w (Shoup pair)
  uint32_t scale_ws;
  int scale;
};

// Tile geometry resolved once per CTA.
struct TileGeo {
  const uint32_t* in;
  uint32_t* out;
  uint32_t pos_base;  // Kind::S: hb << (lo+P) | lchunk << LT ; Kind::C: pos of c == 0
  uint32_t hb;        // Kind::S high block (for M31 twiddles)
  bool spans;         // Kind::C: the tile spans several columns (2^CB > n)
  uint32_t v0;        // Kind::C: virtual (column-major dense) index of the tile start
};

template <class F, bool DESC>
struct Net {
  // GS on canonical values for BabyBear-forward / M31-inverse,
  // lazy CT for BabyBear-inverse / M31-forward.
  static constexpr bool kGS = (F::kMontgomery == DESC);
  static constexpr bool kPerPosition = F::kMontgomery;  // BabyBear twiddles by pos mod 2^L
};

template <class F, bool DESC>
__device__ __forceinline__ void butterfly(uint32_t& a, uint32_t& b, uint2 w) {
  if constexpr (Net<F, DESC>::kGS) {
    const uint32_t s = add_mod<F>(a, b);
    const uint32_t d = a - b + F::P;
    b = mul_shoup<F>(d, w.x, w.y);
    a = s;
  } else {
    const uint32_t ar = reduce2p<F>(a);
    const uint32_t t = mul_shoup<F>(b, w.x, w.y);
    a = ar + t;
    b = ar - t + F::P;
  }
}

// The butterfly with twiddle 1 (same values and representation as
// butterfly() with w = 1, whose Shoup product of x < 2p is x mod p).
template <class F, bool DESC>
__device__ __forceinline__ void butterfly_unit(uint32_t& a, uint32_t& b) {
  if constexpr (Net<F, DESC>::kGS) {
    const uint32_t s = add_mod<F>(a, b);
    b = reduce2p<F>(a - b + F::P);
    a = s;
  } else {
    const uint32_t ar = reduce2p<F>(a);
    const uint32_t t = reduce2p<F>(b);
    a = ar + t;
    b = ar - t + F::P;
  }
}

template <class F, bool DESC, Kind KD, int P, int LT, int R>
struct Pass {
  static constexpr int CB = P + LT;
  static constexpr int NT = 1 << (CB - R);
  static constexpr int E = 1 << R;
  static constexpr int K = Plan<P, R>::K;
  static constexpr uint32_t TMASK = (1u << LT) - 1u;
  static constexpr int SMEM_WORDS = (1 << CB) + ((1 << CB) >> 5);

  // position (within the column) of tile bit pattern c, relative to pos_base
  __device__ static __forceinline__ uint32_t map_pos(uint32_t c, uint32_t lo) {
    if constexpr (KD == Kind::S) return (c & TMASK) | ((c >> LT) << lo);
    else return c;
  }

  __device__ static __forceinline__ uint64_t elem_off(const TileGeo& g, uint32_t c, uint64_t stride,
                                                      const PassArgs& a) {
    if constexpr (KD == Kind::S) {
      return (uint64_t)(g.pos_base | map_pos(c, a.lo));
    } else {
      if (!g.spans) return (uint64_t)(g.pos_base + c);
      const uint32_t vv = g.v0 + c;
      return (uint64_t)(vv >> a.log_n) * stride + (vv & ((1u << a.log_n) - 1u));
    }
  }

  // Twiddle of the butterfly whose lower point has tile bits ctid | cm, at
  // group bit beta (global layer L = lo + beta).
  __device__ static __forceinline__ uint2 twiddle(const TileGeo& g, const PassArgs& a, uint32_t ctid,
                                                  uint32_t cm, int beta) {
    const uint32_t L = a.lo + beta;
    if constexpr (Net<F, DESC>::kPerPosition) {
      uint32_t j;
      if constexpr (KD == Kind::S) {
        const uint32_t em = (1u << beta) - 1u;
        j = (g.pos_base & ((1u << a.lo) - 1u)) | (ctid & TMASK) | (cm & TMASK) |
            ((((ctid | cm) >> LT) & em) << a.lo);
      } else {
        j = (ctid | cm) & ((1u << L) - 1u);
      }
      return __ldg(&a.tw[((1u << L) - 1u) + j]);
    } else {
      const uint32_t n = 1u << a.log_n;
      uint32_t blk;
      if constexpr (KD == Kind::S) {
        blk = (g.hb << (P - beta - 1)) | (((ctid | cm) >> LT) >> (beta + 1));
      } else {
        const uint32_t pos = g.spans ? ((ctid | cm) & (n - 1u)) : (g.pos_base | ctid | cm);
        blk = pos >> (L + 1);
      }
      return __ldg(&a.tw[(n - (n >> L)) + blk]);
    }
  }

  template <int k>
  __device__ static __forceinline__ void round(uint32_t (&v)[E], const TileGeo& g, const PassArgs& a,
                                               uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    constexpr int r = Plan<P, R>::r(k);
    constexpr int b = Plan<P, R>::b(k);
    const uint32_t ct = M::ctid(tid);
#pragma unroll
    for (int jj = 0; jj < r; ++jj) {
      const int j = DESC ? (r - 1 - jj) : jj;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        if (m & (1 << j)) continue;
        const uint2 w = twiddle(g, a, ct, M::cm(m), b + j);
        butterfly<F, DESC>(v[m], v[m | (1 << j)], w);
      }
    }
  }

  template <int k>
  __device__ static __forceinline__ void load_global(uint32_t (&v)[E], const TileGeo& g, const PassArgs& a,
                                                     uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t ct = M::ctid(tid);
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = __ldg(&g.in[elem_off(g, ct | M::cm(m), a.in_stride, a)]);
  }

  template <int k>
  __device__ static __forceinline__ void store_global(uint32_t (&v)[E], const TileGeo& g, const PassArgs& a,
                                                      uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t ct = M::ctid(tid);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      uint32_t x = v[m];
      if (a.scale) x = mul_shoup<F>(x, a.scale_w, a.scale_ws);
      else if constexpr (!Net<F, DESC>::kGS) x = reduce2p<F>(x);
      g.out[elem_off(g, ct | M::cm(m), a.out_stride, a)] = x;
    }
  }

  template <int k>
  __device__ static __forceinline__ void to_smem(uint32_t* sm, const uint32_t (&v)[E], uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t ct = M::ctid(tid);
#pragma unroll
    for (int m = 0; m < E; ++m) sm[sidx(ct | M::cm(m))] = v[m];
  }

  template <int k>
  __device__ static __forceinline__ void from_smem(const uint32_t* sm, uint32_t (&v)[E], uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t ct = M::ctid(tid);
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[sidx(ct | M::cm(m))];
  }

  template <int i>
  __device__ static __forceinline__ void rounds_from(uint32_t* sm, uint32_t (&v)[E], const TileGeo& g,
                                                     const PassArgs& a, uint32_t tid) {
    if constexpr (i < K) {
      constexpr int k = DESC ? (K - 1 - i) : i;
      if constexpr (i > 0) {
        constexpr int kp = DESC ? (K - i) : (i - 1);
        to_smem<kp>(sm, v, tid);
        __syncthreads();
        from_smem<k>(sm, v, tid);
      }
      round<k>(v, g, a, tid);
      rounds_from<i + 1>(sm, v, g, a, tid);
    }
  }

  __device__ static __forceinline__ TileGeo geometry(const PassArgs& a) {
    TileGeo g{};
    const uint32_t t = blockIdx.x;
    if constexpr (KD == Kind::S) {
      const uint32_t tt = t / a.batch;
      const uint32_t col = t - tt * a.batch;
      const uint32_t lchunk_bits = a.lo - LT;
      const uint32_t lchunk = tt & ((1u << lchunk_bits) - 1u);
      g.hb = tt >> lchunk_bits;
      g.pos_base = (g.hb << (a.lo + P)) | (lchunk << LT);
      g.in = a.in + (uint64_t)col * a.in_stride;
      g.out = a.out + (uint64_t)col * a.out_stride;
      g.spans = false;
    } else {
      const uint32_t v0 = t << CB;
      g.v0 = v0;
      if (a.log_n >= (uint32_t)CB) {
        const uint32_t col = v0 >> a.log_n;
        g.pos_base = v0 & ((1u << a.log_n) - 1u);
        g.in = a.in + (uint64_t)col * a.in_stride;
        g.out = a.out + (uint64_t)col * a.out_stride;
        g.spans = false;
      } else {
        g.pos_base = 0;
        g.in = a.in;
        g.out = a.out;
        g.spans = true;
      }
    }
    return g;
  }

  __device__ static __forceinline__ void run(PassArgs a) {
    extern __shared__ uint32_t sm[];  // SMEM_WORDS words (dynamic: tiles reach 66 KB)
    const uint32_t tid = threadIdx.x;
    const TileGeo g = geometry(a);
    uint32_t v[E];
    load_global<DESC ? (K - 1) : 0>(v, g, a, tid);
    rounds_from<0>(sm, v, g, a, tid);
    store_global<DESC ? 0 : (K - 1)>(v, g, a, tid);
  }
};

template <class F, bool DESC, Kind KD, int P, int LT, int R>
__global__ void __launch_bounds__(Pass<F, DESC, KD, P, LT, R>::NT)
pass_kernel(PassArgs a) {
  pdl_enter();
  Pass<F, DESC, KD, P, LT, R>::run(a);
}

}  // namespace sfntt
