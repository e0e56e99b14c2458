// tile_tma.cuh -- persistent, TMA-fed version of the tile engine.
//
// Every tile is 2^13 words = 32 KiB = 256 rows of 128 bytes:
//   Kind::C  2^13 consecutive words (2^(13-P) whole groups of 2^P points);
//   Kind::S  32 consecutive low positions (one 128-byte row each) of a
//            2^P-point group with stride 2^lo, P <= 8 (one TMA box {32,1,2^P}).
// Each CTA owns a strided sequence of tiles.  Thread 0 keeps one tile in
// flight ahead of the compute (double-buffered TMA loads into shared memory,
// completion tracked by mbarriers) and writes finished tiles back with TMA
// stores, so HBM traffic overlaps the integer work and moves with one
// instruction per tile.  The rounds and butterflies are those of ntt_pass.cuh;
// shared-memory exchanges happen in place in the staging buffer, with
// compile-time address offsets and 128-bit accesses wherever a thread owns four
// consecutive words.
//
// Every wait on an mbarrier is bounded (kWaitNs); a CTA that gives up sets the
// error flag, waits for its own TMA stores and returns.
#pragma once
#include <cstdint>

#include "ntt_pass.cuh"
#include "tma.cuh"

namespace sfntt {

constexpr int kTileBits = 13;
constexpr uint32_t kTileWords = 1u << kTileBits;
constexpr uint32_t kTileBytes = 4u << kTileBits;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s: far beyond any tile's latency

// Contiguous tiles are moved with the 128-byte TMA swizzle: word s of the
// shared-memory tile sits at s ^ (((s >> 5) & 7) << 2).  Without it, rounds
// whose threads own tile bits 0..3 (four consecutive words, 128-bit accesses)
// hit 4-way bank conflicts.
constexpr bool kSwizzleC = true;

// Row order of contiguous tiles in shared memory.  Tile word c (c0..c4: the
// word in its 128-byte row, c5..c12: the row) sits at shared word s = lay(c):
// in row order (s = c) the bank of a word is (c0, c1, c2^c5, c3^c6, c4^c7), so
// a round whose slots own tile bits 4..7 (the middle round of 8-, 11- and
// 12-layer passes; lanes on bits 0..3 and 8) reaches only 16 banks: two-way
// conflicts on every access.  Those passes store the rows as
// [c5 c6][c8 .. c11][c7][c12] instead -- bank (c0, c1, c2^c5, c3^c6, c4^c8),
// conflict-free in every round -- by loading each half tile (c12 fixed)
// through a 5-dimensional tensor map (32 words, rows c5..c6, rows c8 and up,
// row c7, column).  The 14-layer pass's 2^14-word tiles keep the same low
// rows, [c5 c6][c8 .. c12][c7][c13] (banks depend on c0 .. c8 alone).  Other
// layer counts are conflict-free in row order.
__host__ __device__ constexpr bool c_row_perm(int P) { return P == 8 || P == 11 || P == 12 || P == 14; }

struct TmaArgs {
  const uint2* tw;     // twiddles (layer-concatenated Shoup pairs)
  uint32_t log_n;      // positions per column of this network
  uint32_t lo;         // first global layer of the pass
  uint32_t ntiles;
  uint32_t log_tpc;    // Kind::C: log2(tiles per column) (n >= 2^13)
  uint32_t batch;
  uint32_t spans;      // Kind::C: tiles span columns (n < 2^13, dense columns)
  uint32_t scale, scale_w, scale_ws;
  int* err;
  // four-step twist applied at this pass's boundary (BabyBear): forward
  // passes multiply their inputs, inverse passes their outputs, by
  // twist[pos & twist_mask]; nullptr = none
  const uint2* twist;
  uint32_t twist_mask;
  // twist_compact: `twist` holds one word per entry, the Shoup companion w' of
  // the twist w, which gives back w = mulhi(w', p) + 1 (w' = floor(w 2^32 / p)
  // and w != 0): half the bytes, for tables that would not stay in L2
  uint32_t twist_compact;
  // M31 contiguous passes: the table's copy of layers 0..3 in first-round
  // order (entry n of an M31 table with n >= 2^13; see round0_permute_kernel);
  // nullptr = read the layers from the table itself
  const uint2* tw0;
  // fused LDE expansion (Expand kernel only)
  const uint2* tw_fwd;
  const uint2* mul;
  uint32_t log_q;
};

// The forward half of the LDE expansion runs in the extended network: the
// forward twiddle table, 2^(log_n + log_q) positions.
struct FwdArgs : TmaArgs {
  __device__ explicit FwdArgs(const TmaArgs& a) : TmaArgs(a) {
    tw = a.tw_fwd;
    log_n = a.log_n + a.log_q;
  }
};
__device__ __forceinline__ FwdArgs fwd_args(const TmaArgs& a) { return FwdArgs(a); }

// Where a tile sits: tensor-map coordinates and the column position of its
// first word (shared by every pass type so fused kernels can mix directions).
struct TileCoord {
  uint32_t pos_base;  // Kind::C: column position of word 0; Kind::S: lchunk << 5
  uint32_t hb;        // Kind::S high block
  int32_t c1, c2;     // Kind::C map coordinates (row, column)
  int32_t s1, s3, s4; // Kind::S map coordinates (lchunk, hb, column)
};

// PLAIN (BabyBear Kind::S only): run the plain 2^P-point sub-transform with
// lane-independent twiddles from shared memory and leave the four-step twist to
// the neighbouring pass; otherwise use the reference's per-position twiddles
// tw[L][pos mod 2^L] from the global table.  TW: this pass applies a boundary
// twist (forward: at load, inverse: at store).  LSTAGE (BabyBear Kind::S,
// per-position twiddles): the caller has staged the twiddles of the tile's
// 32-position chunk in shared memory (see lchunk_entry), so every twiddle is a
// shared-memory load instead of an L2 one.
template <class F, bool DESC, Kind KD, int P, bool PLAIN = false, bool TW = false, bool LSTAGE = false,
          bool HALVES = false>
struct TPass {
  // LSTAGE: each CTA takes a contiguous range of tiles ordered so that it
  // stays on one set of positions across the columns, and stages that set's
  // twiddles in shared memory.  BabyBear strided tiles: the per-position
  // twiddles of a 32-position chunk (the staged lookup takes the lane part of
  // a position from the thread alone: with P = 8 every slot bit of both rounds
  // is a layer bit above the lanes).  M31 contiguous tiles (any layer
  // count): the per-block twiddles of the tile's 2^13 positions.
  static_assert(!LSTAGE || (KD == Kind::S && F::kMontgomery && !PLAIN && P == 8) ||
                    (KD == Kind::C && !F::kMontgomery && !TW),
                "position staging: BabyBear 8-layer strided or M31 contiguous tiles");
  // Tile bits: 2^13-word tiles, except the 14-layer contiguous pass, whose
  // tile is one 2^14-point group (64 KiB, 1024 threads, one CTA per SM).
  static constexpr int TB = (KD == Kind::C && P > kTileBits) ? P : kTileBits;
  static constexpr int LT = (KD == Kind::C) ? (TB - P) : 5;
  static constexpr int CB = P + LT;
  static constexpr int R = 4;
  static constexpr int NT = 1 << (CB - R);
  static constexpr int E = 1 << R;
  static constexpr int K = Plan<P, R>::K;
  static_assert(KD == Kind::C ? (CB == TB && P <= 14) : (P <= 8), "tile shape");
  static constexpr uint32_t TWORDS = 1u << CB;
  static constexpr uint32_t TBYTES = 4u << CB;

  using Geo = TileCoord;

  // Tile t of a pass: Kind::C position-fastest, Kind::S column-fastest, then
  // chunk, then high block.
  __device__ static __forceinline__ Geo geo(const TmaArgs& a, uint32_t t) {
    Geo g{};
    if constexpr (KD == Kind::C) {
      if (a.spans) {
        g.pos_base = 0;
        g.c1 = (int32_t)(t << (CB - 5));
        g.c2 = 0;
      } else {
        const uint32_t r = t & ((1u << a.log_tpc) - 1u);
        g.pos_base = r << CB;
        g.c1 = (int32_t)(r << (CB - 5));
        g.c2 = (int32_t)(t >> a.log_tpc);
      }
    } else {
      const uint32_t tt = t / a.batch;
      const uint32_t col = t - tt * a.batch;
      const uint32_t lbits = a.lo - 5;
      const uint32_t lchunk = tt & ((1u << lbits) - 1u);
      g.hb = tt >> lbits;
      g.pos_base = lchunk << 5;
      g.s1 = (int32_t)lchunk;
      g.s3 = (int32_t)g.hb;
      g.s4 = (int32_t)col;
    }
    return g;
  }

  // The tile order of run(): geo's, except that LSTAGE passes keep a set of
  // positions across the columns -- Kind::C column-fastest; Kind::S chunk
  // slowest, then high block, then column -- so a CTA's contiguous range of
  // tiles shares one staged copy of twiddles for batch (x high blocks) tiles.
  __device__ static __forceinline__ Geo geo_run(const TmaArgs& a, uint32_t t) {
    if constexpr (!LSTAGE) {
      return geo(a, t);
    } else {
      Geo g{};
      if constexpr (KD == Kind::C) {  // n >= 2^13 (never spanning)
        const uint32_t r = t / a.batch;
        g.pos_base = r << CB;
        g.c1 = (int32_t)(r << (CB - 5));
        g.c2 = (int32_t)(t - r * a.batch);
      } else {
        // chunk pairs {2p, 2p+1} slowest, then high block and column, the
        // pair's two chunks alternating: consecutive tiles read neighbouring
        // 128-byte runs of the same rows
        const uint32_t per_pair = (a.batch << (a.log_n - a.lo - P)) << 1;
        const uint32_t pair = t / per_pair;
        const uint32_t r = t - pair * per_pair;
        const uint32_t rest = r >> 1;
        const uint32_t lchunk = 2u * pair + (r & 1u);
        g.hb = rest / a.batch;
        g.pos_base = lchunk << 5;
        g.s1 = (int32_t)lchunk;
        g.s3 = (int32_t)g.hb;
        g.s4 = (int32_t)(rest - g.hb * a.batch);
      }
      return g;
    }
  }

  __device__ static __forceinline__ void tma_load(const CUtensorMap* m, const Geo& g, uint32_t* dst, uint64_t* bar) {
    if constexpr (KD == Kind::C) c_load(m, g.c1, g.c2, dst, bar, true);
    else tma::load_5d(dst, m, 0, g.s1, 0, g.s3, g.s4, bar);
  }

  __device__ static __forceinline__ void tma_store(const CUtensorMap* m, const Geo& g, const uint32_t* src) {
    if constexpr (KD == Kind::C) c_store(m, g.c1, g.c2, src, true);
    else tma::store_5d(m, 0, g.s1, 0, g.s3, g.s4, src);
  }

  // Contiguous tiles: the whole tile at 128-byte row `row` of column `col`
  // (rows [row, row + 256)), or the half tile there (rows [row, row + 128)).
  // A row-ordered map's box is the copy (whole or half, as encoded); a
  // row-permuted map's box is a half tile, so a whole tile takes two copies.
  __device__ static __forceinline__ void c_load(const CUtensorMap* m, int32_t row, int32_t col, uint32_t* dst,
                                                uint64_t* bar, bool whole) {
    if constexpr (kRowPerm) {
      tma::load_5d(dst, m, 0, 0, row >> 3, 0, col, bar);
      if (whole) tma::load_5d(dst + TWORDS / 2, m, 0, 0, (row >> 3) + (int32_t)(TWORDS / 512), 0, col, bar);
    } else {
      tma::load_3d(dst, m, 0, row, col, bar);
    }
  }
  __device__ static __forceinline__ void c_store(const CUtensorMap* m, int32_t row, int32_t col, const uint32_t* src,
                                                 bool whole) {
    if constexpr (kRowPerm) {
      tma::store_5d(m, 0, 0, row >> 3, 0, col, src);
      if (whole) tma::store_5d(m, 0, 0, (row >> 3) + (int32_t)(TWORDS / 512), 0, col, src + TWORDS / 2);
    } else {
      tma::store_3d(m, 0, row, col, src);
    }
  }

  // BabyBear passes read their twiddles from a shared-memory copy of layers
  // [0, P) of the global table: contiguous passes need tw[L][pos mod 2^L]
  // with L < P; strided passes run the plain 2^P-point sub-transform, whose
  // layer-beta twiddle tw[beta][e mod 2^beta] is the same for every lane (the
  // per-position remainder is the boundary twist).
  static constexpr bool kStaged = F::kMontgomery && (KD == Kind::C || PLAIN);

  // M31 contiguous passes whose first round gives thread t the tile words
  // 16 t .. 16 t + 15 (four layers, thread bits 4..12 in order) read that
  // round's per-block twiddles from the table's first-round copy (TmaArgs::tw0).
  static constexpr bool round0_linear() {
    const RoundMap mp = make_map<KD, P, LT, 4>(0);
    return CB == kTileBits && Plan<P, 4>::r(0) == 4 && mp.mpos[0] == 0 && mp.mpos[1] == 1 && mp.mpos[2] == 2 && mp.mpos[3] == 3 &&
           mp.ngrp == 1 && mp.gshift[0] == 4 && mp.gmask[0] == (1u << (kTileBits - 4)) - 1u;
  }
  static constexpr bool kRound0Copy = !F::kMontgomery && KD == Kind::C && round0_linear();
  // M31 12-layer staging keeps layers 0..3 in the first round's thread order
  // (from the table's first-round copy); other layer counts stage every layer
  // in table order.
  static constexpr bool kStageThreadOrder = LSTAGE && KD == Kind::C && P == 12;
  static_assert(!kStageThreadOrder || kRound0Copy, "M31 tile staging starts from the first-round copy");
  // BabyBear staged twiddles: layers [0, min(P, 12)) (32 KiB at most, two CTAs
  // per SM); a 13-layer contiguous pass reads its top layer's 4096 twiddles
  // from the global table.
  static constexpr int kStagedLayers = P < 12 ? P : 12;
  static constexpr uint32_t TW_ENTRIES = kStaged ? ((1u << kStagedLayers) - 1u) : 0u;
  // M31 tile staging: the twiddles of a tile's 2^13 positions, one word each
  // -- the Shoup companion w' = floor(w 2^32 / p), which for the Mersenne
  // prime (2^32 / p = 2 + 2 / p) is 2w + (w >= 2^30), so w = w' >> 1, one
  // shift -- laid out like a
  // 2^13-point table with layer L at 8192 - (8192 >> L); with 12 layers,
  // layers 0..3 (words [0, 7680)) are ordered by thread: layer j gives thread
  // t its 2^(3-j) twiddles as vectors of v = min(2^(3-j), 4) words at
  // v (g NT + t), group g.
  static constexpr uint32_t CTILE_ENTRIES = 8190u;
  // staged twiddle bytes in shared memory, CTAs per SM
  static constexpr uint32_t SMEM_TW_BYTES =
      LSTAGE ? (KD == Kind::S ? 2u * 8u * 32u * ((1u << P) - 1u) : 4u * TWORDS) : 8u * TW_ENTRIES;
  static constexpr int kCtasPerSm = ((LSTAGE && KD == Kind::S) || NT > 512) ? 1 : 2;
  // Tile buffers of the whole-tile pipeline (run): three -- the tiles two and
  // one ahead in flight while one is computed -- for the staged strided passes
  // (one CTA per SM, 227 KiB with the twiddle chunks: 2^20 x 256 natural-order
  // LDE 3.72 -> 3.69 ms), else two.  Three buffers everywhere they fit at the
  // same CTAs per SM (228 KiB per SM, 1 KiB reserved per CTA) was measured:
  // the 2^24-point NTT's twisted strided pass went 45.8 -> 51.1 us (its twist
  // and column compete for L2 with the extra tile in flight), the plain one
  // 34.4 -> 32.0 us, the pair 213 -> 220 us.  The independent halves keep two
  // half-tile buffers per half.
  __host__ __device__ static constexpr int smem_bytes(int stages) {
    return stages * (int)TBYTES + 32 + (int)SMEM_TW_BYTES + 1024;
  }
  static constexpr int kStages = (LSTAGE && KD == Kind::S && (smem_bytes(3) + 1024) * kCtasPerSm <= 233472 &&
                                  smem_bytes(3) <= 232448)
                                     ? 3
                                     : 2;
  static constexpr int kSmemBytes = smem_bytes(HALVES ? 2 : kStages);

  // C = 1, 2 or 4 consecutive staged M31 twiddles (Shoup companions) from
  // shared memory (p aligned to C words) into tv[AT, AT + C) as (w, w') pairs
  template <int C, int AT>
  __device__ static __forceinline__ void staged_w(const uint32_t* p, uint2 (&tv)[E / 2]) {
    uint32_t w[4];
    if constexpr (C == 1) {
      w[0] = p[0];
    } else if constexpr (C == 2) {
      const uint2 q = *reinterpret_cast<const uint2*>(p);
      w[0] = q.x; w[1] = q.y;
    } else {
      static_assert(C == 4, "one vector load");
      const uint4 q = *reinterpret_cast<const uint4*>(p);
      w[0] = q.x; w[1] = q.y; w[2] = q.z; w[3] = q.w;
    }
#pragma unroll
    for (int i = 0; i < C; ++i) tv[AT + i] = make_uint2(w[i] >> 1, w[i]);
  }

  // ---- twiddles: per-layer base pointer + compile-time offset per slot ----
  template <int k>
  __device__ static __forceinline__ uint2 twiddle(const TmaArgs& a, const uint2* tws, const Geo& g, uint32_t ct, int m,
                                                  int beta) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t cm = M::cm(m);
    const uint32_t L = a.lo + beta;
    if constexpr (kStaged) {
      const uint32_t mask = (1u << beta) - 1u;
      if constexpr (KD == Kind::C) {
        if (beta >= (uint32_t)kStagedLayers) return __ldg(a.tw + ((1u << beta) - 1u) + (ct & mask) + (cm & mask));
        return tws[((1u << beta) - 1u) + (ct & mask) + (cm & mask)];
      } else {
        return tws[((1u << beta) - 1u) + ((ct >> 5) & mask) + ((cm >> 5) & mask)];
      }
    } else if constexpr (LSTAGE && KD == Kind::S) {  // tw[L][pos mod 2^L] from the chunk's staged copy
      const uint32_t em = (1u << beta) - 1u;
      return tws[32u * em + ((((ct >> 5) & em) + ((cm >> 5) & em)) << 5) + (ct & 31u)];
    } else if constexpr (LSTAGE && KD == Kind::C) {  // M31: the tile's staged table-order copy (w' = 2w + (w >> 30))
      static_assert(!kStageThreadOrder, "12-layer rounds take their staged twiddles in round()");
      const uint32_t* tw32 = reinterpret_cast<const uint32_t*>(tws) + (TWORDS - (TWORDS >> L));
      const uint32_t ws = tw32[(ct >> (L + 1)) + (cm >> (L + 1))];
      return make_uint2(ws >> 1, ws);
    } else if constexpr (F::kMontgomery) {  // BabyBear strided, per position: tw[L][pos mod 2^L]
      const uint2* base = a.tw + ((1u << L) - 1u);
      const uint32_t em = (1u << beta) - 1u;
      const uint32_t jt = g.pos_base + (ct & 31u) + (((ct >> 5) & em) << a.lo);
      return __ldg(base + jt + (cm & 31u) + (((cm >> 5) & em) << a.lo));
    } else {  // M31: tw[L][pos >> (L+1)]
      const uint32_t n = 1u << a.log_n;
      const uint2* base = a.tw + (n - (n >> L));
      if constexpr (KD == Kind::C) {  // tile bits above log n select the column (spanning tiles)
        return __ldg(base + ((g.pos_base >> (L + 1)) + ((ct & (n - 1u)) >> (L + 1)) + ((cm & (n - 1u)) >> (L + 1))));
      } else {
        return __ldg(base + ((g.hb << (P - beta - 1)) + ((ct >> 5) >> (beta + 1)) + ((cm >> 5) >> (beta + 1))));
      }
    }
  }

  template <int k>
  __device__ static __forceinline__ void round(uint32_t (&v)[E], const TmaArgs& a, const uint2* tws, const Geo& g,
                                               uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    constexpr int r = Plan<P, R>::r(k);
    constexpr int b = Plan<P, R>::b(k);
    const uint32_t ct = M::ctid(tid);
    if constexpr (!F::kMontgomery && r == R) {
      // M31 round without filler bits: slot m sits at group bits m << b, so
      // layer L = lo + b + j needs the per-block twiddles tw[L][base + o] for
      // o = m >> (j+1) < 2^(r-1-j): consecutive entries from an even index
      // (n - n/2^L, the tile's block offset and the thread's bits above the
      // round are even multiples there), fetched as 128-bit pairs.
#pragma unroll
      for (int jj = 0; jj < r; ++jj) {
        const int j = DESC ? (r - 1 - jj) : jj;
        const uint32_t beta = (uint32_t)(b + j);
        const uint32_t L = a.lo + beta;
        const uint32_t n = 1u << a.log_n;
        uint2 tv[E / 2];
        if constexpr (LSTAGE) {
          // this thread's 2^(r-1-j) twiddles of layer j (a constant once unrolled)
          const uint32_t* tw32 = reinterpret_cast<const uint32_t*>(tws) + (TWORDS - (TWORDS >> L));
          if constexpr (k == 0 && kStageThreadOrder) {  // thread-ordered first-round layers
            switch (r - 1 - j) {
              case 3: staged_w<4, 0>(tw32 + 4u * tid, tv); staged_w<4, 4>(tw32 + 4u * (NT + tid), tv); break;
              case 2: staged_w<4, 0>(tw32 + 4u * tid, tv); break;
              case 1: staged_w<2, 0>(tw32 + 2u * tid, tv); break;
              default: staged_w<1, 0>(tw32 + tid, tv); break;
            }
          } else {
            const uint32_t* p = tw32 + (ct >> (L + 1));
            switch (r - 1 - j) {
              case 3: staged_w<4, 0>(p, tv); staged_w<4, 4>(p + 4, tv); break;
              case 2: staged_w<4, 0>(p, tv); break;
              case 1: staged_w<2, 0>(p, tv); break;
              default: staged_w<1, 0>(p, tv); break;
            }
          }
        } else {
          bool copied = false;
          if constexpr (kRound0Copy && k == 0) {
            if (a.tw0) {
              // the table's first-round copy: [tile][layer][pair][thread], coalesced across the CTA
              const uint2* t0 = a.tw0 + (g.pos_base >> 13) * 7680u;
              const uint32_t off = j == 0 ? 0u : j == 1 ? 4096u : j == 2 ? 6144u : 7168u;
              if (j == r - 1) {
                tv[0] = __ldg(t0 + off + tid);
              } else {
#pragma unroll
                for (int o = 0; o < (1 << (r - 1 - j)); o += 2) {
                  const uint4 q = __ldg(reinterpret_cast<const uint4*>(t0 + off) + (uint32_t)(o >> 1) * NT + tid);
                  tv[o] = make_uint2(q.x, q.y);
                  tv[o + 1] = make_uint2(q.z, q.w);
                }
              }
              copied = true;
            }
          }
          if (!copied) {
            const uint2* base = a.tw + (n - (n >> L));
            if constexpr (KD == Kind::C) base += (g.pos_base >> (L + 1)) + ((ct & (n - 1u)) >> (L + 1));
            else base += (g.hb << (P - beta - 1)) + ((ct >> 5) >> (beta + 1));
            if (j == r - 1) {
              tv[0] = __ldg(base);
            } else {
#pragma unroll
              for (int o = 0; o < (1 << (r - 1 - j)); o += 2) {
                const uint4 q = __ldg(reinterpret_cast<const uint4*>(base + o));
                tv[o] = make_uint2(q.x, q.y);
                tv[o + 1] = make_uint2(q.z, q.w);
              }
            }
          }
        }
#pragma unroll
        for (int m = 0; m < E; ++m) {
          if (m & (1 << j)) continue;
          butterfly<F, DESC>(v[m], v[m | (1 << j)], tv[m >> (j + 1)]);
        }
      }
    } else {
#pragma unroll
      for (int jj = 0; jj < r; ++jj) {
        const int j = DESC ? (r - 1 - jj) : jj;
#pragma unroll
        for (int m = 0; m < E; ++m) {
          if (m & (1 << j)) continue;
          if (unit_twiddle<k>(m, b + j))  // a compile-time constant once the loops unroll
            butterfly_unit<F, DESC>(v[m], v[m | (1 << j)]);
          else
            butterfly<F, DESC>(v[m], v[m | (1 << j)], twiddle<k>(a, tws, g, ct, m, b + j));
        }
      }
    }
  }

  // Staged passes index layer beta's twiddle by the group element's low beta
  // bits (tw[beta][e mod 2^beta]).  Where none of round k's thread bits lies
  // among those bits, the index is the slot's alone, and slots whose index is
  // 0 multiply by tw[beta][0] = 1 (g^0 in the forward table and its inverse in
  // the inverse one): their butterflies need no product.  In a 12-layer
  // contiguous pass that is all of layer 0, half of layer 1, a quarter of
  // layer 2 and an eighth of layer 3: 15 of each thread's 96 butterflies.
  __host__ __device__ static constexpr uint32_t thread_tile_bits(int k) {
    const RoundMap mp = make_map<KD, P, LT, R>(k);
    uint32_t t = 0;
    for (int g = 0; g < mp.ngrp; ++g) t |= mp.gmask[g] << mp.gshift[g];
    return t;
  }
  template <int k>
  __device__ static constexpr bool unit_twiddle(int m, int beta) {
    if (!kStaged) return false;
    constexpr int sh = (KD == Kind::C) ? 0 : 5;  // Kind::S: the group element sits above the 32 lanes
    const uint32_t mask = (1u << beta) - 1u;
    return ((thread_tile_bits(k) >> sh) & mask) == 0u && ((RM<KD, P, LT, R, k>::cm(m) >> sh) & mask) == 0u;
  }

  // Round k on two tiles' values at once, with one twiddle load per butterfly
  // pair: the per-position twiddles tw[L][pos mod 2^L] of BabyBear / KoalaBear
  // strided passes are the same for every high block, so the output blocks of
  // one LDE expansion share them.
  template <int k>
  __device__ static __forceinline__ void round2(uint32_t (&va)[E], uint32_t (&vb)[E], const TmaArgs& a,
                                                const uint2* tws, const Geo& g, uint32_t tid) {
    static_assert(F::kMontgomery && KD == Kind::S, "twiddles shared across high blocks: per-position strided");
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
        if (unit_twiddle<k>(m, b + j)) {
          butterfly_unit<F, DESC>(va[m], va[m | (1 << j)]);
          butterfly_unit<F, DESC>(vb[m], vb[m | (1 << j)]);
        } else {
          const uint2 w = twiddle<k>(a, tws, g, ct, m, b + j);
          butterfly<F, DESC>(va[m], va[m | (1 << j)], w);
          butterfly<F, DESC>(vb[m], vb[m | (1 << j)], w);
        }
      }
    }
  }

  // ---- staging-buffer access in round k's layout ----
  template <int k>
  __device__ static constexpr bool vec() {
    constexpr RoundMap mp = make_map<KD, P, LT, R>(k);
    return mp.mpos[0] == 0 && mp.mpos[1] == 1;
  }

  // Shared-memory word of tile word c (the TMA layout of this tile kind: the
  // row order of c_row_perm, then the swizzle).
  static constexpr bool kSwz = (KD == Kind::C) && kSwizzleC;
  static constexpr bool kRowPerm = (KD == Kind::C) && c_row_perm(P);
  __host__ __device__ static constexpr uint32_t lay(uint32_t c) {
    // rows [c5 c6][c8 .. c(TB-2)][c7][c(TB-1)]
    constexpr uint32_t MID = ((1u << (TB - 1)) - 1u) & ~0x7Fu;  // c7 .. c(TB-2)
    return kRowPerm ? ((c & ~MID) | ((c >> 1) & (MID >> 1) & ~0x7Fu) | ((c & 0x80u) << (TB - 9))) : c;
  }
  __host__ __device__ static constexpr uint32_t sw(uint32_t c) {
    const uint32_t s = lay(c);
    return kSwz ? (s ^ (((s >> 5) & 7u) << 2)) : s;
  }
  // Bits that sw(x) may set when x ranges over the bits of `mask`.
  __host__ __device__ static constexpr uint32_t sw_support(uint32_t mask) {
    uint32_t s = 0;
    for (int i = 0; i < 32; ++i)
      if ((mask >> i) & 1u) s |= sw(1u << i);
    return s;
  }
  // sw is linear over GF(2), so sw(ct | cm) = sw(ct) ^ sw(cm).  Round k's
  // thread part and slot part overlap only in the bits `overlap<k>()`; the
  // rest of sw(cm) is added as an immediate offset:
  //   sw(ct | cm) = (sw(ct) ^ (sw(cm) & O)) + (sw(cm) & ~O).
  template <int k>
  __device__ static constexpr uint32_t overlap() {
    constexpr RoundMap mp = make_map<KD, P, LT, R>(k);
    uint32_t tmask = 0, cmask = 0;
    for (int g = 0; g < mp.ngrp; ++g) tmask |= mp.gmask[g] << mp.gshift[g];
    for (int j = 0; j < R; ++j) cmask |= 1u << mp.mpos[j];
    return sw_support(tmask) & sw_support(cmask);
  }
  template <int k>
  __device__ static __forceinline__ uint32_t addr(uint32_t sct, int m) {
    using M = RM<KD, P, LT, R, k>;
    constexpr uint32_t O = overlap<k>();
    const uint32_t scm = sw(M::cm(m));
    return (sct ^ (scm & O)) + (scm & ~O);
  }

  template <int k>
  __device__ static __forceinline__ void ld(const uint32_t* st, uint32_t (&v)[E], uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t sct = sw(M::ctid(tid));
    if constexpr (vec<k>()) {
#pragma unroll
      for (int m = 0; m < E; m += 4) {
        const uint4 q = *reinterpret_cast<const uint4*>(st + addr<k>(sct, m));
        v[m] = q.x; v[m + 1] = q.y; v[m + 2] = q.z; v[m + 3] = q.w;
      }
    } else {
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = st[addr<k>(sct, m)];
    }
  }

  template <int k>
  __device__ static __forceinline__ void st(uint32_t* st, const uint32_t (&v)[E], uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t sct = sw(M::ctid(tid));
    if constexpr (vec<k>()) {
#pragma unroll
      for (int m = 0; m < E; m += 4)
        *reinterpret_cast<uint4*>(st + addr<k>(sct, m)) = make_uint4(v[m], v[m + 1], v[m + 2], v[m + 3]);
    } else {
#pragma unroll
      for (int m = 0; m < E; ++m) st[addr<k>(sct, m)] = v[m];
    }
  }

  // ---- synchronisation of an exchange ----
  // A word written in round kp's layout is read in round k's layout by the
  // thread that owns it there.  Tile bits that are thread bits in both layouts
  // pin the owner's thread-id bits; when they sit at the same thread-id
  // position in both, writer and reader agree on those bits, so only threads
  // that share them exchange data.  If the pinned bits cover every warp bit
  // the exchange stays inside a warp (__syncwarp); if they cover some, inside
  // the warps that share them (a named barrier per group); else the CTA.
  __host__ __device__ static constexpr int tid_bit(int k, int c) {
    const RoundMap mp = make_map<KD, P, LT, R>(k);
    for (int g = 0; g < mp.ngrp; ++g) {
      const int t = c - mp.gshift[g];
      if (t >= 0 && t < 32 && ((mp.gmask[g] >> t) & 1u)) return t;
    }
    return -1;
  }
  __host__ __device__ static constexpr int xfixed_of(int kp, int k) {
    int mask = 0;
    for (int c = 0; c < CB; ++c) {
      const int a = tid_bit(kp, c), b = tid_bit(k, c);
      if (a >= 0 && b >= 0) {
        if (a != b) return -1;
        mask |= 1 << a;
      }
    }
    return mask;
  }
  template <int kp, int k>
  __host__ __device__ static constexpr int xfixed() { return xfixed_of(kp, k); }
  static constexpr int kWarpBits = (NT - 1) & ~31;
  __host__ __device__ static constexpr int popc(int x) { return x ? (x & 1) + popc(x >> 1) : 0; }
  // Named-barrier groups of the exchange between rounds kp and k (0: a warp
  // or CTA barrier).
  __host__ __device__ static constexpr int xgroups(int kp, int k) {
    const int fixed = xfixed_of(kp, k);
    const int wf = fixed < 0 ? 0 : (fixed & kWarpBits);
    if (fixed >= 0 && kWarpBits != 0 && wf == kWarpBits) return 0;
    return (wf != 0 && popc(wf) <= 3) ? (1 << popc(wf)) : 0;
  }
  // First barrier id of the exchange before rounds<i>.  Consecutive exchanges
  // of one tile may group the warps differently with no CTA barrier between
  // them, so a warp can reach the next exchange's barrier while others still
  // wait at this one: every exchange of the pass takes its own ids (1 + the
  // groups of the exchanges before it; ids 14 and 15 are the independent
  // halves' pre-store barriers).
  __host__ __device__ static constexpr int xbase(int i) {
    int b = 1;
    for (int j = 1; j < i; ++j) b += DESC ? xgroups(K - j, K - 1 - j) : xgroups(j - 1, j);
    return b;
  }
  template <int kp, int k, int BASE>
  __device__ static __forceinline__ void xsync(uint32_t tid) {
    constexpr int fixed = xfixed<kp, k>();
    constexpr int wf = fixed < 0 ? 0 : (fixed & kWarpBits);
    if constexpr (fixed >= 0 && kWarpBits != 0 && wf == kWarpBits) {
      __syncwarp();
    } else if constexpr (wf != 0 && __builtin_popcount(wf) <= 3) {
      static_assert(BASE + (1 << __builtin_popcount(wf)) - 1 <= 13, "named barrier ids of the exchanges: 1..13");
      uint32_t id = BASE, i = 0;
#pragma unroll
      for (int bit = 5; bit < 16; ++bit) {
        if ((wf >> bit) & 1) {
          id += ((tid >> bit) & 1u) << i;
          ++i;
        }
      }
      constexpr uint32_t count = (uint32_t)NT >> __builtin_popcount(wf);
      asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
    } else {
      __syncthreads();
    }
  }

  // Warp-shuffle form of an exchange (build-time switch SFNTT_SHFL_EXCHANGE,
  // for comparisons).  Where round k's slot bit j is round kp's lane bit j and
  // the reverse, for every j < R, and the other thread-id bits keep their tile
  // bits, the exchange is a transpose of R slot bits with R lane bits inside a
  // warp: R xor-shuffle stages, stage j swapping slot bit j with lane bit j (per
  // slot pair one shuffle and three selects).  The contiguous 8-, 11- and
  // 12-layer passes' warp-local exchanges have this form (checked on the CPU
  // against the shared-memory exchange's word map).
  __host__ __device__ static constexpr bool shfl_swap(int kp, int k) {
    const RoundMap a = make_map<KD, P, LT, R>(kp), b = make_map<KD, P, LT, R>(k);
    for (int j = 0; j < R; ++j)
      if (tid_bit(k, a.mpos[j]) != j || tid_bit(kp, b.mpos[j]) != j) return false;
    for (int c = 0; c < CB; ++c) {
      const int ta = tid_bit(kp, c), tb = tid_bit(k, c);
      if ((ta >= R || tb >= R) && ta != tb) return false;
    }
    return true;
  }
  __device__ static __forceinline__ void shfl_transpose(uint32_t (&v)[E], uint32_t tid) {
    const uint32_t lane = tid & 31u;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const bool hi = (lane >> j) & 1u;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        if ((m >> j) & 1) continue;
        const uint32_t send = hi ? v[m] : v[m | (1 << j)];
        const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, 1 << j);
        if (hi) v[m] = recv;
        else v[m | (1 << j)] = recv;
      }
    }
  }

  // All K rounds starting from registers in round (DESC ? K-1 : 0)'s layout,
  // exchanging through `buf`; ends in round (DESC ? 0 : K-1)'s layout.
  template <int i>
  __device__ static __forceinline__ void rounds(uint32_t* buf, uint32_t (&v)[E], const TmaArgs& a, const uint2* tws,
                                                const Geo& g, uint32_t tid) {
    if constexpr (i < K) {
      constexpr int k = DESC ? (K - 1 - i) : i;
      if constexpr (i > 0) {
        constexpr int kp = DESC ? (K - i) : (i - 1);
#ifdef SFNTT_SHFL_EXCHANGE
        if constexpr (shfl_swap(kp, k)) {
          shfl_transpose(v, tid);
        } else
#endif
        {
          st<kp>(buf, v, tid);
          xsync<kp, k, xbase(i)>(tid);
          ld<k>(buf, v, tid);
        }
      }
      round<k>(v, a, tws, g, tid);
      rounds<i + 1>(buf, v, a, tws, g, tid);
    }
  }

  static constexpr int kFirst = DESC ? (K - 1) : 0;
  static constexpr int kLast = DESC ? 0 : (K - 1);

  // column position of slot m in round k's layout
  template <int k>
  __device__ static __forceinline__ uint32_t pos_of(const TmaArgs& a, const Geo& g, uint32_t ct, int m) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t cm = M::cm(m);
    if constexpr (KD == Kind::C) return g.pos_base + ct + cm;
    else
      return (g.hb << (a.lo + P)) + g.pos_base + (ct & 31u) + (cm & 31u) + (((ct >> 5) + (cm >> 5)) << a.lo);
  }

  template <int k>
  __device__ static __forceinline__ void twist(uint32_t (&v)[E], const TmaArgs& a, const Geo& g, uint32_t tid) {
    using M = RM<KD, P, LT, R, k>;
    const uint32_t ct = M::ctid(tid);
    if (a.twist_compact) {
      const uint32_t* tc = reinterpret_cast<const uint32_t*>(a.twist);
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const uint32_t ws = __ldg(tc + (pos_of<k>(a, g, ct, m) & a.twist_mask));
        v[m] = mul_shoup<F>(v[m], __umulhi(ws, F::P) + 1u, ws);
      }
    } else {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const uint2 w = __ldg(a.twist + (pos_of<k>(a, g, ct, m) & a.twist_mask));
        v[m] = mul_shoup<F>(v[m], w.x, w.y);
      }
    }
  }

  __device__ static __forceinline__ void finish(uint32_t (&v)[E], const TmaArgs& a, const Geo& g, uint32_t tid) {
    if constexpr (!DESC && TW) twist<kLast>(v, a, g, tid);  // canonical afterwards
#pragma unroll
    for (int m = 0; m < E; ++m) {
      if (a.scale) v[m] = mul_shoup<F>(v[m], a.scale_w, a.scale_ws);
      else if constexpr (!Net<F, DESC>::kGS && (DESC || !TW)) v[m] = reduce2p<F>(v[m]);
    }
  }

  // Copy the twiddle layers [0, P) into shared memory (BabyBear).
  __device__ static __forceinline__ void stage_twiddles(uint2* dst, const uint2* src, uint32_t tid) {
    for (uint32_t i = tid; i < TW_ENTRIES; i += NT) dst[i] = __ldg(src + i);
  }

  // Per-position twiddles of one 32-position chunk of strided tiles (layers
  // lo .. lo+P-1): entry 32 (2^beta - 1) + (e_low << 5) + u holds
  // tw[lo + beta][(e_low << lo) + chunk * 32 + u] for e_low < 2^beta, u < 32.
  static constexpr uint32_t LCHUNK_ENTRIES = 32u * ((1u << P) - 1u);
  __device__ static __forceinline__ void stage_lchunk(uint2* dst, const uint2* src, uint32_t lo, uint32_t chunk,
                                                      uint32_t tid) {
    for (uint32_t i = tid; i < LCHUNK_ENTRIES; i += NT) {
      const uint32_t row = (i >> 5) + 1u;  // 2^beta + e_low
      const uint32_t beta = 31u - __clz(row);
      const uint32_t e_low = row - (1u << beta);
      const uint32_t L = lo + beta;
      dst[i] = __ldg(src + ((1u << L) - 1u) + ((uint64_t)e_low << lo) + (chunk << 5) + (i & 31u));
    }
  }

  // M31 per-block twiddles (Shoup companions) of the 12 layers over tile positions
  // [pos_base, pos_base + 2^13): layers 0..3 from the table's first-round
  // copy ([layer][pair group][thread], a pair group = two pairs), layers
  // 4..11 from the table (2^(12-L) consecutive entries each).
  __device__ static __forceinline__ void stage_ctile(uint32_t* dst, const TmaArgs& a, uint32_t pos_base,
                                                     uint32_t tid) {
    const uint2* src0 = a.tw0 + (pos_base >> 13) * 7680u;
    for (uint32_t d = tid; d < 7680u; d += NT) {
      const uint32_t j = d < 4096u ? 0u : d < 6144u ? 1u : d < 7168u ? 2u : 3u;
      const uint32_t off = 8192u - (8192u >> j);
      const uint32_t rel = d - off;
      const uint32_t v = j <= 1u ? 4u : (j == 2u ? 2u : 1u);
      const uint32_t t = (rel / v) & (NT - 1u);
      const uint32_t o = (rel / (v * NT)) * v + (rel & (v - 1u));  // the thread's o-th twiddle of layer j
      const uint32_t sp = j == 3u ? off + t : off + 2u * ((o >> 1) * NT + t) + (o & 1u);
      dst[d] = __ldg(&src0[sp].y);
    }
    const uint32_t n = 1u << a.log_n;
    for (uint32_t e = 7680u + tid; e < CTILE_ENTRIES; e += NT) {
      const uint32_t L = 12u - (31u - __clz(8191u - e));  // e in [8192 - 2^(13-L), 8192 - 2^(12-L))
      const uint32_t local = e - (8192u - (8192u >> L));
      dst[e] = __ldg(&a.tw[(n - (n >> L)) + (pos_base >> (L + 1)) + local].y);
    }
  }

  // One tile in shared memory, in place: the first round's load, every round,
  // the finish and the last round's store (the work-list kernels' tile step).
  __device__ static __forceinline__ void tile_body(uint32_t* cur, const TmaArgs& a, const uint2* tws, const Geo& g,
                                                   uint32_t tid) {
    uint32_t v[E];
    ld<kFirst>(cur, v, tid);
    if constexpr (DESC && TW) twist<kFirst>(v, a, g, tid);
    rounds<0>(cur, v, a, tws, g, tid);
    finish(v, a, g, tid);
    st<kLast>(cur, v, tid);
  }

  // ---- independent halves (contiguous passes whose rounds all have R layers) ----
  // Tile bit CB-1 is then thread bit log2(NT)-1 in every round, so the two
  // halves of the CTA (256 threads each) work on the two 2^(CB-1)-word halves
  // of a tile without ever exchanging data.  run_halves gives each half its
  // own TMA pipeline (half tiles of 16 KiB, double-buffered, its own
  // mbarriers, its own store) and its own pre-store barrier, so a half never
  // waits for the other: the CTA-wide barriers, and the phase lock-step they
  // impose on all 16 warps, are gone.
  __host__ __device__ static constexpr bool halves_ok() {
    bool ok = KD == Kind::C && !LSTAGE && NT == 512;
    for (int k = 0; k < K && ok; ++k) ok = tid_bit(k, CB - 1) == 8;
    return ok;
  }
  static_assert(!HALVES || halves_ok(), "independent halves: contiguous tiles whose top bit is thread bit 8");
  static constexpr uint32_t HWORDS = TWORDS / 2, HBYTES = TBYTES / 2, HROWS = HWORDS / 32;

  // M31 per-block twiddles (Shoup companions) of every layer L < P over tile
  // positions [pos_base, pos_base + 2^CB), all in table order: 2^(CB-1-L)
  // consecutive entries of layer L at 2^CB - (2^CB >> L).
  __device__ static __forceinline__ void stage_ctile_plain(uint32_t* dst, const TmaArgs& a, uint32_t pos_base,
                                                           uint32_t tid) {
    const uint32_t n = 1u << a.log_n;
    const uint32_t end = TWORDS - (TWORDS >> P);
    for (uint32_t e = tid; e < end; e += NT) {
      // e in [2^CB - 2^(CB-L), 2^CB - 2^(CB-1-L))
      const uint32_t L = (uint32_t)(CB - 1) - (31u - __clz(TWORDS - 1u - e));
      const uint32_t local = e - (TWORDS - (TWORDS >> L));
      dst[e] = __ldg(&a.tw[(n - (n >> L)) + (pos_base >> (L + 1)) + local].y);
    }
  }

  __device__ static void run_halves(const CUtensorMap* min, const CUtensorMap* mout, const TmaArgs& args) {
    extern __shared__ __align__(1024) uint32_t smem_words[];
    const uint32_t tid = threadIdx.x;
    const uint32_t half = tid >> 8;
    const bool leader = (tid & 255u) == 0u;
    uint32_t* stage = smem_words + half * 2u * HWORDS;  // this half's two half-tile buffers
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_words + 2 * TWORDS) + 2u * half;
    uint2* tws = reinterpret_cast<uint2*>(reinterpret_cast<uint64_t*>(smem_words + 2 * TWORDS) + 4);
    const TmaArgs& a = args;
    uint32_t t = blockIdx.x;
    const uint32_t t_end = a.ntiles, t_step = gridDim.x;
    if (t >= t_end) return;
    if constexpr (kStaged) stage_twiddles(tws, a.tw, tid);
    if (leader) {
      tma::prefetch_map(min);
      tma::prefetch_map(mout);
      tma::mbar_init(&bar[0], 1);
      tma::mbar_init(&bar[1], 1);
      tma::fence_mbar_init();
    }
    __syncthreads();  // staged twiddles and barriers: the halves' last shared step
    const int32_t hrow = (int32_t)(half * HROWS);
    if (leader) {
      const Geo g0 = geo(a, t);
      tma::mbar_expect_tx(&bar[0], HBYTES);
      c_load(min, g0.c1 + hrow, g0.c2, stage, &bar[0], false);
    }
    const uint32_t bar_id = 14u + half;  // named barriers 1..13 are the rounds' exchanges
    uint32_t v[E];
    for (uint32_t it = 0; t < t_end; t += t_step, ++it) {
      const uint32_t buf = it & 1u;
      uint32_t* cur = stage + buf * HWORDS;
      // tile word c of this half (bit CB-1 = half) sits at view + sw(c) = cur + sw(c mod 2^(CB-1))
      uint32_t* view = cur - half * HWORDS;
      const uint32_t tn = t + t_step;
      if (leader && tn < t_end) {
        tma::wait_reads();  // the store that last used the other buffer has read it
        const Geo gn = geo(a, tn);
        tma::mbar_expect_tx(&bar[buf ^ 1u], HBYTES);
        c_load(min, gn.c1 + hrow, gn.c2, stage + (buf ^ 1u) * HWORDS, &bar[buf ^ 1u], false);
      }
      const Geo g = geo(a, t);
      const bool ok = tma::mbar_wait(&bar[buf], (it >> 1) & 1u, kWaitNs);
      ld<kFirst>(view, v, tid);
      if constexpr (DESC && TW) twist<kFirst>(v, a, g, tid);
      rounds<0>(view, v, a, tws, g, tid);
      finish(v, a, g, tid);
      st<kLast>(view, v, tid);
      tma::fence_proxy_async();
      uint32_t any_bad;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\t"
          "setp.ne.u32 p, %1, 0;\n\t"
          "bar.red.or.pred q, %2, 256, p;\n\t"
          "selp.u32 %0, 1, 0, q;\n\t}"
          : "=r"(any_bad)
          : "r"(ok ? 0u : 1u), "r"(bar_id)
          : "memory");
      if (any_bad) {
        if (leader) {
          atomicExch(a.err, 1);
          if (tn < t_end) tma::mbar_wait(&bar[buf ^ 1u], ((it + 1) >> 1) & 1u, kWaitNs);
          tma::wait_all();
        }
        return;
      }
      if (leader) {
        c_store(mout, g.c1 + hrow, g.c2, cur, false);
        tma::commit();
      }
    }
    if (leader) tma::wait_all();
  }

  __device__ static void run(const CUtensorMap* min, const CUtensorMap* mout, const TmaArgs& args) {
    if constexpr (HALVES) {
      run_halves(min, mout, args);
      return;
    }
    // Dynamic shared memory is 1024-byte aligned; indexing it directly keeps
    // every access in the shared state space (LDS/STS, not generic LD/ST).
    extern __shared__ __align__(1024) uint32_t smem_words[];
    constexpr uint32_t NS = (uint32_t)kStages;  // tile buffers: tile it in buffer it % NS
    uint32_t* stage = smem_words;
    uint64_t* bar = reinterpret_cast<uint64_t*>(stage + NS * TWORDS);
    uint2* tws = reinterpret_cast<uint2*>(bar + 4);
    const uint32_t tid = threadIdx.x;
    const TmaArgs& a = args;
    uint32_t t, t_end, t_step;
    if constexpr (LSTAGE) {  // contiguous range per CTA
      const uint32_t per = (a.ntiles + gridDim.x - 1) / gridDim.x;
      t = blockIdx.x * per;
      t_end = (t + per < a.ntiles) ? t + per : a.ntiles;
      t_step = 1;
    } else {
      t = blockIdx.x;
      t_end = a.ntiles;
      t_step = gridDim.x;
    }
    if (t >= t_end) return;
    if constexpr (kStaged) stage_twiddles(tws, a.tw, tid);
    if (tid == 0) {
      tma::prefetch_map(min);
      tma::prefetch_map(mout);
      for (uint32_t b = 0; b < NS; ++b) tma::mbar_init(&bar[b], 1);
      tma::fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
      for (uint32_t b = 0; b + 1 < NS; ++b) {  // tiles 0 .. NS-2 of this CTA
        const uint32_t tb = t + b * t_step;
        if (tb < t_end) {
          tma::mbar_expect_tx(&bar[b], TBYTES);
          tma_load(min, geo_run(a, tb), stage + b * TWORDS, &bar[b]);
        }
      }
    }
    uint32_t v[E];
    uint32_t staged = ~0u;  // chunk whose twiddles are in shared memory (LSTAGE)
    for (uint32_t it = 0; t < t_end; t += t_step, ++it) {
      const uint32_t buf = it % NS;
      uint32_t* cur = stage + buf * TWORDS;
      const uint32_t tn = t + (NS - 1u) * t_step;  // the tile NS-1 ahead, into the buffer tile it-1 used
      if (tid == 0 && tn < t_end) {
        const uint32_t nb = (it + NS - 1u) % NS;
        tma::wait_reads();  // the store of tile it-1 (the last one issued) has read that buffer
        tma::mbar_expect_tx(&bar[nb], TBYTES);
        tma_load(min, geo_run(a, tn), stage + nb * TWORDS, &bar[nb]);
      }
      const Geo g = geo_run(a, t);
      if constexpr (LSTAGE) {
        // Every thread passed the previous tile's pre-store barrier after its
        // last twiddle read; the barrier here publishes the new copy (the
        // positions are a function of t, the same for the whole CTA).
        const uint32_t key = (KD == Kind::C) ? g.pos_base : ((uint32_t)g.s1 >> 1);
        if (key != staged) {
          if constexpr (kStageThreadOrder) {
            stage_ctile(reinterpret_cast<uint32_t*>(tws), a, g.pos_base, tid);
          } else if constexpr (KD == Kind::C) {
            stage_ctile_plain(reinterpret_cast<uint32_t*>(tws), a, g.pos_base, tid);
          } else {  // both chunks of the pair
            stage_lchunk(tws, a.tw, a.lo, 2u * key, tid);
            stage_lchunk(tws + LCHUNK_ENTRIES, a.tw, a.lo, 2u * key + 1u, tid);
          }
          staged = key;
          __syncthreads();
        }
      }
      // A wait that ran out is agreed on at the barrier before the store:
      // the rounds in between touch only in-bounds shared memory and
      // twiddles whatever the tile holds, and every thread takes the same
      // barriers, so no extra CTA-wide barrier is needed per tile.
      const bool ok = tma::mbar_wait(&bar[buf], (it / NS) & 1u, kWaitNs);
      ld<kFirst>(cur, v, tid);
      if constexpr (DESC && TW) twist<kFirst>(v, a, g, tid);
      if constexpr (LSTAGE && KD == Kind::S)
        rounds<0>(cur, v, a, tws + ((uint32_t)g.s1 & 1u) * LCHUNK_ENTRIES, g, tid);
      else
        rounds<0>(cur, v, a, tws, g, tid);
      finish(v, a, g, tid);
      st<kLast>(cur, v, tid);
      tma::fence_proxy_async();
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(a.err, 1);
          for (uint32_t d = 1; d < NS; ++d)  // the loads in flight: tiles it+1 .. it+NS-1
            if (t + d * t_step < t_end) tma::mbar_wait(&bar[(it + d) % NS], ((it + d) / NS) & 1u, kWaitNs);
          tma::wait_all();
        }
        return;
      }
      if (tid == 0) {
        tma_store(mout, g, cur);
        tma::commit();
      }
    }
    if (tid == 0) tma::wait_all();
  }
};

// Exchange groups of the 12- and 8-layer contiguous passes and the 8-layer
// strided pass (checked against a brute-force walk over every tile word).
static_assert(TPass<BabyBear, true, Kind::C, 12>::xfixed<2, 1>() == 0x10F, "C12 2->1: tid bits 0-3, 8");
static_assert(TPass<BabyBear, true, Kind::C, 12>::xfixed<1, 0>() == 0x1F0, "C12 1->0: tid bits 4-8 (in a warp)");
static_assert(TPass<BabyBear, false, Kind::C, 8>::xfixed<0, 1>() == 0x1F0, "C8 0->1: in a warp");
static_assert(TPass<BabyBear, false, Kind::S, 8>::xfixed<0, 1>() == 0x1F, "S8: lanes only, whole CTA");
static_assert(TPass<BabyBear, false, Kind::C, 12>::shfl_swap(0, 1) && TPass<BabyBear, true, Kind::C, 12>::shfl_swap(1, 0) &&
                  TPass<BabyBear, false, Kind::C, 8>::shfl_swap(0, 1) && !TPass<BabyBear, false, Kind::C, 12>::shfl_swap(1, 2) &&
                  !TPass<BabyBear, false, Kind::S, 8>::shfl_swap(0, 1),
              "warp-local exchanges of the shuffle form");
// the 11-layer pass's filler (see filler_hint): a grouped exchange and independent halves
static_assert(TPass<BabyBear, false, Kind::C, 11>::xgroups(1, 2) == 2 && TPass<BabyBear, false, Kind::C, 11>::halves_ok(),
              "filler choice of the 11-layer pass");
// 14-layer passes: a warp-local exchange, then two grouped ones (4 groups each)
static_assert(TPass<BabyBear, false, Kind::C, 14>::xgroups(0, 1) == 0 && TPass<BabyBear, false, Kind::C, 14>::xgroups(1, 2) == 4 &&
                  TPass<BabyBear, false, Kind::C, 14>::xgroups(2, 3) == 4 && TPass<BabyBear, false, Kind::C, 14>::xbase(3) == 5 &&
                  TPass<BabyBear, false, Kind::C, 14>::xfixed<0, 1>() >= 0,
              "C14 exchanges: warp, 4 groups, 4 groups");
// 13-layer passes: two grouped exchanges in a row (4 groups each), on disjoint ids
static_assert(TPass<BabyBear, false, Kind::C, 13>::xgroups(1, 2) == 4 && TPass<BabyBear, false, Kind::C, 13>::xgroups(2, 3) == 4 &&
                  TPass<BabyBear, false, Kind::C, 13>::xbase(3) == 5 && TPass<BabyBear, true, Kind::C, 13>::xbase(2) == 5,
              "C13 exchange barrier ids");

// BabyBear LSTAGE passes stage 64 KiB of twiddles besides the two tiles (one
// CTA per SM); M31 contiguous ones 32 KiB (two).
template <class F, bool DESC, Kind KD, int P, bool PLAIN, bool TW, bool LSTAGE = false, bool HALVES = false>
__global__ void __launch_bounds__(TPass<F, DESC, KD, P, PLAIN, TW, LSTAGE, HALVES>::NT,
                                  TPass<F, DESC, KD, P, PLAIN, TW, LSTAGE, HALVES>::kCtasPerSm)
tma_pass_kernel(const __grid_constant__ CUtensorMap min, const __grid_constant__ CUtensorMap mout, TmaArgs a) {
  pdl_enter();
  TPass<F, DESC, KD, P, PLAIN, TW, LSTAGE, HALVES>::run(&min, &mout, a);
}

// ---------------------------------------------------------------------------
// Fused LDE middle step on Kind::S tiles (P <= 8, lo = log_n - P): inverse
// layers [lo, log_n), then for each output block q forward layers [lo, log_n)
// of the extended network (the block's tiles sit in high block q of it);
// block q goes to rows [q n, (q+1) n) of the extended column.
//   BabyBear: before block q's forward layers, the multiplier M_q[pos] (n^-1,
//     coset shift, zero-padded top layers).
//   M31: the inverse result times n^-1 once; the zero-padded top forward layers
//     are a plain replication (CT butterfly on (a, 0) gives (a, a)), so every
//     block starts from the same values.
// The inverse result stays in registers across the blocks.
// LSTAGE (BabyBear, per-position twiddles): each CTA takes a contiguous range
// of tiles; tiles are numbered column-fastest, so consecutive tiles share a
// 32-position chunk and its twiddles, which are staged in shared memory
// (both directions, 2 x 64 KB for P = 8) whenever the chunk changes.
template <class F, int P, bool PLAIN, bool LSTAGE = false>
struct TExpand {
  using Inv = TPass<F, false, Kind::S, P, PLAIN, false, LSTAGE>;
  using Fwd = TPass<F, true, Kind::S, P, PLAIN, false, LSTAGE>;
  static constexpr int K = Inv::K, E = Inv::E, NT = Inv::NT, R = Inv::R, LT = Inv::LT;
  static constexpr uint32_t TWORDS = Inv::TWORDS, TBYTES = Inv::TBYTES;
  static constexpr uint32_t TW_ENTRIES = LSTAGE ? Inv::LCHUNK_ENTRIES : Inv::TW_ENTRIES;  // per direction
  static_assert(F::kMontgomery || !PLAIN, "M31 passes have no plain variant");
  // M31 stages no twiddles (3 x 32 KiB of shared memory) and fits 64 registers:
  // two CTAs per SM; BabyBear / KoalaBear keep their multipliers in registers
  // one block ahead and stage per-position twiddles, one CTA per SM.  The
  // four-step (PLAIN) form stages only the 2 x 255 lane-independent twiddles
  // and loads each multiplier where it is used, so it too fits 64 registers
  // and two CTAs per SM.
  static constexpr int kCtasPerSm = (F::kMontgomery && !PLAIN) ? 1 : 2;

  // Multipliers M_q of the thread's 16 slots (round K-1 layout).  The table is
  // in tile order (kind 2: entry q n + chunk 2^13 + c for tile word c of the
  // chunk's tiles), so from mq = table + q n + chunk 2^13 + ctid every slot is
  // a compile-time offset (its tile bits), and each slot's load is a
  // contiguous 256-byte run across a warp.
  __device__ static __forceinline__ void load_mul(uint2 (&w)[E], const uint2* mq) {
    using M = RM<Kind::S, P, LT, R, K - 1>;
#pragma unroll
    for (int m = 0; m < E; ++m) w[m] = __ldg(mq + M::cm(m));
  }

  // LSTAGE: the 32-position chunk of tile t, whose per-position twiddles the
  // tile reads from shared memory (tiles are numbered column-fastest).
  __device__ static __forceinline__ uint32_t chunk_of(const TmaArgs& ai, uint32_t t) {
    return (t / ai.batch) & ((1u << (ai.lo - 5)) - 1u);
  }

  // One input tile (in `cur`; ok: it arrived) through the inverse layers, then
  // for every output block q the multipliers and forward layers, each block
  // leaving with its own TMA store (block 0 from cur, block 1 from ostage,
  // alternating).  A wait that ran out is agreed on at the barrier before the
  // first store (the inverse and the first block touch only in-bounds shared
  // memory, twiddles and multipliers whatever the tile holds): then nothing is
  // stored and the result is false.
  //
  // BabyBear / KoalaBear with two or more output blocks run them in pairs
  // (tile_body_pairs): blocks 2p and 2p+1 share their forward exchange, their
  // pre-store barrier and every twiddle load of their second forward round.
  // Requires the caller's thread 0 to have waited for the reads of every
  // earlier store (cp.async.bulk.wait_group.read 0) before the tile's first
  // barrier, since block 1 writes ostage without a barrier of its own.
  __device__ static __forceinline__ bool tile_body(uint32_t* cur, uint32_t* ostage, const TmaArgs& ai,
                                                   const uint2* tws_inv, const uint2* tws_fwd, uint32_t t, bool ok,
                                                   const CUtensorMap* mout, uint32_t tid) {
#ifndef SFNTT_NO_X_PAIRS  // (build-time switch for comparisons: one block at a time)
    if constexpr (F::kMontgomery && K == 2 && !PLAIN) {
      if (ai.log_q >= 1) return tile_body_pairs(cur, ostage, ai, tws_inv, tws_fwd, t, ok, mout, tid);
    }
#endif
    using M = RM<Kind::S, P, LT, R, K - 1>;
    const uint32_t ct = M::ctid(tid);
    const uint32_t n = 1u << ai.log_n;
    const uint32_t nq = 1u << ai.log_q;
    uint32_t x[E], v[E];
    const typename Inv::Geo g = Inv::geo(ai, t);
    const uint2* mt = ai.mul + ((uint32_t)g.s1 << kTileBits) + ct;  // this thread's multipliers of block 0
    // BabyBear multipliers are software-pipelined: block q+1's are loaded
    // while block q's forward layers run (block 0's during the inverse); the
    // four-step form loads them where they are used (registers for 2 CTAs).
    constexpr bool kPrefetch = F::kMontgomery && !PLAIN;
    uint2 w[kPrefetch ? E : 1];
    if constexpr (kPrefetch) load_mul(w, mt);
    Inv::template ld<0>(cur, x, tid);
    Inv::template rounds<0>(cur, x, ai, tws_inv, g, tid);  // x: round K-1 layout
    if constexpr (!F::kMontgomery) {
#pragma unroll
      for (int m = 0; m < E; ++m) x[m] = mul_shoup<F>(x[m], ai.scale_w, ai.scale_ws);  // n^-1
    }
    for (uint32_t q = 0; q < nq; ++q) {
      uint32_t* ob = (q & 1u) ? ostage : cur;
      // The TMA store that last read ob is the one before the newest pending
      // store (for q = 1: the previous tile's last ostage store, which no
      // prefetch wait covers on a CTA's last tile).
      if (q >= 1) {
        if (tid == 0) tma::wait_reads_1();
        __syncthreads();
      }
      if constexpr (kPrefetch) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = mul_shoup<F>(x[m], w[m].x, w[m].y);
        if (q + 1 < nq) load_mul(w, mt + (uint64_t)(q + 1) * n);
      } else if constexpr (F::kMontgomery) {
        using MK = RM<Kind::S, P, LT, R, K - 1>;
        const uint2* mq = mt + (uint64_t)q * n;
#pragma unroll
        for (int m = 0; m < E; ++m) {
          const uint2 wm = __ldg(mq + MK::cm(m));
          v[m] = mul_shoup<F>(x[m], wm.x, wm.y);
        }
      } else {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = x[m];
      }
      typename Inv::Geo gq = g;
      gq.hb = q;  // high block of the extended network (M31 per-block twiddles)
      Fwd::template rounds<0>(ob, v, fwd_args(ai), tws_fwd, gq, tid);  // forward starts in round K-1's layout
      if constexpr (!Net<F, true>::kGS) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = reduce2p<F>(v[m]);  // lazy CT values to [0, p)
      }
      Fwd::template st<0>(ob, v, tid);
      tma::fence_proxy_async();
      if (q == 0) {
        if (__syncthreads_or(!ok)) return false;
      } else {
        __syncthreads();
      }
      if (tid == 0) {
        tma::store_5d(mout, 0, g.s1, 0, (int32_t)q, g.s4, ob);
        tma::commit();
      }
    }
    return true;
  }

  __device__ static __forceinline__ bool tile_body_pairs(uint32_t* cur, uint32_t* ostage, const TmaArgs& ai,
                                                         const uint2* tws_inv, const uint2* tws_fwd, uint32_t t,
                                                         bool ok, const CUtensorMap* mout, uint32_t tid) {
    using M = RM<Kind::S, P, LT, R, K - 1>;
    const uint32_t ct = M::ctid(tid);
    const uint32_t n = 1u << ai.log_n;
    const uint32_t nq = 1u << ai.log_q;
    const typename Inv::Geo g = Inv::geo(ai, t);
    const uint2* mt = ai.mul + ((uint32_t)g.s1 << kTileBits) + ct;  // this thread's multipliers of block 0
    const FwdArgs af = fwd_args(ai);
    uint32_t x[E];
    uint2 w[E];
    load_mul(w, mt);  // block 0's multipliers, in flight during the inverse layers
    Inv::template ld<0>(cur, x, tid);
    Inv::template rounds<0>(cur, x, ai, tws_inv, g, tid);  // x: round K-1 layout
    for (uint32_t q = 0; q < nq; q += 2) {
      // blocks q (from cur) and q+1 (from ostage): the stores that last read
      // them are the previous pair's (for q = 0 the previous tile's, whose
      // reads thread 0 waited for before the inverse layers' barrier)
      if (q >= 2) {
        load_mul(w, mt + (uint64_t)q * n);  // (4x and up: not prefetched, to save registers)
        if (tid == 0) tma::wait_reads();
        __syncthreads();
      }
      uint32_t va[E], vb[E];
#pragma unroll
      for (int m = 0; m < E; ++m) va[m] = mul_shoup<F>(x[m], w[m].x, w[m].y);
      load_mul(w, mt + (uint64_t)(q + 1) * n);  // in flight during block q's first round
      Fwd::template round<K - 1>(va, af, tws_fwd, g, tid);
#pragma unroll
      for (int m = 0; m < E; ++m) vb[m] = mul_shoup<F>(x[m], w[m].x, w[m].y);
      Fwd::template round<K - 1>(vb, af, tws_fwd, g, tid);
      Fwd::template st<K - 1>(cur, va, tid);
      Fwd::template st<K - 1>(ostage, vb, tid);
      __syncthreads();  // the exchange of both blocks (strided tiles exchange across the CTA)
      Fwd::template ld<0>(cur, va, tid);
      Fwd::template ld<0>(ostage, vb, tid);
      Fwd::template round2<0>(va, vb, af, tws_fwd, g, tid);
      Fwd::template st<0>(cur, va, tid);
      Fwd::template st<0>(ostage, vb, tid);
      tma::fence_proxy_async();
      if (q == 0) {
        if (__syncthreads_or(!ok)) return false;
      } else {
        __syncthreads();
      }
      if (tid == 0) {
        tma::store_5d(mout, 0, g.s1, 0, (int32_t)q, g.s4, cur);
        tma::store_5d(mout, 0, g.s1, 0, (int32_t)q + 1, g.s4, ostage);
        tma::commit();
      }
    }
    return true;
  }

  __device__ static void run(const CUtensorMap* min, const CUtensorMap* mout, const TmaArgs& args) {
    // Dynamic shared memory is 1024-byte aligned; indexing it directly keeps
    // every access in the shared state space (LDS/STS, not generic LD/ST).
    extern __shared__ __align__(1024) uint32_t smem_words[];
    uint32_t* stage = smem_words;
    uint32_t* ostage = stage + 2 * TWORDS;
    uint64_t* bar = reinterpret_cast<uint64_t*>(stage + 3 * TWORDS);
    uint2* tws_inv = reinterpret_cast<uint2*>(bar + 2);
    uint2* tws_fwd = tws_inv + TW_ENTRIES;
    const uint32_t tid = threadIdx.x;
    const TmaArgs& ai = args;
    uint32_t t, t_end, t_step;
    if constexpr (LSTAGE) {  // contiguous range per CTA
      const uint32_t per = (ai.ntiles + gridDim.x - 1) / gridDim.x;
      t = blockIdx.x * per;
      t_end = (t + per < ai.ntiles) ? t + per : ai.ntiles;
      t_step = 1;
    } else {
      t = blockIdx.x;
      t_end = ai.ntiles;
      t_step = gridDim.x;
    }
    if (t >= t_end) return;
    if constexpr (PLAIN) {
      Inv::stage_twiddles(tws_inv, ai.tw, tid);
      Fwd::stage_twiddles(tws_fwd, ai.tw_fwd, tid);
    }
    if (tid == 0) {
      tma::prefetch_map(min);
      tma::prefetch_map(mout);
      tma::mbar_init(&bar[0], 1);
      tma::mbar_init(&bar[1], 1);
      tma::fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
      tma::mbar_expect_tx(&bar[0], TBYTES);
      Inv::tma_load(min, Inv::geo(ai, t), stage, &bar[0]);
    }
    uint32_t staged = ~0u;  // chunk whose twiddles are in shared memory (LSTAGE)
    for (uint32_t it = 0; t < t_end; t += t_step, ++it) {
      const uint32_t buf = it & 1u;
      uint32_t* cur = stage + buf * TWORDS;
      const uint32_t tn = t + t_step;
      if (tid == 0) {
        tma::wait_reads();  // every earlier store has read its buffer (tile_body relies on it)
        if (tn < t_end) {
          tma::mbar_expect_tx(&bar[buf ^ 1u], TBYTES);
          Inv::tma_load(min, Inv::geo(ai, tn), stage + (buf ^ 1u) * TWORDS, &bar[buf ^ 1u]);
        }
      }
      if constexpr (LSTAGE) {
        // Every thread passed the previous tile's last barrier after its last
        // twiddle read; the barrier here publishes the new copy (the chunk,
        // a function of t, is the same for the whole CTA).
        const uint32_t chunk = chunk_of(ai, t);
        if (chunk != staged) {
          Inv::stage_lchunk(tws_inv, ai.tw, ai.lo, chunk, tid);
          Fwd::stage_lchunk(tws_fwd, ai.tw_fwd, ai.lo, chunk, tid);
          staged = chunk;
          __syncthreads();
        }
      }
      const bool ok = tma::mbar_wait(&bar[buf], (it >> 1) & 1u, kWaitNs);
      if (!tile_body(cur, ostage, ai, tws_inv, tws_fwd, t, ok, mout, tid)) {
        if (tid == 0) {
          atomicExch(ai.err, 1);
          if (tn < t_end) tma::mbar_wait(&bar[buf ^ 1u], ((it + 1) >> 1) & 1u, kWaitNs);
          tma::wait_all();
        }
        return;
      }
    }
    if (tid == 0) tma::wait_all();
  }
};

// Natural-order LDE expansion (BabyBear / KoalaBear, 2x), the mirror image of
// TExpand for natural-order input and output rows.  The strided pass before it
// ran the inverse GS-DIF layers [12, log n) on the natural-order evaluations;
// per contiguous 2^13-word tile this kernel runs the inverse layers [0, 12)
// (GS-DIF, inverse table), which leaves n * coefficient rev(p) at position p,
// then for each coset r in {0, 1}: multiplies by M_r[p] = n^-1 (shift
// g_ext^r)^rev(p) and runs the forward CT-DIT layers [0, 12) of the n-point
// network (forward table).  Coset r's word p belongs at extended position
// 2p + r, so both cosets are interleaved in shared memory and the tile leaves
// as 2^14 contiguous words; the strided pass after it runs the DIT layers
// [12, log n) of every coset on the interleaved column.  The inverse ends and
// the forward starts in round 0's layout, so the coefficients stay in
// registers.
template <class F>
struct TExpandC {
  using Inv = TPass<F, true, Kind::C, 12>;
  using Fwd = TPass<F, false, Kind::C, 12>;
  static constexpr int K = Inv::K, E = Inv::E, NT = Inv::NT, R = Inv::R, LT = Inv::LT;
  static constexpr uint32_t TWORDS = Inv::TWORDS, TBYTES = Inv::TBYTES;
  static constexpr uint32_t TW_ENTRIES = Inv::TW_ENTRIES;  // per direction
  static_assert(F::kMontgomery, "natural-order expansion: BabyBear / KoalaBear");
  static_assert(Inv::kLast == 0 && Fwd::kFirst == 0, "inverse ends and forward starts in round 0's layout");
  using ML = RM<Kind::C, 12, LT, R, K - 1>;

  // Multipliers of the thread's slots (round 0 layout: tile word 16 tid + m)
  // from mq = M_r + pos_base; the table stores word 16 t + m of a tile at
  // m * NT + t, so each slot's load is coalesced across the CTA.
  static_assert(NT == 512 && E == 16, "tile word of round-0 slot m is 16 tid + m");
  __device__ static __forceinline__ void load_mul(uint2 (&w)[E], const uint2* mq, uint32_t tid) {
#pragma unroll
    for (int m = 0; m < E; ++m) w[m] = __ldg(mq + (uint32_t)m * NT + tid);
  }

  // coset r's values (round K-1 layout, canonical) to the interleaved output tile
  __device__ static __forceinline__ void put(uint32_t* ostage, const uint32_t (&v)[E], uint32_t ctl, uint32_t r) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const uint32_t e = ((ctl | ML::cm(m)) << 1) | r;  // 14-bit extended word of the tile
      ostage[(e >> 13) * TWORDS + Inv::sw(e & (TWORDS - 1u))] = v[m];
    }
  }

  __device__ static void run(const CUtensorMap* min, const CUtensorMap* mout, const TmaArgs& args) {
    extern __shared__ __align__(1024) uint32_t smem_words[];
    uint32_t* stage = smem_words;           // 2 x TWORDS: input tiles (double-buffered)
    uint32_t* ostage = stage + 2 * TWORDS;  // 2 x TWORDS: the tile's two output halves
    uint64_t* bar = reinterpret_cast<uint64_t*>(ostage + 2 * TWORDS);
    uint2* tws_inv = reinterpret_cast<uint2*>(bar + 2);
    uint2* tws_fwd = tws_inv + TW_ENTRIES;
    const uint32_t tid = threadIdx.x;
    const TmaArgs& a = args;
    uint32_t t = blockIdx.x;
    if (t >= a.ntiles) return;
    Inv::stage_twiddles(tws_inv, a.tw, tid);
    Fwd::stage_twiddles(tws_fwd, a.tw_fwd, tid);
    if (tid == 0) {
      tma::prefetch_map(min);
      tma::prefetch_map(mout);
      tma::mbar_init(&bar[0], 1);
      tma::mbar_init(&bar[1], 1);
      tma::fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
      tma::mbar_expect_tx(&bar[0], TBYTES);
      Inv::tma_load(min, Inv::geo(a, t), stage, &bar[0]);
    }
    const uint32_t ctl = ML::ctid(tid);
    const uint64_t n = 1ull << a.log_n;
    uint32_t x[E], v[E];
    for (uint32_t it = 0; t < a.ntiles; t += gridDim.x, ++it) {
      const uint32_t buf = it & 1u;
      uint32_t* cur = stage + buf * TWORDS;
      const uint32_t tn = t + gridDim.x;
      if (tid == 0) {
        // The other input buffer was last read by this CTA's previous tile
        // (all threads are past its barriers); ostage, by the previous tile's
        // stores: wait for them here, the barrier before this tile's first
        // ostage write publishes it.
        tma::wait_reads();
        if (tn < a.ntiles) {
          tma::mbar_expect_tx(&bar[buf ^ 1u], TBYTES);
          Inv::tma_load(min, Inv::geo(a, tn), stage + (buf ^ 1u) * TWORDS, &bar[buf ^ 1u]);
        }
      }
      const bool ok = tma::mbar_wait(&bar[buf], (it >> 1) & 1u, kWaitNs);
      const typename Inv::Geo g = Inv::geo(a, t);
      uint2 w[E];
      load_mul(w, a.mul + g.pos_base, tid);  // coset 0's, in flight during the inverse layers
      Inv::template ld<Inv::kFirst>(cur, x, tid);
      Inv::template rounds<0>(cur, x, a, tws_inv, g, tid);  // x: round 0 layout, canonical
#pragma unroll
      for (uint32_t r = 0; r < 2; ++r) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = mul_shoup<F>(x[m], w[m].x, w[m].y);
        if (r == 0) load_mul(w, a.mul + n + g.pos_base, tid);  // coset 1's, during coset 0's layers
        Fwd::template rounds<0>(cur, v, a, tws_fwd, g, tid);
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = reduce2p<F>(v[m]);  // lazy CT values to [0, p)
        // coset 0: every thread is done exchanging through cur before coset 1
        // reuses it, and ostage is free (thread 0 waited at the tile start)
        if (r == 0) __syncthreads();
        put(ostage, v, ctl, r);
      }
      tma::fence_proxy_async();
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(a.err, 1);
          if (tn < a.ntiles) tma::mbar_wait(&bar[buf ^ 1u], ((it + 1) >> 1) & 1u, kWaitNs);
          tma::wait_all();
        }
        return;
      }
      if (tid == 0) {
        // extended rows [2 * pos_base, 2 * pos_base + 2^14) of the column, two boxes of 2^13 words
        Inv::c_store(mout, 2 * g.c1, g.c2, ostage, true);
        Inv::c_store(mout, 2 * g.c1 + (int32_t)(TWORDS / 32), g.c2, ostage + TWORDS, true);
        tma::commit();
      }
    }
    if (tid == 0) tma::wait_all();
  }
};

template <class F>
__global__ void __launch_bounds__(TExpandC<F>::NT, 1)
tma_expand_c_kernel(const __grid_constant__ CUtensorMap min, const __grid_constant__ CUtensorMap mout, TmaArgs a) {
  pdl_enter();
  TExpandC<F>::run(&min, &mout, a);
}

template <class F, int P, bool PLAIN, bool LSTAGE>
__global__ void __launch_bounds__(TExpand<F, P, PLAIN, LSTAGE>::NT, TExpand<F, P, PLAIN, LSTAGE>::kCtasPerSm)
tma_expand_kernel(const __grid_constant__ CUtensorMap min, const __grid_constant__ CUtensorMap mout, TmaArgs a) {
  pdl_enter();
  TExpand<F, P, PLAIN, LSTAGE>::run(&min, &mout, a);
}

}  // namespace sfntt
