// worklist.cu -- the persistent phase kernels of an uneven batch and the
// host code that lays out their work list.
//
// Items of either field (BabyBear, M31) with 2^13 .. 2^21 points per column
// and a blow-up of at most 16 run their LDE in three phases, each ONE launch
// over every such item of the batch:
//   phase 1: inverse layers [0, log n - 8) of every item (contiguous tiles),
//            input -> output columns;
//   phase 2: the expansion of every item: inverse layers [log n - 8, log n),
//            n^-1 / coset shift / zero-padded top layers, forward layers
//            [log n - 8, log n) of every output block (strided tiles);
//   phase 3: forward layers [0, log n - 8) of every item's extended network,
//            in place.
// The per-item kernels do exactly these three steps (lde.cu), so the tiles
// and every value in them are the same; only who runs which tile changes.
#include <algorithm>
#include <vector>

#include "context.hpp"
#include "host_field.hpp"
#include "tma_launch.cuh"
#include "worklist.cuh"

namespace sfntt {
namespace {

constexpr uint32_t kNoTile = 0xFFFFFFFFu;
constexpr uint32_t kBbStaged = 4095u;  // BabyBear twiddle layers [0, 12), staged once per CTA

// Thread 0's cursor over the work list (in shared memory): the unit it is
// consuming, c[0] its item, tiles [c[1], c[2]) still to hand out.
// The next tile of the work list for this CTA (thread 0 only): the rest of the
// current unit, else a freshly popped unit; false when the list is exhausted.
__device__ __forceinline__ bool next_tile(uint32_t* c, const WorkUnit* units, uint32_t n_units, uint32_t* counter,
                                          uint32_t& item, uint32_t& t) {
  if (c[1] >= c[2]) {
    const uint32_t u = atomicAdd(counter, 1u);
    if (u >= n_units) return false;
    const WorkUnit w = units[u];
    c[0] = w.item;
    c[1] = w.t0;
    c[2] = w.t1;
  }
  item = c[0];
  t = c[1]++;
  return true;
}

// ---------------------------------------------------------------- phase 1/3 --
template <bool DESC, class F, int P>
__device__ __forceinline__ void c_tile(uint32_t* cur, const TmaArgs& a, const uint2* tws, uint32_t t, uint32_t tid) {
  using T = TPass<F, DESC, Kind::C, P>;
  T::tile_body(cur, a, tws, T::geo(a, t), tid);
}

#define SFNTT_WL_C(FF, PP) \
  case PP: c_tile<DESC, FF, PP>(cur, a, tws, t, tid); break;

template <bool DESC>
__device__ __forceinline__ void c_dispatch(int field, int P, uint32_t* cur, const TmaArgs& a, const uint2* tws,
                                           uint32_t t, uint32_t tid) {
  if (field == SFNTT_BABYBEAR) {
    switch (P) {
      SFNTT_WL_C(BabyBear, 5) SFNTT_WL_C(BabyBear, 6) SFNTT_WL_C(BabyBear, 7) SFNTT_WL_C(BabyBear, 8)
      SFNTT_WL_C(BabyBear, 9) SFNTT_WL_C(BabyBear, 10) SFNTT_WL_C(BabyBear, 11) SFNTT_WL_C(BabyBear, 12)
      SFNTT_WL_C(BabyBear, 13)
      default: break;
    }
  } else {
    switch (P) {
      SFNTT_WL_C(M31, 5) SFNTT_WL_C(M31, 6) SFNTT_WL_C(M31, 7) SFNTT_WL_C(M31, 8)
      SFNTT_WL_C(M31, 9) SFNTT_WL_C(M31, 10) SFNTT_WL_C(M31, 11) SFNTT_WL_C(M31, 12) SFNTT_WL_C(M31, 13)
      default: break;
    }
  }
}
#undef SFNTT_WL_C

// TMA copies of an item's contiguous tiles.  The tile geometry is field- and
// layer-independent; the copy form is not: 8-, 11- and 12-layer passes keep
// their tiles row-permuted (a 5-dimensional map, half a tile per copy), the
// others in row order (a 3-dimensional map) -- c_row_perm decides both here
// and where worklist_add encodes the item's maps.
template <bool DESC>
struct CCopy {
  using Perm = TPass<BabyBear, DESC, Kind::C, 12>;
  using Rows = TPass<BabyBear, DESC, Kind::C, 10>;
  static_assert(Perm::kRowPerm && !Rows::kRowPerm, "one copy form each");
  __device__ static __forceinline__ void load(const WorkItem& w, uint32_t t, uint32_t* dst, uint64_t* bar) {
    if (c_row_perm(w.P)) Perm::tma_load(&w.min, Perm::geo(w.a, t), dst, bar);
    else Rows::tma_load(&w.min, Rows::geo(w.a, t), dst, bar);
  }
  __device__ static __forceinline__ void store(const WorkItem& w, uint32_t t, const uint32_t* src) {
    if (c_row_perm(w.P)) Perm::tma_store(&w.mout, Perm::geo(w.a, t), src);
    else Rows::tma_store(&w.mout, Rows::geo(w.a, t), src);
  }
};

// Contiguous passes of every item (layers [0, P_item) of its network):
// 2^13-word tiles, the same geometry for every layer count.
template <bool DESC>
__global__ void __launch_bounds__(512, 2)
worklist_c_kernel(const WorkItem* __restrict__ items, const WorkUnit* __restrict__ units, uint32_t n_units,
                  uint32_t* counter, const uint2* bb_tw) {
  using G = CCopy<DESC>;
  extern __shared__ __align__(1024) uint32_t smem_words[];
  uint32_t* stage = smem_words;
  uint64_t* bar = reinterpret_cast<uint64_t*>(stage + 2 * kTileWords);
  // slot [0, 2): item of buffer b; [2, 4): its tile; [4, 7): thread 0's cursor
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 2);
  uint32_t* cursor = slot + 4;
  uint2* tws = reinterpret_cast<uint2*>(slot + 8);
  const uint32_t tid = threadIdx.x;
  // BabyBear items share one (nested) table: layers [0, 12) staged once
  if (bb_tw)
    for (uint32_t i = tid; i < kBbStaged; i += 512u) tws[i] = __ldg(bb_tw + i);
  if (tid == 0) {
    cursor[1] = cursor[2] = 0;
    tma::mbar_init(&bar[0], 1);
    tma::mbar_init(&bar[1], 1);
    tma::fence_mbar_init();
    uint32_t item, t;
    if (next_tile(cursor, units, n_units, counter, item, t)) {
      const WorkItem& w = items[item];
      tma::mbar_expect_tx(&bar[0], kTileBytes);
      G::load(w, t, stage, &bar[0]);
      slot[0] = item;
      slot[2] = t;
    } else {
      slot[0] = kNoTile;
    }
  }
  __syncthreads();
  for (uint32_t it = 0;; ++it) {
    const uint32_t buf = it & 1u;
    const uint32_t item = slot[buf];
    if (item == kNoTile) break;
    const uint32_t t = slot[2 + buf];
    uint32_t* cur = stage + buf * kTileWords;
    bool issued = false;
    if (tid == 0) {
      // every thread read slot[buf ^ 1] (last iteration) before that iteration's barrier
      uint32_t ni, nt;
      if (next_tile(cursor, units, n_units, counter, ni, nt)) {
        tma::wait_reads();  // the store that last used the other buffer has read it
        const WorkItem& wn = items[ni];
        tma::mbar_expect_tx(&bar[buf ^ 1u], kTileBytes);
        G::load(wn, nt, stage + (buf ^ 1u) * kTileWords, &bar[buf ^ 1u]);
        slot[buf ^ 1u] = ni;
        slot[2 + (buf ^ 1u)] = nt;
        issued = true;
      } else {
        slot[buf ^ 1u] = kNoTile;
      }
    }
    const WorkItem& w = items[item];
    const bool ok = tma::mbar_wait(&bar[buf], (it >> 1) & 1u, kWaitNs);
    c_dispatch<DESC>(w.field, w.P, cur, w.a, tws, t, tid);
    tma::fence_proxy_async();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(w.a.err, 1);
        if (issued) tma::mbar_wait(&bar[buf ^ 1u], ((it + 1) >> 1) & 1u, kWaitNs);
        tma::wait_all();
      }
      return;
    }
    if (tid == 0) {
      G::store(w, t, cur);
      tma::commit();
    }
  }
  if (tid == 0) tma::wait_all();
}

// ------------------------------------------------------------------ phase 2 --
using XBbStaged = TExpand<BabyBear, 8, false, true>;
using XM31 = TExpand<M31, 8, false, false>;
static_assert(XBbStaged::TW_ENTRIES == XBbStaged::Inv::LCHUNK_ENTRIES, "staged chunk per direction");

// Expansions of every item (strided 8-layer tiles).  BabyBear items read their
// per-position twiddles from a staged 32-position chunk (restaged when the item
// or the chunk changes; units keep a chunk's columns together); M31 twiddles
// are uniform across a tile's lanes and come from L2.
__global__ void __launch_bounds__(512, 1)
worklist_x_kernel(const WorkItem* __restrict__ items, const WorkUnit* __restrict__ units, uint32_t n_units,
                  uint32_t* counter) {
  using G = XM31::Inv;  // strided tile geometry and TMA (field-independent)
  constexpr uint32_t TW = kTileWords;
  extern __shared__ __align__(1024) uint32_t smem_words[];
  uint32_t* stage = smem_words;
  uint32_t* ostage = stage + 2 * TW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(stage + 3 * TW);
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 2);  // as in worklist_c_kernel
  uint32_t* cursor = slot + 4;
  uint2* tws_inv = reinterpret_cast<uint2*>(slot + 8);
  uint2* tws_fwd = tws_inv + XBbStaged::TW_ENTRIES;
  const uint32_t tid = threadIdx.x;
  if (tid == 0) {
    cursor[1] = cursor[2] = 0;
    tma::mbar_init(&bar[0], 1);
    tma::mbar_init(&bar[1], 1);
    tma::fence_mbar_init();
    uint32_t item, t;
    if (next_tile(cursor, units, n_units, counter, item, t)) {
      const WorkItem& w = items[item];
      tma::mbar_expect_tx(&bar[0], kTileBytes);
      G::tma_load(&w.min, G::geo(w.a, t), stage, &bar[0]);
      slot[0] = item;
      slot[2] = t;
    } else {
      slot[0] = kNoTile;
    }
  }
  __syncthreads();
  uint32_t staged_item = kNoTile, staged_chunk = kNoTile;
  for (uint32_t it = 0;; ++it) {
    const uint32_t buf = it & 1u;
    const uint32_t item = slot[buf];
    if (item == kNoTile) break;
    const uint32_t t = slot[2 + buf];
    uint32_t* cur = stage + buf * TW;
    bool issued = false;
    if (tid == 0) {
      tma::wait_reads();  // every earlier store has read its buffer (the expansion's tile step relies on it)
      uint32_t ni, nt;
      if (next_tile(cursor, units, n_units, counter, ni, nt)) {
        const WorkItem& wn = items[ni];
        tma::mbar_expect_tx(&bar[buf ^ 1u], kTileBytes);
        G::tma_load(&wn.min, G::geo(wn.a, nt), stage + (buf ^ 1u) * TW, &bar[buf ^ 1u]);
        slot[buf ^ 1u] = ni;
        slot[2 + (buf ^ 1u)] = nt;
        issued = true;
      } else {
        slot[buf ^ 1u] = kNoTile;
      }
    }
    const WorkItem& w = items[item];
    if (w.lstage) {
      // every thread passed the previous tile's last barrier after its last
      // twiddle read; the barrier here publishes the new copy
      const uint32_t chunk = XBbStaged::chunk_of(w.a, t);
      if (item != staged_item || chunk != staged_chunk) {
        XBbStaged::Inv::stage_lchunk(tws_inv, w.a.tw, w.a.lo, chunk, tid);
        XBbStaged::Fwd::stage_lchunk(tws_fwd, w.a.tw_fwd, w.a.lo, chunk, tid);
        staged_item = item;
        staged_chunk = chunk;
        __syncthreads();
      }
    }
    const bool ok = tma::mbar_wait(&bar[buf], (it >> 1) & 1u, kWaitNs);
    bool good;
    if (w.field == SFNTT_BABYBEAR) {
      good = XBbStaged::tile_body(cur, ostage, w.a, tws_inv, tws_fwd, t, ok, &w.mout, tid);
    } else {
      good = XM31::tile_body(cur, ostage, w.a, tws_inv, tws_fwd, t, ok, &w.mout, tid);
    }
    if (!good) {
      if (tid == 0) {
        atomicExch(w.a.err, 1);
        if (issued) tma::mbar_wait(&bar[buf ^ 1u], ((it + 1) >> 1) & 1u, kWaitNs);
        tma::wait_all();
      }
      return;
    }
  }
  if (tid == 0) tma::wait_all();
}

constexpr int kSmemC = 2 * (int)kTileBytes + 16 + 32 + 8 * (int)kBbStaged + 1024;
constexpr int kSmemX = 3 * (int)kTileBytes + 16 + 32 + 16 * (int)XBbStaged::TW_ENTRIES + 1024;

// M31 contiguous passes of this layer count read their first round from the
// table's first-round copy (entry n on).
bool m31_round0_copy(bool desc, int P) {
  auto pick = [&](auto d) -> bool {
    constexpr bool D = decltype(d)::value;
    switch (P) {
      case 5: return TPass<M31, D, Kind::C, 5>::kRound0Copy;
      case 6: return TPass<M31, D, Kind::C, 6>::kRound0Copy;
      case 7: return TPass<M31, D, Kind::C, 7>::kRound0Copy;
      case 8: return TPass<M31, D, Kind::C, 8>::kRound0Copy;
      case 9: return TPass<M31, D, Kind::C, 9>::kRound0Copy;
      case 10: return TPass<M31, D, Kind::C, 10>::kRound0Copy;
      case 11: return TPass<M31, D, Kind::C, 11>::kRound0Copy;
      case 12: return TPass<M31, D, Kind::C, 12>::kRound0Copy;
      case 13: return TPass<M31, D, Kind::C, 13>::kRound0Copy;
      default: return false;
    }
  };
  return desc ? pick(std::true_type{}) : pick(std::false_type{});
}

void add_units(WorkPhase& ph, uint32_t item, uint32_t ntiles, uint32_t per) {
  for (uint32_t t = 0; t < ntiles; t += per) ph.units.push_back({item, t, std::min(ntiles, t + per)});
}

}  // namespace

// ------------------------------------------------------------------- host --
bool worklist_eligible(const sfntt_ctx* ctx, const sfntt_lde_item& it) {
  if (ctx->no_tma || it.batch == 0) return false;
  if (it.field != SFNTT_BABYBEAR && it.field != SFNTT_M31) return false;
  if (it.plan != SFNTT_PLAN_AUTO && it.plan != SFNTT_PLAN_TMA) return false;
  if (it.log_n < 13 || it.log_n > 21 || it.added_bits > 4) return false;
  if (it.field == SFNTT_BABYBEAR && ctx->lde_plain) return false;
  const uint64_t tiles = ((uint64_t)it.batch << it.log_n) >> kTileBits;
  if (tiles >= (1ull << 31)) return false;
  const int64_t cap = ctx->worklist_max_tiles < 0 ? 16 * (int64_t)ctx->sm_count : ctx->worklist_max_tiles;
  if (cap > 0 && tiles > (uint64_t)cap) return false;
  return aligned16(it.d_in) && aligned16(it.d_out);
}

// Appends item `it`'s pass of `phase` (0: inverse low layers, 1: expansion,
// 2: forward low layers) to ph, with the tables the per-item kernels use.
Status worklist_add(sfntt_ctx* ctx, WorkPhase& ph, int phase, const sfntt_lde_item& it, cudaStream_t s) {
  const bool bb = it.field == SFNTT_BABYBEAR;
  const uint32_t log_n = it.log_n, log_ext = it.log_n + it.added_bits, lo = it.log_n - 8;
  const uint64_t n = 1ull << log_n, n_ext = 1ull << log_ext;
  const uint2 *tw_inv = nullptr, *tw_fwd = nullptr;
  if (bb) {
    SFNTT_TRY(monty_twiddles(ctx, it.field, true, log_n, s, &tw_inv));
    SFNTT_TRY(monty_twiddles(ctx, it.field, false, log_ext, s, &tw_fwd));
  } else {
    SFNTT_TRY(m31_twiddles(ctx, true, log_n, s, &tw_inv));
    SFNTT_TRY(m31_twiddles(ctx, false, log_ext, s, &tw_fwd));
  }
  WorkItem w{};
  w.field = it.field;
  TmaArgs& a = w.a;
  a.err = ctx->err.as<int>();
  a.batch = it.batch;
  a.ntiles = (uint32_t)(((uint64_t)it.batch * n) >> kTileBits);
  uint32_t per = 8;  // tiles per unit
  if (phase == 1) {
    w.P = 8;
    SFNTT_TRY(encode_s_map(&w.min, it.d_out, lo, 8, 1, n, n_ext, it.batch));
    SFNTT_TRY(encode_s_map(&w.mout, it.d_out, lo, 8, 1ull << it.added_bits, n, n_ext, it.batch));
    a.tw = tw_inv;
    a.tw_fwd = tw_fwd;
    a.log_n = log_n;
    a.lo = lo;
    a.log_q = it.added_bits;
    if (bb) {
      const uint2* mul = nullptr;
      SFNTT_TRY(monty_lde_table(ctx, it.field, log_n, it.added_bits, it.shift_monty, 2, s, &mul));
      a.mul = mul;
      // BabyBear expansions read their per-position twiddles from a staged
      // 32-position chunk (restaged when the item or chunk changes): a unit
      // is one chunk's tiles of up to 32 columns
      w.lstage = 1u;
      {
        const uint32_t chunks = 1u << (lo - 5);
        const uint32_t cols_per = std::min<uint32_t>(it.batch, 32u);
        for (uint32_t c = 0; c < chunks; ++c)
          for (uint32_t c0 = 0; c0 < it.batch; c0 += cols_per)
            ph.units.push_back({(uint32_t)ph.items.size(), c * it.batch + c0,
                                c * it.batch + std::min(it.batch, c0 + cols_per)});
        ph.items.push_back(w);
        return {};
      }
    } else {
      a.scale_w = inv_n_of(SFNTT_M31, log_n);
      a.scale_ws = (uint32_t)(((uint64_t)a.scale_w << 32) / M31::P);
    }
  } else {
    const bool desc = phase == 2;
    w.P = (int32_t)lo;
    const uint32_t lg = desc ? log_ext : log_n;
    const uint64_t nn = 1ull << lg;
    const uint32_t* in = desc ? it.d_out : it.d_in;
    const uint64_t in_stride = desc ? n_ext : n;
    SFNTT_TRY(encode_c_map(&w.min, in, lg, in_stride, it.batch, (int)lo));
    SFNTT_TRY(encode_c_map(&w.mout, it.d_out, lg, n_ext, it.batch, (int)lo));
    a.tw = desc ? tw_fwd : tw_inv;
    a.log_n = lg;
    a.lo = 0;
    a.spans = 0;
    a.log_tpc = lg - kTileBits;
    a.ntiles = (uint32_t)(((uint64_t)it.batch * nn) >> kTileBits);
    if (!bb && m31_round0_copy(desc, (int)lo)) a.tw0 = a.tw + nn;  // M31 tables with n >= 2^13 carry it
    if (bb) {
      if (ph.bb_tw && ph.bb_tw != a.tw) return {SFNTT_INVALID_ARGUMENT, "work list: BabyBear tables differ"};
      ph.bb_tw = a.tw;
    }
  }
  add_units(ph, (uint32_t)ph.items.size(), a.ntiles, per);
  ph.items.push_back(w);
  return {};
}

// Launches phase `phase` over ph's work list (device copies in items / units,
// counter zeroed before the launch).
Status worklist_launch(sfntt_ctx* ctx, int phase, const WorkPhase& ph, const WorkItem* items, const WorkUnit* units,
                       uint32_t* counter, cudaStream_t s) {
  if (ph.units.empty()) return {};
  const uint32_t n_units = (uint32_t)ph.units.size();
  uint64_t tiles = 0;
  for (const WorkUnit& u : ph.units) tiles += u.t1 - u.t0;
  uint64_t bytes = 0;
  for (const WorkItem& w : ph.items) {
    const uint64_t words = (uint64_t)w.a.ntiles << kTileBits;
    bytes += phase == 1 ? words * 4u * (1u + (1u << w.a.log_q)) : words * 8u;
  }
  if (phase == 1) {
    static std::atomic<uint64_t> done{0};
    SFNTT_TRY(smem_limit_once(worklist_x_kernel, kSmemX, ctx->device, done));
    const uint32_t grid = (uint32_t)std::min<uint64_t>(tiles, (uint64_t)ctx->sm_count);
    launch_begin(ctx, s);
    worklist_x_kernel<<<grid, 512, kSmemX, s>>>(items, units, n_units, counter);
    return launch_check(ctx, "worklist_expand", s, bytes);
  }
  const uint32_t grid = (uint32_t)std::min<uint64_t>(tiles, 2ull * (uint64_t)ctx->sm_count);
  if (phase == 0) {
    static std::atomic<uint64_t> done{0};
    SFNTT_TRY(smem_limit_once(worklist_c_kernel<false>, kSmemC, ctx->device, done));
    launch_begin(ctx, s);
    worklist_c_kernel<false><<<grid, 512, kSmemC, s>>>(items, units, n_units, counter, ph.bb_tw);
    return launch_check(ctx, "worklist_inv_C", s, bytes);
  }
  static std::atomic<uint64_t> done{0};
  SFNTT_TRY(smem_limit_once(worklist_c_kernel<true>, kSmemC, ctx->device, done));
  launch_begin(ctx, s);
  worklist_c_kernel<true><<<grid, 512, kSmemC, s>>>(items, units, n_units, counter, ph.bb_tw);
  return launch_check(ctx, "worklist_fwd_C", s, bytes);
}

}  // namespace sfntt
