// cluster_ntt.cu -- one-launch NTT of columns of 2^13 .. 2^16 points on a
// thread-block cluster.
//
// A column of n = 2^(12+X) points is split over CS = 2^(X-1) CTAs of one
// cluster, CTA r owning the contiguous positions [r 2^13, (r+1) 2^13) in
// shared memory.  Layers [0, 12) pair positions inside a 2^13-word block and
// run on the tile engine's rounds (TPass<F, DESC, Kind::C, 12>: registers,
// shared-memory exchanges, staged BabyBear twiddles or the M31 first-round
// copy).  The X cross layers [12, 12+X) pair positions 2^12 apart: the points
// {base + k 2^12 : k < 2^X} (base < 2^12) form one group, and each thread owns
// 16 / 2^X whole groups, so these layers run in registers.  The exchange
// between the two parts goes through distributed shared memory: point k of a
// group lives in CTA k >> 1 at word base + (k & 1) 2^12.
//
//   inverse (layers ascending): load the block, in-block layers, cluster
//     barrier, gather the groups from the cluster's blocks, cross layers and
//     n^-1, store the groups (consecutive threads own consecutive bases:
//     coalesced); a second cluster barrier, split around the last two steps,
//     keeps every block alive until the others have read it.
//   forward (layers descending): load the groups, cross layers, scatter them
//     into the owning blocks, cluster barrier, in-block layers, store the block.
//
// Every global read of a column happens before the cluster's first barrier and
// every global write after it, so the transform works in place.  The
// persistent TMA passes need two launches for these sizes (about 4.5 us each
// for one column); this is one.
#include <cooperative_groups.h>

#include "context.hpp"
#include "pdl.cuh"
#include "tile_tma.cuh"

namespace sfntt {
namespace {

namespace cg = cooperative_groups;

template <class F, bool DESC, int X>
struct ClusterNtt {
  using TP = TPass<F, DESC, Kind::C, 12>;
  static constexpr int CS = 1 << (X - 1);  // CTAs per column
  static constexpr int G = 1 << X;         // points per cross group
  static constexpr int GPT = 16 / G;       // groups per thread
  static constexpr uint32_t NT = TP::NT;
  static constexpr uint32_t LOG_N = 12 + X;
  static constexpr uint32_t BASES = 4096u / CS;  // group bases per CTA
  static_assert(NT == 512 && TP::E == 16 && BASES == GPT * NT, "one thread: 16 points in whole groups");

  // Twiddle of the cross butterfly whose lower point is k (bit j clear) of the
  // group at `base`, layer L = 12 + j: BabyBear / KoalaBear tw[L][pos mod 2^L],
  // M31 tw[L][pos >> (L+1)] (the same for every base).
  __device__ static __forceinline__ uint2 cross_tw(const uint2* tw, uint32_t base, int k, int j) {
    const uint32_t L = 12u + (uint32_t)j;
    if constexpr (F::kMontgomery) {
      return __ldg(tw + ((1u << L) - 1u) + base + ((uint32_t)(k & ((1 << j) - 1)) << 12));
    } else {
      const uint32_t n = 1u << LOG_N;
      return __ldg(tw + (n - (n >> L)) + ((uint32_t)k >> (j + 1)));
    }
  }

  // The X cross layers on the thread's groups (forward: descending, inverse:
  // ascending, then n^-1); canonical values out.
  __device__ static __forceinline__ void cross(uint32_t (&v)[16], uint32_t base0, const uint2* tw, uint32_t scale_w,
                                               uint32_t scale_ws) {
#pragma unroll
    for (int gi = 0; gi < GPT; ++gi) {
      const uint32_t base = base0 + (uint32_t)gi * NT;
#pragma unroll
      for (int jj = 0; jj < X; ++jj) {
        const int j = DESC ? (X - 1 - jj) : jj;
#pragma unroll
        for (int k = 0; k < G; ++k) {
          if (k & (1 << j)) continue;
          butterfly<F, DESC>(v[gi * G + k], v[gi * G + (k | (1 << j))], cross_tw(tw, base, k, j));
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      if constexpr (!DESC) v[m] = mul_shoup<F>(v[m], scale_w, scale_ws);
      else if constexpr (!Net<F, true>::kGS) v[m] = reduce2p<F>(v[m]);  // lazy CT values to [0, p)
    }
  }

  __device__ static void run(uint32_t* d, const uint2* tw, uint32_t scale_w, uint32_t scale_ws) {
    extern __shared__ __align__(1024) uint32_t smem_words[];
    uint32_t* tile = smem_words;                                // the block, in TP's swizzled layout
    uint2* tws = reinterpret_cast<uint2*>(tile + kTileWords);  // BabyBear / KoalaBear layers [0, 12)
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank();
    const uint32_t tid = threadIdx.x;
    const uint64_t n = 1ull << LOG_N;
    uint32_t* col = d + (uint64_t)(blockIdx.x / CS) * n;
    TmaArgs a{};
    a.tw = tw;
    a.log_n = LOG_N;
    a.lo = 0;
    a.batch = 1;
    a.log_tpc = (uint32_t)(X - 1);
    if constexpr (TP::kRound0Copy) a.tw0 = tw + n;  // M31 tables with n >= 2^13 carry it
    TileCoord g{};
    g.pos_base = rank << kTileBits;
    if constexpr (TP::kStaged) TP::stage_twiddles(tws, tw, tid);
    const uint32_t base0 = rank * BASES + tid;  // group gi: base0 + gi NT
    uint32_t v[16];
    if constexpr (DESC) {
      // Distributed shared memory may be written only once every block of the
      // cluster is known to run: arrive here, wait just before the first
      // remote store, so the barrier overlaps the loads and cross layers.
      asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
#pragma unroll
      for (int gi = 0; gi < GPT; ++gi)
#pragma unroll
        for (int k = 0; k < G; ++k) v[gi * G + k] = col[base0 + (uint32_t)gi * NT + ((uint32_t)k << 12)];
      cross(v, base0, tw, 0u, 0u);
      asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
#pragma unroll
      for (int gi = 0; gi < GPT; ++gi)
#pragma unroll
        for (int k = 0; k < G; ++k) {
          uint32_t* owner = cluster.map_shared_rank(tile, (unsigned)(k >> 1));
          owner[TP::sw(base0 + (uint32_t)gi * NT + ((uint32_t)(k & 1) << 12))] = v[gi * G + k];
        }
      cluster.sync();  // every block complete (and the staged twiddles visible)
      TP::template ld<TP::kFirst>(tile, v, tid);
      TP::template rounds<0>(tile, v, a, tws, g, tid);
      TP::finish(v, a, g, tid);
      TP::template st<TP::kLast>(tile, v, tid);
      __syncthreads();
      uint4* out = reinterpret_cast<uint4*>(col + g.pos_base);
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t c = 4u * (tid + i * NT);
        out[c >> 2] = *reinterpret_cast<const uint4*>(tile + TP::sw(c));
      }
    } else {
      const uint4* in = reinterpret_cast<const uint4*>(col + g.pos_base);
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t c = 4u * (tid + i * NT);
        *reinterpret_cast<uint4*>(tile + TP::sw(c)) = in[c >> 2];  // sw keeps 16-byte runs together
      }
      __syncthreads();
      TP::template ld<TP::kFirst>(tile, v, tid);
      TP::template rounds<0>(tile, v, a, tws, g, tid);
      TP::finish(v, a, g, tid);
      TP::template st<TP::kLast>(tile, v, tid);
      cluster.sync();  // every block complete
#pragma unroll
      for (int gi = 0; gi < GPT; ++gi)
#pragma unroll
        for (int k = 0; k < G; ++k) {
          const uint32_t* owner = cluster.map_shared_rank(tile, (unsigned)(k >> 1));
          v[gi * G + k] = owner[TP::sw(base0 + (uint32_t)gi * NT + ((uint32_t)(k & 1) << 12))];
        }
      // No block may leave while another still reads it: arrive once the
      // reads are performed (release), wait only before leaving, so the
      // barrier overlaps the cross layers and the stores.
      asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
      cross(v, base0, tw, scale_w, scale_ws);
#pragma unroll
      for (int gi = 0; gi < GPT; ++gi)
#pragma unroll
        for (int k = 0; k < G; ++k) col[base0 + (uint32_t)gi * NT + ((uint32_t)k << 12)] = v[gi * G + k];
      asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
  }
};

template <class F, bool DESC, int X>
__global__ void __launch_bounds__(512, 1) cluster_ntt_kernel(uint32_t* d, const uint2* tw, uint32_t scale_w,
                                                             uint32_t scale_ws) {
  pdl_enter();
  ClusterNtt<F, DESC, X>::run(d, tw, scale_w, scale_ws);
}

template <class F, bool DESC, int X>
Status launch_cluster(sfntt_ctx* ctx, uint32_t* d, uint32_t batch, const uint2* tw, uint32_t scale_w,
                      cudaStream_t s) {
  using C = ClusterNtt<F, DESC, X>;
  constexpr int smem = 4 * (int)kTileWords + 8 * (int)C::TP::TW_ENTRIES + 1024;
  auto kern = cluster_ntt_kernel<F, DESC, X>;
  static std::atomic<uint64_t> smem_done{0};
  SFNTT_TRY(smem_limit_once(kern, smem, ctx->device, smem_done));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(batch * (uint32_t)C::CS);
  cfg.blockDim = dim3(C::NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)C::CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  // small grids: programmatic dependent launch, as the passes do (pdl.cuh)
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
#ifdef SFNTT_NO_PDL
  cfg.numAttrs = 1;
#else
  cfg.numAttrs = pdl_fits(cfg.gridDim.x) ? 2 : 1;
#endif
  const uint32_t scale_ws = (uint32_t)(((uint64_t)scale_w << 32) / F::P);
  launch_begin(ctx, s);
  SFNTT_CU(cudaLaunchKernelEx(&cfg, kern, d, tw, scale_w, scale_ws));
  static const std::string name = std::string(F::kTag) + (DESC ? "_fwd" : "_inv") + "_cluster" +
                                  std::to_string(C::CS);
  return launch_check(ctx, name.c_str(), s, ((uint64_t)batch << C::LOG_N) * 8u);
}

template <class F, bool DESC>
Status cluster_dispatch(sfntt_ctx* ctx, uint32_t* d, uint32_t log_n, uint32_t batch, const uint2* tw,
                        uint32_t scale_w, cudaStream_t s) {
  switch (log_n) {
    case 13: return launch_cluster<F, DESC, 1>(ctx, d, batch, tw, scale_w, s);
    case 14: return launch_cluster<F, DESC, 2>(ctx, d, batch, tw, scale_w, s);
    case 15: return launch_cluster<F, DESC, 3>(ctx, d, batch, tw, scale_w, s);
    case 16: return launch_cluster<F, DESC, 4>(ctx, d, batch, tw, scale_w, s);
    default: return {SFNTT_INVALID_ARGUMENT, "cluster NTT: 2^13 .. 2^16 points"};
  }
}

}  // namespace

bool cluster_ntt_fits(const sfntt_ctx* ctx, uint32_t log_n, uint32_t batch, const void* d) {
  if (ctx->no_cluster || log_n < 13 || log_n > 16 || batch == 0) return false;
  if ((reinterpret_cast<uintptr_t>(d) & 15u) != 0) return false;
  return ((uint64_t)batch << (log_n - 13)) <= 2ull * (uint64_t)ctx->sm_count;  // one wave
}

Status cluster_ntt_dev(sfntt_ctx* ctx, int field, bool inverse, uint32_t* d, uint32_t log_n, uint32_t batch,
                       const uint2* tw, uint32_t scale_w, cudaStream_t s) {
  return with_field(field, [&](auto f) -> Status {
    using F = decltype(f);
    return inverse ? cluster_dispatch<F, false>(ctx, d, log_n, batch, tw, scale_w, s)
                   : cluster_dispatch<F, true>(ctx, d, log_n, batch, tw, scale_w, s);
  });
}

}  // namespace sfntt
