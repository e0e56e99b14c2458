// layout.cu -- output conventions for LDE / NTT results (SoA batches).
//
// The transforms leave each column's rows in bit-reversed order, SoA
// (data[col * n + row]), as the reference does.  Two conventions used by the
// callers either side of the path:
//   * natural row order (Plonky3's coset_lde_batch returns natural-order rows):
//     out[col * n + r] = in[col * n + bitrev(r)];
//   * row-major rows, the input of Merkle commitment (one leaf per row):
//     out[R * batch + col] = in[col * n + r], R = r or bitrev(r).
// Both are pure permutations, HBM-bound: every word is read once and written
// once.  The reference's own permutation kernel is `bitrev_permute`
// (shaders/m31/m31_ntt_ct_dit_r2.metal:22-41), one word per thread.
//
// Kernels move tiles through shared memory so that global reads and writes are
// whole 128- to 512-byte segments:
//   bitrev_cols: tile (column, mid) holds words (hi << (L-5)) | (mid << 5) | lo
//     for hi, lo < 32; word (hi, mid, lo) goes to (rev5(lo), rev(mid), rev5(hi));
//     tiles mid and rev(mid) swap, so the permutation also runs in place.
//   transpose: tile (32 columns) x (32 consecutive rows); each row of the tile
//     becomes 32 consecutive words of one output row.
#include <algorithm>

#include "context.hpp"

namespace sfntt {
namespace {

constexpr int kLayoutThreads = 256;

__device__ __forceinline__ uint32_t rev_bits(uint32_t x, uint32_t bits) { return bits ? __brev(x) >> (32 - bits) : 0u; }

// log_n >= 10.  tiles = batch << (log_n - 10).  Tiles mid and rev(mid) of a
// column trade places, so one CTA handles the pair (the CTA of the larger mid
// skips): both are read before either is written, which also makes the
// permutation safe in place (in == out).
__global__ void __launch_bounds__(kLayoutThreads) bitrev_cols_kernel(const uint32_t* in, uint64_t in_stride,
                                                                     uint32_t* out, uint64_t out_stride,
                                                                     uint32_t log_n, uint64_t tiles) {
  __shared__ uint32_t ta[32][33], tb[32][33];
  const uint32_t mbits = log_n - 10;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t hi_shift = log_n - 5;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint64_t col = t >> mbits;
    const uint32_t mid = (uint32_t)(t & ((1ull << mbits) - 1ull));
    const uint32_t rmid = rev_bits(mid, mbits);
    if (mid > rmid) continue;  // uniform over the CTA
    const uint32_t* sa = in + col * in_stride + ((uint64_t)mid << 5);
    const uint32_t* sb = in + col * in_stride + ((uint64_t)rmid << 5);
#pragma unroll
    for (uint32_t h = warp; h < 32; h += kLayoutThreads / 32) {
      ta[h][lane] = sa[((uint64_t)h << hi_shift) + lane];
      if (rmid != mid) tb[h][lane] = sb[((uint64_t)h << hi_shift) + lane];
    }
    __syncthreads();
    // tile mid's word (hi, lo) lands in tile rmid at row rev5(lo), word rev5(hi), and vice versa
    uint32_t* da = out + col * out_stride + ((uint64_t)rmid << 5);
    uint32_t* db = out + col * out_stride + ((uint64_t)mid << 5);
#pragma unroll
    for (uint32_t a = warp; a < 32; a += kLayoutThreads / 32) {
      const uint32_t hi = rev_bits(lane, 5), lo = rev_bits(a, 5);
      da[((uint64_t)a << hi_shift) + lane] = ta[hi][lo];
      if (rmid != mid) db[((uint64_t)a << hi_shift) + lane] = tb[hi][lo];
    }
    __syncthreads();
  }
}

// The same permutation on 64 x 64-word tiles (log_n >= 12): 256-byte global
// rows and 32 KB per CTA in flight.  The shared tile is XOR-swizzled, word
// (r, c) at r * 64 + (c ^ ((r >> 1) & 31)), so a row (fixed r) and the
// bit-reversed column read (rows rev6(j) for the 32 lanes j, whose r >> 1 are
// the 32 values rev5(j mod 32)) both touch 32 distinct banks.
constexpr int kWideThreads = 512;

__device__ __forceinline__ uint32_t swz64(uint32_t r, uint32_t c) { return r * 64u + (c ^ ((r >> 1) & 31u)); }

__global__ void __launch_bounds__(kWideThreads) bitrev_cols64_kernel(const uint32_t* in, uint64_t in_stride,
                                                                     uint32_t* out, uint64_t out_stride,
                                                                     uint32_t log_n, uint64_t tiles) {
  __shared__ uint32_t ta[64 * 64], tb[64 * 64];
  const uint32_t mbits = log_n - 12;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t hi_shift = log_n - 6;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint64_t col = t >> mbits;
    const uint32_t mid = (uint32_t)(t & ((1ull << mbits) - 1ull));
    const uint32_t rmid = rev_bits(mid, mbits);
    if (mid > rmid) continue;  // uniform over the CTA
    const uint32_t* sa = in + col * in_stride + ((uint64_t)mid << 6);
    const uint32_t* sb = in + col * in_stride + ((uint64_t)rmid << 6);
#pragma unroll
    for (uint32_t h = warp; h < 64; h += kWideThreads / 32) {
#pragma unroll
      for (uint32_t w = lane; w < 64; w += 32) {
        ta[swz64(h, w)] = sa[((uint64_t)h << hi_shift) + w];
        if (rmid != mid) tb[swz64(h, w)] = sb[((uint64_t)h << hi_shift) + w];
      }
    }
    __syncthreads();
    // tile mid's word (hi, lo) lands in tile rmid at row rev6(lo), word rev6(hi), and vice versa
    uint32_t* da = out + col * out_stride + ((uint64_t)rmid << 6);
    uint32_t* db = out + col * out_stride + ((uint64_t)mid << 6);
#pragma unroll
    for (uint32_t a = warp; a < 64; a += kWideThreads / 32) {
      const uint32_t lo = rev_bits(a, 6);
#pragma unroll
      for (uint32_t j = lane; j < 64; j += 32) {
        const uint32_t hi = rev_bits(j, 6);
        da[((uint64_t)a << hi_shift) + j] = ta[swz64(hi, lo)];
        if (rmid != mid) db[((uint64_t)a << hi_shift) + j] = tb[swz64(hi, lo)];
      }
    }
    __syncthreads();
  }
}

// Row-major on 128-column x 32-row tiles (log_n >= 5, batch >= 128): 128-byte
// reads (32 rows of one column) and 512-byte writes (128 columns of one row),
// so a tile's output is 32 runs of 512 bytes, one per output row.  Tile word
// (column j, row i) at j * 33 + i: a column (fixed j, lanes over i) and a row
// (fixed i, lanes over j) both touch 32 distinct banks.
constexpr uint32_t kWideCols = 128;

__global__ void __launch_bounds__(kWideThreads) transpose_wide_kernel(const uint32_t* __restrict__ in,
                                                                      uint32_t* __restrict__ out, uint32_t log_n,
                                                                      uint32_t batch, uint32_t cblocks, uint32_t tiles,
                                                                      int bitrev) {
  __shared__ uint32_t tile[kWideCols * 33];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Loads: thread reads tile column warp + 16 q (q < 8) at row lane.  Stores:
  // thread writes tile row si + 4 q at column sj.  Addresses advance by
  // shifts from per-tile bases; a bit-reversed row r0 + i (r0 a multiple of
  // 32, i < 32) is rev(r0) + (rev5(i) << (log n - 5)).
  const uint32_t si = warp >> 2, sj = ((warp & 3u) << 5) + lane;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint32_t rb = t / cblocks, cb = t - rb * cblocks;
    const uint32_t c0 = cb * kWideCols;
    const uint64_t r0 = (uint64_t)rb << 5;
    const uint32_t* src = in + ((uint64_t)(c0 + warp) << log_n) + r0 + lane;
#pragma unroll
    for (uint32_t q = 0; q < kWideCols / 16; ++q) {
      const uint32_t j = warp + 16u * q;
      if (c0 + j < batch) tile[j * 33 + lane] = __ldcs(src + ((uint64_t)q << (log_n + 4)));
    }
    __syncthreads();
    if (c0 + sj < batch) {
      uint32_t* dst = out + c0 + sj;
      if (bitrev) {
        const uint64_t rbase = (uint64_t)rev_bits((uint32_t)r0, log_n) + ((uint64_t)rev_bits(si, 5) << (log_n - 5));
        dst += rbase * batch;
        const uint64_t step = (uint64_t)batch << (log_n - 5);  // row rev5(4 q) << (log n - 5) = rev3(q) << (log n - 3)
#pragma unroll
        for (uint32_t q = 0; q < 8; ++q) __stcs(dst + (uint64_t)(rev_bits(4u * q, 5)) * step, tile[sj * 33 + si + 4u * q]);
      } else {
        dst += (r0 + si) * batch;
        const uint64_t step = 4ull * batch;
#pragma unroll
        for (uint32_t q = 0; q < 8; ++q) __stcs(dst + q * step, tile[sj * 33 + si + 4u * q]);
      }
    }
    __syncthreads();
  }
}

// log_n >= 5.  Tiles: ceil(batch / 32) column blocks x (n / 32) row blocks.
__global__ void __launch_bounds__(kLayoutThreads) transpose_kernel(const uint32_t* __restrict__ in,
                                                                   uint32_t* __restrict__ out, uint32_t log_n,
                                                                   uint32_t batch, uint32_t cblocks, uint64_t tiles,
                                                                   int bitrev) {
  __shared__ uint32_t tile[32][33];
  const uint64_t n = 1ull << log_n;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint32_t cb = (uint32_t)(t % cblocks);
    const uint64_t r0 = (t / cblocks) << 5;
    const uint32_t c0 = cb << 5;
#pragma unroll
    for (uint32_t j = warp; j < 32; j += kLayoutThreads / 32)
      if (c0 + j < batch) tile[j][lane] = __ldcs(in + (uint64_t)(c0 + j) * n + r0 + lane);
    __syncthreads();
    const bool col_ok = c0 + lane < batch;
#pragma unroll
    for (uint32_t i = warp; i < 32; i += kLayoutThreads / 32) {
      const uint64_t r = r0 + i;
      const uint64_t R = bitrev ? rev_bits((uint32_t)r, log_n) : r;
      if (col_ok) __stcs(out + R * batch + c0 + lane, tile[lane][i]);
    }
    __syncthreads();
  }
}

// Natural row order of short columns (any size), in place or not: the thread
// owning row r <= bitrev(r) moves the pair.
__global__ void bitrev_pairs_kernel(const uint32_t* in, uint64_t in_stride, uint32_t* out, uint64_t out_stride,
                                    uint32_t log_n, uint64_t total) {
  const uint64_t mask = (1ull << log_n) - 1ull;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = i >> log_n, r = i & mask, rr = rev_bits((uint32_t)r, log_n);
    if (r <= rr) {
      const uint32_t x = in[c * in_stride + r], y = in[c * in_stride + rr];
      out[c * out_stride + rr] = x;
      out[c * out_stride + r] = y;
    }
  }
}

// Any shape (small columns): one word per thread.
__global__ void layout_words_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t log_n,
                                    uint32_t batch, uint64_t total, int flags) {
  const uint64_t mask = (1ull << log_n) - 1ull;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = i >> log_n, r = i & mask;
    const uint64_t R = (flags & SFNTT_LAYOUT_NATURAL) ? rev_bits((uint32_t)r, log_n) : r;
    const uint64_t d = (flags & SFNTT_LAYOUT_ROW_MAJOR) ? R * batch + c : (c << log_n) + R;
    out[d] = in[i];
  }
}

uint32_t grid_for(const sfntt_ctx* ctx, uint64_t work) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(work, (uint64_t)ctx->sm_count * 8));
}

}  // namespace

Status bitrev_cols_dev(sfntt_ctx* ctx, const uint32_t* in, uint64_t in_stride, uint32_t* out, uint64_t out_stride,
                       uint32_t log_n, uint32_t batch, cudaStream_t s) {
  const uint64_t total = (uint64_t)batch << log_n;
  if (total == 0 || log_n == 0) {
    if (total && in != out) SFNTT_CU(cudaMemcpy2DAsync(out, out_stride * 4, in, in_stride * 4, 4, batch,
                                                       cudaMemcpyDeviceToDevice, s));
    return {};
  }
  launch_begin(ctx, s);
  if (log_n >= 12) {
    const uint64_t tiles = (uint64_t)batch << (log_n - 12);
    // 64 CTAs per SM, two resident: the CTAs in flight hold consecutive tiles,
    // whose 256-byte runs share DRAM rows (4 per SM, a stride of 4 x SMs
    // tiles between a CTA's tiles: 0.96 ms for the 2 GiB LDE output; 64: 0.76)
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)ctx->sm_count * 64));
    bitrev_cols64_kernel<<<grid, kWideThreads, 0, s>>>(in, in_stride, out, out_stride, log_n, tiles);
    return launch_check(ctx, "layout_bitrev_cols", s, total * 8);
  }
  if (log_n >= 10) {
    const uint64_t tiles = (uint64_t)batch << (log_n - 10);
    bitrev_cols_kernel<<<grid_for(ctx, tiles), kLayoutThreads, 0, s>>>(in, in_stride, out, out_stride, log_n, tiles);
    return launch_check(ctx, "layout_bitrev_cols", s, total * 8);
  }
  bitrev_pairs_kernel<<<grid_for(ctx, (total + 255) / 256), 256, 0, s>>>(in, in_stride, out, out_stride, log_n, total);
  return launch_check(ctx, "layout_bitrev_pairs", s, total * 8);
}

Status layout_dev(sfntt_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t log_n, uint32_t batch, int flags,
                  cudaStream_t s) {
  if (flags & ~(SFNTT_LAYOUT_NATURAL | SFNTT_LAYOUT_ROW_MAJOR)) return {SFNTT_INVALID_ARGUMENT, "unknown layout flags"};
  if (log_n > 31) return {SFNTT_INVALID_SIZE, "log_n > 31"};
  const uint64_t total = (uint64_t)batch << log_n;
  if (total == 0) return {};
  if (!in || !out) return {SFNTT_INVALID_ARGUMENT, "null buffer"};
  const bool natural = flags & SFNTT_LAYOUT_NATURAL;
  const bool rows = (flags & SFNTT_LAYOUT_ROW_MAJOR) && batch > 1;  // one column is its own row-major form
  const uintptr_t a = reinterpret_cast<uintptr_t>(in), b = reinterpret_cast<uintptr_t>(out);
  const bool same = a == b;
  if (!same && a < b + total * 4 && b < a + total * 4) return {SFNTT_INVALID_ARGUMENT, "layout buffers overlap"};
  if (same && rows) return {SFNTT_INVALID_ARGUMENT, "the row-major layout is out of place"};
  const uint64_t n = 1ull << log_n;
  if (!rows) {
    if (natural) return bitrev_cols_dev(ctx, in, n, out, n, log_n, batch, s);
    if (!same) SFNTT_CU(cudaMemcpyAsync(out, in, total * 4, cudaMemcpyDeviceToDevice, s));
    return {};
  }
  launch_begin(ctx, s);
  if (log_n >= 5 && batch >= kWideCols) {
    const uint32_t cblocks = (batch + kWideCols - 1) / kWideCols;
    const uint64_t tiles = (uint64_t)cblocks << (log_n - 5);  // batch * n / 4096 at most: < 2^29
    // 64 CTAs per SM, as the bit reversal (row-major 0.83 -> 0.80 ms on the 2 GiB LDE output)
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)ctx->sm_count * 64));
    transpose_wide_kernel<<<grid, kWideThreads, 0, s>>>(in, out, log_n, batch, cblocks, (uint32_t)tiles,
                                                        natural ? 1 : 0);
    return launch_check(ctx, natural ? "layout_transpose_bitrev" : "layout_transpose", s, total * 8);
  }
  if (log_n >= 5) {
    const uint32_t cblocks = (batch + 31) / 32;
    const uint64_t tiles = (uint64_t)cblocks << (log_n - 5);
    transpose_kernel<<<grid_for(ctx, tiles), kLayoutThreads, 0, s>>>(in, out, log_n, batch, cblocks, tiles,
                                                                      natural ? 1 : 0);
    return launch_check(ctx, natural ? "layout_transpose_bitrev" : "layout_transpose", s, total * 8);
  }
  layout_words_kernel<<<grid_for(ctx, (total + 255) / 256), 256, 0, s>>>(in, out, log_n, batch, total, flags);
  return launch_check(ctx, "layout_words", s, total * 8);
}

}  // namespace sfntt
