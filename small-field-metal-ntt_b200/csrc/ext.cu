// ext.cu -- the M31 quadratic extension CM31 = M31[i] / (i^2 + 1) (planned in
// the reference, TODOS.md:27-31 "M31 Quadratic Extension Field Support").
//
// Elements are interleaved pairs (re, im) of canonical M31 words, the layout of
// a #[repr(C)] struct of two M31 newtypes.  The Circle NTT's twiddles lie in
// the base field, so the transform of a CM31 column is the base-field
// transform of its real part plus i times that of its imaginary part.  The
// batch of CM31 columns is split into 2 * batch base-field columns (real parts
// first), run through the batched M31 engine, and merged back: split and merge
// each read and write every word once with 8-byte / 4-byte coalesced accesses.
#include <algorithm>

#include "context.hpp"
#include "field.cuh"

namespace sfntt {
namespace {

// planes[k] = pairs[k].x, planes[total + k] = pairs[k].y
__global__ void cm31_split_kernel(const uint2* __restrict__ pairs, uint32_t* __restrict__ planes, uint64_t total) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 v = pairs[k];
    planes[k] = v.x;
    planes[total + k] = v.y;
  }
}

__global__ void cm31_merge_kernel(const uint32_t* __restrict__ planes, uint2* __restrict__ pairs, uint64_t total) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x)
    pairs[k] = make_uint2(planes[k], planes[total + k]);
}

// (a + bi)(c + di) = (ac - bd) + (ad + bc) i, each product Mersenne-folded
__global__ void cm31_mul_kernel(const uint2* __restrict__ x, const uint2* __restrict__ y, uint2* __restrict__ out,
                                uint64_t n) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 a = x[k], b = y[k];
    const uint32_t re = sub_mod<M31>(mul_var<M31>(a.x, b.x), mul_var<M31>(a.y, b.y));
    const uint32_t im = add_mod<M31>(mul_var<M31>(a.x, b.y), mul_var<M31>(a.y, b.x));
    out[k] = make_uint2(re, im);
  }
}

uint32_t grid_of(const sfntt_ctx* ctx, uint64_t n) {
  const uint64_t want = (n + 255) / 256;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 16));
}

}  // namespace

Status cm31_scratch(sfntt_ctx* ctx, uint32_t log_n, uint32_t batch, cudaStream_t s, uint32_t** out) {
  const size_t bytes = ((size_t)batch << log_n) * 8u;
  if (ctx->buf_ext.bytes < bytes) {
    if (capturing(s)) return {SFNTT_INVALID_ARGUMENT, "CM31 scratch not prepared before capture"};
    SFNTT_TRY(ctx->buf_ext.reserve(bytes));
  }
  *out = ctx->buf_ext.as<uint32_t>();
  return {};
}

// Circle NTT over `batch` CM31 columns of 2^log_n interleaved pairs, in place.
Status cm31_ntt_dev(sfntt_ctx* ctx, bool inverse, uint32_t* d_pairs, uint32_t log_n, uint32_t batch,
                    cudaStream_t s) {
  if (log_n > 30) return {SFNTT_INVALID_SIZE, "M31 log_n > 30"};
  if (log_n == 0 || batch == 0) return {};
  if (((uint64_t)batch << log_n) >= (1ull << 39)) return {SFNTT_INVALID_SIZE, "too large"};
  if (!d_pairs) return {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if (reinterpret_cast<uintptr_t>(d_pairs) & 7u) return {SFNTT_INVALID_ARGUMENT, "CM31 pairs must be 8-byte aligned"};
  uint32_t* planes = nullptr;
  SFNTT_TRY(cm31_scratch(ctx, log_n, batch, s, &planes));
  const uint64_t total = (uint64_t)batch << log_n;
  launch_begin(ctx, s);
  cm31_split_kernel<<<grid_of(ctx, total), 256, 0, s>>>(reinterpret_cast<const uint2*>(d_pairs), planes, total);
  SFNTT_TRY(launch_check(ctx, "cm31_split", s, total * 16u));
  SFNTT_TRY(ntt_dev(ctx, SFNTT_M31, SFNTT_BEST, inverse, planes, log_n, 2u * batch, s));
  launch_begin(ctx, s);
  cm31_merge_kernel<<<grid_of(ctx, total), 256, 0, s>>>(planes, reinterpret_cast<uint2*>(d_pairs), total);
  return launch_check(ctx, "cm31_merge", s, total * 16u);
}

Status cm31_mul_dev(sfntt_ctx* ctx, const uint32_t* a, const uint32_t* b, uint32_t* out, size_t n, cudaStream_t s) {
  if (n == 0) return {};
  if (!a || !b || !out) return {SFNTT_INVALID_ARGUMENT, "null buffer"};
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(out)) & 7u)
    return {SFNTT_INVALID_ARGUMENT, "CM31 pairs must be 8-byte aligned"};
  launch_begin(ctx, s);
  cm31_mul_kernel<<<grid_of(ctx, n), 256, 0, s>>>(reinterpret_cast<const uint2*>(a), reinterpret_cast<const uint2*>(b),
                                                  reinterpret_cast<uint2*>(out), n);
  return launch_check(ctx, "cm31_mul", s, (uint64_t)n * 24u);
}

}  // namespace sfntt
