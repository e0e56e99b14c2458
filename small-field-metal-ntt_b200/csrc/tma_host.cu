// tma_host.cu -- tensor-map encoding through the driver entry point.
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include "tma_launch.cuh"

namespace sfntt {
namespace {

// Encoded maps, keyed by every encoding parameter.  A map is a pure function
// of its key (address, shape, strides, box, swizzle), so an entry never goes
// stale; repeated launches on the same buffers skip the encoding.
std::mutex g_map_mu;
std::unordered_map<std::string, CUtensorMap> g_maps;
constexpr size_t kMaxMaps = 4096;

std::string map_key(const void* base, uint32_t rank, const cuuint64_t* dims, const cuuint64_t* strides_bytes,
                    const cuuint32_t* box, bool swizzle128) {
  struct {
    const void* base;
    uint64_t rank_swz;
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5];
  } k;
  std::memset(&k, 0, sizeof k);
  k.base = base;
  k.rank_swz = ((uint64_t)rank << 1) | (swizzle128 ? 1u : 0u);
  std::memcpy(k.dims, dims, rank * sizeof(cuuint64_t));
  std::memcpy(k.strides, strides_bytes, (rank - 1) * sizeof(cuuint64_t));
  std::memcpy(k.box, box, rank * sizeof(cuuint32_t));
  return std::string(reinterpret_cast<const char*>(&k), sizeof k);
}

}  // namespace

Status tensor_map_encode(CUtensorMap* map, const void* base, uint32_t rank, const cuuint64_t* dims,
                         const cuuint64_t* strides_bytes, const cuuint32_t* box, bool swizzle128) {
  if (rank < 1 || rank > 5) return {SFNTT_INVALID_ARGUMENT, "tensor map rank"};
  const std::string key = map_key(base, rank, dims, strides_bytes, box, swizzle128);
  {
    std::lock_guard<std::mutex> lk(g_map_mu);
    auto it = g_maps.find(key);
    if (it != g_maps.end()) {
      *map = it->second;
      return {};
    }
  }
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    cudaGetLastError();
  });
  if (!encode) return {SFNTT_KERNEL_LOAD, "cuTensorMapEncodeTiled unavailable"};
  cuuint32_t elem_strides[5] = {1, 1, 1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, rank, const_cast<void*>(base), dims, strides_bytes, box,
                      elem_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return {SFNTT_INVALID_ARGUMENT, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")"};
  std::lock_guard<std::mutex> lk(g_map_mu);
  if (g_maps.size() >= kMaxMaps) g_maps.clear();
  g_maps.emplace(key, *map);
  return {};
}

}  // namespace sfntt
