// tma_host.cu -- tensor-map encoding through the driver entry point.
#include <mutex>

#include "tma_launch.cuh"

namespace sfntt {

Status tensor_map_encode(CUtensorMap* map, const void* base, uint32_t rank, const cuuint64_t* dims,
                         const cuuint64_t* strides_bytes, const cuuint32_t* box, bool swizzle128) {
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
  return {};
}

}  // namespace sfntt
