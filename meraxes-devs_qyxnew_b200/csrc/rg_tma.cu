// Host side of the TMA tiles: tensor maps through the driver's cuTensorMapEncodeTiled, reached
// through the runtime's driver entry point (the library links no libcuda).
#include <mutex>

#include "rg_tma.cuh"

namespace rg {

namespace {
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(f);
  });
  return fn;
}
}  // namespace

int tma_map_3d(CUtensorMap* map, const void* base, const uint64_t dims[3], const uint64_t strides_bytes[2],
               const uint32_t box[3]) {
  EncodeFn fn = encode_fn();
  if (!fn) return (int)CUDA_ERROR_NOT_FOUND;
  const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
  const cuuint64_t s[2] = {strides_bytes[0], strides_bytes[1]};
  const cuuint32_t b[3] = {box[0], box[1], box[2]};
  const cuuint32_t e[3] = {1, 1, 1};
  return (int)fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), d, s, b, e,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

}  // namespace rg
