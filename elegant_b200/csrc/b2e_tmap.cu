#include "b2e_tmap.h"
#include <cudaTypedefs.h>
#include <mutex>

namespace b2e {

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

cudaError_t make_tmap_rows64(CUtensorMap *map, const void *base, int64_t n_rows, int64_t n_outer, int box_rows) {
  auto fn = encode_fn();
  if (!fn)
    return cudaErrorNotSupported;
  if (((uintptr_t)base & 15u) || box_rows < 1 || box_rows > 256 || n_rows < 1 || n_outer < 1)
    return cudaErrorInvalidValue;
  cuuint64_t dims[3] = {64, (cuuint64_t)n_rows, (cuuint64_t)n_outer};
  cuuint64_t strides[2] = {128, (cuuint64_t)(128 * n_rows)}; /* bytes, dims 1 and 2 */
  cuuint32_t box[3] = {64, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

} // namespace b2e
