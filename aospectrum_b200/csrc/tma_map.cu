// Host-side encoding of 2D FP32 tensor maps for the TMA loads, stores and
// reduce-adds of the tcgen05 kernels (cuTensorMapEncodeTiled, reached through
// the runtime's driver entry point so the library needs no -lcuda).
#include "common.cuh"
#include "tc_common.cuh"

#include <cudaTypedefs.h>

#include <mutex>

namespace aosb {

namespace {
int encoder(PFN_cuTensorMapEncodeTiled_v12000* out, char* err, size_t cap) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (encode == nullptr) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || fn == nullptr)
      return set_error(err, cap, AOSB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  *out = encode;
  return 0;
}
}  // namespace

int encode_staging_5d(void* base, uint64_t plane_slabs, bool half_b, CUtensorMap* map, char* err,
                      size_t cap) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (int rc = encoder(&encode, err, cap)) return rc;
  if (((uintptr_t)base & 15) != 0)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "staging base must be 16-byte aligned");
  if (plane_slabs == 0 || plane_slabs > (uint64_t)INT32_MAX)
    return set_error(err, cap, AOSB_ERR_SIZE, "staging too large for 32-bit TMA coordinates");
  // BF16 elements: 64 per 128-byte core-matrix row, 8 rows per 1 KB group,
  // 2 operand-row halves, 2 K halves, then 4 KB plane slabs
  cuuint64_t gdim[5] = {64, 8, 2, 2, (cuuint64_t)plane_slabs};
  cuuint64_t gstride[4] = {128, 1024, 2048, 4096};
  cuuint32_t box[5] = {64, 8, half_b ? 1u : 2u, 2, 4};
  cuuint32_t estride[5] = {1, 1, 1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, base, gdim, gstride, box, estride,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(err, cap, AOSB_ERR_CUDA, "cuTensorMapEncodeTiled (staging) failed (%d)", (int)r);
  return 0;
}

int encode_f32_2d(void* base, uint64_t inner, uint64_t rows, uint32_t box_x, uint32_t box_y,
                  bool swizzle128, CUtensorMap* map, char* err, size_t cap) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (int rc = encoder(&encode, err, cap)) return rc;
  if (((uintptr_t)base & 15) != 0)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "tensor base must be 16-byte aligned");
  if (rows == 0 || rows > (uint64_t)INT32_MAX)
    return set_error(err, cap, AOSB_ERR_SIZE, "tensor too large for 32-bit TMA rows");
  if ((inner * sizeof(float)) % 16 != 0 || (box_x * sizeof(float)) % 16 != 0)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "tensor rows and boxes must be 16-byte multiples");
  cuuint64_t gdim[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t gstride[1] = {(cuuint64_t)inner * sizeof(float)};
  cuuint32_t box[2] = {box_x, box_y};
  cuuint32_t estride[2] = {1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, gdim, gstride, box, estride,
                      CU_TENSOR_MAP_INTERLEAVE_NONE,
                      swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(err, cap, AOSB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return 0;
}

}  // namespace aosb
