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
