// Shared definitions of the B200 CISS band engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <string>

#include "../../include/aospectrum_b200.h"

namespace aosb {

// Status codes written into aosb_status_t.code by device kernels.
enum DeviceCode : int32_t {
  kDevOk = 0,
  kDevZeroPivot = AOSB_ERR_ZERO_PIVOT,
  kDevNonFinite = AOSB_ERR_NONFINITE_FACTOR,
  kDevTimeout = AOSB_ERR_TIMEOUT,
};

struct c64 { float x, y; };
struct c128 { double x, y; };

__host__ __device__ inline float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline double2 zconj(double2 a) { return make_double2(a.x, -a.y); }

// Error reporting helper shared by every host entry point.
inline int set_error(char* buf, size_t cap, int code, const char* fmt, ...) {
  if (buf != nullptr && cap > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, cap, fmt, ap);
    va_end(ap);
  }
  return code;
}

#define AOSB_CUDA_TRY(expr, buf, cap)                                              \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      return ::aosb::set_error((buf), (cap), AOSB_ERR_CUDA, "%s failed: %s", #expr, \
                               cudaGetErrorString(_e));                            \
    }                                                                              \
  } while (0)

inline int launch_check(char* buf, size_t cap, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    return set_error(buf, cap, AOSB_ERR_CUDA, "%s launch failed: %s", what,
                     cudaGetErrorString(e));
  }
  return 0;
}

inline unsigned ceil_div(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// Number of kernels this library has launched (all devices, all threads).
void count_launches(uint64_t n);

}  // namespace aosb
