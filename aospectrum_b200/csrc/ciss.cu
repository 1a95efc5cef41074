// FP64 kernels of the CISS subspace steps on n x m complex128 blocks.
//
// The reference performs these on the host in complex64 with numpy/scipy
// (src/aospectrum/ciss.py:296-372): S @ probes, the moment axpys, the Gram
// matrix M^H S M, the basis transform, B^H H B, B^H S B and the residual
// norms.  Here they run on the device in FP64 so that the projected
// problems and the reported residuals carry FP64 accuracy.
#include "common.cuh"
#include "timing.h"

#include <mutex>
#include <vector>

namespace aosb {
namespace {

// y = A x: one warp per row, lanes over 32 columns at a time.
__global__ void spmm_kernel(int64_t n, int ncols, const int64_t* __restrict__ indptr,
                            const int32_t* __restrict__ indices, const float2* __restrict__ vals,
                            const double2* __restrict__ x, int64_t ldx, double2* __restrict__ y,
                            int64_t ldy) {
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const int64_t e0 = indptr[row], e1 = indptr[row + 1];
  for (int c0 = 0; c0 < ncols; c0 += 32) {
    const int c = c0 + lane;
    if (c >= ncols) break;
    double sr = 0.0, si = 0.0;
    for (int64_t e = e0; e < e1; ++e) {
      const float2 a = vals[e];
      const double2 v = x[(size_t)indices[e] * ldx + c];
      sr += (double)a.x * v.x - (double)a.y * v.y;
      si += (double)a.x * v.y + (double)a.y * v.x;
    }
    y[(size_t)row * ldy + c] = make_double2(sr, si);
  }
}

__global__ void moments_kernel(int64_t n, int L, int M, const double2* __restrict__ x,
                               const double2* __restrict__ coef, double2* __restrict__ mom) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * L) return;
  const int64_t j = idx / L;
  const int c = (int)(idx - j * L);
  const double2 v = x[idx];
  double2* row = mom + (size_t)j * L * M;
  for (int m = 0; m < M; ++m) {
    const double2 w = coef[m];
    double2 o = row[m * L + c];
    o.x += w.x * v.x - w.y * v.y;
    o.y += w.x * v.y + w.y * v.x;
    row[m * L + c] = o;
  }
}

// Partial Gram blocks: scratch[chunk][p][q] = sum over rows in chunk of
// conj(x[j][a]) y[j][b].  grid = (ceil(p/32), ceil(q/32), chunks).
constexpr int kGramRows = 512;

__global__ void __launch_bounds__(256) gram_partial_kernel(int64_t n, int p, int q,
                                                           const double2* __restrict__ x,
                                                           int64_t ldx,
                                                           const double2* __restrict__ y,
                                                           int64_t ldy,
                                                           double2* __restrict__ part) {
  __shared__ double2 xs[32][33];
  __shared__ double2 ys[32][33];
  const int a0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
  const int64_t r0 = (int64_t)blockIdx.z * kGramRows;
  const int64_t r1 = (n < r0 + kGramRows) ? n : r0 + kGramRows;
  const int tid = threadIdx.x;
  const int ta = tid / 8;          // 32 output rows
  const int tb = (tid % 8) * 4;    // 4 output columns each
  double2 acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = make_double2(0.0, 0.0);
  for (int64_t r = r0; r < r1; r += 32) {
    for (int e = tid; e < 32 * 32; e += 256) {
      const int rr = e / 32, cc = e % 32;
      const int64_t row = r + rr;
      xs[rr][cc] = (row < r1 && a0 + cc < p) ? x[(size_t)row * ldx + a0 + cc] : make_double2(0, 0);
      ys[rr][cc] = (row < r1 && b0 + cc < q) ? y[(size_t)row * ldy + b0 + cc] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < 32; ++rr) {
      const double2 xv = xs[rr][ta];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 yv = ys[rr][tb + j];
        // conj(xv) * yv
        acc[j].x = fma(xv.x, yv.x, fma(xv.y, yv.y, acc[j].x));
        acc[j].y = fma(xv.x, yv.y, fma(-xv.y, yv.x, acc[j].y));
      }
    }
    __syncthreads();
  }
  const int a = a0 + ta;
  if (a < p) {
    double2* out = part + (size_t)blockIdx.z * p * q;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (b0 + tb + j < q) out[(size_t)a * q + b0 + tb + j] = acc[j];
  }
}

__global__ void gram_reduce_kernel(int chunks, int64_t pq, const double2* __restrict__ part,
                                   double2* __restrict__ g) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pq) return;
  double sr = 0.0, si = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const double2 v = part[(size_t)c * pq + i];
    sr += v.x;
    si += v.y;
  }
  g[i] = make_double2(sr, si);
}

// y (n x r) = x (n x p) t (p x r); CTA = 32 rows x 64 columns.
__global__ void __launch_bounds__(256) dense_mul_kernel(int64_t n, int p, int r,
                                                        const double2* __restrict__ x,
                                                        int64_t ldx,
                                                        const double2* __restrict__ t,
                                                        double2* __restrict__ y, int64_t ldy) {
  __shared__ double2 xs[32][17];
  __shared__ double2 ts[16][64];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 64;
  const int tid = threadIdx.x;
  const int tr = tid / 16;        // 16 row groups of 2 rows
  const int tc = tid % 16;        // 16 column groups of 4 columns (strided)
  double2 acc[2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0, 0);
  for (int k0 = 0; k0 < p; k0 += 16) {
    for (int e = tid; e < 32 * 16; e += 256) {
      const int rr = e / 16, kk = e % 16;
      const int64_t row = r0 + rr;
      xs[rr][kk] = (row < n && k0 + kk < p) ? x[(size_t)row * ldx + k0 + kk] : make_double2(0, 0);
    }
    for (int e = tid; e < 16 * 64; e += 256) {
      const int kk = e / 64, cc = e % 64;
      ts[kk][cc] = (k0 + kk < p && c0 + cc < r) ? t[(size_t)(k0 + kk) * r + c0 + cc]
                                                 : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double2 a = xs[tr * 2 + i][kk];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double2 b = ts[kk][tc + 16 * j];
          acc[i][j].x = fma(a.x, b.x, fma(-a.y, b.y, acc[i][j].x));
          acc[i][j].y = fma(a.x, b.y, fma(a.y, b.x, acc[i][j].y));
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int64_t row = r0 + tr * 2 + i;
    if (row >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = c0 + tc + 16 * j;
      if (col < r) y[(size_t)row * ldy + col] = acc[i][j];
    }
  }
}

// out[j] = || a[:, j] - e[j] b[:, j] ||; CTA = 32 columns x 8 row lanes.
__global__ void column_norms_kernel(int64_t n, int m, const double2* __restrict__ a,
                                    const double2* __restrict__ b, int64_t ld,
                                    const double* __restrict__ e, double* __restrict__ out) {
  __shared__ double part[8][32];
  const int cl = threadIdx.x % 32, rl = threadIdx.x / 32;
  const int j = blockIdx.x * 32 + cl;
  double s = 0.0;
  if (j < m) {
    const double ej = e[j];
    for (int64_t i = rl; i < n; i += 8) {
      const double2 av = a[(size_t)i * ld + j], bv = b[(size_t)i * ld + j];
      const double dr = av.x - ej * bv.x, di = av.y - ej * bv.y;
      s += dr * dr + di * di;
    }
  }
  part[rl][cl] = s;
  __syncthreads();
  if (rl == 0 && j < m) {
    double t = 0.0;
    for (int q = 0; q < 8; ++q) t += part[q][cl];
    out[j] = sqrt(t);
  }
}

}  // namespace
}  // namespace aosb

extern "C" {

int aosb_spmm(int64_t n, int32_t ncols, const int64_t* indptr, const int32_t* indices,
              const aosb_complex64* values, const aosb_complex128* x, int64_t ldx,
              aosb_complex128* y, int64_t ldy, void* stream, char* err, size_t cap) {
  if (indptr == nullptr || indices == nullptr || values == nullptr || x == nullptr || y == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || ncols <= 0 || ldx < ncols || ldy < ncols)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid spmm shape");
  cudaEvent_t ev[2];
  const bool timed = aosb::timing_begin((cudaStream_t)stream, ev);
  aosb::spmm_kernel<<<aosb::ceil_div(n, 8), 256, 0, (cudaStream_t)stream>>>(
      n, ncols, indptr, indices, (const float2*)values, (const double2*)x, ldx, (double2*)y, ldy);
  aosb::count_launches(1);
  if (timed) {
    // nnz of a pattern, read once per indptr array (timing runs only)
    static std::mutex mu;
    static std::vector<std::pair<const int64_t*, int64_t>> seen;
    int64_t nnz = -1;
    {
      std::lock_guard<std::mutex> lock(mu);
      for (auto& e : seen)
        if (e.first == indptr + n) nnz = e.second;
    }
    if (nnz < 0) {
      cudaMemcpy(&nnz, indptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost);
      std::lock_guard<std::mutex> lock(mu);
      seen.emplace_back(indptr + n, nnz);
    }
    aosb::timing_end(aosb::kTimedSpmm, (cudaStream_t)stream, ev, 8.0 * nnz * ncols,
                     12.0 * nnz + (double)n * ncols * 32.0);
  }
  return aosb::launch_check(err, cap, "spmm");
}

int aosb_moments_accumulate(int64_t n, int32_t L, int32_t M, const aosb_complex128* x,
                            const aosb_complex128* coef, aosb_complex128* mom, void* stream,
                            char* err, size_t cap) {
  if (x == nullptr || coef == nullptr || mom == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || L <= 0 || M <= 0)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid moment shape");
  aosb::moments_kernel<<<aosb::ceil_div(n * L, 256), 256, 0, (cudaStream_t)stream>>>(
      n, L, M, (const double2*)x, (const double2*)coef, (double2*)mom);
  aosb::count_launches(1);
  return aosb::launch_check(err, cap, "moments");
}

size_t aosb_gram_scratch_bytes(int64_t n, int32_t p, int32_t q) {
  if (n <= 0 || p <= 0 || q <= 0) return 0;
  const int64_t chunks = (n + aosb::kGramRows - 1) / aosb::kGramRows;
  return (size_t)chunks * (size_t)p * (size_t)q * sizeof(double2);
}

namespace aosb {
// The partial-sum grid is (ceil(p/32), ceil(q/32), ceil(n/512)); its y and z
// extents are limited to 65535, so n above 33,553,920 rows (or q above
// 2,097,120 columns) is rejected before anything is launched.
static int gram_grid_check(int64_t n, int32_t q, char* err, size_t cap) {
  const int64_t chunks = (n + kGramRows - 1) / kGramRows;
  if (chunks > 65535 || ceil_div((int64_t)q, 32) > 65535)
    return set_error(err, cap, AOSB_ERR_SIZE,
                     "gram: n=%lld rows in %lld chunks of %d (or q=%d) exceeds the launch grid "
                     "limit of 65535 chunks", (long long)n, (long long)chunks, kGramRows, q);
  return 0;
}
}  // namespace aosb

int aosb_gram(int64_t n, int32_t p, int32_t q, const aosb_complex128* x, int64_t ldx,
              const aosb_complex128* y, int64_t ldy, aosb_complex128* g, void* scratch,
              void* stream, char* err, size_t cap) {
  if (x == nullptr || y == nullptr || g == nullptr || scratch == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || p <= 0 || q <= 0 || ldx < p || ldy < q)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid gram shape");
  if (int rc = aosb::gram_grid_check(n, q, err, cap)) return rc;
  const int chunks = (int)((n + aosb::kGramRows - 1) / aosb::kGramRows);
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid(aosb::ceil_div(p, 32), aosb::ceil_div(q, 32), chunks);
  aosb::gram_partial_kernel<<<grid, 256, 0, st>>>(n, p, q, (const double2*)x, ldx,
                                                  (const double2*)y, ldy, (double2*)scratch);
  const int64_t pq = (int64_t)p * q;
  aosb::gram_reduce_kernel<<<aosb::ceil_div(pq, 256), 256, 0, st>>>(
      chunks, pq, (const double2*)scratch, (double2*)g);
  aosb::count_launches(2);
  return aosb::launch_check(err, cap, "gram");
}

int aosb_dense_mul(int64_t n, int32_t p, int32_t r, const aosb_complex128* x, int64_t ldx,
                   const aosb_complex128* t, aosb_complex128* y, int64_t ldy, void* stream,
                   char* err, size_t cap) {
  if (x == nullptr || t == nullptr || y == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || p <= 0 || r <= 0 || ldx < p || ldy < r)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid dense_mul shape");
  dim3 grid(aosb::ceil_div(n, 32), aosb::ceil_div(r, 64));
  aosb::dense_mul_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
      n, p, r, (const double2*)x, ldx, (const double2*)t, (double2*)y, ldy);
  aosb::count_launches(1);
  return aosb::launch_check(err, cap, "dense_mul");
}

int aosb_column_norms(int64_t n, int32_t m, const aosb_complex128* a, const aosb_complex128* b,
                      int64_t ld, const double* e, double* out, void* stream, char* err,
                      size_t cap) {
  if (a == nullptr || b == nullptr || e == nullptr || out == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || m <= 0 || ld < m)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid norm shape");
  aosb::column_norms_kernel<<<aosb::ceil_div(m, 32), 256, 0, (cudaStream_t)stream>>>(
      n, m, (const double2*)a, (const double2*)b, ld, e, out);
  aosb::count_launches(1);
  return aosb::launch_check(err, cap, "column_norms");
}

// ---------------------------------------------------------------------------
// Gram product without any allocation, for callers that cannot allocate
// device memory at the point of the call: code running inside another
// framework's stream-ordered memory pool or under a memory cap that forbids
// new cudaMalloc, real-time or callback contexts where an allocation could
// block or deadlock, and embedders that must not grow the device heap after
// start-up.  The partial sums live in one file-scope device array of
// kNoAllocGramBytes (16 MiB); every GPU that loads this library's device
// code holds it until the process exits.
constexpr size_t kNoAllocGramBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_noalloc_gram_scratch[kNoAllocGramBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

}  // namespace aosb

extern "C" int aosb_gram_noalloc(int64_t n, int32_t p, int32_t q, const aosb_complex128* x,
                                 int64_t ldx, const aosb_complex128* y, int64_t ldy,
                                 aosb_complex128* g, void* stream, char* err, size_t cap) {
  using namespace aosb;
  if (x == nullptr || y == nullptr || g == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || p <= 0 || q <= 0 || ldx < p || ldy < q)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid gram shape");
  if (int rc = gram_grid_check(n, q, err, cap)) return rc;
  const size_t need = aosb_gram_scratch_bytes(n, p, q);
  if (need > kNoAllocGramBytes)
    return set_error(err, cap, AOSB_ERR_SIZE,
                     "aosb_gram_noalloc: n=%lld, p=%d, q=%d needs %zu bytes of partial sums, "
                     "more than its fixed %zu-byte scratch (ceil(n/512)*p*q*16 must not exceed "
                     "it); use aosb_gram with caller-provided scratch",
                     (long long)n, p, q, need, kNoAllocGramBytes);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return set_error(err, cap, AOSB_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "device index %d not supported", dev);
  void* scratch = nullptr;
  {
    // First call on a device: resolve the array's device address once, with
    // that device current (a synchronous runtime call; make this first call
    // before any stream capture).
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_gram_scratch);
      if (e != cudaSuccess || ptr == nullptr)
        return set_error(err, cap, AOSB_ERR_CUDA, "cudaGetSymbolAddress failed: %s",
                         cudaGetErrorString(e));
      g_noalloc_ptr[dev] = ptr;
    }
    scratch = g_noalloc_ptr[dev];
  }
  // Nothing in the scratch needs clearing: the partial kernel writes every
  // element that the reduction then reads.
  const int chunks = (int)((n + kGramRows - 1) / kGramRows);
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid(ceil_div(p, 32), ceil_div(q, 32), chunks);
  gram_partial_kernel<<<grid, 256, 0, st>>>(n, p, q, (const double2*)x, ldx, (const double2*)y,
                                            ldy, (double2*)scratch);
  const int64_t pq = (int64_t)p * q;
  gram_reduce_kernel<<<ceil_div(pq, 256), 256, 0, st>>>(chunks, pq, (const double2*)scratch,
                                                        (double2*)g);
  count_launches(2);
  return launch_check(err, cap, "gram_noalloc");
}
