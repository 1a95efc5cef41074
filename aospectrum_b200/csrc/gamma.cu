// Real symmetric shifted factorization with inertia at the Gamma point
// (replaces aospectrum_cudss_shift_factor_{create_device,refactor_device,
// solve,get_stats,destroy}, native/src/aospectrum_cudss_shift_factor.c:
// 232-329 and 541-742, whose cuDSS symmetric factorization reports the
// inertia that drives the reference's ordinal locator,
// src/aospectrum/primme.py:281-397).
//
// A = H - sigma S is taken, as the reference's upper-triangle cuDSS view
// takes it, from the upper triangle (diagonal included) of the caller's CSR
// values, mirrored below.  It is factored by the same tile engine as the
// shifted pencils: symbolic plan (natural or nested-dissection order,
// whichever needs fewer flops), block elimination over 32/64/128-wide tiles
// with FP32 tile updates and partial pivoting inside each diagonal tile (a
// real A keeps every imaginary part exactly zero).
//
// Inertia.  The block elimination leaves on each diagonal tile k, just
// before its own LU, the Schur complement S_kk of everything eliminated
// before it: exactly the symmetric block elimination of P A P^T whatever
// the in-tile row pivoting was, because A_ik inv(A_kk) A_kj does not depend
// on how A_kk was factored.  By the inertia additivity of Schur complements
// (Haynsworth), In(A) = In(A_11) + In(A / A_11), applied tile by tile,
// In(A) = sum_k In(S_kk), and by Sylvester's law In(A) counts the
// eigenvalues of the pencil (H, S) (S positive definite) below, at and
// above sigma.  A hook on the factorization stream runs, before each
// diagonal LU, a Bunch-Kaufman symmetric-indefinite LDL^T of S_kk in FP64
// shared memory (1x1 and 2x2 pivots, alpha = (1 + sqrt(17)) / 8) and adds
// the signs of its D blocks to the counters.  Padding rows of the plan are
// identity rows: each adds one positive count, removed on the host.
#include "plan.h"
#include "factor.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

namespace aosb {
namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

constexpr int kInertiaThreads = 256;

template <int T>
constexpr size_t inertia_smem_bytes() {
  return (size_t)T * (T + 1) * sizeof(double);
}

// Block-wide max of |v| with its index (ties: smallest index).  All
// threads get the result.
__device__ __forceinline__ void block_argmax(double v, int idx, double* s_val, int* s_idx,
                                             double& out_v, int& out_i) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
  }
  if (lane == 0) { s_val[warp] = v; s_idx[warp] = idx; }
  __syncthreads();
  if (warp == 0) {
    v = lane < kInertiaThreads / 32 ? s_val[lane] : -1.0;
    idx = lane < kInertiaThreads / 32 ? s_idx[lane] : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, v, o);
      const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
      if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
    if (lane == 0) { s_val[0] = v; s_idx[0] = idx; }
  }
  __syncthreads();
  out_v = s_val[0];
  out_i = s_idx[0];
  __syncthreads();
}

// Inertia of the symmetric diagonal tile (k, k) of pencil blockIdx.x by a
// Bunch-Kaufman LDL^T (partial pivoting) in FP64 shared memory; adds
// (negative, zero, positive) counts and the number of symmetric
// interchanges to counts[p][0..3].  The real plane of the tile is read; it
// is symmetrized as (A + A^T) / 2 against FP32 rounding of the updates.
template <int T>
__global__ void __launch_bounds__(kInertiaThreads) tile_inertia_kernel(
    int k, const int32_t* __restrict__ diag_slot, int64_t n_slots,
    const float* __restrict__ factor, int32_t* __restrict__ counts) {
  constexpr int LD = T + 1;
  extern __shared__ double a[];
  __shared__ double s_val[kInertiaThreads / 32];
  __shared__ int s_idx[kInertiaThreads / 32];
  __shared__ int s_step, s_kind, s_swap_from, s_swap_to;
  const int p = blockIdx.x, tid = threadIdx.x;
  const float* g = factor + ((size_t)p * n_slots + diag_slot[k]) * (size_t)(2 * T * T);
  for (int e = tid; e < T * T; e += kInertiaThreads) {
    const int r = e / T, c = e % T;
    a[r * LD + c] = 0.5 * ((double)g[r * T + c] + (double)g[c * T + r]);
  }
  __syncthreads();
  const double alpha = (1.0 + sqrt(17.0)) / 8.0;
  int neg = 0, zero = 0, pos = 0, swaps = 0;   // kept by thread 0
  for (int j = 0; j < T;) {
    // lambda = max_{i > j} |a_ij|, at row r
    double lam;
    int r;
    {
      double v = -1.0;
      int idx = 0x7fffffff;
      for (int i = j + 1 + tid; i < T; i += kInertiaThreads) {
        const double m = fabs(a[i * LD + j]);
        if (m > v) { v = m; idx = i; }
      }
      block_argmax(v, idx, s_val, s_idx, lam, r);
    }
    // sigma = max_{i >= j, i != r} |a_ri| (only meaningful when lam > 0)
    double sig = 0.0;
    if (lam > 0.0) {
      double v = -1.0;
      int idx = 0x7fffffff, unused;
      for (int i = j + tid; i < T; i += kInertiaThreads)
        if (i != r) {
          const double m = fabs(a[r * LD + i]);
          if (m > v) { v = m; idx = i; }
        }
      block_argmax(v, idx, s_val, s_idx, sig, unused);
    }
    if (tid == 0) {
      const double ajj = fabs(a[j * LD + j]);
      int kind = 1, from = -1, to = -1;   // 1x1 / 2x2 pivot; swap rows/cols from <-> to
      if (lam <= 0.0 && ajj == 0.0) {
        kind = 0;                                    // zero column: exact zero pivot
      } else if (ajj >= alpha * lam) {
        kind = 1;
      } else if (ajj * sig >= alpha * lam * lam) {
        kind = 1;
      } else if (fabs(a[r * LD + r]) >= alpha * sig) {
        kind = 1; from = j; to = r;
      } else {
        kind = 2; from = j + 1; to = r;
      }
      if (j + 1 >= T && kind == 2) kind = 1;       // cannot happen: lam > 0 needs a row below
      s_kind = kind;
      s_swap_from = from;
      s_swap_to = to;
      if (from >= 0 && from != to) ++swaps;
    }
    __syncthreads();
    const int kind = s_kind, from = s_swap_from, to = s_swap_to;
    if (from >= 0 && from != to) {
      // symmetric interchange of rows/columns from <-> to in the trailing block
      for (int c = j + tid; c < T; c += kInertiaThreads) {
        const double x = a[from * LD + c];
        a[from * LD + c] = a[to * LD + c];
        a[to * LD + c] = x;
      }
      __syncthreads();
      for (int rr = j + tid; rr < T; rr += kInertiaThreads) {
        const double x = a[rr * LD + from];
        a[rr * LD + from] = a[rr * LD + to];
        a[rr * LD + to] = x;
      }
      __syncthreads();
    }
    if (kind == 0) {
      if (tid == 0) ++zero;
      j += 1;
    } else if (kind == 1) {
      const double d = a[j * LD + j];
      if (tid == 0) {
        if (d < 0.0) ++neg;
        else if (d > 0.0) ++pos;
        else ++zero;
      }
      if (d != 0.0) {
        const int m = T - j - 1;
        for (int e = tid; e < m * m; e += kInertiaThreads) {
          const int rr = j + 1 + e / m, cc = j + 1 + e % m;
          a[rr * LD + cc] -= a[rr * LD + j] * a[j * LD + cc] / d;
        }
      }
      __syncthreads();
      j += 1;
    } else {
      const double d11 = a[j * LD + j], d21 = a[(j + 1) * LD + j], d22 = a[(j + 1) * LD + j + 1];
      const double det = d11 * d22 - d21 * d21;
      if (tid == 0) {
        if (det < 0.0) { ++neg; ++pos; }
        else if (det > 0.0) { if (d11 + d22 > 0.0) pos += 2; else neg += 2; }
        else { ++zero; if (d11 + d22 > 0.0) ++pos; else if (d11 + d22 < 0.0) ++neg; else ++zero; }
      }
      if (det != 0.0) {
        // trailing -= C inv(D) C^T with C = a[j+2:, j:j+2]
        const double i11 = d22 / det, i12 = -d21 / det, i22 = d11 / det;
        const int m = T - j - 2;
        for (int e = tid; e < m * m; e += kInertiaThreads) {
          const int rr = j + 2 + e / m, cc = j + 2 + e % m;
          const double c1 = a[rr * LD + j], c2 = a[rr * LD + j + 1];
          const double e1 = a[j * LD + cc], e2 = a[(j + 1) * LD + cc];
          a[rr * LD + cc] -= c1 * (i11 * e1 + i12 * e2) + c2 * (i12 * e1 + i22 * e2);
        }
      }
      __syncthreads();
      j += 2;
    }
  }
  if (tid == 0) {
    atomicAdd(&counts[4 * p + 0], neg);
    atomicAdd(&counts[4 * p + 1], zero);
    atomicAdd(&counts[4 * p + 2], pos);
    atomicAdd(&counts[4 * p + 3], swaps);
  }
  (void)s_step;
}

// Symmetric-pattern values from the caller's real CSR values: entry q of
// the mirrored upper triangle takes the value at source position src[q].
__global__ void gather_upper_kernel(int64_t nnz, const int32_t* __restrict__ src,
                                    const float* __restrict__ h, const float* __restrict__ s,
                                    float2* __restrict__ hc, float2* __restrict__ sc) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnz) return;
  const int32_t e = src[q];
  hc[q] = make_float2(h[e], 0.0f);
  sc[q] = make_float2(s[e], 0.0f);
}

// work[i][c] = rhs[perm[i] + c * ld] (column-major real), 0 for padding.
__global__ void rhs_in_kernel(int64_t n_pad, int L, const int32_t* __restrict__ perm,
                              const float* __restrict__ rhs, int64_t ld,
                              float2* __restrict__ work) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_pad * L) return;
  const int64_t i = e / L;
  const int c = (int)(e - i * L);
  const int32_t r = perm[i];
  work[e] = make_float2(r >= 0 ? rhs[(int64_t)r + c * ld] : 0.0f, 0.0f);
}

// solution[r + c * ld] = Re work[pinv[r]][c].
__global__ void sol_out_kernel(int64_t n, int L, const int32_t* __restrict__ pinv,
                               const float2* __restrict__ work, float* __restrict__ sol,
                               int64_t ld) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * L) return;
  const int c = (int)(e / n);
  const int64_t r = e - (int64_t)c * n;
  sol[r + c * ld] = work[(int64_t)pinv[r] * L + c].x;
}

}  // namespace
}  // namespace aosb

struct aosb_shift_factor {
  aosb_plan* plan = nullptr;
  int64_t n = 0, nnz_sym = 0;
  int32_t max_rhs = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  int32_t* d_src = nullptr;
  float2* d_h = nullptr;
  float2* d_s = nullptr;
  float* d_factor = nullptr;
  int32_t* d_piv = nullptr;
  int32_t* d_status = nullptr;
  int32_t* d_pk = nullptr;
  double2* d_shift = nullptr;
  int32_t* d_counts = nullptr;
  float2* d_work = nullptr;
  void* d_scratch = nullptr;
  aosb_shift_factor_stats stats{};
};

namespace aosb {
namespace {

int inertia_hook(void* ctx, int64_t k, cudaStream_t st, char* err, size_t cap) {
  aosb_shift_factor* f = (aosb_shift_factor*)ctx;
  const aosb_plan* P = f->plan;
  switch (P->T) {
    case 32:
      tile_inertia_kernel<32><<<1, kInertiaThreads, inertia_smem_bytes<32>(), st>>>(
          (int)k, P->d_diag_slot, P->n_slots, f->d_factor, f->d_counts);
      break;
    case 64:
      tile_inertia_kernel<64><<<1, kInertiaThreads, inertia_smem_bytes<64>(), st>>>(
          (int)k, P->d_diag_slot, P->n_slots, f->d_factor, f->d_counts);
      break;
    case 128:
      tile_inertia_kernel<128><<<1, kInertiaThreads, inertia_smem_bytes<128>(), st>>>(
          (int)k, P->d_diag_slot, P->n_slots, f->d_factor, f->d_counts);
      break;
    default:
      return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "unsupported tile size");
  }
  count_launches(1);
  return 0;
}

int inertia_attributes(int T, char* err, size_t cap) {
  cudaError_t e = cudaSuccess;
  if (T == 64)
    e = cudaFuncSetAttribute(tile_inertia_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)inertia_smem_bytes<64>());
  else if (T == 128)
    e = cudaFuncSetAttribute(tile_inertia_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)inertia_smem_bytes<128>());
  if (e != cudaSuccess)
    return set_error(err, cap, AOSB_ERR_CUDA, "tile inertia smem attribute: %s",
                     cudaGetErrorString(e));
  return 0;
}

int pick_gamma_tile(int64_t n) { return n <= 512 ? 32 : (n <= 6000 ? 64 : 128); }

// Factor the current values at `shift` and read the inertia back.
int factorize(aosb_shift_factor* f, float shift, char* err, size_t cap) {
  const aosb_plan* P = f->plan;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  f->stats.free_device_bytes_before_factorization = free_b;
  f->stats.factorization_seconds = 0.0;
  f->stats.solve_seconds = 0.0;
  f->stats.solve_calls = 0;
  f->stats.solved_rhs = 0;
  const double t0 = now_s();
  const double2 z = make_double2((double)shift, 0.0);
  AOSB_CUDA_TRY(cudaMemcpyAsync(f->d_shift, &z, sizeof(z), cudaMemcpyHostToDevice, f->stream),
                err, cap);
  AOSB_CUDA_TRY(cudaMemsetAsync(f->d_counts, 0, 4 * sizeof(int32_t), f->stream), err, cap);
  AOSB_CUDA_TRY(cudaMemsetAsync(f->d_status, 0, sizeof(int32_t), f->stream), err, cap);
  aosb_factor_args_v1 fa{AOSPECTRUM_B200_ABI_VERSION, sizeof(aosb_factor_args_v1), 1,
                         AOSB_PRECISION_PLAIN, (const aosb_complex64*)f->d_h,
                         (const aosb_complex64*)f->d_s, f->d_pk, (const aosb_complex128*)f->d_shift,
                         f->d_factor, f->d_piv, f->d_status, nullptr, f->stream};
  if (int rc = inertia_attributes((int)P->T, err, cap)) return rc;
  if (int rc = factor_assemble(P, &fa, err, cap)) return rc;
  if (int rc = factor_plain(P, &fa, err, cap, inertia_hook, f)) return rc;
  int32_t counts[4] = {0, 0, 0, 0}, status = 0;
  AOSB_CUDA_TRY(cudaMemcpyAsync(counts, f->d_counts, sizeof(counts), cudaMemcpyDeviceToHost,
                                f->stream), err, cap);
  AOSB_CUDA_TRY(cudaMemcpyAsync(&status, f->d_status, sizeof(status), cudaMemcpyDeviceToHost,
                                f->stream), err, cap);
  AOSB_CUDA_TRY(cudaStreamSynchronize(f->stream), err, cap);
  f->stats.factorization_seconds = now_s() - t0;
  if (status != 0)
    return set_error(err, cap, AOSB_ERR_DEVICE_INFO,
                     "shifted symmetric factorization reported status %d (%s)", status,
                     status == AOSB_ERR_ZERO_PIVOT ? "singular at this shift" : "non-finite");
  const int64_t padding = P->n_pad - P->n;
  f->stats.inertia_negative = counts[0];
  f->stats.inertia_positive = (int32_t)(counts[2] - padding);
  f->stats.pivot_count = counts[3];
  f->stats.factor_nnz = P->n_slots * P->T * P->T;
  cudaMemGetInfo(&free_b, &total_b);
  f->stats.free_device_bytes_after_factorization = free_b;
  if (counts[0] < 0 || counts[2] - padding < 0 || counts[0] + counts[2] - padding > f->n)
    return set_error(err, cap, AOSB_ERR_DEVICE_INFO, "inertia counts are invalid");
  return 0;
}

int gather_values(aosb_shift_factor* f, const float* h, const float* s, char* err, size_t cap) {
  gather_upper_kernel<<<ceil_div(f->nnz_sym, 256), 256, 0, f->stream>>>(f->nnz_sym, f->d_src, h, s,
                                                                        f->d_h, f->d_s);
  count_launches(1);
  return launch_check(err, cap, "gamma value gather");
}

}  // namespace
}  // namespace aosb

extern "C" {

void aosb_shift_factor_destroy(aosb_shift_factor_t* f) {
  if (f == nullptr) return;
  cudaFree(f->d_src);
  cudaFree(f->d_h);
  cudaFree(f->d_s);
  cudaFree(f->d_factor);
  cudaFree(f->d_piv);
  cudaFree(f->d_status);
  cudaFree(f->d_pk);
  cudaFree(f->d_shift);
  cudaFree(f->d_counts);
  cudaFree(f->d_work);
  cudaFree(f->d_scratch);
  if (f->plan) aosb_plan_destroy(f->plan);
  delete f;
}

int aosb_shift_factor_create_device(aosb_shift_factor_t** out, int64_t n, int64_t nnz,
                                    const int32_t* indptr, const int32_t* indices,
                                    const float* device_h, const float* device_s, float shift,
                                    int32_t maximum_rhs, void* stream, char* err, size_t cap) {
  using namespace aosb;
  if (out == nullptr) return set_error(err, cap, AOSB_ERR_NULL, "factor output pointer is null");
  *out = nullptr;
  if (n <= 0 || n > INT32_MAX || nnz <= 0 || nnz > INT32_MAX || indptr == nullptr ||
      indices == nullptr || device_h == nullptr || device_s == nullptr || !std::isfinite(shift) ||
      maximum_rhs <= 0 || maximum_rhs > 256)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid shift-factor request");
  if (indptr[0] != 0 || indptr[n] != nnz)
    return set_error(err, cap, AOSB_ERR_INDPTR, "CSR row offsets do not span the declared nnz");
  const double t_prep = now_s();
  // Upper triangle (diagonal included) with its source positions, then the
  // mirrored symmetric pattern sorted by column in every row.
  std::vector<std::vector<std::pair<int32_t, int32_t>>> rows((size_t)n);
  int64_t upper = 0, diag = 0;
  for (int64_t r = 0; r < n; ++r) {
    const int32_t b = indptr[r], e = indptr[r + 1];
    if (b < 0 || e < b || e > nnz)
      return set_error(err, cap, AOSB_ERR_CSR_MONOTONIC, "CSR row offsets are not monotonic");
    int32_t prev = -1;
    for (int32_t q = b; q < e; ++q) {
      const int32_t c = indices[q];
      if (c < 0 || c >= n)
        return set_error(err, cap, AOSB_ERR_CSR_COLUMN, "CSR column index is outside the matrix");
      if (c <= prev)
        return set_error(err, cap, AOSB_ERR_CSR_ORDER, "CSR columns must be sorted and duplicate-free");
      prev = c;
      if (c < r) continue;
      ++upper;
      rows[(size_t)r].emplace_back(c, q);
      if (c == r) ++diag;
      else rows[(size_t)c].emplace_back((int32_t)r, q);
    }
  }
  if (diag != n)
    return set_error(err, cap, AOSB_ERR_DIAGONAL,
                     "shifted matrix is missing diagonal entries: %lld/%lld", (long long)diag,
                     (long long)n);
  std::vector<int64_t> sp((size_t)n + 1, 0);
  for (int64_t r = 0; r < n; ++r) sp[(size_t)r + 1] = sp[(size_t)r] + (int64_t)rows[(size_t)r].size();
  const int64_t nsym = sp[(size_t)n];
  std::vector<int32_t> si((size_t)nsym), src((size_t)nsym);
  for (int64_t r = 0; r < n; ++r) {
    auto& v = rows[(size_t)r];
    std::sort(v.begin(), v.end());
    for (size_t t = 0; t < v.size(); ++t) {
      si[(size_t)sp[(size_t)r] + t] = v[t].first;
      src[(size_t)sp[(size_t)r] + t] = v[t].second;
    }
  }
  rows.clear();
  rows.shrink_to_fit();
  aosb_shift_factor* f = new aosb_shift_factor();
  f->n = n;
  f->nnz_sym = nsym;
  f->max_rhs = maximum_rhs;
  f->stream = (cudaStream_t)stream;
  cudaGetDevice(&f->device);
  f->stats.upper_nnz = upper;
  f->stats.preparation_seconds = now_s() - t_prep;
  // Symbolic analysis: both orderings, the one with fewer flops.
  const double t_an = now_s();
  const int T = pick_gamma_tile(n);
  for (int ordering = 0; ordering < 2; ++ordering) {
    aosb_plan_options_v1 opt{AOSPECTRUM_B200_ABI_VERSION, sizeof(aosb_plan_options_v1), T, ordering,
                             4 * T, 1};
    aosb_plan* cand = nullptr;
    if (int rc = aosb_plan_create(n, sp.data(), si.data(), nullptr, 0, &opt, &cand, err, cap)) {
      aosb_shift_factor_destroy(f);
      return rc;
    }
    if (f->plan == nullptr || cand->flops < f->plan->flops) {
      if (f->plan) aosb_plan_destroy(f->plan);
      f->plan = cand;
    } else {
      aosb_plan_destroy(cand);
    }
  }
  int rc = aosb_plan_upload(f->plan, err, cap);
  f->stats.analysis_seconds = now_s() - t_an;
  if (rc) {
    aosb_shift_factor_destroy(f);
    return rc;
  }
  const aosb_plan* P = f->plan;
  const double t_up = now_s();
  auto alloc = [&](void** p, size_t bytes, const char* what) -> int {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) return 0;
    return set_error(err, cap, e == cudaErrorMemoryAllocation ? AOSB_ERR_MEMORY : AOSB_ERR_CUDA,
                     "%s allocation failed: %s", what, cudaGetErrorString(e));
  };
  const size_t fbytes = aosb_factor_bytes(P, 1);
  const size_t scratch = aosb_solve_scratch_bytes(P, 1, maximum_rhs);
  const int32_t zero = 0;
  if ((rc = alloc((void**)&f->d_src, sizeof(int32_t) * nsym, "source positions")) ||
      (rc = alloc((void**)&f->d_h, sizeof(float2) * nsym, "H values")) ||
      (rc = alloc((void**)&f->d_s, sizeof(float2) * nsym, "S values")) ||
      (rc = alloc((void**)&f->d_factor, fbytes, "factor")) ||
      (rc = alloc((void**)&f->d_piv, sizeof(int32_t) * P->n_pad, "pivots")) ||
      (rc = alloc((void**)&f->d_status, sizeof(int32_t), "status")) ||
      (rc = alloc((void**)&f->d_pk, sizeof(int32_t), "pencil index")) ||
      (rc = alloc((void**)&f->d_shift, sizeof(double2), "shift")) ||
      (rc = alloc((void**)&f->d_counts, 4 * sizeof(int32_t), "inertia counters")) ||
      (rc = alloc((void**)&f->d_work, sizeof(float2) * P->n_pad * maximum_rhs, "solve block")) ||
      (rc = alloc(&f->d_scratch, scratch > 16 ? scratch : 16, "solve scratch"))) {
    aosb_shift_factor_destroy(f);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(f->d_src, src.data(), sizeof(int32_t) * nsym,
                                  cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(f->d_pk, &zero, sizeof(zero), cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) {
    aosb_shift_factor_destroy(f);
    return set_error(err, cap, AOSB_ERR_CUDA, "shift-factor upload failed: %s", cudaGetErrorString(e));
  }
  f->stats.permanent_device_bytes = fbytes + sizeof(int32_t) * P->n_pad +
                                    (sizeof(int32_t) + 2 * sizeof(float2)) * nsym;
  f->stats.peak_device_bytes = f->stats.permanent_device_bytes +
                               sizeof(float2) * P->n_pad * maximum_rhs + scratch;
  f->stats.permanent_host_bytes = 0;
  f->stats.peak_host_bytes = (sizeof(int32_t) * 2 + sizeof(int64_t)) * (size_t)nsym;
  if ((rc = gather_values(f, device_h, device_s, err, cap))) {
    aosb_shift_factor_destroy(f);
    return rc;
  }
  f->stats.upload_seconds = now_s() - t_up;
  if ((rc = factorize(f, shift, err, cap))) {
    aosb_shift_factor_destroy(f);
    return rc;
  }
  *out = f;
  return 0;
}

int aosb_shift_factor_refactor_device(aosb_shift_factor_t* f, const float* device_h,
                                      const float* device_s, float shift, char* err, size_t cap) {
  using namespace aosb;
  if (f == nullptr || device_h == nullptr || device_s == nullptr || !std::isfinite(shift))
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid refactor request");
  f->stats.preparation_seconds = 0.0;
  f->stats.upload_seconds = 0.0;
  f->stats.analysis_seconds = 0.0;
  const double t0 = now_s();
  if (int rc = gather_values(f, device_h, device_s, err, cap)) return rc;
  f->stats.upload_seconds = now_s() - t0;
  return factorize(f, shift, err, cap);
}

int aosb_shift_factor_solve(aosb_shift_factor_t* f, const float* rhs, int64_t leading_rhs,
                            float* solution, int64_t leading_solution, int32_t rhs_count,
                            char* err, size_t cap) {
  using namespace aosb;
  if (f == nullptr || rhs == nullptr || solution == nullptr || rhs_count <= 0 ||
      rhs_count > f->max_rhs || leading_rhs < f->n || leading_solution < f->n)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid shifted-solve request");
  const aosb_plan* P = f->plan;
  const double t0 = now_s();
  const int L = rhs_count;
  rhs_in_kernel<<<ceil_div(P->n_pad * L, 256), 256, 0, f->stream>>>(P->n_pad, L, P->d_perm, rhs,
                                                                    leading_rhs, f->d_work);
  count_launches(1);
  aosb_solve_args_v1 sa{AOSPECTRUM_B200_ABI_VERSION, sizeof(aosb_solve_args_v1), 1, L, 0, 0,
                        f->d_factor, f->d_piv, (aosb_complex64*)f->d_work, f->d_scratch, f->stream};
  if (int rc = aosb_solve(P, &sa, err, cap)) return rc;
  sol_out_kernel<<<ceil_div(f->n * L, 256), 256, 0, f->stream>>>(f->n, L, P->d_pinv, f->d_work,
                                                                 solution, leading_solution);
  count_launches(1);
  AOSB_CUDA_TRY(cudaStreamSynchronize(f->stream), err, cap);
  if (int rc = launch_check(err, cap, "shifted symmetric solve")) return rc;
  f->stats.solve_seconds += now_s() - t0;
  ++f->stats.solve_calls;
  f->stats.solved_rhs += rhs_count;
  return 0;
}

void aosb_shift_factor_get_stats(const aosb_shift_factor_t* f, aosb_shift_factor_stats* stats) {
  if (stats == nullptr) return;
  if (f == nullptr) {
    std::memset(stats, 0, sizeof(*stats));
    return;
  }
  *stats = f->stats;
}

}  // extern "C"
