// Numeric tile LU of shifted pencils A_p = H(k_p) - z_p S(k_p) (plain FP32).
//
// Storage: factor[p][slot][2][T][T] floats, real plane then imaginary
// plane, each row-major.  Right-looking over tile steps k:
//   1. diag_lu: LU of tile (k,k) with partial pivoting inside the tile,
//      then in-place inversion of both triangles; the slot keeps inv(L_kk)
//      strictly below the diagonal and inv(U_kk) on and above it.
//   2. panel:   L_ik = A_ik inv(U_kk)        (i > k, CTA owns row strips)
//               U_kj = inv(L_kk) P_k A_kj    (j > k, CTA owns column strips)
//   3. schur:   A_ij -= L_ik U_kj            for every (i, j) target.
// All kernels batch over pencils (grid.y / grid.x).
#include <atomic>
#include "plan.h"
#include "cgemm.cuh"
#include "factor.h"

namespace aosb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ size_t tile_base(int64_t p, int64_t n_slots, int64_t slot, int T) {
  return ((size_t)p * (size_t)n_slots + (size_t)slot) * (size_t)(2 * T * T);
}

// ---------------------------------------------------------------------------
// Assembly of H - z S into the tile storage (factor must be zeroed first).
__global__ void assemble_kernel(int64_t n, int64_t nnz, const int64_t* __restrict__ indptr,
                                const int32_t* __restrict__ indices,
                                const float2* __restrict__ hv, const float2* __restrict__ sv,
                                const int32_t* __restrict__ pencil_k,
                                const double2* __restrict__ shifts,
                                const int32_t* __restrict__ pinv, const int32_t* __restrict__ slot,
                                int64_t nb, int64_t n_slots, int T, float* __restrict__ factor) {
  const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.y;
  if (warp >= n) return;
  const int64_t r = warp;
  const int64_t kp = pencil_k[p];
  const double2 zd = shifts[p];
  const float2 z = make_float2((float)zd.x, (float)zd.y);
  const float2* h = hv + kp * nnz;
  const float2* s = sv != nullptr ? sv + kp * nnz : nullptr;
  const int pr = pinv[r];
  const int I = pr / T, rr = pr - I * T;
  for (int64_t e = indptr[r] + lane; e < indptr[r + 1]; e += 32) {
    const int pc = pinv[indices[e]];
    const int J = pc / T, cc = pc - J * T;
    const int sl = slot[(int64_t)I * nb + J];
    const float2 hval = h[e];
    const float2 sval = s != nullptr ? s[e] : make_float2(0.f, 0.f);
    const float re = hval.x - (z.x * sval.x - z.y * sval.y);
    const float im = hval.y - (z.x * sval.y + z.y * sval.x);
    const size_t b = tile_base(p, n_slots, sl, T) + (size_t)rr * T + cc;
    factor[b] = re;
    factor[b + (size_t)T * T] = im;
  }
}

// Padding rows and columns carry an identity diagonal.
__global__ void pad_identity_kernel(int64_t n_pad, const int32_t* __restrict__ perm,
                                    const int32_t* __restrict__ diag_slot, int64_t n_slots, int T,
                                    float* __restrict__ factor) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.y;
  if (i >= n_pad || perm[i] >= 0) return;
  const int k = (int)(i / T), r = (int)(i - (int64_t)k * T);
  factor[tile_base(p, n_slots, diag_slot[k], T) + (size_t)r * T + r] = 1.0f;
}

// ---------------------------------------------------------------------------
// Diagonal tile: LU with partial pivoting in shared memory + triangle inverses.
// Rows are padded to T+1 floats so that walking a column touches 32
// different banks; 512 threads.
constexpr int kDiagThreads = 512;

template <int T>
constexpr size_t diag_smem_bytes() {
  // tile (2 planes, padded rows) + scratch column (2T) + perm (T) + the
  // recursive-inverse temporaries (2 planes of T*T/2)
  return (size_t)(2 * T * (T + 1) + 2 * T) * sizeof(float) + T * sizeof(int) +
         (size_t)T * T * sizeof(float);
}

template <int T>
__global__ void __launch_bounds__(kDiagThreads) diag_lu_kernel(int k, const int32_t* __restrict__ diag_slot,
                                                               int64_t n_slots, int64_t n_pad,
                                                               float* __restrict__ factor,
                                                               int32_t* __restrict__ pivots,
                                                               int32_t* __restrict__ status) {
  constexpr int LD = T + 1;
  extern __shared__ float smem[];
  float* ar = smem;               // T x LD
  float* ai = smem + T * LD;      // T x LD
  float* colr = ai + T * LD;      // T  (scratch column)
  float* coli = colr + T;         // T
  int* perm = (int*)(coli + T);   // T
  const int p = blockIdx.x;
  const int tid = threadIdx.x;
  float* g = factor + tile_base(p, n_slots, diag_slot[k], T);
  for (int e = tid; e < T * T; e += kDiagThreads) {
    const int r = e / T, c = e % T;  // T is a power of two
    ar[r * LD + c] = g[e];
    ai[r * LD + c] = g[e + T * T];
  }
  for (int r = tid; r < T; r += kDiagThreads) perm[r] = r;
  __syncthreads();
  int bad = 0;
  // Blocked right-looking LU with partial pivoting (LAPACK getrf order):
  // warp 0 factors each NB-column panel with warp-level syncs only, then all
  // threads apply the panel's row interchanges to the other columns, form
  // U12 = inv(L11) A12 and apply the rank-NB update of the trailing block.
  constexpr int NB = 8;
  __shared__ int s_swap[NB];
  const int warp = tid / 32, lane = tid % 32;
  const int ty = tid / 32, tx = tid % 32;
  for (int j0 = 0; j0 < T; j0 += NB) {
    if (warp == 0) {
      for (int j = j0; j < j0 + NB; ++j) {
        float best = -1.0f;
        int bi = j;
        for (int r = j + lane; r < T; r += 32) {
          const float m = fabsf(ar[r * LD + j]) + fabsf(ai[r * LD + j]);
          if (m > best) { best = m; bi = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        // every lane now holds the same (best, bi)
        if (bi != j && lane < NB) {
          const int c = j0 + lane;
          float t = ar[j * LD + c]; ar[j * LD + c] = ar[bi * LD + c]; ar[bi * LD + c] = t;
          t = ai[j * LD + c]; ai[j * LD + c] = ai[bi * LD + c]; ai[bi * LD + c] = t;
        }
        if (lane == 0) s_swap[j - j0] = bi;
        __syncwarp();
        float pr = ar[j * LD + j], pi = ai[j * LD + j];
        float d = pr * pr + pi * pi;
        if (!(d > 0.0f) || !isfinite(d)) {
          if (lane == 0) bad = isfinite(d) ? kDevZeroPivot : kDevNonFinite;
          pr = 1.0f; pi = 0.0f; d = 1.0f;
        }
        __syncwarp();
        if (lane == 0) { ar[j * LD + j] = pr; ai[j * LD + j] = pi; }
        const float ipr = pr / d, ipi = -pi / d;
        for (int r = j + 1 + lane; r < T; r += 32) {
          const float xr = ar[r * LD + j], xi = ai[r * LD + j];
          const float lr = xr * ipr - xi * ipi, li = xr * ipi + xi * ipr;
          ar[r * LD + j] = lr;
          ai[r * LD + j] = li;
          // rank-1 update of the remaining panel columns of row r
          for (int c = j + 1; c < j0 + NB; ++c) {
            const float ur = ar[j * LD + c], ui = ai[j * LD + c];
            ar[r * LD + c] -= lr * ur - li * ui;
            ai[r * LD + c] -= lr * ui + li * ur;
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // row interchanges of this panel, applied in order to the other columns
    for (int c = tid; c < T; c += kDiagThreads) {
      if (c >= j0 && c < j0 + NB) continue;
      for (int t = 0; t < NB; ++t) {
        const int j = j0 + t, bi = s_swap[t];
        if (bi != j) {
          float x = ar[j * LD + c]; ar[j * LD + c] = ar[bi * LD + c]; ar[bi * LD + c] = x;
          x = ai[j * LD + c]; ai[j * LD + c] = ai[bi * LD + c]; ai[bi * LD + c] = x;
        }
      }
    }
    if (tid == 0) {
      for (int t = 0; t < NB; ++t) {
        const int j = j0 + t, bi = s_swap[t];
        if (bi != j) { int x = perm[j]; perm[j] = perm[bi]; perm[bi] = x; }
      }
    }
    __syncthreads();
    // U12 = inv(L11) A12: forward substitution down each column c >= j0+NB
    for (int c = j0 + NB + tid; c < T; c += kDiagThreads) {
      for (int j = j0 + 1; j < j0 + NB; ++j) {
        float sr = ar[j * LD + c], si = ai[j * LD + c];
        for (int q = j0; q < j; ++q) {
          const float lr = ar[j * LD + q], li = ai[j * LD + q];
          const float ur = ar[q * LD + c], ui = ai[q * LD + c];
          sr -= lr * ur - li * ui;
          si -= lr * ui + li * ur;
        }
        ar[j * LD + c] = sr;
        ai[j * LD + c] = si;
      }
    }
    __syncthreads();
    // trailing update A22 -= L21 U12 (rank NB)
    for (int r = j0 + NB + ty; r < T; r += kDiagThreads / 32) {
      float lr[NB], li[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        lr[q] = ar[r * LD + j0 + q];
        li[q] = ai[r * LD + j0 + q];
      }
      for (int c = j0 + NB + tx; c < T; c += 32) {
        float sr = ar[r * LD + c], si = ai[r * LD + c];
#pragma unroll
        for (int q = 0; q < NB; ++q) {
          const float ur = ar[(j0 + q) * LD + c], ui = ai[(j0 + q) * LD + c];
          sr -= lr[q] * ur - li[q] * ui;
          si -= lr[q] * ui + li[q] * ur;
        }
        ar[r * LD + c] = sr;
        ai[r * LD + c] = si;
      }
    }
    __syncthreads();
  }
  // Triangle inverses by recursive 2x2 blocking: invert the 8x8 diagonal
  // blocks (one warp each), then for b = 8, 16, ... , T/2 combine adjacent
  // blocks:  X12 = -X11 U12 X22  (upper)  and  X21 = -X22 L21 X11  (unit
  // lower).  tr/ti hold the b x b temporaries of all pairs of a level.
  float* tr = colr + 2 * T + T;   // after perm (see diag_smem_bytes)
  float* ti = tr + T * T / 2;
  // ---- base: 8x8 diagonal blocks, warp w < T/8 takes block w
  if (warp < T / 8) {
    const int b0 = warp * 8;
    const int i = lane % 8;
    // upper, non-unit: column by column, lane i = row
    for (int j = 0; j < 8; ++j) {
      float cr[8], ci[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        cr[q] = ar[(b0 + q) * LD + b0 + j];
        ci[q] = ai[(b0 + q) * LD + b0 + j];
      }
      __syncwarp();
      const float dd = cr[j] * cr[j] + ci[j] * ci[j];
      const float dr = cr[j] / dd, di = -ci[j] / dd;
      if (lane < 8 && i <= j) {
        if (i == j) {
          ar[(b0 + j) * LD + b0 + j] = dr;
          ai[(b0 + j) * LD + b0 + j] = di;
        } else {
          float sr = 0.0f, si = 0.0f;
          for (int q = i; q < j; ++q) {
            const float xr = ar[(b0 + i) * LD + b0 + q], xi = ai[(b0 + i) * LD + b0 + q];
            sr += xr * cr[q] - xi * ci[q];
            si += xr * ci[q] + xi * cr[q];
          }
          ar[(b0 + i) * LD + b0 + j] = -(sr * dr - si * di);
          ai[(b0 + i) * LD + b0 + j] = -(sr * di + si * dr);
        }
      }
      __syncwarp();
    }
    // unit lower: columns right to left
    for (int j = 6; j >= 0; --j) {
      float cr[8], ci[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        cr[q] = ar[(b0 + q) * LD + b0 + j];
        ci[q] = ai[(b0 + q) * LD + b0 + j];
      }
      __syncwarp();
      if (lane < 8 && i > j) {
        float sr = cr[i], si = ci[i];
        for (int q = j + 1; q < i; ++q) {
          const float xr = ar[(b0 + i) * LD + b0 + q], xi = ai[(b0 + i) * LD + b0 + q];
          sr += xr * cr[q] - xi * ci[q];
          si += xr * ci[q] + xi * cr[q];
        }
        ar[(b0 + i) * LD + b0 + j] = -sr;
        ai[(b0 + i) * LD + b0 + j] = -si;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // ---- combine levels
  for (int b = 8; b < T; b *= 2) {
    const int pairs = T / (2 * b);
    const int per = b * b;
    // upper: T1 = U12 X22 (X22 upper incl. diagonal)
    for (int e = tid; e < pairs * per; e += kDiagThreads) {
      const int m = e / per, r = (e % per) / b, c = e % b;
      const int A0 = 2 * b * m, B0 = A0 + b;
      float sr = 0.0f, si = 0.0f;
      for (int q = 0; q <= c; ++q) {
        const float ur = ar[(A0 + r) * LD + B0 + q], ui = ai[(A0 + r) * LD + B0 + q];
        const float xr = ar[(B0 + q) * LD + B0 + c], xi = ai[(B0 + q) * LD + B0 + c];
        sr += ur * xr - ui * xi;
        si += ur * xi + ui * xr;
      }
      tr[e] = sr;
      ti[e] = si;
    }
    __syncthreads();
    // X12 = -X11 T1 (X11 upper incl. diagonal), written over U12
    for (int e = tid; e < pairs * per; e += kDiagThreads) {
      const int m = e / per, r = (e % per) / b, c = e % b;
      const int A0 = 2 * b * m, B0 = A0 + b;
      float sr = 0.0f, si = 0.0f;
      for (int q = r; q < b; ++q) {
        const float xr = ar[(A0 + r) * LD + A0 + q], xi = ai[(A0 + r) * LD + A0 + q];
        const float t_r = tr[m * per + q * b + c], t_i = ti[m * per + q * b + c];
        sr += xr * t_r - xi * t_i;
        si += xr * t_i + xi * t_r;
      }
      ar[(A0 + r) * LD + B0 + c] = -sr;
      ai[(A0 + r) * LD + B0 + c] = -si;
    }
    __syncthreads();
    // lower: T1 = L21 X11 (X11 unit lower)
    for (int e = tid; e < pairs * per; e += kDiagThreads) {
      const int m = e / per, r = (e % per) / b, c = e % b;
      const int A0 = 2 * b * m, B0 = A0 + b;
      float sr = ar[(B0 + r) * LD + A0 + c], si = ai[(B0 + r) * LD + A0 + c];
      for (int q = c + 1; q < b; ++q) {
        const float lr = ar[(B0 + r) * LD + A0 + q], li = ai[(B0 + r) * LD + A0 + q];
        const float xr = ar[(A0 + q) * LD + A0 + c], xi = ai[(A0 + q) * LD + A0 + c];
        sr += lr * xr - li * xi;
        si += lr * xi + li * xr;
      }
      tr[e] = sr;
      ti[e] = si;
    }
    __syncthreads();
    // X21 = -X22 T1 (X22 unit lower), written over L21
    for (int e = tid; e < pairs * per; e += kDiagThreads) {
      const int m = e / per, r = (e % per) / b, c = e % b;
      const int A0 = 2 * b * m, B0 = A0 + b;
      float sr = tr[m * per + r * b + c], si = ti[m * per + r * b + c];
      for (int q = 0; q < r; ++q) {
        const float xr = ar[(B0 + r) * LD + B0 + q], xi = ai[(B0 + r) * LD + B0 + q];
        const float t_r = tr[m * per + q * b + c], t_i = ti[m * per + q * b + c];
        sr += xr * t_r - xi * t_i;
        si += xr * t_i + xi * t_r;
      }
      ar[(B0 + r) * LD + A0 + c] = -sr;
      ai[(B0 + r) * LD + A0 + c] = -si;
    }
    __syncthreads();
  }
  for (int e = tid; e < T * T; e += kDiagThreads) {
    const int r = e / T, c = e % T;
    g[e] = ar[r * LD + c];
    g[e + T * T] = ai[r * LD + c];
  }
  for (int r = tid; r < T; r += kDiagThreads) pivots[(size_t)p * n_pad + (size_t)k * T + r] = perm[r];
  if (tid == 0 && bad != 0 && status[p] == 0) status[p] = bad;
}

// ---------------------------------------------------------------------------
// Panel updates.  blockIdx.x enumerates (tile, strip); blockIdx.y = pencil.
// L strips are 32 rows x T columns, U strips are T rows x 32 columns.
template <int T>
struct PanelCfg {
  static constexpr int kStrip = 32;
  static constexpr int kStrips = T / kStrip;
  // micro tiles so that (rows / TM) * (cols / TN) == 256
  static constexpr int LTM = T == 128 ? 4 : 2, LTN = T == 32 ? 2 : 4;   // 32 x T
  static constexpr int UTM = T == 32 ? 2 : (T == 64 ? 2 : 4), UTN = T == 32 ? 2 : 4;  // T x 32
  static_assert((32 / LTM) * (T / LTN) == 256, "L panel layout");
  static_assert((T / UTM) * (32 / UTN) == 256, "U panel layout");
};

template <int T>
__global__ void __launch_bounds__(kThreads) panel_kernel(int k, int nL, int nU,
                                                         const int32_t* __restrict__ lslot,
                                                         const int32_t* __restrict__ uslot,
                                                         const int32_t* __restrict__ diag_slot,
                                                         int64_t n_slots, int64_t n_pad,
                                                         float* __restrict__ factor,
                                                         const int32_t* __restrict__ pivots) {
  using C = PanelCfg<T>;
  constexpr int S = C::kStrip;
  constexpr size_t kRaw = 2 * (sizeof(CgemmSmem<S, T>) > sizeof(CgemmSmem<T, S>)
                                   ? sizeof(CgemmSmem<S, T>) : sizeof(CgemmSmem<T, S>));
  __shared__ __align__(16) unsigned char raw[kRaw];
  const int p = blockIdx.y;
  const int item = blockIdx.x / C::kStrips, strip = blockIdx.x % C::kStrips;
  const float* D = factor + tile_base(p, n_slots, diag_slot[k], T);
  if (item < nL) {
    // rows [strip*S, +S) of A_ik times inv(U_kk) (upper incl. diagonal)
    constexpr int TM = C::LTM, TN = C::LTN;
    auto& sm = *reinterpret_cast<CgemmSmem<S, T>(*)[2]>(raw);
    float* A = factor + tile_base(p, n_slots, lslot[item], T);
    float accr[TM][TN] = {}, acci[TM][TN] = {};
    const int r0 = strip * S;
    auto la = [&](int m, int q) {
      const size_t o = (size_t)(r0 + m) * T + q;
      return make_float2(A[o], A[o + T * T]);
    };
    auto lb = [&](int q, int c) {
      if (q > c) return make_float2(0.f, 0.f);
      const size_t o = (size_t)q * T + c;
      return make_float2(D[o], D[o + T * T]);
    };
    cgemm_cta<S, T, TM, TN>(accr, acci, T, sm, la, lb);
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const size_t o = (size_t)(r0 + cg_row<S, T, TM, TN>(i)) * T + cg_col<S, T, TM, TN>(j);
        A[o] = accr[i][j];
        A[o + T * T] = acci[i][j];
      }
  } else if (item < nL + nU) {
    // columns [strip*S, +S) of inv(L_kk) (P_k A_kj)
    constexpr int TM = C::UTM, TN = C::UTN;
    auto& sm = *reinterpret_cast<CgemmSmem<T, S>(*)[2]>(raw);
    float* A = factor + tile_base(p, n_slots, uslot[item - nL], T);
    const int32_t* pv = pivots + (size_t)p * n_pad + (size_t)k * T;
    float accr[TM][TN] = {}, acci[TM][TN] = {};
    const int c0 = strip * S;
    auto la = [&](int r, int q) {
      if (q > r) return make_float2(0.f, 0.f);
      if (q == r) return make_float2(1.f, 0.f);
      const size_t o = (size_t)r * T + q;
      return make_float2(D[o], D[o + T * T]);
    };
    auto lb = [&](int q, int c) {
      const size_t o = (size_t)pv[q] * T + c0 + c;
      return make_float2(A[o], A[o + T * T]);
    };
    cgemm_cta<T, S, TM, TN>(accr, acci, T, sm, la, lb);
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const size_t o = (size_t)cg_row<T, S, TM, TN>(i) * T + c0 + cg_col<T, S, TM, TN>(j);
        A[o] = accr[i][j];
        A[o + T * T] = acci[i][j];
      }
  }
}

// ---------------------------------------------------------------------------
// Schur update: blockIdx.x = (pair, sub-block), blockIdx.y = pencil.
template <int T>
struct SchurCfg {
  static constexpr int BM = T >= 64 ? 64 : 32;
  static constexpr int BN = T >= 64 ? 64 : 32;
  static constexpr int TM = T >= 64 ? 4 : 2;
  static constexpr int TN = T >= 64 ? 4 : 2;
  static constexpr int kSub = (T / BM) * (T / BN);
};

template <int T>
__global__ void __launch_bounds__(kThreads) schur_kernel(int nU, const int32_t* __restrict__ lslot,
                                                         const int32_t* __restrict__ uslot,
                                                         const int32_t* __restrict__ tslot,
                                                         int64_t n_slots, float* __restrict__ factor) {
  using C = SchurCfg<T>;
  constexpr int BM = C::BM, BN = C::BN, TM = C::TM, TN = C::TN;
  __shared__ CgemmSmem<BM, BN> sm[2];
  const int p = blockIdx.y;
  const int pair = blockIdx.x / C::kSub, sub = blockIdx.x % C::kSub;
  const int a = pair / nU, b = pair % nU;
  const int m0 = (sub / (T / BN)) * BM, n0 = (sub % (T / BN)) * BN;
  const float* L = factor + tile_base(p, n_slots, lslot[a], T);
  const float* U = factor + tile_base(p, n_slots, uslot[b], T);
  float* Cc = factor + tile_base(p, n_slots, tslot[pair], T);
  float accr[TM][TN] = {}, acci[TM][TN] = {};
  auto la = [&](int m, int q) {
    const size_t o = (size_t)(m0 + m) * T + q;
    return make_float2(L[o], L[o + T * T]);
  };
  auto lb = [&](int q, int c) {
    const size_t o = (size_t)q * T + n0 + c;
    return make_float2(U[o], U[o + T * T]);
  };
  cgemm_cta<BM, BN, TM, TN>(accr, acci, T, sm, la, lb);
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const size_t o = (size_t)(m0 + cg_row<BM, BN, TM, TN>(i)) * T + n0 + cg_col<BM, BN, TM, TN>(j);
      Cc[o] -= accr[i][j];
      Cc[o + T * T] -= acci[i][j];
    }
}

template <int T>
int ensure_diag_attr(char* err, size_t cap) {
  // kernel attributes belong to each device's context: set once per device
  // (devices past 63 set it on every call)
  static std::atomic<uint64_t> attr_devices{0};
  int device = 0;
  cudaGetDevice(&device);
  const uint64_t dev_bit = device < 64 ? (uint64_t)1 << device : 0;
  if (dev_bit != 0 && (attr_devices.load() & dev_bit) != 0) return 0;
  const size_t diag_smem = diag_smem_bytes<T>();
  cudaError_t e = cudaFuncSetAttribute(diag_lu_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)diag_smem);
  if (e != cudaSuccess)
    return set_error(err, cap, AOSB_ERR_CUDA, "diag_lu smem attribute: %s", cudaGetErrorString(e));
  attr_devices.fetch_or(dev_bit);
  return 0;
}

// Diagonal LU and panel updates of step k (FP32 SIMT).
template <int T>
void step_panels(const aosb_plan* P, const aosb_factor_args_v1* a, int64_t k) {
  cudaStream_t st = (cudaStream_t)a->stream;
  const int np = a->n_pencils;
  const size_t diag_smem = diag_smem_bytes<T>();
  diag_lu_kernel<T><<<np, kDiagThreads, diag_smem, st>>>((int)k, P->d_diag_slot, P->n_slots, P->n_pad,
                                                    a->factor, a->pivots, a->status);
  count_launches(1);
  const int nL = P->lb_off[k + 1] - P->lb_off[k];
  const int nU = P->ur_off[k + 1] - P->ur_off[k];
  if (nL + nU > 0) {
    dim3 grid((unsigned)((nL + nU) * PanelCfg<T>::kStrips), np);
    panel_kernel<T><<<grid, kThreads, 0, st>>>((int)k, nL, nU, P->d_lb_slot + P->lb_off[k],
                                               P->d_ur_slot + P->ur_off[k], P->d_diag_slot,
                                               P->n_slots, P->n_pad, a->factor, a->pivots);
    count_launches(1);
  }
}

template <int T>
int run_plain(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap,
              StepHook hook, void* hook_ctx) {
  cudaStream_t st = (cudaStream_t)a->stream;
  const int np = a->n_pencils;
  if (int rc = ensure_diag_attr<T>(err, cap)) return rc;
  for (int64_t k = 0; k < P->nb; ++k) {
    if (hook != nullptr)
      if (int rc = hook(hook_ctx, k, st, err, cap)) return rc;
    step_panels<T>(P, a, k);
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    if (nL > 0 && nU > 0) {
      const int64_t blocks = (int64_t)nL * nU * SchurCfg<T>::kSub;
      if (blocks > INT32_MAX) return set_error(err, cap, AOSB_ERR_SIZE, "schur grid too large");
      dim3 grid((unsigned)blocks, np);
      schur_kernel<T><<<grid, kThreads, 0, st>>>(nU, P->d_lb_slot + P->lb_off[k],
                                                 P->d_ur_slot + P->ur_off[k],
                                                 P->d_sc_slot + P->sc_off[k], P->n_slots, a->factor);
      count_launches(1);
    }
  }
  return launch_check(err, cap, "plain factorization");
}

}  // namespace

int factor_assemble(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap) {
  cudaStream_t st = (cudaStream_t)a->stream;
  const int np = a->n_pencils;
  const size_t bytes = (size_t)np * P->n_slots * 2 * P->T * P->T * sizeof(float);
  AOSB_CUDA_TRY(cudaMemsetAsync(a->factor, 0, bytes, st), err, cap);
  dim3 g1(ceil_div(P->n, 8), np);
  assemble_kernel<<<g1, 256, 0, st>>>(P->n, P->nnz, P->d_indptr, P->d_indices,
                                      (const float2*)a->h_values, (const float2*)a->s_values,
                                      a->pencil_k, (const double2*)a->shifts, P->d_pinv, P->d_slot,
                                      P->nb, P->n_slots, (int)P->T, a->factor);
  dim3 g2(ceil_div(P->n_pad, 256), np);
  pad_identity_kernel<<<g2, 256, 0, st>>>(P->n_pad, P->d_perm, P->d_diag_slot, P->n_slots,
                                          (int)P->T, a->factor);
  count_launches(2);
  return launch_check(err, cap, "assemble");
}

int factor_step_panels(const aosb_plan* P, const aosb_factor_args_v1* a, int k, char* err,
                       size_t cap) {
  switch (P->T) {
    case 32: if (int rc = ensure_diag_attr<32>(err, cap)) return rc; step_panels<32>(P, a, k); return 0;
    case 64: if (int rc = ensure_diag_attr<64>(err, cap)) return rc; step_panels<64>(P, a, k); return 0;
    case 128: if (int rc = ensure_diag_attr<128>(err, cap)) return rc; step_panels<128>(P, a, k); return 0;
  }
  return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "unsupported tile size");
}

int factor_step_diag(const aosb_plan* P, const aosb_factor_args_v1* a, int k, cudaStream_t st,
                     char* err, size_t cap) {
  if (P->T != 128) return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "diagonal step needs tile 128");
  if (int rc = ensure_diag_attr<128>(err, cap)) return rc;
  diag_lu_kernel<128><<<a->n_pencils, kDiagThreads, diag_smem_bytes<128>(), st>>>(
      k, P->d_diag_slot, P->n_slots, P->n_pad, a->factor, a->pivots, a->status);
  count_launches(1);
  return 0;
}

int factor_plain(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap,
                 StepHook hook, void* hook_ctx) {
  switch (P->T) {
    case 32: return run_plain<32>(P, a, err, cap, hook, hook_ctx);
    case 64: return run_plain<64>(P, a, err, cap, hook, hook_ctx);
    case 128: return run_plain<128>(P, a, err, cap, hook, hook_ctx);
  }
  return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "unsupported tile size");
}

}  // namespace aosb

extern "C" {

size_t aosb_factor_bytes(const aosb_plan_t* p, int32_t n_pencils) {
  if (p == nullptr || n_pencils <= 0) return 0;
  return (size_t)n_pencils * (size_t)p->n_slots * (size_t)(2 * p->T * p->T) * sizeof(float);
}

int aosb_factor(const aosb_plan_t* plan, const aosb_factor_args_v1* a, char* err, size_t cap) {
  using aosb::set_error;
  if (plan == nullptr || a == nullptr) return set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (a->abi_version != AOSPECTRUM_B200_ABI_VERSION || a->struct_size != sizeof(*a))
    return set_error(err, cap, AOSB_ERR_ABI, "factor args ABI mismatch");
  if (a->n_pencils <= 0 || a->n_pencils > 65535)
    return set_error(err, cap, AOSB_ERR_BATCH, "n_pencils must be in 1..65535");
  if (a->h_values == nullptr || a->pencil_k == nullptr ||
      a->shifts == nullptr || a->factor == nullptr || a->pivots == nullptr || a->status == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "required pointer is null");
  if (!plan->uploaded)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "call aosb_plan_upload first");
  int rc = aosb::factor_assemble(plan, a, err, cap);
  if (rc) return rc;
  if (a->precision == AOSB_PRECISION_PLAIN) return aosb::factor_plain(plan, a, err, cap);
  if (a->precision == AOSB_PRECISION_BF16X3 || a->precision == AOSB_PRECISION_BF16X3_FP32_PANELS ||
      a->precision == AOSB_PRECISION_BF16X3_ONE_STEP)
    return aosb::factor_tc(plan, a, err, cap);
  return set_error(err, cap, AOSB_ERR_ARGUMENT, "unknown precision %d", a->precision);
}

}  // extern "C"
