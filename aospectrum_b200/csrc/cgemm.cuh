// CTA-level complex GEMM on FP32 SIMT cores: acc(BM x BN) += A(BM x K) B(K x BN).
//
// 256 threads; each owns a TM x TN micro-tile of complex accumulators.
// Operands are fetched through loader functors so the same core serves
// tiles stored planar (factor), interleaved (solve blocks), transposed,
// conjugated, triangular or row-permuted operands.  Shared memory holds one
// BK slice of each operand, A transposed (k-major) so the inner loop reads
// TM consecutive rows with one vector load.
#pragma once

#include "common.cuh"

namespace aosb {

template <int BM, int BN, int TM, int TN>
struct CgemmShape {
  static constexpr int kThreads = 256;
  static constexpr int kRowThreads = BM / TM;
  static constexpr int kColThreads = BN / TN;
  static_assert(kRowThreads * kColThreads == kThreads, "thread layout");
  static constexpr int BK = 16;
};

// Shared-memory staging for one BK slice.
template <int BM, int BN>
struct CgemmSmem {
  float ar[16][BM + 1];  // +1 keeps the transposed stores conflict-free
  float ai[16][BM + 1];
  float br[16][BN];
  float bi[16][BN];
};

// Runs the K loop. LoadA(m, k) -> float2, LoadB(k, n) -> float2 return the
// operand element (zero outside the valid range is the loader's job).
template <int BM, int BN, int TM, int TN, typename LoadA, typename LoadB>
__device__ __forceinline__ void cgemm_cta(float (&accr)[TM][TN], float (&acci)[TM][TN], int K,
                                          CgemmSmem<BM, BN>& sm, LoadA loadA, LoadB loadB) {
  using S = CgemmShape<BM, BN, TM, TN>;
  constexpr int BK = S::BK;
  const int tid = threadIdx.x;
  const int tr = tid / S::kColThreads;  // row group
  const int tc = tid % S::kColThreads;  // column group
  for (int k0 = 0; k0 < K; k0 += BK) {
    // Stage A: BM x BK elements, 256 threads.
#pragma unroll
    for (int e = tid; e < BM * BK; e += 256) {
      const int m = e / BK, kk = e % BK;
      float2 v = loadA(m, k0 + kk);
      sm.ar[kk][m] = v.x;
      sm.ai[kk][m] = v.y;
    }
#pragma unroll
    for (int e = tid; e < BK * BN; e += 256) {
      const int kk = e / BN, n = e % BN;
      float2 v = loadB(k0 + kk, n);
      sm.br[kk][n] = v.x;
      sm.bi[kk][n] = v.y;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a_r[TM], a_i[TM], b_r[TN], b_i[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) {
        a_r[i] = sm.ar[kk][tr * TM + i];
        a_i[i] = sm.ai[kk][tr * TM + i];
      }
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        b_r[j] = sm.br[kk][tc + j * S::kColThreads];
        b_i[j] = sm.bi[kk][tc + j * S::kColThreads];
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          accr[i][j] = fmaf(a_r[i], b_r[j], accr[i][j]);
          accr[i][j] = fmaf(-a_i[i], b_i[j], accr[i][j]);
          acci[i][j] = fmaf(a_r[i], b_i[j], acci[i][j]);
          acci[i][j] = fmaf(a_i[i], b_r[j], acci[i][j]);
        }
    }
    __syncthreads();
  }
}

// Output coordinates of accumulator (i, j) for the calling thread.
template <int BM, int BN, int TM, int TN>
__device__ __forceinline__ int cg_row(int i) {
  using S = CgemmShape<BM, BN, TM, TN>;
  return (threadIdx.x / S::kColThreads) * TM + i;
}
template <int BM, int BN, int TM, int TN>
__device__ __forceinline__ int cg_col(int j) {
  using S = CgemmShape<BM, BN, TM, TN>;
  return (threadIdx.x % S::kColThreads) + j * S::kColThreads;
}

}  // namespace aosb
