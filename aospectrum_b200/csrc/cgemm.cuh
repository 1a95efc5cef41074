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
// Two shared-memory slices: the global loads of slice s+1 are issued into
// registers before slice s is multiplied, then stored to the other slice.
// A_MN: consecutive threads fetch consecutive rows m of A (for operands
// read from a transposed tile, so that a warp reads along memory); by
// default consecutive threads fetch consecutive k.
template <int BM, int BN, int TM, int TN, bool A_MN = false, typename LoadA, typename LoadB>
__device__ __forceinline__ void cgemm_cta(float (&accr)[TM][TN], float (&acci)[TM][TN], int K,
                                          CgemmSmem<BM, BN> (&sm)[2], LoadA loadA, LoadB loadB) {
  using S = CgemmShape<BM, BN, TM, TN>;
  constexpr int BK = S::BK;
  constexpr int NA = (BM * BK + 255) / 256, NB = (BK * BN + 255) / 256;
  const int tid = threadIdx.x;
  const int tr = tid / S::kColThreads;  // row group
  const int tc = tid % S::kColThreads;  // column group
  float2 ra[NA], rb[NB];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int t = 0; t < NA; ++t) {
      const int e = tid + t * 256;
      if (e < BM * BK) {
        if (A_MN) ra[t] = loadA(e % BM, k0 + e / BM);
        else ra[t] = loadA(e / BK, k0 + e % BK);
      }
    }
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int e = tid + t * 256;
      if (e < BK * BN) rb[t] = loadB(k0 + e / BN, e % BN);
    }
  };
  auto stash = [&](CgemmSmem<BM, BN>& buf) {
#pragma unroll
    for (int t = 0; t < NA; ++t) {
      const int e = tid + t * 256;
      if (e < BM * BK) {
        const int m = A_MN ? e % BM : e / BK, kk = A_MN ? e / BM : e % BK;
        buf.ar[kk][m] = ra[t].x;
        buf.ai[kk][m] = ra[t].y;
      }
    }
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int e = tid + t * 256;
      if (e < BK * BN) {
        buf.br[e / BN][e % BN] = rb[t].x;
        buf.bi[e / BN][e % BN] = rb[t].y;
      }
    }
  };
  fetch(0);
  stash(sm[0]);
  __syncthreads();
  int cur = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    const bool more = k0 + BK < K;
    if (more) fetch(k0 + BK);
    const CgemmSmem<BM, BN>& b = sm[cur];
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a_r[TM], a_i[TM], b_r[TN], b_i[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) {
        a_r[i] = b.ar[kk][tr * TM + i];
        a_i[i] = b.ai[kk][tr * TM + i];
      }
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        b_r[j] = b.br[kk][tc + j * S::kColThreads];
        b_i[j] = b.bi[kk][tc + j * S::kColThreads];
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
    if (more) stash(sm[cur ^ 1]);
    __syncthreads();
    cur ^= 1;
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
