// Tensor-core (tcgen05) update step of the block-RHS triangular sweeps for
// tile 128: X_i -= op(F) Y for every listed tile F of the step, with
// op(F) = F (plain) or F^H (adjoint sweeps) and Y the step's diagonal
// result (T x n_rhs complex64, computed by the SIMT diagonal kernel).
//
// One CTA (4 warps) per (tile, 64-column RHS strip, pencil):
//   * the Y strip is split into four BF16 planes (re_hi, re_lo, im_hi,
//     im_lo; x = hi + lo) as the K-major B operand (N = strip columns
//     rounded up to 16, K = 128) in shared memory;
//   * the FP32 factor tile is read from HBM in 16-wide K slabs, split the
//     same way into the K-major A operand (M = 128) in a two-slab ring, and
//     for each slab one thread issues 12 tcgen05.mma.kind::f16 into two
//     FP32 TMEM accumulators (the split-BF16 complex product of the
//     factorization: hi*hi + hi*lo + lo*hi per real product);
//   * each warp reads its 32 rows of the accumulators with tcgen05.ld and
//     subtracts them from X_i.
// The conversion of slab s+1 overlaps the MMAs of slab s; each slab buffer
// is rewritten only after the tcgen05.commit of the MMAs that read it has
// arrived on its mbarrier.  Every wait is bounded: on expiry the CTA
// records AOSB_ERR_TIMEOUT in the pencil status, skips the rest, waits
// (bounded) for MMAs in flight and frees its TMEM.
#include "plan.h"
#include "tc_common.cuh"

#include <cuda_bf16.h>

namespace aosb {
namespace {

using namespace tc;

constexpr int kT = 128;
constexpr int kNS = 64;                    // RHS columns per CTA
constexpr int kSK = 16;                    // K per slab
constexpr int kSlabsS = kT / kSK;          // 8
constexpr int kSThreads = 128;
constexpr int kACols = 2 * kNS;            // TMEM columns: re [0, kNS), im [kNS, 2 kNS)
constexpr int kAPlane = kT * kSK * 2;      // 4096 bytes: one plane of one A slab
constexpr int kASlab = 4 * kAPlane;        // 16 KB
constexpr int kBPlaneSlab = kNS * kSK * 2;  // 2048 bytes
constexpr int kBSlab = 4 * kBPlaneSlab;    // 8 KB
constexpr int kCopyCtas = 4;

enum SolveOp { kOpPlain = 0, kOpConjT = 1 };

struct SShared {
  alignas(1024) unsigned char b[kSlabsS][kBSlab];   // 64 KB
  alignas(1024) unsigned char a[2][kASlab];          // 32 KB
  uint64_t done[2];
  uint32_t tmem_base;
  int failed;
};

// K-major no-swizzle core-matrix layout (8 rows x 16 bytes), the two 8-wide
// K halves of a slab `rows / 8 * 128` bytes apart.
__device__ __forceinline__ uint32_t a_off(int m, int k, int plane) {
  return (uint32_t)(plane * kAPlane + (k / 8) * ((kT / 8) * 128) + (m / 8) * 128 + (m % 8) * 16 +
                    (k % 8) * 2);
}
__device__ __forceinline__ uint32_t b_off(int n, int k, int plane) {
  const int slab = k / kSK, kk = k % kSK;
  return (uint32_t)(slab * kBSlab + plane * kBPlaneSlab + (kk / 8) * ((kNS / 8) * 128) +
                    (n / 8) * 128 + (n % 8) * 16 + (kk % 8) * 2);
}

__device__ __forceinline__ void split2(float x0, float x1, __nv_bfloat162& hi, __nv_bfloat162& lo) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
  hi.x = h0;
  hi.y = h1;
  lo.x = __float2bfloat16_rn(x0 - __bfloat162float(h0));
  lo.y = __float2bfloat16_rn(x1 - __bfloat162float(h1));
}

template <int OP>
__global__ void __launch_bounds__(kSThreads) solve_tc_kernel(
    int k, int n_items, int nrhs, int64_t n_pad, const int32_t* __restrict__ tiles,
    const int32_t* __restrict__ slots, int64_t n_slots, const float* __restrict__ factor,
    float2* __restrict__ work, const float2* __restrict__ ytmp, int32_t* __restrict__ status) {
  const int p = blockIdx.y;
  const int strips = (nrhs + kNS - 1) / kNS;
  const int work_blocks = n_items * strips;
  const float2* Y = ytmp + (size_t)p * kT * nrhs;
  if ((int)blockIdx.x >= work_blocks) {
    // copy-back CTAs: X_k = Y
    const int cb = blockIdx.x - work_blocks;
    float2* Xk = work + ((size_t)p * n_pad + (size_t)k * kT) * nrhs;
    const int total = kT * nrhs;
    for (int e = cb * kSThreads + threadIdx.x; e < total; e += kCopyCtas * kSThreads) Xk[e] = Y[e];
    return;
  }
  extern __shared__ unsigned char dyn[];
  SShared& sh = *reinterpret_cast<SShared*>(
      (reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
  const int item = blockIdx.x / strips, strip = blockIdx.x % strips;
  const int c0 = strip * kNS;
  const int ncols = nrhs - c0 < kNS ? nrhs - c0 : kNS;
  const int n16 = (ncols + 15) & ~15;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const float* F = factor + ((size_t)p * (size_t)n_slots + (size_t)slots[item]) * (2 * kT * kT);
  float2* Xi = work + ((size_t)p * n_pad + (size_t)tiles[item] * kT) * nrhs;

  if (tid == 0) {
    mbar_init(&sh.done[0], 1);
    mbar_init(&sh.done[1], 1);
    sh.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem_base)),
                 "r"(kACols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // B operand: element (n, q) = Y[q][c0 + n], zero beyond the strip
  for (int e = tid; e < kNS * (kT / 2); e += kSThreads) {
    const int n = e % kNS, q = (e / kNS) * 2;
    float2 y0 = make_float2(0.f, 0.f), y1 = y0;
    if (n < ncols) {
      y0 = Y[(size_t)q * nrhs + c0 + n];
      y1 = Y[(size_t)(q + 1) * nrhs + c0 + n];
    }
    __nv_bfloat162 rh, rl, ih, il;
    split2(y0.x, y1.x, rh, rl);
    split2(y0.y, y1.y, ih, il);
    unsigned char* b = &sh.b[0][0];
    *reinterpret_cast<__nv_bfloat162*>(b + b_off(n, q, 0)) = rh;
    *reinterpret_cast<__nv_bfloat162*>(b + b_off(n, q, 1)) = rl;
    *reinterpret_cast<__nv_bfloat162*>(b + b_off(n, q, 2)) = ih;
    *reinterpret_cast<__nv_bfloat162*>(b + b_off(n, q, 3)) = il;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem_base;
  const uint32_t id_pos = umma_idesc_mn(kT, n16, false), id_neg = umma_idesc_mn(kT, n16, true);
  int issued = 0;  // slabs whose MMAs were committed

  for (int s = 0; s < kSlabsS; ++s) {
    const int buf = s & 1;
    if (s >= 2) {
      const bool ok = mbar_wait(&sh.done[buf], (uint32_t)(((s - 2) >> 1) & 1));
      if (!ok && tid == 0) sh.failed = 1;
    }
    __syncthreads();
    if (sh.failed) break;
    unsigned char* a = sh.a[buf];
    const int k0 = s * kSK;
    // A operand slab: element (m, q) = F[m][k0 + q] or conj(F[k0 + q][m])
    for (int e = tid; e < kT * (kSK / 2); e += kSThreads) {
      int m, q;
      float r0, r1, i0, i1;
      if (OP == kOpPlain) {
        m = e / (kSK / 2);
        q = (e % (kSK / 2)) * 2;
        const size_t o = (size_t)m * kT + k0 + q;
        const float2 rr = *reinterpret_cast<const float2*>(F + o);
        const float2 ii = *reinterpret_cast<const float2*>(F + kT * kT + o);
        r0 = rr.x; r1 = rr.y; i0 = ii.x; i1 = ii.y;
      } else {
        m = e % kT;
        q = (e / kT) * 2;
        const size_t o0 = (size_t)(k0 + q) * kT + m, o1 = o0 + kT;
        r0 = F[o0]; r1 = F[o1];
        i0 = -F[kT * kT + o0]; i1 = -F[kT * kT + o1];
      }
      __nv_bfloat162 rh, rl, ih, il;
      split2(r0, r1, rh, rl);
      split2(i0, i1, ih, il);
      *reinterpret_cast<__nv_bfloat162*>(a + a_off(m, q, 0)) = rh;
      *reinterpret_cast<__nv_bfloat162*>(a + a_off(m, q, 1)) = rl;
      *reinterpret_cast<__nv_bfloat162*>(a + a_off(m, q, 2)) = ih;
      *reinterpret_cast<__nv_bfloat162*>(a + a_off(m, q, 3)) = il;
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(a), sb = smem_u32(sh.b[s]);
      const uint32_t alb = (kT / 8) * 128, blb = (kNS / 8) * 128;
      uint64_t A[4], Bv[4];
#pragma unroll
      for (int pl = 0; pl < 4; ++pl) {
        A[pl] = umma_desc(sa + pl * kAPlane, alb, 128);
        Bv[pl] = umma_desc(sb + pl * kBPlaneSlab, blb, 128);
      }
      const uint32_t re = tmem, im = tmem + kNS;
      const uint32_t first = s == 0 ? 0u : 1u;
      umma_bf16(re, A[0], Bv[0], id_pos, first);
      umma_bf16(re, A[0], Bv[1], id_pos, 1);
      umma_bf16(re, A[1], Bv[0], id_pos, 1);
      umma_bf16(re, A[2], Bv[2], id_neg, 1);
      umma_bf16(re, A[2], Bv[3], id_neg, 1);
      umma_bf16(re, A[3], Bv[2], id_neg, 1);
      umma_bf16(im, A[0], Bv[2], id_pos, first);
      umma_bf16(im, A[0], Bv[3], id_pos, 1);
      umma_bf16(im, A[1], Bv[2], id_pos, 1);
      umma_bf16(im, A[2], Bv[0], id_pos, 1);
      umma_bf16(im, A[2], Bv[1], id_pos, 1);
      umma_bf16(im, A[3], Bv[0], id_pos, 1);
      umma_commit(&sh.done[buf]);
    }
    issued = s + 1;
  }
  // wait for the MMAs of the last two committed slabs (bounded)
  bool ok = true;
  for (int s = issued - 2 < 0 ? 0 : issued - 2; s < issued; ++s)
    ok = mbar_wait(&sh.done[s & 1], (uint32_t)((s >> 1) & 1)) && ok;
  if (!ok || issued < kSlabsS) {
    if (tid == 0) atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // X_i rows 32 w + lane -= acc (columns [0, ncols) of the strip)
    const int row = warp * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
    float2* xr = Xi + (size_t)row * nrhs + c0;
    for (int c = 0; c < n16; c += 16) {
      float vr[16], vi[16];
      tmem_ld16(tmem + lane_addr + c, vr);
      tmem_ld16(tmem + lane_addr + kNS + c, vi);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        if (c + j < ncols) {
          float2 v = xr[c + j];
          v.x -= vr[j];
          v.y -= vi[j];
          xr[c + j] = v;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kACols));
  }
}

}  // namespace

size_t solve_tc_smem() { return sizeof(SShared) + 1024; }

// Launch the tensor-core update of step k for n tiles (device lists).
int solve_tc_update(int k, int n, const int32_t* dtiles, const int32_t* dslots, int op,
                    int np, int nrhs, const aosb_plan* P, const float* factor, float2* work,
                    const float2* ytmp, int32_t* status, cudaStream_t st, char* err, size_t cap) {
  static bool attr_done[2] = {false, false};
  const size_t smem = solve_tc_smem();
  static_assert(sizeof(SShared) + 1024 <= 232448, "shared memory budget");
  if (!attr_done[op]) {
    cudaError_t e = op == kOpPlain
                        ? cudaFuncSetAttribute(solve_tc_kernel<kOpPlain>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                        : cudaFuncSetAttribute(solve_tc_kernel<kOpConjT>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
      return set_error(err, cap, AOSB_ERR_CUDA, "solve_tc smem attribute: %s", cudaGetErrorString(e));
    attr_done[op] = true;
  }
  const int strips = (nrhs + kNS - 1) / kNS;
  dim3 g((unsigned)(n * strips + kCopyCtas), np);
  if (op == kOpPlain)
    solve_tc_kernel<kOpPlain><<<g, kSThreads, smem, st>>>(k, n, nrhs, P->n_pad, dtiles, dslots,
                                                          P->n_slots, factor, work, ytmp, status);
  else
    solve_tc_kernel<kOpConjT><<<g, kSThreads, smem, st>>>(k, n, nrhs, P->n_pad, dtiles, dslots,
                                                          P->n_slots, factor, work, ytmp, status);
  count_launches(1);
  return 0;
}

}  // namespace aosb
