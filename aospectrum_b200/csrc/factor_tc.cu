// Tensor-core (tcgen05) factorization path: split-BF16 Schur updates.
//
// Same right-looking tile LU as factor.cu (diagonal LU and panels stay FP32
// SIMT); the Schur update A_ij -= L_ik U_kj of every step runs on the 5th
// generation tensor cores:
//
//   * stage_kernel converts the step's L tiles (i,k) and U tiles (k,j) into
//     four BF16 planes each -- re_hi, re_lo, im_hi, im_lo with
//     x = hi + lo, hi = bf16(x), lo = bf16(x - hi) -- laid out as UMMA
//     K-major, no-swizzle core matrices (8 rows x 16 bytes), cut into 16-wide
//     K slabs so that one slab of one tile is a single contiguous bulk copy.
//     For U the operand rows are U's columns (B is K-major).
//   * schur_tc_kernel: one CTA (4 warps) per (target tile, pencil).  Lane 0
//     of warp 0 streams slabs with cp.async.bulk into a 3-stage mbarrier
//     ring; lane 0 of warp 1 issues, per 16-wide K step, 12
//     tcgen05.mma.kind::f16 (M=128, N=128) into two FP32 TMEM accumulators:
//       Re += Lr_h Ur_h + Lr_h Ur_l + Lr_l Ur_h - (Li_h Ui_h + Li_h Ui_l + Li_l Ui_h)
//       Im += Lr_h Ui_h + Lr_h Ui_l + Lr_l Ui_h + Li_h Ur_h + Li_h Ur_l + Li_l Ur_h
//     (the minus via the instruction's negate-A bit; lo*lo is dropped).
//     All four warps then read the accumulators with tcgen05.ld and apply
//     C -= acc to the FP32 tile in HBM.
//   Every mbarrier wait is bounded; on expiry the CTA records
//   AOSB_ERR_TIMEOUT in the pencil status, skips the remaining work, and
//   still frees its TMEM.
#include "plan.h"
#include "factor.h"
#include "cgemm.cuh"

#include <cuda_bf16.h>

namespace aosb {
namespace {

constexpr int kTcT = 128;                 // tile edge supported by this path
constexpr int kSlabK = 16;                // K per slab (one MMA K step)
constexpr int kSlabs = kTcT / kSlabK;     // 8
constexpr int kPlaneSlabBytes = kTcT * kSlabK * 2;          // 4096
constexpr int kOperandSlabBytes = 4 * kPlaneSlabBytes;      // 16384
constexpr int kStagedTileBytes = kSlabs * kOperandSlabBytes;  // 131072
constexpr long long kWaitLimit = 1ll << 22;  // polls (with backoff) before timeout

__device__ __forceinline__ size_t tile_base(int64_t p, int64_t n_slots, int64_t slot) {
  return ((size_t)p * (size_t)n_slots + (size_t)slot) * (size_t)(2 * kTcT * kTcT);
}

// Byte offset of operand element (row, k) of plane `plane` in a staged tile.
__host__ __device__ __forceinline__ uint32_t staged_offset(int row, int k, int plane) {
  const int slab = k / kSlabK, kk = k % kSlabK;
  return (uint32_t)(slab * kOperandSlabBytes + plane * kPlaneSlabBytes +
                    (kk / 8) * ((kTcT / 8) * 128) + (row / 8) * 128 + (row % 8) * 16 +
                    (kk % 8) * 2);
}

// ---------------------------------------------------------------------------
// Staging: blockIdx.x = item (L tiles first, then U tiles), blockIdx.y = pencil.
__global__ void __launch_bounds__(256) stage_kernel(int nL, int nU, const int32_t* __restrict__ lslot,
                                                    const int32_t* __restrict__ uslot,
                                                    int64_t n_slots, const float* __restrict__ factor,
                                                    unsigned char* __restrict__ staging,
                                                    int64_t staging_pencil_stride) {
  const int item = blockIdx.x, p = blockIdx.y;
  const bool is_l = item < nL;
  const int slot = is_l ? lslot[item] : uslot[item - nL];
  const float* F = factor + tile_base(p, n_slots, slot);
  unsigned char* out = staging + (size_t)p * staging_pencil_stride + (size_t)item * kStagedTileBytes;
  // Each thread converts pairs of consecutive k for one operand row, so a
  // 4-byte store writes two BF16 values.
  for (int e = threadIdx.x; e < kTcT * (kTcT / 2); e += blockDim.x) {
    int row, k;
    float r0, i0, r1, i1;
    if (is_l) {
      // A = L (row-major): operand row = tile row, k = tile column
      row = e / (kTcT / 2);
      k = (e % (kTcT / 2)) * 2;
      const size_t o = (size_t)row * kTcT + k;
      r0 = F[o]; r1 = F[o + 1];
      i0 = F[o + kTcT * kTcT]; i1 = F[o + 1 + kTcT * kTcT];
    } else {
      // B = U (row-major, k x n): operand row = column n, k = tile row
      k = (e / kTcT) * 2;
      row = e % kTcT;
      const size_t o0 = (size_t)k * kTcT + row, o1 = (size_t)(k + 1) * kTcT + row;
      r0 = F[o0]; r1 = F[o1];
      i0 = F[o0 + kTcT * kTcT]; i1 = F[o1 + kTcT * kTcT];
    }
    const float re[2] = {r0, r1}, im[2] = {i0, i1};
    __nv_bfloat162 plane[4];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const __nv_bfloat16 rh = __float2bfloat16_rn(re[t]);
      const __nv_bfloat16 rl = __float2bfloat16_rn(re[t] - __bfloat162float(rh));
      const __nv_bfloat16 ih = __float2bfloat16_rn(im[t]);
      const __nv_bfloat16 il = __float2bfloat16_rn(im[t] - __bfloat162float(ih));
      if (t == 0) {
        plane[0].x = rh; plane[1].x = rl; plane[2].x = ih; plane[3].x = il;
      } else {
        plane[0].y = rh; plane[1].y = rl; plane[2].y = ih; plane[3].y = il;
      }
    }
#pragma unroll
    for (int pl = 0; pl < 4; ++pl)
      *reinterpret_cast<__nv_bfloat162*>(out + staged_offset(row, k, pl)) = plane[pl];
  }
}

// ---------------------------------------------------------------------------
// PTX helpers.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait on phase `parity`; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(128);
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// UMMA shared-memory descriptor: K-major, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (Blackwell)
  return d;               // base offset 0, lbo mode 0, layout SWIZZLE_NONE (0)
}

// Instruction descriptor: BF16 x BF16 -> F32, K-major A and B, M = N = 128.
__host__ __device__ constexpr uint32_t umma_idesc(bool negate_a) {
  return (1u << 4)                    // D format F32
         | (1u << 7)                  // A format BF16
         | (1u << 10)                 // B format BF16
         | ((negate_a ? 1u : 0u) << 13)
         | ((uint32_t)(kTcT >> 3) << 17)   // N / 8
         | ((uint32_t)(kTcT >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Persistent, warp-specialized Schur update.  Each CTA (one per SM) walks
// the step's (pencil, target) items with stride gridDim.x:
//   warp 8 lane 0  producer: 16-wide K slabs of A (L_ik) and B (U_kj) into a
//                  kStages-deep ring (cp.async.bulk + mbarrier complete_tx);
//   warp 9 lane 0  MMA issuer: 12 tcgen05.mma per slab into accumulator set
//                  acc (TMEM columns acc*256 + [0,128) real, +[128,256) imag);
//   warps 0-7      epilogue: C rows 32*(w%4) + lane, columns 64*(w/4) ..+63;
//                  the C values are loaded before the accumulator is ready,
//                  then C -= acc is stored.
// Two accumulator sets let the epilogue of one item overlap the MMAs of the
// next.
constexpr int kStagesP = 4;
constexpr int kEpiWarps = 8;
constexpr int kXpLd = 36;  // padded row (floats) of the epilogue transposition tile
constexpr int kPThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kTmemColsP = 512;

struct PShared {
  alignas(1024) unsigned char a[kStagesP][kOperandSlabBytes];
  alignas(1024) unsigned char b[kStagesP][kOperandSlabBytes];
  uint64_t full[kStagesP];
  uint64_t empty[kStagesP];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tmem_base;
  int failed;
  // per epilogue warp: 32 x 32 re and im blocks for the transposition
  alignas(16) float xp[kEpiWarps][2][32 * kXpLd];
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(kPThreads, 1) schur_tc_kernel(
    int nU, int step_items, int n_pairs, int n_pencils, const int32_t* __restrict__ tslot,
    int64_t n_slots, float* __restrict__ factor, const unsigned char* __restrict__ staging,
    int64_t staging_pencil_stride, int32_t* __restrict__ status) {
  extern __shared__ unsigned char dyn[];
  PShared& sh = *reinterpret_cast<PShared*>(
      (reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int total = n_pairs * n_pencils;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesP; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sh.acc_full[b], 1);
      mbar_init(&sh.acc_empty[b], kEpiWarps);
    }
    sh.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem_base)),
                 "r"(kTmemColsP));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem_base;

  if (warp == kEpiWarps) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (int it = blockIdx.x; it < total && !sh.failed; it += gridDim.x) {
        const int p = it / n_pairs, pair = it % n_pairs;
        const unsigned char* stA = staging + (size_t)p * staging_pencil_stride +
                                   (size_t)(pair / nU) * kStagedTileBytes;
        const unsigned char* stB = staging + (size_t)p * staging_pencil_stride +
                                   (size_t)(step_items + pair % nU) * kStagedTileBytes;
        for (int s = 0; s < kSlabs; ++s) {
          if (!mbar_wait(&sh.empty[stage], phase ^ 1)) {
            sh.failed = 1;
            atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
            break;
          }
          mbar_expect_tx(&sh.full[stage], 2 * kOperandSlabBytes);
          bulk_g2s(sh.a[stage], stA + (size_t)s * kOperandSlabBytes, kOperandSlabBytes,
                   &sh.full[stage]);
          bulk_g2s(sh.b[stage], stB + (size_t)s * kOperandSlabBytes, kOperandSlabBytes,
                   &sh.full[stage]);
          if (++stage == kStagesP) { stage = 0; phase ^= 1; }
        }
      }
    }
  } else if (warp == kEpiWarps + 1) {
    if (lane == 0) {
      const uint32_t id_pos = umma_idesc(false), id_neg = umma_idesc(true);
      const uint32_t lbo = (kTcT / 8) * 128, sbo = 128;
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      for (int it = blockIdx.x; it < total && !sh.failed; it += gridDim.x) {
        const int p = it / n_pairs;
        if (!mbar_wait(&sh.acc_empty[acc], acc_phase ^ 1)) {
          sh.failed = 1;
          atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t re = tmem + (uint32_t)acc * 256, im = re + kTcT;
        bool ok = true;
        for (int s = 0; s < kSlabs; ++s) {
          if (!mbar_wait(&sh.full[stage], phase)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sa = smem_u32(sh.a[stage]), sb = smem_u32(sh.b[stage]);
          uint64_t A[4], Bv[4];
#pragma unroll
          for (int pl = 0; pl < 4; ++pl) {
            A[pl] = umma_desc(sa + pl * kPlaneSlabBytes, lbo, sbo);
            Bv[pl] = umma_desc(sb + pl * kPlaneSlabBytes, lbo, sbo);
          }
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
          umma_commit(&sh.empty[stage]);
          if (++stage == kStagesP) { stage = 0; phase ^= 1; }
        }
        if (!ok) {
          sh.failed = 1;
          atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
          break;
        }
        umma_commit(&sh.acc_full[acc]);
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
    }
  } else {
    // Epilogue warps.  Warp w owns rows 32*(w%4) .. +31 and columns
    // 64*(w/4) .. +63 of the target tile, processed as two 32 x 32 blocks.
    // C is read and written coalesced: lane l covers row 4*i + l/8 and
    // columns 4*(l%8) .. +3 of a block; the accumulator (one row per lane
    // after tcgen05.ld) is transposed through the warp's padded tile xp.
    const int quarter = warp % 4, half = warp / 4;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const int ro = lane / 8, cg = lane % 8;
    float* xre = sh.xp[warp][0];
    float* xim = sh.xp[warp][1];
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int it = blockIdx.x; it < total; it += gridDim.x) {
      const int p = it / n_pairs, pair = it % n_pairs;
      float* C = factor + tile_base(p, n_slots, tslot[pair]);
      // prefetch: 2 blocks x 8 row groups x (re, im)
      float4 cre[2][8], cim[2][8];
#pragma unroll
      for (int bk = 0; bk < 2; ++bk)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const size_t o = (size_t)(quarter * 32 + 4 * i + ro) * kTcT + half * 64 + bk * 32 + 4 * cg;
          cre[bk][i] = *reinterpret_cast<const float4*>(C + o);
          cim[bk][i] = *reinterpret_cast<const float4*>(C + kTcT * kTcT + o);
        }
      const bool ready = __all_sync(0xffffffffu, mbar_wait(&sh.acc_full[acc], acc_phase) ? 1 : 0);
      if (!ready) {
        if (lane == 0) {
          sh.failed = 1;
          atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
        }
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = tmem + (uint32_t)acc * 256 + (uint32_t)half * 64 + lane_addr;
#pragma unroll
      for (int bk = 0; bk < 2; ++bk) {
        float v[16];
        // real part: columns bk*32 .. +31 of this warp's half
        tmem_ld16(base + bk * 32, v);
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(xre + lane * kXpLd + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        tmem_ld16(base + bk * 32 + 16, v);
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(xre + lane * kXpLd + 16 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        tmem_ld16(base + kTcT + bk * 32, v);
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(xim + lane * kXpLd + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        tmem_ld16(base + kTcT + bk * 32 + 16, v);
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(xim + lane * kXpLd + 16 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float4 ar = *reinterpret_cast<const float4*>(xre + (4 * i + ro) * kXpLd + 4 * cg);
          const float4 ai = *reinterpret_cast<const float4*>(xim + (4 * i + ro) * kXpLd + 4 * cg);
          float4& x = cre[bk][i];
          float4& y = cim[bk][i];
          x.x -= ar.x; x.y -= ar.y; x.z -= ar.z; x.w -= ar.w;
          y.x -= ai.x; y.y -= ai.y; y.z -= ai.z; y.w -= ai.w;
        }
        __syncwarp();
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.acc_empty[acc]);
#pragma unroll
      for (int bk = 0; bk < 2; ++bk)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const size_t o = (size_t)(quarter * 32 + 4 * i + ro) * kTcT + half * 64 + bk * 32 + 4 * cg;
          *reinterpret_cast<float4*>(C + o) = cre[bk][i];
          *reinterpret_cast<float4*>(C + kTcT * kTcT + o) = cim[bk][i];
        }
      if (++acc == 2) { acc = 0; acc_phase ^= 1; }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemColsP));
  }
}

}  // namespace

size_t factor_tc_workspace(const aosb_plan* P, int32_t n_pencils) {
  if (P->T != kTcT) return 0;
  int64_t most = 0;
  for (int64_t k = 0; k < P->nb; ++k) {
    const int64_t items = (P->lb_off[k + 1] - P->lb_off[k]) + (P->ur_off[k + 1] - P->ur_off[k]);
    most = items > most ? items : most;
  }
  return (size_t)(most > 0 ? most : 1) * kStagedTileBytes * (size_t)n_pencils;
}

int factor_tc(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap) {
  if (P->T != kTcT)
    return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "tensor-core path needs tile = 128");
  if (a->workspace == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "tensor-core path needs a staging workspace");
  cudaStream_t st = (cudaStream_t)a->stream;
  const int np = a->n_pencils;
  const size_t smem = sizeof(PShared) + 1024;
  static_assert(sizeof(PShared) + 1024 <= 232448, "shared memory budget");
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(schur_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess)
      return set_error(err, cap, AOSB_ERR_CUDA, "schur_tc smem attribute: %s", cudaGetErrorString(e));
    attr_done = true;
  }
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int64_t most = 0;
  for (int64_t k = 0; k < P->nb; ++k) {
    const int64_t items = (P->lb_off[k + 1] - P->lb_off[k]) + (P->ur_off[k + 1] - P->ur_off[k]);
    most = items > most ? items : most;
  }
  const int64_t pencil_stride = (most > 0 ? most : 1) * (int64_t)kStagedTileBytes;
  unsigned char* staging = (unsigned char*)a->workspace;
  for (int64_t k = 0; k < P->nb; ++k) {
    int rc = factor_step_panels(P, a, (int)k, err, cap);
    if (rc) return rc;
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    if (nL == 0 || nU == 0) continue;
    stage_kernel<<<dim3(nL + nU, np), 256, 0, st>>>(nL, nU, P->d_lb_slot + P->lb_off[k],
                                                   P->d_ur_slot + P->ur_off[k], P->n_slots,
                                                   a->factor, staging, pencil_stride);
    const int64_t items = (int64_t)nL * nU * np;
    if ((int64_t)nL * nU > INT32_MAX / 65536)
      return set_error(err, cap, AOSB_ERR_SIZE, "too many Schur targets in one step");
    const int grid = (int)(items < sms ? items : sms);
    schur_tc_kernel<<<grid, kPThreads, smem, st>>>(nU, nL, nL * nU, np, P->d_sc_slot + P->sc_off[k],
                                                   P->n_slots, a->factor, staging, pencil_stride,
                                                   a->status);
    count_launches(2);
  }
  return launch_check(err, cap, "tensor-core factorization");
}

}  // namespace aosb
