// Tensor-core (tcgen05) update step of the block-RHS triangular sweeps for
// tile 128: X_i -= op(F) Y for every listed tile F of the step, with
// op(F) = F (plain) or F^H (adjoint sweeps) and Y the step's diagonal
// result (T x n_rhs complex64, written by the SIMT diagonal kernel together
// with its split-BF16 copy, the B operand: four BF16 planes re_hi, re_lo,
// im_hi, im_lo per 32-column RHS strip).
//
// Persistent and warp specialized; each CTA walks the step's (pencil,
// strip, tile) items with stride gridDim.x:
//   warp 0 lane 0   producer: per item one bulk copy of the Y strip planes
//                   (32 KB) into a two-buffer ring, and per 16-wide K slab two
//                   TMA tensor loads of the FP32 factor tile (real and
//                   imaginary plane boxes) into a kRawStages-deep ring;
//   warps 2-5       converters: split each FP32 slab into the four BF16
//                   planes of the K-major A operand (M = 128) in a
//                   kAStages-deep ring (op(F) = F^H reads the slab transposed
//                   and negates the imaginary part);
//   warp 1 lane 0   MMA issuer: 12 tcgen05.mma.kind::f16 (M = 128, N = strip
//                   width rounded up to 16) per slab into one of two TMEM
//                   accumulator pairs (re, im): hi*hi + hi*lo + lo*hi per real
//                   product, FP32 accumulation;
//   warps 6-9       epilogue: first the CTA's slice of the copy X_k = Y
//                   (the step's diagonal result), then per item tcgen05.ld
//                   of the accumulator (warp w reads lanes 32 (w % 4) ..);
//                   -acc goes through 128B-swizzled shared boxes into TMA
//                   reduce-adds on X_i (coalesced and asynchronous: X never
//                   passes through the registers).
// Two accumulator pairs let one item's epilogue overlap the next item's
// MMAs.  Every mbarrier wait is bounded: on expiry the CTA records
// AOSB_ERR_TIMEOUT in the pencil status and stops; a CTA that stops waits
// (bounded) for its own copies and MMAs in flight and frees its TMEM.
#include "plan.h"
#include "tc_common.cuh"

#include <cuda_bf16.h>

#include <atomic>

namespace aosb {
namespace {

using namespace tc;

constexpr int kT = 128;
constexpr int kNS = kSolveNS;              // RHS columns per item (32)
constexpr int kSK = 16;                    // K per slab
constexpr int kSlabsS = kT / kSK;          // 8
constexpr int kConvWarps = 4, kEpiWarps = 4;
constexpr int kConvWarp0 = 2, kEpiWarp0 = kConvWarp0 + kConvWarps;  // 2, 6
constexpr int kSThreads = (kEpiWarp0 + kEpiWarps) * 32;              // 320
constexpr int kACols = 4 * kNS;            // two accumulator pairs (re, im) = 128 columns
constexpr int kAPlane = kT * kSK * 2;      // 4096 bytes: one BF16 plane of one A slab
constexpr int kASlab = 4 * kAPlane;        // 16 KB
constexpr int kRawPlane = kT * kSK;        // floats in one FP32 plane box of a slab
constexpr uint32_t kRawBytes = 2 * kRawPlane * sizeof(float);  // 16 KB per slab

enum SolveOp { kOpPlain = 0, kOpConjT = 1 };

// Ring depths and CTAs per SM.  Form 1: one CTA per SM with deep rings
// (FP32 slabs 4, BF16 slabs 3, Y strips 2, two epilogue boxes per warp;
// 208 KB).  Form 2: two CTAs per SM with shallow rings (2, 1, 1, one box per
// warp; 96 KB), so that one CTA's waits overlap the other's work.
template <int CTAS>
struct SolveCfg;
template <>
struct SolveCfg<1> {
  static constexpr int kRawStages = 4, kAStages = 3, kBStages = 2, kEpBoxes = 2;
};
template <>
struct SolveCfg<2> {
  static constexpr int kRawStages = 2, kAStages = 1, kBStages = 1, kEpBoxes = 1;
};

template <int CTAS>
struct SShared {
  using C = SolveCfg<CTAS>;
  // per epilogue warp: its 32 rows x 32 complex of -acc as two 32 x 32 FP32
  // boxes (complex columns 0-15 and 16-31, re/im interleaved; with one box
  // the halves take turns), laid out as the TMA 128-byte swizzle expects
  alignas(1024) float ep[kEpiWarps][C::kEpBoxes][32 * 32];
  alignas(128) float raw[C::kRawStages][2][kRawPlane];
  alignas(128) unsigned char a[C::kAStages][kASlab];
  alignas(128) unsigned char b[C::kBStages][kSolveBBytes];
  uint64_t raw_full[C::kRawStages], raw_empty[C::kRawStages];
  uint64_t a_full[C::kAStages], a_empty[C::kAStages];
  uint64_t b_full[C::kBStages], b_empty[C::kBStages];
  uint64_t acc_full[2], acc_empty[2];
  uint64_t drain;  // the MMA issuer's last commit after a failure
  uint32_t tmem_base;
  int failed;
};

// K-major no-swizzle core-matrix layout (8 rows x 16 bytes), the two 8-wide
// K halves of a slab (kT / 8) * 128 bytes apart.
__device__ __forceinline__ uint32_t a_off(int m, int k, int plane) {
  return (uint32_t)(plane * kAPlane + (k / 8) * ((kT / 8) * 128) + (m / 8) * 128 + (m % 8) * 16 +
                    (k % 8) * 2);
}

__device__ __forceinline__ void split2(float x0, float x1, __nv_bfloat162& hi, __nv_bfloat162& lo) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
  hi.x = h0;
  hi.y = h1;
  lo.x = __float2bfloat16_rn(x0 - __bfloat162float(h0));
  lo.y = __float2bfloat16_rn(x1 - __bfloat162float(h1));
}

struct ItemOf {
  int p, strip, tile_idx;
};
__device__ __forceinline__ ItemOf item_of(int it, int n_items, int strips) {
  const int per_pencil = n_items * strips;
  ItemOf r;
  r.p = it / per_pencil;
  const int rem = it % per_pencil;
  r.strip = rem / n_items;
  r.tile_idx = rem % n_items;
  return r;
}

template <typename SH>
__device__ __forceinline__ void fail(SH& sh, int32_t* status, int p) {
  sh.failed = 1;
  atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
}

template <int OP, int CTAS>
__global__ void __launch_bounds__(kSThreads, CTAS) solve_tc_kernel(
    int k, int n_items, int nrhs, int n_pencils, int64_t n_pad, const int32_t* __restrict__ tiles,
    const int32_t* __restrict__ slots, int64_t n_slots, float2* __restrict__ work,
    const float2* __restrict__ ytmp, const unsigned char* __restrict__ ystaged,
    int32_t* __restrict__ status, const __grid_constant__ CUtensorMap fmap,
    const __grid_constant__ CUtensorMap xmap, int x_tma, int copy_y, long long wl) {
  const int strips = (nrhs + kNS - 1) / kNS;
  const int total = n_items * strips * n_pencils;
  const int work_ctas = (int)gridDim.x;
  using C = SolveCfg<CTAS>;
  constexpr int kRawStages = C::kRawStages, kAStages = C::kAStages, kBStages = C::kBStages;
  extern __shared__ unsigned char dyn[];
  SShared<CTAS>& sh = *reinterpret_cast<SShared<CTAS>*>(
      (reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kRawStages; ++s) {
      mbar_init(&sh.raw_full[s], 1);
      mbar_init(&sh.raw_empty[s], kConvWarps);
    }
    for (int s = 0; s < kAStages; ++s) {
      mbar_init(&sh.a_full[s], kConvWarps);
      mbar_init(&sh.a_empty[s], 1);
    }
    for (int b = 0; b < kBStages; ++b) {
      mbar_init(&sh.b_full[b], 1);
      mbar_init(&sh.b_empty[b], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sh.acc_full[b], 1);
      mbar_init(&sh.acc_empty[b], kEpiWarps);
    }
    mbar_init(&sh.drain, 1);
    sh.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem_base)),
                 "r"(kACols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem_base;
  // What the producer and the MMA issuer have in flight, for the drain
  // after a failure: the FP32-slab and Y-strip ring stages the producer
  // filled (bit s) with the phase parity of the last fill of each, and
  // whether any MMA was issued.
  uint32_t raw_filled = 0, raw_parity = 0, b_filled = 0, b_parity = 0;
  bool issued = false;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int g = 0;  // slab counter over all items of this CTA
      int j = 0;  // item counter
      for (int it = blockIdx.x; it < total && !sh.failed; it += work_ctas, ++j) {
        const ItemOf w = item_of(it, n_items, strips);
        const int bb = j % kBStages;
        if (!mbar_wait(&sh.b_empty[bb], (uint32_t)(((j / kBStages) & 1) ^ 1), wl)) {
          fail(sh, status, w.p);
          break;
        }
        b_filled |= 1u << bb;
        b_parity = (b_parity & ~(1u << bb)) | ((uint32_t)((j / kBStages) & 1) << bb);
        mbar_expect_tx(&sh.b_full[bb], kSolveBBytes);
        bulk_g2s(sh.b[bb], ystaged + ((size_t)w.p * strips + w.strip) * kSolveBBytes,
                 kSolveBBytes, &sh.b_full[bb]);
        const int64_t row0 = ((int64_t)w.p * n_slots + slots[w.tile_idx]) * (2 * kT);
        bool ok = true;
        for (int s = 0; s < kSlabsS; ++s, ++g) {
          const int st = g % kRawStages;
          if (!mbar_wait(&sh.raw_empty[st], (uint32_t)(((g / kRawStages) & 1) ^ 1), wl)) {
            ok = false;
            break;
          }
          raw_filled |= 1u << st;
          raw_parity = (raw_parity & ~(1u << st)) | ((uint32_t)((g / kRawStages) & 1) << st);
          mbar_expect_tx(&sh.raw_full[st], kRawBytes);
          if (OP == kOpPlain) {
            tma_load_2d(sh.raw[st][0], &fmap, s * kSK, (int)row0, &sh.raw_full[st]);
            tma_load_2d(sh.raw[st][1], &fmap, s * kSK, (int)(row0 + kT), &sh.raw_full[st]);
          } else {
            tma_load_2d(sh.raw[st][0], &fmap, 0, (int)(row0 + s * kSK), &sh.raw_full[st]);
            tma_load_2d(sh.raw[st][1], &fmap, 0, (int)(row0 + kT + s * kSK), &sh.raw_full[st]);
          }
        }
        if (!ok) { fail(sh, status, w.p); break; }
      }
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t alb = (kT / 8) * 128, blb = (kNS / 8) * 128;
      int g = 0, j = 0;
      for (int it = blockIdx.x; it < total && !sh.failed; it += work_ctas, ++j) {
        const ItemOf w = item_of(it, n_items, strips);
        const int ncols = nrhs - w.strip * kNS < kNS ? nrhs - w.strip * kNS : kNS;
        const int n16 = (ncols + 15) & ~15;
        const uint32_t id_pos = umma_idesc_mn(kT, n16, false), id_neg = umma_idesc_mn(kT, n16, true);
        const int acc = j & 1, bb = j % kBStages;
        if (!mbar_wait(&sh.acc_empty[acc], (uint32_t)(((j >> 1) & 1) ^ 1), wl) ||
            !mbar_wait(&sh.b_full[bb], (uint32_t)((j / kBStages) & 1), wl)) {
          fail(sh, status, w.p);
          break;
        }
        const uint32_t re = tmem + (uint32_t)acc * (2 * kNS), im = re + kNS;
        bool ok = true;
        for (int s = 0; s < kSlabsS; ++s, ++g) {
          const int ab = g % kAStages;
          if (!mbar_wait(&sh.a_full[ab], (uint32_t)((g / kAStages) & 1), wl)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          issued = true;
          const uint32_t sa = smem_u32(sh.a[ab]), sb = smem_u32(sh.b[bb]) + s * kSolveBSlab;
          uint64_t A[4], Bv[4];
#pragma unroll
          for (int pl = 0; pl < 4; ++pl) {
            A[pl] = umma_desc(sa + pl * kAPlane, alb, 128);
            Bv[pl] = umma_desc(sb + pl * kSolveBPlaneSlab, blb, 128);
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
          umma_commit(&sh.a_empty[ab]);
        }
        if (!ok) { fail(sh, status, w.p); break; }
        umma_commit(&sh.acc_full[acc]);
        umma_commit(&sh.b_empty[bb]);
      }
    }
  } else if (warp < kEpiWarp0) {
    // ---------------------------------------------------------- converters
    const int ct = threadIdx.x - kConvWarp0 * 32;  // 0 .. 127
    int g = 0;
    for (int it = blockIdx.x; it < total; it += work_ctas) {
      bool ok = true;
      for (int s = 0; s < kSlabsS; ++s, ++g) {
        const int st = g % kRawStages, ab = g % kAStages;
        const bool ready = mbar_wait(&sh.raw_full[st], (uint32_t)((g / kRawStages) & 1), wl) &&
                           mbar_wait(&sh.a_empty[ab], (uint32_t)(((g / kAStages) & 1) ^ 1), wl);
        if (!__all_sync(0xffffffffu, ready ? 1 : 0) || sh.failed) {
          ok = false;
          break;
        }
        unsigned char* a = sh.a[ab];
        const float* rre = sh.raw[st][0];
        const float* rim = sh.raw[st][1];
#pragma unroll 4
        for (int e = ct; e < kT * (kSK / 2); e += kConvWarps * 32) {
          int m, q;
          float r0, r1, i0, i1;
          if (OP == kOpPlain) {  // raw box [128 rows][16 cols]
            m = e / (kSK / 2);
            q = (e % (kSK / 2)) * 2;
            const float2 rr = *reinterpret_cast<const float2*>(rre + m * kSK + q);
            const float2 ii = *reinterpret_cast<const float2*>(rim + m * kSK + q);
            r0 = rr.x; r1 = rr.y; i0 = ii.x; i1 = ii.y;
          } else {  // raw box [16 rows][128 cols]
            m = e % kT;
            q = (e / kT) * 2;
            r0 = rre[q * kT + m]; r1 = rre[(q + 1) * kT + m];
            i0 = -rim[q * kT + m]; i1 = -rim[(q + 1) * kT + m];
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
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&sh.raw_empty[st]);
          mbar_arrive(&sh.a_full[ab]);
        }
      }
      if (!ok) {
        if (lane == 0) fail(sh, status, item_of(it, n_items, strips).p);
        break;
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // X rows of an item are contiguous (n_rhs complex each).  With x_tma the
    // warp writes -acc for its 32 rows into its swizzled boxes and lane 0
    // hands them to TMA reduce-adds into X in L2 (coalesced, asynchronous);
    // otherwise every lane read-modify-writes its row.
    const int quarter = warp % 4;
    const int ew = warp - kEpiWarp0;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const int row = quarter * 32 + lane;
    const int sw = lane & 7;
    if (copy_y) {
      // While the first accumulator fills, the epilogue warps of every CTA
      // copy one slice of the step's diagonal result into X_k (X_k = Y for
      // every pencil; no item of this step touches rows of tile k): the
      // copy rides along with the launch instead of adding CTAs that would
      // wait for the persistent ones to leave.
      const int et = threadIdx.x - kEpiWarp0 * 32;  // 0 .. 127
      const int64_t per = (int64_t)kT * nrhs;      // float2 per pencil
      if ((nrhs & 1) == 0) {
        const int64_t per4 = per / 2, n4 = per4 * n_pencils;
        const int64_t e0 = n4 * blockIdx.x / work_ctas, e1 = n4 * (blockIdx.x + 1) / work_ctas;
        for (int64_t e = e0 + et; e < e1; e += kEpiWarps * 32) {
          const int64_t p = e / per4, r = e - p * per4;
          reinterpret_cast<float4*>(work + ((size_t)p * n_pad + (size_t)k * kT) * nrhs)[r] =
              reinterpret_cast<const float4*>(ytmp + (size_t)p * per)[r];
        }
      } else {
        const int64_t n2 = per * n_pencils;
        const int64_t e0 = n2 * blockIdx.x / work_ctas, e1 = n2 * (blockIdx.x + 1) / work_ctas;
        for (int64_t e = e0 + et; e < e1; e += kEpiWarps * 32) {
          const int64_t p = e / per, r = e - p * per;
          work[((size_t)p * n_pad + (size_t)k * kT) * nrhs + r] = ytmp[(size_t)p * per + r];
        }
      }
    }
    int j = 0;
    for (int it = blockIdx.x; it < total; it += work_ctas, ++j) {
      const ItemOf w = item_of(it, n_items, strips);
      const int acc = j & 1;
      const bool ready = mbar_wait(&sh.acc_full[acc], (uint32_t)((j >> 1) & 1), wl);
      if (!__all_sync(0xffffffffu, ready ? 1 : 0)) {
        if (lane == 0) fail(sh, status, w.p);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int c0 = w.strip * kNS;
      const int ncols = nrhs - c0 < kNS ? nrhs - c0 : kNS;
      const uint32_t base = tmem + (uint32_t)acc * (2 * kNS) + lane_addr;
      float vr[2][16], vi[2][16];
      tmem_ld16(base, vr[0]);
      tmem_ld16(base + 16, vr[1]);
      tmem_ld16(base + kNS, vi[0]);
      tmem_ld16(base + kNS + 16, vi[1]);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.acc_empty[acc]);
      const int64_t xrow = (int64_t)w.p * n_pad + (int64_t)tiles[w.tile_idx] * kT;
      if (x_tma && C::kEpBoxes == 2) {
        if (lane == 0) bulk_wait_read_all();   // the boxes' previous reduce has read them
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float* box = sh.ep[ew][h % C::kEpBoxes];
          // 16 complex = 32 floats = 8 chunks of 16 bytes: (re, im, re, im)
#pragma unroll
          for (int c = 0; c < 8; ++c)
            *reinterpret_cast<float4*>(box + lane * 32 + ((c ^ sw) * 4)) =
                make_float4(-vr[h][2 * c], -vi[h][2 * c], -vr[h][2 * c + 1], -vi[h][2 * c + 1]);
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          const int y = (int)(xrow + quarter * 32);
          tma_reduce_add_2d(&xmap, sh.ep[ew][0], 2 * c0, y);
          if (ncols > 16) tma_reduce_add_2d(&xmap, sh.ep[ew][1 % C::kEpBoxes], 2 * c0 + 32, y);
          bulk_commit();
        }
      } else if (x_tma) {
        // one box per warp: each half waits until the box's previous reduce
        // has read it
        float* box = sh.ep[ew][0];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (h == 1 && ncols <= 16) break;
          if (lane == 0) bulk_wait_read_all();
          __syncwarp();
#pragma unroll
          for (int c = 0; c < 8; ++c)
            *reinterpret_cast<float4*>(box + lane * 32 + ((c ^ sw) * 4)) =
                make_float4(-vr[h][2 * c], -vi[h][2 * c], -vr[h][2 * c + 1], -vi[h][2 * c + 1]);
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_reduce_add_2d(&xmap, box, 2 * c0 + 32 * h, (int)(xrow + quarter * 32));
            bulk_commit();
          }
        }
      } else {
        float2* xr = work + (size_t)(xrow + row) * nrhs + c0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float2 xv[16];
#pragma unroll
          for (int c = 0; c < 16; ++c)
            xv[c] = h * 16 + c < ncols ? xr[h * 16 + c] : make_float2(0.f, 0.f);
#pragma unroll
          for (int c = 0; c < 16; ++c)
            if (h * 16 + c < ncols)
              xr[h * 16 + c] = make_float2(xv[c].x - vr[h][c], xv[c].y - vi[h][c]);
        }
      }
    }
    // the X updates must be complete (not only read) before exit
    if (x_tma && lane == 0) bulk_wait_all();
    __syncwarp();
  }
  // Every role has left its loop (all waits are bounded).  After a failure
  // the producer waits (bounded) until each stage it filled has received
  // its bytes, and the MMA issuer commits once more and waits until its
  // MMAs are done, so no copy or MMA lands in shared memory or TMEM after
  // they are released.
  __syncthreads();
  if (sh.failed) {
    if (warp == 0 && lane == 0) {
      for (int s = 0; s < kRawStages; ++s)
        if (raw_filled & (1u << s)) mbar_wait(&sh.raw_full[s], (raw_parity >> s) & 1u);
      for (int b = 0; b < kBStages; ++b)
        if (b_filled & (1u << b)) mbar_wait(&sh.b_full[b], (b_parity >> b) & 1u);
    }
    if (warp == 1 && lane == 0 && issued) {
      umma_commit(&sh.drain);
      mbar_wait(&sh.drain, 0);
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

template <int CTAS>
size_t solve_tc_smem() { return sizeof(SShared<CTAS>) + 1024; }
static_assert(sizeof(SShared<1>) + 1024 <= 232448, "shared memory budget");
// two CTAs and their 1 KB system reservations in the SM's 228 KB
static_assert(2 * (sizeof(SShared<2>) + 1024 + 1024) <= 233472, "two CTAs per SM");

// CTAs per SM of the tensor-core solve update (1 or 2; 2 measured ~5 %
// faster per launch on c2); process-wide.
std::atomic<int> g_solve_ctas{2};

template <int OP, int CTAS>
int solve_tc_launch(int k, int n, const int32_t* dtiles, const int32_t* dslots, int np, int nrhs,
                    const aosb_plan* P, float2* work, const float2* ytmp,
                    const unsigned char* ystaged, int32_t* status, const CUtensorMap& fmap,
                    const CUtensorMap& xmap, int x_tma, int copy_y, int sms, cudaStream_t st,
                    char* err, size_t cap) {
  const size_t smem = solve_tc_smem<CTAS>();
  // kernel attributes belong to each device's context: set once per device
  static std::atomic<uint64_t> attr_devices{0};
  int device = 0;
  cudaGetDevice(&device);
  const uint64_t dev_bit = device < 64 ? (uint64_t)1 << device : 0;
  if (dev_bit == 0 || (attr_devices.load() & dev_bit) == 0) {
    cudaError_t e = cudaFuncSetAttribute(solve_tc_kernel<OP, CTAS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && CTAS > 1)
      e = cudaFuncSetAttribute(solve_tc_kernel<OP, CTAS>,
                               cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess)
      return set_error(err, cap, AOSB_ERR_CUDA, "solve_tc attributes: %s", cudaGetErrorString(e));
    attr_devices.fetch_or(dev_bit);
  }
  const int strips = (nrhs + kNS - 1) / kNS;
  const int64_t items = (int64_t)n * strips * np;
  const int64_t slots = (int64_t)CTAS * sms;
  // at least one CTA when the launch copies Y into X_k: a step without
  // tiles still does that copy
  const int work_ctas =
      (int)(items < slots ? (items > 0 ? items : (copy_y ? 1 : 0)) : slots);
  if (work_ctas == 0) return 0;
  dim3 g((unsigned)work_ctas);
  solve_tc_kernel<OP, CTAS><<<g, kSThreads, smem, st>>>(k, n, nrhs, np, P->n_pad, dtiles, dslots,
                                                        P->n_slots, work, ytmp, ystaged, status,
                                                        fmap, xmap, x_tma, copy_y,
                                                        tc_wait_limit());
  count_launches(1);
  return 0;
}

// Launch the tensor-core update of step k for n tiles (device lists).
int solve_tc_update(int k, int n, const int32_t* dtiles, const int32_t* dslots, int op,
                    int np, int nrhs, const aosb_plan* P, const float* factor, float2* work,
                    const float2* ytmp, const unsigned char* ystaged, int32_t* status,
                    cudaStream_t st, char* err, size_t cap, int copy_y) {
  if (n == 0 && !copy_y) return 0;
  // the factor as [rows][128] FP32; plain slabs are {16, 128} boxes,
  // adjoint slabs {128, 16}
  CUtensorMap fmap;
  const uint64_t rows = (uint64_t)np * P->n_slots * 2 * kT;
  if (int rc = op == kOpPlain
                   ? encode_f32_2d((void*)factor, kT, rows, kSK, kT, false, &fmap, err, cap)
                   : encode_f32_2d((void*)factor, kT, rows, kT, kSK, false, &fmap, err, cap))
    return rc;
  // X as [n_pencils * n_pad rows][2 n_rhs] FP32, 32 x 32 boxes, 128-byte
  // swizzle: the destination of the epilogue's reduce-adds (rows of 2 n_rhs
  // floats must be a multiple of 16 bytes: n_rhs even)
  CUtensorMap xmap;
  const int x_tma = (nrhs % 2 == 0) ? 1 : 0;
  if (x_tma) {
    if (int rc = encode_f32_2d((void*)work, (uint64_t)2 * nrhs, (uint64_t)np * P->n_pad, 32, 32,
                               true, &xmap, err, cap))
      return rc;
  } else {
    xmap = fmap;  // unused
  }
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const bool two = g_solve_ctas.load() == 2;
  if (op == kOpPlain)
    return two ? solve_tc_launch<kOpPlain, 2>(k, n, dtiles, dslots, np, nrhs, P, work, ytmp,
                                              ystaged, status, fmap, xmap, x_tma, copy_y, sms, st, err, cap)
               : solve_tc_launch<kOpPlain, 1>(k, n, dtiles, dslots, np, nrhs, P, work, ytmp,
                                              ystaged, status, fmap, xmap, x_tma, copy_y, sms, st, err, cap);
  return two ? solve_tc_launch<kOpConjT, 2>(k, n, dtiles, dslots, np, nrhs, P, work, ytmp, ystaged,
                                            status, fmap, xmap, x_tma, copy_y, sms, st, err, cap)
             : solve_tc_launch<kOpConjT, 1>(k, n, dtiles, dslots, np, nrhs, P, work, ytmp, ystaged,
                                            status, fmap, xmap, x_tma, copy_y, sms, st, err, cap);
}

}  // namespace aosb

extern "C" int32_t aosb_solve_set_ctas_per_sm(int32_t ctas) {
  if (ctas < 0 || ctas > 2) return -1;
  return aosb::g_solve_ctas.exchange(ctas == 0 ? 2 : ctas);
}
