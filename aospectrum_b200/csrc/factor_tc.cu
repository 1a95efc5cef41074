// Tensor-core (tcgen05) factorization path: split-BF16 panel products and
// Schur updates.
//
// Same right-looking tile LU as factor.cu.  The diagonal tile LU (with
// pivoting and the two triangle inverses) stays FP32 SIMT; the panel
// products L_ik = A_ik inv(U_kk), U_kj = inv(L_kk) P_k A_kj and the Schur
// update A_ij -= L_ik U_kj of every step run on the 5th generation tensor
// cores:
//
//   * stage_kernel converts the step's L tiles (i,k) and U tiles (k,j) into
//     four BF16 planes each -- re_hi, re_lo, im_hi, im_lo with
//     x = hi + lo, hi = bf16(x), lo = bf16(x - hi) -- laid out as UMMA
//     K-major, no-swizzle core matrices (8 rows x 16 bytes), cut into 16-wide
//     K slabs so that one slab of one tile is a single contiguous bulk copy.
//     For U the operand rows are U's columns (B is K-major).
//   * schur_tc_kernel: persistent and warp specialized (see the kernel).  Per
//     16-wide K slab the MMA warp issues 12 tcgen05.mma.kind::f16 (M=N=128)
//     into two FP32 TMEM accumulators:
//       Re += Lr_h Ur_h + Lr_h Ur_l + Lr_l Ur_h - (Li_h Ui_h + Li_h Ui_l + Li_l Ui_h)
//       Im += Lr_h Ui_h + Lr_h Ui_l + Lr_l Ui_h + Li_h Ur_h + Li_h Ur_l + Li_l Ur_h
//     (the minus via the instruction's negate-A bit; lo*lo is dropped).
//     The epilogue writes -acc into 128B-swizzled shared tiles and the TMA
//     unit adds them into the FP32 target tile in L2
//     (cp.reduce.async.bulk.tensor .add.f32), so C never passes through
//     the SM's registers.
//   Every mbarrier wait is bounded; on expiry the CTA records
//   AOSB_ERR_TIMEOUT in the pencil status, skips the remaining work, and
//   still frees its TMEM.
#include "plan.h"
#include "factor.h"
#include "cgemm.cuh"
#include "tc_common.cuh"
#include "timing.h"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

namespace aosb {

namespace {

using namespace tc;

constexpr int kTcT = 128;                 // tile edge supported by this path
constexpr int kSlabK = 16;                // K per slab (one MMA K step)
constexpr int kSlabs = kTcT / kSlabK;     // 8
constexpr int kPlaneSlabBytes = kTcT * kSlabK * 2;          // 4096
constexpr int kOperandSlabBytes = 4 * kPlaneSlabBytes;      // 16384
constexpr int kStagedTileBytes = kSlabs * kOperandSlabBytes;  // 131072

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
// Staging.  Operand kinds:
//   A          tile as the A operand (row-major: operand row = tile row,
//              k = tile column)
//   B          tile as the B operand (operand row = tile column n, k = tile
//              row)
//   B_PERM     B with the tile's rows taken through the pivot order of the
//              step: k -> row pv[k] (for U_kj = inv(L_kk) P_k A_kj)
//   A_UNIT_LO  the strictly lower triangle of the diagonal slot with a unit
//              diagonal and zeros above (inv(L_kk))
//   B_UPPER    the upper triangle (with diagonal) of the diagonal slot and
//              zeros below (inv(U_kk))
enum StageKind : int { kStageA = 0, kStageB = 1, kStageBPerm = 2, kStageAUnitLower = 3, kStageBUpper = 4 };

__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void stage_tile(const float* __restrict__ F, unsigned char* __restrict__ out,
                                           int kind, const int32_t* __restrict__ pv) {
  const bool a_side = kind == kStageA || kind == kStageAUnitLower;
  // Each thread converts 8 consecutive k of one operand row into one 16-byte
  // chunk of every plane.  Consecutive threads take consecutive operand rows,
  // whose chunks are adjacent in the staged layout, so a warp stores 512
  // contiguous bytes per plane; A-side reads are whole 32-byte row segments,
  // B-side reads are 128-byte row runs of the tile.
  for (int e = threadIdx.x; e < kTcT * (kTcT / 8); e += blockDim.x) {
    const int row = e % kTcT;
    const int k0 = (e / kTcT) * 8;
    float re[8], im[8];
    if (a_side) {
      const float4* sr = reinterpret_cast<const float4*>(F + (size_t)row * kTcT + k0);
      const float4* si = reinterpret_cast<const float4*>(F + kTcT * kTcT + (size_t)row * kTcT + k0);
      const float4 r0 = sr[0], r1 = sr[1], i0 = si[0], i1 = si[1];
      re[0] = r0.x; re[1] = r0.y; re[2] = r0.z; re[3] = r0.w;
      re[4] = r1.x; re[5] = r1.y; re[6] = r1.z; re[7] = r1.w;
      im[0] = i0.x; im[1] = i0.y; im[2] = i0.z; im[3] = i0.w;
      im[4] = i1.x; im[5] = i1.y; im[6] = i1.z; im[7] = i1.w;
      if (kind == kStageAUnitLower) {
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const int q = k0 + t;
          if (q >= row) {
            re[t] = q == row ? 1.0f : 0.0f;
            im[t] = 0.0f;
          }
        }
      }
    } else {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int q = kind == kStageBPerm ? pv[k0 + t] : k0 + t;
        const size_t o = (size_t)q * kTcT + row;
        re[t] = F[o];
        im[t] = F[o + kTcT * kTcT];
      }
      if (kind == kStageBUpper) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (k0 + t > row) re[t] = im[t] = 0.0f;
      }
    }
    uint32_t plane[4][4];
#pragma unroll
    for (int t = 0; t < 8; t += 2) {
      __nv_bfloat16 h[4][2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const __nv_bfloat16 rh = __float2bfloat16_rn(re[t + u]);
        const __nv_bfloat16 ih = __float2bfloat16_rn(im[t + u]);
        h[0][u] = rh;
        h[1][u] = __float2bfloat16_rn(re[t + u] - __bfloat162float(rh));
        h[2][u] = ih;
        h[3][u] = __float2bfloat16_rn(im[t + u] - __bfloat162float(ih));
      }
#pragma unroll
      for (int pl = 0; pl < 4; ++pl) plane[pl][t / 2] = pack_bf16x2(h[pl][0], h[pl][1]);
    }
#pragma unroll
    for (int pl = 0; pl < 4; ++pl)
      *reinterpret_cast<uint4*>(out + staged_offset(row, k0, pl)) =
          make_uint4(plane[pl][0], plane[pl][1], plane[pl][2], plane[pl][3]);
  }
}

// blockIdx.x = item, blockIdx.y = pencil.
//   Schur staging (panel == 0): items [0, nL) = L_ik as A, [nL, nL+nU) =
//     U_kj as B.
//   Panel staging (panel == 1): items [0, nL) = A_ik as A, [nL, nL+nU) =
//     P_k A_kj as B, nL+nU = inv(L_kk) as A, nL+nU+1 = inv(U_kk) as B.
__global__ void __launch_bounds__(256) stage_kernel(int nL, int nU, int panel, int k,
                                                    const int32_t* __restrict__ lslot,
                                                    const int32_t* __restrict__ uslot, int diag_slot,
                                                    int64_t n_slots, int64_t n_pad,
                                                    const float* __restrict__ factor,
                                                    const int32_t* __restrict__ pivots,
                                                    unsigned char* __restrict__ staging,
                                                    int64_t staging_pencil_stride) {
  const int item = blockIdx.x, p = blockIdx.y;
  int slot, kind;
  if (item < nL) {
    slot = lslot[item];
    kind = kStageA;
  } else if (item < nL + nU) {
    slot = uslot[item - nL];
    kind = panel ? kStageBPerm : kStageB;
  } else {
    slot = diag_slot;
    kind = item == nL + nU ? kStageAUnitLower : kStageBUpper;
  }
  const float* F = factor + tile_base(p, n_slots, slot);
  const int32_t* pv = pivots + (size_t)p * n_pad + (size_t)k * kTcT;
  unsigned char* out = staging + (size_t)p * staging_pencil_stride + (size_t)item * kStagedTileBytes;
  stage_tile(F, out, kind, pv);
}

// Persistent, warp-specialized Schur update.  Each CTA (one per SM) walks
// the step's (pencil, target) items with stride gridDim.x:
//   warp 8 lane 0  producer: 16-wide K slabs of A (L_ik) and B (U_kj) into a
//                  kStages-deep ring (cp.async.bulk + mbarrier complete_tx);
//   warp 9 lane 0  MMA issuer: 12 tcgen05.mma per slab into accumulator set
//                  acc (TMEM columns acc*256 + [0,128) real, +[128,256) imag);
//   warps 0-7      epilogue: rows 32*(w%4) .. +31 (TMEM lanes), columns
//                  64*(w/4) .. +63 as two 32 x 32 blocks; each block's -acc
//                  goes through the warp's swizzled shared tile into a TMA
//                  reduce-add on the target tile.
// Two accumulator sets let the epilogue of one item overlap the MMAs of the
// next.
// Depth of the operand slab ring (build-time: -DAOSB_SCHUR_STAGES=n; 5 is
// the most that fits beside the epilogue tiles in 227 KB).
#ifndef AOSB_SCHUR_STAGES
#define AOSB_SCHUR_STAGES 4
#endif
constexpr int kStagesP = AOSB_SCHUR_STAGES;
constexpr int kEpiWarps = 8;
constexpr int kPThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kTmemColsP = 512;
constexpr int kItemRing = 8;  // > items the producer can run ahead of the epilogue (~4)

struct PShared {
  alignas(1024) unsigned char a[kStagesP][kOperandSlabBytes];
  alignas(1024) unsigned char b[kStagesP][kOperandSlabBytes];
  uint64_t full[kStagesP];
  uint64_t empty[kStagesP];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint64_t drain;  // the MMA issuer's last commit after a failure
  uint32_t tmem_base;
  int failed;
  // claimed item of the producer's j-th item (j % kItemRing), -1 = no more
  int items[8];
  // per epilogue warp: one 32 x 32 block of -acc (re, im planes), laid out
  // as the TMA 128-byte swizzle expects (row r at r * 128 bytes, 16-byte
  // chunk c of the row at chunk position c ^ (r % 8))
  alignas(1024) float ep[kEpiWarps][2][32 * 32];
};

// Work item -> (staged A index, staged B index, target slot).
//   kMapSchur: pair = a * nU + b over the step's L x U tiles; the target
//     gets C -= A B (TMA reduce-add of -acc).
//   kMapPanel: pair < nL: L_ik = A_ik inv(U_kk); else U_kj = inv(L_kk) P_k
//     A_kj; the target is overwritten with A B (TMA store of acc).
//   kMapCross / kMapRest: the Schur pairs split for lookahead.  With a0
//     (b0) = 1 when the step's first L (U) tile is in tile row (column)
//     k + 1, "cross" holds the pairs with a < a0 or b < b0 -- every target
//     in tile row or column k + 1, which step k + 1's diagonal LU and panels
//     read -- and "rest" the pairs with a >= a0 and b >= b0.
//   kMapList: two-step (K = 256) Schur items from the plan's super-step
//     lists: item = (target slot, A and B staged index of the first step or
//     -1, of the second step or -1); the first step's tiles come from
//     `staging`, the second's from `staging1`.
enum MapKind : int { kMapSchur = 0, kMapPanel = 1, kMapCross = 2, kMapRest = 3, kMapList = 4 };

struct ItemMap {
  int kind, nL, nU, n_pairs, a0, b0;
  const int32_t* tslot;  // Schur targets [nL * nU]
  const int32_t* lslot;  // panel L targets [nL]
  const int32_t* uslot;  // panel U targets [nU]
  const int32_t* list;   // kMapList items [n_pairs][5]
};

// K halves of an item: staged (A, B) indices and which staging buffer
// (0 = `staging`, 1 = `staging1`); returns how many (1 or 2).
__device__ __forceinline__ int item_halves(const ItemMap& m, int pair, int (&ia)[2], int (&ib)[2],
                                           int (&buf)[2]);

__device__ __forceinline__ void item_pair(const ItemMap& m, int pair, int& a, int& b) {
  if (m.kind == kMapSchur) {
    a = pair / m.nU;
    b = pair % m.nU;
  } else if (m.kind == kMapRest) {
    const int w = m.nU - m.b0;
    a = m.a0 + pair / w;
    b = m.b0 + pair % w;
  } else {  // kMapCross
    const int head = m.a0 * m.nU;
    if (pair < head) {
      a = pair / m.nU;
      b = pair % m.nU;
    } else {
      const int i = pair - head;
      a = m.a0 + i / m.b0;
      b = i % m.b0;
    }
  }
}

__device__ __forceinline__ void item_operands(const ItemMap& m, int pair, int& ia, int& ib) {
  if (m.kind == kMapPanel) {
    if (pair < m.nL) {
      ia = pair;
      ib = m.nL + m.nU + 1;
    } else {
      ia = m.nL + m.nU;
      ib = pair;
    }
    return;
  }
  int a, b;
  item_pair(m, pair, a, b);
  ia = a;
  ib = m.nL + b;
}

__device__ __forceinline__ int item_halves(const ItemMap& m, int pair, int (&ia)[2], int (&ib)[2],
                                           int (&buf)[2]) {
  if (m.kind != kMapList) {
    item_operands(m, pair, ia[0], ib[0]);
    buf[0] = 0;
    return 1;
  }
  const int32_t* e = m.list + (size_t)pair * 5;
  int nh = 0;
  if (e[1] >= 0) {
    ia[nh] = e[1];
    ib[nh] = e[2];
    buf[nh] = 0;
    ++nh;
  }
  if (e[3] >= 0) {
    ia[nh] = e[3];
    ib[nh] = e[4];
    buf[nh] = 1;
    ++nh;
  }
  return nh;
}

__device__ __forceinline__ int item_target(const ItemMap& m, int pair) {
  if (m.kind == kMapList) return m.list[(size_t)pair * 5];
  if (m.kind == kMapPanel) return pair < m.nL ? m.lslot[pair] : m.uslot[pair - m.nL];
  int a, b;
  item_pair(m, pair, a, b);
  return m.tslot[a * m.nU + b];
}

__global__ void __launch_bounds__(kPThreads, 1) schur_tc_kernel(
    const ItemMap map, int n_pencils, int64_t n_slots, const unsigned char* __restrict__ staging,
    const unsigned char* __restrict__ staging1, int64_t staging_pencil_stride,
    int32_t* __restrict__ status, int* __restrict__ claim,
    const __grid_constant__ CUtensorMap tmap_c, long long wl) {
  const int n_pairs = map.n_pairs;
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
    mbar_init(&sh.drain, 1);
    sh.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // What the producer and the MMA issuer have in flight, for the drain
  // after a failure: the ring stages the producer filled (bit s) and the
  // phase parity of its last fill of each; whether any MMA was issued.
  uint32_t filled = 0, fill_parity = 0;
  bool issued = false;
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
      // The next item's index (a claim from the shared counter, or the
      // static stride) and its list entry are fetched one item ahead: the
      // atomic and the dependent list load then overlap the current item's
      // copies instead of draining the ring at every item boundary.  A
      // claimed item is always processed by the CTA that claimed it.
      int cur = claim != nullptr ? atomicAdd(claim, 1) : (int)blockIdx.x;
      int ia[2], ib[2], bf[2], nh = 0;
      if (cur < total) nh = item_halves(map, cur % n_pairs, ia, ib, bf);
      int nxt = claim != nullptr ? atomicAdd(claim, 1) : cur + (int)gridDim.x;
      for (int j = 0; !sh.failed; ++j) {
        int it = cur < total ? cur : -1;
        if (claim != nullptr) {
          // dynamic: the item index reaches the MMA issuer and the epilogue
          // through sh.items, published by this thread's arrive on full[]
          sh.items[j % kItemRing] = it;
          if (it < 0) {
            // stop token: one slab slot whose full[] completes without data
            if (!mbar_wait(&sh.empty[stage], phase ^ 1, wl)) {
              sh.failed = 1;
              atomicCAS(&status[0], 0, (int)AOSB_ERR_TIMEOUT);
              break;
            }
            mbar_arrive(&sh.full[stage]);
            break;
          }
        } else if (it < 0) {
          break;
        }
        const int p = it / n_pairs;
        const int nslabs = nh * kSlabs;
        int na[2] = {0, 0}, nb[2] = {0, 0}, nf[2] = {0, 0}, nnh = 0;
        for (int s = 0; s < nslabs; ++s) {
          if (s == 2 && nxt < total) nnh = item_halves(map, nxt % n_pairs, na, nb, nf);
          const int h = s / kSlabs, sl = s % kSlabs;
          const unsigned char* base = (bf[h] ? staging1 : staging) + (size_t)p * staging_pencil_stride;
          const unsigned char* stA = base + (size_t)ia[h] * kStagedTileBytes;
          const unsigned char* stB = base + (size_t)ib[h] * kStagedTileBytes;
          if (!mbar_wait(&sh.empty[stage], phase ^ 1, wl)) {
            sh.failed = 1;
            atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
            break;
          }
          filled |= 1u << stage;
          fill_parity = (fill_parity & ~(1u << stage)) | (phase << stage);
          mbar_expect_tx(&sh.full[stage], 2 * kOperandSlabBytes);
          bulk_g2s(sh.a[stage], stA + (size_t)sl * kOperandSlabBytes, kOperandSlabBytes,
                   &sh.full[stage]);
          bulk_g2s(sh.b[stage], stB + (size_t)sl * kOperandSlabBytes, kOperandSlabBytes,
                   &sh.full[stage]);
          if (++stage == kStagesP) { stage = 0; phase ^= 1; }
        }
        if (sh.failed) break;
        cur = nxt;
        nh = nnh;
        for (int q = 0; q < 2; ++q) {
          ia[q] = na[q];
          ib[q] = nb[q];
          bf[q] = nf[q];
        }
        nxt = cur >= total ? total : claim != nullptr ? atomicAdd(claim, 1) : cur + (int)gridDim.x;
      }
    }
  } else if (warp == kEpiWarps + 1) {
    if (lane == 0) {
      const uint32_t id_pos = umma_idesc_mn(kTcT, kTcT, false), id_neg = umma_idesc_mn(kTcT, kTcT, true);
      const uint32_t lbo = (kTcT / 8) * 128, sbo = 128;
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      for (int j = 0; !sh.failed; ++j) {
        int it = blockIdx.x + j * (int)gridDim.x;
        if (claim == nullptr && it >= total) break;
        if (!mbar_wait(&sh.acc_empty[acc], acc_phase ^ 1, wl)) {
          sh.failed = 1;
          atomicCAS(&status[claim == nullptr ? it / n_pairs : 0], 0, (int)AOSB_ERR_TIMEOUT);
          break;
        }
        bool first_waited = false;
        if (claim != nullptr) {
          // the item index is published with the item's first slab
          if (!mbar_wait(&sh.full[stage], phase, wl)) {
            sh.failed = 1;
            atomicCAS(&status[0], 0, (int)AOSB_ERR_TIMEOUT);
            break;
          }
          it = *reinterpret_cast<volatile int*>(&sh.items[j % kItemRing]);
          if (it < 0) {
            mbar_arrive(&sh.acc_full[acc]);  // stop token for the epilogue
            break;
          }
          first_waited = true;
        }
        const int p = it / n_pairs;
        int ia[2], ib[2], bf[2];
        const int nslabs = item_halves(map, it % n_pairs, ia, ib, bf) * kSlabs;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t re = tmem + (uint32_t)acc * 256, im = re + kTcT;
        bool ok = true;
        for (int s = 0; s < nslabs; ++s) {
          if (!(s == 0 && first_waited) && !mbar_wait(&sh.full[stage], phase, wl)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          issued = true;
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
    // Epilogue warps.  Warp w owns TMEM lanes (tile rows) 32*(w%4) .. +31
    // and columns 64*(w/4) .. +63, as two 32 x 32 blocks.  Lane l holds row
    // l of a block after tcgen05.ld; it writes the negated values into the
    // warp's swizzled shared tile, and lane 0 hands the tile to the TMA
    // unit, which adds it into the target tile (C -= acc).  The tile is
    // rewritten only after the previous reduce has finished reading it.
    const int quarter = warp % 4, half = warp / 4;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    float* bre = sh.ep[warp][0];
    float* bim = sh.ep[warp][1];
    const int sw = lane & 7;
    const bool store = map.kind == kMapPanel;
    const float sgn = store ? 1.0f : -1.0f;  // store acc / add -acc
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int j = 0;; ++j) {
      int it = blockIdx.x + j * (int)gridDim.x;
      if (claim == nullptr && it >= total) break;
      const bool ready =
          __all_sync(0xffffffffu, mbar_wait(&sh.acc_full[acc], acc_phase, wl) ? 1 : 0);
      if (!ready) {
        if (lane == 0) {
          sh.failed = 1;
          atomicCAS(&status[claim == nullptr ? it / n_pairs : 0], 0, (int)AOSB_ERR_TIMEOUT);
        }
        break;
      }
      if (claim != nullptr) {
        it = *reinterpret_cast<volatile int*>(&sh.items[j % kItemRing]);
        if (it < 0) break;
      }
      const int p = it / n_pairs, pair = it % n_pairs;
      // first row of the target tile's real plane in the [rows][128] view
      const int64_t row0 = ((int64_t)p * n_slots + item_target(map, pair)) * (2 * kTcT);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = tmem + (uint32_t)acc * 256 + (uint32_t)half * 64 + lane_addr;
#pragma unroll
      for (int bk = 0; bk < 2; ++bk) {
        float vr[2][16], vi[2][16];
        tmem_ld16(base + bk * 32, vr[0]);
        tmem_ld16(base + bk * 32 + 16, vr[1]);
        tmem_ld16(base + kTcT + bk * 32, vi[0]);
        tmem_ld16(base + kTcT + bk * 32 + 16, vi[1]);
        if (bk == 1) {
          // every TMEM read of this accumulator is done: release it
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(&sh.acc_empty[acc]);
        }
        if (lane == 0) bulk_wait_read_all();
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int h = c / 4, j = (c % 4) * 4;
          const int off = lane * 32 + ((c ^ sw) * 4);
          *reinterpret_cast<float4*>(bre + off) = make_float4(
              sgn * vr[h][j], sgn * vr[h][j + 1], sgn * vr[h][j + 2], sgn * vr[h][j + 3]);
          *reinterpret_cast<float4*>(bim + off) = make_float4(
              sgn * vi[h][j], sgn * vi[h][j + 1], sgn * vi[h][j + 2], sgn * vi[h][j + 3]);
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          const int x = half * 64 + bk * 32;
          const int y = (int)(row0 + quarter * 32);
          if (store) {
            tma_store_2d(&tmap_c, bre, x, y);
            tma_store_2d(&tmap_c, bim, x, y + kTcT);
          } else {
            tma_reduce_add_2d(&tmap_c, bre, x, y);
            tma_reduce_add_2d(&tmap_c, bim, x, y + kTcT);
          }
          bulk_commit();
        }
      }
      if (++acc == 2) { acc = 0; acc_phase ^= 1; }
    }
    // the target updates must be complete (not only read) before exit
    if (lane == 0) bulk_wait_all();
    __syncwarp();
  }
  // Every role has left its loop (all waits are bounded).  After a failure
  // the producer waits (bounded) until each stage it filled has received
  // its bytes, and the MMA issuer commits once more and waits until its
  // MMAs are done, so no copy or MMA lands in shared memory or TMEM after
  // they are released.
  __syncthreads();
  if (sh.failed) {
    if (warp == kEpiWarps && lane == 0)
      for (int s = 0; s < kStagesP; ++s)
        if (filled & (1u << s)) mbar_wait(&sh.full[s], (fill_parity >> s) & 1u);
    if (warp == kEpiWarps + 1 && lane == 0 && issued) {
      umma_commit(&sh.drain);
      mbar_wait(&sh.drain, 0);
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

static int64_t staged_tiles_per_pencil(const aosb_plan* P) {
  int64_t most = 0;
  for (int64_t k = 0; k < P->nb; ++k) {
    const int64_t items = (P->lb_off[k + 1] - P->lb_off[k]) + (P->ur_off[k + 1] - P->ur_off[k]);
    most = items > most ? items : most;
  }
  return most + 2;
}

// Four staging buffers (tile step k uses buffer k % 4): with two-step
// updates and lookahead, steps k + 2 and k + 3 are staged while the
// two-step update of steps k and k + 1 still reads theirs.  After them, 256
// bytes hold the item counter of the shared two-step updates.
constexpr size_t kClaimBytes = 256;
size_t factor_tc_workspace(const aosb_plan* P, int32_t n_pencils) {
  if (P->T != kTcT) return 0;
  return 4 * (size_t)staged_tiles_per_pencil(P) * kStagedTileBytes * (size_t)n_pencils +
         kClaimBytes;
}

// Side stream of a caller stream for the lookahead panels (created once,
// non-blocking, kept for the life of the process).
static int side_stream(cudaStream_t main, cudaStream_t* out, char* err, size_t cap) {
  static std::mutex mu;
  static std::vector<std::pair<cudaStream_t, cudaStream_t>> table;
  int device = 0;
  cudaGetDevice(&device);
  std::lock_guard<std::mutex> lock(mu);
  for (auto& e : table) {
    if (e.first == main) {
      int dev2 = -1;
      if (cudaStreamGetDevice(e.second, &dev2) == cudaSuccess && dev2 == device) {
        *out = e.second;
        return 0;
      }
    }
  }
  cudaStream_t s = nullptr;
  AOSB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), err, cap);
  table.emplace_back(main, s);
  *out = s;
  return 0;
}

// Tensor map of the factor storage as a [rows][T] FP32 matrix (each tile is
// 2 planes x T rows), 32 x 32 boxes, 128-byte swizzle: the destination of
// the epilogue's bulk reduce-add and store.
static int factor_tensor_map(void* factor, int64_t rows, CUtensorMap* map, char* err, size_t cap) {
  return encode_f32_2d(factor, kTcT, (uint64_t)rows, 32, 32, true, map, err, cap);
}

// SMs left to the lookahead side stream (0 = the default rule); process-wide.
std::atomic<int> g_lookahead_sms{0};

// 1: the two-step Schur updates run as two-CTA pairs (schur_pair.cu);
// process-wide.
std::atomic<int> g_schur_pairs{0};

// Polls of one mbarrier wait before a tensor-core kernel gives up and
// records AOSB_ERR_TIMEOUT; process-wide, read at each launch.
std::atomic<long long> g_tc_wait_limit{tc::kTcWaitLimit};
long long tc::tc_wait_limit() { return g_tc_wait_limit.load(); }

int factor_tc(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap) {
  if (P->T != kTcT)
    return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "tensor-core path needs tile = 128");
  if (a->workspace == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "tensor-core path needs a staging workspace");
  cudaStream_t st = (cudaStream_t)a->stream;
  const int np = a->n_pencils;
  const size_t smem = sizeof(PShared) + 1024;
  static_assert(sizeof(PShared) + 1024 <= 232448, "shared memory budget");
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  // kernel attributes belong to each device's context: set once per device
  static std::atomic<uint64_t> attr_devices{0};
  const uint64_t dev_bit = device < 64 ? (uint64_t)1 << device : 0;
  if (dev_bit == 0 || (attr_devices.load() & dev_bit) == 0) {
    cudaError_t e = cudaFuncSetAttribute(schur_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess)
      return set_error(err, cap, AOSB_ERR_CUDA, "schur_tc smem attribute: %s", cudaGetErrorString(e));
    attr_devices.fetch_or(dev_bit);
  }
  // staged tiles per pencil: the step's L and U tiles plus the two
  // diagonal inverses of the panel product
  const int64_t pencil_stride = staged_tiles_per_pencil(P) * (int64_t)kStagedTileBytes;
  unsigned char* staging = (unsigned char*)a->workspace;
  CUtensorMap tmap_c;
  if (int rc = factor_tensor_map(a->factor, (int64_t)np * P->n_slots * 2 * kTcT, &tmap_c, err, cap))
    return rc;
  const bool tc_panels = a->precision != AOSB_PRECISION_BF16X3_FP32_PANELS;
  const long long wl = tc_wait_limit();
  auto grid_for = [&](int64_t items, int cap_ctas) {
    return (int)(items < cap_ctas ? items : cap_ctas);
  };
  // Lookahead (tensor-core panels): step k's Schur targets in tile row and
  // column k + 1 go first ("cross"); then step k + 1's diagonal LU, panel
  // products and staging run on a side stream on `reserve` SMs while the
  // rest of step k's Schur update runs on the others.
  const bool lookahead = tc_panels && sms >= 32;
  const int chosen = g_lookahead_sms.load();
  // default: 5/4 of the pencils (the side stream's diagonal LU runs one CTA
  // per pencil), at most a third of the SMs; the reserved SMs join the rest
  // of the two-step update once the panels are done, so a generous reserve
  // costs little (c2: 48 SMs beat 37 at 64 pencils, 40 beat 24 and 16 at 32)
  const int reserve = !lookahead ? 0
                      : chosen > 0 ? std::min(chosen, sms / 2)
                                   : std::min(std::max(np * 5 / 4, 8), sms / 3);
  cudaStream_t side = nullptr;
  cudaEvent_t ev_cross = nullptr, ev_panel = nullptr;
  if (lookahead) {
    if (int rc = side_stream(st, &side, err, cap)) return rc;
    AOSB_CUDA_TRY(cudaEventCreateWithFlags(&ev_cross, cudaEventDisableTiming), err, cap);
    if (cudaEventCreateWithFlags(&ev_panel, cudaEventDisableTiming) != cudaSuccess) {
      cudaEventDestroy(ev_cross);
      return set_error(err, cap, AOSB_ERR_CUDA, "cudaEventCreate failed");
    }
  }
  struct EventGuard {
    cudaEvent_t a, b;
    ~EventGuard() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } guard{ev_cross, ev_panel};
  const int64_t buffer_bytes = (int64_t)np * pencil_stride;
  auto stage_buf = [&](int64_t k) { return staging + (k & 3) * buffer_bytes; };

  // diagonal LU + panel products of step k on stream s (panel grid <= cap_ctas)
  auto panels = [&](int64_t k, cudaStream_t s, int cap_ctas) -> int {
    if (int rc = factor_step_diag(P, a, (int)k, s, err, cap)) return rc;
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    if (nL + nU == 0) return 0;
    const int32_t* lslot = P->d_lb_slot + P->lb_off[k];
    const int32_t* uslot = P->d_ur_slot + P->ur_off[k];
    // L_ik = A_ik inv(U_kk), U_kj = inv(L_kk) P_k A_kj on the tensor cores
    stage_kernel<<<dim3(nL + nU + 2, np), 256, 0, s>>>(
        nL, nU, 1, (int)k, lslot, uslot, P->diag_slot[k], P->n_slots, P->n_pad, a->factor,
        a->pivots, stage_buf(k), pencil_stride);
    const ItemMap pm{kMapPanel, nL, nU, nL + nU, 0, 0, nullptr, lslot, uslot, nullptr};
    schur_tc_kernel<<<grid_for((int64_t)(nL + nU) * np, cap_ctas), kPThreads, smem, s>>>(
        pm, np, P->n_slots, stage_buf(k), stage_buf(k), pencil_stride, a->status, nullptr, tmap_c, wl);
    count_launches(2);
    return 0;
  };
  // Schur staging of step k (L_ik as A, U_kj as B) on stream s
  auto stage_schur = [&](int64_t k, cudaStream_t s) {
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    if (nL == 0 || nU == 0) return;
    stage_kernel<<<dim3(nL + nU, np), 256, 0, s>>>(nL, nU, 0, (int)k, P->d_lb_slot + P->lb_off[k],
                                                  P->d_ur_slot + P->ur_off[k], 0, P->n_slots,
                                                  P->n_pad, a->factor, a->pivots, stage_buf(k),
                                                  pencil_stride);
    count_launches(1);
  };
  // Schur update of step k (the pairs `kind` selects) on stream s, untimed
  auto schur_on = [&](int64_t k, int kind, int a0, int b0, int n_pairs, int cap_ctas,
                      cudaStream_t s) {
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    const ItemMap sm{kind, nL, nU, n_pairs, a0, b0, P->d_sc_slot + P->sc_off[k], nullptr, nullptr,
                     nullptr};
    schur_tc_kernel<<<grid_for((int64_t)n_pairs * np, cap_ctas), kPThreads, smem, s>>>(
        sm, np, P->n_slots, stage_buf(k), stage_buf(k), pencil_stride, a->status, nullptr, tmap_c, wl);
    count_launches(1);
  };
  // Schur update of step k (the pairs `kind` selects) on the caller stream,
  // timed
  auto schur = [&](int64_t k, int kind, int a0, int b0, int n_pairs, int cap_ctas) {
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    const int64_t items = (int64_t)n_pairs * np;
    cudaEvent_t ev[2];
    const bool timed = timing_begin(st, ev);
    const ItemMap sm{kind, nL, nU, n_pairs, a0, b0, P->d_sc_slot + P->sc_off[k], nullptr, nullptr,
                     nullptr};
    schur_tc_kernel<<<grid_for(items, cap_ctas), kPThreads, smem, st>>>(
        sm, np, P->n_slots, stage_buf(k), stage_buf(k), pencil_stride, a->status, nullptr, tmap_c, wl);
    count_launches(1);
    if (timed)
      timing_end(kTimedSchur, st, ev, (double)items * 8.0 * kTcT * kTcT * kTcT,
                 (double)items * 2.0 * 2 * kTcT * kTcT * sizeof(float) +
                     (double)(nL + nU) * np * kStagedTileBytes * ((double)n_pairs / (nL * nU)));
  };

  // targets of step k in tile row or column k + 1 (K = 128), on stream s
  auto inner = [&](int64_t k, cudaStream_t s, int cap_ctas) {
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    if (nL == 0 || nU == 0) return;
    const int a0 = P->lb_tile[P->lb_off[k]] == k + 1 ? 1 : 0;
    const int b0 = P->ur_tile[P->ur_off[k]] == k + 1 ? 1 : 0;
    const int cross = nL * nU - (nL - a0) * (nU - b0);
    if (cross > 0) schur_on(k, kMapCross, a0, b0, cross, cap_ctas, s);
  };
  // two-step update of super-step ss (tile steps 2 ss, 2 ss + 1), the cross
  // or the rest items, on stream s (timed); with `claim` the launch takes
  // items from the shared counter instead of a fixed share
  int* claim_counter = reinterpret_cast<int*>(staging + 4 * (int64_t)np * pencil_stride);
  const bool pairs = g_schur_pairs.load() != 0 && P->d_sp_rest != nullptr;
  int pair_rc = 0;
  auto two_step = [&](int64_t ss, bool cross, int cap_ctas, cudaStream_t s = nullptr,
                      int* claim = nullptr, bool count_work = true) {
    if (s == nullptr) s = st;
    const std::vector<int64_t>& off = cross ? P->ss_cross_off : P->ss_rest_off;
    const std::vector<int32_t>& host = cross ? P->ss_cross : P->ss_rest;
    const int32_t* dev = cross ? P->d_ss_cross : P->d_ss_rest;
    const int64_t n = off[ss + 1] - off[ss];
    if (n == 0) return;
    const int64_t k0 = 2 * ss;
    double halves = 0;
    for (int64_t i = off[ss]; i < off[ss + 1]; ++i)
      halves += (host[5 * i + 1] >= 0 ? 1 : 0) + (host[5 * i + 3] >= 0 ? 1 : 0);
    cudaEvent_t ev[2];
    const bool timed = count_work && timing_begin(s, ev);
    if (pairs) {
      // the same items as pairs of targets sharing a column: two-CTA MMAs
      const std::vector<int64_t>& poff = cross ? P->sp_cross_off : P->sp_rest_off;
      const int32_t* pdev = cross ? P->d_sp_cross : P->d_sp_rest;
      const int rc = schur_pair_launch(pdev + 8 * poff[ss], poff[ss + 1] - poff[ss], np,
                                       P->n_slots, staging, 4 * buffer_bytes,
                                       (k0 & 3) * buffer_bytes, ((k0 + 1) & 3) * buffer_bytes,
                                       pencil_stride, a->status, claim, tmap_c, cap_ctas, s, err,
                                       cap);
      if (rc != 0 && pair_rc == 0) pair_rc = rc;
    } else {
      const ItemMap lm{kMapList, 0, 0, (int)n, 0, 0, nullptr, nullptr, nullptr, dev + 5 * off[ss]};
      schur_tc_kernel<<<grid_for(n * np, cap_ctas), kPThreads, smem, s>>>(
          lm, np, P->n_slots, stage_buf(k0), stage_buf(k0 + 1), pencil_stride, a->status, claim,
          tmap_c, wl);
      count_launches(1);
    }
    // algorithmic bytes: every target read and written once, the staged L
    // and U tiles of both steps read once.  Of two launches sharing one
    // counter, the main one is timed with all the work: the second joins
    // later on other SMs and ends within about one item of the first.
    const double staged = (double)(P->lb_off[k0 + 1] - P->lb_off[k0] + P->ur_off[k0 + 1] -
                                   P->ur_off[k0] + P->lb_off[k0 + 2] - P->lb_off[k0 + 1] +
                                   P->ur_off[k0 + 2] - P->ur_off[k0 + 1]);
    if (timed)
      timing_end(kTimedSchur, s, ev, halves * np * 8.0 * kTcT * kTcT * kTcT,
                 (double)n * np * 2.0 * 2 * kTcT * kTcT * sizeof(float) +
                     staged * np * kStagedTileBytes);
  };

  // Two-step (K = 256) updates with lookahead: per super-step (k, k + 1),
  // after step k's cross targets (K = 128) and step k + 1's panels, one
  // update applies both steps to every other target, reading and writing
  // each target once instead of twice.  The items in tile rows/columns
  // k + 2, k + 3 go first; the side stream then prepares the next
  // super-step's two panels beside the rest.
  const bool two_steps = tc_panels && lookahead && a->precision == AOSB_PRECISION_BF16X3 &&
                         P->d_ss_rest != nullptr;
  if (two_steps) {
    const int64_t nb = P->nb;
    if (int rc = panels(0, st, sms)) return rc;
    stage_schur(0, st);
    if (nb > 1) {
      inner(0, st, sms);
      if (int rc = panels(1, st, sms)) return rc;
      stage_schur(1, st);
    }
    for (int64_t ss = 0; 2 * ss + 1 < nb; ++ss) {
      const int64_t k2 = 2 * ss + 2, k3 = 2 * ss + 3;
      two_step(ss, true, sms);
      if (k2 < nb) {
        // the rest items are shared through a counter: the main launch on
        // sms - reserve SMs starts at once, a second launch on the reserved
        // SMs joins it once the side stream's panel work is done
        AOSB_CUDA_TRY(cudaMemsetAsync(claim_counter, 0, sizeof(int), st), err, cap);
        AOSB_CUDA_TRY(cudaEventRecord(ev_cross, st), err, cap);
        AOSB_CUDA_TRY(cudaStreamWaitEvent(side, ev_cross, 0), err, cap);
        if (int rc = panels(k2, side, reserve)) return rc;
        stage_schur(k2, side);
        if (k3 < nb) {
          inner(k2, side, reserve);
          if (int rc = panels(k3, side, reserve)) return rc;
          stage_schur(k3, side);
        }
        // main launch first: it starts at once either way, and a profiler
        // that serializes launches then sees the full-grid launch take the
        // items
        two_step(ss, false, sms - reserve, st, claim_counter, true);
        two_step(ss, false, reserve, side, claim_counter, false);
        AOSB_CUDA_TRY(cudaEventRecord(ev_panel, side), err, cap);
        AOSB_CUDA_TRY(cudaStreamWaitEvent(st, ev_panel, 0), err, cap);
      } else {
        two_step(ss, false, sms);
      }
      if (pair_rc != 0) return pair_rc;
    }
    return launch_check(err, cap, "tensor-core factorization");
  }

  for (int64_t k = 0; k < P->nb; ++k) {
    const int nL = P->lb_off[k + 1] - P->lb_off[k];
    const int nU = P->ur_off[k + 1] - P->ur_off[k];
    // the kernel enumerates (target, pencil) items in 32-bit ints
    if ((int64_t)nL * nU * np > INT32_MAX)
      return set_error(err, cap, AOSB_ERR_SIZE, "too many Schur targets x pencils in one step");
    if (!tc_panels) {
      if (int rc = factor_step_panels(P, a, (int)k, err, cap)) return rc;
      stage_schur(k, st);
      if (nL > 0 && nU > 0) schur(k, kMapSchur, 0, 0, nL * nU, sms);
      continue;
    }
    if (k == 0) {
      if (int rc = panels(0, st, sms)) return rc;
      stage_schur(0, st);
    }
    const bool has_next = k + 1 < P->nb;
    if (nL == 0 || nU == 0) {
      if (has_next) {
        if (int rc = panels(k + 1, st, sms)) return rc;
        stage_schur(k + 1, st);
      }
      continue;
    }
    if (!lookahead || !has_next) {
      schur(k, kMapSchur, 0, 0, nL * nU, sms);
      if (has_next) {
        if (int rc = panels(k + 1, st, sms)) return rc;
        stage_schur(k + 1, st);
      }
      continue;
    }
    const int a0 = P->lb_tile[P->lb_off[k]] == k + 1 ? 1 : 0;
    const int b0 = P->ur_tile[P->ur_off[k]] == k + 1 ? 1 : 0;
    const int rest = (nL - a0) * (nU - b0);
    const int cross = nL * nU - rest;
    if (cross > 0) schur(k, kMapCross, a0, b0, cross, sms);
    AOSB_CUDA_TRY(cudaEventRecord(ev_cross, st), err, cap);
    AOSB_CUDA_TRY(cudaStreamWaitEvent(side, ev_cross, 0), err, cap);
    if (int rc = panels(k + 1, side, reserve)) return rc;
    stage_schur(k + 1, side);
    AOSB_CUDA_TRY(cudaEventRecord(ev_panel, side), err, cap);
    if (rest > 0) schur(k, kMapRest, a0, b0, rest, sms - reserve);
    AOSB_CUDA_TRY(cudaStreamWaitEvent(st, ev_panel, 0), err, cap);
  }
  return launch_check(err, cap, "tensor-core factorization");
}

}  // namespace aosb

extern "C" int32_t aosb_factor_set_schur_pairs(int32_t on) {
  if (on < 0 || on > 1) return -1;
  return aosb::g_schur_pairs.exchange(on);
}

extern "C" int64_t aosb_tc_set_wait_limit(int64_t polls) {
  if (polls < 0) return -1;
  return aosb::g_tc_wait_limit.exchange(polls == 0 ? aosb::tc::kTcWaitLimit : polls);
}

extern "C" int32_t aosb_factor_set_lookahead_sms(int32_t sms) {
  if (sms < 0) return -1;
  return aosb::g_lookahead_sms.exchange(sms);
}
