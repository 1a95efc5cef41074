// Two-CTA (cta_group::2, M = 256) split-BF16 Schur update of the two-step
// (K = 256) factorization lists.
//
// Why pairs.  One CTA applying a 128 x 128 x 16 slab with 12
// tcgen05.mma.kind::f16 (M = N = 128) makes the tensor core read 8 KB of
// operands from shared memory per MMA, about 121 B/clk at the tensor peak,
// while the TMA brings 32 KB per slab into the same shared memory and the
// epilogue stages every target through it: the single-CTA kernel runs out
// of shared-memory and L2 bandwidth before it runs out of tensor cycles.
// Here a cluster of two CTAs on one TPC updates two targets (i1, j), (i2, j)
// of the same tile column, which share their B tile U_kj (the plan's pair
// lists).  The even CTA issues one M = 256 MMA for both: each CTA holds its
// own target's A slab (128 rows) and one half of the shared B slab (64
// columns), and each CTA's TMEM receives its own target's 128 x 128
// accumulator.  Per CTA and slab that is 24 KB in from L2 instead of 32 KB
// and 6 KB of operand reads per MMA instead of 8 KB, with the two
// accumulator sets still double buffered.
//
// Roles (320 threads per CTA):
//   warp 8 lane 0   producer (both CTAs): one tensor-map load of the CTA's
//                   A slab and one of its half of the B slab per 16-wide K
//                   slab, into a kStages-deep ring; both CTAs' loads count
//                   on the even CTA's full[] barrier (.cta_group::2 loads),
//                   whose expected bytes the even CTA posts for the pair.
//                   With a shared item counter the even CTA claims each item
//                   and hands its index to the odd CTA (remote store +
//                   remote arrive on item_full[]);
//   warp 9 lane 0   even CTA: MMA issuer -- waits for full[], issues 12
//                   M = 256 MMAs per slab, commits the slab's release to
//                   empty[] of both CTAs and the accumulator to acc_full[] of
//                   both (multicast commits);
//   warps 0-7       epilogue (both CTAs): TMEM -> 128B-swizzled shared tiles
//                   -> TMA reduce-add into the CTA's own target (C -= acc);
//                   every warp of both CTAs releases the accumulator on the
//                   even CTA's acc_empty[] (count 16).
// Every wait is bounded; after a failure each producer waits (bounded) for
// its own copies, the MMA issuer for its MMAs, and the two CTAs meet at a
// cluster barrier before freeing TMEM.
#include "plan.h"
#include "factor.h"
#include "tc_common.cuh"
#include "timing.h"

#include <cuda.h>

#include <atomic>

namespace aosb {
namespace {

using namespace tc;

constexpr int kT = 128;
constexpr int kSlabK = 16;
constexpr int kSlabs = kT / kSlabK;                 // 8 per tile step
constexpr int kASlabBytes = 4 * kT * kSlabK * 2;    // 16 KB: four planes, 128 rows
constexpr int kBHalfBytes = kASlabBytes / 2;        // 8 KB: four planes, 64 rows
constexpr int kAPlane = kASlabBytes / 4;            // 4096
constexpr int kBPlane = kBHalfBytes / 4;            // 2048
constexpr int kPlanesPerTile = 32;                  // 4 KB plane slabs per staged tile
#ifndef AOSB_PAIR_STAGES
#define AOSB_PAIR_STAGES 6
#endif
constexpr int kStages = AOSB_PAIR_STAGES;
constexpr int kEpiWarps = 8;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kTmemCols = 512;
constexpr int kRing = 8;

struct PairShared {
  alignas(1024) unsigned char a[kStages][kASlabBytes];
  alignas(1024) unsigned char b[kStages][kBHalfBytes];
  alignas(1024) float ep[kEpiWarps][2][32 * 32];
  uint64_t full[kStages];       // even CTA: both CTAs' TMA bytes of a stage
  uint64_t empty[kStages];      // the even CTA's MMA commit, both CTAs
  uint64_t acc_full[2];         // the even CTA's accumulator commit, both CTAs
  uint64_t acc_empty[2];        // even CTA: 16 epilogue warps of both CTAs
  uint64_t item_full[kRing];    // odd CTA: item handed over by the even CTA
  uint64_t drain;
  uint32_t tmem_base;
  int failed;
  int items[kRing];
};

__device__ __forceinline__ uint32_t cta_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t map_to(const void* p, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_u32(p)), "r"(rank));
  return out;
}
__device__ __forceinline__ void remote_arrive(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void remote_store(uint32_t cluster_addr, int v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(cluster_addr), "r"(v) : "memory");
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" :::
                   "memory");
}
// Bounded wait with cluster-scope acquire (barriers that other CTAs arrive on).
__device__ __forceinline__ bool mbar_wait_cl(uint64_t* bar, uint32_t parity, long long limit) {
  const uint32_t addr = smem_u32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 4096) __nanosleep(64);
  }
  return false;
}
// Tensor-map load into this CTA's shared memory whose completion is
// counted on the barrier at cluster address `bar` (the even CTA's; the
// .cta_group::2 form lets the odd CTA's loads signal the even CTA).
__device__ __forceinline__ void tma_load_5d_pair(void* dst, const CUtensorMap* map, int c2, int c4,
                                                 uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(0), "r"(0), "r"(c2), "r"(0), "r"(c4)
      : "memory");
}
__device__ __forceinline__ void umma2_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive on `bar` (same offset) in both CTAs once this thread's MMAs are done.
__device__ __forceinline__ void umma2_commit_both(uint64_t* bar) {
  const uint16_t mask = 3;
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
      "[%0], %1;" ::"r"(smem_u32(bar)),
      "h"(mask)
      : "memory");
}
__device__ __forceinline__ void umma2_commit_local(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

struct Halves {
  int n;         // 1 or 2 tile steps
  int a[2];      // staged A index of this CTA per half
  int b[2];      // shared staged B index per half
  int buf[2];    // 0: first step's buffer, 1: second's
};
__device__ __forceinline__ Halves halves_of(const int32_t* e, uint32_t rank) {
  Halves h;
  h.n = 0;
  if (e[2] >= 0) {
    h.a[h.n] = rank ? e[3] : e[2];
    h.b[h.n] = e[4];
    h.buf[h.n] = 0;
    ++h.n;
  }
  if (e[5] >= 0) {
    h.a[h.n] = rank ? e[6] : e[5];
    h.b[h.n] = e[7];
    h.buf[h.n] = 1;
    ++h.n;
  }
  return h;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1) schur_pair_kernel(
    const int32_t* __restrict__ list, int n_pairs, int n_pencils, int64_t n_slots,
    int64_t buf0_planes, int64_t buf1_planes, int64_t pencil_planes, int32_t* __restrict__ status,
    int* __restrict__ claim, const __grid_constant__ CUtensorMap tm_a,
    const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tmap_c,
    long long wl) {
  extern __shared__ unsigned char dyn[];
  PairShared& sh = *reinterpret_cast<PairShared*>(
      (reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t rank = cta_rank();
  const int cluster = blockIdx.x / 2, n_clusters = gridDim.x / 2;
  const int total = n_pairs * n_pencils;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sh.acc_full[b], 1);
      mbar_init(&sh.acc_empty[b], 2 * kEpiWarps);
    }
    for (int r = 0; r < kRing; ++r) mbar_init(&sh.item_full[r], 1);
    mbar_init(&sh.drain, 1);
    sh.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // both CTAs' barriers and TMEM exist before either side signals the other
  cluster_sync();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem_base;
  uint32_t filled = 0, fill_parity = 0;   // producer: stages filled, parity of the last fill
  bool issued = false;                    // even CTA's MMA issuer: any MMA issued

  if (warp == kEpiWarps) {
    // ------------------------------------------------------------- producer
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (int j = 0; !sh.failed; ++j) {
        int it = cluster + j * n_clusters;
        if (claim != nullptr) {
          const int r = j % kRing;
          if (rank == 0) {
            it = atomicAdd(claim, 1);
            if (it >= total) it = -1;
            sh.items[r] = it;
            remote_store(map_to(&sh.items[r], 1), it);
            remote_arrive(map_to(&sh.item_full[r], 1));
            if (it < 0) {
              // stop token for this CTA's MMA issuer: a slot whose full[]
              // completes without data
              if (!mbar_wait(&sh.empty[stage], phase ^ 1, wl)) {
                sh.failed = 1;
                atomicCAS(&status[0], 0, (int)AOSB_ERR_TIMEOUT);
                break;
              }
              mbar_arrive(&sh.full[stage]);
              break;
            }
          } else {
            if (!mbar_wait_cl(&sh.item_full[r], (uint32_t)((j / kRing) & 1), wl)) {
              sh.failed = 1;
              atomicCAS(&status[0], 0, (int)AOSB_ERR_TIMEOUT);
              break;
            }
            it = *reinterpret_cast<volatile int*>(&sh.items[r]);
            if (it < 0) break;
          }
        } else if (it >= total) {
          break;
        }
        const int p = it / n_pairs;
        const Halves h = halves_of(list + (size_t)(it % n_pairs) * 8, rank);
        bool ok = true;
        const uint32_t full0 = map_to(&sh.full[0], 0);
        for (int s = 0; s < h.n * kSlabs; ++s) {
          const int hh = s / kSlabs, sl = s % kSlabs;
          const int64_t base = (h.buf[hh] ? buf1_planes : buf0_planes) + (int64_t)p * pencil_planes;
          if (!mbar_wait_cl(&sh.empty[stage], phase ^ 1, wl)) {
            ok = false;
            break;
          }
          filled |= 1u << stage;
          fill_parity = (fill_parity & ~(1u << stage)) | (phase << stage);
          // the even CTA's full[] counts both CTAs' bytes; the odd CTA's
          // loads signal it directly
          if (rank == 0) mbar_expect_tx(&sh.full[stage], 2 * (kASlabBytes + kBHalfBytes));
          const uint32_t bar = full0 + (uint32_t)(stage * sizeof(uint64_t));
          tma_load_5d_pair(sh.a[stage], &tm_a, 0,
                           (int)(base + (int64_t)h.a[hh] * kPlanesPerTile + sl * 4), bar);
          tma_load_5d_pair(sh.b[stage], &tm_b, (int)rank,
                           (int)(base + (int64_t)h.b[hh] * kPlanesPerTile + sl * 4), bar);
          if (++stage == kStages) { stage = 0; phase ^= 1; }
        }
        if (!ok) {
          sh.failed = 1;
          atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
          break;
        }
      }
    }
  } else if (warp == kEpiWarps + 1) {
    if (lane == 0 && rank == 0) {
      // --------------------------------------------------------- MMA issuer
      const uint32_t idesc_pos = umma_idesc_mn(2 * kT, kT, false);
      const uint32_t idesc_neg = umma_idesc_mn(2 * kT, kT, true);
      const uint32_t alb = (kT / 8) * 128, blb = (kT / 16) * 128, sbo = 128;
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      for (int j = 0; !sh.failed; ++j) {
        int it = cluster + j * n_clusters;
        if (claim == nullptr && it >= total) break;
        if (!mbar_wait_cl(&sh.acc_empty[acc], acc_phase ^ 1, wl)) {
          sh.failed = 1;
          atomicCAS(&status[claim == nullptr ? it / n_pairs : 0], 0, (int)AOSB_ERR_TIMEOUT);
          break;
        }
        bool first_waited = false;
        if (claim != nullptr) {
          if (!mbar_wait_cl(&sh.full[stage], phase, wl)) {
            sh.failed = 1;
            atomicCAS(&status[0], 0, (int)AOSB_ERR_TIMEOUT);
            break;
          }
          it = *reinterpret_cast<volatile int*>(&sh.items[j % kRing]);
          if (it < 0) {
            mbar_arrive(&sh.acc_full[acc]);   // stop token for this CTA's epilogue
            break;
          }
          first_waited = true;
        }
        const int p = it / n_pairs;
        const Halves h = halves_of(list + (size_t)(it % n_pairs) * 8, 0);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t re = tmem + (uint32_t)acc * 256, im = re + kT;
        bool ok = true;
        for (int s = 0; s < h.n * kSlabs; ++s) {
          if (!(s == 0 && first_waited) && !mbar_wait_cl(&sh.full[stage], phase, wl)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          issued = true;
          const uint32_t sa = smem_u32(sh.a[stage]), sb = smem_u32(sh.b[stage]);
          uint64_t A[4], Bv[4];
#pragma unroll
          for (int pl = 0; pl < 4; ++pl) {
            A[pl] = umma_desc(sa + pl * kAPlane, alb, sbo);
            Bv[pl] = umma_desc(sb + pl * kBPlane, blb, sbo);
          }
          // the two accumulators alternate, and MMAs that read the same A
          // plane follow each other
          const uint32_t first = s == 0 ? 0u : 1u;
          umma2_bf16(re, A[0], Bv[0], idesc_pos, first);
          umma2_bf16(im, A[0], Bv[2], idesc_pos, first);
          umma2_bf16(re, A[0], Bv[1], idesc_pos, 1);
          umma2_bf16(im, A[0], Bv[3], idesc_pos, 1);
          umma2_bf16(re, A[1], Bv[0], idesc_pos, 1);
          umma2_bf16(im, A[1], Bv[2], idesc_pos, 1);
          umma2_bf16(re, A[2], Bv[2], idesc_neg, 1);
          umma2_bf16(im, A[2], Bv[0], idesc_pos, 1);
          umma2_bf16(re, A[2], Bv[3], idesc_neg, 1);
          umma2_bf16(im, A[2], Bv[1], idesc_pos, 1);
          umma2_bf16(re, A[3], Bv[2], idesc_neg, 1);
          umma2_bf16(im, A[3], Bv[0], idesc_pos, 1);
          umma2_commit_both(&sh.empty[stage]);
          if (++stage == kStages) { stage = 0; phase ^= 1; }
        }
        if (!ok) {
          sh.failed = 1;
          atomicCAS(&status[p], 0, (int)AOSB_ERR_TIMEOUT);
          break;
        }
        umma2_commit_both(&sh.acc_full[acc]);
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
    }
  } else {
    // ------------------------------------------------------------- epilogue
    // Warp w owns TMEM lanes (target rows) 32 (w % 4) .. +31 and columns
    // 64 (w / 4) .. +63 as two 32 x 32 blocks; -acc goes through the warp's
    // swizzled shared tile into a TMA reduce-add on this CTA's target.
    const int quarter = warp % 4, half = warp / 4;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    float* bre = sh.ep[warp][0];
    float* bim = sh.ep[warp][1];
    const int sw = lane & 7;
    const uint32_t acc_empty0 = map_to(&sh.acc_empty[0], 0);
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int j = 0;; ++j) {
      int it = cluster + j * n_clusters;
      if (claim == nullptr && it >= total) break;
      if (claim != nullptr && rank == 1) {
        const bool got = __all_sync(
            0xffffffffu, mbar_wait_cl(&sh.item_full[j % kRing], (uint32_t)((j / kRing) & 1), wl));
        if (!got) {
          if (lane == 0) {
            sh.failed = 1;
            atomicCAS(&status[0], 0, (int)AOSB_ERR_TIMEOUT);
          }
          break;
        }
        it = *reinterpret_cast<volatile int*>(&sh.items[j % kRing]);
        if (it < 0) break;
      }
      const bool ready = __all_sync(0xffffffffu, mbar_wait_cl(&sh.acc_full[acc], acc_phase, wl));
      if (!ready) {
        if (lane == 0) {
          sh.failed = 1;
          atomicCAS(&status[claim == nullptr ? it / n_pairs : 0], 0, (int)AOSB_ERR_TIMEOUT);
        }
        break;
      }
      if (claim != nullptr && rank == 0) {
        it = *reinterpret_cast<volatile int*>(&sh.items[j % kRing]);
        if (it < 0) break;
      }
      const int p = it / n_pairs;
      const int32_t* e = list + (size_t)(it % n_pairs) * 8;
      const int slot = rank ? e[1] : e[0];
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (slot < 0) {
        // single: this CTA's accumulator holds a product nobody needs
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          if (rank == 0) mbar_arrive(&sh.acc_empty[acc]);
          else remote_arrive(acc_empty0 + (uint32_t)(acc * sizeof(uint64_t)));
        }
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
        continue;
      }
      const int64_t row0 = ((int64_t)p * n_slots + slot) * (2 * kT);
      const uint32_t base = tmem + (uint32_t)acc * 256 + (uint32_t)half * 64 + lane_addr;
#pragma unroll
      for (int bk = 0; bk < 2; ++bk) {
        float vr[2][16], vi[2][16];
        tmem_ld16(base + bk * 32, vr[0]);
        tmem_ld16(base + bk * 32 + 16, vr[1]);
        tmem_ld16(base + kT + bk * 32, vi[0]);
        tmem_ld16(base + kT + bk * 32 + 16, vi[1]);
        if (bk == 1) {
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            if (rank == 0) mbar_arrive(&sh.acc_empty[acc]);
            else remote_arrive(acc_empty0 + (uint32_t)(acc * sizeof(uint64_t)));
          }
        }
        if (lane == 0) bulk_wait_read_all();
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int hh = c / 4, q = (c % 4) * 4;
          const int off = lane * 32 + ((c ^ sw) * 4);
          *reinterpret_cast<float4*>(bre + off) =
              make_float4(-vr[hh][q], -vr[hh][q + 1], -vr[hh][q + 2], -vr[hh][q + 3]);
          *reinterpret_cast<float4*>(bim + off) =
              make_float4(-vi[hh][q], -vi[hh][q + 1], -vi[hh][q + 2], -vi[hh][q + 3]);
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          const int x = half * 64 + bk * 32;
          const int y = (int)(row0 + quarter * 32);
          tma_reduce_add_2d(&tmap_c, bre, x, y);
          tma_reduce_add_2d(&tmap_c, bim, x, y + kT);
          bulk_commit();
        }
      }
      if (++acc == 2) { acc = 0; acc_phase ^= 1; }
    }
    if (lane == 0) bulk_wait_all();
    __syncwarp();
  }
  // Every role has left its loop.  After a failure the even CTA's producer
  // waits (bounded) until each stage it filled has both CTAs' bytes, and its
  // MMA issuer until its MMAs are done.  The odd CTA cannot observe its own
  // loads (they count on the even CTA's barrier); after a failure it pauses
  // (bounded, ~0.2 ms) so that any load of a stage the even CTA never
  // accounted lands first.  Then both CTAs meet before TMEM is freed (the
  // even CTA's MMAs write the odd CTA's TMEM and the odd CTA's loads and
  // epilogue signal the even CTA's barriers).
  __syncthreads();
  if (sh.failed) {
    if (warp == kEpiWarps && lane == 0 && rank == 0)
      for (int s = 0; s < kStages; ++s)
        if (filled & (1u << s)) mbar_wait_cl(&sh.full[s], (fill_parity >> s) & 1u, kTcWaitLimit);
    if (warp == kEpiWarps && lane == 0 && rank == 1 && filled)
      for (int i = 0; i < 200; ++i) __nanosleep(1000);
    if (warp == kEpiWarps + 1 && lane == 0 && rank == 0 && issued) {
      umma2_commit_local(&sh.drain);
      mbar_wait(&sh.drain, 0);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

}  // namespace

size_t schur_pair_smem() { return sizeof(PairShared) + 1024; }
static_assert(sizeof(PairShared) + 1024 <= 232448, "shared memory budget");

int schur_pair_launch(const int32_t* d_list, int64_t n_pairs, int n_pencils, int64_t n_slots,
                      unsigned char* staging, int64_t staging_bytes, int64_t buf0_bytes,
                      int64_t buf1_bytes, int64_t pencil_stride, int32_t* status, int* claim,
                      const CUtensorMap& tmap_c, int ctas, cudaStream_t st, char* err,
                      size_t cap) {
  if (n_pairs <= 0) return 0;
  if (n_pairs * (int64_t)n_pencils > INT32_MAX)
    return set_error(err, cap, AOSB_ERR_SIZE, "too many Schur pairs x pencils in one launch");
  if ((buf0_bytes | buf1_bytes | pencil_stride | staging_bytes) % 4096 != 0)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "staging offsets must be 4 KB multiples");
  const size_t smem = schur_pair_smem();
  static std::atomic<uint64_t> attr_devices{0};
  int device = 0;
  cudaGetDevice(&device);
  const uint64_t dev_bit = device < 64 ? (uint64_t)1 << device : 0;
  if (dev_bit == 0 || (attr_devices.load() & dev_bit) == 0) {
    cudaError_t e = cudaFuncSetAttribute(schur_pair_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
      return set_error(err, cap, AOSB_ERR_CUDA, "schur_pair smem attribute: %s",
                       cudaGetErrorString(e));
    attr_devices.fetch_or(dev_bit);
  }
  CUtensorMap tm_a, tm_b;
  const uint64_t planes = (uint64_t)staging_bytes / 4096;
  if (int rc = encode_staging_5d(staging, planes, false, &tm_a, err, cap)) return rc;
  if (int rc = encode_staging_5d(staging, planes, true, &tm_b, err, cap)) return rc;
  const int64_t items = n_pairs * n_pencils;
  int clusters = ctas / 2;
  if (clusters < 1) clusters = 1;
  if (claim == nullptr && items < clusters) clusters = (int)items;
  schur_pair_kernel<<<2 * clusters, kThreads, smem, st>>>(
      d_list, (int)n_pairs, n_pencils, n_slots, buf0_bytes / 4096, buf1_bytes / 4096,
      pencil_stride / 4096, status, claim, tm_a, tm_b, tmap_c, tc_wait_limit());
  count_launches(1);
  return 0;
}

}  // namespace aosb
