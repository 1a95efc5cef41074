// Inline-PTX helpers of the tcgen05 kernels (sm_100a): mbarriers with
// bounded waits, bulk copies, UMMA shared-memory and instruction
// descriptors, tcgen05.mma / commit / ld, and TMA tensor stores and
// reduce-adds.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace aosb {

// FP32 [rows][inner] tensor map with (box_x, box_y) boxes (tma_map.cu).
int encode_f32_2d(void* base, uint64_t inner, uint64_t rows, uint32_t box_x, uint32_t box_y,
                  bool swizzle128, CUtensorMap* map, char* err, size_t cap);

// BF16 view of the split-BF16 staging buffer for the two-CTA Schur update:
// [plane_slabs][2 K halves][2 operand-row halves][8 rows][64 elements]; a
// box is one 16 KB A slab (four planes, both row halves) or, with half_b,
// one 8 KB half of a B slab (four planes, one row half) (tma_map.cu).
int encode_staging_5d(void* base, uint64_t plane_slabs, bool half_b, CUtensorMap* map, char* err,
                      size_t cap);

namespace tc {

// Polls (with backoff) of one mbarrier wait before it gives up: the default
// of the process-wide limit the kernels are launched with
// (aosb_tc_set_wait_limit), and the fixed bound of the drain waits a CTA
// makes on its own copies and MMAs after a failure.
constexpr long long kTcWaitLimit = 1ll << 22;

// Current process-wide wait limit (factor_tc.cu).
long long tc_wait_limit();

// B operand of the tensor-core solve update: one 32-column RHS strip of a
// step's diagonal result Y (K = 128 rows) as four BF16 planes (re_hi,
// re_lo, im_hi, im_lo), K-major no-swizzle core matrices, 16-wide K slabs.
constexpr int kSolveNS = 32;
constexpr int kSolveBPlaneSlab = kSolveNS * 16 * 2;  // 1024 bytes
constexpr int kSolveBSlab = 4 * kSolveBPlaneSlab;     // 4096 bytes
constexpr int kSolveBBytes = 8 * kSolveBSlab;         // 32 KB per strip
__host__ __device__ __forceinline__ uint32_t solve_b_offset(int n, int k, int plane) {
  const int slab = k / 16, kk = k % 16;
  return (uint32_t)(slab * kSolveBSlab + plane * kSolveBPlaneSlab + (kk / 8) * ((kSolveNS / 8) * 128) +
                    (n / 8) * 128 + (n % 8) * 16 + (kk % 8) * 2);
}

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

// Bounded wait on phase `parity` (at most `limit` polls); returns false on
// timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          long long limit = kTcWaitLimit) {
  const uint32_t addr = smem_u32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 4096) __nanosleep(64);   // spin first: pipeline handoffs are sub-microsecond
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

// Instruction descriptor: BF16 x BF16 -> F32, K-major A and B, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_mn(int m, int n, bool negate_a) {
  return (1u << 4)                    // D format F32
         | (1u << 7)                  // A format BF16
         | (1u << 10)                 // B format BF16
         | ((negate_a ? 1u : 0u) << 13)
         | ((uint32_t)(n >> 3) << 17)   // N / 8
         | ((uint32_t)(m >> 4) << 24);  // M / 16
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

// smem tile = global box at (x, y); completion counted on `bar` (bytes).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// C[box at (x, y)] += smem tile (FP32 add in L2), one bulk group per commit.
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, const void* src, int x,
                                                  int y) {
  asm volatile(
      "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(smem_u32(src)), "r"(x), "r"(y)
      : "memory");
}
// C[box at (x, y)] = smem tile.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

}  // namespace tc
}  // namespace aosb
