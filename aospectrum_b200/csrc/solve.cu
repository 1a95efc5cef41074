// Block-RHS triangular solves with the tile factors, plus the gather /
// scatter between the original dof order (complex128) and the permuted,
// padded solver order (complex64), and the FP64 shifted residual used by
// iterative refinement.
//
// With P A = L U (P block diagonal, one permutation per tile row):
//   A X = B    forward  y_k = inv(L_kk) P_k (b_k - sum_{j<k} L_kj y_j)
//              backward x_k = inv(U_kk) (y_k - sum_{j>k} U_kj x_j)
//   A^H X = B  forward  w_k = inv(U_kk)^H (b_k - sum_{j<k} U_jk^H w_j)
//              backward x_k = P_k^T inv(L_kk)^H (w_k - sum_{j>k} L_jk^H x_j)
// (the stored L_kj, j < k, are in the row order of tile row k before its
// own pivoting, which is why P_k is applied after the accumulation.)
// Each sweep is right-looking: a diagonal kernel per step, then an update
// kernel for every off-diagonal tile of that step.
#include "plan.h"
#include "cgemm.cuh"
#include "tc_common.cuh"
#include "timing.h"

#include <cuda_bf16.h>

#include <atomic>
#include <mutex>
#include <vector>

namespace aosb {
int solve_graph(const aosb_plan* P, const aosb_solve_args_v1* a, char* err, size_t cap,
                int (*direct)(const aosb_plan*, const aosb_solve_args_v1*, char*, size_t));
int solve_tc_update(int k, int n, const int32_t* dtiles, const int32_t* dslots, int op, int np,
                    int nrhs, const aosb_plan* P, const float* factor, float2* work,
                    const float2* ytmp, const unsigned char* ystaged, int32_t* status,
                    cudaStream_t st, char* err, size_t cap, int copy_y);

// 1: the tensor-core sweeps run the next step's diagonal solve on a side
// stream beside the current step's remaining updates; process-wide.
std::atomic<int> g_solve_lookahead{0};

// Scratch block of aosb_solve: a status word per pencil (tensor-core
// updates), the diagonal result Y [np][T][L] complex64 and, for tile 128,
// Y as BF16 B-operand planes [np][strips][32 KB]; the tensor-core path
// keeps two of each (the lookahead writes step k+1's while step k's is
// read).  Each part starts on a 256-byte boundary.
struct ScratchLayout {
  int32_t* status = nullptr;
  float2* y[2] = {nullptr, nullptr};
  unsigned char* ystaged[2] = {nullptr, nullptr};
  size_t bytes = 0;
};
static ScratchLayout scratch_layout(const aosb_plan* P, int np, int nrhs, void* base) {
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  ScratchLayout l;
  unsigned char* p = (unsigned char*)base;
  size_t off = 0;
  l.status = (int32_t*)(p + off);
  off = up(off + (size_t)np * sizeof(int32_t));
  const size_t ybytes = up((size_t)np * P->T * nrhs * sizeof(float2));
  const int copies = P->T == 128 ? 2 : 1;
  for (int c = 0; c < copies; ++c) {
    l.y[c] = (float2*)(p + off);
    off += ybytes;
  }
  if (P->T == 128) {
    const size_t strips = (size_t)((nrhs + tc::kSolveNS - 1) / tc::kSolveNS);
    const size_t sb = up((size_t)np * strips * tc::kSolveBBytes);
    for (int c = 0; c < 2; ++c) {
      l.ystaged[c] = p + off;
      off += sb;
    }
  }
  l.bytes = off;
  return l;
}

// Side stream of a caller stream for the solve lookahead (created once,
// non-blocking, kept for the life of the process).
static int solve_side_stream(cudaStream_t main, cudaStream_t* out, char* err, size_t cap) {
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

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ size_t tile_base(int64_t p, int64_t n_slots, int64_t slot, int T) {
  return ((size_t)p * (size_t)n_slots + (size_t)slot) * (size_t)(2 * T * T);
}

enum DiagOp { kLinv = 0, kUinv = 1, kUinvH = 2, kLinvH = 3 };

constexpr int kCopyBlocks = 4;  // CTAs that copy the diagonal result back

// Diagonal step, out of place: Y = op(D_kk) X_k, one CTA per (32-column
// strip, 32-row block, pencil).  kLinv gathers rows of X_k through P_k;
// kLinvH stores row r of the product at row P_k[r] (x_k = P_k^T v_k).
// Y is a per-pencil T x n_rhs scratch block; the update launch of the same
// step copies it back into X_k.
template <int T, int OP>
__global__ void __launch_bounds__(kThreads) solve_diag_kernel(int k, int nrhs, int64_t n_pad,
                                                              const int32_t* __restrict__ diag_slot,
                                                              int64_t n_slots,
                                                              const float* __restrict__ factor,
                                                              const int32_t* __restrict__ pivots,
                                                              const float2* __restrict__ work,
                                                              float2* __restrict__ ytmp,
                                                              unsigned char* __restrict__ ystaged) {
  constexpr int BM = 32, BN = 32, TM = 2, TN = 2;
  static_assert((BM / TM) * (BN / TN) == 256, "layout");
  __shared__ CgemmSmem<BM, BN> sm[2];
  const int p = blockIdx.z;
  const int c0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  const float* D = factor + tile_base(p, n_slots, diag_slot[k], T);
  const int32_t* pv = pivots + (size_t)p * n_pad + (size_t)k * T;
  const float2* X = work + ((size_t)p * n_pad + (size_t)k * T) * nrhs;
  float2* Y = ytmp + (size_t)p * T * nrhs;
  float accr[TM][TN] = {}, acci[TM][TN] = {};
  auto la = [&](int m, int q) -> float2 {
    const int r = m0 + m;
    if (OP == kLinv) {
      if (q > r) return make_float2(0.f, 0.f);
      if (q == r) return make_float2(1.f, 0.f);
      const size_t o = (size_t)r * T + q;
      return make_float2(D[o], D[o + T * T]);
    } else if (OP == kUinv) {
      if (q < r) return make_float2(0.f, 0.f);
      const size_t o = (size_t)r * T + q;
      return make_float2(D[o], D[o + T * T]);
    } else if (OP == kUinvH) {  // conj(Uinv[q][r]), nonzero for q <= r
      if (q > r) return make_float2(0.f, 0.f);
      const size_t o = (size_t)q * T + r;
      return make_float2(D[o], -D[o + T * T]);
    } else {  // kLinvH: conj(Linv[q][r]), unit diagonal, nonzero for q >= r
      if (q < r) return make_float2(0.f, 0.f);
      if (q == r) return make_float2(1.f, 0.f);
      const size_t o = (size_t)q * T + r;
      return make_float2(D[o], -D[o + T * T]);
    }
  };
  auto lb = [&](int q, int c) -> float2 {
    const int col = c0 + c;
    if (col >= nrhs) return make_float2(0.f, 0.f);
    const int row = OP == kLinv ? pv[q] : q;
    return X[(size_t)row * nrhs + col];
  };
  cgemm_cta<BM, BN, TM, TN, (OP == kUinvH || OP == kLinvH)>(accr, acci, T, sm, la, lb);
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int r = m0 + cg_row<BM, BN, TM, TN>(i), col = c0 + cg_col<BM, BN, TM, TN>(j);
      if (col >= nrhs) continue;
      const int row = OP == kLinvH ? pv[r] : r;
      Y[(size_t)row * nrhs + col] = make_float2(accr[i][j], acci[i][j]);
      if (ystaged != nullptr) {
        // the same value as the tensor-core update's B operand (strip of 32
        // columns): four BF16 planes, x = hi + lo
        const int strips = (nrhs + tc::kSolveNS - 1) / tc::kSolveNS;
        unsigned char* sp = ystaged + ((size_t)p * strips + col / tc::kSolveNS) * tc::kSolveBBytes;
        const int n = col % tc::kSolveNS;
        const __nv_bfloat16 rh = __float2bfloat16_rn(accr[i][j]);
        const __nv_bfloat16 ih = __float2bfloat16_rn(acci[i][j]);
        *reinterpret_cast<__nv_bfloat16*>(sp + tc::solve_b_offset(n, row, 0)) = rh;
        *reinterpret_cast<__nv_bfloat16*>(sp + tc::solve_b_offset(n, row, 1)) =
            __float2bfloat16_rn(accr[i][j] - __bfloat162float(rh));
        *reinterpret_cast<__nv_bfloat16*>(sp + tc::solve_b_offset(n, row, 2)) = ih;
        *reinterpret_cast<__nv_bfloat16*>(sp + tc::solve_b_offset(n, row, 3)) =
            __float2bfloat16_rn(acci[i][j] - __bfloat162float(ih));
      }
    }
}

enum UpdOp { kPlain = 0, kConjT = 1 };

// Update step: X_i -= op(F_t) Y for the listed tiles, Y = the step's
// diagonal result.  blockIdx.x = (item, row block, column strip); the last
// `copy_blocks` CTAs copy Y into X_k.  op = plain tile or conjugate transpose.
template <int T, int OP>
__global__ void __launch_bounds__(kThreads) solve_update_kernel(
    int k, int n_items, int nrhs, int64_t n_pad, const int32_t* __restrict__ tiles,
    const int32_t* __restrict__ slots, int64_t n_slots, const float* __restrict__ factor,
    float2* __restrict__ work, const float2* __restrict__ ytmp) {
  constexpr int BM = T >= 64 ? 64 : 32;
  constexpr int BN = 32;
  constexpr int TM = BM == 64 ? 4 : 2, TN = 2;
  static_assert((BM / TM) * (BN / TN) == 256, "layout");
  constexpr int kRowBlocks = T / BM;
  __shared__ CgemmSmem<BM, BN> sm[2];
  const int p = blockIdx.y;
  const int ncs = (nrhs + BN - 1) / BN;
  const int work_blocks = n_items * kRowBlocks * ncs;
  const float2* Y = ytmp + (size_t)p * T * nrhs;
  if ((int)blockIdx.x >= work_blocks) {
    // copy-back CTAs
    const int cb = blockIdx.x - work_blocks;
    float2* Xk = work + ((size_t)p * n_pad + (size_t)k * T) * nrhs;
    const int total = T * nrhs;
    for (int e = cb * kThreads + threadIdx.x; e < total; e += kCopyBlocks * kThreads) Xk[e] = Y[e];
    return;
  }
  const int item = blockIdx.x / (kRowBlocks * ncs);
  const int rem = blockIdx.x % (kRowBlocks * ncs);
  const int m0 = (rem / ncs) * BM, c0 = (rem % ncs) * BN;
  const int i = tiles[item];
  const float* F = factor + tile_base(p, n_slots, slots[item], T);
  float2* Xi = work + ((size_t)p * n_pad + (size_t)i * T) * nrhs;
  float accr[TM][TN] = {}, acci[TM][TN] = {};
  auto la = [&](int m, int q) -> float2 {
    if (OP == kPlain) {
      const size_t o = (size_t)(m0 + m) * T + q;
      return make_float2(F[o], F[o + T * T]);
    } else {
      const size_t o = (size_t)q * T + (m0 + m);
      return make_float2(F[o], -F[o + T * T]);
    }
  };
  auto lb = [&](int q, int c) -> float2 {
    const int col = c0 + c;
    if (col >= nrhs) return make_float2(0.f, 0.f);
    return Y[(size_t)q * nrhs + col];
  };
  cgemm_cta<BM, BN, TM, TN, OP == kConjT>(accr, acci, T, sm, la, lb);
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) {
      const int r = m0 + cg_row<BM, BN, TM, TN>(a), col = c0 + cg_col<BM, BN, TM, TN>(b);
      if (col >= nrhs) continue;
      float2 v = Xi[(size_t)r * nrhs + col];
      v.x -= accr[a][b];
      v.y -= acci[a][b];
      Xi[(size_t)r * nrhs + col] = v;
    }
}

template <int T>
int run_solve(const aosb_plan* P, const aosb_solve_args_v1* a, char* err, size_t cap) {
  cudaStream_t st = (cudaStream_t)a->stream;
  const int np = a->n_pencils, L = a->n_rhs;
  const int ncs = (L + 31) / 32;
  constexpr int BM = T >= 64 ? 64 : 32;
  const int rowblocks = T / BM;
  float2* W = (float2*)a->work;
  const bool tc = T == 128 && (a->flags & AOSB_SOLVE_TENSOR_CORES) != 0;
  const ScratchLayout sl = scratch_layout(P, np, L, a->scratch);
  int32_t* tc_status = sl.status;
  auto diag = [&](int k, int op, int buf, cudaStream_t s) {
    count_launches(1);
    dim3 g(ncs, T / 32, np);
    cudaEvent_t ev[2];
    const bool timed = timing_begin(s, ev);
    float2* Y = sl.y[buf];
    unsigned char* ys = tc ? sl.ystaged[buf] : nullptr;
    switch (op) {
      case kLinv: solve_diag_kernel<T, kLinv><<<g, kThreads, 0, s>>>(k, L, P->n_pad, P->d_diag_slot, P->n_slots, a->factor, a->pivots, W, Y, ys); break;
      case kUinv: solve_diag_kernel<T, kUinv><<<g, kThreads, 0, s>>>(k, L, P->n_pad, P->d_diag_slot, P->n_slots, a->factor, a->pivots, W, Y, ys); break;
      case kUinvH: solve_diag_kernel<T, kUinvH><<<g, kThreads, 0, s>>>(k, L, P->n_pad, P->d_diag_slot, P->n_slots, a->factor, a->pivots, W, Y, ys); break;
      default: solve_diag_kernel<T, kLinvH><<<g, kThreads, 0, s>>>(k, L, P->n_pad, P->d_diag_slot, P->n_slots, a->factor, a->pivots, W, Y, ys); break;
    }
    // algorithmic: one triangular T x T tile times T x L per pencil
    if (timed)
      timing_end(kTimedSolveDiag, s, ev, 4.0 * T * T * L * np,
                 (double)np * (2.0 * T * T * sizeof(float) + 2.0 * T * L * sizeof(float2)));
  };
  if (tc) AOSB_CUDA_TRY(cudaMemsetAsync(tc_status, 0, (size_t)np * sizeof(int32_t), st), err, cap);
  int tc_rc = 0;
  // update of step k with the list entries [b, e) of off[k] .. off[k + 1]
  auto update = [&](int k, int64_t b, int64_t e, const int32_t* dtiles, const int32_t* dslots,
                    int op, int buf, bool copy) {
    const int n = (int)(e - b);
    if (tc && n == 0 && !copy) return;
    cudaEvent_t ev[2];
    const bool timed = timing_begin(st, ev);
    // algorithmic: n tiles x (T x T) x (T x L) complex per pencil; factor
    // tiles read once, X tiles read and written
    const double uflops = 8.0 * T * T * L * (double)n * np;
    const double ubytes = (double)n * np * (2.0 * T * T * sizeof(float) + 2.0 * T * L * sizeof(float2));
    if (tc) {
      if (tc_rc == 0)
        tc_rc = solve_tc_update(k, n, dtiles + b, dslots + b, op, np, L, P, a->factor, W,
                                sl.y[buf], sl.ystaged[buf], tc_status, st, err, cap, copy ? 1 : 0);
      if (timed) timing_end(kTimedSolveUpdate, st, ev, uflops, ubytes);
      return;
    }
    dim3 g((unsigned)(n * rowblocks * ncs + kCopyBlocks), np);
    count_launches(1);
    if (op == kPlain)
      solve_update_kernel<T, kPlain><<<g, kThreads, 0, st>>>(k, n, L, P->n_pad, dtiles + b, dslots + b, P->n_slots, a->factor, W, sl.y[buf]);
    else
      solve_update_kernel<T, kConjT><<<g, kThreads, 0, st>>>(k, n, L, P->n_pad, dtiles + b, dslots + b, P->n_slots, a->factor, W, sl.y[buf]);
    if (timed) timing_end(kTimedSolveUpdate, st, ev, uflops, ubytes);
  };
  const int nb = (int)P->nb;
  const bool lookahead = tc && g_solve_lookahead.load() != 0 && nb > 1;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_next = nullptr, ev_diag = nullptr;
  if (lookahead) {
    if (int rc = solve_side_stream(st, &side, err, cap)) return rc;
    AOSB_CUDA_TRY(cudaEventCreateWithFlags(&ev_next, cudaEventDisableTiming), err, cap);
    if (cudaEventCreateWithFlags(&ev_diag, cudaEventDisableTiming) != cudaSuccess) {
      cudaEventDestroy(ev_next);
      return set_error(err, cap, AOSB_ERR_CUDA, "cudaEventCreate failed");
    }
  }
  struct EventGuard {
    cudaEvent_t a, b;
    ~EventGuard() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } guard{ev_next, ev_diag};
  // One sweep over the steps in `order`: without lookahead, per step the
  // diagonal solve and then all updates.  With lookahead, step k first
  // updates the tile of the next step (the first list entry going forward,
  // the last going backward), then the next step's diagonal solve runs on
  // the side stream into the other Y buffer while the rest of step k's
  // updates (and the copy X_k = Y) run on the caller stream.
  auto sweep = [&](bool forward, const std::vector<int32_t>& off,
                   const std::vector<int32_t>& host_tiles, const int32_t* dtiles,
                   const int32_t* dslots, int dop, int uop) -> int {
    auto step_at = [&](int i) { return forward ? i : nb - 1 - i; };
    if (!lookahead) {
      for (int i = 0; i < nb; ++i) {
        const int k = step_at(i);
        diag(k, dop, 0, st);
        update(k, off[k], off[k + 1], dtiles, dslots, uop, 0, true);
      }
      return 0;
    }
    diag(step_at(0), dop, 0, st);
    for (int i = 0; i < nb; ++i) {
      const int k = step_at(i), buf = i & 1;
      const int64_t b = off[k], e = off[k + 1];
      int64_t nb0 = b, nb1 = b, rb = b, re = e;   // next-step entry [nb0, nb1), rest [rb, re)
      if (i + 1 < nb) {
        const int kn = step_at(i + 1);
        if (forward && e > b && host_tiles[b] == kn) { nb1 = b + 1; rb = b + 1; }
        if (!forward && e > b && host_tiles[e - 1] == kn) { nb0 = e - 1; nb1 = e; re = e - 1; }
        update(k, nb0, nb1, dtiles, dslots, uop, buf, false);
        AOSB_CUDA_TRY(cudaEventRecord(ev_next, st), err, cap);
        AOSB_CUDA_TRY(cudaStreamWaitEvent(side, ev_next, 0), err, cap);
        diag(kn, dop, buf ^ 1, side);
        AOSB_CUDA_TRY(cudaEventRecord(ev_diag, side), err, cap);
        update(k, rb, re, dtiles, dslots, uop, buf, true);
        AOSB_CUDA_TRY(cudaStreamWaitEvent(st, ev_diag, 0), err, cap);
      } else {
        update(k, b, e, dtiles, dslots, uop, buf, true);
      }
    }
    return 0;
  };
  int rc = 0;
  if (!a->adjoint) {
    rc = sweep(true, P->lb_off, P->lb_tile, P->d_lb_tile, P->d_lb_slot, kLinv, kPlain);
    if (rc == 0) rc = sweep(false, P->ua_off, P->ua_tile, P->d_ua_tile, P->d_ua_slot, kUinv, kPlain);
  } else {
    // forward: X_i -= U_ki^H w_k for U tiles (k, i), i > k; backward:
    // X_i -= L_ki^H x_k for L tiles (k, i), i < k
    rc = sweep(true, P->ur_off, P->ur_tile, P->d_ur_tile, P->d_ur_slot, kUinvH, kConjT);
    if (rc == 0) rc = sweep(false, P->ll_off, P->ll_tile, P->d_ll_tile, P->d_ll_slot, kLinvH, kConjT);
  }
  if (rc) return rc;
  if (tc_rc) return tc_rc;
  return launch_check(err, cap, "solve");
}

__global__ void gather_rhs_kernel(int64_t n_pad, int nrhs, const int32_t* __restrict__ perm,
                                  const double2* __restrict__ src, int64_t src_stride,
                                  float2* __restrict__ work) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.y;
  if (idx >= n_pad * nrhs) return;
  const int64_t i = idx / nrhs, c = idx - (idx / nrhs) * nrhs;
  const int32_t o = perm[i];
  float2 v = make_float2(0.f, 0.f);
  if (o >= 0) {
    const double2 s = src[(size_t)p * src_stride + (size_t)o * nrhs + c];
    v = make_float2((float)s.x, (float)s.y);
  }
  work[((size_t)p * n_pad) * nrhs + idx] = v;
}

__global__ void scatter_solution_kernel(int64_t n, int64_t n_pad, int nrhs,
                                        const int32_t* __restrict__ pinv,
                                        const float2* __restrict__ work, double2* __restrict__ x,
                                        int accumulate) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.y;
  if (idx >= n * nrhs) return;
  const int64_t j = idx / nrhs, c = idx - (idx / nrhs) * nrhs;
  const float2 w = work[((size_t)p * n_pad + pinv[j]) * nrhs + c];
  double2* o = x + (size_t)p * n * nrhs + idx;
  if (accumulate) {
    double2 v = *o;
    v.x += (double)w.x;
    v.y += (double)w.y;
    *o = v;
  } else {
    *o = make_double2((double)w.x, (double)w.y);
  }
}

// r = b - (H - z S) x, one warp per row, lanes over right-hand sides.
__global__ void shifted_residual_kernel(int64_t n, int nrhs, const int64_t* __restrict__ indptr,
                                        const int32_t* __restrict__ indices,
                                        const float2* __restrict__ hv,
                                        const float2* __restrict__ sv, int64_t nnz,
                                        const int32_t* __restrict__ pencil_k,
                                        const double2* __restrict__ shifts,
                                        const double2* __restrict__ b, int64_t b_stride,
                                        const double2* __restrict__ x, double2* __restrict__ r) {
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.y;
  if (row >= n) return;
  const int64_t kp = pencil_k[p];
  const double2 z = shifts[p];
  const float2* h = hv + kp * nnz;
  const float2* s = sv != nullptr ? sv + kp * nnz : nullptr;
  const double2* xp = x + (size_t)p * n * nrhs;
  for (int c0 = 0; c0 < nrhs; c0 += 32) {
    const int c = c0 + lane;
    double hr = 0, hi = 0, sr = 0, si = 0;
    if (c < nrhs) {
      for (int64_t e = indptr[row]; e < indptr[row + 1]; ++e) {
        const int64_t col = indices[e];
        const float2 hh = h[e];
        const float2 ss = s != nullptr ? s[e] : make_float2(0.f, 0.f);
        const double2 xv = xp[(size_t)col * nrhs + c];
        hr += (double)hh.x * xv.x - (double)hh.y * xv.y;
        hi += (double)hh.x * xv.y + (double)hh.y * xv.x;
        sr += (double)ss.x * xv.x - (double)ss.y * xv.y;
        si += (double)ss.x * xv.y + (double)ss.y * xv.x;
      }
      // A x = H x - z (S x)
      const double ar = hr - (z.x * sr - z.y * si);
      const double ai = hi - (z.x * si + z.y * sr);
      const double2 bv = b[(size_t)p * b_stride + (size_t)row * nrhs + c];
      r[((size_t)p * n + row) * nrhs + c] = make_double2(bv.x - ar, bv.y - ai);
    }
  }
}

// Row-block kernels: rows [rb[b], rb[b+1]) share one column pattern (the
// rows of one atom) and are stored one after another with equal lengths.
// One CTA of kResWarps warps per (block, 32-column strip, pencil), pencils
// fastest; the warps split the block's nonzeros.  Per chunk of 32 nonzeros each lane forms the
// FP64 matrix entries of one nonzero for every row of the block into shared
// memory (so A is converted once, not once per lane); then every lane walks
// the chunk, loading each x row once for all rows of the block, with the
// loads of the next kXRows x rows issued before the products of the current
// ones.  Partial sums of the warps are added in shared memory.
//
// kResidual: A = H(k_p) - z_p S(k_p) and y[p] = b[p] - A x[p] (FP64 residual
// of every pencil of a batch).  Otherwise A = the single complex64 value
// array and y = A x (the CISS products S Y, H B, S B).
constexpr int kResWarps = 4;
constexpr int kXRows = 4;

struct RowBlockArgs {
  int np;  // pencils (1 for the product)
  int64_t n_blocks;
  const int32_t* rb;
  int ncols;
  const int64_t* indptr;
  const int32_t* indices;
  const float2* hv;  // residual: H values [k][nnz]; product: A values [nnz]
  const float2* sv;  // residual: S values [k][nnz] or null
  int64_t nnz;
  const int32_t* pencil_k;
  const double2* shifts;
  const double2* b;  // residual: b[p * b_stride + row * ldy + c]
  int64_t b_stride;
  const double2* x;  // x[p * x_stride + col * ldx + c]
  int64_t ldx, x_stride;
  double2* y;        // y[p * y_stride + row * ldy + c]
  int64_t ldy, y_stride;
};

template <int R, bool kResidual>
__global__ void __launch_bounds__(kResWarps * 32, 4) row_block_kernel(const RowBlockArgs a) {
  __shared__ double2 as[kResWarps][R][32];
  __shared__ int32_t cs[kResWarps][32];
  // CTA index = (block, strip) * np + pencil: the CTAs of all pencils of one
  // row block run together and share its H, S values in L2
  const int ncs = (a.ncols + 31) / 32;
  const int p = (int)(blockIdx.x % a.np);
  const int64_t bs = blockIdx.x / a.np;
  const int64_t blk = bs / ncs;
  const int c = (int)(bs % ncs) * 32 + (threadIdx.x & 31);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (blk >= a.n_blocks) return;
  const int r0 = a.rb[blk], nr = a.rb[blk + 1] - a.rb[blk];
  const int nq = nr < R ? nr : R;
  const float2* h = a.hv;
  const float2* s = nullptr;
  double2 z = make_double2(0.0, 0.0);
  if (kResidual) {
    const int64_t kp = a.pencil_k[p];
    z = a.shifts[p];
    h = a.hv + kp * a.nnz;
    s = a.sv != nullptr ? a.sv + kp * a.nnz : nullptr;
  }
  const double2* xp = a.x + (size_t)p * a.x_stride;
  const bool active = c < a.ncols;
  // row q of the block starts at base0 + q * len
  const int64_t base0 = a.indptr[r0];
  const int64_t len = a.indptr[r0 + 1] - base0;
  const int64_t per = (len + kResWarps - 1) / kResWarps;
  const int64_t w0 = (int64_t)warp * per;
  const int64_t w1 = w0 + per < len ? w0 + per : len;
  double ar[R], ai[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    ar[q] = 0.0;
    ai[q] = 0.0;
  }
  for (int64_t e0 = w0; e0 < w1; e0 += 32) {
    const int cnt = (int)(w1 - e0 < 32 ? w1 - e0 : 32);
    if (lane < cnt) {
      cs[warp][lane] = a.indices[base0 + e0 + lane];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        double2 v = make_double2(0.0, 0.0);  // rows past the block add nothing
        if (q < nq) {
          const int64_t at = base0 + (int64_t)q * len + e0 + lane;
          const float2 hh = h[at];
          if (kResidual) {
            const float2 ss = s != nullptr ? s[at] : make_float2(0.f, 0.f);
            v = make_double2((double)hh.x - (z.x * ss.x - z.y * ss.y),
                             (double)hh.y - (z.x * ss.y + z.y * ss.x));
          } else {
            v = make_double2((double)hh.x, (double)hh.y);
          }
        }
        as[warp][q][lane] = v;
      }
    }
    __syncwarp();
    double2 xa[kXRows], xb[kXRows];
    auto load = [&](double2(&buf)[kXRows], int j) {
#pragma unroll
      for (int u = 0; u < kXRows; ++u)
        buf[u] = (j + u < cnt && active) ? xp[(size_t)cs[warp][j + u] * a.ldx + c]
                                         : make_double2(0.0, 0.0);
    };
    auto madd = [&](const double2(&buf)[kXRows], int j) {
#pragma unroll
      for (int u = 0; u < kXRows; ++u) {
        if (j + u >= cnt) break;
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const double2 m = as[warp][q][j + u];
          // four FMAs per complex product (no separate multiply and add)
          ar[q] = fma(m.x, buf[u].x, ar[q]);
          ar[q] = fma(-m.y, buf[u].y, ar[q]);
          ai[q] = fma(m.x, buf[u].y, ai[q]);
          ai[q] = fma(m.y, buf[u].x, ai[q]);
        }
      }
    };
    load(xa, 0);
    for (int j0 = 0; j0 < cnt; j0 += 2 * kXRows) {
      load(xb, j0 + kXRows);
      madd(xa, j0);
      load(xa, j0 + 2 * kXRows);
      madd(xb, j0 + kXRows);
    }
    __syncwarp();
  }
  // cross-warp sum: reuse `as` as [warp][row][lane]
  __syncthreads();
#pragma unroll
  for (int q = 0; q < R; ++q) as[warp][q][lane] = make_double2(ar[q], ai[q]);
  __syncthreads();
  if (!active) return;
  for (int q = warp; q < nr; q += kResWarps) {
    const int64_t row = r0 + q;
    double2* out = a.y + (size_t)p * a.y_stride + (size_t)row * a.ldy + c;
    if (q >= R) {
      // blocks longer than R break the launch contract: poison those rows
      *out = make_double2(__longlong_as_double(0x7ff8000000000000ll),
                          __longlong_as_double(0x7ff8000000000000ll));
      continue;
    }
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int w = 0; w < kResWarps; ++w) {
      sr += as[w][q][lane].x;
      si += as[w][q][lane].y;
    }
    if (kResidual) {
      const double2 bv = a.b[(size_t)p * a.b_stride + (size_t)row * a.ldy + c];
      *out = make_double2(bv.x - sr, bv.y - si);
    } else {
      *out = make_double2(sr, si);
    }
  }
}

// Launches row_block_kernel with the smallest row count R >= max_rows.
template <bool kResidual>
int launch_row_blocks(const RowBlockArgs& a, int max_rows, int np, cudaStream_t st, char* err,
                      size_t cap) {
  const int ncs = (a.ncols + 31) / 32;
  if (a.n_blocks * ncs * np > INT32_MAX)
    return set_error(err, cap, AOSB_ERR_SIZE, "too many row blocks x pencils");
  if (max_rows < 1 || max_rows > 16)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "max_block_rows must be in 1..16");
  if (a.np != np) return set_error(err, cap, AOSB_ERR_ARGUMENT, "pencil count mismatch");
  dim3 g((unsigned)(a.n_blocks * ncs * np));
  const int th = kResWarps * 32;
  if (max_rows <= 4)
    row_block_kernel<4, kResidual><<<g, th, 0, st>>>(a);
  else if (max_rows <= 8)
    row_block_kernel<8, kResidual><<<g, th, 0, st>>>(a);
  else if (max_rows <= 13)
    row_block_kernel<13, kResidual><<<g, th, 0, st>>>(a);
  else
    row_block_kernel<16, kResidual><<<g, th, 0, st>>>(a);
  count_launches(1);
  return 0;
}

}  // namespace

// CUDA-graph replay of whole solves.  The launch sequence of one aosb_solve
// (a diagonal and an update launch per tile step and sweep) depends only on
// the plan, the batch shape, the flags and the buffer addresses, so it is
// captured once per such key and replayed with cudaGraphLaunch afterwards.
// Graphs referring to a plan are dropped when the plan is destroyed.
struct SolveGraphKey {
  const aosb_plan* P;
  int device, np, L, adjoint, flags;
  const void *factor, *pivots, *work, *scratch;
  bool operator==(const SolveGraphKey& o) const {
    return P == o.P && device == o.device && np == o.np && L == o.L && adjoint == o.adjoint &&
           flags == o.flags && factor == o.factor && pivots == o.pivots && work == o.work &&
           scratch == o.scratch;
  }
};
struct SolveGraph {
  SolveGraphKey key;
  cudaGraphExec_t exec;
  size_t kernels;
  uint64_t last_use;
};
static std::mutex g_graph_mu;
static std::vector<SolveGraph> g_graphs;
static uint64_t g_graph_clock = 0;
constexpr size_t kMaxSolveGraphs = 32;

void solve_graphs_forget(const aosb_plan* P) {
  std::lock_guard<std::mutex> lock(g_graph_mu);
  for (size_t i = 0; i < g_graphs.size();) {
    if (g_graphs[i].key.P == P) {
      cudaGraphExecDestroy(g_graphs[i].exec);
      g_graphs[i] = g_graphs.back();
      g_graphs.pop_back();
    } else {
      ++i;
    }
  }
}

int solve_graph(const aosb_plan* P, const aosb_solve_args_v1* a, char* err, size_t cap,
                int (*direct)(const aosb_plan*, const aosb_solve_args_v1*, char*, size_t)) {
  cudaStream_t st = (cudaStream_t)a->stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  AOSB_CUDA_TRY(cudaStreamIsCapturing(st, &cs), err, cap);
  if (cs != cudaStreamCaptureStatusNone || st == nullptr) return direct(P, a, err, cap);
  int device = 0;
  AOSB_CUDA_TRY(cudaGetDevice(&device), err, cap);
  const SolveGraphKey key{P, device, a->n_pencils, a->n_rhs, a->adjoint, a->flags,
                          a->factor, a->pivots, a->work, a->scratch};
  {
    std::lock_guard<std::mutex> lock(g_graph_mu);
    for (auto& g : g_graphs) {
      if (g.key == key) {
        g.last_use = ++g_graph_clock;
        AOSB_CUDA_TRY(cudaGraphLaunch(g.exec, st), err, cap);
        count_launches(g.kernels);
        return 0;
      }
    }
  }
  // capture (thread-local mode: other threads keep issuing CUDA calls)
  AOSB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), err, cap);
  const int rc = direct(P, a, err, cap);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (rc != 0) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess)
    return set_error(err, cap, AOSB_ERR_CUDA, "solve capture failed: %s", cudaGetErrorString(e));
  size_t nodes = 0;
  cudaGraphGetNodes(graph, nullptr, &nodes);
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess)
    return set_error(err, cap, AOSB_ERR_CUDA, "solve graph instantiate: %s", cudaGetErrorString(ei));
  AOSB_CUDA_TRY(cudaGraphLaunch(exec, st), err, cap);
  std::lock_guard<std::mutex> lock(g_graph_mu);
  if (g_graphs.size() >= kMaxSolveGraphs) {
    size_t old = 0;
    for (size_t i = 1; i < g_graphs.size(); ++i)
      if (g_graphs[i].last_use < g_graphs[old].last_use) old = i;
    cudaGraphExecDestroy(g_graphs[old].exec);
    g_graphs[old] = g_graphs.back();
    g_graphs.pop_back();
  }
  g_graphs.push_back({key, exec, nodes, ++g_graph_clock});
  return 0;
}

}  // namespace aosb

extern "C" {

size_t aosb_solve_scratch_bytes(const aosb_plan_t* P, int32_t np, int32_t nrhs) {
  if (P == nullptr || np <= 0 || nrhs <= 0) return 0;
  return aosb::scratch_layout(P, np, nrhs, nullptr).bytes;
}

int aosb_solve_check(const aosb_plan_t* P, const aosb_solve_args_v1* a, char* err, size_t cap) {
  using aosb::set_error;
  if (P == nullptr || a == nullptr || a->scratch == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (a->n_pencils <= 0 || a->n_pencils > 65535 || a->n_rhs <= 0)
    return set_error(err, cap, AOSB_ERR_BATCH, "invalid pencil or right-hand-side count");
  cudaStream_t st = (cudaStream_t)a->stream;
  AOSB_CUDA_TRY(cudaStreamSynchronize(st), err, cap);
  if (P->T != 128 || (a->flags & AOSB_SOLVE_TENSOR_CORES) == 0) return 0;
  std::vector<int32_t> host((size_t)a->n_pencils);
  const int32_t* words = aosb::scratch_layout(P, a->n_pencils, a->n_rhs, a->scratch).status;
  AOSB_CUDA_TRY(cudaMemcpy(host.data(), words, host.size() * sizeof(int32_t),
                           cudaMemcpyDeviceToHost), err, cap);
  for (size_t i = 0; i < host.size(); ++i)
    if (host[i] != 0)
      return set_error(err, cap, host[i], "tensor-core solve update of pencil %zu gave up a bounded "
                       "wait (status %d)", i, host[i]);
  return 0;
}

static int solve_direct(const aosb_plan_t* P, const aosb_solve_args_v1* a, char* err, size_t cap) {
  switch (P->T) {
    case 32: return aosb::run_solve<32>(P, a, err, cap);
    case 64: return aosb::run_solve<64>(P, a, err, cap);
    case 128: return aosb::run_solve<128>(P, a, err, cap);
  }
  return aosb::set_error(err, cap, AOSB_ERR_UNSUPPORTED, "unsupported tile size");
}

int aosb_solve(const aosb_plan_t* P, const aosb_solve_args_v1* a, char* err, size_t cap) {
  using aosb::set_error;
  if (P == nullptr || a == nullptr) return set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (a->abi_version != AOSPECTRUM_B200_ABI_VERSION || a->struct_size != sizeof(*a))
    return set_error(err, cap, AOSB_ERR_ABI, "solve args ABI mismatch");
  if (a->n_pencils <= 0 || a->n_pencils > 65535 || a->n_rhs <= 0 || a->n_rhs > 256)
    return set_error(err, cap, AOSB_ERR_BATCH, "invalid pencil or right-hand-side count");
  if (a->factor == nullptr || a->pivots == nullptr || a->work == nullptr || a->scratch == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "required pointer is null");
  if (!P->uploaded) return set_error(err, cap, AOSB_ERR_ARGUMENT, "call aosb_plan_upload first");
  if ((a->flags & AOSB_SOLVE_GRAPH) == 0) return solve_direct(P, a, err, cap);
  return aosb::solve_graph(P, a, err, cap, solve_direct);
}

int aosb_gather_rhs(const aosb_plan_t* P, int32_t np, int32_t nrhs, const aosb_complex128* src,
                    int64_t src_stride, aosb_complex64* work, void* stream, char* err, size_t cap) {
  if (P == nullptr || src == nullptr || work == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (!P->uploaded) return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "plan not uploaded");
  if (np <= 0 || np > 65535 || nrhs <= 0)
    return aosb::set_error(err, cap, AOSB_ERR_BATCH, "invalid batch");
  dim3 g(aosb::ceil_div(P->n_pad * nrhs, 256), np);
  aosb::gather_rhs_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(
      P->n_pad, nrhs, P->d_perm, (const double2*)src, src_stride, (float2*)work);
  aosb::count_launches(1);
  return aosb::launch_check(err, cap, "gather_rhs");
}

int aosb_scatter_solution(const aosb_plan_t* P, int32_t np, int32_t nrhs,
                          const aosb_complex64* work, aosb_complex128* x, int32_t accumulate,
                          void* stream, char* err, size_t cap) {
  if (P == nullptr || work == nullptr || x == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (!P->uploaded) return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "plan not uploaded");
  if (np <= 0 || np > 65535 || nrhs <= 0)
    return aosb::set_error(err, cap, AOSB_ERR_BATCH, "invalid batch");
  dim3 g(aosb::ceil_div(P->n * nrhs, 256), np);
  aosb::scatter_solution_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(
      P->n, P->n_pad, nrhs, P->d_pinv, (const float2*)work, (double2*)x, accumulate);
  aosb::count_launches(1);
  return aosb::launch_check(err, cap, "scatter_solution");
}

int aosb_shifted_residual_blocks(int64_t n, int32_t nrhs, int32_t np, int64_t n_blocks,
                                 const int32_t* row_blocks, int32_t max_block_rows,
                                 const int64_t* indptr, const int32_t* indices,
                                 const aosb_complex64* h_values, const aosb_complex64* s_values,
                                 int64_t nnz, const int32_t* pencil_k,
                                 const aosb_complex128* shifts, const aosb_complex128* b,
                                 int64_t b_stride, const aosb_complex128* x, aosb_complex128* r,
                                 void* stream, char* err, size_t cap) {
  if (row_blocks == nullptr || indptr == nullptr || indices == nullptr || h_values == nullptr ||
      pencil_k == nullptr || shifts == nullptr || b == nullptr || x == nullptr || r == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (np <= 0 || np > 65535 || nrhs <= 0 || n <= 0 || n_blocks <= 0)
    return aosb::set_error(err, cap, AOSB_ERR_BATCH, "invalid batch");
  aosb::RowBlockArgs a{np, n_blocks, row_blocks, nrhs, indptr, indices, (const float2*)h_values,
                       (const float2*)s_values, nnz, pencil_k, (const double2*)shifts,
                       (const double2*)b, b_stride, (const double2*)x, nrhs, n * nrhs,
                       (double2*)r, nrhs, n * nrhs};
  cudaEvent_t ev[2];
  const bool timed = aosb::timing_begin((cudaStream_t)stream, ev);
  int rc = aosb::launch_row_blocks<true>(a, max_block_rows, np, (cudaStream_t)stream, err, cap);
  if (rc) return rc;
  // algorithmic: 8 FP64 flops per (nonzero, column, pencil); H and S values
  // once per k, x read and r written once per pencil
  if (timed)
    aosb::timing_end(aosb::kTimedResidual, (cudaStream_t)stream, ev, 8.0 * nnz * nrhs * np,
                     16.0 * nnz + (double)np * n * nrhs * 16.0 * 3.0);
  return aosb::launch_check(err, cap, "shifted_residual_blocks");
}

int aosb_spmm_blocks(int64_t n, int32_t ncols, int64_t n_blocks, const int32_t* row_blocks,
                     int32_t max_block_rows, const int64_t* indptr, const int32_t* indices,
                     const aosb_complex64* values, int64_t nnz, const aosb_complex128* x,
                     int64_t ldx, aosb_complex128* y, int64_t ldy, void* stream, char* err,
                     size_t cap) {
  if (row_blocks == nullptr || indptr == nullptr || indices == nullptr || values == nullptr ||
      x == nullptr || y == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (n <= 0 || ncols <= 0 || n_blocks <= 0 || ldx < ncols || ldy < ncols)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "invalid spmm shape");
  aosb::RowBlockArgs a{1, n_blocks, row_blocks, ncols, indptr, indices, (const float2*)values,
                       nullptr, nnz, nullptr, nullptr, nullptr, 0, (const double2*)x, ldx, 0,
                       (double2*)y, ldy, 0};
  cudaEvent_t ev[2];
  const bool timed = aosb::timing_begin((cudaStream_t)stream, ev);
  int rc = aosb::launch_row_blocks<false>(a, max_block_rows, 1, (cudaStream_t)stream, err, cap);
  if (rc) return rc;
  // algorithmic: 8 FP64 flops per (nonzero, column); A once, x read and y
  // written once
  if (timed)
    aosb::timing_end(aosb::kTimedSpmm, (cudaStream_t)stream, ev, 8.0 * nnz * ncols,
                     8.0 * nnz + (double)n * ncols * 32.0);
  return aosb::launch_check(err, cap, "spmm_blocks");
}

int aosb_shifted_residual(int64_t n, int32_t nrhs, int32_t np, const int64_t* indptr,
                          const int32_t* indices, const aosb_complex64* h_values,
                          const aosb_complex64* s_values, int64_t nnz, const int32_t* pencil_k,
                          const aosb_complex128* shifts, const aosb_complex128* b,
                          int64_t b_stride, const aosb_complex128* x, aosb_complex128* r,
                          void* stream, char* err, size_t cap) {
  if (indptr == nullptr || indices == nullptr || h_values == nullptr ||
      pencil_k == nullptr || shifts == nullptr || b == nullptr || x == nullptr || r == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "null argument");
  if (np <= 0 || np > 65535 || nrhs <= 0 || n <= 0)
    return aosb::set_error(err, cap, AOSB_ERR_BATCH, "invalid batch");
  dim3 g(aosb::ceil_div(n, 8), np);
  aosb::shifted_residual_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(
      n, nrhs, indptr, indices, (const float2*)h_values, (const float2*)s_values, nnz, pencil_k,
      (const double2*)shifts, (const double2*)b, b_stride, (const double2*)x, (double2*)r);
  aosb::count_launches(1);
  return aosb::launch_check(err, cap, "shifted_residual");
}

}  // extern "C"

extern "C" int32_t aosb_solve_set_lookahead(int32_t on) {
  if (on < 0 || on > 1) return -1;
  return aosb::g_solve_lookahead.exchange(on);
}
