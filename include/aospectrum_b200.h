/*
 * C ABI of the B200 CISS band engine (libaospectrum_b200.so, sm_100a).
 *
 * Every entry point takes plain pointers and sizes.  Pointers documented as
 * "device" must be CUDA device memory on the current device; "host" pointers
 * are ordinary host memory.  Functions return 0 on success and a nonzero
 * status code otherwise; when an error buffer is passed, a NUL-terminated
 * message is written into it.  Kernels are enqueued on the caller's stream
 * (a cudaStream_t passed as void*; NULL is the legacy default stream) and
 * the functions return without synchronising unless stated otherwise.
 *
 * Reference interfaces that each group replaces (paths inside the
 * yumiaoyi-o/AOSpectrum project):
 *   - aospectrum_b200_solve_complex64_ubatch_v1 replaces
 *     aospectrum_cudss_solve_complex64_ubatch_v1
 *     (native/include/aospectrum_cudss_complex64_ubatch.h:64-66); the
 *     request and result structs keep that header's field order (18-62).
 *   - aosb_bloch_* replace BlochPattern.from_bundle and
 *     BlochWorkspace.update (src/aospectrum/sparse.py:64-140, 181-245).
 *   - aosb_plan_*, aosb_factor, aosb_solve and the IR helpers replace the
 *     cuDSS ANALYSIS / FACTORIZATION / SOLVE phases called from
 *     native/src/aospectrum_cudss_complex64_ubatch.c:446-600.
 *   - aosb_spmm(_blocks), aosb_moments_accumulate, aosb_gram, aosb_dense_mul
 *     and aosb_column_norms replace the host numpy/scipy steps of
 *     CudssCissSolver.solve_interval (src/aospectrum/ciss.py:284-372).
 */
#ifndef AOSPECTRUM_B200_H
#define AOSPECTRUM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AOSPECTRUM_B200_ABI_VERSION 1u
#define AOSPECTRUM_B200_ERROR_CAPACITY 512u

/* Status codes.  10-14, 20-22, 30-36 and 40 keep the meaning they have in
 * native/src/aospectrum_cudss_complex64_ubatch.c:56-241. */
#define AOSB_OK 0
#define AOSB_ERR_ABI 10
#define AOSB_ERR_DIMS 11
#define AOSB_ERR_BATCH 12
#define AOSB_ERR_NULL 13
#define AOSB_ERR_INDPTR 14
#define AOSB_ERR_CUDA 20
#define AOSB_ERR_ENGINE 21
#define AOSB_ERR_DEVICE_INFO 22
#define AOSB_ERR_CSR_MONOTONIC 30
#define AOSB_ERR_CSR_COLUMN 31
#define AOSB_ERR_CSR_ORDER 32
#define AOSB_ERR_DIAGONAL 33
#define AOSB_ERR_SIZE 34
#define AOSB_ERR_NONFINITE_MATRIX 35
#define AOSB_ERR_NONFINITE_RHS 36
#define AOSB_ERR_MEMORY 40
#define AOSB_ERR_TOPOLOGY 41
#define AOSB_ERR_ZERO_PIVOT 50
#define AOSB_ERR_NONFINITE_FACTOR 51
#define AOSB_ERR_TIMEOUT 52
#define AOSB_ERR_ARGUMENT 53
#define AOSB_ERR_UNSUPPORTED 54

typedef struct {
  float real;
  float imag;
} aosb_complex64;

typedef struct {
  double real;
  double imag;
} aosb_complex128;

/* Build facts: ABI version and a static string naming arch and options. */
uint32_t aosb_abi_version(void);
const char *aosb_build_info(void);
/* Kernels launched by this library since load (all devices and threads). */
uint64_t aosb_launch_count(void);

/* Measurement hook (no counterpart in the reference, whose cuDSS calls are
 * opaque): aosb_kernel_timing(1) clears and starts CUDA-event timing of
 * every tensor-core Schur-update launch (schur_tc_kernel) on the stream it
 * is launched on; aosb_kernel_timing(0) stops.  _read synchronizes on the
 * recorded events and returns the summed device time (ms), the algorithmic
 * flops (8 T^3 per target tile and pencil), the algorithmic bytes (target
 * read + write, staged operands read once) and the number of launches. */
int aosb_kernel_timing(int32_t enable);
int aosb_kernel_timing_read(double *total_ms, double *flops, double *bytes,
                            int64_t *launches);
/* The same for a category: 0 = tensor-core Schur updates, 1 = solve
 * diagonal steps (4 T^2 L flops per pencil), 2 = solve tile updates
 * (8 T^2 L flops per tile and pencil; factor tile read, X tile read and
 * written), 3 = FP64 shifted residuals (8 flops per nonzero, column and
 * pencil), 4 = FP64 SpMM (8 flops per nonzero and column), 5 = Bloch sums
 * (bytes: stored H and S values read once, complex64 H(k), S(k) written
 * once per k point).  Timing skips launches issued while a stream is
 * captured. */
int aosb_kernel_timing_read_category(int32_t category, double *total_ms, double *flops,
                                     double *bytes, int64_t *launches);

/* ------------------------------------------------------------------------
 * Drop-in uniform-batch shifted solve with host buffers.
 * Replaces aospectrum_cudss_solve_complex64_ubatch_v1
 * (native/include/aospectrum_cudss_complex64_ubatch.h:64-66).
 * values: batch_count x nnz shifted matrices H - z_b S in CSR order;
 * rhs/solution: batch_count x rhs_count x n, column-major per batch entry
 * (the layout native/src/bindings.cpp:153-157 packs).
 * The symbolic plan of the last pattern is cached inside the library, so
 * repeated calls with the same indptr/indices skip the analysis.
 * ------------------------------------------------------------------------ */
typedef struct {
  uint32_t abi_version;
  uint32_t struct_size;
  int64_t n;
  int64_t nnz;
  int32_t batch_count;
  int32_t rhs_count;
  const int32_t *indptr;
  const int32_t *indices;
  const aosb_complex64 *values;
  const aosb_complex64 *rhs;
  aosb_complex64 *solution;
} aospectrum_b200_ubatch_request_v1;

typedef struct {
  uint32_t abi_version;
  uint32_t struct_size;
  int32_t status;
  int32_t engine_status; /* device status of the factorization (0 = ok) */
  int64_t n;
  int64_t nnz;
  int64_t diagonal_count;
  int64_t reported_factor_nnz; /* stored factor entries (tile level) */
  int32_t reported_pivot_count; /* row interchanges inside diagonal tiles */
  int32_t batch_count;
  int32_t rhs_count;
  int32_t iterative_refinement_steps;
  double upload_seconds;
  double descriptor_setup_seconds;
  double analysis_seconds;
  double factorization_seconds;
  double solve_seconds;
  double download_seconds;
  double total_seconds;
  uint64_t permanent_device_bytes;
  uint64_t peak_device_bytes;
  uint64_t permanent_host_bytes;
  uint64_t peak_host_bytes;
  uint64_t free_device_bytes_before;
  uint64_t free_device_bytes_after_upload;
  uint64_t free_device_bytes_after_factorization;
  uint64_t free_device_bytes_after_solve;
  uint64_t total_device_bytes;
  char error_message[AOSPECTRUM_B200_ERROR_CAPACITY];
} aospectrum_b200_ubatch_result_v1;

int aospectrum_b200_solve_complex64_ubatch_v1(
    const aospectrum_b200_ubatch_request_v1 *request,
    aospectrum_b200_ubatch_result_v1 *result);

/* ------------------------------------------------------------------------
 * Bloch pattern and Bloch sum.
 * Replaces BlochPattern.from_bundle (src/aospectrum/sparse.py:64-140) and
 * BlochWorkspace.update / _fill / _project_hermitian (sparse.py:25-36,
 * 181-245).
 * ------------------------------------------------------------------------ */
typedef struct aosb_bloch aosb_bloch_t;

/* Host inputs are the operator block table of the bundle.  Builds the CSR
 * pattern (sorted, duplicate-free columns) and the block maps on the host
 * (no device call).  Fails with AOSB_ERR_TOPOLOGY when some block has no
 * mirror block (the topology is not Hermitian). */
int aosb_bloch_create(int64_t n_orbitals, int64_t n_atoms,
                      const int64_t *atom_offsets, int64_t n_blocks,
                      const int32_t *row_atom, const int32_t *col_atom,
                      const int32_t *lattice_shift, const int64_t *block_offsets,
                      aosb_bloch_t **out, char *err, size_t err_cap);
/* Copies the tables to the current device; required before the device
 * entry points below.  Synchronous; call it before any stream capture. */
int aosb_bloch_upload(aosb_bloch_t *b, char *err, size_t err_cap);
/* nnz of the CSR pattern, number of distinct lattice shifts. */
int aosb_bloch_info(const aosb_bloch_t *b, int64_t *nnz, int64_t *n_shifts);
/* Host outputs: indptr[n+1], indices[nnz], shifts[n_shifts*3] (distinct
 * shifts in lexicographic order), block_shift[n_blocks] (shift index). */
int aosb_bloch_export(const aosb_bloch_t *b, int64_t *indptr, int32_t *indices,
                      int32_t *shifts, int32_t *block_shift);
/* Host copies of the Bloch kernel's tables (no counterpart in the
 * reference): per group of blocks with one atom pair (i, j), in
 * (row atom, column atom) order, group_info[4g..4g+3] = (rows, columns, CSR
 * row length of atom i, mirror group (j, i)), group_dst[g] = CSR position
 * of the group's entry (0, 0), group_members[2g..2g+1] = [begin, end) of its
 * member blocks; per member block, member_off = offset of its values and
 * member_shift = its lattice-shift index.  Pass null arrays to read the
 * counts first. */
int aosb_bloch_export_groups(const aosb_bloch_t *b, int64_t *n_groups, int64_t *n_members,
                             int32_t *group_info, int64_t *group_dst,
                             int32_t *group_members, int64_t *member_off,
                             int32_t *member_shift);
/* Device CSR pattern arrays owned by the handle (valid until destroy). */
int aosb_bloch_device_pattern(const aosb_bloch_t *b, const int64_t **indptr,
                              const int32_t **indices);
/* H(k), S(k) for n_k k points: value_kind 0 = float32 block values,
 * 1 = complex64.  phases: device [n_k][n_shifts] exp(2 pi i R.k);
 * outputs: device [n_k][nnz] complex64, Hermitian-projected. */
int aosb_bloch_apply(const aosb_bloch_t *b, int32_t value_kind,
                     const void *h_values, const void *s_values,
                     const aosb_complex64 *phases, int32_t n_k,
                     aosb_complex64 *h_out, aosb_complex64 *s_out, void *stream,
                     char *err, size_t err_cap);
void aosb_bloch_destroy(aosb_bloch_t *b);

/* ------------------------------------------------------------------------
 * Symbolic analysis, once per CSR pattern: supervariables, nested
 * dissection on the supervariable graph, tile padding, tile-level fill and
 * the per-step tile lists.  Replaces the cuDSS ANALYSIS phase that the
 * reference re-runs on every call (aospectrum_cudss_complex64_ubatch.c:
 * 446-474).
 * ------------------------------------------------------------------------ */
typedef struct aosb_plan aosb_plan_t;

typedef struct {
  uint32_t abi_version;
  uint32_t struct_size;
  int32_t tile;           /* 32, 64 or 128 */
  int32_t ordering;       /* 0 natural order, 1 nested dissection */
  int32_t leaf_dofs;      /* nested dissection stops below this many dofs */
  int32_t pad_nodes;      /* 1: every ordering node starts on a tile edge */
} aosb_plan_options_v1;

typedef struct {
  int64_t n;
  int64_t n_pad;
  int64_t nnz;
  int64_t n_tiles;
  int64_t n_slots;
  int64_t n_supervariables;
  int64_t n_nodes;
  int64_t schur_tile_updates;
  int64_t tree_levels;
  int32_t tile;
  int32_t reserved;
  double factor_flops;      /* real flops of one factorization, tile level */
  double factor_flops_alg;  /* same, padded rows and columns excluded */
  double factor_bytes;      /* bytes of one stored factor */
} aosb_plan_info_v1;

int aosb_plan_create(int64_t n, const int64_t *indptr, const int32_t *indices,
                     const int64_t *sv_offsets, int64_t n_sv,
                     const aosb_plan_options_v1 *options, aosb_plan_t **out,
                     char *err, size_t err_cap);
/* Host-only: aosb_plan_create performs no device call.  aosb_plan_upload
 * copies the plan tables to the current device (synchronous, before any
 * stream capture); factor, solve, gather and scatter require it. */
int aosb_plan_upload(aosb_plan_t *plan, char *err, size_t err_cap);
int aosb_plan_info(const aosb_plan_t *plan, aosb_plan_info_v1 *info);
/* perm[n_pad]: original dof of each permuted position, -1 for padding. */
int aosb_plan_export_perm(const aosb_plan_t *plan, int32_t *perm);
/* slot[n_tiles*n_tiles]: storage slot of each tile, -1 if structurally 0. */
int aosb_plan_export_slots(const aosb_plan_t *plan, int32_t *slot);
/* The two-step (K = 256) Schur item lists of the plan (host copies), for
 * inspection and tests; no counterpart in the reference.  Call with null
 * arrays for the sizes: n_super super-steps (tile steps 2s, 2s+1),
 * cross_off / rest_off [n_super + 1] item offsets, items of 5 ints (target
 * slot, staged A and B index of step 2s or -1, of step 2s+1 or -1). */
int aosb_plan_export_super_steps(const aosb_plan_t *plan, int64_t *n_super, int64_t *n_cross,
                                 int64_t *n_rest, int64_t *cross_off, int64_t *rest_off,
                                 int32_t *cross, int32_t *rest);
/* The same items as pairs for the two-CTA (M = 256) Schur update, host
 * copies for inspection and tests; no counterpart in the reference.  Pairs
 * of 8 ints: target slot of the even CTA, of the odd CTA (-1: single),
 * then for step 2s and step 2s+1 the staged A index of the even CTA, of the
 * odd CTA and the shared staged B index (-1 when that step's half is
 * absent).  cross_off / rest_off hold [n_super + 1] pair offsets. */
int aosb_plan_export_pair_steps(const aosb_plan_t *plan, int64_t *n_cross, int64_t *n_rest,
                                int64_t *cross_off, int64_t *rest_off, int32_t *cross,
                                int32_t *rest);
void aosb_plan_destroy(aosb_plan_t *plan);

/* ------------------------------------------------------------------------
 * Numeric factorization P A_p = L_p U_p of A_p = H(k_p) - z_p S(k_p) for a
 * batch of pencils, all on the plan's pattern.  Row interchanges stay
 * inside diagonal tiles (partial pivoting on the tile).  The diagonal tile
 * slot stores inv(L_kk) strictly below and inv(U_kk) on and above its
 * diagonal.
 * ------------------------------------------------------------------------ */
#define AOSB_PRECISION_PLAIN 0  /* complex64, FP32 SIMT updates */
#define AOSB_PRECISION_BF16X3 1 /* split-BF16 tcgen05 panels and two-step
                                   (K = 256) Schur updates with lookahead,
                                   FP32 accumulate (tile 128) */
#define AOSB_PRECISION_BF16X3_FP32_PANELS 2 /* split-BF16 tcgen05 Schur updates,
                                               FP32 SIMT panels (tile 128) */
#define AOSB_PRECISION_BF16X3_ONE_STEP 3 /* as 1 with one-step (K = 128) Schur
                                            updates */

typedef struct {
  uint32_t abi_version;
  uint32_t struct_size;
  int32_t n_pencils;
  int32_t precision;
  const aosb_complex64 *h_values; /* device [n_k][nnz] */
  const aosb_complex64 *s_values; /* device [n_k][nnz] */
  const int32_t *pencil_k;        /* device [n_pencils] row of h/s values */
  const aosb_complex128 *shifts;  /* device [n_pencils] z_p */
  float *factor;                  /* device [n_pencils][n_slots][2][T][T] */
  int32_t *pivots;                /* device [n_pencils][n_pad] */
  int32_t *status;                /* device [n_pencils], 0 = ok */
  void *workspace;                /* device, aosb_factor_workspace_bytes */
  void *stream;
} aosb_factor_args_v1;

size_t aosb_factor_bytes(const aosb_plan_t *plan, int32_t n_pencils);
/* Tensor-core precisions: four staging buffers of split-BF16 panel tiles
 * plus 256 bytes for the item counter that the two-step update's main and
 * lookahead launches share; 0 for precision 0.  A workspace sized for
 * n_pencils serves any batch of at most n_pencils; one factorization at a
 * time per workspace. */
size_t aosb_factor_workspace_bytes(const aosb_plan_t *plan, int32_t n_pencils,
                                   int32_t precision);
int aosb_factor(const aosb_plan_t *plan, const aosb_factor_args_v1 *args,
                char *err, size_t err_cap);
/* SMs that the tensor-core factorization leaves to its lookahead side
 * stream (next steps' diagonal LU, panel products and staging) while the
 * Schur update runs on the others; 0 restores the default rule
 * min(max(5 n_pencils / 4, 8), SMs / 3); values are capped at SMs / 2.
 * Process-wide; returns the previous setting (-1 for sms < 0).  No
 * counterpart in the reference (cuDSS schedules internally). */
int32_t aosb_factor_set_lookahead_sms(int32_t sms);
/* 1: the two-step tensor-core Schur updates run as pairs of targets of one
 * tile column on two-CTA clusters (tcgen05 cta_group::2, M = 256: the pair
 * shares the B operand, a quarter less operand traffic per MMA); 0: one
 * target per CTA.  Process-wide; returns the previous setting (-1 for
 * other values).  No counterpart in the reference. */
int32_t aosb_factor_set_schur_pairs(int32_t on);
/* Polls of one mbarrier wait in the tensor-core kernels (factorization
 * Schur/panel products and solve updates) before the waiting CTA gives up:
 * it records AOSB_ERR_TIMEOUT in the pencil's status word, waits (with the
 * default bound) for its own copies and MMAs in flight, frees its TMEM and
 * returns, so the context stays usable.  The default is 4,194,304 polls
 * with backoff (well over a second of waiting); 0 restores it.
 * Process-wide, read at each launch; returns the previous value (-1 for a
 * negative argument).  No counterpart in the reference (cuDSS has no
 * bounded waits to set). */
int64_t aosb_tc_set_wait_limit(int64_t polls);

/* ------------------------------------------------------------------------
 * Block-RHS triangular solves in the permuted, padded order:
 * adjoint = 0 solves A X = B, adjoint = 1 solves A^H X = B (the conjugate
 * shift of a contour node pair reuses one factorization this way).
 * work: device [n_pencils][n_pad][n_rhs] complex64, overwritten.
 * scratch: device, aosb_solve_scratch_bytes(plan, n_pencils, n_rhs).
 * flags: AOSB_SOLVE_TENSOR_CORES (tile 128) runs the off-diagonal tile
 * updates on the tensor cores in split BF16 (FP32 accumulation); 0 keeps
 * them in FP32 SIMT.  The tensor-core updates bound their waits; after the
 * solves, aosb_solve_check synchronizes the stream and reports a timeout.
 * ------------------------------------------------------------------------ */
#define AOSB_SOLVE_TENSOR_CORES 1
/* AOSB_SOLVE_GRAPH: capture the solve's launch sequence into a CUDA graph
 * the first time a (plan, n_pencils, n_rhs, adjoint, flags, factor, pivots,
 * work, scratch) combination is seen and replay it afterwards; ignored while
 * the stream is being captured by the caller.  Graphs are released with
 * their plan. */
#define AOSB_SOLVE_GRAPH 2

typedef struct {
  uint32_t abi_version;
  uint32_t struct_size;
  int32_t n_pencils;
  int32_t n_rhs;
  int32_t adjoint;
  int32_t flags;
  const float *factor;
  const int32_t *pivots;
  aosb_complex64 *work;
  void *scratch;
  void *stream;
} aosb_solve_args_v1;

size_t aosb_solve_scratch_bytes(const aosb_plan_t *plan, int32_t n_pencils, int32_t n_rhs);
int aosb_solve(const aosb_plan_t *plan, const aosb_solve_args_v1 *args,
               char *err, size_t err_cap);
/* Synchronizes args->stream and returns AOSB_ERR_TIMEOUT when a
 * tensor-core update of an aosb_solve call with these args gave up on a
 * bounded wait (status words kept in the scratch block, cleared by each
 * aosb_solve). */
int aosb_solve_check(const aosb_plan_t *plan, const aosb_solve_args_v1 *args,
                     char *err, size_t err_cap);
/* CTAs per SM of the tensor-core solve update (AOSB_SOLVE_TENSOR_CORES):
 * 1 (deep slab and RHS rings, 208 KB of shared memory) or 2 (default:
 * shallow rings, 96 KB each, so one CTA's waits overlap the other's work;
 * bit-identical results); 0 restores the default.  Process-wide; graphs captured before a change
 * keep the form they captured.  Returns the previous setting (-1 for values
 * outside 0..2).  No counterpart in the reference (cuDSS schedules
 * internally). */
int32_t aosb_solve_set_ctas_per_sm(int32_t ctas);
/* 1: the tensor-core sweeps (AOSB_SOLVE_TENSOR_CORES) update the next
 * step's tile first and run the next diagonal solve on a side stream
 * beside the rest of the current step's updates (double-buffered diagonal
 * results; same arithmetic, same results); 0: one diagonal solve and one
 * update per step in order.  Process-wide; returns the previous setting (-1
 * for other values).  No counterpart in the reference. */
int32_t aosb_solve_set_lookahead(int32_t on);

/* work[p][i][:] = complex64(src[p*src_stride + perm[i]*n_rhs + :]), zero for
 * padding rows (src: device complex128 [.][n][n_rhs]). */
int aosb_gather_rhs(const aosb_plan_t *plan, int32_t n_pencils, int32_t n_rhs,
                    const aosb_complex128 *src, int64_t src_stride,
                    aosb_complex64 *work, void *stream, char *err, size_t err_cap);
/* x[p][j][:] (+)= complex128(work[p][pinv[j]][:]); accumulate 0 overwrites. */
int aosb_scatter_solution(const aosb_plan_t *plan, int32_t n_pencils, int32_t n_rhs,
                          const aosb_complex64 *work, aosb_complex128 *x,
                          int32_t accumulate, void *stream, char *err, size_t err_cap);
/* FP64 residual r[p] = b[p*b_stride] - (H(k_p) - z_p S(k_p)) x[p] on the CSR
 * pattern (indptr/indices device). */
int aosb_shifted_residual(int64_t n, int32_t n_rhs, int32_t n_pencils,
                          const int64_t *indptr, const int32_t *indices,
                          const aosb_complex64 *h_values,
                          const aosb_complex64 *s_values, int64_t nnz,
                          const int32_t *pencil_k, const aosb_complex128 *shifts,
                          const aosb_complex128 *b, int64_t b_stride,
                          const aosb_complex128 *x, aosb_complex128 *r,
                          void *stream, char *err, size_t err_cap);

/* The same residual for patterns whose rows come in blocks with identical
 * column sets (the orbitals of one atom): row_blocks[n_blocks+1] (device)
 * are block start rows, every block at most max_block_rows (1..16) rows;
 * rows of a block longer than that come back NaN.  Each x row is read once
 * per block. */
int aosb_shifted_residual_blocks(int64_t n, int32_t n_rhs, int32_t n_pencils,
                                 int64_t n_blocks, const int32_t *row_blocks,
                                 int32_t max_block_rows,
                                 const int64_t *indptr, const int32_t *indices,
                                 const aosb_complex64 *h_values,
                                 const aosb_complex64 *s_values, int64_t nnz,
                                 const int32_t *pencil_k, const aosb_complex128 *shifts,
                                 const aosb_complex128 *b, int64_t b_stride,
                                 const aosb_complex128 *x, aosb_complex128 *r,
                                 void *stream, char *err, size_t err_cap);

/* ------------------------------------------------------------------------
 * FP64 CISS kernels on n x m complex128 blocks (row-major, leading
 * dimension = row stride in elements).
 * ------------------------------------------------------------------------ */
/* y = A x, A complex64 CSR, x and y complex128. */
int aosb_spmm(int64_t n, int32_t ncols, const int64_t *indptr,
              const int32_t *indices, const aosb_complex64 *values,
              const aosb_complex128 *x, int64_t ldx, aosb_complex128 *y,
              int64_t ldy, void *stream, char *err, size_t err_cap);
/* y = A x on a row-blocked pattern (row_blocks and max_block_rows as for
 * aosb_shifted_residual_blocks): each x row is read once per block. */
int aosb_spmm_blocks(int64_t n, int32_t ncols, int64_t n_blocks,
                     const int32_t *row_blocks, int32_t max_block_rows,
                     const int64_t *indptr, const int32_t *indices,
                     const aosb_complex64 *values, int64_t nnz,
                     const aosb_complex128 *x, int64_t ldx, aosb_complex128 *y,
                     int64_t ldy, void *stream, char *err, size_t err_cap);
/* mom[:, m*L:(m+1)*L] += coef[m] * x for m < n_moments. */
int aosb_moments_accumulate(int64_t n, int32_t n_rhs, int32_t n_moments,
                            const aosb_complex128 *x, const aosb_complex128 *coef,
                            aosb_complex128 *mom, void *stream, char *err,
                            size_t err_cap);
/* g (p x q) = x^H y; scratch: device, aosb_gram_scratch_bytes(n, p, q). */
size_t aosb_gram_scratch_bytes(int64_t n, int32_t p, int32_t q);
int aosb_gram(int64_t n, int32_t p, int32_t q, const aosb_complex128 *x,
              int64_t ldx, const aosb_complex128 *y, int64_t ldy,
              aosb_complex128 *g, void *scratch, void *stream, char *err,
              size_t err_cap);
/* aosb_gram without any allocation (no counterpart in the reference).
 * For callers that cannot allocate device memory when they call: code inside
 * another framework's memory pool or under a device-memory cap, real-time or
 * callback contexts where cudaMalloc could block or deadlock, embedders that
 * must not grow the device heap after start-up.  The partial sums use one
 * fixed 16 MiB device array inside the library (held on every GPU that
 * loads it until exit); sizes with ceil(n/512)*p*q*16 bytes above 16 MiB are
 * rejected with AOSB_ERR_SIZE.  The first call on a device resolves that
 * array's address with a synchronous runtime call: make it before any stream
 * capture.  All calls share the one array, so calls that overlap on the GPU
 * (other streams, other host threads) race; serialise them. */
int aosb_gram_noalloc(int64_t n, int32_t p, int32_t q, const aosb_complex128 *x,
                      int64_t ldx, const aosb_complex128 *y, int64_t ldy,
                      aosb_complex128 *g, void *stream, char *err, size_t err_cap);
/* y (n x r) = x (n x p) t (p x r), t row-major p x r. */
int aosb_dense_mul(int64_t n, int32_t p, int32_t r, const aosb_complex128 *x,
                   int64_t ldx, const aosb_complex128 *t, aosb_complex128 *y,
                   int64_t ldy, void *stream, char *err, size_t err_cap);
/* out[j] = || a[:, j] - e[j] * b[:, j] ||_2 for j < m. */
int aosb_column_norms(int64_t n, int32_t m, const aosb_complex128 *a,
                      const aosb_complex128 *b, int64_t ld, const double *e,
                      double *out, void *stream, char *err, size_t err_cap);

/* ------------------------------------------------------------------------
 * Real symmetric shifted factorization with inertia (Gamma point).
 * Replaces aospectrum_cudss_shift_factor_{create_device,refactor_device,
 * solve,get_stats,destroy} (native/include/aospectrum_cudss_shift_factor.h:
 * 15-76, native/src/aospectrum_cudss_shift_factor.c:232-742): same
 * arguments in the same order, the same statistics block, and the same
 * meaning -- A = H - shift * S from the upper triangle (diagonal included)
 * of the caller's real float32 CSR values on the DEVICE, int32 CSR pattern
 * on the host; inertia_negative / inertia_positive count the eigenvalues of
 * the pencil (H, S) below / above the shift (S positive definite), so
 * n - negative - positive is the count at the shift.  Differences: the
 * factorization is this library's tile block elimination (FP32 tile
 * updates, partial pivoting inside diagonal tiles) with the inertia taken
 * tile by tile from a Bunch-Kaufman LDL^T of each eliminated diagonal tile;
 * pivot_count is the number of symmetric interchanges those LDL^Ts made;
 * factor_nnz counts the stored tile entries.  Functions return 0 or an
 * AOSB_ERR_* status (the reference returns 1 for every failure); a shift at
 * which a diagonal tile is exactly singular fails with AOSB_ERR_DEVICE_INFO.
 * rhs / solution of aosb_shift_factor_solve are device float32 column-major
 * blocks (leading dimension >= n), as the reference's PRIMME preconditioner
 * passes them; the call synchronizes the stream.
 * ------------------------------------------------------------------------ */
typedef struct aosb_shift_factor aosb_shift_factor_t;

typedef struct {
  int64_t upper_nnz;
  int64_t factor_nnz;
  int32_t pivot_count;
  int32_t inertia_positive;
  int32_t inertia_negative;
  int32_t solve_calls;
  int64_t solved_rhs;
  double preparation_seconds;
  double upload_seconds;
  double analysis_seconds;
  double factorization_seconds;
  double solve_seconds;
  uint64_t permanent_device_bytes;
  uint64_t peak_device_bytes;
  uint64_t permanent_host_bytes;
  uint64_t peak_host_bytes;
  uint64_t free_device_bytes_before_factorization;
  uint64_t free_device_bytes_after_factorization;
} aosb_shift_factor_stats;

int aosb_shift_factor_create_device(aosb_shift_factor_t **factor, int64_t n, int64_t nnz,
                                    const int32_t *indptr, const int32_t *indices,
                                    const float *device_hamiltonian_values,
                                    const float *device_overlap_values, float shift,
                                    int32_t maximum_rhs, void *stream, char *err,
                                    size_t err_cap);
int aosb_shift_factor_refactor_device(aosb_shift_factor_t *factor,
                                      const float *device_hamiltonian_values,
                                      const float *device_overlap_values, float shift,
                                      char *err, size_t err_cap);
int aosb_shift_factor_solve(aosb_shift_factor_t *factor, const float *rhs,
                            int64_t leading_rhs, float *solution, int64_t leading_solution,
                            int32_t rhs_count, char *err, size_t err_cap);
void aosb_shift_factor_get_stats(const aosb_shift_factor_t *factor,
                                 aosb_shift_factor_stats *stats);
void aosb_shift_factor_destroy(aosb_shift_factor_t *factor);

#ifdef __cplusplus
}
#endif

#endif /* AOSPECTRUM_B200_H */
