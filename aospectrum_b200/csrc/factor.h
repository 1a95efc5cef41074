// Internal entry points of the factorization modules.
#pragma once

#include "plan.h"

#include <cuda.h>

namespace aosb {
int factor_assemble(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap);
int factor_step_panels(const aosb_plan* P, const aosb_factor_args_v1* a, int k, char* err,
                       size_t cap);
int factor_step_diag(const aosb_plan* P, const aosb_factor_args_v1* a, int k, cudaStream_t st,
                     char* err, size_t cap);
// Called by the plain factorization before the diagonal LU of tile step k,
// on the factorization's stream: the diagonal tile (k, k) then holds the
// Schur complement that the steps before k left (nonzero return aborts).
using StepHook = int (*)(void* ctx, int64_t k, cudaStream_t stream, char* err, size_t cap);
int factor_plain(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap,
                 StepHook hook = nullptr, void* hook_ctx = nullptr);
int factor_tc(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap);
size_t factor_tc_workspace(const aosb_plan* P, int32_t n_pencils);
// Two-CTA (M = 256) Schur update of one pair list (schur_pair.cu): the
// pairs d_list[0 .. n_pairs) x n_pencils, operands from the staging buffers
// at byte offsets buf0_bytes (first tile step) and buf1_bytes (second),
// `ctas` CTAs (clusters of two); with `claim` the pairs are taken from that
// counter, shared with another launch of the same list.
int schur_pair_launch(const int32_t* d_list, int64_t n_pairs, int n_pencils, int64_t n_slots,
                      unsigned char* staging, int64_t staging_bytes, int64_t buf0_bytes,
                      int64_t buf1_bytes, int64_t pencil_stride, int32_t* status, int* claim,
                      const CUtensorMap& tmap_c, int ctas, cudaStream_t st, char* err,
                      size_t cap);
}  // namespace aosb
