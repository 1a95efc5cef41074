// Internal entry points of the factorization modules.
#pragma once

#include "plan.h"

namespace aosb {
int factor_assemble(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap);
int factor_step_panels(const aosb_plan* P, const aosb_factor_args_v1* a, int k, char* err,
                       size_t cap);
int factor_step_diag(const aosb_plan* P, const aosb_factor_args_v1* a, int k, cudaStream_t st,
                     char* err, size_t cap);
int factor_plain(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap);
int factor_tc(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap);
size_t factor_tc_workspace(const aosb_plan* P, int32_t n_pencils);
}  // namespace aosb
