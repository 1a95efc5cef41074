// Tensor-core (tcgen05) factorization path: split-BF16 Schur updates.
#include "factor.h"

namespace aosb {

size_t factor_tc_workspace(const aosb_plan* P, int32_t n_pencils) {
  (void)P;
  (void)n_pencils;
  return 0;
}

int factor_tc(const aosb_plan* P, const aosb_factor_args_v1* a, char* err, size_t cap) {
  (void)P;
  (void)a;
  return set_error(err, cap, AOSB_ERR_UNSUPPORTED, "tensor-core path not built");
}

}  // namespace aosb
