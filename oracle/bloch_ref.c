/*
 * Plain C restatement of the reference Bloch sum -- test oracle only.
 *
 * Given the expanded, sorted entry tables of the reference pattern builder
 * (src/aospectrum/sparse.py:64-140 of yumiaoyi-o/AOSpectrum: source index,
 * phase group and segment start per CSR entry) this computes
 *   out[p] = sum_{s in segment p} value[source[s]] * phase[group[s]]
 * in float32 complex arithmetic, left to right (sparse.py:181-197), then the
 * Hermitian projection of sparse.py:25-36.  Real (float32) or complex64
 * values.  Complex products are formed as (ac - bd, ad + bc) with every
 * operation rounded to float32; compile without FMA contraction.
 */
#include <stdint.h>

typedef struct { float re, im; } c64;

static c64 cmul(c64 a, c64 b) {
  volatile float ac = a.re * b.re, bd = a.im * b.im, ad = a.re * b.im, bc = a.im * b.re;
  c64 r = {ac - bd, ad + bc};
  return r;
}

void oracle_bloch_sum(int64_t nnz, int64_t n_entries, const int64_t *starts,
                      const int64_t *source, const int64_t *group, int value_kind,
                      const void *values, const c64 *phase, c64 *out) {
  for (int64_t p = 0; p < nnz; ++p) {
    const int64_t b = starts[p], e = (p + 1 < nnz) ? starts[p + 1] : n_entries;
    c64 acc = {0.0f, 0.0f};
    for (int64_t s = b; s < e; ++s) {
      c64 v;
      if (value_kind == 0) {
        v.re = ((const float *)values)[source[s]];
        v.im = 0.0f;
      } else {
        v = ((const c64 *)values)[source[s]];
      }
      c64 t = cmul(v, phase[group[s]]);
      if (s == b) {
        acc = t;
      } else {
        acc.re = acc.re + t.re;
        acc.im = acc.im + t.im;
      }
    }
    out[p] = acc;
  }
}

void oracle_project_hermitian(int64_t n_upper, const int64_t *upper, const int64_t *lower,
                              int64_t n_diag, const int64_t *diag, c64 *v) {
  for (int64_t i = 0; i < n_upper; ++i) {
    c64 a = v[upper[i]], b = v[lower[i]];
    c64 m = {(a.re + b.re) * 0.5f, (a.im - b.im) * 0.5f};
    v[upper[i]] = m;
    c64 cm = {m.re, -m.im};
    v[lower[i]] = cm;
  }
  for (int64_t i = 0; i < n_diag; ++i) v[diag[i]].im = 0.0f;
}
