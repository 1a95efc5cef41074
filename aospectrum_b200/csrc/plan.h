// Symbolic plan shared by the factorization and solve modules.
#pragma once

#include "common.cuh"

#include <vector>

struct aosb_plan {
  int64_t n = 0, n_pad = 0, nnz = 0, nb = 0, T = 0, n_slots = 0;
  int64_t n_sv = 0, n_nodes = 0, schur_updates = 0, tree_levels = 0;
  double flops = 0.0, flops_alg = 0.0;
  std::vector<int32_t> perm;  // n_pad
  std::vector<int32_t> pinv;  // n
  std::vector<int32_t> slot;  // nb*nb
  std::vector<int32_t> real_dofs;  // per tile
  // Per-step tile lists: offsets [nb+1] and (tile, slot) entries.
  std::vector<int32_t> lb_off, lb_tile, lb_slot;  // L column k, rows i > k
  std::vector<int32_t> ur_off, ur_tile, ur_slot;  // U row k, cols j > k
  std::vector<int32_t> ua_off, ua_tile, ua_slot;  // U column k, rows i < k
  std::vector<int32_t> ll_off, ll_tile, ll_slot;  // L row k, cols j < k
  std::vector<int64_t> sc_off;                    // Schur target offsets [nb+1]
  std::vector<int32_t> sc_slot;                   // |L_k| x |U_k| target slots per step
  std::vector<int32_t> diag_slot;                 // slot of (k, k)
  // Two-step (K = 256) Schur updates, super-step s = tile steps (2s, 2s+1):
  // the targets of step 2s outside tile row/column 2s+1 merged with the
  // targets of step 2s+1, 5 ints per item: target slot, then the staged A
  // and B indices of step 2s (L index a, nL + U index b) or -1, then those of
  // step 2s+1 or -1.  "cross" items lie in tile row or column 2s+2 or 2s+3
  // (read by the next super-step's panels), "rest" items elsewhere.
  std::vector<int64_t> ss_cross_off, ss_rest_off;  // [n_super + 1], in items
  std::vector<int32_t> ss_cross, ss_rest;
  // The same items as pairs for the two-CTA (cta_group::2, M = 256) Schur
  // update: two targets (i1, j), (i2, j) of one tile column with the same
  // halves present share the B tiles; 8 ints per pair: target slot of the
  // even CTA, of the odd CTA (-1 for a single: the odd CTA then computes a
  // copy of the even CTA's product and discards it), then per step (2s, then
  // 2s+1) the staged A index of the even CTA, of the odd CTA and the shared
  // staged B index (all -1 when the step's half is absent).  Pairs are
  // ordered by (first target row, column) so that neighbouring pairs share
  // their A tiles.
  std::vector<int64_t> sp_cross_off, sp_rest_off;  // [n_super + 1], in pairs
  std::vector<int32_t> sp_cross, sp_rest;
  // Device copies.
  int32_t *d_perm = nullptr, *d_pinv = nullptr, *d_slot = nullptr;
  int32_t *d_lb_slot = nullptr, *d_ur_slot = nullptr, *d_ua_slot = nullptr, *d_ll_slot = nullptr;
  int32_t *d_lb_tile = nullptr, *d_ur_tile = nullptr, *d_ua_tile = nullptr, *d_ll_tile = nullptr;
  int32_t *d_sc_slot = nullptr, *d_diag_slot = nullptr;
  int32_t *d_ss_cross = nullptr, *d_ss_rest = nullptr;
  int32_t *d_sp_cross = nullptr, *d_sp_rest = nullptr;
  // Pattern copies for the shifted-value assembly (host and device).
  std::vector<int64_t> h_indptr;
  std::vector<int32_t> h_indices;
  bool uploaded = false;
  int64_t* d_indptr = nullptr;
  int32_t* d_indices = nullptr;
};

namespace aosb {
int plan_upload(aosb_plan* p, char* err, size_t cap);
void plan_free_device(aosb_plan* p);
void solve_graphs_forget(const aosb_plan* p);
void build_super_steps(aosb_plan* p);
}  // namespace aosb
