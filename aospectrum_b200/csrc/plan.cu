// Symbolic analysis, once per CSR pattern (host C++).
//
// 1. Supervariables: maximal runs of consecutive rows with identical column
//    sets in the symmetrised pattern (one per atom for AO bundles).
// 2. Ordering: nested dissection on the supervariable graph with
//    dof weights.  A part is split at a breadth-first level set started
//    from a pseudo-peripheral vertex; separator vertices that touch only one
//    side are moved to that side.  Parts below leaf_dofs become leaves.
// 3. Layout: the ordering nodes are laid out in elimination order; with
//    pad_nodes each node starts on a tile edge, so no tile mixes two nodes
//    and the tile-level fill follows the dissection tree exactly.  Padding
//    rows are decoupled identity rows.
// 4. Tile fill: symbolic elimination on the tile graph with row bitsets.
// 5. Step lists: for every tile step k the L tiles below, U tiles right,
//    U tiles above and L tiles left, and the |L_k| x |U_k| Schur targets.
#include "plan.h"

#include <unordered_map>

#include <algorithm>
#include <deque>
#include <map>
#include <tuple>
#include <numeric>
#include <vector>

namespace {

struct Graph {
  int64_t nv = 0;
  std::vector<int64_t> off;
  std::vector<int32_t> adj;
  std::vector<int64_t> w;  // dofs per vertex
};

// Breadth-first levels of the vertices in `mark == tag` reachable from s.
// Returns the vertices in visit order; level[v] is filled.
std::vector<int32_t> bfs(const Graph& g, int32_t s, const std::vector<int32_t>& mark, int32_t tag,
                         std::vector<int32_t>& level) {
  std::vector<int32_t> order;
  order.push_back(s);
  level[s] = 0;
  for (size_t h = 0; h < order.size(); ++h) {
    int32_t v = order[h];
    for (int64_t e = g.off[v]; e < g.off[v + 1]; ++e) {
      int32_t u = g.adj[e];
      if (mark[u] == tag && level[u] < 0) {
        level[u] = level[v] + 1;
        order.push_back(u);
      }
    }
  }
  return order;
}

struct Dissector {
  const Graph& g;
  int64_t leaf_dofs;
  std::vector<int32_t> mark, level;
  std::vector<std::vector<int32_t>> nodes;  // elimination-ordered nodes
  int32_t next_tag = 1;

  Dissector(const Graph& graph, int64_t leaf) : g(graph), leaf_dofs(leaf) {
    mark.assign(g.nv, 0);
    level.assign(g.nv, -1);
  }

  int64_t weight(const std::vector<int32_t>& vs) const {
    int64_t s = 0;
    for (int32_t v : vs) s += g.w[v];
    return s;
  }

  void run(std::vector<int32_t> verts) {
    // Explicit stack of work items: (vertex set, separator to emit after).
    struct Item {
      std::vector<int32_t> verts;
      std::vector<int32_t> sep;
      int stage;  // 0 = dissect, 1 = emit separator
    };
    std::vector<Item> stack;
    stack.push_back({std::move(verts), {}, 0});
    while (!stack.empty()) {
      Item it = std::move(stack.back());
      stack.pop_back();
      if (it.stage == 1) {
        if (!it.sep.empty()) nodes.push_back(std::move(it.sep));
        continue;
      }
      if (it.verts.empty()) continue;
      if (weight(it.verts) <= leaf_dofs) {
        nodes.push_back(std::move(it.verts));
        continue;
      }
      const int32_t tag = next_tag++;
      for (int32_t v : it.verts) {
        mark[v] = tag;
        level[v] = -1;
      }
      // Connected components.
      std::vector<std::vector<int32_t>> comps;
      for (int32_t v : it.verts) {
        if (level[v] >= 0) continue;
        comps.push_back(bfs(g, v, mark, tag, level));
      }
      if (comps.size() > 1) {
        // Independent components: push in reverse so the first is ordered first.
        for (auto c = comps.rbegin(); c != comps.rend(); ++c) stack.push_back({std::move(*c), {}, 0});
        continue;
      }
      std::vector<int32_t>& comp = comps[0];
      // Pseudo-peripheral start vertex: repeated BFS to the farthest vertex.
      int32_t s = comp.back();
      int last_depth = -1;
      for (int rep = 0; rep < 4; ++rep) {
        for (int32_t v : comp) level[v] = -1;
        auto ord = bfs(g, s, mark, tag, level);
        int depth = level[ord.back()];
        // farthest vertex with the smallest degree among the last level
        int32_t best = ord.back();
        int64_t bestdeg = g.off[best + 1] - g.off[best];
        for (auto r = ord.rbegin(); r != ord.rend() && level[*r] == depth; ++r) {
          int64_t d = g.off[*r + 1] - g.off[*r];
          if (d < bestdeg) { best = *r; bestdeg = d; }
        }
        if (depth <= last_depth) break;
        last_depth = depth;
        s = best;
      }
      for (int32_t v : comp) level[v] = -1;
      auto ord = bfs(g, s, mark, tag, level);
      const int depth = level[ord.back()];
      if (depth < 2) {
        // Too dense to separate: one leaf.
        nodes.push_back(std::move(comp));
        continue;
      }
      std::vector<int64_t> lw(depth + 1, 0);
      for (int32_t v : ord) lw[level[v]] += g.w[v];
      const int64_t total = std::accumulate(lw.begin(), lw.end(), (int64_t)0);
      // Candidate separator levels 1..depth-1 with balance in [0.2, 0.8];
      // choose the lightest, ties to the most balanced.
      int best_l = -1;
      double best_score = 1e300;
      int64_t before = lw[0];
      for (int l = 1; l < depth; ++l) {
        const int64_t after = total - before - lw[l];
        const double frac = (double)before / (double)(before + after);
        if (frac >= 0.2 && frac <= 0.8) {
          const double score = (double)lw[l] * (1.0 + 0.5 * std::abs(frac - 0.5));
          if (score < best_score) { best_score = score; best_l = l; }
        }
        before += lw[l];
      }
      if (best_l < 0) {
        // fall back to the median level
        int64_t acc = 0;
        for (int l = 0; l <= depth; ++l) {
          acc += lw[l];
          if (2 * acc >= total) { best_l = std::min(std::max(l, 1), depth - 1); break; }
        }
      }
      std::vector<int32_t> A, S, B;
      for (int32_t v : ord) {
        if (level[v] < best_l) A.push_back(v);
        else if (level[v] == best_l) S.push_back(v);
        else B.push_back(v);
      }
      // Refinement: separator vertices touching only one side join it.
      std::vector<int32_t> side(0);
      {
        // 1 = A, 2 = S, 3 = B using level as scratch label
        for (int32_t v : A) level[v] = 1;
        for (int32_t v : S) level[v] = 2;
        for (int32_t v : B) level[v] = 3;
        std::vector<int32_t> keep;
        for (int32_t v : S) {
          bool ta = false, tb = false;
          for (int64_t e = g.off[v]; e < g.off[v + 1]; ++e) {
            int32_t u = g.adj[e];
            if (mark[u] != tag) continue;
            if (level[u] == 1) ta = true;
            if (level[u] == 3) tb = true;
          }
          if (!tb) { level[v] = 1; A.push_back(v); }
          else if (!ta) { level[v] = 3; B.push_back(v); }
          else keep.push_back(v);
        }
        S.swap(keep);
      }
      if (A.empty() || B.empty()) {
        nodes.push_back(std::move(comp));
        continue;
      }
      // Order: A, then B, then S.
      stack.push_back({{}, std::move(S), 1});
      stack.push_back({std::move(B), {}, 0});
      stack.push_back({std::move(A), {}, 0});
    }
  }
};

}  // namespace

namespace aosb {

template <typename T>
static int up(T** dst, const std::vector<T>& src, char* err, size_t cap) {
  size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(T);
  cudaError_t e = cudaMalloc((void**)dst, bytes);
  if (e != cudaSuccess)
    return set_error(err, cap, AOSB_ERR_MEMORY, "cudaMalloc(%zu) failed: %s", bytes,
                     cudaGetErrorString(e));
  if (!src.empty()) {
    e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
      return set_error(err, cap, AOSB_ERR_CUDA, "cudaMemcpy failed: %s", cudaGetErrorString(e));
  }
  return 0;
}

int plan_upload(aosb_plan* p, char* err, size_t cap) {
  int rc = 0;
  if ((rc = up(&p->d_perm, p->perm, err, cap)) || (rc = up(&p->d_pinv, p->pinv, err, cap)) ||
      (rc = up(&p->d_slot, p->slot, err, cap)) || (rc = up(&p->d_lb_slot, p->lb_slot, err, cap)) ||
      (rc = up(&p->d_ur_slot, p->ur_slot, err, cap)) ||
      (rc = up(&p->d_ua_slot, p->ua_slot, err, cap)) ||
      (rc = up(&p->d_ll_slot, p->ll_slot, err, cap)) ||
      (rc = up(&p->d_lb_tile, p->lb_tile, err, cap)) ||
      (rc = up(&p->d_ur_tile, p->ur_tile, err, cap)) ||
      (rc = up(&p->d_ua_tile, p->ua_tile, err, cap)) ||
      (rc = up(&p->d_ll_tile, p->ll_tile, err, cap)) ||
      (rc = up(&p->d_sc_slot, p->sc_slot, err, cap)) ||
      (rc = up(&p->d_diag_slot, p->diag_slot, err, cap)))
    return rc;
  return 0;
}

// Two-step Schur item lists (see plan.h).
void build_super_steps(aosb_plan* P) {
  const int64_t nb = P->nb;
  P->ss_cross_off.assign(1, 0);
  P->ss_rest_off.assign(1, 0);
  P->ss_cross.clear();
  P->ss_rest.clear();
  P->sp_cross_off.assign(1, 0);
  P->sp_rest_off.assign(1, 0);
  P->sp_cross.clear();
  P->sp_rest.clear();
  struct Item {
    int32_t i, j, slot, a0, b0, a1, b1;
  };
  std::vector<Item> items;
  for (int64_t k0 = 0; k0 + 1 < nb; k0 += 2) {
    const int64_t k1 = k0 + 1, k2 = k0 + 2, k3 = k0 + 3;
    items.clear();
    const int32_t l0 = P->lb_off[k0], nL0 = P->lb_off[k0 + 1] - l0;
    const int32_t u0 = P->ur_off[k0], nU0 = P->ur_off[k0 + 1] - u0;
    const int32_t l1 = P->lb_off[k1], nL1 = P->lb_off[k1 + 1] - l1;
    const int32_t u1 = P->ur_off[k1], nU1 = P->ur_off[k1 + 1] - u1;
    // dense index over the (i, j) targets of this super-step: i, j in
    // [k2, nb) -> item position
    std::unordered_map<int64_t, int32_t> at;
    at.reserve((size_t)(nL0 * nU0 + nL1 * nU1) * 2 + 16);
    auto get = [&](int32_t i, int32_t j) -> Item& {
      const int64_t key = (int64_t)i * nb + j;
      auto f = at.find(key);
      if (f != at.end()) return items[f->second];
      at.emplace(key, (int32_t)items.size());
      items.push_back({i, j, P->slot[key], -1, -1, -1, -1});
      return items.back();
    };
    for (int32_t a = 0; a < nL0; ++a) {
      const int32_t i = P->lb_tile[l0 + a];
      if (i == k1) continue;
      for (int32_t b = 0; b < nU0; ++b) {
        const int32_t j = P->ur_tile[u0 + b];
        if (j == k1) continue;
        Item& it = get(i, j);
        it.a0 = a;
        it.b0 = nL0 + b;
      }
    }
    for (int32_t a = 0; a < nL1; ++a) {
      const int32_t i = P->lb_tile[l1 + a];
      for (int32_t b = 0; b < nU1; ++b) {
        const int32_t j = P->ur_tile[u1 + b];
        Item& it = get(i, j);
        it.a1 = a;
        it.b1 = nL1 + b;
      }
    }
    std::sort(items.begin(), items.end(), [](const Item& x, const Item& y) {
      return x.i != y.i ? x.i < y.i : x.j < y.j;
    });
    for (const Item& it : items) {
      const bool cross = it.i == k2 || it.i == k3 || it.j == k2 || it.j == k3;
      std::vector<int32_t>& dst = cross ? P->ss_cross : P->ss_rest;
      dst.insert(dst.end(), {it.slot, it.a0, it.b0, it.a1, it.b1});
    }
    P->ss_cross_off.push_back((int64_t)P->ss_cross.size() / 5);
    P->ss_rest_off.push_back((int64_t)P->ss_rest.size() / 5);
    // pairs: group each list's items by (column, halves present), pair them
    // in row order, then order the pairs by (first row, column)
    for (int list = 0; list < 2; ++list) {
      std::map<std::tuple<int32_t, bool, bool>, std::vector<const Item*>> groups;
      for (const Item& it : items) {
        const bool cross = it.i == k2 || it.i == k3 || it.j == k2 || it.j == k3;
        if (cross != (list == 0)) continue;
        groups[std::make_tuple(it.j, it.a0 >= 0, it.a1 >= 0)].push_back(&it);
      }
      std::vector<std::pair<const Item*, const Item*>> pairs;
      for (auto& g : groups)
        for (size_t t = 0; t < g.second.size(); t += 2)
          pairs.emplace_back(g.second[t], t + 1 < g.second.size() ? g.second[t + 1] : nullptr);
      std::sort(pairs.begin(), pairs.end(), [](const auto& x, const auto& y) {
        return x.first->i != y.first->i ? x.first->i < y.first->i : x.first->j < y.first->j;
      });
      std::vector<int32_t>& dst = list == 0 ? P->sp_cross : P->sp_rest;
      for (const auto& pr : pairs) {
        const Item& e = *pr.first;
        const Item& o = pr.second ? *pr.second : *pr.first;
        dst.insert(dst.end(), {e.slot, pr.second ? o.slot : -1, e.a0, o.a0, e.b0, e.a1, o.a1,
                               e.b1});
      }
    }
    P->sp_cross_off.push_back((int64_t)P->sp_cross.size() / 8);
    P->sp_rest_off.push_back((int64_t)P->sp_rest.size() / 8);
  }
}

void plan_free_device(aosb_plan* p) {
  int32_t** arrs[] = {&p->d_perm, &p->d_pinv, &p->d_slot, &p->d_lb_slot, &p->d_ur_slot,
                      &p->d_ua_slot, &p->d_ll_slot, &p->d_lb_tile, &p->d_ur_tile,
                      &p->d_ua_tile, &p->d_ll_tile, &p->d_sc_slot, &p->d_diag_slot,
                      &p->d_indices, &p->d_ss_cross, &p->d_ss_rest, &p->d_sp_cross,
                      &p->d_sp_rest};
  for (int32_t** a : arrs) {
    if (*a) cudaFree(*a);
    *a = nullptr;
  }
  if (p->d_indptr) cudaFree(p->d_indptr);
  p->d_indptr = nullptr;
  p->uploaded = false;
}

}  // namespace aosb

extern "C" {

int aosb_plan_create(int64_t n, const int64_t* indptr, const int32_t* indices,
                     const int64_t* sv_offsets, int64_t n_sv_in,
                     const aosb_plan_options_v1* opt, aosb_plan_t** out, char* err, size_t cap) {
  using aosb::set_error;
  if (out == nullptr || indptr == nullptr || indices == nullptr || opt == nullptr)
    return set_error(err, cap, AOSB_ERR_NULL, "required pointer is null");
  *out = nullptr;
  if (opt->abi_version != AOSPECTRUM_B200_ABI_VERSION || opt->struct_size != sizeof(*opt))
    return set_error(err, cap, AOSB_ERR_ABI, "plan options ABI mismatch");
  const int64_t T = opt->tile;
  if (T != 32 && T != 64 && T != 128)
    return set_error(err, cap, AOSB_ERR_ARGUMENT, "tile must be 32, 64 or 128");
  if (n <= 0 || n > INT32_MAX / 2)
    return set_error(err, cap, AOSB_ERR_DIMS, "invalid matrix dimension");
  const int64_t nnz = indptr[n];
  if (indptr[0] != 0 || nnz <= 0)
    return set_error(err, cap, AOSB_ERR_INDPTR, "CSR row offsets do not span the declared nnz");
  for (int64_t r = 0; r < n; ++r) {
    if (indptr[r + 1] < indptr[r])
      return set_error(err, cap, AOSB_ERR_CSR_MONOTONIC, "CSR row offsets are not monotonic");
    bool diag = false;
    for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) {
      if (indices[e] < 0 || indices[e] >= n)
        return set_error(err, cap, AOSB_ERR_CSR_COLUMN, "CSR column index is outside the matrix");
      if (e > indptr[r] && indices[e] <= indices[e - 1])
        return set_error(err, cap, AOSB_ERR_CSR_ORDER, "CSR columns must be sorted and duplicate-free");
      diag |= indices[e] == r;
    }
    if (!diag)
      return set_error(err, cap, AOSB_ERR_DIAGONAL, "matrix row %lld has no diagonal entry",
                       (long long)r);
  }
  // Symmetrised pattern (rows of A + A^T).
  std::vector<int64_t> soff(n + 1, 0);
  std::vector<int32_t> sadj;
  {
    std::vector<int64_t> cnt(n, 0);
    for (int64_t r = 0; r < n; ++r)
      for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) {
        cnt[r]++;
        cnt[indices[e]]++;
      }
    for (int64_t r = 0; r < n; ++r) soff[r + 1] = soff[r] + cnt[r];
    sadj.resize(soff[n]);
    std::vector<int64_t> pos(soff.begin(), soff.end() - 1);
    for (int64_t r = 0; r < n; ++r)
      for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) {
        sadj[pos[r]++] = indices[e];
        sadj[pos[indices[e]]++] = (int32_t)r;
      }
    int64_t w = 0;
    std::vector<int64_t> noff(n + 1, 0);
    for (int64_t r = 0; r < n; ++r) {
      auto b = sadj.begin() + soff[r], e = sadj.begin() + soff[r + 1];
      std::sort(b, e);
      auto u = std::unique(b, e);
      for (auto it = b; it != u; ++it) sadj[w++] = *it;
      noff[r + 1] = w;
    }
    sadj.resize(w);
    soff.swap(noff);
  }
  // Supervariables.
  std::vector<int64_t> sv;
  if (sv_offsets != nullptr && n_sv_in > 0) {
    if (sv_offsets[0] != 0 || sv_offsets[n_sv_in] != n)
      return set_error(err, cap, AOSB_ERR_ARGUMENT, "supervariable offsets must span 0..n");
    sv.assign(sv_offsets, sv_offsets + n_sv_in + 1);
  } else {
    sv.push_back(0);
    for (int64_t r = 1; r < n; ++r) {
      const int64_t la = soff[r] - soff[r - 1], lb = soff[r + 1] - soff[r];
      bool same = la == lb && std::equal(sadj.begin() + soff[r - 1], sadj.begin() + soff[r],
                                         sadj.begin() + soff[r]);
      if (!same) sv.push_back(r);
    }
    sv.push_back(n);
  }
  const int64_t nsv = (int64_t)sv.size() - 1;
  std::vector<int32_t> sv_of(n);
  for (int64_t s = 0; s < nsv; ++s)
    for (int64_t r = sv[s]; r < sv[s + 1]; ++r) sv_of[r] = (int32_t)s;
  // Supervariable graph (union over the rows of each supervariable).
  Graph g;
  g.nv = nsv;
  g.off.assign(nsv + 1, 0);
  g.w.resize(nsv);
  {
    std::vector<int32_t> stamp(nsv, -1);
    for (int64_t s = 0; s < nsv; ++s) {
      g.w[s] = sv[s + 1] - sv[s];
      for (int64_t r = sv[s]; r < sv[s + 1]; ++r)
        for (int64_t e = soff[r]; e < soff[r + 1]; ++e) {
          int32_t t = sv_of[sadj[e]];
          if (t != s && stamp[t] != (int32_t)s) {
            stamp[t] = (int32_t)s;
            g.adj.push_back(t);
          }
        }
      g.off[s + 1] = (int64_t)g.adj.size();
      std::sort(g.adj.begin() + g.off[s], g.adj.end());
    }
  }
  // Ordering nodes.
  std::vector<std::vector<int32_t>> nodes;
  if (opt->ordering == 1) {
    Dissector d(g, std::max<int64_t>(opt->leaf_dofs, 1));
    std::vector<int32_t> all(nsv);
    std::iota(all.begin(), all.end(), 0);
    d.run(std::move(all));
    nodes = std::move(d.nodes);
  } else {
    std::vector<int32_t> all(nsv);
    std::iota(all.begin(), all.end(), 0);
    nodes.push_back(std::move(all));
  }
  auto* P = new aosb_plan();
  P->n = n;
  P->nnz = nnz;
  P->T = T;
  P->n_sv = nsv;
  P->n_nodes = (int64_t)nodes.size();
  // Layout with optional padding.
  {
    std::vector<int32_t> perm;
    for (const auto& node : nodes) {
      if (opt->pad_nodes)
        while (perm.size() % T) perm.push_back(-1);
      for (int32_t s : node)
        for (int64_t r = sv[s]; r < sv[s + 1]; ++r) perm.push_back((int32_t)r);
    }
    while (perm.size() % T) perm.push_back(-1);
    P->perm = std::move(perm);
  }
  P->n_pad = (int64_t)P->perm.size();
  P->nb = P->n_pad / T;
  const int64_t nb = P->nb;
  P->pinv.assign(n, -1);
  for (int64_t i = 0; i < P->n_pad; ++i)
    if (P->perm[i] >= 0) P->pinv[P->perm[i]] = (int32_t)i;
  P->real_dofs.assign(nb, 0);
  for (int64_t i = 0; i < P->n_pad; ++i)
    if (P->perm[i] >= 0) P->real_dofs[i / T]++;
  // Tile pattern of A (symmetrised) with row bitsets.
  const int64_t words = (nb + 63) / 64;
  std::vector<uint64_t> bits(nb * words, 0);
  auto setb = [&](int64_t i, int64_t j) { bits[i * words + (j >> 6)] |= 1ull << (j & 63); };
  auto getb = [&](int64_t i, int64_t j) { return (bits[i * words + (j >> 6)] >> (j & 63)) & 1ull; };
  for (int64_t k = 0; k < nb; ++k) setb(k, k);
  for (int64_t s = 0; s < nsv; ++s) {
    // tiles spanned by supervariable s
    int64_t lo = INT64_MAX, hi = -1;
    for (int64_t r = sv[s]; r < sv[s + 1]; ++r) {
      lo = std::min<int64_t>(lo, P->pinv[r] / T);
      hi = std::max<int64_t>(hi, P->pinv[r] / T);
    }
    auto mark_pair = [&](int64_t t) {
      int64_t lo2 = INT64_MAX, hi2 = -1;
      for (int64_t r = sv[t]; r < sv[t + 1]; ++r) {
        lo2 = std::min<int64_t>(lo2, P->pinv[r] / T);
        hi2 = std::max<int64_t>(hi2, P->pinv[r] / T);
      }
      for (int64_t a = lo; a <= hi; ++a)
        for (int64_t b = lo2; b <= hi2; ++b) {
          setb(a, b);
          setb(b, a);
        }
    };
    mark_pair(s);
    for (int64_t e = g.off[s]; e < g.off[s + 1]; ++e) mark_pair(g.adj[e]);
  }
  // Symbolic elimination on tiles (symmetric structure).
  {
    std::vector<uint64_t> col(words);
    for (int64_t k = 0; k < nb; ++k) {
      // col = row k restricted to indices > k
      for (int64_t w = 0; w < words; ++w) col[w] = bits[k * words + w];
      for (int64_t j = 0; j <= k; ++j) col[j >> 6] &= ~(1ull << (j & 63));
      for (int64_t w = 0; w < words; ++w) {
        uint64_t m = col[w];
        while (m) {
          int b = __builtin_ctzll(m);
          m &= m - 1;
          int64_t i = w * 64 + b;
          uint64_t* row = &bits[i * words];
          for (int64_t x = 0; x < words; ++x) row[x] |= col[x];
        }
      }
    }
  }
  // Slots (row-major) and lists.
  P->slot.assign(nb * nb, -1);
  int64_t ns = 0;
  for (int64_t i = 0; i < nb; ++i)
    for (int64_t j = 0; j < nb; ++j)
      if (getb(i, j)) P->slot[i * nb + j] = (int32_t)ns++;
  P->n_slots = ns;
  P->diag_slot.resize(nb);
  P->lb_off.assign(1, 0);
  P->ur_off.assign(1, 0);
  P->ua_off.assign(1, 0);
  P->ll_off.assign(1, 0);
  P->sc_off.assign(1, 0);
  std::vector<int32_t> parent(nb, -1);
  const double T3 = (double)T * T * T;
  for (int64_t k = 0; k < nb; ++k) {
    P->diag_slot[k] = P->slot[k * nb + k];
    for (int64_t i = 0; i < nb; ++i) {
      if (i == k) continue;
      if (getb(i, k)) {
        if (i > k) { P->lb_tile.push_back((int32_t)i); P->lb_slot.push_back(P->slot[i * nb + k]); }
        else { P->ua_tile.push_back((int32_t)i); P->ua_slot.push_back(P->slot[i * nb + k]); }
      }
      if (getb(k, i)) {
        if (i > k) { P->ur_tile.push_back((int32_t)i); P->ur_slot.push_back(P->slot[k * nb + i]); }
        else { P->ll_tile.push_back((int32_t)i); P->ll_slot.push_back(P->slot[k * nb + i]); }
      }
    }
    const int64_t l0 = P->lb_off.back(), l1 = (int64_t)P->lb_tile.size();
    const int64_t u0 = P->ur_off.back(), u1 = (int64_t)P->ur_tile.size();
    double rl = 0, ru = 0;
    for (int64_t a = l0; a < l1; ++a) {
      rl += P->real_dofs[P->lb_tile[a]];
      for (int64_t b = u0; b < u1; ++b) {
        int32_t s = P->slot[(int64_t)P->lb_tile[a] * nb + P->ur_tile[b]];
        if (s < 0) {
          delete P;
          return set_error(err, cap, AOSB_ERR_ENGINE, "symbolic fill is inconsistent");
        }
        P->sc_slot.push_back(s);
      }
    }
    for (int64_t b = u0; b < u1; ++b) ru += P->real_dofs[P->ur_tile[b]];
    if (l1 > l0) parent[k] = P->lb_tile[l0];
    const double nl = (double)(l1 - l0), nu = (double)(u1 - u0);
    P->flops += 8.0 * (T3 / 3.0 + (nl + nu) * T3 / 2.0 + nl * nu * T3);
    const double d = P->real_dofs[k];
    P->flops_alg += 8.0 * (d * d * d / 3.0 + d * d * (rl + ru) / 2.0 + d * rl * ru);
    P->schur_updates += (l1 - l0) * (u1 - u0);
    P->lb_off.push_back((int32_t)l1);
    P->ur_off.push_back((int32_t)u1);
    P->ua_off.push_back((int32_t)P->ua_tile.size());
    P->ll_off.push_back((int32_t)P->ll_tile.size());
    P->sc_off.push_back((int64_t)P->sc_slot.size());
  }
  // Tree levels of the tile elimination tree.
  {
    std::vector<int32_t> lev(nb, 0);
    int32_t mx = 0;
    for (int64_t k = 0; k < nb; ++k) {
      if (parent[k] >= 0) lev[parent[k]] = std::max(lev[parent[k]], lev[k] + 1);
      mx = std::max(mx, lev[k]);
    }
    P->tree_levels = mx + 1;
  }
  aosb::build_super_steps(P);
  P->h_indptr.assign(indptr, indptr + n + 1);
  P->h_indices.assign(indices, indices + nnz);
  *out = P;
  return 0;
}

int aosb_plan_upload(aosb_plan_t* P, char* err, size_t cap) {
  if (P == nullptr) return aosb::set_error(err, cap, AOSB_ERR_NULL, "null plan");
  if (P->uploaded) return 0;
  int rc = aosb::plan_upload(P, err, cap);
  if (rc == 0) rc = aosb::up(&P->d_indptr, P->h_indptr, err, cap);
  if (rc == 0 && !P->ss_cross.empty()) rc = aosb::up(&P->d_ss_cross, P->ss_cross, err, cap);
  if (rc == 0 && !P->ss_rest.empty()) rc = aosb::up(&P->d_ss_rest, P->ss_rest, err, cap);
  if (rc == 0 && !P->sp_cross.empty()) rc = aosb::up(&P->d_sp_cross, P->sp_cross, err, cap);
  if (rc == 0 && !P->sp_rest.empty()) rc = aosb::up(&P->d_sp_rest, P->sp_rest, err, cap);
  if (rc == 0) rc = aosb::up(&P->d_indices, P->h_indices, err, cap);
  if (rc != 0) {
    aosb::plan_free_device(P);
    return rc;
  }
  P->uploaded = true;
  return 0;
}

int aosb_plan_info(const aosb_plan_t* p, aosb_plan_info_v1* info) {
  if (p == nullptr || info == nullptr) return AOSB_ERR_NULL;
  std::memset(info, 0, sizeof(*info));
  info->n = p->n;
  info->n_pad = p->n_pad;
  info->nnz = p->nnz;
  info->n_tiles = p->nb;
  info->n_slots = p->n_slots;
  info->n_supervariables = p->n_sv;
  info->n_nodes = p->n_nodes;
  info->schur_tile_updates = p->schur_updates;
  info->tree_levels = p->tree_levels;
  info->tile = (int32_t)p->T;
  info->factor_flops = p->flops;
  info->factor_flops_alg = p->flops_alg;
  info->factor_bytes = (double)p->n_slots * (double)(p->T * p->T) * 8.0;
  return 0;
}

int aosb_plan_export_perm(const aosb_plan_t* p, int32_t* perm) {
  if (p == nullptr || perm == nullptr) return AOSB_ERR_NULL;
  std::copy(p->perm.begin(), p->perm.end(), perm);
  return 0;
}

int aosb_plan_export_slots(const aosb_plan_t* p, int32_t* slot) {
  if (p == nullptr || slot == nullptr) return AOSB_ERR_NULL;
  std::copy(p->slot.begin(), p->slot.end(), slot);
  return 0;
}

int aosb_plan_export_super_steps(const aosb_plan_t* p, int64_t* n_super, int64_t* n_cross,
                                 int64_t* n_rest, int64_t* cross_off, int64_t* rest_off,
                                 int32_t* cross, int32_t* rest) {
  if (p == nullptr) return AOSB_ERR_NULL;
  if (n_super) *n_super = (int64_t)p->ss_cross_off.size() - 1;
  if (n_cross) *n_cross = (int64_t)p->ss_cross.size() / 5;
  if (n_rest) *n_rest = (int64_t)p->ss_rest.size() / 5;
  if (cross_off) std::copy(p->ss_cross_off.begin(), p->ss_cross_off.end(), cross_off);
  if (rest_off) std::copy(p->ss_rest_off.begin(), p->ss_rest_off.end(), rest_off);
  if (cross) std::copy(p->ss_cross.begin(), p->ss_cross.end(), cross);
  if (rest) std::copy(p->ss_rest.begin(), p->ss_rest.end(), rest);
  return 0;
}

int aosb_plan_export_pair_steps(const aosb_plan_t* p, int64_t* n_cross, int64_t* n_rest,
                                int64_t* cross_off, int64_t* rest_off, int32_t* cross,
                                int32_t* rest) {
  if (p == nullptr) return AOSB_ERR_NULL;
  if (n_cross) *n_cross = (int64_t)p->sp_cross.size() / 8;
  if (n_rest) *n_rest = (int64_t)p->sp_rest.size() / 8;
  if (cross_off) std::copy(p->sp_cross_off.begin(), p->sp_cross_off.end(), cross_off);
  if (rest_off) std::copy(p->sp_rest_off.begin(), p->sp_rest_off.end(), rest_off);
  if (cross) std::copy(p->sp_cross.begin(), p->sp_cross.end(), cross);
  if (rest) std::copy(p->sp_rest.begin(), p->sp_rest.end(), rest);
  return 0;
}

void aosb_plan_destroy(aosb_plan_t* p) {
  if (p == nullptr) return;
  aosb::solve_graphs_forget(p);
  aosb::plan_free_device(p);
  delete p;
}

}  // extern "C"
