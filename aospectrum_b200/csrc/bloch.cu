// Bloch pattern (host, once per bundle) and Bloch sum (device, per k).
//
// The reference expands every block entry into (row, col, source, phase)
// tuples and argsorts them (src/aospectrum/sparse.py:64-140), then per k
// gathers, multiplies and segment-sums them (sparse.py:181-245).  Here the
// pattern is built at block granularity: blocks with the same atom pair
// (i, j) form one "group" whose entries land in the same 2D window of the
// CSR arrays, because every row of atom i has the same column structure.
// Entry (a, c) of group (i, j) sits at dst_base + a * rowlen_i + c.
//
// The device kernel gives one warp to each group (window) and chunk of up
// to four k points: it sums the member blocks of (i, j) and of its mirror
// (j, i) in block order (the order the reference's stable sort leaves them
// in), applies the Hermitian projection of sparse.py:25-36 and writes the
// window row by row for every k point of the chunk.  With
// real block values the products v * phase are exact, so the output is
// bit-identical to the reference's numpy path.
#include "common.cuh"
#include "timing.h"

#include <algorithm>
#include <numeric>
#include <vector>

struct aosb_bloch {
  int64_t n = 0, n_atoms = 0, n_blocks = 0, nnz = 0;
  std::vector<int64_t> indptr;
  std::vector<int32_t> indices;
  std::vector<int32_t> shifts;       // n_shifts * 3
  std::vector<int32_t> block_shift;  // n_blocks
  // device tables
  int64_t n_groups = 0, n_members = 0;
  int64_t* d_indptr = nullptr;
  int32_t* d_indices = nullptr;
  int4* d_group = nullptr;        // (nr, nc, rowlen, mirror)
  int64_t* d_group_dst = nullptr;  // dst base
  int2* d_group_members = nullptr; // [begin, end) into members
  int64_t* d_member_off = nullptr; // value offset of each member block
  int32_t* d_member_shift = nullptr;
  // host copies of the device tables (uploaded by aosb_bloch_upload)
  std::vector<int4> g_info;
  std::vector<int64_t> g_dst;
  std::vector<int2> g_mem;
  std::vector<int64_t> m_off;
  std::vector<int32_t> m_shift;
  int64_t n_values = 0;  // stored block values (sum of block sizes), set at upload
  bool uploaded = false;
};

namespace {

template <typename T>
int upload(T** dst, const std::vector<T>& src, char* err, size_t cap) {
  size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(T);
  cudaError_t e = cudaMalloc((void**)dst, bytes);
  if (e != cudaSuccess)
    return aosb::set_error(err, cap, AOSB_ERR_MEMORY, "cudaMalloc(%zu) failed: %s", bytes,
                           cudaGetErrorString(e));
  if (!src.empty()) {
    e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
      return aosb::set_error(err, cap, AOSB_ERR_CUDA, "cudaMemcpy failed: %s",
                             cudaGetErrorString(e));
  }
  return 0;
}

template <typename V>
__device__ __forceinline__ float2 load_value(const V* v, int64_t i);
template <>
__device__ __forceinline__ float2 load_value<float>(const float* v, int64_t i) {
  return make_float2(v[i], 0.0f);
}
template <>
__device__ __forceinline__ float2 load_value<float2>(const float2* v, int64_t i) {
  return v[i];
}

// Complex product without FMA contraction, matching a plain
// (ac - bd, ad + bc) evaluation in float32.
__device__ __forceinline__ float2 cmul_rn(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// k points per warp: one warp reads its blocks once and writes this many
// H(k), S(k) windows (four keeps the kernel at 64 registers, 32 warps per SM)
constexpr int kBlochKChunk = 4;

// Sums of one element over the member blocks [range.x, range.y) of a group
// for the k points k0 .. k0+nk-1 (nk <= kBlochKChunk): each member value is
// loaded once and multiplied by the phase of its lattice shift at every k.
// Members are added in block order, first product first, for every k.
template <typename V>
__device__ __forceinline__ void group_sums(const V* vals, const int64_t* moff, const int32_t* msh,
                                           const float2* ph0, int64_t n_shifts, int nk,
                                           int2 range, int64_t elem,
                                           float2 (&s)[kBlochKChunk]) {
#pragma unroll
  for (int q = 0; q < kBlochKChunk; ++q) s[q] = make_float2(0.0f, 0.0f);
  for (int m = range.x; m < range.y; ++m) {
    const float2 v = load_value<V>(vals, moff[m] + elem);
    const float2* ph = ph0 + msh[m];
#pragma unroll
    for (int q = 0; q < kBlochKChunk; ++q) {
      if (q < nk) {
        const float2 p = cmul_rn(v, ph[q * n_shifts]);
        if (m == range.x) {
          s[q] = p;
        } else {
          s[q].x = __fadd_rn(s[q].x, p.x);
          s[q].y = __fadd_rn(s[q].y, p.y);
        }
      }
    }
  }
}

__device__ __forceinline__ float2 hermitian_mean(float2 x, float2 y) {
  return make_float2(__fmul_rn(__fadd_rn(x.x, y.x), 0.5f), __fmul_rn(__fsub_rn(x.y, y.y), 0.5f));
}

// One warp per group (i, j) writes that group's window.  Groups are sorted by
// (row atom, column atom), so the 8 warps of a CTA write neighbouring windows
// of the same CSR rows at the same time and the 32-byte sectors they share
// at window boundaries are completed in L2 instead of leaving it partly
// written.  Element (a, c) of window (i, j) and element (c, a) of its mirror
// (j, i) hold the Hermitian mean of the pair and its conjugate: the upper
// window (i < j) writes mean(x_ij(a, c), x_ji(c, a)), the lower window writes
// the conjugate of its upper mirror's mean formed the same way.
template <typename V>
__global__ void __launch_bounds__(256, 4) bloch_windows_kernel(
    int64_t n_groups, const int4* __restrict__ group, const int64_t* __restrict__ gdst,
    const int2* __restrict__ gmem, const int64_t* __restrict__ moff,
    const int32_t* __restrict__ msh, const V* __restrict__ hv, const V* __restrict__ sv,
    const float2* __restrict__ phases, int64_t n_shifts, int64_t nnz, int n_k,
    float2* __restrict__ hout, float2* __restrict__ sout) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (warp >= n_groups) return;
  const int k0 = blockIdx.y * kBlochKChunk;
  const int nk = min(n_k - k0, kBlochKChunk);
  const float2* ph0 = phases + (int64_t)k0 * n_shifts;
  const int64_t out0 = (int64_t)k0 * nnz;
  const int g = (int)warp;
  const int4 gi = group[g];  // nr, nc, rowlen, mirror
  const int nr = gi.x, nc = gi.y, rl = gi.z, gm = gi.w;
  const int ne = nr * nc;
  const int64_t base = gdst[g];
  const int2 rg = gmem[g];
  float2 x[kBlochKChunk], y[kBlochKChunk];
  if (gm == g) {
    // diagonal window: t runs over [matrix H|S][row-major element]; the mean
    // of the pair (lo, hi) is formed the same way for both of its entries
    for (int t = lane; t < 2 * ne; t += 32) {
      const int which = t >= ne;
      const int e = t - which * ne;
      const int a = e / nc, c = e - (e / nc) * nc;
      const V* vals = which == 0 ? hv : sv;
      float2* out = (which == 0 ? hout : sout) + out0 + base + (int64_t)a * rl + c;
      const int lo = min(a, c), hi = max(a, c);
      group_sums<V>(vals, moff, msh, ph0, n_shifts, nk, rg, lo * nc + hi, x);
      if (a != c) group_sums<V>(vals, moff, msh, ph0, n_shifts, nk, rg, hi * nc + lo, y);
#pragma unroll
      for (int q = 0; q < kBlochKChunk; ++q) {
        if (q < nk) {
          float2 v;
          if (a == c) {
            v = make_float2(x[q].x, 0.0f);
          } else {
            const float2 mean = hermitian_mean(x[q], y[q]);
            v = a < c ? mean : make_float2(mean.x, -mean.y);
          }
          out[q * nnz] = v;
        }
      }
    }
    return;
  }
  const bool lower = gm < g;
  const int2 mr = gmem[gm];
  // the mean's first operand comes from the upper group of the pair
  const int2 r1 = lower ? mr : rg, r2 = lower ? rg : mr;
  if (r1.y - r1.x == 1 && r2.y - r2.x == 1) {
    // One member block each way (a single lattice image, the common case):
    // value offsets and phases are warp-uniform and loaded once; each lane
    // keeps two elements' value loads in flight.
    const int64_t o1 = moff[r1.x], o2 = moff[r2.x];
    const float2* ph1 = ph0 + msh[r1.x];
    const float2* ph2 = ph0 + msh[r2.x];
    float2 p1[kBlochKChunk], p2[kBlochKChunk];
#pragma unroll
    for (int q = 0; q < kBlochKChunk; ++q) {
      p1[q] = q < nk ? ph1[q * n_shifts] : make_float2(0.0f, 0.0f);
      p2[q] = q < nk ? ph2[q * n_shifts] : make_float2(0.0f, 0.0f);
    }
    for (int t0 = lane; t0 < 2 * ne; t0 += 64) {
      float2 v1[2], v2[2];
      float2* out[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int t = t0 + 32 * u;
        out[u] = nullptr;
        v1[u] = v2[u] = make_float2(0.0f, 0.0f);
        if (t < 2 * ne) {
          const int which = t >= ne;
          const int e = t - which * ne;
          const int a = e / nc, c = e - a * nc;
          const int eg = a * nc + c, em = c * nr + a;
          const V* vals = which == 0 ? hv : sv;
          out[u] = (which == 0 ? hout : sout) + out0 + base + (int64_t)a * rl + c;
          v1[u] = load_value<V>(vals, o1 + (lower ? em : eg));
          v2[u] = load_value<V>(vals, o2 + (lower ? eg : em));
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (out[u] == nullptr) continue;
#pragma unroll
        for (int q = 0; q < kBlochKChunk; ++q) {
          if (q < nk) {
            const float2 mean = hermitian_mean(cmul_rn(v1[u], p1[q]), cmul_rn(v2[u], p2[q]));
            out[u][q * nnz] = lower ? make_float2(mean.x, -mean.y) : mean;
          }
        }
      }
    }
    return;
  }
  // general: t runs over [matrix H|S][row-major element]
  for (int t = lane; t < 2 * ne; t += 32) {
    const int which = t >= ne;
    const int e = t - which * ne;
    const int a = e / nc, c = e - a * nc;
    const int eg = a * nc + c, em = c * nr + a;
    const V* vals = which == 0 ? hv : sv;
    float2* out = (which == 0 ? hout : sout) + out0 + base + (int64_t)a * rl + c;
    group_sums<V>(vals, moff, msh, ph0, n_shifts, nk, r1, lower ? em : eg, x);
    group_sums<V>(vals, moff, msh, ph0, n_shifts, nk, r2, lower ? eg : em, y);
#pragma unroll
    for (int q = 0; q < kBlochKChunk; ++q) {
      if (q < nk) {
        const float2 mean = hermitian_mean(x[q], y[q]);
        out[q * nnz] = lower ? make_float2(mean.x, -mean.y) : mean;
      }
    }
  }
}

}  // namespace

extern "C" {

int aosb_bloch_create(int64_t n_orbitals, int64_t n_atoms, const int64_t* atom_offsets,
                      int64_t n_blocks, const int32_t* row_atom, const int32_t* col_atom,
                      const int32_t* lattice_shift, const int64_t* block_offsets,
                      aosb_bloch_t** out, char* err, size_t cap) {
  if (out == nullptr || atom_offsets == nullptr || row_atom == nullptr || col_atom == nullptr ||
      lattice_shift == nullptr || block_offsets == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "required pointer is null");
  *out = nullptr;
  if (n_orbitals <= 0 || n_atoms <= 0 || n_blocks <= 0 || atom_offsets[n_atoms] != n_orbitals)
    return aosb::set_error(err, cap, AOSB_ERR_DIMS, "invalid bundle dimensions");
  for (int64_t b = 0; b < n_blocks; ++b) {
    if (row_atom[b] < 0 || row_atom[b] >= n_atoms || col_atom[b] < 0 || col_atom[b] >= n_atoms)
      return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "block %lld references an unknown atom",
                             (long long)b);
    const int64_t nr = atom_offsets[row_atom[b] + 1] - atom_offsets[row_atom[b]];
    const int64_t nc = atom_offsets[col_atom[b] + 1] - atom_offsets[col_atom[b]];
    if (block_offsets[b + 1] - block_offsets[b] != nr * nc)
      return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "block %lld size mismatch", (long long)b);
  }
  auto* B = new aosb_bloch();
  B->n = n_orbitals;
  B->n_atoms = n_atoms;
  B->n_blocks = n_blocks;

  // Distinct lattice shifts, lexicographic (the order numpy.unique(axis=0) gives).
  std::vector<int64_t> sidx(n_blocks);
  std::iota(sidx.begin(), sidx.end(), 0);
  auto shift_less = [&](int64_t a, int64_t b) {
    for (int d = 0; d < 3; ++d) {
      int32_t x = lattice_shift[a * 3 + d], y = lattice_shift[b * 3 + d];
      if (x != y) return x < y;
    }
    return false;
  };
  std::stable_sort(sidx.begin(), sidx.end(), shift_less);
  B->block_shift.assign(n_blocks, 0);
  int32_t ns = -1;
  for (int64_t t = 0; t < n_blocks; ++t) {
    if (t == 0 || shift_less(sidx[t - 1], sidx[t])) {
      ++ns;
      for (int d = 0; d < 3; ++d) B->shifts.push_back(lattice_shift[sidx[t] * 3 + d]);
    }
    B->block_shift[sidx[t]] = ns;
  }

  // Groups: blocks sorted by (row atom, col atom), block order kept inside.
  std::vector<int64_t> order(n_blocks);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    if (row_atom[a] != row_atom[b]) return row_atom[a] < row_atom[b];
    return col_atom[a] < col_atom[b];
  });
  std::vector<int32_t> g_row, g_col;
  std::vector<int2> g_mem;
  std::vector<int64_t> m_off;
  std::vector<int32_t> m_shift;
  for (int64_t t = 0; t < n_blocks; ++t) {
    const int64_t b = order[t];
    if (t == 0 || row_atom[b] != row_atom[order[t - 1]] || col_atom[b] != col_atom[order[t - 1]]) {
      g_row.push_back(row_atom[b]);
      g_col.push_back(col_atom[b]);
      g_mem.push_back(make_int2((int)m_off.size(), (int)m_off.size()));
    }
    m_off.push_back(block_offsets[b]);
    m_shift.push_back(B->block_shift[b]);
    g_mem.back().y = (int)m_off.size();
  }
  const int64_t ng = (int64_t)g_row.size();
  B->n_groups = ng;
  // Row structure per atom.
  std::vector<int64_t> rowlen(n_atoms, 0), first_group(n_atoms + 1, ng);
  std::vector<int64_t> colpos(ng, 0);
  for (int64_t g = ng - 1; g >= 0; --g) first_group[g_row[g]] = g;
  for (int64_t a = n_atoms - 1; a >= 0; --a)
    if (first_group[a] == ng) first_group[a] = first_group[a + 1];
  for (int64_t g = 0; g < ng; ++g) {
    const int32_t i = g_row[g], j = g_col[g];
    colpos[g] = rowlen[i];
    rowlen[i] += atom_offsets[j + 1] - atom_offsets[j];
  }
  B->indptr.assign(n_orbitals + 1, 0);
  for (int64_t a = 0; a < n_atoms; ++a)
    for (int64_t r = atom_offsets[a]; r < atom_offsets[a + 1]; ++r)
      B->indptr[r + 1] = B->indptr[r] + rowlen[a];
  B->nnz = B->indptr[n_orbitals];
  if (B->nnz == 0) {
    delete B;
    return aosb::set_error(err, cap, AOSB_ERR_DIMS, "empty pattern");
  }
  B->indices.resize(B->nnz);
  for (int64_t g = 0; g < ng; ++g) {
    const int32_t i = g_row[g], j = g_col[g];
    for (int64_t r = atom_offsets[i]; r < atom_offsets[i + 1]; ++r) {
      int64_t p = B->indptr[r] + colpos[g];
      for (int64_t c = atom_offsets[j]; c < atom_offsets[j + 1]; ++c) B->indices[p++] = (int32_t)c;
    }
  }
  for (int64_t r = 0; r < n_orbitals; ++r)
    if (B->indptr[r + 1] == B->indptr[r]) {
      // Rows without entries are allowed by the reference pattern builder;
      // the solver rejects them later (missing diagonal).
    }
  // Mirror groups (Hermitian topology).
  std::vector<int4> g_info(ng);
  std::vector<int64_t> g_dst(ng);
  for (int64_t g = 0; g < ng; ++g) {
    const int32_t i = g_row[g], j = g_col[g];
    int64_t lo = first_group[j], hi = first_group[j + 1];
    int64_t m = -1;
    while (lo < hi) {
      int64_t mid = (lo + hi) / 2;
      if (g_col[mid] < i) lo = mid + 1; else hi = mid;
    }
    if (lo < first_group[j + 1] && g_col[lo] == i) m = lo;
    if (m < 0) {
      delete B;
      return aosb::set_error(err, cap, AOSB_ERR_TOPOLOGY, "operator topology is not Hermitian");
    }
    const int nr = (int)(atom_offsets[i + 1] - atom_offsets[i]);
    const int nc = (int)(atom_offsets[j + 1] - atom_offsets[j]);
    g_info[g] = make_int4(nr, nc, (int)rowlen[i], (int)m);
    g_dst[g] = B->indptr[atom_offsets[i]] + colpos[g];
  }
  B->n_members = (int64_t)m_off.size();
  B->g_info = std::move(g_info);
  B->g_dst = std::move(g_dst);
  B->g_mem = std::move(g_mem);
  B->m_off = std::move(m_off);
  B->m_shift = std::move(m_shift);
  *out = B;
  return 0;
}

int aosb_bloch_upload(aosb_bloch_t* B, char* err, size_t cap) {
  if (B == nullptr) return aosb::set_error(err, cap, AOSB_ERR_NULL, "null handle");
  if (B->uploaded) return 0;
  int rc = 0;
  if ((rc = upload(&B->d_indptr, B->indptr, err, cap)) ||
      (rc = upload(&B->d_indices, B->indices, err, cap)) ||
      (rc = upload(&B->d_group, B->g_info, err, cap)) ||
      (rc = upload(&B->d_group_dst, B->g_dst, err, cap)) ||
      (rc = upload(&B->d_group_members, B->g_mem, err, cap)) ||
      (rc = upload(&B->d_member_off, B->m_off, err, cap)) ||
      (rc = upload(&B->d_member_shift, B->m_shift, err, cap)))
    return rc;
  int64_t values = 0;
  for (size_t g = 0; g < B->g_info.size(); ++g)
    values += (int64_t)B->g_info[g].x * B->g_info[g].y * (B->g_mem[g].y - B->g_mem[g].x);
  B->n_values = values;
  B->uploaded = true;
  return 0;
}

int aosb_bloch_info(const aosb_bloch_t* b, int64_t* nnz, int64_t* n_shifts) {
  if (b == nullptr) return AOSB_ERR_NULL;
  if (nnz) *nnz = b->nnz;
  if (n_shifts) *n_shifts = (int64_t)(b->shifts.size() / 3);
  return 0;
}

int aosb_bloch_export(const aosb_bloch_t* b, int64_t* indptr, int32_t* indices, int32_t* shifts,
                      int32_t* block_shift) {
  if (b == nullptr) return AOSB_ERR_NULL;
  if (indptr) std::copy(b->indptr.begin(), b->indptr.end(), indptr);
  if (indices) std::copy(b->indices.begin(), b->indices.end(), indices);
  if (shifts) std::copy(b->shifts.begin(), b->shifts.end(), shifts);
  if (block_shift) std::copy(b->block_shift.begin(), b->block_shift.end(), block_shift);
  return 0;
}

int aosb_bloch_export_groups(const aosb_bloch_t* b, int64_t* n_groups, int64_t* n_members,
                             int32_t* group_info, int64_t* group_dst, int32_t* group_members,
                             int64_t* member_off, int32_t* member_shift) {
  if (b == nullptr) return AOSB_ERR_NULL;
  if (n_groups) *n_groups = (int64_t)b->g_info.size();
  if (n_members) *n_members = (int64_t)b->m_off.size();
  for (size_t g = 0; g < b->g_info.size(); ++g) {
    if (group_info) {
      group_info[4 * g] = b->g_info[g].x;
      group_info[4 * g + 1] = b->g_info[g].y;
      group_info[4 * g + 2] = b->g_info[g].z;
      group_info[4 * g + 3] = b->g_info[g].w;
    }
    if (group_dst) group_dst[g] = b->g_dst[g];
    if (group_members) {
      group_members[2 * g] = b->g_mem[g].x;
      group_members[2 * g + 1] = b->g_mem[g].y;
    }
  }
  if (member_off) std::copy(b->m_off.begin(), b->m_off.end(), member_off);
  if (member_shift) std::copy(b->m_shift.begin(), b->m_shift.end(), member_shift);
  return 0;
}

int aosb_bloch_device_pattern(const aosb_bloch_t* b, const int64_t** indptr,
                              const int32_t** indices) {
  if (b == nullptr) return AOSB_ERR_NULL;
  if (!b->uploaded) return AOSB_ERR_ARGUMENT;
  if (indptr) *indptr = b->d_indptr;
  if (indices) *indices = b->d_indices;
  return 0;
}

int aosb_bloch_apply(const aosb_bloch_t* b, int32_t value_kind, const void* h_values,
                     const void* s_values, const aosb_complex64* phases, int32_t n_k,
                     aosb_complex64* h_out, aosb_complex64* s_out, void* stream, char* err,
                     size_t cap) {
  if (b == nullptr || h_values == nullptr || s_values == nullptr || phases == nullptr ||
      h_out == nullptr || s_out == nullptr)
    return aosb::set_error(err, cap, AOSB_ERR_NULL, "required pointer is null");
  if (!b->uploaded)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "call aosb_bloch_upload first");
  if (n_k <= 0 || n_k > 65535)
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "n_k must be in 1..65535");
  const int warps = 8;
  dim3 grid(aosb::ceil_div(b->n_groups, warps), aosb::ceil_div(n_k, kBlochKChunk));
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nsh = (int64_t)(b->shifts.size() / 3);
  cudaEvent_t ev[2];
  const bool timed = aosb::timing_begin(st, ev);
  if (value_kind == 0) {
    bloch_windows_kernel<float><<<grid, warps * 32, 0, st>>>(
        b->n_groups, b->d_group, b->d_group_dst, b->d_group_members, b->d_member_off,
        b->d_member_shift, (const float*)h_values, (const float*)s_values,
        (const float2*)phases, nsh, b->nnz, n_k, (float2*)h_out, (float2*)s_out);
  } else if (value_kind == 1) {
    bloch_windows_kernel<float2><<<grid, warps * 32, 0, st>>>(
        b->n_groups, b->d_group, b->d_group_dst, b->d_group_members, b->d_member_off,
        b->d_member_shift, (const float2*)h_values, (const float2*)s_values,
        (const float2*)phases, nsh, b->nnz, n_k, (float2*)h_out, (float2*)s_out);
  } else {
    return aosb::set_error(err, cap, AOSB_ERR_ARGUMENT, "value_kind must be 0 or 1");
  }
  aosb::count_launches(1);
  // algorithmic bytes: the stored H and S block values read once per launch,
  // the complex64 H(k) and S(k) CSR values written once per k point
  if (timed)
    aosb::timing_end(aosb::kTimedBloch, st, ev, 0.0,
                     (double)b->n_values * 2.0 * (value_kind ? 8.0 : 4.0) +
                         (double)n_k * (double)b->nnz * 2.0 * 8.0);
  return aosb::launch_check(err, cap, "bloch_windows_kernel");
}

void aosb_bloch_destroy(aosb_bloch_t* b) {
  if (b == nullptr) return;
  cudaFree(b->d_indptr);
  cudaFree(b->d_indices);
  cudaFree(b->d_group);
  cudaFree(b->d_group_dst);
  cudaFree(b->d_group_members);
  cudaFree(b->d_member_off);
  cudaFree(b->d_member_shift);
  delete b;
}

}  // extern "C"
