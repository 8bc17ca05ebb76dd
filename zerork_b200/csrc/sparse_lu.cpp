// sparse_lu.cpp -- ordering and symbolic factorization (see sparse_lu.h).
#include "sparse_lu.h"

#include <algorithm>
#include <cstdint>
#include <stdexcept>

namespace zrk {
namespace {

struct Bits {
  int n = 0, w = 0;
  std::vector<uint64_t> v;
  Bits() = default;
  explicit Bits(int n_) : n(n_), w((n_ + 63) / 64), v(w, 0) {}
  void set(int i) { v[i >> 6] |= (uint64_t)1 << (i & 63); }
  void reset(int i) { v[i >> 6] &= ~((uint64_t)1 << (i & 63)); }
  bool get(int i) const { return (v[i >> 6] >> (i & 63)) & 1; }
  void or_with(const Bits &o) {
    for (int k = 0; k < w; ++k) v[k] |= o.v[k];
  }
  int count_and(const Bits &mask) const {
    int c = 0;
    for (int k = 0; k < w; ++k) c += __builtin_popcountll(v[k] & mask.v[k]);
    return c;
  }
};

}  // namespace

LUSymbolic analyze_lu(const JacPattern &p) {
  const int n = p.n, ns = n - 1;  // variable n-1 is temperature
  LUSymbolic s;
  s.n = n;
  // symmetric structure of the species block
  std::vector<Bits> adj(ns, Bits(ns));
  for (int j = 0; j < ns; ++j)
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
      int i = p.row_idx[k];
      if (i < ns && i != j) {
        adj[i].set(j);
        adj[j].set(i);
      }
    }
  // minimum degree (exact external degree on the elimination graph)
  Bits alive(ns);
  for (int i = 0; i < ns; ++i) alive.set(i);
  s.perm.clear();
  for (int step = 0; step < ns; ++step) {
    int best = -1, bd = 1 << 30;
    for (int i = 0; i < ns; ++i) {
      if (!alive.get(i)) continue;
      int d = adj[i].count_and(alive);
      if (d < bd) {
        bd = d;
        best = i;
      }
    }
    s.perm.push_back(best);
    alive.reset(best);
    // clique of the eliminated node's live neighbours
    std::vector<int> nb;
    for (int i = 0; i < ns; ++i)
      if (alive.get(i) && adj[best].get(i)) nb.push_back(i);
    for (int u : nb) {
      adj[u].or_with(adj[best]);
      adj[u].reset(u);
      adj[u].reset(best);
    }
  }
  s.perm.push_back(ns);  // temperature last
  s.iperm.assign(n, 0);
  for (int k = 0; k < n; ++k) s.iperm[s.perm[k]] = k;
  // symbolic Gaussian elimination on the permuted pattern (rows as bitsets)
  std::vector<Bits> row(n, Bits(n));
  for (int j = 0; j < n; ++j)
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k)
      row[s.iperm[p.row_idx[k]]].set(s.iperm[j]);
  for (int i = 0; i < n; ++i) row[i].set(i);
  for (int k = 0; k < n; ++k) {
    // U part of row k beyond k
    Bits uk(n);
    for (int j = k + 1; j < n; ++j)
      if (row[k].get(j)) uk.set(j);
    for (int i = k + 1; i < n; ++i)
      if (row[i].get(k)) row[i].or_with(uk);
  }
  // CSC of L+U
  s.col_ptr.assign(n + 1, 0);
  std::vector<std::vector<int>> cols(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (row[i].get(j)) cols[j].push_back(i);
  for (int j = 0; j < n; ++j) {
    s.col_ptr[j + 1] = s.col_ptr[j] + (int)cols[j].size();
    for (int i : cols[j]) s.row_idx.push_back(i);
  }
  s.nnz = s.col_ptr[n];
  s.diag_pos.assign(n, -1);
  for (int j = 0; j < n; ++j)
    for (int k = s.col_ptr[j]; k < s.col_ptr[j + 1]; ++k)
      if (s.row_idx[k] == j) s.diag_pos[j] = k;
  auto find = [&](int i, int j) {
    auto b = s.row_idx.begin() + s.col_ptr[j], e = s.row_idx.begin() + s.col_ptr[j + 1];
    auto it = std::lower_bound(b, e, i);
    if (it == e || *it != i) throw std::runtime_error("symbolic LU: missing entry");
    return (int)(it - s.row_idx.begin());
  };
  s.jac_to_lu.resize(p.nnz);
  for (int j = 0; j < n; ++j)
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k)
      s.jac_to_lu[k] = find(s.iperm[p.row_idx[k]], s.iperm[j]);
  s.diag_of_orig.resize(n);
  for (int v = 0; v < n; ++v) s.diag_of_orig[v] = s.diag_pos[s.iperm[v]];
  long fl = 0;
  for (int j = 0; j < n; ++j)
    for (int k = s.col_ptr[j]; k < s.diag_pos[j]; ++k) {
      int kk = s.row_idx[k];
      fl += s.col_ptr[kk + 1] - s.diag_pos[kk] - 1;
    }
  s.flops = fl;
  return s;
}

}  // namespace zrk
