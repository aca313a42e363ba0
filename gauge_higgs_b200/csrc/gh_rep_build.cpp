// gh_rep_build.cpp -- host-side construction of general SU(N) irreps: the basis W
// of the irrep inside V^{x n} and the generators T^a_R.  Runs once per context;
// the MD kernels only consume the resulting tables.
//
// The construction is the one the reference defines (src/rep/rep_general.hpp):
// the irrep space is the image of the Young symmetriser c = b a (a: symmetrise
// over the rows of the canonical tableau, b: antisymmetrise over its columns)
// applied to every standard tuple in index order, orthonormalised by modified
// Gram-Schmidt with a 1e-9 rank cut (:364-398); single-row diagrams use the
// normalised sums over distinct permutations of each multiset (:338-362); the
// generators act as derivations on the n slots and are restricted to the span
// of W (:400-411).  The order of construction fixes the basis, and the basis
// fixes the meaning of every scalar-field component, so the order is kept.
#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>
#include <map>
#include <functional>
#include <vector>
#include "../../include/gauge_higgs_b200.h"

namespace {
typedef std::complex<double> cd;

struct Builder {
  int N = 0, n = 0;
  long dimT = 1;
  std::vector<int> rows;
  std::vector<long> powN;
  std::vector<std::vector<cd>> W;

  long tup2idx(const std::vector<int>& t) const {
    long idx = 0;
    for (int j = 0; j < n; ++j) idx += (long)t[j] * powN[n - 1 - j];
    return idx;
  }
  std::vector<int> idx2tup(long idx) const {
    std::vector<int> t(n);
    for (int j = 0; j < n; ++j) t[j] = (int)((idx / powN[n - 1 - j]) % N);
    return t;
  }
  static cd inner(const std::vector<cd>& a, const std::vector<cd>& b) {
    cd s(0, 0);
    for (size_t i = 0; i < a.size(); ++i) s += std::conj(a[i]) * b[i];
    return s;
  }
  std::vector<int> permute(const std::vector<int>& sigma, const std::vector<int>& t) const {
    std::vector<int> u(n);
    for (int j = 0; j < n; ++j) u[sigma[j]] = t[j];
    return u;
  }
  static int parity_sign(const std::vector<int>& p) {
    std::vector<char> seen(p.size(), 0);
    int sign = 1;
    for (size_t i = 0; i < p.size(); ++i) {
      if (seen[i]) continue;
      int len = 0;
      for (size_t j = i; !seen[j]; j = p[j]) { seen[j] = 1; ++len; }
      if (len % 2 == 0) sign = -sign;
    }
    return sign;
  }
  // product of the symmetric groups of disjoint position blocks, as full permutations
  void group(const std::vector<std::vector<int>>& blocks, std::vector<std::vector<int>>& perms, std::vector<int>& signs) const {
    std::vector<int> id(n);
    std::iota(id.begin(), id.end(), 0);
    perms.assign(1, id);
    for (const auto& blk : blocks) {
      std::vector<int> src = blk;
      std::sort(src.begin(), src.end());
      std::vector<std::vector<int>> dsts;
      std::vector<int> cur = src;
      do { dsts.push_back(cur); } while (std::next_permutation(cur.begin(), cur.end()));
      std::vector<std::vector<int>> next;
      next.reserve(perms.size() * dsts.size());
      for (const auto& g : perms)
        for (const auto& dst : dsts) {
          std::vector<int> g2 = g;
          for (size_t k = 0; k < src.size(); ++k) g2[src[k]] = dst[k];
          next.push_back(g2);
        }
      perms.swap(next);
    }
    signs.resize(perms.size());
    for (size_t i = 0; i < perms.size(); ++i) signs[i] = parity_sign(perms[i]);
  }
  // Single-row diagram {n}: one basis vector per multiset of n slot indices, the
  // normalised sum of every tensor index whose digits form that multiset.  The order is
  // the reference's (ascending sorted tuples), which is the digit histograms in
  // descending lexicographic order: at the first value where two histograms differ, the
  // one with more copies of it has that value where the other's tuple has a larger one.
  void basis_symmetric() {
    std::map<std::vector<int>, std::vector<long>, std::greater<std::vector<int>>> by_hist;
    for (long t = 0; t < dimT; ++t) {
      std::vector<int> hist(N, 0);
      for (int digit : idx2tup(t)) ++hist[digit];
      by_hist[hist].push_back(t);
    }
    for (const auto& group : by_hist) {
      std::vector<cd> v(dimT, cd(0, 0));
      const double w = 1.0 / std::sqrt((double)group.second.size());
      for (long t : group.second) v[t] = cd(w, 0);
      W.push_back(v);
    }
  }
  void basis_young() {
    std::vector<std::vector<int>> rb(rows.size()), cb(rows[0]);
    int pos = 0;
    for (size_t i = 0; i < rows.size(); ++i)
      for (int j = 0; j < rows[i]; ++j) { rb[i].push_back(pos); cb[j].push_back(pos); ++pos; }
    std::vector<std::vector<int>> R, C;
    std::vector<int> Rs, Cs;
    group(rb, R, Rs);
    group(cb, C, Cs);
    for (long tc = 0; tc < dimT; ++tc) {
      const std::vector<int> t = idx2tup(tc);
      std::vector<cd> v1(dimT, cd(0, 0)), v(dimT, cd(0, 0));
      for (const auto& p : R) v1[tup2idx(permute(p, t))] += cd(1, 0);
      for (long idx = 0; idx < dimT; ++idx) {
        const cd c = v1[idx];
        if (c == cd(0, 0)) continue;
        const std::vector<int> ta = idx2tup(idx);
        for (size_t q = 0; q < C.size(); ++q) v[tup2idx(permute(C[q], ta))] += cd(Cs[q], 0) * c;
      }
      for (const auto& w : W) {
        const cd ov = inner(w, v);
        for (long i = 0; i < dimT; ++i) v[i] -= ov * w[i];
      }
      const double nrm = std::sqrt(std::max(0.0, inner(v, v).real()));
      if (nrm > 1e-9) {
        const cd inv(1.0 / nrm, 0);
        for (auto& z : v) z *= inv;
        W.push_back(v);
      }
    }
  }
  // generalised Gell-Mann T^a_F (src/group/algebra.hpp:23-49)
  std::vector<cd> gen(int a) const {
    std::vector<cd> T(N * N, cd(0, 0));
    int k = 0;
    for (int j = 0; j < N; ++j)
      for (int l = j + 1; l < N; ++l, ++k)
        if (k == a) { T[j * N + l] += cd(0.5, 0); T[l * N + j] += cd(0.5, 0); }
    for (int j = 0; j < N; ++j)
      for (int l = j + 1; l < N; ++l, ++k)
        if (k == a) { T[j * N + l] += cd(0, -0.5); T[l * N + j] += cd(0, 0.5); }
    for (int l = 1; l <= N - 1; ++l, ++k)
      if (k == a) {
        const double c = std::sqrt(2.0 / ((double)l * (l + 1)));
        for (int j = 0; j < l; ++j) T[j * N + j] += cd(0.5 * c, 0);
        T[l * N + l] += cd(-0.5 * c * l, 0);
      }
    return T;
  }
  std::vector<cd> onebody(const std::vector<cd>& M, const std::vector<cd>& v, int s) const {
    std::vector<cd> out(dimT, cd(0, 0));
    const long blk = powN[n - 1 - s];
    for (long idx = 0; idx < dimT; ++idx) {
      const cd c = v[idx];
      if (c == cd(0, 0)) continue;
      const int digit = (int)((idx / blk) % N);
      const long base = idx - (long)digit * blk;
      for (int j = 0; j < N; ++j) out[base + (long)j * blk] += M[j * N + digit] * c;
    }
    return out;
  }
};

int setup(Builder& b, int N, const int* rows, int nrows) {
  if (N < 2 || N > 4 || !rows || nrows < 1) return GH_ERR_ARG;
  b.N = N;
  b.rows.assign(rows, rows + nrows);
  while (!b.rows.empty() && b.rows.back() == 0) b.rows.pop_back();
  if (b.rows.empty()) return GH_ERR_REP;
  for (size_t i = 0; i + 1 < b.rows.size(); ++i) if (b.rows[i] < b.rows[i + 1]) return GH_ERR_REP;
  if ((int)b.rows.size() > N - 1) return GH_ERR_REP;
  b.n = std::accumulate(b.rows.begin(), b.rows.end(), 0);
  if (b.n > 17) return GH_ERR_REP;        // N^n <= 200000 below bounds n by 17 (SU(2))
  b.powN.assign(b.n + 1, 1);
  for (int k = 1; k <= b.n; ++k) b.powN[k] = b.powN[k - 1] * N;
  b.dimT = b.powN[b.n];
  if (b.dimT > 200000) return GH_ERR_REP;
  if (b.rows.size() == 1) b.basis_symmetric(); else b.basis_young();
  return GH_OK;
}
}  // namespace

extern "C" {

int gh_rep_general_info(int N, const int* rows, int nrows, int* d, int* n_boxes, long* dimT) {
  Builder b;
  const int rc = setup(b, N, rows, nrows);
  if (rc) return rc;
  if (d) *d = (int)b.W.size();
  if (n_boxes) *n_boxes = b.n;
  if (dimT) *dimT = b.dimT;
  return GH_OK;
}

int gh_rep_general_build(int N, const int* rows, int nrows, double* T, double* W) {
  Builder b;
  const int rc = setup(b, N, rows, nrows);
  if (rc) return rc;
  const int d = (int)b.W.size();
  if (W)
    for (int l = 0; l < d; ++l)
      for (long i = 0; i < b.dimT; ++i) { W[2 * ((size_t)l * b.dimT + i)] = b.W[l][i].real(); W[2 * ((size_t)l * b.dimT + i) + 1] = b.W[l][i].imag(); }
  if (T)
    for (int a = 0; a < N * N - 1; ++a) {
      const std::vector<cd> Ta = b.gen(a);
      for (int l = 0; l < d; ++l) {
        std::vector<cd> v(b.dimT, cd(0, 0));
        for (int s = 0; s < b.n; ++s) {
          const std::vector<cd> tmp = b.onebody(Ta, b.W[l], s);
          for (long i = 0; i < b.dimT; ++i) v[i] += tmp[i];
        }
        for (int k = 0; k < d; ++k) {
          const cd z = Builder::inner(b.W[k], v);
          const size_t o = 2 * (((size_t)a * d + k) * d + l);
          T[o] = z.real();
          T[o + 1] = z.imag();
        }
      }
    }
  return GH_OK;
}

}  // extern "C"
