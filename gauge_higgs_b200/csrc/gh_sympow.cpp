// Closed-form D(U) for the single-row irreps: term lists and host checks.
#include "gh_sympow.h"

#include <algorithm>
#include <cmath>
#include <complex>

namespace ghsym {
namespace {

typedef std::complex<double> cd;

double factorial(int k) {
  double f = 1.0;
  for (int i = 2; i <= k; ++i) f *= i;
  return f;
}

// all N x N non-negative integer matrices with the given row and column sums
struct Tables {
  int N;
  std::vector<int> row, col;
  std::vector<unsigned char> K;
  std::vector<std::vector<unsigned char>> out;
  long cap;
  bool overflow = false;
  void rec(int cell) {
    if (overflow) return;
    if (cell == N * N) {
      for (int j = 0; j < N; ++j)
        if (col[j]) return;
      if ((long)out.size() >= cap) { overflow = true; return; }
      out.push_back(K);
      return;
    }
    const int i = cell / N, j = cell % N;
    if (j == N - 1) {                       // last cell of a row takes what the row has left
      const int v = row[i];
      if (v > col[j]) return;
      K[cell] = (unsigned char)v; row[i] -= v; col[j] -= v;
      rec(cell + 1);
      row[i] += v; col[j] += v;
      return;
    }
    const int hi = std::min(row[i], col[j]);
    for (int v = 0; v <= hi; ++v) {
      K[cell] = (unsigned char)v; row[i] -= v; col[j] -= v;
      rec(cell + 1);
      row[i] += v; col[j] += v;
    }
  }
};

void su_link(int N, int which, cd* U) {
  // a fixed, generic SU(N) link: exp(i H) of a Hermitian H, by eigen-free series
  // with scaling and squaring (host check only)
  std::vector<cd> H(N * N);
  for (int i = 0; i < N; ++i)
    for (int j = i; j < N; ++j) {
      const double re = 0.37 * std::sin(1.0 + 3 * i + 5 * j + 2.0 * which) + 0.11 * (which + 1);
      const double im = (i == j) ? 0.0 : 0.29 * std::cos(2.0 + i + 7 * j + which);
      H[i * N + j] = cd(re, im);
      H[j * N + i] = cd(re, -im);
    }
  cd tr = 0;
  for (int i = 0; i < N; ++i) tr += H[i * N + i];
  for (int i = 0; i < N; ++i) H[i * N + i] -= tr / double(N);
  const int sq = 8;
  for (auto& h : H) h *= cd(0.0, 1.0 / (1 << sq));
  std::vector<cd> E(N * N, 0.0), term(N * N, 0.0), tmp(N * N);
  for (int i = 0; i < N; ++i) { E[i * N + i] = 1.0; term[i * N + i] = 1.0; }
  for (int k = 1; k < 20; ++k) {
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        cd s = 0;
        for (int q = 0; q < N; ++q) s += term[i * N + q] * H[q * N + j];
        tmp[i * N + j] = s / double(k);
      }
    term = tmp;
    for (int i = 0; i < N * N; ++i) E[i] += term[i];
  }
  for (int r = 0; r < sq; ++r) {
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        cd s = 0;
        for (int q = 0; q < N; ++q) s += E[i * N + q] * E[q * N + j];
        tmp[i * N + j] = s;
      }
    E = tmp;
  }
  for (int i = 0; i < N * N; ++i) U[i] = E[i];
}

}  // namespace

bool build(int N, int n, int d, long dimT, const double* W, long max_terms, Terms& out, std::string* why) {
  auto no = [&](const char* m) { if (why) *why = m; return false; };
  if (N < 2 || n < 1 || d < 1 || dimT < 1 || !W) return no("bad arguments");
  if (N * N * (n + 1) > 255) return no("power table too large for byte offsets");
  long pw = 1;
  for (int k = 0; k < n; ++k) pw *= N;
  if (pw != dimT) return no("dimT != N^n");
  const cd* w = reinterpret_cast<const cd*>(W);
  // multiset and common entry of every basis vector
  std::vector<std::vector<int>> occ(d, std::vector<int>(N, 0));
  std::vector<cd> omega(d);
  for (int l = 0; l < d; ++l) {
    long nnz = 0;
    bool first = true;
    const cd* row = w + (size_t)l * dimT;
    double amax = 0.0;
    for (long i = 0; i < dimT; ++i) amax = std::max(amax, std::abs(row[i]));
    if (amax == 0.0) return no("zero basis vector");
    for (long i = 0; i < dimT; ++i) {
      if (std::abs(row[i]) <= 1e-12 * amax) continue;
      ++nnz;
      std::vector<int> m(N, 0);
      long r = i;
      for (int s = n - 1; s >= 0; --s) { m[r % N]++; r /= N; }
      if (first) { occ[l] = m; omega[l] = row[i]; first = false; continue; }
      if (m != occ[l]) return no("basis vector mixes multisets (not a single-row irrep)");
      if (std::abs(row[i] - omega[l]) > 1e-12 * amax) return no("basis vector is not a constant times the symmetrised multiset");
    }
    double arr = factorial(n);
    for (int i = 0; i < N; ++i) arr /= factorial(occ[l][i]);
    if (std::fabs((double)nnz - arr) > 0.5) return no("basis vector does not cover every arrangement of its multiset");
  }
  out = Terms();
  out.N = N; out.n = n; out.d = d;
  out.ptr.assign((size_t)d * d + 1, 0);
  Tables tb;
  tb.N = N;
  tb.K.assign(N * N, 0);
  for (int k = 0; k < d; ++k) {
    double arrk = factorial(n);
    for (int i = 0; i < N; ++i) arrk /= factorial(occ[k][i]);
    for (int l = 0; l < d; ++l) {
      tb.row = occ[k];
      tb.col = occ[l];
      tb.out.clear();
      tb.cap = max_terms - (long)out.c.size() / 2;
      tb.rec(0);
      if (tb.overflow) return no("more terms than the limit");
      const cd pre = std::conj(omega[k]) * omega[l] * arrk;
      for (const auto& K : tb.out) {
        double coef = 1.0;
        for (int i = 0; i < N; ++i) {
          coef *= factorial(occ[k][i]);
          for (int j = 0; j < N; ++j) coef /= factorial(K[i * N + j]);
        }
        const cd c = pre * coef;
        out.c.push_back(c.real());
        out.c.push_back(c.imag());
        out.e.insert(out.e.end(), K.begin(), K.end());
        out.e.resize(out.e.size() + (4 - (N * N) % 4) % 4, 0);   // whole 32-bit words per term
        const size_t o0 = out.off.size();
        for (int ij = 0; ij < N * N; ++ij)
          if (N == 2 || K[ij] > 0) out.off.push_back((unsigned char)(ij * (n + 1) + K[ij]));
        out.off.resize(o0 + (N * N + 3) / 4 * 4, 0xFF);
      }
      out.ptr[(size_t)k * d + l + 1] = (int)(out.c.size() / 2);
    }
  }
  // check against the tensor construction on two generic links
  std::vector<cd> U(N * N), Dt((size_t)d * d), Dc((size_t)d * d);
  for (int t = 0; t < 2; ++t) {
    su_link(N, t, U.data());
    tensor_matrix(N, n, d, dimT, W, reinterpret_cast<const double*>(U.data()), reinterpret_cast<double*>(Dt.data()));
    eval(out, reinterpret_cast<const double*>(U.data()), reinterpret_cast<double*>(Dc.data()));
    double worst = 0.0;
    for (size_t i = 0; i < Dt.size(); ++i) worst = std::max(worst, std::abs(Dt[i] - Dc[i]));
    if (!(worst < 1e-10)) return no("closed form disagrees with the tensor construction");
  }
  return true;
}

void eval(const Terms& t, const double* Uin, double* Dout) {
  const int N = t.N, n = t.n, d = t.d;
  const cd* U = reinterpret_cast<const cd*>(Uin);
  cd* D = reinterpret_cast<cd*>(Dout);
  std::vector<cd> P((size_t)N * N * (n + 1));
  for (int ij = 0; ij < N * N; ++ij) {
    P[(size_t)ij * (n + 1)] = 1.0;
    for (int p = 1; p <= n; ++p) P[(size_t)ij * (n + 1) + p] = P[(size_t)ij * (n + 1) + p - 1] * U[ij];
  }
  for (int e = 0; e < d * d; ++e) {
    cd s = 0;
    for (int q = t.ptr[e]; q < t.ptr[e + 1]; ++q) {
      cd pr(t.c[2 * (size_t)q], t.c[2 * (size_t)q + 1]);
      for (int ij = 0; ij < N * N; ++ij) {
        const int k = t.e[(size_t)q * ((N * N + 3) / 4 * 4) + ij];
        if (k) pr *= P[(size_t)ij * (n + 1) + k];
      }
      s += pr;
    }
    D[e] = s;
  }
}

void tensor_matrix(int N, int n, int d, long dimT, const double* Win, const double* Uin, double* Dout) {
  const cd* W = reinterpret_cast<const cd*>(Win);
  const cd* U = reinterpret_cast<const cd*>(Uin);
  cd* D = reinterpret_cast<cd*>(Dout);
  std::vector<cd> v(dimT), tmp(N);
  // nonzeros of every basis vector (the projection runs over these only)
  std::vector<std::vector<long>> supp(d);
  for (int k = 0; k < d; ++k)
    for (long i = 0; i < dimT; ++i)
      if (W[(size_t)k * dimT + i] != cd(0.0, 0.0)) supp[k].push_back(i);
  for (int l = 0; l < d; ++l) {
    for (long i = 0; i < dimT; ++i) v[i] = W[(size_t)l * dimT + i];
    long blk = dimT;
    for (int s = 0; s < n; ++s) {            // slot s: digit of weight N^(n-1-s)
      blk /= N;
      for (long hi = 0; hi < dimT; hi += blk * N)
        for (long lo = 0; lo < blk; ++lo) {
          for (int j = 0; j < N; ++j) {
            cd acc = 0;
            for (int g = 0; g < N; ++g) acc += U[j * N + g] * v[hi + lo + g * blk];
            tmp[j] = acc;
          }
          for (int j = 0; j < N; ++j) v[hi + lo + j * blk] = tmp[j];
        }
    }
    for (int k = 0; k < d; ++k) {
      cd s = 0;
      for (long i : supp[k]) s += std::conj(W[(size_t)k * dimT + i]) * v[i];
      D[(size_t)k * d + l] = s;
    }
  }
}

}  // namespace ghsym

// ---- C ABI (host only; no GPU needed) ----
#include "../../include/gauge_higgs_b200.h"
#include "gh_potential.h"

extern "C" int gh_sympow_matrix(int N, const gh_rep_desc* rep, const double* U, double* D, long* n_terms) {
  if (!rep || !U || !D) { ghpot::set_host_error("null argument"); return GH_ERR_ARG; }
  if (rep->kind != GH_REP_GENERAL || !rep->W || rep->dimT <= 0 || rep->dimT > 200000 || rep->n_boxes < 1 ||
      rep->n_boxes > 17) {
    ghpot::set_host_error("closed-form matrices need a general irrep with its W table (N^n <= 200000)");
    return GH_ERR_REP;
  }
  ghsym::Terms t;
  std::string why;
  if (!ghsym::build(N, rep->n_boxes, rep->d, rep->dimT, rep->W, 1L << 22, t, &why)) {
    ghpot::set_host_error("no closed form for this irrep: " + why);
    return GH_ERR_REP;
  }
  ghsym::eval(t, U, D);
  if (n_terms) *n_terms = (long)(t.c.size() / 2);
  return GH_OK;
}
