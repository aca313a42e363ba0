// gh_adjprod.cpp -- general irreps as a piece of a product of adjoints (see gh_adjprod.h).
#include "gh_adjprod.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "../../include/gauge_higgs_b200.h"
#include "gh_potential.h"
#include "gh_sympow.h"

namespace ghadj {
namespace {

using cd = std::complex<double>;

// sign of the permutation idx[0..m-1] of distinct values, 0 when a value repeats
int levi_civita(const int* idx, int m) {
  int sg = 1;
  for (int i = 0; i < m; ++i)
    for (int j = i + 1; j < m; ++j) {
      if (idx[i] == idx[j]) return 0;
      if (idx[i] > idx[j]) sg = -sg;
    }
  return sg;
}

// One nonzero of a column of the embedding: the digits of its n slots and its value.
struct Entry {
  int dig[6];
  cd v;
};

// Columns b of E1: the adjoint basis vector T^b as an element of V (x) Lambda^(N-1) V,
//   E1[(i, k_1 .. k_{N-1})][b] = sum_j T^b_ij eps_{j k_1 .. k_{N-1}}.
std::vector<std::vector<Entry>> embed_adjoint(int N) {
  const int ng = N * N - 1;
  const std::vector<cd> T = ghpot::gell_mann(N);
  int total = 1;
  for (int s = 0; s < N; ++s) total *= N;
  std::vector<std::vector<Entry>> cols(ng);
  for (int b = 0; b < ng; ++b)
    for (int code = 0; code < total; ++code) {
      Entry e{};
      int r = code;
      for (int s = N - 1; s >= 0; --s) { e.dig[s] = r % N; r /= N; }
      cd v = 0.0;
      for (int j = 0; j < N; ++j) {
        int idx[4] = {j, 0, 0, 0};
        for (int s = 1; s < N; ++s) idx[s] = e.dig[s];
        const int sg = levi_civita(idx, N);
        if (sg) v += T[((size_t)b * N + e.dig[0]) * N + j] * (double)sg;
      }
      if (v != cd(0.0, 0.0)) {
        e.v = v;
        cols[b].push_back(e);
      }
    }
  return cols;
}

// A generic SU(N) link for the self-check: the Cayley transform (1 + iH)(1 - iH)^-1 of
// a fixed Hermitian H, its determinant phase removed (N <= 3: explicit inverse).
void check_link(int N, int which, cd* U) {
  cd H[9], A[9], B[9];
  for (int i = 0; i < N; ++i)
    for (int j = i; j < N; ++j) {
      const double re = 0.41 * std::cos(0.7 + 2 * i + 3 * j + 1.3 * which) + 0.07 * (which + 1);
      const double im = (i == j) ? 0.0 : 0.33 * std::sin(1.1 + 5 * i + j + 0.9 * which);
      H[i * N + j] = cd(re, im);
      H[j * N + i] = cd(re, -im);
    }
  for (int i = 0; i < N * N; ++i) {
    const bool diag = (i / N) == (i % N);
    A[i] = (diag ? 1.0 : 0.0) + cd(0, 1) * H[i];
    B[i] = (diag ? 1.0 : 0.0) - cd(0, 1) * H[i];
  }
  cd Bi[9];
  if (N == 2) {
    const cd det = B[0] * B[3] - B[1] * B[2];
    Bi[0] = B[3] / det; Bi[1] = -B[1] / det; Bi[2] = -B[2] / det; Bi[3] = B[0] / det;
  } else {
    const cd det = B[0] * (B[4] * B[8] - B[5] * B[7]) - B[1] * (B[3] * B[8] - B[5] * B[6]) +
                   B[2] * (B[3] * B[7] - B[4] * B[6]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const int r0 = (j + 1) % 3, r1 = (j + 2) % 3, c0 = (i + 1) % 3, c1 = (i + 2) % 3;
        Bi[i * 3 + j] = (B[r0 * 3 + c0] * B[r1 * 3 + c1] - B[r0 * 3 + c1] * B[r1 * 3 + c0]) / det;
      }
  }
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      cd s = 0.0;
      for (int k = 0; k < N; ++k) s += A[i * N + k] * Bi[k * N + j];
      U[i * N + j] = s;
    }
  cd det = (N == 2) ? U[0] * U[3] - U[1] * U[2]
                    : U[0] * (U[4] * U[8] - U[5] * U[7]) - U[1] * (U[3] * U[8] - U[5] * U[6]) +
                          U[2] * (U[3] * U[7] - U[4] * U[6]);
  const cd ph = std::pow(det / std::abs(det), -1.0 / N);
  for (int i = 0; i < N * N; ++i) U[i] *= ph;
}

}  // namespace

void adjoint_matrix(int N, const double* Uin, double* Dadj) {
  const int ng = N * N - 1;
  const cd* U = reinterpret_cast<const cd*>(Uin);
  const std::vector<cd> T = ghpot::gell_mann(N);
  std::vector<cd> M(N * N), UT(N * N);
  for (int b = 0; b < ng; ++b) {
    const cd* Tb = T.data() + (size_t)b * N * N;
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        cd s = 0.0;
        for (int k = 0; k < N; ++k) s += U[i * N + k] * Tb[k * N + j];
        UT[i * N + j] = s;
      }
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        cd s = 0.0;
        for (int k = 0; k < N; ++k) s += UT[i * N + k] * std::conj(U[j * N + k]);
        M[i * N + j] = s;
      }
    for (int a = 0; a < ng; ++a) {
      const cd* Ta = T.data() + (size_t)a * N * N;
      cd tr = 0.0;
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) tr += Ta[i * N + j] * M[j * N + i];
      Dadj[a * ng + b] = 2.0 * tr.real();
    }
  }
}

void eval(const Product& p, const double* U, double* Dout) {
  const int ng = p.N * p.N - 1, A = p.A, d = p.d;
  std::vector<double> G((size_t)ng * ng);
  adjoint_matrix(p.N, U, G.data());
  cd* D = reinterpret_cast<cd*>(Dout);
  std::vector<cd> x(A), y(A), z(A);
  for (int l = 0; l < d; ++l) {
    for (int r = 0; r < A; ++r) x[r] = p.Q[(size_t)r * d + l];
    if (p.K == 1) {
      for (int a = 0; a < ng; ++a) {
        cd s = 0.0;
        for (int k = 0; k < ng; ++k) s += G[a * ng + k] * x[k];
        y[a] = s;
      }
    } else {
      // X -> G X G^T on the ng x ng coefficient matrix X_ab = x[a ng + b]
      for (int a = 0; a < ng; ++a)
        for (int b = 0; b < ng; ++b) {
          cd s = 0.0;
          for (int k = 0; k < ng; ++k) s += G[a * ng + k] * x[k * ng + b];
          z[a * ng + b] = s;
        }
      for (int a = 0; a < ng; ++a)
        for (int b = 0; b < ng; ++b) {
          cd s = 0.0;
          for (int k = 0; k < ng; ++k) s += z[a * ng + k] * G[b * ng + k];
          y[a * ng + b] = s;
        }
    }
    for (int k = 0; k < d; ++k) {
      cd s = 0.0;
      for (int r = 0; r < A; ++r) s += std::conj(p.Q[(size_t)r * d + k]) * y[r];
      D[(size_t)k * d + l] = s;
    }
  }
}

bool build(int N, int n, int d, long dimT, const double* Win, Product& out, std::string* why) {
  auto no = [&](const char* m) { if (why) *why = m; return false; };
  if (N != 2 && N != 3) return no("product of adjoints is built for SU(2) and SU(3)");
  if (n % N != 0 || n / N < 1 || n / N > 2) return no("needs n = K N boxes with K = 1 or 2");
  const int K = n / N, ng = N * N - 1;
  const int A = (K == 1) ? ng : ng * ng;
  if (d <= 0 || d > A) return no("irrep larger than the adjoint product");
  long pw = 1;
  for (int s = 0; s < n; ++s) pw *= N;
  if (pw != dimT) return no("dimT must equal N^n");
  const cd* W = reinterpret_cast<const cd*>(Win);
  // the columns of the K-fold embedding, slot digits concatenated factor by factor
  const std::vector<std::vector<Entry>> e1 = embed_adjoint(N);
  std::vector<std::vector<Entry>> cols(A);
  if (K == 1) {
    cols = e1;
  } else {
    for (int a = 0; a < ng; ++a)
      for (int b = 0; b < ng; ++b)
        for (const Entry& x : e1[a])
          for (const Entry& y : e1[b]) {
            Entry z{};
            for (int s = 0; s < N; ++s) { z.dig[s] = x.dig[s]; z.dig[N + s] = y.dig[s]; }
            z.v = x.v * y.v;
            cols[a * ng + b].push_back(z);
          }
  }
  // the basis vectors of R by tensor index
  std::vector<std::vector<std::pair<int, cd>>> wt(dimT);
  for (int l = 0; l < d; ++l)
    for (long t = 0; t < dimT; ++t)
      if (W[(size_t)l * dimT + t] != cd(0.0, 0.0)) wt[t].push_back({l, W[(size_t)l * dimT + t]});
  // every slot order of the embedding; keep the one with the largest overlap
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::vector<cd> M((size_t)A * d), best;
  double best_c2 = 0.0;
  do {
    std::fill(M.begin(), M.end(), cd(0.0, 0.0));
    for (int r = 0; r < A; ++r)
      for (const Entry& e : cols[r]) {
        long t = 0;
        for (int s = 0; s < n; ++s) t = t * N + e.dig[perm[s]];
        for (const auto& lw : wt[t]) M[(size_t)r * d + lw.first] += std::conj(e.v) * lw.second;
      }
    double c2 = 0.0;
    for (const cd& m : M) c2 += std::norm(m);
    c2 /= d;
    if (c2 > best_c2 * (1.0 + 1e-9)) { best_c2 = c2; best = M; }
  } while (std::next_permutation(perm.begin(), perm.end()));
  if (!(best_c2 > 1e-8)) return no("the irrep does not overlap the adjoint product");
  // M^dag M = c^2 I (Schur): the overlap is a multiple of an isometry
  for (int l = 0; l < d; ++l)
    for (int m = 0; m < d; ++m) {
      cd g = 0.0;
      for (int r = 0; r < A; ++r) g += std::conj(best[(size_t)r * d + l]) * best[(size_t)r * d + m];
      if (std::abs(g - (l == m ? best_c2 : 0.0)) > 1e-9 * best_c2) return no("overlap is not an intertwiner");
    }
  out.N = N; out.K = K; out.d = d; out.A = A; out.c2 = best_c2;
  out.Q.resize((size_t)A * d);
  const double inv = 1.0 / std::sqrt(best_c2);
  for (size_t i = 0; i < best.size(); ++i) out.Q[i] = best[i] * inv;
  // the rows the device lifts into: a symmetric / antisymmetric coefficient matrix needs
  // only the pairs a <= b / a < b
  out.sym = 0;
  if (K == 2) {
    double es = 0.0, ea = 0.0, mx = 0.0;
    for (int a = 0; a < ng; ++a)
      for (int b = 0; b < ng; ++b)
        for (int k = 0; k < d; ++k) {
          const std::complex<double> x = out.Q[(size_t)(a * ng + b) * d + k], y = out.Q[(size_t)(b * ng + a) * d + k];
          es = std::max(es, std::abs(x - y));
          ea = std::max(ea, std::abs(x + y));
          mx = std::max(mx, std::abs(x));
        }
    if (es <= 1e-13 * mx) out.sym = 1;
    else if (ea <= 1e-13 * mx) out.sym = -1;
  }
  out.rows.clear();
  if (out.sym == 1)
    for (int a = 0; a < ng; ++a) out.rows.push_back(a * ng + a);
  out.ndiag = (int)out.rows.size();
  if (out.sym != 0) {
    for (int a = 0; a < ng; ++a)
      for (int b = a + 1; b < ng; ++b) out.rows.push_back(a * ng + b);
  } else {
    for (int r = 0; r < A; ++r) out.rows.push_back(r);
    out.ndiag = A;
  }
  out.Qr.resize(out.rows.size() * (size_t)d);
  for (size_t r = 0; r < out.rows.size(); ++r)
    for (int k = 0; k < d; ++k) out.Qr[r * d + k] = out.Q[(size_t)out.rows[r] * d + k];
  // against the tensor construction on two generic links
  std::vector<cd> Dp((size_t)d * d), Dt((size_t)d * d);
  for (int which = 0; which < 2; ++which) {
    cd U[9];
    check_link(N, which, U);
    eval(out, reinterpret_cast<const double*>(U), reinterpret_cast<double*>(Dp.data()));
    ghsym::tensor_matrix(N, n, d, dimT, Win, reinterpret_cast<const double*>(U), reinterpret_cast<double*>(Dt.data()));
    double worst = 0.0;
    for (size_t i = 0; i < Dp.size(); ++i) worst = std::max(worst, std::abs(Dp[i] - Dt[i]));
    if (!(worst < 1e-10)) return no("product of adjoints disagrees with the tensor construction");
  }
  return true;
}

}  // namespace ghadj

// ---- C ABI (host only; no GPU needed) ----
extern "C" int gh_rep_product_matrix(int N, const gh_rep_desc* rep, const double* U, double* D, int* K) {
  if (!rep || !U || !D) { ghpot::set_host_error("null argument"); return GH_ERR_ARG; }
  if (rep->kind != GH_REP_GENERAL || !rep->W || rep->dimT <= 0 || rep->dimT > 200000 || rep->n_boxes < 1 ||
      rep->n_boxes > 17) {
    ghpot::set_host_error("the product of adjoints needs a general irrep with its W table");
    return GH_ERR_REP;
  }
  ghadj::Product p;
  std::string why;
  if (!ghadj::build(N, rep->n_boxes, rep->d, rep->dimT, rep->W, p, &why)) {
    ghpot::set_host_error("no product-of-adjoints form for this irrep: " + why);
    return GH_ERR_REP;
  }
  ghadj::eval(p, U, D);
  if (K) *K = p.K;
  return GH_OK;
}
