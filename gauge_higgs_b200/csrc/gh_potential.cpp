// gh_potential.cpp -- host set-up of the multi-invariant onsite potential
//   V[phi] = -mu2 phi^dag phi + sum_c f_c || P_c(phi phi^dag) ||^2
// (src/action/scalar_invariants.hpp:19-206).  The channels c are the eigenspaces
// of the adjoint Casimir superoperator Chat(M) = sum_a [T^a_R, [T^a_R, M]] on the
// d x d matrices; P_c is the projector onto channel c.  Everything the device
// needs is the combined superoperator A = sum_c 2 f_c P_c (d^2 x d^2), because
//   dV/dphi^* = -mu2 phi + A(M) phi   and   V = -mu2 phi^dag phi + Re phi^dag A(M) phi / 2,
// M = phi phi^dag (the first is the reference's dV_dphibar_cached, :120-148; the
// second is sum_c f_c Re Tr(M^dag P_c M), :69-74, since the P_c are orthogonal
// projectors).  Matrices are vectorised row-major: vec(M)[i*d + j] = M_ij.
//
// Channels: Lanczos with full reorthogonalisation on Chat from a fixed generic
// Hermitian start (every channel holds Hermitian matrices, so the Krylov space
// stops at exactly one vector per distinct eigenvalue), eigenvalues of the small
// tridiagonal by cyclic Jacobi, merged when closer than 1e-4 and sorted ascending
// -- the channel order of the reference (find_channels, :152-187), which fixes the
// meaning of f_c.  Projectors: the Lagrange polynomial in Chat, as the reference
// (apply_proj, :43-52), applied to each basis matrix E_ij with a sparse Chat.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/gauge_higgs_b200.h"
#include "gh_potential.h"

namespace {

using cd = std::complex<double>;

// Generalised Gell-Mann generators / 2 in the order of the momentum components
// (symmetric pairs j<k, antisymmetric pairs, diagonal; src/group/algebra.hpp:23-49).
std::vector<cd> fund_generators(int N) {
  const int ng = N * N - 1;
  std::vector<cd> T((size_t)ng * N * N, cd(0, 0));
  int a = 0;
  for (int j = 0; j < N; ++j)
    for (int k = j + 1; k < N; ++k, ++a) {
      T[((size_t)a * N + j) * N + k] = cd(0.5, 0);
      T[((size_t)a * N + k) * N + j] = cd(0.5, 0);
    }
  for (int j = 0; j < N; ++j)
    for (int k = j + 1; k < N; ++k, ++a) {
      T[((size_t)a * N + j) * N + k] = cd(0, -0.5);
      T[((size_t)a * N + k) * N + j] = cd(0, 0.5);
    }
  for (int l = 1; l < N; ++l, ++a) {
    const double c = std::sqrt(2.0 / (double)(l * (l + 1)));
    for (int j = 0; j < l; ++j) T[((size_t)a * N + j) * N + j] = cd(0.5 * c, 0);
    T[((size_t)a * N + l) * N + l] = cd(-0.5 * l * c, 0);
  }
  return T;
}

// Adjoint generators (T^a)_bc = -i f^abc, f^abc = 2 Im Tr([T^a, T^b] T^c)
// (src/rep/rep_adjoint.hpp:12-24, src/group/algebra.hpp:103-120).
std::vector<cd> adj_generators(int N) {
  const int ng = N * N - 1;
  const std::vector<cd> t = fund_generators(N);
  auto el = [&](int a, int i, int j) { return t[((size_t)a * N + i) * N + j]; };
  std::vector<cd> T((size_t)ng * ng * ng, cd(0, 0));
  for (int a = 0; a < ng; ++a)
    for (int b = 0; b < ng; ++b)
      for (int c = 0; c < ng; ++c) {
        cd tr(0, 0);   // Tr([T^a, T^b] T^c)
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j)
            for (int k = 0; k < N; ++k) tr += (el(a, i, j) * el(b, j, k) - el(b, i, j) * el(a, j, k)) * el(c, k, i);
        T[((size_t)a * ng + b) * ng + c] = cd(0, -2.0 * tr.imag());
      }
  return T;
}

struct Sparse {           // CSR of the Casimir superoperator
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<cd> val;
  void apply(const std::vector<cd>& x, std::vector<cd>& y) const {
    for (int r = 0; r < n; ++r) {
      cd s(0, 0);
      for (int p = ptr[r]; p < ptr[r + 1]; ++p) s += val[p] * x[col[p]];
      y[r] = s;
    }
  }
};

// Chat[(i,j),(k,l)] = sum_a [(T_a^2)_ik delta_lj - 2 (T_a)_ik (T_a)_lj + delta_ik (T_a^2)_lj]
Sparse casimir_superop(const std::vector<cd>& T, int ng, int d) {
  const int n = d * d;
  std::vector<cd> dense((size_t)n * n, cd(0, 0));
  std::vector<cd> T2((size_t)d * d);
  for (int a = 0; a < ng; ++a) {
    const cd* t = &T[(size_t)a * d * d];
    for (int i = 0; i < d; ++i)
      for (int k = 0; k < d; ++k) {
        cd s(0, 0);
        for (int m = 0; m < d; ++m) s += t[i * d + m] * t[m * d + k];
        T2[i * d + k] = s;
      }
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j) {
        cd* row = &dense[(size_t)(i * d + j) * n];
        for (int k = 0; k < d; ++k) row[k * d + j] += T2[i * d + k];   // (T_a^2 M)_ij
        for (int l = 0; l < d; ++l) row[i * d + l] += T2[l * d + j];   // (M T_a^2)_ij
        for (int k = 0; k < d; ++k) {                                  // -2 (T_a M T_a)_ij
          if (t[i * d + k] == cd(0, 0)) continue;
          for (int l = 0; l < d; ++l)
            if (t[l * d + j] != cd(0, 0)) row[k * d + l] -= 2.0 * t[i * d + k] * t[l * d + j];
        }
      }
  }
  Sparse S;
  S.n = n;
  S.ptr.assign(n + 1, 0);
  for (int r = 0; r < n; ++r) {
    for (int c = 0; c < n; ++c) {
      const cd v = dense[(size_t)r * n + c];
      if (std::abs(v) > 1e-15) { S.col.push_back(c); S.val.push_back(v); }
    }
    S.ptr[r + 1] = (int)S.col.size();
  }
  return S;
}

cd dot(const std::vector<cd>& x, const std::vector<cd>& y) {
  cd s(0, 0);
  for (size_t i = 0; i < x.size(); ++i) s += std::conj(x[i]) * y[i];
  return s;
}

// Eigenvalues of a real symmetric m x m matrix (row-major) by cyclic Jacobi rotations.
std::vector<double> jacobi_eigenvalues(std::vector<double> A, int m) {
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) off += A[p * m + q] * A[p * m + q];
    if (off < 1e-30) break;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = A[p * m + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = 0.5 * (A[q * m + q] - A[p * m + p]) / apq;
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < m; ++k) {   // columns p, q
          const double akp = A[k * m + p], akq = A[k * m + q];
          A[k * m + p] = c * akp - s * akq;
          A[k * m + q] = s * akp + c * akq;
        }
        for (int k = 0; k < m; ++k) {   // rows p, q
          const double apk = A[p * m + k], aqk = A[q * m + k];
          A[p * m + k] = c * apk - s * aqk;
          A[q * m + k] = s * apk + c * aqk;
        }
      }
  }
  std::vector<double> ev(m);
  for (int i = 0; i < m; ++i) ev[i] = A[i * m + i];
  return ev;
}

// Distinct eigenvalues of the Hermitian superoperator, ascending.
std::vector<double> distinct_eigenvalues(const Sparse& C, int d) {
  const int n = C.n;
  // generic Hermitian start: entries from a fixed splitmix64 stream, M + M^dag
  std::vector<cd> v(n);
  uint64_t st = 0x9E3779B97F4A7C15ULL ^ (uint64_t)d;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * 0x1.0p-53 - 0.5;
  };
  std::vector<cd> R(n);
  for (int i = 0; i < n; ++i) R[i] = cd(next(), next());
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) v[i * d + j] = R[i * d + j] + std::conj(R[j * d + i]);
  double nv = std::sqrt(dot(v, v).real());
  for (auto& x : v) x /= nv;
  std::vector<std::vector<cd>> Q{v};
  std::vector<double> alpha, beta;
  std::vector<cd> w(n);
  double scale = 0.0;
  for (int k = 0; k < n; ++k) {
    C.apply(Q[k], w);
    const double a = dot(Q[k], w).real();
    alpha.push_back(a);
    scale = std::max(scale, std::fabs(a));
    for (int i = 0; i < n; ++i) w[i] -= a * Q[k][i];
    if (k > 0)
      for (int i = 0; i < n; ++i) w[i] -= beta[k - 1] * Q[k - 1][i];
    for (int pass = 0; pass < 2; ++pass)   // full reorthogonalisation, twice
      for (const auto& u : Q) {
        const cd o = dot(u, w);
        for (int i = 0; i < n; ++i) w[i] -= o * u[i];
      }
    const double b = std::sqrt(std::max(0.0, dot(w, w).real()));
    if (b <= 1e-9 * std::max(1.0, scale)) break;
    beta.push_back(b);
    for (auto& x : w) x /= b;
    Q.push_back(w);
  }
  const int m = (int)alpha.size();
  std::vector<double> Tri((size_t)m * m, 0.0);
  for (int i = 0; i < m; ++i) Tri[i * m + i] = alpha[i];
  for (int i = 0; i + 1 < m; ++i) Tri[i * m + i + 1] = Tri[(i + 1) * m + i] = beta[i];
  std::vector<double> ev = jacobi_eigenvalues(Tri, m);
  std::sort(ev.begin(), ev.end());
  std::vector<double> out;
  for (double e : ev)
    if (out.empty() || std::fabs(e - out.back()) > 1e-4) out.push_back(e);
  return out;
}

bool generators(int N, int kind, int d, const double* Tgen, std::vector<cd>& T, std::string& err) {
  const int ng = N * N - 1;
  if (kind == GH_REP_FUND) {
    if (d != N) { err = "fundamental representation needs d = N"; return false; }
    T = fund_generators(N);
  } else if (kind == GH_REP_ADJ) {
    if (d != ng) { err = "adjoint representation needs d = N*N-1"; return false; }
    T = adj_generators(N);
  } else if (kind == GH_REP_GENERAL) {
    if (!Tgen || d <= 0) { err = "general representation needs d and its generators T"; return false; }
    T.resize((size_t)ng * d * d);
    for (size_t i = 0; i < T.size(); ++i) T[i] = cd(Tgen[2 * i], Tgen[2 * i + 1]);
  } else {
    err = "the potential needs a scalar representation (fundamental, adjoint or general)";
    return false;
  }
  return true;
}

}  // namespace

namespace ghpot {

std::vector<std::complex<double>> gell_mann(int N) { return fund_generators(N); }

int channels(int N, int kind, int d, const double* Tgen, std::vector<double>& c2, std::string& err) {
  if (N != 2 && N != 3) { err = "N must be 2 or 3"; return GH_ERR_UNSUPPORTED; }
  if (d > POT_DMAX) { err = "representation dimension above the potential's limit of " + std::to_string(POT_DMAX); return GH_ERR_UNSUPPORTED; }
  std::vector<cd> T;
  if (!generators(N, kind, d, Tgen, T, err)) return GH_ERR_REP;
  c2 = distinct_eigenvalues(casimir_superop(T, N * N - 1, d), d);
  return GH_OK;
}

int superop(int N, int kind, int d, const double* Tgen, const std::vector<double>& f, std::vector<double>& c2,
            std::vector<double>& A, std::string& err) {
  if (N != 2 && N != 3) { err = "N must be 2 or 3"; return GH_ERR_UNSUPPORTED; }
  if (d > POT_DMAX) { err = "representation dimension above the potential's limit of " + std::to_string(POT_DMAX); return GH_ERR_UNSUPPORTED; }
  std::vector<cd> T;
  if (!generators(N, kind, d, Tgen, T, err)) return GH_ERR_REP;
  const Sparse C = casimir_superop(T, N * N - 1, d);
  c2 = distinct_eigenvalues(C, d);
  const int nch = (int)c2.size();
  if ((int)f.size() != nch) {
    err = "need " + std::to_string(nch) + " channel couplings, got " + std::to_string(f.size());
    return GH_ERR_ARG;
  }
  const int n = d * d;
  A.assign((size_t)2 * n * n, 0.0);
  std::vector<cd> x(n), y(n), col(n);
  for (int e = 0; e < n; ++e) {            // column e of A = sum_c 2 f_c P_c(E_e)
    std::fill(col.begin(), col.end(), cd(0, 0));
    for (int c = 0; c < nch; ++c) {
      if (f[c] == 0.0) continue;
      std::fill(x.begin(), x.end(), cd(0, 0));
      x[e] = cd(1, 0);
      for (int cp = 0; cp < nch; ++cp) {   // P_c = prod_{c' != c} (Chat - l_c') / (l_c - l_c')
        if (cp == c) continue;
        C.apply(x, y);
        const double inv = 1.0 / (c2[c] - c2[cp]);
        for (int i = 0; i < n; ++i) x[i] = (y[i] - c2[cp] * x[i]) * inv;
      }
      for (int i = 0; i < n; ++i) col[i] += 2.0 * f[c] * x[i];
    }
    for (int r = 0; r < n; ++r) {
      A[2 * ((size_t)r * n + e)] = col[r].real();
      A[2 * ((size_t)r * n + e) + 1] = col[r].imag();
    }
  }
  return GH_OK;
}

}  // namespace ghpot

extern "C" int gh_casimir_channels(int N, const gh_rep_desc* rep, double* c2, int cap, int* n_channels) {
  if (!rep) { ghpot::set_host_error("null representation"); return GH_ERR_ARG; }
  std::vector<double> v;
  std::string err;
  const int rc = ghpot::channels(N, rep->kind, rep->d, rep->T, v, err);
  if (rc) { ghpot::set_host_error(err); return rc; }
  if (n_channels) *n_channels = (int)v.size();
  if (c2)
    for (int c = 0; c < (int)v.size() && c < cap; ++c) c2[c] = v[c];
  return GH_OK;
}

extern "C" int gh_multi_superop(int N, const gh_rep_desc* rep, int n_channels, const double* f, double* A) {
  if (!rep || !A || (n_channels > 0 && !f)) { ghpot::set_host_error("null representation, couplings or output"); return GH_ERR_ARG; }
  std::vector<double> c2, Av;
  std::string err;
  const int rc = ghpot::superop(N, rep->kind, rep->d, rep->T, std::vector<double>(f, f + std::max(n_channels, 0)), c2, Av, err);
  if (rc) { ghpot::set_host_error(err); return rc; }
  std::copy(Av.begin(), Av.end(), A);
  return GH_OK;
}
