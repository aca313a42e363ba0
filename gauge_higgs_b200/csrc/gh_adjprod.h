// General irreps as a piece of a product of adjoints (host set-up, gh_adjprod.cpp).
//
// The reference applies a general irrep R of SU(N) on the tensor space V^(x)n
// (src/rep/rep_general.hpp:184-220): lift with its basis W, act with U on each of the
// n slots, project.  When n = K N, the adjoint representation's K-fold tensor
// product also lives in V^(x)n: the adjoint vector phi = sum_b phi_b T^b is the matrix
// Phi in V (x) Vbar, and Vbar is Lambda^(N-1) V for SU(N) (conj(e_j) -> the
// Levi-Civita tensor eps_{j k ...}), so
//   E1: phi -> sum_{i j k..} (sum_b phi_b T^b_ij) eps_{j k..} e_i (x) e_k (x) ...
// commutes with the group action (U Phi U^dag on the left, U^(x)N on the right,
// because det U = 1).  For any permutation pi of the n slots, M = E_pi^dag W^T is then
// an intertwiner from R (the reference's basis) into the K-fold adjoint product, and
// by Schur's lemma M^dag M = c^2 I.  With Q = M / c (an isometry) the representation
// matrix in the reference's basis is exactly
//   D_R(U) = Q^dag (D_adj(U) (x) ... (x) D_adj(U)) Q,   D_adj(U)_ab = 2 Re Tr(T^a U T^b U^dag),
// D_adj a real (N^2-1) x (N^2-1) matrix.  For the SU(3) 27-plet {4,2} (n = 6, K = 2)
// that is a 64 x 27 lift, two 8 x 8 products per link and a 27 x 64 projection, in
// place of six slot sweeps over 729 entries.  The slot permutation is the one with
// the largest overlap c; the result is checked against the tensor construction on
// two generic links before a context uses it.
#pragma once
#include <complex>
#include <string>
#include <vector>

namespace ghadj {

struct Product {
  int N = 0, K = 0, d = 0, A = 0;          // A = (N^2 - 1)^K
  std::vector<std::complex<double>> Q;     // [A][d]: isometric intertwiner R -> adjoint^(x)K
  double c2 = 0.0;                         // squared overlap of the chosen slot order
  // The rows the device lifts into.  K = 2 and every column of Q a symmetric (sym = +1) or
  // antisymmetric (sym = -1) ng x ng matrix: only the pairs a <= b (a < b) are lifted,
  // the mirror entry written as +-x, and the projection weights the off-diagonal pairs by 2.
  // Otherwise (sym = 0) every row.  rows[r] = a ng + b; the first ndiag rows are diagonal.
  int sym = 0;
  int ndiag = 0;
  std::vector<int> rows;
  std::vector<std::complex<double>> Qr;    // [rows.size()][d]: the rows of Q the device uses
};

// Builds Q for the irrep whose basis is W ([d][dimT] complex, slot 0 the most
// significant base-N digit of the tensor index) when n = K N with K = 1 or 2 and
// N = 2 or 3; false (reason in *why) when the irrep is not reached that way.
bool build(int N, int n, int d, long dimT, const double* W, Product& out, std::string* why);

// Adjoint matrix of an SU(N) link (host): D[a][b] = 2 Re Tr(T^a U T^b U^dag).
void adjoint_matrix(int N, const double* U, double* Dadj);

// D_R(U) = Q^dag (D_adj (x)...(x) D_adj) Q (host).  U: N x N complex; D: d x d complex.
void eval(const Product& p, const double* U, double* D);

}  // namespace ghadj
