// Closed-form representation matrices of the single-row (totally symmetric) irreps
// of SU(N) in the reference's GeneralRep basis (src/rep/rep_general.hpp:54-84,330-362).
//
// For a single-row Young diagram [n] every basis vector of the reference is one
// multiset m of slot indices (m_i slots hold index i), written as a constant times
// the sum over the n!/prod(m_i!) distinct arrangements of that multiset.  Then
//   D(U)[k][l] = <W_k| U^(x)n |W_l>
//              = conj(w_k) w_l A(m_k) sum_K prod_i [m_k(i)! / prod_j K_ij!] prod_ij U_ij^K_ij
// where w_k is the common entry of W_k, A(m) = n!/prod(m_i!) the number of
// arrangements, and K runs over the N x N non-negative integer matrices with row sums
// m_k and column sums m_l.  This is the tensor construction rep_matrix_tensor
// (src/rep/rep_general.hpp:122-131) summed in closed form, so it is exact; its cost
// is the number of (k, l, K) terms instead of the N^n tensor.  The reference's own
// fast path for these irreps, exp(i w.T_R) with w taken from the fundamental link
// (src/rep/rep_general.hpp:94-112,165-179), agrees with the tensor matrix to its 1e-7 check.
#pragma once
#include <string>
#include <vector>

namespace ghsym {

struct Terms {
  int N = 0, n = 0, d = 0;
  std::vector<int> ptr;            // d*d + 1: terms of entry k*d + l
  std::vector<double> c;           // 2 per term: complex coefficient
  std::vector<unsigned char> e;    // per term: exponents K_ij (row-major), N*N bytes padded to a multiple of 4
  // per term, for the device: offsets ij*(n+1) + K_ij into the table of powers U_ij^p, as
  // bytes in whole 32-bit words.  N = 2: all four factors (an exponent 0 points at the
  // table's 1); N > 2: the factors with K_ij > 0, in ij order, then 0xFF.
  std::vector<unsigned char> off;
};

// Builds the term list when W ([d][dimT] complex, slot 0 the most significant base-N
// digit of the tensor index) is a symmetric-power basis with at most max_terms terms,
// and checks it against the tensor construction on two fixed SU(N) links (max entry
// difference below 1e-10).  Returns false, with the reason in *why, otherwise.
bool build(int N, int n, int d, long dimT, const double* W, long max_terms, Terms& out, std::string* why);

// D(U) from the term list (host).  U: N x N complex row-major; D: d x d complex.
void eval(const Terms& t, const double* U, double* D);

// D(U) by the tensor construction (host): lift W_l, apply U on every slot, project.
void tensor_matrix(int N, int n, int d, long dimT, const double* W, const double* U, double* D);

}  // namespace ghsym
