// gh_potential.h -- host set-up of the multi-invariant onsite potential (gh_potential.cpp).
#pragma once
#include <complex>
#include <string>
#include <vector>

namespace ghpot {
constexpr int POT_DMAX = 32;   // largest representation dimension the potential accepts
// Distinct adjoint-Casimir eigenvalues of R (x) Rbar, ascending (the channel order).
int channels(int N, int kind, int d, const double* Tgen, std::vector<double>& c2, std::string& err);
// The channels and A = sum_c 2 f_c P_c, [(p*d+q)*d*d + (i*d+j)] complex as re, im pairs.
int superop(int N, int kind, int d, const double* Tgen, const std::vector<double>& f, std::vector<double>& c2,
            std::vector<double>& A, std::string& err);
// Generalised Gell-Mann generators / 2, [a][i][j], in the momentum components' order.
std::vector<std::complex<double>> gell_mann(int N);
// Message of a failed context-free call, read back by gh_last_error(NULL) (gh_ctx.cu).
void set_host_error(const std::string& m);
}  // namespace ghpot
