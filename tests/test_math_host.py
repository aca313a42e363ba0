"""The SU(N) arithmetic of gauge_higgs_b200/csrc/gh_math.cuh compiled for the host (the
header's functions are host-and-device): the staple products that form their last row
from unitarity (mm_su) against the full products, the Hermitian determinant against
the general one, and the SU(3) exponential (Cayley-Hamilton-reduced series, two terms
per trip) against a long-double Taylor series with scaling and squaring
(src/group/sun.hpp:11-29 computes the same exponential by a plain Taylor series).
The kernels use these functions unchanged, so the checks pin the device arithmetic."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r'''
#include "gh_math.cuh"
#include <cstdio>
#include <cmath>
#include <complex>
#include <random>
using namespace ghm;
typedef std::complex<long double> LC;
template <int N> Mat<N, double> su(std::mt19937_64& g, double s) {
  std::normal_distribution<double> n(0, 1);
  double v[N * N - 1];
  for (auto& x : v) x = s * n(g);
  return expi<N>(alg_to_mat<N, double>(v));
}
template <int N> double diff(const Mat<N, double>& a, const Mat<N, double>& b) {
  double m = 0;
  for (int i = 0; i < N * N; ++i) m = std::fmax(m, std::hypot(a.e[i].re - b.e[i].re, a.e[i].im - b.e[i].im));
  return m;
}
int main() {
  std::mt19937_64 g(7);
  std::normal_distribution<double> n(0, 1);
  double w3 = 0, w2 = 0, wdet = 0, wexp = 0, wexpf = 0;
  for (int t = 0; t < 20000; ++t) {
    const Mat<3, double> A = su<3>(g, 0.9), B = su<3>(g, 0.9);
    w3 = std::fmax(w3, diff<3>(mm_su<3, double, false, true>(A, B), mm_nd(A, B)));
    w3 = std::fmax(w3, diff<3>(mm_su<3, double, true, true>(A, B), mm_dd(A, B)));
    const Mat<2, double> C = su<2>(g, 0.9), D = su<2>(g, 0.9);
    w2 = std::fmax(w2, diff<2>(mm_su<2, double, false, true>(C, D), mm_nd(C, D)));
    w2 = std::fmax(w2, diff<2>(mm_su<2, double, true, true>(C, D), mm_dd(C, D)));
    // a Hermitian traceless H of norm ~1e-5 .. 2 (the drift's eps P and beyond the scaling threshold)
    const double sc = (t % 4 == 0) ? 2.0 : (t % 4 == 1) ? 0.3 : (t % 4 == 2) ? 0.06 : 1e-5;
    double v[8];
    for (auto& x : v) x = sc * n(g);
    const Mat<3, double> H = alg_to_mat<3, double>(v);
    wdet = std::fmax(wdet, std::fabs(det_herm3(H) - det<3, double>(H).re));
    // reference exp(iH): long-double Taylor, scaled to norm <= 0.1, squared back
    LC X[9], R[9], T[9];
    long double nr = 0;
    for (int i = 0; i < 9; ++i) nr += (long double)H.e[i].re * H.e[i].re + (long double)H.e[i].im * H.e[i].im;
    nr = std::sqrt(nr);
    int s = 0;
    while (nr > 0.1L) { nr /= 2; ++s; }
    for (int i = 0; i < 9; ++i) {
      X[i] = LC(0, 1) * LC(H.e[i].re, H.e[i].im) / std::pow(2.0L, s);
      R[i] = T[i] = (i % 4 == 0) ? 1 : 0;
    }
    for (int k = 1; k < 30; ++k) {
      LC Y[9];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Y[i * 3 + j] = 0; for (int l = 0; l < 3; ++l) Y[i * 3 + j] += T[i * 3 + l] * X[l * 3 + j]; }
      for (int i = 0; i < 9; ++i) { T[i] = Y[i] / (long double)k; R[i] += T[i]; }
    }
    for (int q = 0; q < s; ++q) {
      LC Y[9];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Y[i * 3 + j] = 0; for (int l = 0; l < 3; ++l) Y[i * 3 + j] += R[i * 3 + l] * R[l * 3 + j]; }
      for (int i = 0; i < 9; ++i) R[i] = Y[i];
    }
    const Mat<3, double> E = expi<3>(H);
    Mat<3, float> Hf;
    for (int i = 0; i < 9; ++i) Hf.e[i] = mk<float>((float)H.e[i].re, (float)H.e[i].im);
    const Mat<3, float> Ef = expi<3>(Hf);
    for (int i = 0; i < 9; ++i) {
      wexp = std::fmax(wexp, (double)std::abs(LC(E.e[i].re, E.e[i].im) - R[i]));
      wexpf = std::fmax(wexpf, (double)std::abs(LC(Ef.e[i].re, Ef.e[i].im) - R[i]));
    }
  }
  std::printf("%.3e %.3e %.3e %.3e %.3e\n", w3, w2, wdet, wexp, wexpf);
  return 0;
}
'''


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    d = tmp_path_factory.mktemp("mathhost")
    src, exe = d / "math_host.cpp", d / "math_host"
    src.write_text(SRC)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    "-I" + os.path.join(ROOT, "gauge_higgs_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    return dict(zip(["su3", "su2", "det", "exp", "expf"], map(float, out)))


def test_su_products_equal_full_products(results):
    assert results["su3"] < 1e-14
    assert results["su2"] < 1e-14


def test_hermitian_determinant(results):
    assert results["det"] < 1e-14


def test_exponential_against_long_double_taylor(results):
    assert results["exp"] < 1e-14
    assert results["expf"] < 5e-6      # FP32 arithmetic on the FP32-rounded H
