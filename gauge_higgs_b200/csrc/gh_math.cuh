// gh_math.cuh -- register-resident SU(N) algebra for the MD kernels.
//
// Conventions are the reference's (docs/conventions.md): Hermitian generators
// T^a = Lambda^a / 2 in generalised Gell-Mann order (symmetric pairs,
// antisymmetric pairs, diagonal; src/group/algebra.hpp:23-49), Tr T^aT^b = d/2.
// Nothing here materialises T^a: projections Im Tr(T^a M), 2 Tr(T^a M) and the
// map v -> sum_a v_a T^a are written out entry by entry from the sparse
// structure of the generators, which is what makes them cheap in registers.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define GH_HD __host__ __device__ __forceinline__
#define GH_D __device__ __forceinline__
#else
#define GH_HD inline
#define GH_D inline
#endif

namespace ghm {

template <typename T> struct cx { T re, im; };

template <typename T> GH_HD cx<T> mk(T r, T i) { cx<T> z; z.re = r; z.im = i; return z; }
template <typename T> GH_HD cx<T> zero() { return mk<T>(T(0), T(0)); }
template <typename T> GH_HD cx<T> add(cx<T> a, cx<T> b) { return mk<T>(a.re + b.re, a.im + b.im); }
template <typename T> GH_HD cx<T> sub(cx<T> a, cx<T> b) { return mk<T>(a.re - b.re, a.im - b.im); }
template <typename T> GH_HD cx<T> mul(cx<T> a, cx<T> b) { return mk<T>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
// a * conj(b)
template <typename T> GH_HD cx<T> mulc(cx<T> a, cx<T> b) { return mk<T>(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im); }
// conj(a) * b
template <typename T> GH_HD cx<T> cmul(cx<T> a, cx<T> b) { return mk<T>(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re); }
// conj(a) * conj(b)
template <typename T> GH_HD cx<T> cmulc(cx<T> a, cx<T> b) { return mk<T>(a.re * b.re - a.im * b.im, -(a.re * b.im + a.im * b.re)); }
template <typename T> GH_HD cx<T> conj(cx<T> a) { return mk<T>(a.re, -a.im); }
template <typename T> GH_HD cx<T> scale(cx<T> a, T s) { return mk<T>(a.re * s, a.im * s); }
template <typename T> GH_HD T norm2(cx<T> a) { return a.re * a.re + a.im * a.im; }
template <typename T, typename S> GH_HD cx<T> cvt(cx<S> a) { return mk<T>((T)a.re, (T)a.im); }

template <int N, typename T> struct Mat { cx<T> e[N * N]; };

template <int N, typename T> GH_HD void set_zero(Mat<N, T>& A) {
#pragma unroll
  for (int i = 0; i < N * N; ++i) A.e[i] = zero<T>();
}
template <int N, typename T> GH_HD void set_ident(Mat<N, T>& A) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) A.e[i * N + j] = mk<T>(i == j ? T(1) : T(0), T(0));
}
template <int N, typename T> GH_HD void acc(Mat<N, T>& A, const Mat<N, T>& B) {
#pragma unroll
  for (int i = 0; i < N * N; ++i) A.e[i] = add(A.e[i], B.e[i]);
}

// Fused multiply-add, rounded once, on host and device alike.
GH_HD float fmad(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
GH_HD double fmad(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

// s + a b and s + conj(a) b as four fused multiply-adds each
template <typename T> GH_HD cx<T> cfma(cx<T> s, cx<T> a, cx<T> b) {
  s.re = fmad(a.re, b.re, s.re);
  s.re = fmad(-a.im, b.im, s.re);
  s.im = fmad(a.re, b.im, s.im);
  s.im = fmad(a.im, b.re, s.im);
  return s;
}
template <typename T> GH_HD cx<T> cfma_cj(cx<T> s, cx<T> a, cx<T> b) {
  s.re = fmad(a.re, b.re, s.re);
  s.re = fmad(a.im, b.im, s.re);
  s.im = fmad(a.re, b.im, s.im);
  s.im = fmad(-a.im, b.re, s.im);
  return s;
}

// Matrix products C (+)= op(A) op(B), op = identity or dagger (DA, DB).  Every
// output entry is one chain of fused multiply-adds over k = 0..N-1: a complex
// multiply-accumulate is 4 FMAs (re += ar br -/+ ai bi, im += ar bi +/- ai br, the
// conjugation signs folded into operand negations), where the written-out form
// s + (ar br - ai bi) costs 6 (one product of each pair cannot fuse).
// Rows 0 .. ROWS-1 of the output only.
template <int N, typename T, bool DA, bool DB, bool ACC, int ROWS = N>
GH_HD void mm_core(const Mat<N, T>& A, const Mat<N, T>& B, Mat<N, T>& C) {
#pragma unroll
  for (int i = 0; i < ROWS; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<T> s = ACC ? C.e[i * N + j] : zero<T>();
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const cx<T> a = DA ? A.e[k * N + i] : A.e[i * N + k];
        const cx<T> b = DB ? B.e[j * N + k] : B.e[k * N + j];
        const T ai = DA ? -a.im : a.im;       // im of op(A)_ik
        const T bi = DB ? -b.im : b.im;       // im of op(B)_kj
        if (!ACC && k == 0) {
          s.re = a.re * b.re;
          s.im = a.re * bi;
        } else {
          s.re = fmad(a.re, b.re, s.re);
          s.im = fmad(a.re, bi, s.im);
        }
        s.re = fmad(-ai, bi, s.re);
        s.im = fmad(ai, b.re, s.im);
      }
      C.e[i * N + j] = s;
    }
}
// C = A B ; C = A B^dag ; C = A^dag B ; C = A^dag B^dag
template <int N, typename T> GH_HD Mat<N, T> mm(const Mat<N, T>& A, const Mat<N, T>& B) {
  Mat<N, T> C;
  mm_core<N, T, false, false, false>(A, B, C);
  return C;
}
template <int N, typename T> GH_HD Mat<N, T> mm_nd(const Mat<N, T>& A, const Mat<N, T>& B) {
  Mat<N, T> C;
  mm_core<N, T, false, true, false>(A, B, C);
  return C;
}
template <int N, typename T> GH_HD Mat<N, T> mm_dn(const Mat<N, T>& A, const Mat<N, T>& B) {
  Mat<N, T> C;
  mm_core<N, T, true, false, false>(A, B, C);
  return C;
}
template <int N, typename T> GH_HD Mat<N, T> mm_dd(const Mat<N, T>& A, const Mat<N, T>& B) {
  Mat<N, T> C;
  mm_core<N, T, true, true, false>(A, B, C);
  return C;
}
// conj(a b - c d), one chain of fused multiply-adds per part
template <typename T> GH_HD cx<T> conj_cross(const cx<T>& a, const cx<T>& b, const cx<T>& c, const cx<T>& d) {
  T re = c.im * d.im;
  re = fmad(-c.re, d.re, re);
  re = fmad(-a.im, b.im, re);
  re = fmad(a.re, b.re, re);
  T im = c.re * d.im;
  im = fmad(c.im, d.re, im);
  im = fmad(-a.re, b.im, im);
  im = fmad(-a.im, b.re, im);
  return mk<T>(re, im);
}
// Product of two SU(N) matrices, N = 2 or 3: the first N-1 rows as products, the last
// from them through unitarity and det = 1 (SU(3): row 2 = conj(row 0 x row 1); SU(2):
// row 1 = (-conj c01, conj c00)).  The last row costs 24 multiply-adds instead of 36
// (SU(3)), and the operand entries only it would read -- the last row of op(A) -- are
// never used, so their loads drop out.  The result differs from the full product by
// the operands' distance from SU(N) (rounding level for links of the HMC state).
// Other N: the full product.
template <int N, typename T, bool DA, bool DB> GH_HD Mat<N, T> mm_su(const Mat<N, T>& A, const Mat<N, T>& B) {
  Mat<N, T> C;
  if constexpr (N == 3) {
    mm_core<N, T, DA, DB, false, 2>(A, B, C);
    C.e[6] = conj_cross(C.e[1], C.e[5], C.e[2], C.e[4]);
    C.e[7] = conj_cross(C.e[2], C.e[3], C.e[0], C.e[5]);
    C.e[8] = conj_cross(C.e[0], C.e[4], C.e[1], C.e[3]);
  } else if constexpr (N == 2) {
    mm_core<N, T, DA, DB, false, 1>(A, B, C);
    C.e[2] = mk<T>(-C.e[1].re, C.e[1].im);
    C.e[3] = mk<T>(C.e[0].re, -C.e[0].im);
  } else {
    mm_core<N, T, DA, DB, false>(A, B, C);
  }
  return C;
}
// C += A B ; C += A B^dag
template <int N, typename T> GH_HD void mm_acc(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  mm_core<N, T, false, false, true>(A, B, C);
}
template <int N, typename T> GH_HD void mm_nd_acc(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  mm_core<N, T, false, true, true>(A, B, C);
}
// Re Tr(A B^dag) = sum_ij Re(A_ij conj(B_ij))
template <int N, typename T> GH_HD T retr_nd(const Mat<N, T>& A, const Mat<N, T>& B) {
  T s = T(0);
#pragma unroll
  for (int i = 0; i < N * N; ++i) s += A.e[i].re * B.e[i].re + A.e[i].im * B.e[i].im;
  return s;
}
template <int N, typename T> GH_HD T fnorm2(const Mat<N, T>& A) {
  T s = T(0);
#pragma unroll
  for (int i = 0; i < N * N; ++i) s += norm2(A.e[i]);
  return s;
}

// ---------------------------------------------------------------------------
// Generator maps (generalised Gell-Mann, T = Lambda/2).
// ---------------------------------------------------------------------------
template <int N> GH_HD constexpr int ngen() { return N * N - 1; }
template <int N> GH_HD constexpr int npair() { return N * (N - 1) / 2; }

// diagonal generator l (1..N-1): T_jj = c_l/2 (j<l), T_ll = -l c_l/2, c_l = sqrt(2/(l(l+1)))
GH_HD double diag_c(int l) {
  return (l == 1) ? 1.0 : (l == 2) ? 0.57735026918962573 : (l == 3) ? 0.40824829046386302 : sqrt(2.0 / (double)(l * (l + 1)));
}

// F_a = Im Tr(T^a M)   (the component projection of src/action/gauge_wilson.hpp:80-81)
template <int N, typename T> GH_HD void im_tr_proj(const Mat<N, T>& M, T* F) {
  int a = 0;
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int k = j + 1; k < N; ++k) F[a++] = T(0.5) * (M.e[k * N + j].im + M.e[j * N + k].im);
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int k = j + 1; k < N; ++k) F[a++] = T(0.5) * (M.e[j * N + k].re - M.e[k * N + j].re);
#pragma unroll
  for (int l = 1; l < N; ++l) {
    T s = T(0);
#pragma unroll
    for (int j = 0; j < l; ++j) s += M.e[j * N + j].im;
    F[a++] = T(0.5 * diag_c(l)) * (s - T(l) * M.e[l * N + l].im);
  }
}
// z_a = 2 Tr(T^a M) (complex); the inverse of alg_to_mat on traceless matrices
template <int N, typename T> GH_HD void tr2_proj(const Mat<N, T>& M, cx<T>* z) {
  int a = 0;
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int k = j + 1; k < N; ++k) z[a++] = add(M.e[k * N + j], M.e[j * N + k]);
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int k = j + 1; k < N; ++k) {
      const cx<T> d = sub(M.e[j * N + k], M.e[k * N + j]);   // -i M_kj + i M_jk = i (M_jk - M_kj)
      z[a++] = mk<T>(-d.im, d.re);
    }
#pragma unroll
  for (int l = 1; l < N; ++l) {
    cx<T> s = zero<T>();
#pragma unroll
    for (int j = 0; j < l; ++j) s = add(s, M.e[j * N + j]);
    s = sub(s, scale(M.e[l * N + l], T(l)));
    z[a++] = scale(s, T(diag_c(l)));
  }
}
// M = sum_a v_a T^a for real v (src/group/algebra.hpp:59-71)
template <int N, typename T> GH_HD Mat<N, T> alg_to_mat(const T* v) {
  Mat<N, T> M;
  set_zero(M);
  int a = 0;
  const int np = npair<N>();
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int k = j + 1; k < N; ++k, ++a) {
      const T s = T(0.5) * v[a], t = T(0.5) * v[a + np];
      M.e[j * N + k] = mk<T>(s, -t);
      M.e[k * N + j] = mk<T>(s, t);
    }
  a += np;
#pragma unroll
  for (int l = 1; l < N; ++l, ++a) {
    const T h = T(0.5 * diag_c(l)) * v[a];
#pragma unroll
    for (int j = 0; j < l; ++j) M.e[j * N + j].re += h;
    M.e[l * N + l].re -= T(l) * h;
  }
  return M;
}
// M = sum_a z_a T^a for complex z
template <int N, typename T> GH_HD Mat<N, T> alg_to_mat_c(const cx<T>* z) {
  Mat<N, T> M;
  set_zero(M);
  int a = 0;
  const int np = npair<N>();
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int k = j + 1; k < N; ++k, ++a) {
      const cx<T> s = scale(z[a], T(0.5)), t = scale(z[a + np], T(0.5));
      // T_sym: 1/2 at (j,k),(k,j); T_anti: -i/2 at (j,k), +i/2 at (k,j)
      M.e[j * N + k] = add(s, mk<T>(t.im, -t.re));
      M.e[k * N + j] = add(s, mk<T>(-t.im, t.re));
    }
  a += np;
#pragma unroll
  for (int l = 1; l < N; ++l, ++a) {
    const cx<T> h = scale(z[a], T(0.5 * diag_c(l)));
#pragma unroll
    for (int j = 0; j < l; ++j) M.e[j * N + j] = add(M.e[j * N + j], h);
    M.e[l * N + l] = sub(M.e[l * N + l], scale(h, T(l)));
  }
  return M;
}

template <int N, typename T> GH_HD cx<T> det(const Mat<N, T>& U);

// ---------------------------------------------------------------------------
// exp(iH), H Hermitian traceless, in FP64 (src/group/sun.hpp:11-45).
// General N: scaling and squaring to ||A||_F <= 1/2, then the Taylor series,
// stopped once a term falls below 1e-18 (the reference always sums 18 terms;
// the terms it adds past that point are below FP64 resolution).
// SU(2): the closed form cos r + i sin(r)/r H.
// ---------------------------------------------------------------------------
// Series cut-off per arithmetic type: a term below it no longer changes an O(1)
// coefficient (FP64: 1e-18; FP32: 1e-9, below half an FP32 ulp of 1).
template <typename T> struct ExpTol { static constexpr double v = 1e-18; };
template <> struct ExpTol<float> { static constexpr double v = 1e-9; };

template <int N, typename T> GH_HD Mat<N, T> expi_series(const Mat<N, T>& H) {
  const T nrm = sqrt(fnorm2(H));
  int s = 0;
  T scaled = nrm;
  while (scaled > T(0.5) && s < 64) { scaled *= T(0.5); ++s; }   // bounded: a non-finite H ends as NaN
  const T inv2s = (T)ldexp(1.0, -s);
  Mat<N, T> A, term, res;
#pragma unroll
  for (int i = 0; i < N * N; ++i) A.e[i] = mk<T>(-H.e[i].im * inv2s, H.e[i].re * inv2s);
  set_ident(term);
  set_ident(res);
  for (int k = 1; k <= 18; ++k) {
    term = mm(term, A);
    const T ik = (T)(1.0 / k);
#pragma unroll
    for (int i = 0; i < N * N; ++i) term.e[i] = scale(term.e[i], ik);
    acc(res, term);
    if (fnorm2(term) < T(ExpTol<T>::v * ExpTol<T>::v)) break;
  }
  for (int i = 0; i < s; ++i) res = mm(res, res);
  return res;
}
// SU(3): the same Taylor series sum_n (iQ)^n / n!, Q = H / 2^s, with every power
// reduced by the Cayley-Hamilton identity Q^3 = c1 Q + c0 I (c1 = Tr Q^2 / 2,
// c0 = det Q for traceless Q): Q^n = a_n I + b_n Q + g_n Q^2 with
// (a, b, g)_{n+1} = (c0 g_n, a_n + c1 g_n, b_n).  The series runs on three
// scalars instead of 3x3 matrices; exp(iQ) = f0 I + f1 Q + f2 Q^2.
// 1/n for the series coefficients (multiplications instead of FP64 divisions)
GH_HD double inv_int(int n) {
  switch (n) {
    case 1: return 1.0; case 2: return 0.5; case 3: return 1.0 / 3.0; case 4: return 0.25; case 5: return 0.2;
    case 6: return 1.0 / 6.0; case 7: return 1.0 / 7.0; case 8: return 0.125; case 9: return 1.0 / 9.0;
    case 10: return 0.1; case 11: return 1.0 / 11.0; case 12: return 1.0 / 12.0; case 13: return 1.0 / 13.0;
    case 14: return 1.0 / 14.0; case 15: return 1.0 / 15.0; case 16: return 0.0625; case 17: return 1.0 / 17.0;
    case 18: return 1.0 / 18.0; case 19: return 1.0 / 19.0; case 20: return 0.05; default: return 1.0 / n;
  }
}
// Q^2 of a Hermitian 3x3 Q: the diagonal is the squared row norms, the upper
// triangle three complex dot products, the lower triangle their conjugates (54
// multiply-adds instead of the general product's 108).
template <typename T> GH_HD Mat<3, T> herm_sq3(const Mat<3, T>& Q) {
  Mat<3, T> R;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T d = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) d = fmad(Q.e[i * 3 + k].re, Q.e[i * 3 + k].re, fmad(Q.e[i * 3 + k].im, Q.e[i * 3 + k].im, d));
    R.e[i * 4] = mk<T>(d, T(0));
#pragma unroll
    for (int j = i + 1; j < 3; ++j) {
      cx<T> z = zero<T>();
#pragma unroll
      for (int k = 0; k < 3; ++k) z = cfma(z, Q.e[i * 3 + k], Q.e[k * 3 + j]);
      R.e[i * 3 + j] = z;
      R.e[j * 3 + i] = conj(z);
    }
  }
  return R;
}
// det of a Hermitian 3x3 (real diagonal d_i, upper entries a = q01, b = q02, c = q12):
//   d0 d1 d2 + 2 Re(a c conj(b)) - d0 |c|^2 - d1 |b|^2 - d2 |a|^2
template <typename T> GH_HD T det_herm3(const Mat<3, T>& Q) {
  const T d0 = Q.e[0].re, d1 = Q.e[4].re, d2 = Q.e[8].re;
  const cx<T> a = Q.e[1], b = Q.e[2], c = Q.e[5];
  const cx<T> ac = mul(a, c);
  T r = d0 * d1 * d2;
  r = fmad(T(2), fmad(ac.re, b.re, ac.im * b.im), r);
  r = fmad(-d0, norm2(c), r);
  r = fmad(-d1, norm2(b), r);
  r = fmad(-d2, norm2(a), r);
  return r;
}
template <typename T> GH_HD Mat<3, T> expi3(const Mat<3, T>& H) {
  T nrm2 = fnorm2(H);               // scale until ||H||_F / 2^s <= 1/2, compared squared
  int s = 0;
  while (nrm2 > T(0.25) && s < 64) { nrm2 *= T(0.25); ++s; }   // bounded: a non-finite H ends as NaN
  Mat<3, T> Q = H;
  if (s > 0) {                      // rare: the MD step keeps ||eps P|| well below 1/2
    const T sc = (T)ldexp(1.0, -s);
#pragma unroll
    for (int i = 0; i < 9; ++i) Q.e[i] = scale(H.e[i], sc);
  }
  const Mat<3, T> Q2 = herm_sq3(Q);   // H (and Q) Hermitian: built from real algebra coefficients
  const T c1 = T(0.5) * (Q2.e[0].re + Q2.e[4].re + Q2.e[8].re);
  const T c0 = det_herm3(Q);
  // (a, b, g): the coefficients of Q^n / n! in (I, Q, Q^2), advanced two terms per trip
  // (i^n = i, -1 for n = 4k+1, 4k+2 and -i, 1 for n = 4k+3, 4k+4)
  T a = 1, b = 0, g = 0;
  T f0r = 1, f0i = 0, f1r = 0, f1i = 0, f2r = 0, f2i = 0;
#pragma unroll
  for (int n = 1; n < 40; n += 2) {
    const T sg = (n & 2) ? T(-1) : T(1);
    T r = (T)inv_int(n);
    T an = c0 * g * r, bn = fmad(c1, g, a) * r, gn = b * r;
    f0i = fmad(sg, an, f0i); f1i = fmad(sg, bn, f1i); f2i = fmad(sg, gn, f2i);
    r = (T)inv_int(n + 1);
    a = c0 * gn * r; b = fmad(c1, gn, an) * r; g = bn * r;
    f0r = fmad(-sg, a, f0r); f1r = fmad(-sg, b, f1r); f2r = fmad(-sg, g, f2r);
    if (fabs(a) + fabs(b) + fabs(g) < T(ExpTol<T>::v)) break;
  }
  Mat<3, T> E;
#pragma unroll
  for (int i = 0; i < 9; ++i)
    E.e[i] = add(mul(mk<T>(f1r, f1i), Q.e[i]), mul(mk<T>(f2r, f2i), Q2.e[i]));
  E.e[0].re += f0r; E.e[0].im += f0i;
  E.e[4].re += f0r; E.e[4].im += f0i;
  E.e[8].re += f0r; E.e[8].im += f0i;
  for (int i = 0; i < s; ++i) E = mm(E, E);
  return E;
}
template <typename T> GH_HD Mat<2, T> expi2(const Mat<2, T>& H) {
  // r^2 = Tr(H^2)/2
  T trh2 = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int k = 0; k < 2; ++k) trh2 += mul(H.e[i * 2 + k], H.e[k * 2 + i]).re;
  const T r2 = T(0.5) * trh2;
  const T r = sqrt(r2 > T(0) ? r2 : T(0));
  T c, sinc;
  // below the cut-off the next terms of cos r and sin(r)/r are under the type's resolution
  const T rsmall = sizeof(T) == sizeof(double) ? T(1e-8) : T(1e-4);
  if (r < rsmall) { c = T(1) - T(0.5) * r2; sinc = T(1) - r2 / T(6); }
  else { T sn; sincos(r, &sn, &c); sinc = sn / r; }
  Mat<2, T> U;
#pragma unroll
  for (int i = 0; i < 4; ++i) U.e[i] = mk<T>(-sinc * H.e[i].im, sinc * H.e[i].re);
  U.e[0].re += c;
  U.e[3].re += c;
  return U;
}
// exp(iH) in the arithmetic type of H
template <int N, typename T> GH_HD Mat<N, T> expi(const Mat<N, T>& H) {
  if constexpr (N == 3) return expi3<T>(H);
  else if constexpr (N == 2) return expi2<T>(H);
  else return expi_series<N, T>(H);
}

// Determinant (N <= 4), Gaussian elimination without pivoting for N=4 falls back
// to cofactors; N=2,3 closed forms.
template <int N, typename T> GH_HD cx<T> det(const Mat<N, T>& U) {
  if (N == 2) return sub(mul(U.e[0], U.e[3]), mul(U.e[1], U.e[2]));
  if (N == 3) {
    const cx<T> c0 = sub(mul(U.e[4], U.e[8]), mul(U.e[5], U.e[7]));
    const cx<T> c1 = sub(mul(U.e[5], U.e[6]), mul(U.e[3], U.e[8]));
    const cx<T> c2 = sub(mul(U.e[3], U.e[7]), mul(U.e[4], U.e[6]));
    return add(add(mul(U.e[0], c0), mul(U.e[1], c1)), mul(U.e[2], c2));
  }
  // generic: elimination with partial pivoting on a copy
  Mat<N, T> m = U;
  cx<T> d = mk<T>(T(1), T(0));
  for (int col = 0; col < N; ++col) {
    int piv = col;
    T best = norm2(m.e[col * N + col]);
    for (int r = col + 1; r < N; ++r) { T v = norm2(m.e[r * N + col]); if (v > best) { best = v; piv = r; } }
    if (best == T(0)) return zero<T>();
    if (piv != col) {
      for (int j = 0; j < N; ++j) { cx<T> t = m.e[piv * N + j]; m.e[piv * N + j] = m.e[col * N + j]; m.e[col * N + j] = t; }
      d = mk<T>(-d.re, -d.im);
    }
    d = mul(d, m.e[col * N + col]);
    const T in2 = T(1) / norm2(m.e[col * N + col]);
    const cx<T> inv = scale(conj(m.e[col * N + col]), in2);
    for (int r = col + 1; r < N; ++r) {
      const cx<T> f = mul(m.e[r * N + col], inv);
      for (int j = col; j < N; ++j) m.e[r * N + j] = sub(m.e[r * N + j], mul(f, m.e[col * N + j]));
    }
  }
  return d;
}

// Modified Gram-Schmidt on rows, then det phase removed from row 0
// (src/group/sun.hpp:48-71).
template <int N, typename T> GH_HD void reunitarize(Mat<N, T>& U) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int k = 0; k < i; ++k) {
      cx<T> p = zero<T>();
#pragma unroll
      for (int j = 0; j < N; ++j) p = add(p, cmul(U.e[k * N + j], U.e[i * N + j]));
#pragma unroll
      for (int j = 0; j < N; ++j) U.e[i * N + j] = sub(U.e[i * N + j], mul(p, U.e[k * N + j]));
    }
    T n = T(0);
#pragma unroll
    for (int j = 0; j < N; ++j) n += norm2(U.e[i * N + j]);
    const T inv = T(1) / sqrt(n);
#pragma unroll
    for (int j = 0; j < N; ++j) U.e[i * N + j] = scale(U.e[i * N + j], inv);
  }
  const cx<T> d = det<N, T>(U);
  const T ad = sqrt(norm2(d));
  if (ad > T(0)) {
    const cx<T> ph = mk<T>(d.re / ad, -d.im / ad);   // conj(d/|d|)
#pragma unroll
    for (int j = 0; j < N; ++j) U.e[j] = mul(U.e[j], ph);
  }
}

}  // namespace ghm
