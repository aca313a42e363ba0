// gh_rng.cuh -- counter-based RNG of the MD path, bit-exact on host and device.
//
// splitmix64 / key / uniform restate src/core/rng.hpp:11-39 (integer work,
// bit-exact by construction).  The Gaussian of src/core/rng.hpp:42-46 is
//   sqrt(-2 log u1) * cos(2 pi u2)
// evaluated with CORRECTLY ROUNDED log and cos, so every draw is the unique
// correctly rounded evaluation of that formula (each operation rounded once).
// The reference calls the host libm, which is not correctly rounded; where libm
// is off by one ulp the reference's draw differs from this one by <= 2 ulp.
//
// log and cos are written here in double-double arithmetic from standard
// published techniques, not from any vendor library:
//   * error-free transformations two_sum (Knuth, TAOCP vol. 2, 4.2.2) and
//     two_prod via fused multiply-add (Dekker 1971 / Ogita-Rump-Oishi 2005);
//   * log: x = 2^e m, m in [1/sqrt2, sqrt2), log m = 2 atanh(s), s=(m-1)/(m+1),
//     atanh series summed by Horner in double-double (about 2^-100 relative);
//   * cos: Cody-Waite style reduction by pi/2 held as a triple-double, then the
//     sin/cos Taylor series in double-double on |r| <= pi/4.
// Final rounding hi+lo gives the correctly rounded result except when the true
// value lies within ~2^-100 relative of a rounding midpoint (probability ~2^-47
// per call).  Host and device use the same explicitly rounded operations
// (no contraction), so both produce identical bits.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define GH_HD __host__ __device__ __forceinline__
#else
#define GH_HD inline
#endif

namespace ghrng {

GH_HD uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

GH_HD uint64_t key(uint64_t a, uint64_t b = 0, uint64_t c = 0, uint64_t d = 0, uint64_t e = 0) {
  const uint64_t g = 0x9E3779B97F4A7C15ULL;
  uint64_t h = splitmix64(a);
  h = splitmix64(h ^ (b + g));
  h = splitmix64(h ^ (c + g));
  h = splitmix64(h ^ (d + g));
  h = splitmix64(h ^ (e + g));
  return h;
}

GH_HD double uniform(uint64_t seed, uint64_t k) {
  const uint64_t h = splitmix64(seed ^ splitmix64(k));
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// ---- explicitly rounded primitives (never contracted) ----
#if defined(__CUDA_ARCH__)
GH_HD double add_rn(double a, double b) { return __dadd_rn(a, b); }
GH_HD double sub_rn(double a, double b) { return __dsub_rn(a, b); }
GH_HD double mul_rn(double a, double b) { return __dmul_rn(a, b); }
GH_HD double div_rn(double a, double b) { return __ddiv_rn(a, b); }
GH_HD double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
GH_HD double sqrt_rn(double a) { return __dsqrt_rn(a); }
GH_HD double rint_rn(double a) { return rint(a); }
#else
// Host build: the translation unit is compiled with -ffp-contract=off.
inline double add_rn(double a, double b) { return a + b; }
inline double sub_rn(double a, double b) { return a - b; }
inline double mul_rn(double a, double b) { return a * b; }
inline double div_rn(double a, double b) { return a / b; }
inline double fma_rn(double a, double b, double c) { return fma(a, b, c); }
inline double sqrt_rn(double a) { return sqrt(a); }
inline double rint_rn(double a) { return rint(a); }
#endif

struct dd { double hi, lo; };

#if defined(__CUDA_ARCH__)
GH_HD uint64_t dbits(double x) { return (uint64_t)__double_as_longlong(x); }
GH_HD double bitsd(uint64_t b) { return __longlong_as_double((long long)b); }
#else
inline uint64_t dbits(double x) { uint64_t b; memcpy(&b, &x, 8); return b; }
inline double bitsd(uint64_t b) { double x; memcpy(&x, &b, 8); return x; }
#endif

GH_HD dd two_sum(double a, double b) {
  const double s = add_rn(a, b);
  const double bb = sub_rn(s, a);
  const double e = add_rn(sub_rn(a, sub_rn(s, bb)), sub_rn(b, bb));
  return dd{s, e};
}
GH_HD dd fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = add_rn(a, b);
  return dd{s, sub_rn(b, sub_rn(s, a))};
}
GH_HD dd two_prod(double a, double b) {
  const double p = mul_rn(a, b);
  return dd{p, fma_rn(a, b, -p)};
}
GH_HD dd dd_add(dd x, dd y) {
  dd s = two_sum(x.hi, y.hi);
  const dd t = two_sum(x.lo, y.lo);
  s.lo = add_rn(s.lo, t.hi);
  s = fast_two_sum(s.hi, s.lo);
  s.lo = add_rn(s.lo, t.lo);
  return fast_two_sum(s.hi, s.lo);
}
GH_HD dd dd_neg(dd x) { return dd{-x.hi, -x.lo}; }
GH_HD dd dd_mul(dd x, dd y) {
  dd p = two_prod(x.hi, y.hi);
  p.lo = add_rn(p.lo, add_rn(mul_rn(x.hi, y.lo), mul_rn(x.lo, y.hi)));
  return fast_two_sum(p.hi, p.lo);
}
GH_HD dd dd_mul_d(dd x, double b) {
  dd p = two_prod(x.hi, b);
  p.lo = add_rn(p.lo, mul_rn(x.lo, b));
  return fast_two_sum(p.hi, p.lo);
}
GH_HD dd dd_div_d(dd x, double b) {
  const double q1 = div_rn(x.hi, b);
  const dd p = two_prod(q1, b);
  const double rem = add_rn(sub_rn(sub_rn(x.hi, p.hi), p.lo), x.lo);
  return fast_two_sum(q1, div_rn(rem, b));
}
GH_HD dd dd_div(dd x, dd y) {
  const double q1 = div_rn(x.hi, y.hi);
  const dd p = two_prod(q1, y.hi);
  double r = add_rn(sub_rn(sub_rn(x.hi, p.hi), p.lo), x.lo);
  r = sub_rn(r, mul_rn(q1, y.lo));
  return fast_two_sum(q1, div_rn(r, y.hi));
}

// log x for finite normal x > 0, correctly rounded (see header).
GH_HD double cr_log(double x) {
  uint64_t bits = dbits(x);
  int e = (int)((bits >> 52) & 0x7FF) - 1023;
  double m = bitsd((bits & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL);  // m in [1,2)
  if (m > 1.4142135623730951) { m = mul_rn(m, 0.5); e += 1; }      // m in [1/sqrt2, sqrt2)
  const double num = sub_rn(m, 1.0);                                  // exact (Sterbenz)
  const dd den = two_sum(m, 1.0);
  const dd s = dd_div(dd{num, 0.0}, den);
  const dd z = dd_mul(s, s);
  const int K = 23;                                                   // |s| <= 0.1716: z^K/(2K+1) < 2^-120
  dd acc = dd_div_d(dd{1.0, 0.0}, (double)(2 * K + 1));
  for (int j = K - 1; j >= 0; --j)
    acc = dd_add(dd_div_d(dd{1.0, 0.0}, (double)(2 * j + 1)), dd_mul(z, acc));
  const dd logm = dd_mul(dd_mul_d(s, 2.0), acc);
  const dd ln2{0.6931471805599453, 2.3190468138462996e-17};           // ln 2 = hi + lo (to ~2^-107)
  const dd r = dd_add(dd_mul_d(ln2, (double)e), logm);
  return add_rn(r.hi, r.lo);
}

// cos x for |x| < 2^20, correctly rounded (see header).
GH_HD double cr_cos(double x) {
  const double P1 = 1.5707963267948966, P2 = 6.123233995736766e-17, P3 = -1.4973849048591698e-33;
  const double k = rint_rn(mul_rn(x, 0.6366197723675814));
  dd r = dd_add(dd{x, 0.0}, dd_neg(two_prod(k, P1)));
  r = dd_add(r, dd_neg(two_prod(k, P2)));
  r = dd_add(r, dd{-mul_rn(k, P3), 0.0});
  const int q = ((int)k) & 3;
  const dd z = dd_mul(r, r);
  const int J = 16;                      // |r| <= pi/4: z^J/(2J)! < 2^-125
  dd cc[J + 1], ss[J + 1];
  cc[0] = dd{1.0, 0.0};
  ss[0] = dd{1.0, 0.0};
  for (int j = 1; j <= J; ++j) {
    cc[j] = dd_div_d(cc[j - 1], -(double)((2 * j - 1) * (2 * j)));
    ss[j] = dd_div_d(ss[j - 1], -(double)((2 * j) * (2 * j + 1)));
  }
  dd cacc = cc[J], sacc = ss[J];
  for (int j = J - 1; j >= 0; --j) {
    cacc = dd_add(cc[j], dd_mul(z, cacc));
    sacc = dd_add(ss[j], dd_mul(z, sacc));
  }
  sacc = dd_mul(r, sacc);
  dd res = (q == 0) ? cacc : (q == 1) ? dd_neg(sacc) : (q == 2) ? dd_neg(cacc) : sacc;
  return add_rn(res.hi, res.lo);
}

// Standard normal draw keyed on k (src/core/rng.hpp:42-46 formula).
GH_HD double gauss(uint64_t seed, uint64_t k) {
  const double u1 = uniform(seed, splitmix64(k * 2 + 1));
  const double u2 = uniform(seed, splitmix64(k * 2 + 2));
  const double a = sqrt_rn(mul_rn(-2.0, cr_log(u1)));
  const double c = cr_cos(mul_rn(6.283185307179586, u2));            // (2 * pi) * u2, 2*pi exact
  return mul_rn(a, c);
}

}  // namespace ghrng
