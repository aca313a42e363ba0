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
//   * table-driven argument reduction in the manner of Tang (ACM TOMS 1989/1990)
//     with double-double tables from gen_rng_tables.py (mpmath, 400 bits);
//   * log: x = 2^e m, m in [1/sqrt2, sqrt2), m = c (1 + r) with c = i/128,
//     log m = log c + 2 atanh(s), s = (m - c)/(m + c), series in double-double;
//   * cos: Cody-Waite style reduction by pi/32 held as a triple-double, then
//     the addition formula with tabulated cos / sin(j pi/32) and the sin/cos
//     Taylor series in double-double on |r| <= pi/64.
// Final rounding hi+lo gives the correctly rounded result except when the true
// value lies within ~2^-100 relative of a rounding midpoint (probability ~2^-47
// per call).  The Gaussian calls them through a cheaper first phase (Ziv's
// strategy, cr_log_fast / cr_cos_fast) that returns the same value whenever its
// own error bound settles the rounding, and falls back to them otherwise.  Host and device use the same explicitly rounded operations
// (no contraction), so both produce identical bits.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>
#include "gh_rng_tables.cuh"

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

// Table storage: global memory on the device (threads of a warp index it at
// random, which constant memory would serialise), static arrays on the host.
#if defined(__CUDACC__)
static __device__ const double g_logc_d[] = {GH_TAB_LOGC};
static __device__ const double g_cos_d[] = {GH_TAB_COS};
static __device__ const double g_sin_d[] = {GH_TAB_SIN};
static __device__ const double g_odd_d[] = {GH_TAB_ODD};
static __device__ const double g_cfac_d[] = {GH_TAB_CFAC};
static __device__ const double g_sfac_d[] = {GH_TAB_SFAC};
#endif
static const double g_logc_h[] = {GH_TAB_LOGC};
static const double g_cos_h[] = {GH_TAB_COS};
static const double g_sin_h[] = {GH_TAB_SIN};
static const double g_odd_h[] = {GH_TAB_ODD};
static const double g_cfac_h[] = {GH_TAB_CFAC};
static const double g_sfac_h[] = {GH_TAB_SFAC};
#if defined(__CUDA_ARCH__)
#define GH_TAB(name, i) dd{__ldg(&g_##name##_d[2 * (i)]), __ldg(&g_##name##_d[2 * (i) + 1])}
#else
#define GH_TAB(name, i) dd{g_##name##_h[2 * (i)], g_##name##_h[2 * (i) + 1]}
#endif

// log x for finite normal x > 0, correctly rounded (see header).
// x = 2^e m, m in [1/sqrt2, sqrt2); c = i/128 nearest to m (i = 91..181);
// log m = log c + 2 atanh(s), s = (m - c)/(m + c), |s| < 0.0028 (7 series terms).
GH_HD double cr_log(double x) {
  const uint64_t bits = dbits(x);
  int e = (int)((bits >> 52) & 0x7FF) - 1023;
  double m = bitsd((bits & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL);  // m in [1,2)
  if (m > 1.4142135623730951) { m = mul_rn(m, 0.5); e += 1; }                 // exact
  const double ci = rint_rn(mul_rn(m, 128.0));
  const int i = (int)ci;
  const double c = mul_rn(ci, 0.0078125);                                      // i/128, exact
  const double t = sub_rn(m, c);                                               // exact, |t| <= 1/256
  const dd s = dd_div(dd{t, 0.0}, two_sum(mul_rn(2.0, c), t));
  const dd z = dd_mul(s, s);
  dd acc = GH_TAB(odd, 7);
  for (int j = 6; j >= 0; --j) acc = dd_add(GH_TAB(odd, j), dd_mul(z, acc));
  const dd lm = dd_add(GH_TAB(logc, i - 90), dd_mul(dd_mul_d(s, 2.0), acc));
  const dd r = dd_add(dd_mul_d(dd{GH_LN2_HI, GH_LN2_LO}, (double)e), lm);
  return add_rn(r.hi, r.lo);
}

// cos x for |x| < 2^20, correctly rounded (see header).
// x = k pi/32 + r, |r| <= pi/64 (pi/32 as a triple-double); with j = k mod 64,
// cos x = cos(j pi/32) cos r - sin(j pi/32) sin r, series to z^9 (z = r^2).
GH_HD double cr_cos(double x) {
  const double k = rint_rn(mul_rn(x, GH_32_OVER_PI));
  dd r = dd_add(dd{x, 0.0}, dd_neg(two_prod(k, GH_PI32_1)));
  r = dd_add(r, dd_neg(two_prod(k, GH_PI32_2)));
  r = dd_add(r, dd{-mul_rn(k, GH_PI32_3), 0.0});
  const int j = ((int)k) & 63;
  const dd z = dd_mul(r, r);
  dd ca = GH_TAB(cfac, 9), sa = GH_TAB(sfac, 9);
  for (int q = 8; q >= 0; --q) {
    ca = dd_add(GH_TAB(cfac, q), dd_mul(z, ca));
    sa = dd_add(GH_TAB(sfac, q), dd_mul(z, sa));
  }
  sa = dd_mul(r, sa);
  const dd res = dd_add(dd_mul(GH_TAB(cos, j), ca), dd_neg(dd_mul(GH_TAB(sin, j), sa)));
  return add_rn(res.hi, res.lo);
}

// Two-phase evaluation (Ziv's strategy): a first phase accurate to ~2^-66 whose
// result comes with an error bound E; when hi + lo - E and hi + lo + E round to the
// same double, that double is the correctly rounded value, and the first phase
// returns it.  Otherwise (about one call in 2^12) the double-double evaluation
// above decides.  Either way the result is the one cr_log / cr_cos give.
GH_HD bool ziv_round(dd r, double E, double* y) {
  const double a = add_rn(r.hi, add_rn(r.lo, E)), b = add_rn(r.hi, sub_rn(r.lo, E));
  *y = add_rn(r.hi, r.lo);
  return a == b;
}

// log x, first phase: the reduction of cr_log, then log m = log c + 2s + tail with the
// tail 2s (s^2/3 + s^4/5 + s^6/7 + s^8/9) in double (it is below 2^-18 of 2s for
// |s| < 0.0028; the terms dropped are below 2^-86 of 2s).  Error: the tail's rounding,
// under 2^-70 |2s|, and the double-double steps, under 2^-100 |log x|; E doubles both.
GH_HD double cr_log_fast(double x) {
  const uint64_t bits = dbits(x);
  int e = (int)((bits >> 52) & 0x7FF) - 1023;
  double m = bitsd((bits & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL);
  if (m > 1.4142135623730951) { m = mul_rn(m, 0.5); e += 1; }
  const double ci = rint_rn(mul_rn(m, 128.0));
  const int i = (int)ci;
  const double c = mul_rn(ci, 0.0078125);
  const double t = sub_rn(m, c);
  const dd s = dd_div(dd{t, 0.0}, two_sum(mul_rn(2.0, c), t));
  const double z = mul_rn(s.hi, s.hi);
  double q = fma_rn(z, 0.1111111111111111, 0.14285714285714285);    // 1/9, 1/7
  q = fma_rn(z, q, 0.2);
  q = fma_rn(z, q, 0.3333333333333333);
  const double tail = mul_rn(mul_rn(mul_rn(2.0, s.hi), z), q);
  const dd u = dd_add(dd{mul_rn(2.0, s.hi), mul_rn(2.0, s.lo)}, dd{tail, 0.0});
  const dd lm = dd_add(GH_TAB(logc, i - 90), u);
  const dd r = dd_add(dd_mul_d(dd{GH_LN2_HI, GH_LN2_LO}, (double)e), lm);
  const double E = add_rn(mul_rn(fabs(s.hi), 0x1p-67), mul_rn(fabs(r.hi), 0x1p-98));
  double y;
  return ziv_round(r, E, &y) ? y : cr_log(x);
}

// cos x, first phase: the reduction of cr_cos (r = x - k pi/32 in double-double), then
//   cos r = 1 - r^2/2 + z^2 (1/24 - z/720 + z^2/40320 - z^3/3628800),  z = r_hi^2,
//   sin r = r_hi + (r_lo + r_hi ts),  ts = -z/6 + z^2/120 - ... + z^5/39916800 (double),
// |r| <= pi/64: the leading r^2/2 in double-double, the rest in double.  Error: sin r
// under 2^-52.6 |r_hi| z (ts to 2^-50.4 relative, times |r_hi ts| <= |r_hi| z / 6, and the
// fma's rounding), cos r under 2^-54.5 z^2 (the double tail), the reduction, tables and
// double-double steps under 2^-100; E = 2^-52 |r_hi| z + 2^-54 z^2 + 2^-99, so that the
// bound shrinks with r where cos x is near zero.
GH_HD double cr_cos_fast(double x) {
  const double k = rint_rn(mul_rn(x, GH_32_OVER_PI));
  dd r = dd_add(dd{x, 0.0}, dd_neg(two_prod(k, GH_PI32_1)));
  r = dd_add(r, dd_neg(two_prod(k, GH_PI32_2)));
  r = dd_add(r, dd{-mul_rn(k, GH_PI32_3), 0.0});
  const int j = ((int)k) & 63;
  const dd zz = two_prod(r.hi, r.hi);
  const double z = zz.hi;
  double tc = fma_rn(z, -2.755731922398589e-07, 2.48015873015873e-05);   // -1/3628800, 1/40320
  tc = fma_rn(z, tc, -0.001388888888888889);                            // -1/720
  tc = fma_rn(z, tc, 0.041666666666666664);                             // 1/24
  tc = mul_rn(mul_rn(z, z), tc);
  const double zl = fma_rn(mul_rn(2.0, r.hi), r.lo, zz.lo);                   // r^2 = z + zl to 2^-106
  const dd cosr = dd_add(dd{1.0, 0.0}, dd_add(dd{mul_rn(-0.5, z), mul_rn(-0.5, zl)}, dd{tc, 0.0}));
  double ts = fma_rn(z, 2.505210838544172e-08, -2.7557319223985893e-06);  // 1/39916800, -1/362880
  ts = fma_rn(z, ts, 0.0001984126984126984);                               // 1/5040
  ts = fma_rn(z, ts, -0.008333333333333333);                              // -1/120
  ts = fma_rn(z, ts, 0.16666666666666666);                                // 1/6
  ts = mul_rn(-z, ts);
  const dd sinr = fast_two_sum(r.hi, fma_rn(r.hi, ts, r.lo));
  const dd res = dd_add(dd_mul(GH_TAB(cos, j), cosr), dd_neg(dd_mul(GH_TAB(sin, j), sinr)));
  double y;
  const double E = add_rn(add_rn(mul_rn(mul_rn(fabs(r.hi), z), 0x1p-52), mul_rn(mul_rn(z, z), 0x1p-54)), 0x1p-99);
  return ziv_round(res, E, &y) ? y : cr_cos(x);
}

// Standard normal draw keyed on k (src/core/rng.hpp:42-46 formula).
GH_HD double gauss(uint64_t seed, uint64_t k) {
  const double u1 = uniform(seed, splitmix64(k * 2 + 1));
  const double u2 = uniform(seed, splitmix64(k * 2 + 2));
  const double a = sqrt_rn(mul_rn(-2.0, cr_log_fast(u1)));
  const double c = cr_cos_fast(mul_rn(6.283185307179586, u2));       // (2 * pi) * u2, 2*pi exact
  return mul_rn(a, c);
}

#if defined(__CUDACC__)
// The same draw with the CUDA math library's FP64 log and cos (within 1-2 ulp of
// the correctly rounded value).  Used where the result is rounded to FP32 at once
// (momentum refresh of the FP32-MD mode): after that rounding it equals gauss()
// except with probability ~1e-8 per draw, at a fraction of the cost.
__device__ __forceinline__ double gauss_md(uint64_t seed, uint64_t k) {
  const double u1 = uniform(seed, splitmix64(k * 2 + 1));
  const double u2 = uniform(seed, splitmix64(k * 2 + 2));
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
#endif

}  // namespace ghrng
