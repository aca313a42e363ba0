/* gh_oracle.c -- CPU restatement of the reference MD path (TEST INFRASTRUCTURE ONLY).
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the hlammiv/gauge_higgs project root).  Arithmetic order follows the
 * reference so that, compiled with -ffp-contract=off, most quantities agree
 * with a contraction-free build of the reference to the last bit; the parity
 * gate itself is 1e-12 relative.
 *
 * Gaussian draws use the host libm (log, cos) exactly as src/core/rng.hpp:42-46
 * does, so this oracle inherits glibc's (not correctly rounded) libm.
 */
#include "gh_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cx;

static inline cx cmk(double r, double i) { cx z; z.re = r; z.im = i; return z; }
static inline cx cadd(cx a, cx b) { return cmk(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return cmk(a.re - b.re, a.im - b.im); }
static inline cx cmul(cx a, cx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx cconj(cx a) { return cmk(a.re, -a.im); }
static inline cx cscal(cx a, double s) { return cmk(a.re * s, a.im * s); }
static inline double cnorm(cx a) { return a.re * a.re + a.im * a.im; }
static inline int ciszero(cx a) { return a.re == 0.0 && a.im == 0.0; }

/* Smith's (1962) complex division a/b. */
static cx cdiv(cx a, cx b) {
  double r, den;
  if (fabs(b.re) >= fabs(b.im)) {
    r = b.im / b.re; den = b.re + b.im * r;
    return cmk((a.re + a.im * r) / den, (a.im - a.re * r) / den);
  }
  r = b.re / b.im; den = b.re * r + b.im;
  return cmk((a.re * r + a.im) / den, (a.im * r - a.re) / den);
}

#define CX(p, i) (((cx*)(p))[(i)])
#define NG(N) ((N) * (N) - 1)

/* ------------------------------------------------------------------------ */
/* Lattice: src/core/geometry.hpp:20-49 (mixed radix, direction 0 fastest).  */
/* ------------------------------------------------------------------------ */
void gho_lattice_init(gho_lattice* lat, int D, int N, const int* L) {
  lat->D = D; lat->N = N; lat->vol = 1;
  for (int mu = 0; mu < GHO_MAXD; ++mu) { lat->L[mu] = 1; lat->stride[mu] = 0; }
  for (int mu = 0; mu < D; ++mu) { lat->L[mu] = L[mu]; lat->stride[mu] = lat->vol; lat->vol *= L[mu]; }
}
static inline int gho_coord(const gho_lattice* lat, int64_t s, int mu) {
  return (int)((s / lat->stride[mu]) % lat->L[mu]);
}
int64_t gho_fwd(const gho_lattice* lat, int64_t s, int mu) {
  int x = gho_coord(lat, s, mu);
  return (x + 1 < lat->L[mu]) ? s + lat->stride[mu] : s - (int64_t)x * lat->stride[mu];
}
int64_t gho_bwd(const gho_lattice* lat, int64_t s, int mu) {
  int x = gho_coord(lat, s, mu);
  return (x > 0) ? s - lat->stride[mu] : s + (int64_t)(lat->L[mu] - 1) * lat->stride[mu];
}
static int64_t n_plaq(const gho_lattice* lat) {  /* geometry.hpp:52 */
  return lat->vol * ((int64_t)lat->D * (lat->D - 1) / 2);
}

/* ------------------------------------------------------------------------ */
/* RNG: src/core/rng.hpp:11-46                                                */
/* ------------------------------------------------------------------------ */
uint64_t gho_splitmix64(uint64_t x) {            /* rng.hpp:11-16 */
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
uint64_t gho_key(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e) {  /* rng.hpp:24-32 */
  const uint64_t g = 0x9E3779B97F4A7C15ULL;
  uint64_t h = gho_splitmix64(a);
  h = gho_splitmix64(h ^ (b + g));
  h = gho_splitmix64(h ^ (c + g));
  h = gho_splitmix64(h ^ (d + g));
  h = gho_splitmix64(h ^ (e + g));
  return h;
}
double gho_uniform(uint64_t seed, uint64_t k) {  /* rng.hpp:35-39 */
  uint64_t h = gho_splitmix64(seed ^ gho_splitmix64(k));
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
double gho_gauss(uint64_t seed, uint64_t k) {    /* rng.hpp:42-46 */
  const double kPi = 3.14159265358979323846264338327950288;
  const double u1 = gho_uniform(seed, gho_splitmix64(k * 2 + 1));
  const double u2 = gho_uniform(seed, gho_splitmix64(k * 2 + 2));
  return sqrt(-2.0 * log(u1)) * cos(2.0 * kPi * u2);
}

/* ------------------------------------------------------------------------ */
/* Small N x N complex matrices (src/core/linalg.hpp:16-96).                  */
/* ------------------------------------------------------------------------ */
static void mzero(int N, cx* A) { for (int i = 0; i < N * N; ++i) A[i] = cmk(0, 0); }
static void mident(int N, cx* A) { mzero(N, A); for (int i = 0; i < N; ++i) A[i * N + i] = cmk(1, 0); }
/* C = A*B, loop order and zero skip of linalg.hpp:66-75 */
static void mmul(int N, const cx* A, const cx* B, cx* C) {
  cx T[GHO_MAXN * GHO_MAXN];
  mzero(N, T);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < N; ++k) {
      const cx aik = A[i * N + k];
      if (ciszero(aik)) continue;
      for (int j = 0; j < N; ++j) T[i * N + j] = cadd(T[i * N + j], cmul(aik, B[k * N + j]));
    }
  memcpy(C, T, sizeof(cx) * N * N);
}
static void mdag(int N, const cx* A, cx* R) {
  cx T[GHO_MAXN * GHO_MAXN];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) T[i * N + j] = cconj(A[j * N + i]);
  memcpy(R, T, sizeof(cx) * N * N);
}
static cx mtrace(int N, const cx* A) {
  cx t = cmk(0, 0);
  for (int i = 0; i < N; ++i) t = cadd(t, A[i * N + i]);
  return t;
}
static cx trprod(int N, const cx* A, const cx* B) {       /* linalg.hpp:90-96 */
  cx s = cmk(0, 0);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < N; ++k) s = cadd(s, cmul(A[i * N + k], B[k * N + i]));
  return s;
}
static double fnorm(int N, const cx* A) {
  double s = 0.0;
  for (int i = 0; i < N * N; ++i) s += cnorm(A[i]);
  return sqrt(s);
}
static cx mdet(int N, const cx* M) {                       /* linalg.hpp:98-125 */
  cx m[GHO_MAXN * GHO_MAXN];
  memcpy(m, M, sizeof(cx) * N * N);
  cx d = cmk(1, 0);
  for (int col = 0; col < N; ++col) {
    int piv = col;
    double best = hypot(m[col * N + col].re, m[col * N + col].im);
    for (int r = col + 1; r < N; ++r) {
      double v = hypot(m[r * N + col].re, m[r * N + col].im);
      if (v > best) { best = v; piv = r; }
    }
    if (best == 0.0) return cmk(0, 0);
    if (piv != col) {
      for (int j = 0; j < N; ++j) { cx t = m[piv * N + j]; m[piv * N + j] = m[col * N + j]; m[col * N + j] = t; }
      d = cmk(-d.re, -d.im);
    }
    d = cmul(d, m[col * N + col]);
    const cx inv = cdiv(cmk(1, 0), m[col * N + col]);
    for (int r = col + 1; r < N; ++r) {
      const cx f = cmul(m[r * N + col], inv);
      if (ciszero(f)) continue;
      for (int j = col; j < N; ++j) m[r * N + j] = csub(m[r * N + j], cmul(f, m[col * N + j]));
    }
  }
  return d;
}

/* ------------------------------------------------------------------------ */
/* su(N): src/group/algebra.hpp:23-120                                        */
/* ------------------------------------------------------------------------ */
void gho_generators(int N, double* Tout) {                 /* algebra.hpp:23-49 */
  cx* T = (cx*)Tout;
  const int ng = NG(N);
  for (int i = 0; i < ng * N * N; ++i) T[i] = cmk(0, 0);
  int a = 0;
  for (int j = 0; j < N; ++j)
    for (int k = j + 1; k < N; ++k, ++a) {
      T[a * N * N + j * N + k] = cadd(T[a * N * N + j * N + k], cmk(0.5, 0));
      T[a * N * N + k * N + j] = cadd(T[a * N * N + k * N + j], cmk(0.5, 0));
    }
  for (int j = 0; j < N; ++j)
    for (int k = j + 1; k < N; ++k, ++a) {
      T[a * N * N + j * N + k] = cadd(T[a * N * N + j * N + k], cmk(0, -0.5));
      T[a * N * N + k * N + j] = cadd(T[a * N * N + k * N + j], cmk(0, 0.5));
    }
  for (int l = 1; l <= N - 1; ++l, ++a) {
    const double c = sqrt(2.0 / ((double)l * (l + 1)));
    for (int j = 0; j < l; ++j) T[a * N * N + j * N + j] = cadd(T[a * N * N + j * N + j], cmk(0.5 * c, 0));
    T[a * N * N + l * N + l] = cadd(T[a * N * N + l * N + l], cmk(-0.5 * c * l, 0));
  }
}

static const cx* gens(int N) {  /* cached generator tables for N = 2..4 */
  static cx tab[GHO_MAXN + 1][NG(GHO_MAXN) * GHO_MAXN * GHO_MAXN];
  static int built[GHO_MAXN + 1];
  if (!built[N]) { gho_generators(N, (double*)tab[N]); built[N] = 1; }
  return tab[N];
}

void gho_structure_constants(int N, double* f) {           /* algebra.hpp:102-120 */
  const cx* T = gens(N);
  const int n = NG(N), NN = N * N;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      cx ab[GHO_MAXN * GHO_MAXN], ba[GHO_MAXN * GHO_MAXN], comm[GHO_MAXN * GHO_MAXN];
      mmul(N, T + a * NN, T + b * NN, ab);
      mmul(N, T + b * NN, T + a * NN, ba);
      for (int i = 0; i < NN; ++i) comm[i] = csub(ab[i], ba[i]);
      for (int c = 0; c < n; ++c) f[((size_t)a * n + b) * n + c] = 2.0 * trprod(N, comm, T + c * NN).im;
    }
}

void gho_alg_to_mat(int N, const double* v, double* Mout) {  /* algebra.hpp:59-71 */
  const cx* T = gens(N);
  cx M[GHO_MAXN * GHO_MAXN];
  mzero(N, M);
  for (int a = 0; a < NG(N); ++a) {
    const double va = v[a];
    if (va == 0.0) continue;
    for (int i = 0; i < N * N; ++i) M[i] = cadd(M[i], cscal(T[a * N * N + i], va));
  }
  memcpy(Mout, M, sizeof(cx) * N * N);
}

/* exp(iH): src/group/sun.hpp:11-29 (general N), :33-45 (SU(2) closed form). */
void gho_expi(int N, const double* Hin, double* Uout) {
  const cx* H = (const cx*)Hin;
  cx* U = (cx*)Uout;
  if (N == 2) {
    const double r2 = 0.5 * trprod(2, H, H).re;
    const double r = sqrt(r2 > 0.0 ? r2 : 0.0);
    double c, sinc;
    if (r < 1e-8) { c = 1.0 - 0.5 * r2; sinc = 1.0 - r2 / 6.0; }
    else { c = cos(r); sinc = sin(r) / r; }
    cx R[4];
    mident(2, R);
    for (int i = 0; i < 4; ++i) R[i] = cmul(R[i], cmk(c, 0));
    for (int i = 0; i < 4; ++i) R[i] = cadd(R[i], cmul(H[i], cmk(0, sinc)));
    memcpy(U, R, sizeof(R));
    return;
  }
  const double nrm = fnorm(N, H);
  int s = 0;
  double scaled = nrm;
  while (scaled > 0.5) { scaled *= 0.5; ++s; }
  const double inv2s = pow(0.5, s);
  cx A[GHO_MAXN * GHO_MAXN], term[GHO_MAXN * GHO_MAXN], res[GHO_MAXN * GHO_MAXN];
  for (int i = 0; i < N * N; ++i) A[i] = cmul(H[i], cmk(0, inv2s));
  mident(N, term); mident(N, res);
  for (int k = 1; k <= 18; ++k) {
    mmul(N, term, A, term);
    for (int i = 0; i < N * N; ++i) term[i] = cmul(term[i], cmk(1.0 / k, 0));
    for (int i = 0; i < N * N; ++i) res[i] = cadd(res[i], term[i]);
  }
  for (int i = 0; i < s; ++i) mmul(N, res, res, res);
  memcpy(U, res, sizeof(cx) * N * N);
}

/* Modified Gram-Schmidt on rows + det phase: src/group/sun.hpp:48-71. */
void gho_reunitarize(int N, double* Uio) {
  cx* U = (cx*)Uio;
  for (int i = 0; i < N; ++i) {
    for (int k = 0; k < i; ++k) {
      cx proj = cmk(0, 0);
      for (int j = 0; j < N; ++j) proj = cadd(proj, cmul(cconj(U[k * N + j]), U[i * N + j]));
      for (int j = 0; j < N; ++j) U[i * N + j] = csub(U[i * N + j], cmul(proj, U[k * N + j]));
    }
    double nrm = 0.0;
    for (int j = 0; j < N; ++j) nrm += cnorm(U[i * N + j]);
    nrm = sqrt(nrm);
    const cx inv = cmk(1.0 / nrm, 0);
    for (int j = 0; j < N; ++j) U[i * N + j] = cmul(U[i * N + j], inv);
  }
  const cx d = mdet(N, U);
  const double ad = hypot(d.re, d.im);
  if (ad > 0.0) {
    const cx phase = cmk(d.re / ad, d.im / ad);
    const cx inv = cconj(phase);
    for (int j = 0; j < N; ++j) U[j] = cmul(U[j], inv);
  }
}

/* ------------------------------------------------------------------------ */
/* Representations: src/rep/representation.hpp, rep_fundamental.hpp,         */
/* rep_adjoint.hpp, rep_general.hpp                                            */
/* ------------------------------------------------------------------------ */
int gho_rep_init(gho_rep* r, int kind, int N, int d, int real, int n, long dimT,
                 const double* T, const double* W) {
  memset(r, 0, sizeof(*r));
  r->kind = kind; r->N = N;
  const int ng = NG(N);
  if (kind == GHO_REP_FUND) {                              /* rep_fundamental.hpp:15-25 */
    r->d = N; r->real = 0;
    r->T = (double*)malloc(sizeof(cx) * ng * N * N);
    memcpy(r->T, gens(N), sizeof(cx) * ng * N * N);
  } else if (kind == GHO_REP_ADJ) {                        /* rep_adjoint.hpp:10-25 */
    r->d = ng; r->real = 1;
    double* f = (double*)malloc(sizeof(double) * ng * ng * ng);
    gho_structure_constants(N, f);
    r->T = (double*)malloc(sizeof(cx) * ng * ng * ng);
    cx* Tc = (cx*)r->T;
    for (int a = 0; a < ng; ++a)
      for (int b = 0; b < ng; ++b)
        for (int c = 0; c < ng; ++c) Tc[(a * ng + b) * ng + c] = cmk(0.0, -f[((size_t)a * ng + b) * ng + c]);
    free(f);
  } else if (kind == GHO_REP_GENERAL) {                    /* rep_general.hpp:54-84 */
    r->d = d; r->real = real; r->n = n; r->dimT = dimT;
    r->T = (double*)malloc(sizeof(cx) * ng * d * d);
    memcpy(r->T, T, sizeof(cx) * ng * d * d);
    r->W = (double*)malloc(sizeof(cx) * d * dimT);
    memcpy(r->W, W, sizeof(cx) * d * dimT);
  } else {
    r->kind = GHO_REP_NONE; r->d = 0;
  }
  return 0;
}
void gho_rep_free(gho_rep* r) { free(r->T); free(r->W); r->T = r->W = 0; }

/* D_ab = 2 Re Tr(T^a U T^b U^dag): rep_adjoint.hpp:27-40 */
static void adj_matrix(int N, const cx* U, cx* Dm) {
  const cx* T = gens(N);
  const int n = NG(N), NN = N * N;
  cx Ud[GHO_MAXN * GHO_MAXN];
  mdag(N, U, Ud);
  for (int a = 0; a < n; ++a) {
    cx TaU[GHO_MAXN * GHO_MAXN];
    mmul(N, T + a * NN, U, TaU);
    for (int b = 0; b < n; ++b) {
      cx t1[GHO_MAXN * GHO_MAXN], t2[GHO_MAXN * GHO_MAXN];
      mmul(N, TaU, T + b * NN, t1);
      mmul(N, t1, Ud, t2);
      Dm[a * n + b] = cmk(2.0 * mtrace(N, t2).re, 0.0);
    }
  }
}

/* V^{xn} slot apply: rep_general.hpp:184-194 */
static void onebody(const gho_rep* r, const cx* M, const cx* src, cx* dst, int s, const long* powN) {
  const int N = r->N;
  for (long i = 0; i < r->dimT; ++i) dst[i] = cmk(0, 0);
  const long blk = powN[r->n - 1 - s];
  for (long idx = 0; idx < r->dimT; ++idx) {
    const cx c = src[idx];
    if (ciszero(c)) continue;
    const int digit = (int)((idx / blk) % N);
    const long base = idx - (long)digit * blk;
    for (int j = 0; j < N; ++j) dst[base + (long)j * blk] = cadd(dst[base + (long)j * blk], cmul(M[j * N + digit], c));
  }
}

/* matrix-free lift / slot applies / project: rep_general.hpp:196-220 */
static void apply_tensor(const gho_rep* r, const cx* U, const cx* phi, cx* out, int dag) {
  const int N = r->N, d = r->d;
  const long dimT = r->dimT;
  long powN[32];
  powN[0] = 1;
  for (int k = 1; k <= r->n; ++k) powN[k] = powN[k - 1] * N;
  cx* sa = (cx*)malloc(sizeof(cx) * dimT);
  cx* sb = (cx*)malloc(sizeof(cx) * dimT);
  const cx* W = (const cx*)r->W;
  for (long i = 0; i < dimT; ++i) sa[i] = cmk(0, 0);
  for (int l = 0; l < d; ++l) {
    const cx c = phi[l];
    if (ciszero(c)) continue;
    for (long i = 0; i < dimT; ++i) sa[i] = cadd(sa[i], cmul(c, W[(size_t)l * dimT + i]));
  }
  cx M[GHO_MAXN * GHO_MAXN];
  if (dag) mdag(N, U, M); else memcpy(M, U, sizeof(cx) * N * N);
  cx* cur = sa; cx* oth = sb;
  for (int s = 0; s < r->n; ++s) { onebody(r, M, cur, oth, s, powN); cx* t = cur; cur = oth; oth = t; }
  for (int k = 0; k < d; ++k) {
    cx acc = cmk(0, 0);
    for (long i = 0; i < dimT; ++i) acc = cadd(acc, cmul(cconj(W[(size_t)k * dimT + i]), cur[i]));
    out[k] = acc;
  }
  free(sa); free(sb);
}

void gho_rep_matrix(const gho_rep* r, const double* Uin, double* Dout) {
  const cx* U = (const cx*)Uin;
  cx* Dm = (cx*)Dout;
  const int N = r->N, d = r->d;
  if (r->kind == GHO_REP_FUND) { memcpy(Dm, U, sizeof(cx) * N * N); return; }
  if (r->kind == GHO_REP_ADJ) { adj_matrix(N, U, Dm); return; }
  /* tensor materialisation <W_k|U^{xn}|W_l>: rep_general.hpp:122-131 */
  cx* e = (cx*)malloc(sizeof(cx) * d);
  cx* col = (cx*)malloc(sizeof(cx) * d);
  for (int l = 0; l < d; ++l) {
    for (int k = 0; k < d; ++k) e[k] = cmk(k == l ? 1.0 : 0.0, 0.0);
    apply_tensor(r, U, e, col, 0);
    for (int k = 0; k < d; ++k) Dm[k * d + l] = col[k];
  }
  free(e); free(col);
}

/* y = M x (DMat*DVec, linalg.hpp:302-307) */
static void dmatvec(int d, const cx* M, const cx* x, cx* y, int dag) {
  for (int i = 0; i < d; ++i) {
    cx acc = cmk(0, 0);
    for (int j = 0; j < d; ++j) acc = cadd(acc, cmul(dag ? cconj(M[j * d + i]) : M[i * d + j], x[j]));
    y[i] = acc;
  }
}

/* rotate / rotate_dag: representation.hpp:28-32 (default, also the *_cached
 * variants :68-75 used by kick for link-cacheable reps) and rep_general.hpp:137-150. */
void gho_rep_rotate(const gho_rep* r, const double* Uin, const double* phiin, double* outp, int dag) {
  const cx* U = (const cx*)Uin;
  const cx* phi = (const cx*)phiin;
  cx* out = (cx*)outp;
  if (r->kind == GHO_REP_GENERAL) { apply_tensor(r, U, phi, out, dag); return; }
  cx Dm[(NG(GHO_MAXN)) * (NG(GHO_MAXN))];
  gho_rep_matrix(r, Uin, (double*)Dm);
  dmatvec(r->d, Dm, phi, out, dag);
}

/* hop_link_g: g^a = -2 Im(phi_x^dag T^a_R D(U) phi_y): representation.hpp:36-46,
 * rep_general.hpp:151-159. */
void gho_rep_hop_link_g(const gho_rep* r, const double* Uin, const double* phixin,
                        const double* phiyin, double* g) {
  const int d = r->d, ng = NG(r->N);
  const cx* phix = (const cx*)phixin;
  const cx* T = (const cx*)r->T;
  cx* Dy = (cx*)malloc(sizeof(cx) * d);
  cx* t = (cx*)malloc(sizeof(cx) * d);
  gho_rep_rotate(r, Uin, phiyin, (double*)Dy, 0);
  for (int a = 0; a < ng; ++a) {
    dmatvec(d, T + (size_t)a * d * d, Dy, t, 0);
    cx z = cmk(0, 0);
    for (int i = 0; i < d; ++i) z = cadd(z, cmul(cconj(phix[i]), t[i]));
    g[a] = -2.0 * z.im;
  }
  free(Dy); free(t);
}

/* ------------------------------------------------------------------------ */
/* Field initialisation                                                       */
/* ------------------------------------------------------------------------ */
/* GaugeField::hot: src/core/fields.hpp:25-34 */
void gho_hot_start(const gho_lattice* lat, uint64_t seed, double sigma, double* U) {
  const int D = lat->D, N = lat->N, NN = N * N;
  for (int64_t s = 0; s < lat->vol; ++s)
    for (int mu = 0; mu < D; ++mu) {
      double v[NG(GHO_MAXN)];
      cx H[GHO_MAXN * GHO_MAXN];
      for (int a = 0; a < NG(N); ++a) v[a] = sigma * gho_gauss(seed, gho_key(1, (uint64_t)s, (uint64_t)mu, (uint64_t)a, 0));
      gho_alg_to_mat(N, v, (double*)H);
      gho_expi(N, (double*)H, U + 2 * (size_t)(s * D + mu) * NN);
    }
}
void gho_cold_start(const gho_lattice* lat, double* U) {   /* fields.hpp:23 */
  const int N = lat->N;
  for (int64_t l = 0; l < lat->vol * lat->D; ++l) mident(N, (cx*)U + l * N * N);
}
/* CVecField::gaussian: src/core/scalar_field.hpp:40-50 */
void gho_phi_gaussian(const gho_lattice* lat, int d, uint64_t seed, uint64_t stream,
                      int real, double sigma, double* phi) {
  for (int64_t s = 0; s < lat->vol; ++s)
    for (int k = 0; k < d; ++k) {
      const double re = sigma * gho_gauss(seed, gho_key(stream, (uint64_t)s, (uint64_t)(2 * k), 0, 0));
      const double im = real ? 0.0 : sigma * gho_gauss(seed, gho_key(stream, (uint64_t)s, (uint64_t)(2 * k + 1), 0, 0));
      CX(phi, s * d + k) = cmk(re, im);
    }
}
/* LinkMom::refresh: src/core/fields.hpp:59-66 */
void gho_mom_refresh(const gho_lattice* lat, uint64_t seed, uint64_t stream, double* P) {
  const int D = lat->D, ng = NG(lat->N);
  for (int64_t s = 0; s < lat->vol; ++s)
    for (int mu = 0; mu < D; ++mu)
      for (int a = 0; a < ng; ++a)
        P[(s * D + mu) * ng + a] = gho_gauss(seed, gho_key(stream, (uint64_t)s, (uint64_t)mu, (uint64_t)a, 0));
}

/* ------------------------------------------------------------------------ */
/* Gauge action and force: src/action/gauge_wilson.hpp                        */
/* ------------------------------------------------------------------------ */
#define LINK(U, s, mu) ((const cx*)(U) + ((size_t)(s) * D + (mu)) * NN)

static double sum_retr_plaq(const gho_lattice* lat, const double* U) {  /* gauge_wilson.hpp:31-47 */
  const int D = lat->D, N = lat->N, NN = N * N;
  double sum = 0.0;
  for (int64_t s = 0; s < lat->vol; ++s)
    for (int mu = 0; mu < D; ++mu) {
      const int64_t spmu = gho_fwd(lat, s, mu);
      for (int nu = mu + 1; nu < D; ++nu) {
        const int64_t spnu = gho_fwd(lat, s, nu);
        cx A[GHO_MAXN * GHO_MAXN], B[GHO_MAXN * GHO_MAXN];
        mmul(N, LINK(U, s, mu), LINK(U, spmu, nu), A);
        mdag(N, LINK(U, spnu, mu), B); mmul(N, A, B, A);
        mdag(N, LINK(U, s, nu), B);    mmul(N, A, B, A);
        sum += mtrace(N, A).re;
      }
    }
  return sum;
}
double gho_gauge_action(const gho_lattice* lat, const double* U, double beta) {
  const int N = lat->N;
  return (beta / N) * ((double)N * n_plaq(lat) - sum_retr_plaq(lat, U));
}
double gho_avg_plaquette(const gho_lattice* lat, const double* U) {  /* gauge_wilson.hpp:50-65 */
  return sum_retr_plaq(lat, U) / ((double)lat->N * n_plaq(lat));
}

/* staple: gauge_wilson.hpp:11-27 */
static void staple(const gho_lattice* lat, const double* U, int64_t s, int mu, cx* sig) {
  const int D = lat->D, N = lat->N, NN = N * N;
  mzero(N, sig);
  const int64_t spmu = gho_fwd(lat, s, mu);
  for (int nu = 0; nu < D; ++nu) {
    if (nu == mu) continue;
    const int64_t spnu = gho_fwd(lat, s, nu), smnu = gho_bwd(lat, s, nu);
    const int64_t spmu_mnu = gho_bwd(lat, spmu, nu);
    cx A[GHO_MAXN * GHO_MAXN], B[GHO_MAXN * GHO_MAXN];
    mdag(N, LINK(U, spnu, mu), B); mmul(N, LINK(U, spmu, nu), B, A);
    mdag(N, LINK(U, s, nu), B);    mmul(N, A, B, A);
    for (int i = 0; i < NN; ++i) sig[i] = cadd(sig[i], A[i]);
    mdag(N, LINK(U, spmu_mnu, nu), A);
    mdag(N, LINK(U, smnu, mu), B); mmul(N, A, B, A);
    mmul(N, A, LINK(U, smnu, nu), A);
    for (int i = 0; i < NN; ++i) sig[i] = cadd(sig[i], A[i]);
  }
}
/* F^a += (beta/N) Im Tr(T^a U Sigma): gauge_wilson.hpp:70-83 */
void gho_add_gauge_force(const gho_lattice* lat, const double* U, double beta, double* F) {
  const int D = lat->D, N = lat->N, NN = N * N, ng = NG(N);
  const cx* T = gens(N);
  const double c = beta / N;
  for (int64_t s = 0; s < lat->vol; ++s)
    for (int mu = 0; mu < D; ++mu) {
      cx sig[GHO_MAXN * GHO_MAXN], Om[GHO_MAXN * GHO_MAXN];
      staple(lat, U, s, mu, sig);
      mmul(N, LINK(U, s, mu), sig, Om);
      double* Fa = F + (s * D + mu) * ng;
      for (int a = 0; a < ng; ++a) Fa[a] += c * trprod(N, T + a * NN, Om).im;
    }
}

/* ------------------------------------------------------------------------ */
/* Scalar sector: src/action/scalar_higgs.hpp                                 */
/* ------------------------------------------------------------------------ */
static double vnorm2(int d, const cx* v) { double s = 0; for (int k = 0; k < d; ++k) s += cnorm(v[k]); return s; }
static cx vdot(int d, const cx* x, const cx* y) {
  cx s = cmk(0, 0);
  for (int i = 0; i < d; ++i) s = cadd(s, cmul(cconj(x[i]), y[i]));
  return s;
}

/* scalar_higgs.hpp:43-65 with QuarticPotential::value :30-33 */
/* Onsite potential: the quartic phi^dag phi + lambda (phi^dag phi - 1)^2
 * (QuarticPotential, src/action/scalar_higgs.hpp:25-40) or the multi-invariant
 * -mu2 phi^dag phi + sum_c f_c Tr(M^dag P_c M) given by its combined channel
 * superoperator A = sum_c 2 f_c P_c (src/action/scalar_invariants.hpp:60-148):
 * y = A vec(M), vec(M)[i*d+j] = phi_i conj(phi_j);  V = -mu2 n2 + Re <vec M, y> / 2;
 * dV/dphibar = -mu2 phi + mat(y) phi. */
typedef struct { int multi; double lambda; const double* A; double mu2; } gho_pot;

static void multi_y(int d, const double* A, const cx* px, cx* y) {
  const int dd = d * d;
  for (int r = 0; r < dd; ++r) {
    cx acc = cmk(0.0, 0.0);
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j) {
        const cx a = cmk(A[2 * ((size_t)r * dd + i * d + j)], A[2 * ((size_t)r * dd + i * d + j) + 1]);
        acc = cadd(acc, cmul(a, cmul(px[i], cconj(px[j]))));
      }
    y[r] = acc;
  }
}

static double pot_value(const gho_pot* p, int d, const cx* px) {
  const double n2 = vnorm2(d, px);
  if (!p->multi) return n2 + p->lambda * (n2 - 1.0) * (n2 - 1.0);
  cx* y = (cx*)malloc(sizeof(cx) * d * d);
  multi_y(d, p->A, px, y);
  double re = 0.0;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) re += cmul(cconj(cmul(px[i], cconj(px[j]))), y[i * d + j]).re;
  free(y);
  return -p->mu2 * n2 + 0.5 * re;
}

static void pot_dV(const gho_pot* p, int d, const cx* px, cx* g) {
  if (!p->multi) {
    const double c = 1.0 + 2.0 * p->lambda * (vnorm2(d, px) - 1.0);
    for (int k = 0; k < d; ++k) g[k] = cmul(cmk(c, 0), px[k]);
    return;
  }
  cx* y = (cx*)malloc(sizeof(cx) * d * d);
  multi_y(d, p->A, px, y);
  for (int k = 0; k < d; ++k) {
    cx acc = cscal(px[k], -p->mu2);
    for (int q = 0; q < d; ++q) acc = cadd(acc, cmul(y[k * d + q], px[q]));
    g[k] = acc;
  }
  free(y);
}

void gho_multi_potential(int d, const double* A, double mu2, const double* phi, double* value, double* dV) {
  const gho_pot p = {1, 0.0, A, mu2};
  if (value) *value = pot_value(&p, d, (const cx*)phi);
  if (dV) pot_dV(&p, d, (const cx*)phi, (cx*)dV);
}

/* scalar_higgs.hpp:43-65 */
static double scalar_action_pot(const gho_lattice* lat, const gho_rep* r, const double* U,
                                const double* phi, double kappa, const gho_pot* pot) {
  const int D = lat->D, N = lat->N, NN = N * N, d = r->d;
  cx* Dpy = (cx*)malloc(sizeof(cx) * d);
  double S = 0.0;
  for (int64_t s = 0; s < lat->vol; ++s) {
    const cx* px = (const cx*)phi + s * d;
    S += pot_value(pot, d, px);
    for (int mu = 0; mu < D; ++mu) {
      const cx* py = (const cx*)phi + gho_fwd(lat, s, mu) * d;
      gho_rep_rotate(r, (const double*)LINK(U, s, mu), (const double*)py, (double*)Dpy, 0);
      S -= 2.0 * kappa * vdot(d, px, Dpy).re;
    }
  }
  free(Dpy);
  (void)NN;
  return S;
}

/* scalar_higgs.hpp:71-108 */
static void scalar_force_pot(const gho_lattice* lat, const gho_rep* r, const double* U,
                             const double* phi, double kappa, const gho_pot* pot, double* Fphi) {
  const int D = lat->D, N = lat->N, NN = N * N, d = r->d;
  cx* Dpf = (cx*)malloc(sizeof(cx) * d);
  cx* Dpb = (cx*)malloc(sizeof(cx) * d);
  cx* F = (cx*)malloc(sizeof(cx) * d);
  cx* g = (cx*)malloc(sizeof(cx) * d);
  for (int64_t s = 0; s < lat->vol; ++s) {
    const cx* px = (const cx*)phi + s * d;
    pot_dV(pot, d, px, g);
    for (int k = 0; k < d; ++k) F[k] = cscal(g[k], -2.0);
    for (int mu = 0; mu < D; ++mu) {
      const int64_t yf = gho_fwd(lat, s, mu), yb = gho_bwd(lat, s, mu);
      gho_rep_rotate(r, (const double*)LINK(U, s, mu), (const double*)((const cx*)phi + yf * d), (double*)Dpf, 0);
      gho_rep_rotate(r, (const double*)LINK(U, yb, mu), (const double*)((const cx*)phi + yb * d), (double*)Dpb, 1);
      for (int k = 0; k < d; ++k) F[k] = cadd(F[k], cscal(cadd(Dpf[k], Dpb[k]), 2.0 * kappa));
    }
    memcpy((cx*)Fphi + s * d, F, sizeof(cx) * d);
  }
  free(Dpf); free(Dpb); free(F); free(g);
  (void)NN;
}

double gho_scalar_action(const gho_lattice* lat, const gho_rep* r, const double* U,
                         const double* phi, double kappa, double lambda) {
  const gho_pot p = {0, lambda, NULL, 0.0};
  return scalar_action_pot(lat, r, U, phi, kappa, &p);
}
void gho_scalar_force(const gho_lattice* lat, const gho_rep* r, const double* U,
                      const double* phi, double kappa, double lambda, double* Fphi) {
  const gho_pot p = {0, lambda, NULL, 0.0};
  scalar_force_pot(lat, r, U, phi, kappa, &p, Fphi);
}
double gho_scalar_action_multi(const gho_lattice* lat, const gho_rep* r, const double* U,
                               const double* phi, double kappa, const double* A, double mu2) {
  const gho_pot p = {1, 0.0, A, mu2};
  return scalar_action_pot(lat, r, U, phi, kappa, &p);
}
void gho_scalar_force_multi(const gho_lattice* lat, const gho_rep* r, const double* U,
                            const double* phi, double kappa, const double* A, double mu2, double* Fphi) {
  const gho_pot p = {1, 0.0, A, mu2};
  scalar_force_pot(lat, r, U, phi, kappa, &p, Fphi);
}

/* scalar_higgs.hpp:113-128 */
void gho_add_matter_link_force(const gho_lattice* lat, const gho_rep* r, const double* U,
                               const double* phi, double kappa, double* F) {
  const int D = lat->D, N = lat->N, NN = N * N, d = r->d, ng = NG(N);
  double g[NG(GHO_MAXN)];
  for (int64_t s = 0; s < lat->vol; ++s)
    for (int mu = 0; mu < D; ++mu) {
      const int64_t y = gho_fwd(lat, s, mu);
      gho_rep_hop_link_g(r, (const double*)LINK(U, s, mu), (const double*)((const cx*)phi + s * d),
                         (const double*)((const cx*)phi + y * d), g);
      double* Fa = F + (s * D + mu) * ng;
      for (int a = 0; a < ng; ++a) Fa[a] += -kappa * g[a];
    }
}

/* scalar_higgs.hpp:132-144 */
double gho_link_energy(const gho_lattice* lat, const gho_rep* r, const double* U, const double* phi) {
  const int D = lat->D, N = lat->N, NN = N * N, d = r->d;
  cx* Dpy = (cx*)malloc(sizeof(cx) * d);
  double sum = 0.0;
  for (int64_t x = 0; x < lat->vol; ++x)
    for (int mu = 0; mu < D; ++mu) {
      gho_rep_rotate(r, (const double*)LINK(U, x, mu), (const double*)((const cx*)phi + gho_fwd(lat, x, mu) * d),
                     (double*)Dpy, 0);
      sum += vdot(d, (const cx*)phi + x * d, Dpy).re;
    }
  free(Dpy);
  return sum / ((double)lat->vol * D);
}
/* scalar_higgs.hpp:147-154 */
double gho_higgs_length(const gho_lattice* lat, int d, const double* phi) {
  double s = 0.0;
  for (int64_t x = 0; x < lat->vol; ++x) s += vnorm2(d, (const cx*)phi + x * d);
  return s / (double)lat->vol;
}
/* src/measure/observables.hpp:17-34 */
double gho_polyakov(const gho_lattice* lat, const double* U, int tdir) {
  const int D = lat->D, N = lat->N, NN = N * N;
  const int Lt = lat->L[tdir];
  double sum = 0.0;
  int64_t count = 0;
  for (int64_t s = 0; s < lat->vol; ++s) {
    if (gho_coord(lat, s, tdir) != 0) continue;
    cx P[GHO_MAXN * GHO_MAXN];
    memcpy(P, LINK(U, s, tdir), sizeof(cx) * NN);
    int64_t cur = gho_fwd(lat, s, tdir);
    for (int t = 1; t < Lt; ++t) { mmul(N, P, LINK(U, cur, tdir), P); cur = gho_fwd(lat, cur, tdir); }
    sum += mtrace(N, P).re;
    ++count;
  }
  return sum / ((double)count * N);
}
/* LinkMom::kinetic fields.hpp:69-74; CVecField::kinetic scalar_field.hpp:53-57 */
double gho_kinetic_mom(const gho_lattice* lat, const double* P) {
  const int64_t n = lat->vol * lat->D * NG(lat->N);
  double e = 0.0;
  for (int64_t i = 0; i < n; ++i) e += P[i] * P[i];
  return 0.5 * e;
}
double gho_kinetic_vec(const gho_lattice* lat, int d, const double* pi) {
  double e = 0.0;
  for (int64_t i = 0; i < lat->vol * d; ++i) e += cnorm(CX(pi, i));
  return 0.5 * e;
}

/* ------------------------------------------------------------------------ */
/* HMC: src/hmc/gauge_higgs_hmc.hpp:15-195 and src/hmc/hmc.hpp:12-96          */
/* ------------------------------------------------------------------------ */
static int has_scalar(const gho_hmc* h) { return h->rep && h->rep->kind != GHO_REP_NONE; }

int gho_hmc_init(gho_hmc* h, int D, int N, const int* L, const gho_rep* r, uint64_t seed) {
  memset(h, 0, sizeof(*h));
  gho_lattice_init(&h->lat, D, N, L);
  h->rep = r; h->seed = seed;
  h->beta = 2.3; h->kappa = 0.1; h->lambda = 0.5; h->tau = 1.0;
  h->nmd = 20; h->integ = GHO_OMELYAN; h->reunit_each_traj = 1;
  const int64_t V = h->lat.vol;
  h->U = (double*)calloc((size_t)V * D * N * N * 2, sizeof(double));
  h->P = (double*)calloc((size_t)V * D * NG(N), sizeof(double));
  const int d = (r && r->kind != GHO_REP_NONE) ? r->d : 1;
  h->phi = (double*)calloc((size_t)V * d * 2, sizeof(double));
  h->pi = (double*)calloc((size_t)V * d * 2, sizeof(double));
  return 0;
}
void gho_hmc_free(gho_hmc* h) { free(h->U); free(h->P); free(h->phi); free(h->pi); }

double gho_hmc_hamiltonian(const gho_hmc* h) {           /* gauge_higgs_hmc.hpp:105-110, hmc.hpp:29 */
  if (!has_scalar(h)) return gho_kinetic_mom(&h->lat, h->P) + gho_gauge_action(&h->lat, h->U, h->beta);
  return gho_kinetic_mom(&h->lat, h->P) + gho_kinetic_vec(&h->lat, h->rep->d, h->pi)
       + gho_gauge_action(&h->lat, h->U, h->beta)
       + gho_scalar_action(&h->lat, h->rep, h->U, h->phi, h->kappa, h->lambda);
}

void gho_hmc_kick(gho_hmc* h, double eps) {              /* gauge_higgs_hmc.hpp:112-134, hmc.hpp:35-41 */
  const gho_lattice* lat = &h->lat;
  const int64_t nl = lat->vol * lat->D;
  const int ng = NG(lat->N);
  double* F = (double*)calloc((size_t)nl * ng, sizeof(double));
  gho_add_gauge_force(lat, h->U, h->beta, F);
  if (has_scalar(h)) gho_add_matter_link_force(lat, h->rep, h->U, h->phi, h->kappa, F);
  for (int64_t i = 0; i < nl * ng; ++i) h->P[i] -= eps * F[i];
  free(F);
  if (has_scalar(h)) {
    const int d = h->rep->d;
    double* Fp = (double*)malloc(sizeof(double) * 2 * lat->vol * d);
    gho_scalar_force(lat, h->rep, h->U, h->phi, h->kappa, h->lambda, Fp);
    for (int64_t i = 0; i < lat->vol * d; ++i) CX(h->pi, i) = cadd(CX(h->pi, i), cscal(CX(Fp, i), eps));
    free(Fp);
  }
}

void gho_hmc_drift(gho_hmc* h, double eps) {             /* gauge_higgs_hmc.hpp:136-147, hmc.hpp:44-52 */
  const gho_lattice* lat = &h->lat;
  const int N = lat->N, NN = N * N, ng = NG(N);
  for (int64_t l = 0; l < lat->vol * lat->D; ++l) {
    cx Pm[GHO_MAXN * GHO_MAXN], E[GHO_MAXN * GHO_MAXN];
    gho_alg_to_mat(N, h->P + l * ng, (double*)Pm);
    for (int i = 0; i < NN; ++i) Pm[i] = cmul(Pm[i], cmk(eps, 0));
    gho_expi(N, (double*)Pm, (double*)E);
    cx* U = (cx*)h->U + l * NN;
    mmul(N, E, U, U);
  }
  if (has_scalar(h))
    for (int64_t i = 0; i < lat->vol * h->rep->d; ++i) CX(h->phi, i) = cadd(CX(h->phi, i), cscal(CX(h->pi, i), eps));
}

void gho_hmc_md_evolve(gho_hmc* h) {                     /* gauge_higgs_hmc.hpp:149-165 */
  const double eps = h->tau / h->nmd;
  if (h->integ == GHO_LEAPFROG) {
    gho_hmc_kick(h, 0.5 * eps);
    for (int i = 0; i < h->nmd; ++i) { gho_hmc_drift(h, eps); if (i != h->nmd - 1) gho_hmc_kick(h, eps); }
    gho_hmc_kick(h, 0.5 * eps);
  } else {
    const double lam = 0.1931833275037836;               /* src/core/config.hpp:25 */
    gho_hmc_kick(h, lam * eps);
    for (int i = 0; i < h->nmd; ++i) {
      gho_hmc_drift(h, 0.5 * eps);
      gho_hmc_kick(h, (1.0 - 2.0 * lam) * eps);
      gho_hmc_drift(h, 0.5 * eps);
      gho_hmc_kick(h, (i != h->nmd - 1 ? 2.0 * lam : lam) * eps);
    }
  }
}

void gho_hmc_refresh_momenta(gho_hmc* h) {               /* gauge_higgs_hmc.hpp:167-173, hmc.hpp:75-76 */
  if (!has_scalar(h)) {
    gho_mom_refresh(&h->lat, h->seed, gho_key(0xA1, h->traj_count, 0, 0, 0), h->P);
    return;
  }
  const uint64_t sg = gho_key(0xC3, h->traj_count, 0, 0, 0);
  const uint64_t ss = gho_key(0xD4, h->traj_count, 0, 0, 0);
  gho_mom_refresh(&h->lat, h->seed, sg, h->P);
  gho_phi_gaussian(&h->lat, h->rep->d, h->seed, ss, h->rep->real, 1.0, h->pi);
}

void gho_hmc_reunitarize_all(gho_hmc* h) {               /* fields.hpp:36 */
  const int N = h->lat.N, NN = N * N;
  for (int64_t l = 0; l < h->lat.vol * h->lat.D; ++l) gho_reunitarize(N, h->U + 2 * l * NN);
}

int gho_hmc_trajectory(gho_hmc* h) {                     /* gauge_higgs_hmc.hpp:175-192, hmc.hpp:73-91 */
  const gho_lattice* lat = &h->lat;
  const size_t nU = (size_t)lat->vol * lat->D * lat->N * lat->N * 2;
  const int d = has_scalar(h) ? h->rep->d : 0;
  const size_t nphi = (size_t)lat->vol * d * 2;
  gho_hmc_refresh_momenta(h);
  double* Us = (double*)malloc(sizeof(double) * nU);
  double* ps = (double*)malloc(sizeof(double) * (nphi ? nphi : 1));
  memcpy(Us, h->U, sizeof(double) * nU);
  if (nphi) memcpy(ps, h->phi, sizeof(double) * nphi);
  const double Hi = gho_hmc_hamiltonian(h);
  gho_hmc_md_evolve(h);
  if (h->reunit_each_traj) gho_hmc_reunitarize_all(h);
  const double Hf = gho_hmc_hamiltonian(h);
  h->last_dH = Hf - Hi;
  ++h->traj_count;
  const uint64_t ck = has_scalar(h) ? 0xE5 : 0xB2;
  const double r = gho_uniform(h->seed, gho_key(ck, h->traj_count, 0, 0, 0));
  const int accept = (h->last_dH <= 0.0) || (r < exp(-h->last_dH));
  if (accept) ++h->accept_count;
  else { memcpy(h->U, Us, sizeof(double) * nU); if (nphi) memcpy(h->phi, ps, sizeof(double) * nphi); }
  free(Us); free(ps);
  return accept;
}
