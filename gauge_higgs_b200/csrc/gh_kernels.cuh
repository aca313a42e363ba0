// gh_kernels.cuh -- sm_100a kernels of the gauge + Higgs molecular-dynamics path.
//
// Device layout (component-major, so that a warp's load of one component for 32
// consecutive sites is one 512 B (FP64) or 256 B (FP32) coalesced transaction;
// complex = {re,im} vector load):
//   U   [lat][mu][site/32][i*N+j][site%32]  complex R  (reference: [site*D+mu] N x N, src/core/fields.hpp:12-20)
//        blocks of 32 sites, the N*N components of a block side by side: the
//        components of one link lie at a fixed stride of 32 elements, so one
//        address serves all N*N loads (immediate offsets); the volume is padded
//        to a multiple of 32 (LatDev::Vp)
//   P   [lat][mu][site/32][a][site%32]  real R     (reference: [site*D+mu][a], src/core/fields.hpp:46-57)
//   phi [lat][site/32][k][site%32]      complex R  (reference: [site*d+k], src/core/scalar_field.hpp:15)
// R = double (FP64 mode) or float (FP32-MD mode).  Several lattices of unequal
// extents live back to back; every kernel walks a table of Work items (lattice,
// direction, first site, count), one per block, so a single launch covers all
// lattices of a batch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "gh_math.cuh"
#include "gh_rng.cuh"

namespace ghk {
using namespace ghm;

enum { REP_NONE = 0, REP_FUND = 1, REP_ADJ = 2, REP_GEN = 3 };
enum { F_GAUGE = 1, F_MATTER = 2 };
enum { M_UPDATE = 0, M_WRITE = 1 };
constexpr int KBLOCK = 128;    // threads per block of site/link kernels
#ifndef GH_KICK_LOG2
#define GH_KICK_LOG2 7
#endif
constexpr int KICK_LOG2 = GH_KICK_LOG2;      // sites per kick tile (= threads per kick block), log2
constexpr int KICK_BLOCK = 1 << KICK_LOG2;
constexpr int GEN_WARPS = 4;   // warps per block of the general-irrep kernel
constexpr int NRED = 6;        // per-site partial sums of the measure kernel
constexpr int ULANE = 32;      // sites per block of the link-field layout
enum { POT_QUARTIC = 0, POT_MULTI = 1 };
// Multi-invariant potential superoperator A[(r*d+q)][(i*d+j)], nonzeros only: CSR over
// the row pairs rq = r*d + q, column pair ij packed as i | j << 8, values in the
// precision of the arithmetic that reads them (double2 or float2).
struct PotA { const int* ptr; const unsigned short* ij; const void* v; };
constexpr int POT_DMAX = 32;   // largest representation the multi-invariant potential accepts

// Programmatic dependent launch: kernels of the MD path are launched so that the
// next one in the stream may be scheduled while this one finishes.  Each waits for
// its predecessor's results (griddepcontrol.wait: the predecessor grid has completed
// and its writes are visible) before reading anything, then lets its own successor
// launch.  Without the launch attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

struct LatDev {
  int L[4];
  int stride[4];
  int V;
  int Vp;                        // V rounded up to a multiple of ULANE (link-field plane size)
  int cidx;                      // coupling index (tempering bookkeeping)
  long long u_off, p_off, f_off, g_off;  // complex / real / complex / complex element offsets
  double beta, kappa, lambda;
  unsigned long long seed;
  unsigned long long traj, accepted, nonfinite;
  int last_acc;
  int lt[4];                     // kick tile shape: log2 of the tile extent per direction
  // Domain decomposition (src/mpi/gauge_mpi.hpp:26-80): a subdomain is stored with a
  // width-1 halo in every split direction.  Kernels act on the active box [lo, hi) only
  // (the whole lattice when not decomposed), and the counter RNG is keyed on the global
  // site index sum_mu (x_mu - lo_mu + goff_mu) * gstr_mu, so a decomposed lattice draws
  // the same numbers as the whole one.
  int lo[4], hi[4];
  int goff[4];
  long long gstr[4];
  int Vi;                        // active sites (normalises the lattice's sums)
  int dec;                       // 1: a subdomain with halo sites
};
// Site s inside the active box (always true for a lattice that is not decomposed).
__device__ __forceinline__ bool active_site(const LatDev& L, int s) {
  if (!L.dec) return true;
  int r = s;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const int x = r % L.L[mu];
    r /= L.L[mu];
    if (x < L.lo[mu] || x >= L.hi[mu]) return false;
  }
  return true;
}
// Below the active box's upper end in every direction: the interior and the lower halo
// layer, where the general-irrep link kernels also write psi_b = D(U)^dag phi, which the
// scalar force of the first interior layer reads at x - mu.
template <int D> __device__ __forceinline__ bool below_hi(const LatDev& L, const int* x) {
  bool in = true;
#pragma unroll
  for (int mu = 0; mu < D; ++mu) in = in && (x[mu] < L.hi[mu]);
  return in;
}
template <int D> __device__ __forceinline__ bool in_box(const LatDev& L, const int* x) {
  bool in = true;
#pragma unroll
  for (int mu = 0; mu < D; ++mu) in = in && (x[mu] >= L.lo[mu]) && (x[mu] < L.hi[mu]);
  return in;
}
// Global site index of local site s (the RNG key's site).
__device__ __forceinline__ long long global_site(const LatDev& L, int s) {
  if (!L.dec) return s;
  long long g = 0;
  int r = s;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const int x = r % L.L[mu];
    r /= L.L[mu];
    g += (long long)(x - L.lo[mu] + L.goff[mu]) * L.gstr[mu];
  }
  return g;
}
// Block work item.  Linear items: sites s0 .. s0+n-1.  Kick items (tiles): s0 is
// the tile's origin site and n packs the origin coordinates, 8 bits each.
// mu = -1 marks a site item, mu >= 0 a link item of direction mu.
struct Work { int lat, mu, s0, n; };

struct GenTables {                 // general irrep (src/rep/rep_general.hpp), sparse
  int d, n, dimT, ng;
  int powN[18];
  // division by powN[k] as a multiply-high: q = umulhi(f, pmag[k]) for k >= 1 (exact for
  // f * powN[k] < 2^32, which N^n <= 200000 guarantees); powN[0] = 1 needs none
  unsigned pmag[18];
  const int* wt_ptr; const int* wt_l; const double2* wt_v;   // lift: CSR over tensor index
  const int* w_ptr;  const int* w_i;  const double2* w_v;    // project: CSR over basis vector
  const int* t_ptr;  const int* t_j;  const double2* t_v;    // T^a_R: CSR over (a, row)
  // single-row irreps: D(U) in closed form (host term lists, gh_sympow.h); null: tensor path
  const int* sp_ptr; const double2* sp_c; const unsigned char* sp_e;
  int warp_bytes;                                            // shared memory of one warp
  int px_off;                                                // byte offset of px in a warp's region
  // irreps inside the K-fold adjoint product (host: gh_adjprod.h): the isometric
  // intertwiner Q [A][d] in both precisions; null: not available
  // rows of Q the kernel lifts into (all A, or for a symmetric / antisymmetric coefficient
  // matrix the pairs a <= b / a < b): prow[r] = a ng + b, the first pndiag diagonal
  const double2* pq64; const float2* pq32;
  const int* prow;
  int pK, pnrows, pndiag, psym;
  // two-slot irreps (n = 2): the basis W [d][N*N] dense in both precisions; null: not used
  const double2* w2_64; const float2* w2_32;
};

template <typename R> struct V2;
template <> struct V2<double> { typedef double2 t; };
template <> struct V2<float> { typedef float2 t; };
template <typename R> struct Cmp { typedef R t; };

template <typename C, typename R> __device__ __forceinline__ cx<C> ldc(const R* __restrict__ p, long long i) {
  const typename V2<R>::t v = __ldg(reinterpret_cast<const typename V2<R>::t*>(p) + i);
  return mk<C>((C)v.x, (C)v.y);
}
template <typename C, typename R> __device__ __forceinline__ cx<C> ldc_rw(const R* p, long long i) {
  const typename V2<R>::t v = reinterpret_cast<const typename V2<R>::t*>(p)[i];
  return mk<C>((C)v.x, (C)v.y);
}
template <typename C, typename R> __device__ __forceinline__ void stc(R* p, long long i, cx<C> z) {
  typename V2<R>::t v;
  v.x = (R)z.re;
  v.y = (R)z.im;
  reinterpret_cast<typename V2<R>::t*>(p)[i] = v;
}
// Sites are never negative: the 32-site block and lane come from a shift and a mask
// (a signed division by 32 costs the rounding fix-up on every address).
__device__ __forceinline__ long long site_blk(int s) { return (long long)((unsigned)s >> 5); }
__device__ __forceinline__ int site_lane(int s) { return (int)((unsigned)s & (ULANE - 1)); }
// Element index of component c of link (mu, s); component c + k sits k * ULANE further on.
__device__ __forceinline__ long long u_index(const LatDev& L, int nn, int mu, int c, int s) {
  return L.u_off + (long long)mu * nn * L.Vp + (site_blk(s) * nn + c) * ULANE + site_lane(s);
}
// Momenta P: [mu][site/32][a][site%32] (ng components, direction planes of ng * Vp)
__device__ __forceinline__ long long p_index(const LatDev& L, int ng, int mu, int g, int s) {
  return L.p_off + (long long)mu * ng * L.Vp + (site_blk(s) * ng + g) * ULANE + site_lane(s);
}
// Scalar fields phi, pi: [site/32][k][site%32] (d components)
__device__ __forceinline__ long long f_index(const LatDev& L, int d, int k, int s) {
  return L.f_off + (site_blk(s) * d + k) * ULANE + site_lane(s);
}
// General-irrep scratch psi_f, psi_b: [mu][site/32][k][site%32]
__device__ __forceinline__ long long g_index(const LatDev& L, int d, int mu, int k, int s) {
  return L.g_off + (long long)mu * d * L.Vp + (site_blk(s) * d + k) * ULANE + site_lane(s);
}
template <int N, typename C, typename R>
__device__ __forceinline__ Mat<N, C> ld_link(const R* __restrict__ U, const LatDev& L, int mu, int s) {
  Mat<N, C> M;
  const long long base = u_index(L, N * N, mu, 0, s);
#pragma unroll
  for (int c = 0; c < N * N; ++c) M.e[c] = ldc<C>(U, base + c * ULANE);
  return M;
}
template <int N, typename C, typename R>
__device__ __forceinline__ Mat<N, C> ld_link_rw(const R* U, const LatDev& L, int mu, int s) {
  Mat<N, C> M;
  const long long base = u_index(L, N * N, mu, 0, s);
#pragma unroll
  for (int c = 0; c < N * N; ++c) M.e[c] = ldc_rw<C>(U, base + c * ULANE);
  return M;
}
template <int N, typename C, typename R>
__device__ __forceinline__ void st_link(R* U, const LatDev& L, int mu, int s, const Mat<N, C>& M) {
  const long long base = u_index(L, N * N, mu, 0, s);
#pragma unroll
  for (int c = 0; c < N * N; ++c) stc<C>(U, base + c * ULANE, M.e[c]);
}

template <int D> __device__ __forceinline__ void coords(const LatDev& L, int s, int* x) {
  int r = s;
#pragma unroll
  for (int mu = 0; mu < D; ++mu) { x[mu] = r % L.L[mu]; r /= L.L[mu]; }
}
// neighbour of site s (whose coordinate in direction mu is xm) in +mu / -mu
__device__ __forceinline__ int nfwd(const LatDev& L, int s, int xm, int mu) {
  return (xm + 1 < L.L[mu]) ? s + L.stride[mu] : s - xm * L.stride[mu];
}
__device__ __forceinline__ int nbwd(const LatDev& L, int s, int xm, int mu) {
  return (xm > 0) ? s - L.stride[mu] : s + (L.L[mu] - 1) * L.stride[mu];
}
// Site of thread `tid` inside a kick tile: the tile's origin comes from the work
// item, the offset from tid split by the power-of-two tile extents.  Threads that
// fall outside the lattice's active box (partial tiles, halo sites) return false.
template <int D>
__device__ __forceinline__ bool tile_site(const LatDev& L, const Work& w, int tid, int& s, int* x) {
  s = w.s0;
  bool in = true;
  int r = tid;
#pragma unroll
  for (int mu = 0; mu < D; ++mu) {
    const int l = r & ((1 << L.lt[mu]) - 1);
    r >>= L.lt[mu];
    x[mu] = ((w.n >> (8 * mu)) & 0xFF) + l;
    in = in && (x[mu] >= L.lo[mu]) && (x[mu] < L.hi[mu]);
    s += l * L.stride[mu];
  }
  return in && (r == 0);
}

// ---------------------------------------------------------------------------
// Representation apply for the register-resident reps.
// Fundamental: D(U) = U (src/rep/rep_fundamental.hpp:15-25).
// Adjoint: D_ab = 2 Re Tr(T^a U T^b U^dag) (src/rep/rep_adjoint.hpp:27-40) applied
// without forming D: (D phi)_a = 2 Tr(T^a U Phi U^dag), Phi = sum_b phi_b T^b.
// ---------------------------------------------------------------------------
template <int N, typename C>
__device__ __forceinline__ void fund_apply(const Mat<N, C>& U, const cx<C>* v, cx<C>* o, bool dag) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    cx<C> s = zero<C>();
#pragma unroll
    for (int j = 0; j < N; ++j) s = dag ? cfma_cj(s, U.e[j * N + i], v[j]) : cfma(s, U.e[i * N + j], v[j]);
    o[i] = s;
  }
}
template <int N, typename C>
__device__ __forceinline__ void adj_apply(const Mat<N, C>& U, const cx<C>* v, cx<C>* o, bool dag) {
  const Mat<N, C> Phi = alg_to_mat_c<N, C>(v);
  Mat<N, C> Psi = dag ? mm(mm_dn(U, Phi), U) : mm_nd(mm(U, Phi), U);
  tr2_proj<N, C>(Psi, o);
}

template <int N, int REP> struct RepDim { static constexpr int d = (REP == REP_FUND) ? N : (REP == REP_ADJ) ? N * N - 1 : 1; };

// ---------------------------------------------------------------------------
// Kick: link items (gauge force + matter back-reaction, P -= eps F) and site
// items (scalar force, pi += eps F_phi) of one launch.
//   gauge force  F^a = (beta/N) Im Tr(T^a U Sigma)      src/action/gauge_wilson.hpp:11-27,70-83
//   matter force F^a = -kappa g^a                        src/action/scalar_higgs.hpp:113-128
//   scalar force F_phi = -2 dV/dphi* + 2 kappa sum_mu [D phi_{x+mu} + D^dag phi_{x-mu}]
//                                                        src/action/scalar_higgs.hpp:71-108
// Fundamental rep: -kappa g^a = 2 kappa Im Tr(T^a psi phi_x^dag), psi = U phi_{x+mu},
// so one projection of (beta/N) U Sigma + 2 kappa psi phi_x^dag gives the total link force.
// Adjoint rep: -kappa g^a = -4 kappa Im Tr(T^a [conj(Phi_x), U Phi_y U^dag]).
// ---------------------------------------------------------------------------
struct KickArgs {
  const Work* work;
  const LatDev* lats;
  const void* U;
  void* P;
  const void* phi;
  void* pi;
  const void* psif;   // general irrep scratch: D(U_mu(x)) phi_{x+mu}
  const void* psib;   // general irrep scratch: D(U_mu(x))^dag phi_x
  double eps;
  int mode;           // M_UPDATE or M_WRITE
  int flags;          // F_GAUGE | F_MATTER
  int d;              // rep dimension (general irreps)
  double* out;        // M_WRITE destination (SoA like P / like phi, FP64)
  int pot;            // POT_QUARTIC or POT_MULTI
  double mu2;         // multi-invariant potential: -mu2 phi^dag phi
  PotA sa;            // multi-invariant potential: A = sum_c 2 f_c P_c, values in the field precision
  const double2* wpot;  // general irreps: w = A(M) phi per site, written by k_gen_links
};

// The direction is a template parameter so that every index into the lattice
// descriptor is static (no local-memory copy of the descriptor).
template <int D, int N, typename R, int REP, int MU>
__device__ __forceinline__ void kick_link(const KickArgs& a, const LatDev& L, int s, const int* x) {
  typedef typename Cmp<R>::t C;
  constexpr int mu = MU;
  const R* U = (const R*)a.U;
  const int spm = nfwd(L, s, x[mu], mu);
  // U_mu(x) is loaded after the staple loop: its 2 N^2 registers stay free while the
  // neighbour links are in flight (measured: FP64 kick -7%, FP32 -1%)
  Mat<N, C> Om;
  set_zero(Om);
  Mat<N, C> Umu;
  if (!(a.flags & F_GAUGE)) Umu = ld_link<N, C>(U, L, mu, s);
  if (a.flags & F_GAUGE) {
    Mat<N, C> sig;
    set_zero(sig);
#pragma unroll
    for (int nu = 0; nu < D; ++nu) {
      if (nu == mu) continue;
      const int spn = nfwd(L, s, x[nu], nu);
      const int smn = nbwd(L, s, x[nu], nu);
      const int spm_mn = nbwd(L, spm, x[nu], nu);
      // upper staple U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, lower U_nu(x+mu-nu)^dag U_mu(x-nu)^dag U_nu(x-nu)
      // (the inner products of two links through mm_su: their last row from unitarity)
      mm_nd_acc(sig, mm_su<N, C, false, true>(ld_link<N, C>(U, L, nu, spm), ld_link<N, C>(U, L, mu, spn)),
                ld_link<N, C>(U, L, nu, s));
      mm_acc(sig, mm_su<N, C, true, true>(ld_link<N, C>(U, L, nu, spm_mn), ld_link<N, C>(U, L, mu, smn)),
             ld_link<N, C>(U, L, nu, smn));
    }
    Umu = ld_link<N, C>(U, L, mu, s);
    Om = mm(Umu, sig);
    const C c = (C)(L.beta / N);
#pragma unroll
    for (int i = 0; i < N * N; ++i) Om.e[i] = scale(Om.e[i], c);
  }
  if ((a.flags & F_MATTER) && (REP == REP_FUND || REP == REP_ADJ)) {
    constexpr int d = RepDim<N, REP>::d;
    const R* phi = (const R*)a.phi;
    cx<C> px[d], py[d];
#pragma unroll
    for (int k = 0; k < d; ++k) {
      px[k] = ldc<C>(phi, f_index(L, d, k, s));
      py[k] = ldc<C>(phi, f_index(L, d, k, spm));
    }
    const C kap = (C)L.kappa;
    if (REP == REP_FUND) {
      cx<C> psi[N];
      fund_apply<N, C>(Umu, py, psi, false);
      const C k2 = C(2) * kap;
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) Om.e[i * N + j] = add(Om.e[i * N + j], scale(mulc(psi[i], px[j]), k2));
    } else {
      cx<C> pxc[d];
#pragma unroll
      for (int k = 0; k < d; ++k) pxc[k] = conj(px[k]);
      const Mat<N, C> Phx = alg_to_mat_c<N, C>(pxc);
      const Mat<N, C> Psi = mm_nd(mm(Umu, alg_to_mat_c<N, C>(py)), Umu);
      const Mat<N, C> c1 = mm(Phx, Psi), c2 = mm(Psi, Phx);
      const C k4 = C(-4) * kap;
#pragma unroll
      for (int i = 0; i < N * N; ++i) Om.e[i] = add(Om.e[i], scale(sub(c1.e[i], c2.e[i]), k4));
    }
  }
  C F[N * N - 1];
  im_tr_proj<N, C>(Om, F);
  constexpr int ng = N * N - 1;
  const long long pb = p_index(L, ng, mu, 0, s);
  if (a.mode == M_UPDATE) {
    R* P = (R*)a.P;
    const C eps = (C)a.eps;
#pragma unroll
    for (int g = 0; g < ng; ++g) P[pb + g * ULANE] = (R)((C)P[pb + g * ULANE] - eps * F[g]);
  } else {
#pragma unroll
    for (int g = 0; g < ng; ++g) a.out[pb + g * ULANE] = (double)F[g];
  }
}

// ---------------------------------------------------------------------------
// Multi-invariant onsite potential at site s (src/action/scalar_invariants.hpp):
// with M = phi phi^dag and A = sum_c 2 f_c P_c the combined channel superoperator
// ((d^2) x (d^2), vec index i*d + j),
//   w = A(M) phi,  dV/dphi^* = -mu2 phi + w,  V = -mu2 phi^dag phi + Re(phi^dag w) / 2.
// Writes w (when given) and returns V.  One thread per site; A is held sparse (the
// weight of the Cartan generators is conserved, so 75-95% of its d^4 entries
// vanish: 1469 of 28561 for SU(2){12}), read through L1 (every thread of a warp
// reads the same entry).
// ---------------------------------------------------------------------------
template <typename C, typename R>
__device__ __noinline__ C pot_multi(const R* phi, const LatDev& L, int d, int s, const PotA A, C mu2, cx<C>* w) {
  typedef typename V2<C>::t VT;
  const VT* __restrict__ av = reinterpret_cast<const VT*>(A.v);
  cx<C> p[POT_DMAX];
  C n2 = C(0);
  for (int k = 0; k < d; ++k) {
    p[k] = ldc<C>(phi, f_index(L, d, k, s));
    n2 += norm2(p[k]);
  }
  C re = C(0);
  for (int r = 0; r < d; ++r) {
    cx<C> acc = zero<C>();
    for (int q = 0; q < d; ++q) {
      const int b = __ldg(A.ptr + r * d + q), e = __ldg(A.ptr + r * d + q + 1);
      if (b == e) continue;
      cx<C> y = zero<C>();                 // A(M)_rq = sum_ij A_{rq,ij} phi_i conj(phi_j)
      for (int z = b; z < e; ++z) {
        const int ij = __ldg(A.ij + z);
        const VT a = __ldg(av + z);
        y = cfma(y, mk<C>(a.x, a.y), mulc(p[ij & 0xFF], p[ij >> 8]));
      }
      acc = cfma(acc, y, p[q]);
    }
    if (w) w[r] = acc;
    re = fmad(p[r].re, acc.re, fmad(p[r].im, acc.im, re));
  }
  return -mu2 * n2 + C(0.5) * re;
}

template <int D, int N, typename R, int REP>
__device__ __forceinline__ void kick_site(const KickArgs& a, const LatDev& L, int s, const int* x) {
  typedef typename Cmp<R>::t C;
  const R* U = (const R*)a.U;
  const R* phi = (const R*)a.phi;
  const C kap2 = C(2) * (C)L.kappa;
  if (REP == REP_FUND || REP == REP_ADJ) {
    constexpr int d = RepDim<N, REP>::d;
    cx<C> F[d], v[d], o[d];
    C n2 = C(0);
#pragma unroll
    for (int k = 0; k < d; ++k) { v[k] = ldc<C>(phi, f_index(L, d, k, s)); n2 += norm2(v[k]); }
    if (a.pot == POT_MULTI) {          // -2 dV/dphi^* = 2 mu2 phi - 2 A(M) phi
      cx<C> w[d];
      pot_multi<C, R>(phi, L, d, s, a.sa, (C)a.mu2, w);
#pragma unroll
      for (int k = 0; k < d; ++k) F[k] = sub(scale(v[k], C(2) * (C)a.mu2), scale(w[k], C(2)));
    } else {                           // -2 dV/dphi^* = -2 [1 + 2 lambda (n2 - 1)] phi
      const C cc = C(1) + C(2) * (C)L.lambda * (n2 - C(1));
#pragma unroll
      for (int k = 0; k < d; ++k) F[k] = scale(v[k], C(-2) * cc);
    }
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
      const int yf = nfwd(L, s, x[mu], mu), yb = nbwd(L, s, x[mu], mu);
      cx<C> o2[d];
#pragma unroll
      for (int k = 0; k < d; ++k) v[k] = ldc<C>(phi, f_index(L, d, k, yf));
      {
        const Mat<N, C> Uf = ld_link<N, C>(U, L, mu, s);
        if (REP == REP_FUND) fund_apply<N, C>(Uf, v, o, false); else adj_apply<N, C>(Uf, v, o, false);
      }
#pragma unroll
      for (int k = 0; k < d; ++k) v[k] = ldc<C>(phi, f_index(L, d, k, yb));
      {
        const Mat<N, C> Ub = ld_link<N, C>(U, L, mu, yb);
        if (REP == REP_FUND) fund_apply<N, C>(Ub, v, o2, true); else adj_apply<N, C>(Ub, v, o2, true);
      }
#pragma unroll
      for (int k = 0; k < d; ++k) F[k] = add(F[k], scale(add(o[k], o2[k]), kap2));
    }
    const long long fb = f_index(L, d, 0, s);
    if (a.mode == M_UPDATE) {
      R* pi = (R*)a.pi;
      const C eps = (C)a.eps;
#pragma unroll
      for (int k = 0; k < d; ++k) stc<C>(pi, fb + k * ULANE, add(ldc_rw<C>(pi, fb + k * ULANE), scale(F[k], eps)));
    } else {
      double2* out = reinterpret_cast<double2*>(a.out);
#pragma unroll
      for (int k = 0; k < d; ++k) out[fb + k * ULANE] = make_double2((double)F[k].re, (double)F[k].im);
    }
  } else if (REP == REP_GEN) {
    const int d = a.d;
    const R* psif = (const R*)a.psif;
    const R* psib = (const R*)a.psib;
    C n2 = C(0);
    for (int k = 0; k < d; ++k) n2 += norm2(ldc<C>(phi, f_index(L, d, k, s)));
    const C cc = C(1) + C(2) * (C)L.lambda * (n2 - C(1));
    int yb[D];
#pragma unroll
    for (int mu = 0; mu < D; ++mu) yb[mu] = nbwd(L, s, x[mu], mu);
    for (int k = 0; k < d; ++k) {
      const cx<C> pk = ldc<C>(phi, f_index(L, d, k, s));
      cx<C> F;
      if (a.pot == POT_MULTI) {
        const double2 wk = a.wpot[f_index(L, d, k, s)];
        F = sub(scale(pk, C(2) * (C)a.mu2), scale(mk<C>((C)wk.x, (C)wk.y), C(2)));
      } else {
        F = scale(pk, C(-2) * cc);
      }
#pragma unroll
      for (int mu = 0; mu < D; ++mu) {
        
        F = add(F, scale(add(ldc<C>(psif, g_index(L, d, mu, k, s)), ldc<C>(psib, g_index(L, d, mu, k, yb[mu]))), kap2));
      }
      const long long fi = f_index(L, d, k, s);
      if (a.mode == M_UPDATE) {
        R* pi = (R*)a.pi;
        stc<C>(pi, fi, add(ldc_rw<C>(pi, fi), scale(F, (C)a.eps)));
      } else {
        reinterpret_cast<double2*>(a.out)[fi] = make_double2((double)F.re, (double)F.im);
      }
    }
  }
}

template <int D, int N, typename R, int REP>
__device__ __forceinline__ void kick_link_dispatch(const KickArgs& a, const LatDev& L, int mu, int s, const int* x) {
  if (mu == 0) kick_link<D, N, R, REP, 0>(a, L, s, x);
  else if (mu == 1) kick_link<D, N, R, REP, 1>(a, L, s, x);
  else if constexpr (D > 2) {
    if (mu == 2) kick_link<D, N, R, REP, 2>(a, L, s, x);
    else if constexpr (D > 3) kick_link<D, N, R, REP, 3>(a, L, s, x);
  }
}

// Occupancy: resident kick blocks per SM.  FP32 fundamental: 7 (72 registers, 40 bytes
// spilled); other FP32 kicks: 5 (the adjoint's commutator terms spill 432 bytes at 72
// registers against 28 at 96); FP64 fundamental: 4 (128 registers, 64 bytes spilled),
// other FP64 kicks 3 (the adjoint spills 1.3 KB at 128 registers).  Measured at
// SU(3) 16^4 (fundamental): the kick alone runs the same at FP32 5 and 7 blocks (24.5
// us) and at FP64 3 and 4 (40.7 / 40.9 us), while the trajectory with the higher
// occupancy is 1.4% (FP32) and 1.7% (FP64) faster -- the next launch's blocks find room
// sooner; FP32 6 blocks (80 registers) was 2.5% slower; FP32 4 / FP64 2 lose ~4%.
#ifndef GH_KICK_MINB_F32
#define GH_KICK_MINB_F32 5
#endif
#ifndef GH_KICK_MINB_F32_FUND
#define GH_KICK_MINB_F32_FUND 7
#endif
#ifndef GH_KICK_MINB_F64
#define GH_KICK_MINB_F64 3
#endif
#ifndef GH_KICK_MINB_F64_FUND
#define GH_KICK_MINB_F64_FUND 4
#endif
template <typename R, int REP> struct KickMinBlocks {
  static constexpr int v = (REP == REP_FUND ? GH_KICK_MINB_F32_FUND : GH_KICK_MINB_F32) * 128 / KICK_BLOCK;
};
template <int REP> struct KickMinBlocks<double, REP> {
  static constexpr int b = REP == REP_FUND ? GH_KICK_MINB_F64_FUND : GH_KICK_MINB_F64;
  static constexpr int v = b * 128 / KICK_BLOCK > 0 ? b * 128 / KICK_BLOCK : 1;
};

template <int D, int N, typename R, int REP>
__global__ void __launch_bounds__(KICK_BLOCK, KickMinBlocks<R, REP>::v) k_kick(const KickArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  const LatDev& L = a.lats[w.lat];
  int s, x[D];
  if (!tile_site<D>(L, w, threadIdx.x, s, x)) return;
  if (w.mu >= 0) kick_link_dispatch<D, N, R, REP>(a, L, w.mu, s, x);
  else if (REP != REP_NONE) kick_site<D, N, R, REP>(a, L, s, x);
}

// ---------------------------------------------------------------------------
// General irrep: one warp per link.  D^(R)(U) phi is applied matrix-free on the
// tensor space V^{xn} exactly as src/rep/rep_general.hpp:184-220 does (lift with
// the basis W, apply U on each of the n slots, project with W^dag), but W and
// T^a_R are held sparse (97% / 94% zeros for the SU(3) 27-plet) and the lanes of
// the warp split the tensor index / slot fibres / basis vectors between them.
// Single-row irreps whose term list the host built (GenTables::sp_ptr) take D(U)
// in closed form instead (sympow_matrix: the lanes split the d*d entries), then
// two d x d matrix-vector products.
//   mode 0: psi_f = D phi_{x+mu}, psi_b = D^dag phi_x -> scratch; P -= eps F_matter
//   mode 1: psi_f only (for the scalar action and the link energy)
//   mode 2: F_matter -> out (no P update), psi_f, psi_b -> scratch
// hop_link_g: src/rep/representation.hpp:36-46 / rep_general.hpp:151-159.
// ---------------------------------------------------------------------------
struct GenArgs {
  const Work* work;
  const LatDev* lats;
  const void* U;
  void* P;
  const void* phi;
  void* psif;
  void* psib;
  GenTables t;
  double eps;
  int mode;
  double* out;
  int pot;            // POT_MULTI: the warps of mu = 0 also write w = A(M) phi_x
  PotA sa;            // superoperator rows, FP64 values
  double2* wpot;      // w per site, FP64, laid out like phi
};

template <int N, typename C>
__device__ void gen_apply(const GenTables& t, const Mat<N, C>& M, bool dag, const cx<C>* vin, cx<C>* buf,
                          cx<C>* vout, int lane) {
  // lift: buf[i] = sum_l vin[l] W_l[i]
  for (int i = lane; i < t.dimT; i += 32) {
    cx<C> s = zero<C>();
    for (int p = t.wt_ptr[i]; p < t.wt_ptr[i + 1]; ++p) {
      const double2 w = t.wt_v[p];
      s = cfma(s, vin[t.wt_l[p]], mk<C>((C)w.x, (C)w.y));
    }
    buf[i] = s;
  }
  __syncwarp();
  // slot applies: fibre f of slot sl holds the N entries base + j*blk
  const int nf = t.dimT / N;
  for (int sl = 0; sl < t.n; ++sl) {
    const int k = t.n - 1 - sl;
    const int blk = t.powN[k];
    const unsigned mag = t.pmag[k];
    // fibre f = hi * blk + lo starts at hi * blk * N + lo.  Odd N in FP64 with more than
    // 64 fibres per slot (over two per lane) walks them as f = lo * N^(n-1-k) + hi instead (consecutive
    // lanes step hi): the same fibres, each computed alike, so the results do not change;
    // SU(3) 27-plet FP64 trajectories +8%, while the sextet, the octet and FP32 ran 1-4%
    // slower with it, so they keep the plain order
    const int kq = t.n - 1 - k;
    const unsigned magq = t.pmag[kq];
    const bool swap = (sizeof(C) == 8) && (N & 1) && nf > 64;
    for (int f = lane; f < nf; f += 32) {
      int base;
      if (swap) {
        const int lo = (kq == 0) ? f : (int)__umulhi((unsigned)f, magq);
        base = (f - lo * t.powN[kq]) * blk * N + lo;
      } else {
        const int q = (k == 0) ? f : (int)__umulhi((unsigned)f, mag);
        base = q * blk * (N - 1) + f;              // (f / blk) * blk * N + f % blk
      }
      cx<C> v[N];
#pragma unroll
      for (int j = 0; j < N; ++j) v[j] = buf[base + j * blk];
#pragma unroll
      for (int j = 0; j < N; ++j) {
        cx<C> s = zero<C>();
#pragma unroll
        for (int g = 0; g < N; ++g) s = dag ? cfma_cj(s, M.e[g * N + j], v[g]) : cfma(s, M.e[j * N + g], v[g]);
        buf[base + j * blk] = s;
      }
    }
    __syncwarp();
  }
  // project: vout[k] = sum_i conj(W_k[i]) buf[i]
  for (int k = lane; k < t.d; k += 32) {
    cx<C> s = zero<C>();
    for (int p = t.w_ptr[k]; p < t.w_ptr[k + 1]; ++p) {
      const double2 w = t.w_v[p];
      s = cfma_cj(s, mk<C>((C)w.x, (C)w.y), buf[t.w_i[p]]);
    }
    vout[k] = s;
  }
  __syncwarp();
}

// D(U) of a single-row irrep from its term list, FP64, one warp:
//   D[k][l] = sum_terms c prod_ij U_ij^K_ij
// with the powers U_ij^p (p = 0..n) tabulated first (entry ij*(n+1) + p) and each term
// given by its offsets into that table.  Dm: d*d, Pw: N*N*(n+1) entries of this warp's
// shared memory.
template <int N, typename C>
__device__ void sympow_matrix(const GenTables& t, const Mat<N, C>& M, cx<double>* Dm, cx<double>* Pw, int lane) {
  const int n = t.n, d = t.d;
  if (lane < N * N) {
    const cx<double> u = mk<double>((double)M.e[lane].re, (double)M.e[lane].im);
    cx<double> p = mk<double>(1.0, 0.0);
    for (int q = 0; q <= n; ++q) {
      Pw[lane * (n + 1) + q] = p;
      p = mul(p, u);
    }
  }
  __syncwarp();
  for (int e = lane; e < d * d; e += 32) {
    cx<double> acc = zero<double>();
    for (int q = t.sp_ptr[e]; q < t.sp_ptr[e + 1]; ++q) {
      const double2 c = t.sp_c[q];
      cx<double> pr = mk<double>(c.x, c.y);
      // offsets into the power table, N*N bytes per term in whole 32-bit words: SU(2)
      // multiplies all four factors (an exponent 0 points at a 1), larger N the nonzero
      // factors up to the first 0xFF
      constexpr int EW = (N * N + 3) / 4;
      const unsigned* ex = reinterpret_cast<const unsigned*>(t.sp_e) + (size_t)q * EW;
      unsigned w[EW];
#pragma unroll
      for (int i = 0; i < EW; ++i) w[i] = __ldg(ex + i);
      if constexpr (N == 2) {
#pragma unroll
        for (int f = 0; f < 4; ++f) pr = mul(pr, Pw[(w[0] >> (8 * f)) & 0xFF]);
      } else {
#pragma unroll
        for (int f = 0; f < N * N; ++f) {
          const unsigned o = (w[f >> 2] >> (8 * (f & 3))) & 0xFF;
          if (o == 0xFF) break;
          pr = mul(pr, Pw[o]);
        }
      }
      acc = add(acc, pr);
    }
    Dm[e] = acc;
  }
  __syncwarp();
}

template <int D, int N, typename R>
__global__ void __launch_bounds__(GEN_WARPS * 32) k_gen_links(const GenArgs a) {
  pdl_enter();
  typedef typename Cmp<R>::t C;
  extern __shared__ unsigned char smem_raw[];
  const Work w = a.work[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= w.n) return;
  const LatDev L = a.lats[w.lat];
  const int mu = w.mu, s = w.s0 + warp;
  const int d = a.t.d, dimT = a.t.dimT;
  // this warp's shared memory: tensor path [buf: dimT][px py pf pb: d each];
  // closed-form path [Dm: d*d][Pw: N*N*(n+1)] (FP64) then [px py pf pb]
  unsigned char* wbase = smem_raw + (size_t)warp * a.t.warp_bytes;
  const bool sp = a.t.sp_ptr != nullptr;
  cx<double>* Dm = reinterpret_cast<cx<double>*>(wbase);
  cx<double>* Pw = Dm + d * d;
  cx<C>* buf = reinterpret_cast<cx<C>*>(wbase);
  // the region before px (the tensor buffer or D and the powers) also holds, before it
  // is filled, A(M) of the potential (d*d FP64 complex) where that fits, and, after,
  // the matter force's partial sums (ng*d doubles, which the host makes room for)
  cx<C>* px = reinterpret_cast<cx<C>*>(wbase + a.t.px_off);
  cx<C>* py = px + d;
  cx<C>* pf = py + d;
  cx<C>* pb = pf + d;
  const R* U = (const R*)a.U;
  const R* phi = (const R*)a.phi;
  int x[D];
  coords<D>(L, s, x);
  if (!below_hi<D>(L, x)) return;                // upper halo link of a subdomain (whole warp)
  const bool own = in_box<D>(L, x);              // the link's momentum belongs to this subdomain
  const int spm = nfwd(L, s, x[mu], mu);
  const Mat<N, C> M = ld_link<N, C>(U, L, mu, s);
  for (int k = lane; k < d; k += 32) {
    px[k] = ldc<C>(phi, f_index(L, d, k, s));
    py[k] = ldc<C>(phi, f_index(L, d, k, spm));
  }
  __syncwarp();
  if (a.pot == POT_MULTI && mu == 0) {
    // multi-invariant potential of site s (FP64):
    //   A(M)_rq = sum_ij A_{rq,ij} phi_i conj(phi_j),  w_r = sum_q A(M)_rq phi_q.
    // Where A(M) fits in the region before px (always on the closed-form path) the
    // lanes split the row pairs rq, then one lane per r sums over q; otherwise one
    // lane per r does both.  Fixed summation order either way.
    const double2* __restrict__ av = reinterpret_cast<const double2*>(a.sa.v);
    const bool split = (size_t)d * d * sizeof(cx<double>) <= (size_t)a.t.px_off;
    cx<double>* AM = reinterpret_cast<cx<double>*>(wbase);
    auto am = [&](int rq) {
      const int b = __ldg(a.sa.ptr + rq), e = __ldg(a.sa.ptr + rq + 1);
      cx<double> y = zero<double>();
      for (int z = b; z < e; ++z) {
        const int ij = __ldg(a.sa.ij + z);
        const double2 v = __ldg(av + z);
        const cx<C> pi = px[ij & 0xFF], pj = px[ij >> 8];
        y = cfma(y, mk<double>(v.x, v.y), mulc(mk<double>(pi.re, pi.im), mk<double>(pj.re, pj.im)));
      }
      return y;
    };
    if (split) {
      for (int rq = lane; rq < d * d; rq += 32) AM[rq] = am(rq);
      __syncwarp();
    }
    for (int r = lane; r < d; r += 32) {
      cx<double> acc = zero<double>();
      for (int q = 0; q < d; ++q) acc = cfma(acc, split ? AM[r * d + q] : am(r * d + q), mk<double>(px[q].re, px[q].im));
      a.wpot[f_index(L, d, r, s)] = make_double2(acc.re, acc.im);
    }
    __syncwarp();
  }
  if (sp) {
    sympow_matrix<N, C>(a.t, M, Dm, Pw, lane);
    // psi_f = D phi_y on lanes 0..d-1, psi_b = D^dag phi_x on the next d lanes
    const int nv = a.mode == 1 ? d : 2 * d;
    for (int t = lane; t < nv; t += 32) {
      cx<double> acc = zero<double>();
      if (t < d) {
        for (int l = 0; l < d; ++l) acc = cfma(acc, Dm[t * d + l], mk<double>((double)py[l].re, (double)py[l].im));
        pf[t] = mk<C>((C)acc.re, (C)acc.im);
      } else {
        const int k = t - d;
        for (int l = 0; l < d; ++l) acc = cfma_cj(acc, Dm[l * d + k], mk<double>((double)px[l].re, (double)px[l].im));
        pb[k] = mk<C>((C)acc.re, (C)acc.im);
      }
    }
    __syncwarp();
  } else {
    gen_apply<N, C>(a.t, M, false, py, buf, pf, lane);
    if (a.mode != 1) gen_apply<N, C>(a.t, M, true, px, buf, pb, lane);
  }
  R* psif = (R*)a.psif;
  R* psib = (R*)a.psib;
  for (int k = lane; k < d; k += 32) {
    const long long gi = g_index(L, d, mu, k, s);
    stc<C>(psif, gi, pf[k]);
    if (a.mode != 1) stc<C>(psib, gi, pb[k]);
  }
  if (a.mode == 1 || !own) return;
  // matter force: g^a = -2 Im(phi_x^dag T^a_R psi_f), F^a = -kappa g^a.  The lanes
  // split the (a, row) pairs; the rows of each a are then summed in order.
  constexpr int ng = N * N - 1;
  double* zc = reinterpret_cast<double*>(wbase);
  for (int r = lane; r < ng * d; r += 32) {
    const int i = r % d;
    cx<C> ti = zero<C>();
    for (int p = a.t.t_ptr[r]; p < a.t.t_ptr[r + 1]; ++p) {
      const double2 tv = a.t.t_v[p];
      ti = cfma(ti, mk<C>((C)tv.x, (C)tv.y), pf[a.t.t_j[p]]);
    }
    zc[r] = (double)px[i].re * (double)ti.im - (double)px[i].im * (double)ti.re;   // Im(conj(phi_i) t_i)
  }
  __syncwarp();
  for (int g = lane; g < ng; g += 32) {
    double zim = 0.0;
    for (int i = 0; i < d; ++i) zim += zc[g * d + i];
    const C F = -(C)L.kappa * (C(-2) * (C)zim);
    const long long pi_ = p_index(L, ng, mu, g, s);
    if (a.mode == 0) {
      R* P = (R*)a.P;
      P[pi_] = (R)((C)P[pi_] - (C)a.eps * F);
    } else {
      a.out[pi_] = (double)F;
    }
  }
}

// ---------------------------------------------------------------------------
// General irreps inside the K-fold adjoint product (K = 1, 2; host set-up and the
// algebra in gh_adjprod.h): with the fixed isometric intertwiner Q (A x d,
// A = (N^2 - 1)^K) from the reference's basis into the product,
//   D_R(U) phi = Q^dag (G (x) ... (x) G) Q phi,   G_ab = 2 Re Tr(T^a U T^b U^dag),
// and D_R(U)^dag phi with G^T.  One block takes the 32 links of one 32-site block and
// one direction, 8 threads per link: the lift Q phi and the projection Q^dag y are
// 64 x 27 and 27 x 64 products shared by the 32 links (every warp reads the same Q
// entry, every lane its own link); G (x) G acts as X -> G X G^T on each link's 8 x 8
// coefficient matrix, one row per thread.  Same modes and outputs as k_gen_links
// (psi_f, psi_b, matter force); the multi-invariant potential's w stays there.
// The matter force is g^a = -2 Im(phi_x^dag T^a_R psi_f) (src/rep/rep_general.hpp:151-159),
// one generator per thread, rows summed in order.
// ---------------------------------------------------------------------------
constexpr int GP_LINKS = 32;      // links per block (one 32-site block, one direction)
constexpr int GP_THREADS = 256;   // 8 per link
template <int N, int K> struct AdjProd {
  static constexpr int NG = N * N - 1;
  static constexpr int A = (K == 1) ? NG : NG * NG;
  static constexpr int RA = (A + 7) / 8;      // rows of A (and of d <= A) per thread
};
template <int N, int K, typename C> __host__ __device__ constexpr size_t gen_prod_smem(int d, int nrows) {
  return (size_t)nrows * d * sizeof(cx<C>) + (size_t)(2 * d + AdjProd<N, K>::A) * GP_LINKS * sizeof(cx<C>) +
         (size_t)AdjProd<N, K>::NG * AdjProd<N, K>::NG * GP_LINKS * sizeof(C);
}

// out[i] = (D phi)_k, k = q + 8 i, for the link in lane c; Pin: [d][32] input vectors;
// Qs: [nrows][d] the rows of Q in shared memory; X: [A][32] work space; G: [NG][NG][32]
// adjoint matrices.  Every thread of the block calls it.
template <int N, int K, typename C>
__device__ __forceinline__ void gp_apply(const GenTables& t, const cx<C>* Qs, int d, const cx<C>* Pin, cx<C>* X,
                                         const C* G, bool dag, int c, int q, cx<C>* out) {
  constexpr int NG = AdjProd<N, K>::NG, A = AdjProd<N, K>::A, RA = AdjProd<N, K>::RA, LB = GP_LINKS;
  const int nr = t.pnrows;
  cx<C> acc[RA];
#pragma unroll
  for (int i = 0; i < RA; ++i) acc[i] = zero<C>();
  for (int l = 0; l < d; ++l) {                         // lift: the needed rows of X = Q phi
    const cx<C> p = Pin[l * LB + c];
#pragma unroll
    for (int i = 0; i < RA; ++i) {
      const int r = q + 8 * i;
      if (r < nr) acc[i] = cfma(acc[i], Qs[r * d + l], p);
    }
  }
  __syncthreads();                                      // earlier readers of X are done
  if (K == 2 && t.psym < 0 && q < NG) X[(q * NG + q) * LB + c] = zero<C>();   // antisymmetric: zero diagonal
#pragma unroll
  for (int i = 0; i < RA; ++i) {
    const int r = q + 8 * i;
    if (r < nr) {
      const int e = __ldg(t.prow + r);
      X[e * LB + c] = acc[i];
      if (K == 2 && t.psym != 0) {
        const int a = e / NG, b = e - a * NG;
        if (a != b) X[(b * NG + a) * LB + c] = t.psym > 0 ? acc[i] : mk<C>(-acc[i].re, -acc[i].im);
      }
    }
  }
  __syncthreads();
  auto g = [&](int a, int b) { return dag ? G[(b * NG + a) * LB + c] : G[(a * NG + b) * LB + c]; };
  if constexpr (K == 1) {                               // y = G x
    cx<C> y = zero<C>();
    const int a = q;
    if (a < NG)
#pragma unroll
      for (int k = 0; k < NG; ++k) y = add(y, scale(X[k * LB + c], g(a, k)));
    __syncthreads();
    if (a < NG) X[a * LB + c] = y;
  } else {                                              // Y = G X G^T, row a of this thread
    const int a = q;
    cx<C> y[NG];
    if (a < NG) {
      cx<C> z[NG];
#pragma unroll
      for (int b = 0; b < NG; ++b) {
        cx<C> sacc = zero<C>();
#pragma unroll
        for (int k = 0; k < NG; ++k) sacc = add(sacc, scale(X[(k * NG + b) * LB + c], g(a, k)));
        z[b] = sacc;
      }
#pragma unroll
      for (int b = 0; b < NG; ++b) {
        cx<C> sacc = zero<C>();
#pragma unroll
        for (int k = 0; k < NG; ++k) sacc = add(sacc, scale(z[k], g(b, k)));
        y[b] = sacc;
      }
    }
    __syncthreads();
    if (a < NG)
#pragma unroll
      for (int b = 0; b < NG; ++b) X[(a * NG + b) * LB + c] = y[b];
  }
  __syncthreads();
  // project: out = Q^dag y over the needed rows; off-diagonal pairs of a symmetric or
  // antisymmetric coefficient matrix count twice (their mirror entries are equal terms)
#pragma unroll
  for (int i = 0; i < RA; ++i) {
    const int k = q + 8 * i;
    cx<C> s1 = zero<C>(), s2 = zero<C>();
    if (k < d) {
      for (int r = 0; r < t.pndiag; ++r) s1 = cfma_cj(s1, Qs[r * d + k], X[__ldg(t.prow + r) * LB + c]);
      for (int r = t.pndiag; r < nr; ++r) s2 = cfma_cj(s2, Qs[r * d + k], X[__ldg(t.prow + r) * LB + c]);
    }
    out[i] = add(s1, scale(s2, C(2)));
  }
}

template <int D, int N, typename R, int K>
__global__ void __launch_bounds__(GP_THREADS) k_gen_prod(const GenArgs a) {
  pdl_enter();
  typedef typename Cmp<R>::t C;
  constexpr int NG = AdjProd<N, K>::NG, A = AdjProd<N, K>::A, RA = AdjProd<N, K>::RA, LB = GP_LINKS;
  extern __shared__ unsigned char smem_raw[];
  const Work w = a.work[blockIdx.x];
  const LatDev& L = a.lats[w.lat];
  const int d = a.t.d;
  const int c = threadIdx.x & (LB - 1), q = threadIdx.x >> 5;
  cx<C>* Qs = reinterpret_cast<cx<C>*>(smem_raw);       // [nrows][d] the rows of Q the lift uses
  cx<C>* Px = Qs + a.t.pnrows * d;                      // [d][32] phi_x
  cx<C>* Py = Px + d * LB;                              // [d][32] phi_{x+mu}, then psi_f
  cx<C>* X = Py + d * LB;                               // [A][32]
  C* G = reinterpret_cast<C*>(X + A * LB);              // [NG][NG][32]
  {
    const typename V2<C>::t* Qv = reinterpret_cast<const typename V2<C>::t*>(
        sizeof(C) == sizeof(double) ? (const void*)a.t.pq64 : (const void*)a.t.pq32);
    for (int i = threadIdx.x; i < a.t.pnrows * d; i += GP_THREADS) {
      const typename V2<C>::t v = __ldg(Qv + i);
      Qs[i] = mk<C>(v.x, v.y);
    }
  }
  const int mu = w.mu;
  const int s = w.s0 + (c < w.n ? c : 0);              // lanes past the lattice's end compute on site s0
  int x[D];
  coords<D>(L, s, x);
  const bool live = c < w.n && below_hi<D>(L, x);      // and store nothing, as upper halo sites of a subdomain
  const bool own = live && in_box<D>(L, x);            // momentum updates: interior links only
  const int spm = nfwd(L, s, x[mu], mu);
  const R* phi = (const R*)a.phi;
  for (int k = q; k < d; k += 8) {
    Px[k * LB + c] = ldc<C>(phi, f_index(L, d, k, s));
    Py[k * LB + c] = ldc<C>(phi, f_index(L, d, k, spm));
  }
  {
    const Mat<N, C> U = ld_link<N, C>((const R*)a.U, L, mu, s);
    for (int b = q; b < NG; b += 8) {                   // column b of G: 2 Tr(T^a U T^b U^dag)
      C e[NG];
#pragma unroll
      for (int k = 0; k < NG; ++k) e[k] = (k == b) ? C(1) : C(0);
      const Mat<N, C> M = mm_nd(mm(U, alg_to_mat<N, C>(e)), U);
      cx<C> o[NG];
      tr2_proj<N, C>(M, o);
#pragma unroll
      for (int k = 0; k < NG; ++k) G[(k * NG + b) * LB + c] = o[k].re;
    }
  }
  __syncthreads();
  R* psif = (R*)a.psif;
  R* psib = (R*)a.psib;
  cx<C> o[RA];
  gp_apply<N, K, C>(a.t, Qs, d, Py, X, G, false, c, q, o);  // psi_f = D phi_{x+mu}
#pragma unroll
  for (int i = 0; i < RA; ++i) {
    const int k = q + 8 * i;
    if (k < d) {
      Py[k * LB + c] = o[i];
      if (live) stc<C>(psif, g_index(L, d, mu, k, s), o[i]);
    }
  }
  if (a.mode == 1) return;
  gp_apply<N, K, C>(a.t, Qs, d, Px, X, G, true, c, q, o);   // psi_b = D^dag phi_x
#pragma unroll
  for (int i = 0; i < RA; ++i) {
    const int k = q + 8 * i;
    if (k < d && live) stc<C>(psib, g_index(L, d, mu, k, s), o[i]);
  }
  __syncthreads();
  for (int gi = q; gi < NG; gi += 8) {                  // matter force, generator gi
    double zim = 0.0;
    for (int i = 0; i < d; ++i) {
      const int r = gi * d + i;
      cx<C> ti = zero<C>();
      for (int p = a.t.t_ptr[r]; p < a.t.t_ptr[r + 1]; ++p) {
        const double2 tv = a.t.t_v[p];
        ti = cfma(ti, mk<C>((C)tv.x, (C)tv.y), Py[a.t.t_j[p] * LB + c]);
      }
      const cx<C> pxi = Px[i * LB + c];
      zim += (double)pxi.re * (double)ti.im - (double)pxi.im * (double)ti.re;   // Im(conj(phi_i) t_i)
    }
    if (!own) continue;
    const C F = -(C)L.kappa * (C(-2) * (C)zim);
    const long long pi_ = p_index(L, NG, mu, gi, s);
    if (a.mode == 0) {
      R* P = (R*)a.P;
      P[pi_] = (R)((C)P[pi_] - (C)a.eps * F);
    } else {
      a.out[pi_] = (double)F;
    }
  }
}

// ---------------------------------------------------------------------------
// Two-slot irreps (n = 2: the symmetric and antisymmetric squares of V, e.g. the SU(3)
// sextet {2} and antitriplet {1,1}) in registers, one thread per link.  With the irrep
// basis W ([d][N*N], tensor index i*N + j for the slots (i, j)) the reference's tensor
// apply (src/rep/rep_general.hpp:184-220: lift with W, U on each slot, project with W^H)
// is, as N x N matrices,
//   Phi = sum_b phi_b W_b,  Psi = U Phi U^T,  psi_b = sum_ij conj(W_b,ij) Psi_ij,
// and D^dag phi the same with Psi = U^dag Phi conj(U).  Every W_b is symmetric or
// antisymmetric, so phi_x^dag T^a_R psi_f = Tr(Phi_x^dag (T^a Psi + Psi T^aT))
// = 2 Tr(T^a Psi Phi_x^dag), and the matter force -kappa g^a, g^a = -2 Im(phi_x^dag
// T^a_R D phi_{x+mu}) (src/rep/representation.hpp:36-46), is 4 kappa Im Tr(T^a Psi
// Phi_x^dag): one N x N product and the projection the fundamental uses.  Outputs and
// modes as k_gen_links: psi_f, psi_b to the scratch fields; mode 0 P -= eps F, mode 2
// F -> out, mode 1 psi_f only.
// ---------------------------------------------------------------------------
template <int N, typename C, typename R>
__device__ __forceinline__ Mat<N, C> pair_lift(const typename V2<C>::t* Wt, int d, const R* phi, const LatDev& L, int s) {
  Mat<N, C> M;
  set_zero(M);
  for (int b = 0; b < d; ++b) {
    const cx<C> f = ldc<C>(phi, f_index(L, d, b, s));
#pragma unroll
    for (int t = 0; t < N * N; ++t) {
      const typename V2<C>::t v = __ldg(Wt + b * N * N + t);
      M.e[t] = cfma(M.e[t], f, mk<C>(v.x, v.y));
    }
  }
  return M;
}
template <int N, typename C, typename R>
__device__ __forceinline__ void pair_project(const typename V2<C>::t* Wt, int d, const Mat<N, C>& M, R* out,
                                             const LatDev& L, int mu, int s) {
  for (int b = 0; b < d; ++b) {
    cx<C> z = zero<C>();
#pragma unroll
    for (int t = 0; t < N * N; ++t) {
      const typename V2<C>::t v = __ldg(Wt + b * N * N + t);
      z = cfma(z, mk<C>(v.x, -v.y), M.e[t]);
    }
    stc<C>(out, g_index(L, d, mu, b, s), z);
  }
}
template <int N, typename C> __device__ __forceinline__ Mat<N, C> conj_mat(const Mat<N, C>& A) {
  Mat<N, C> B;
#pragma unroll
  for (int i = 0; i < N * N; ++i) B.e[i] = conj(A.e[i]);
  return B;
}
template <int D, int N, typename R>
__global__ void __launch_bounds__(KBLOCK) k_gen_pair(const GenArgs a) {
  pdl_enter();
  typedef typename Cmp<R>::t C;
  const Work w = a.work[blockIdx.x];
  if ((int)threadIdx.x >= w.n) return;
  const LatDev& L = a.lats[w.lat];
  const int mu = w.mu, s = w.s0 + threadIdx.x;
  int x[D];
  coords<D>(L, s, x);
  if (!below_hi<D>(L, x)) return;                      // upper halo sites of a subdomain store nothing
  const int d = a.t.d;
  const typename V2<C>::t* Wt = reinterpret_cast<const typename V2<C>::t*>(
      sizeof(C) == sizeof(double) ? (const void*)a.t.w2_64 : (const void*)a.t.w2_32);
  const R* phi = (const R*)a.phi;
  const Mat<N, C> U = ld_link<N, C>((const R*)a.U, L, mu, s);
  const Mat<N, C> Uc = conj_mat(U);
  const int spm = nfwd(L, s, x[mu], mu);
  // psi_f = D phi_{x+mu}: U Phi U^T = (U Phi) conj(U)^dag
  const Mat<N, C> Psi = mm_nd(mm(U, pair_lift<N, C>(Wt, d, phi, L, spm)), Uc);
  pair_project<N, C>(Wt, d, Psi, (R*)a.psif, L, mu, s);
  if (a.mode == 1) return;
  const Mat<N, C> Phx = pair_lift<N, C>(Wt, d, phi, L, s);
  // psi_b = D^dag phi_x: U^dag Phi conj(U)
  pair_project<N, C>(Wt, d, mm(mm_dn(U, Phx), Uc), (R*)a.psib, L, mu, s);
  if (!in_box<D>(L, x)) return;                        // momentum updates: interior links only
  Mat<N, C> M = mm_nd(Psi, Phx);
  const C k4 = C(4) * (C)L.kappa;
#pragma unroll
  for (int i = 0; i < N * N; ++i) M.e[i] = scale(M.e[i], k4);
  constexpr int ng = N * N - 1;
  C F[ng];
  im_tr_proj<N, C>(M, F);
  const long long pb = p_index(L, ng, mu, 0, s);
  if (a.mode == 0) {
    R* P = (R*)a.P;
    const C eps = (C)a.eps;
#pragma unroll
    for (int g = 0; g < ng; ++g) P[pb + g * ULANE] = (R)((C)P[pb + g * ULANE] - eps * F[g]);
  } else {
#pragma unroll
    for (int g = 0; g < ng; ++g) a.out[pb + g * ULANE] = (double)F[g];
  }
}

// ---------------------------------------------------------------------------
// Drift: U <- exp(i eps P) U (src/hmc/gauge_higgs_hmc.hpp:136-143); site items:
// phi += eps pi (:145-146).  The link update (exponential, product with U,
// projection) runs in the arithmetic type A, whatever the storage type R:
//   FP64 mode       R = double, A = double, no projection (the reference's
//                   reunitarisation once per trajectory, k_reunit);
//   FP32-MD         R = float,  A = double: FP32 links and momenta are widened,
//                   exp(i eps P) (scaling, Cayley-Hamilton series), its product
//                   with U and the Gram-Schmidt projection back to SU(N) are
//                   FP64, the result is rounded to FP32 once;
//   FP32-MD, all    R = float,  A = float: the same steps in FP32 (non-default
//   FP32            variant, GH_PREC_FP32_ALL).
// ---------------------------------------------------------------------------
// Projection back to SU(N) after each FP32-MD drift: Gram-Schmidt on the first
// N-1 rows, the last row fixed by det = 1 (SU(2): (-conj u01, conj u00); SU(3):
// conj(row0 x row1)).  The trajectory-end reunitarisation of the FP64 mode keeps
// the reference's algorithm (k_reunit).
template <int N, typename T>
__device__ __forceinline__ void project_su(Mat<N, T>& U) {
  // rows stay within ~1e-6 of unit norm between projections: one Newton step of
  // 1/sqrt from 1 (x^-1/2 ~ (3 - x)/2) is exact to ~1e-12, a second to FP64 resolution
  T n0 = 0;
#pragma unroll
  for (int j = 0; j < N; ++j) n0 += norm2(U.e[j]);
  T i0 = T(1.5) - T(0.5) * n0;
  i0 = i0 * (T(1.5) - T(0.5) * n0 * i0 * i0);
  if (fabs(n0 - T(1)) > T(1e-3)) i0 = rsqrt(n0);    // far from unitary (links set by the caller)
#pragma unroll
  for (int j = 0; j < N; ++j) U.e[j] = scale(U.e[j], i0);
  if (N == 2) {
    U.e[2] = mk<T>(-U.e[1].re, U.e[1].im);
    U.e[3] = mk<T>(U.e[0].re, -U.e[0].im);
    return;
  }
  cx<T> p = zero<T>();
#pragma unroll
  for (int j = 0; j < N; ++j) p = add(p, cmul(U.e[j], U.e[N + j]));
  T n1 = 0;
#pragma unroll
  for (int j = 0; j < N; ++j) { U.e[N + j] = sub(U.e[N + j], mul(p, U.e[j])); n1 += norm2(U.e[N + j]); }
  T i1 = T(1.5) - T(0.5) * n1;
  i1 = i1 * (T(1.5) - T(0.5) * n1 * i1 * i1);
  if (fabs(n1 - T(1)) > T(1e-3)) i1 = rsqrt(n1);
#pragma unroll
  for (int j = 0; j < N; ++j) U.e[N + j] = scale(U.e[N + j], i1);
  if (N == 3) {
    U.e[6] = conj(sub(mul(U.e[1], U.e[5]), mul(U.e[2], U.e[4])));
    U.e[7] = conj(sub(mul(U.e[2], U.e[3]), mul(U.e[0], U.e[5])));
    U.e[8] = conj(sub(mul(U.e[0], U.e[4]), mul(U.e[1], U.e[3])));
  }
}

struct DriftArgs {
  const Work* work;
  const LatDev* lats;
  void* U;
  const void* P;
  void* phi;
  void* pi;
  double eps;
  int d;
  int frozen;          // |phi_x| = 1: geodesic (great-circle) drift of (phi, pi)
};
// PROJ: the link update is projected back to SU(N) (the FP32 modes' drift)
template <int N, typename R, typename A, bool PROJ>
__global__ void __launch_bounds__(KBLOCK) k_drift(const DriftArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  if ((int)threadIdx.x >= w.n) return;
  const LatDev L = a.lats[w.lat];
  const int s = w.s0 + threadIdx.x;
  if (!active_site(L, s)) return;
  if (w.mu >= 0) {
    const int mu = w.mu;
    constexpr int ng = N * N - 1;
    const R* P = (const R*)a.P;
    A v[ng];
    const long long pb = p_index(L, ng, mu, 0, s);
    const A eps = (A)a.eps;
#pragma unroll
    for (int g = 0; g < ng; ++g) v[g] = (A)P[pb + g * ULANE] * eps;   // eps P in algebra coefficients
    const Mat<N, A> E = expi<N>(alg_to_mat<N, A>(v));
    const Mat<N, A> Uo = ld_link_rw<N, A>((const R*)a.U, L, mu, s);
    Mat<N, A> Un;
    if constexpr (PROJ) {
      // the projection reads the first N-1 rows of E U and rebuilds the last, so the
      // last row of the product (and of E) is never formed
      mm_core<N, A, false, false, false, N - 1>(E, Uo, Un);
      project_su<N, A>(Un);
    } else {
      Un = mm(E, Uo);
    }
    st_link<N, A>((R*)a.U, L, mu, s, Un);
  } else if (a.frozen) {
    // Frozen length (src/hmc/gauge_higgs_hmc.hpp:84-102): the exact constrained free
    // flow on the unit sphere, r = |pi|:
    //   phi' = cos(r eps) phi + sin(r eps) pi / r,  pi' = -r sin(r eps) phi + cos(r eps) pi.
    // FP64 arithmetic in both precisions; FP32 fields are put back on the sphere
    // (phi' / |phi'|) before they are stored, so that FP32 rounding does not let
    // |phi| wander over many steps.
    R* phi = (R*)a.phi;
    R* pi = (R*)a.pi;
    double r2 = 0.0;
    for (int k = 0; k < a.d; ++k) r2 += norm2(ldc_rw<double>(pi, f_index(L, a.d, k, s)));
    const double r = sqrt(r2);
    if (r < 1e-300) return;
    double sn, c;
    sincos(r * a.eps, &sn, &c);
    const double sr = sn / r, rs = -r * sn;
    double inv = 1.0;
    if (sizeof(R) != sizeof(double)) {
      double n2 = 0.0;
      for (int k = 0; k < a.d; ++k) {
        const long long i = f_index(L, a.d, k, s);
        n2 += norm2(add(scale(ldc_rw<double>(phi, i), c), scale(ldc_rw<double>(pi, i), sr)));
      }
      inv = 1.0 / sqrt(n2);
    }
    for (int k = 0; k < a.d; ++k) {
      const long long i = f_index(L, a.d, k, s);
      const cx<double> f = ldc_rw<double>(phi, i), p = ldc_rw<double>(pi, i);
      stc<double>(phi, i, scale(add(scale(f, c), scale(p, sr)), inv));
      stc<double>(pi, i, add(scale(f, rs), scale(p, c)));
    }
  } else {
    typedef typename Cmp<R>::t C;
    R* phi = (R*)a.phi;
    const R* pi = (const R*)a.pi;
    for (int k = 0; k < a.d; ++k) {
      const long long i = f_index(L, a.d, k, s);
      stc<C>(phi, i, add(ldc_rw<C>(phi, i), scale(ldc<C>(pi, i), (C)a.eps)));
    }
  }
}

// ---------------------------------------------------------------------------
// Frozen-length scalar helpers, one thread per site (src/hmc/gauge_higgs_hmc.hpp:61-82):
//   what 0: pi <- pi - Re(phi^dag pi) phi   (momentum onto the sphere's tangent space)
//   what 1: phi <- phi / |phi|              (put the field on the unit sphere)
// FP64 arithmetic in both precisions.
// ---------------------------------------------------------------------------
struct SphereArgs { const Work* work; const LatDev* lats; void* phi; void* pi; int d; int what; };
template <typename R>
__global__ void __launch_bounds__(KBLOCK) k_sphere(const SphereArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  if ((int)threadIdx.x >= w.n) return;
  const LatDev& L = a.lats[w.lat];
  const int s = w.s0 + threadIdx.x;
  if (!active_site(L, s)) return;
  R* phi = (R*)a.phi;
  R* pi = (R*)a.pi;
  if (a.what == 0) {
    double rp = 0.0;
    for (int k = 0; k < a.d; ++k) {
      const long long i = f_index(L, a.d, k, s);
      const cx<double> f = ldc_rw<double>(phi, i), p = ldc_rw<double>(pi, i);
      rp += f.re * p.re + f.im * p.im;
    }
    for (int k = 0; k < a.d; ++k) {
      const long long i = f_index(L, a.d, k, s);
      stc<double>(pi, i, sub(ldc_rw<double>(pi, i), scale(ldc_rw<double>(phi, i), rp)));
    }
  } else {
    double n2 = 0.0;
    for (int k = 0; k < a.d; ++k) n2 += norm2(ldc_rw<double>(phi, f_index(L, a.d, k, s)));
    if (!(n2 > 0.0)) return;
    const double inv = 1.0 / sqrt(n2);
    for (int k = 0; k < a.d; ++k) {
      const long long i = f_index(L, a.d, k, s);
      stc<double>(phi, i, scale(ldc_rw<double>(phi, i), inv));
    }
  }
}

// Reunitarise all links (src/core/fields.hpp:36, src/group/sun.hpp:48-71), FP64.
struct LinkArgs { const Work* work; const LatDev* lats; void* U; const void* Us; };
template <int N, typename R>
__global__ void __launch_bounds__(KBLOCK) k_reunit(const LinkArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  if ((int)threadIdx.x >= w.n || w.mu < 0) return;
  const LatDev L = a.lats[w.lat];
  const int s = w.s0 + threadIdx.x;
  if (!active_site(L, s)) return;
  Mat<N, double> M = ld_link_rw<N, double>((const R*)a.U, L, w.mu, s);
  reunitarize<N, double>(M);
  st_link<N, double>((R*)a.U, L, w.mu, s, M);
}

// ---------------------------------------------------------------------------
// Measure: one pass over sites producing the six per-site sums behind
// H = 1/2 sum P^2 + 1/2 sum |pi|^2 + S_g + S_H (src/hmc/gauge_higgs_hmc.hpp:105-110)
// and the observables plaquette, L_link, L_phi (src/action/gauge_wilson.hpp:31-65,
// src/action/scalar_higgs.hpp:43-65,132-154), all accumulated in FP64:
//   r0 sum_{mu<nu} Re Tr U_pl   r1 sum V(phi)   r2 sum_mu Re phi_x^dag D phi_{x+mu}
//   r3 sum P^2                  r4 sum |pi|^2   r5 sum |phi|^2
// Warp-shuffle tree reduction, then one partial per block (deterministic order).
// ---------------------------------------------------------------------------
struct MeasArgs {
  const Work* work;
  const LatDev* lats;
  const void* U;
  const void* P;
  const void* phi;
  const void* pi;
  const void* psif;
  int pot;
  double mu2;
  PotA sa;               // multi-invariant potential superoperator (FP64 values)
  const double2* wpot;   // general irreps: w = A(M) phi per site, written by k_gen_links
  int d;
  int scalar;
  double* partials;   // [block][NRED]
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int D, int N, typename R, int REP>
__global__ void __launch_bounds__(KBLOCK) k_measure(const MeasArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  double r[NRED] = {0, 0, 0, 0, 0, 0};
  if ((int)threadIdx.x < w.n && active_site(a.lats[w.lat], w.s0 + (int)threadIdx.x)) {
    const LatDev L = a.lats[w.lat];
    const int s = w.s0 + threadIdx.x;
    const R* U = (const R*)a.U;
    int x[D];
    coords<D>(L, s, x);
    // plaquettes: Re Tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag) = Re Tr(A B^dag)
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
      const int spm = nfwd(L, s, x[mu], mu);
      const Mat<N, double> Umu = ld_link<N, double>(U, L, mu, s);
#pragma unroll
      for (int nu = mu + 1; nu < D; ++nu) {
        const int spn = nfwd(L, s, x[nu], nu);
        const Mat<N, double> A = mm(Umu, ld_link<N, double>(U, L, nu, spm));
        const Mat<N, double> B = mm(ld_link<N, double>(U, L, nu, s), ld_link<N, double>(U, L, mu, spn));
        r[0] += retr_nd(A, B);
      }
    }
    constexpr int ng = N * N - 1;
    const R* P = (const R*)a.P;
#pragma unroll
    for (int mu = 0; mu < D; ++mu)
#pragma unroll
      for (int g = 0; g < ng; ++g) {
        const double p = (double)P[p_index(L, ng, mu, g, s)];
        r[3] += p * p;
      }
    if (a.scalar) {
      const R* phi = (const R*)a.phi;
      const R* pi = (const R*)a.pi;
      double n2 = 0.0;
      for (int k = 0; k < a.d; ++k) {
        n2 += norm2(ldc<double>(phi, f_index(L, a.d, k, s)));
        r[4] += norm2(ldc<double>(pi, f_index(L, a.d, k, s)));
      }
      r[5] = n2;
      if (a.pot != POT_MULTI) {
        r[1] = n2 + L.lambda * (n2 - 1.0) * (n2 - 1.0);
      } else if (REP == REP_GEN) {         // V = -mu2 phi^dag phi + Re(phi^dag w) / 2, w from k_gen_links
        double re = 0.0;
        for (int k = 0; k < a.d; ++k) {
          const cx<double> pk = ldc<double>(phi, f_index(L, a.d, k, s));
          const double2 wk = a.wpot[f_index(L, a.d, k, s)];
          re = fmad(pk.re, wk.x, fmad(pk.im, wk.y, re));
        }
        r[1] = -a.mu2 * n2 + 0.5 * re;
      } else {
        r[1] = pot_multi<double, R>(phi, L, a.d, s, a.sa, a.mu2, nullptr);
      }
      if (REP == REP_FUND || REP == REP_ADJ) {
        constexpr int d = RepDim<N, REP>::d;
        cx<double> px[d], py[d], o[d];
#pragma unroll
        for (int k = 0; k < d; ++k) px[k] = ldc<double>(phi, f_index(L, d, k, s));
#pragma unroll
        for (int mu = 0; mu < D; ++mu) {
          const int y = nfwd(L, s, x[mu], mu);
#pragma unroll
          for (int k = 0; k < d; ++k) py[k] = ldc<double>(phi, f_index(L, d, k, y));
          const Mat<N, double> Umu = ld_link<N, double>(U, L, mu, s);
          if (REP == REP_FUND) fund_apply<N, double>(Umu, py, o, false); else adj_apply<N, double>(Umu, py, o, false);
          double h = 0.0;
#pragma unroll
          for (int k = 0; k < d; ++k) h += px[k].re * o[k].re + px[k].im * o[k].im;
          r[2] += h;
        }
      } else if (REP == REP_GEN) {
        const R* psif = (const R*)a.psif;
#pragma unroll
        for (int mu = 0; mu < D; ++mu) {
          double h = 0.0;
          for (int k = 0; k < a.d; ++k) {
            const cx<double> p = ldc<double>(phi, f_index(L, a.d, k, s));
            const cx<double> o = ldc<double>(psif, g_index(L, a.d, mu, k, s));
            h += p.re * o.re + p.im * o.im;
          }
          r[2] += h;
        }
      }
    }
  }
  __shared__ double red[KBLOCK / 32][NRED];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NRED; ++k) {
    const double v = warp_sum(r[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < NRED) {
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < KBLOCK / 32; ++q) v += red[q][threadIdx.x];
    a.partials[(size_t)blockIdx.x * NRED + threadIdx.x] = v;
  }
}

// Per-lattice totals of the measure partials and the derived quantities.
// res[l][slot][k]: 0 H, 1 S_g, 2 S_H, 3 kin_P, 4 kin_pi, 5 plaquette, 6 L_link, 7 L_phi
constexpr int NRES = 8;
struct FinArgs {
  const LatDev* lats;
  const int* blk_first;   // [nlat+1] block range of each lattice in the measure launch
  const double* partials;
  double* res;
  int slot;               // 0 or 1 (initial / final configuration)
  int D, N;
  int scalar;
};
static __global__ void k_finalize(const FinArgs a) {
  pdl_enter();
  const int l = blockIdx.x;
  const int b0 = a.blk_first[l], b1 = a.blk_first[l + 1];
  __shared__ double sh[NRED][32];
  double v[NRED] = {0, 0, 0, 0, 0, 0};
  for (int b = b0 + (int)threadIdx.x; b < b1; b += 32)
#pragma unroll
    for (int k = 0; k < NRED; ++k) v[k] += a.partials[(size_t)b * NRED + k];
#pragma unroll
  for (int k = 0; k < NRED; ++k) sh[k][threadIdx.x] = v[k];
  __syncwarp();
  if (threadIdx.x == 0) {
    double t[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) { t[k] = 0.0; for (int q = 0; q < 32; ++q) t[k] += sh[k][q]; }
    const LatDev L = a.lats[l];
    const double Vd = (double)L.Vi;              // active sites (all of a lattice that is not decomposed)
    const double nplaq = Vd * (a.D * (a.D - 1) / 2);
    const double Sg = (L.beta / a.N) * ((double)a.N * nplaq - t[0]);
    const double SH = a.scalar ? (t[1] - 2.0 * L.kappa * t[2]) : 0.0;
    const double kP = 0.5 * t[3], kpi = 0.5 * t[4];
    double* o = a.res + ((size_t)l * 2 + a.slot) * NRES;
    o[0] = kP + kpi + Sg + SH;
    o[1] = Sg;
    o[2] = SH;
    o[3] = kP;
    o[4] = kpi;
    o[5] = t[0] / ((double)a.N * nplaq);
    o[6] = a.scalar ? t[2] / (Vd * a.D) : 0.0;
    o[7] = a.scalar ? t[5] / Vd : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Metropolis (src/hmc/gauge_higgs_hmc.hpp:183-191, src/hmc/hmc.hpp:280-287): one
// thread per lattice; dH from the two measure slots, ++traj, coin
// uniform(key(0xE5 | 0xB2, traj)); NaN/Inf dH rejects (as in the reference,
// where every comparison with NaN is false) and is counted.  Appends a record.
// ---------------------------------------------------------------------------
struct TrajRec { double dH; int accepted; int traj; double plaq, L_phi, L_link, kappa, beta; };
struct MetroArgs { LatDev* lats; const double* res; TrajRec* hist; int hist_cap; int nlat; int pure; };
static __global__ void k_metropolis(const MetroArgs a) {
  pdl_enter();
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.nlat) return;
  LatDev& L = a.lats[l];
  const double* r0 = a.res + (size_t)l * 2 * NRES;
  const double* r1 = r0 + NRES;
  const double dH = r1[0] - r0[0];
  L.traj += 1;
  const double u = ghrng::uniform(L.seed, ghrng::key(a.pure ? 0xB2 : 0xE5, L.traj));
  const bool finite = isfinite(dH);
  const int acc = (dH <= 0.0) || (u < exp(-dH));
  if (!finite) L.nonfinite += 1;
  L.last_acc = acc;
  L.accepted += acc;
  if (a.hist && a.hist_cap > 0) {
    TrajRec& h = a.hist[(size_t)l * a.hist_cap + (int)((L.traj - 1) % (unsigned long long)a.hist_cap)];
    const double* ro = acc ? r1 : r0;
    h.dH = dH;
    h.accepted = acc;
    h.traj = (int)L.traj;
    h.plaq = ro[5];
    h.L_phi = ro[7];
    h.L_link = ro[6];
    h.kappa = L.kappa;
    h.beta = L.beta;
  }
}

// Restore the saved configuration of lattices whose trajectory was rejected.
struct RestoreArgs { const Work* work; const LatDev* lats; void* U; const void* Us; void* phi; const void* phis; int N; int d; };
template <typename R>
__global__ void __launch_bounds__(KBLOCK) k_restore(const RestoreArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  if ((int)threadIdx.x >= w.n) return;
  const LatDev& L = a.lats[w.lat];
  if (L.last_acc) return;
  const int s = w.s0 + threadIdx.x;
  typedef typename V2<R>::t V;
  if (w.mu >= 0) {
    const int NN = a.N * a.N;
    const long long b = u_index(L, NN, w.mu, 0, s);
    for (int c = 0; c < NN; ++c) reinterpret_cast<V*>(a.U)[b + c * ULANE] = reinterpret_cast<const V*>(a.Us)[b + c * ULANE];
  } else {
    for (int k = 0; k < a.d; ++k) {
      const long long i = f_index(L, a.d, k, s);
      reinterpret_cast<V*>(a.phi)[i] = reinterpret_cast<const V*>(a.phis)[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Halo planes of a subdomain (src/mpi/gauge_mpi.hpp:101-139): gather (pack) or scatter
// (unpack) every site of the local lattice with x_nu = layer, all components of the
// links (kind 0: D N^2 complex per site) or of phi (kind 1: d complex per site), to or
// from a contiguous buffer [component][plane site], the plane's sites in mixed radix
// over the other directions, direction 0 fastest.  Whole planes, halo sites of the other
// directions included, so that exchanging the split directions one after the other
// also fills the edges and corners, as the reference's sequential exchange does.
// ---------------------------------------------------------------------------
struct HaloArgs {
  const LatDev* lats;
  int lat;
  void* f;              // the field (U or phi)
  void* buf;            // device buffer, ncomp * nplane complex R
  int kind, nu, layer, unpack, D, nn, d;
  long long nplane;
  int ncomp;
};
template <typename R>
__global__ void __launch_bounds__(256) k_halo(const HaloArgs a) {
  typedef typename V2<R>::t V;
  const LatDev& L = a.lats[a.lat];
  const long long total = a.nplane * a.ncomp;
  V* f = reinterpret_cast<V*>(a.f);
  V* b = reinterpret_cast<V*>(a.buf);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(i / a.nplane);
    long long r = i - (long long)comp * a.nplane;
    int s = a.layer * L.stride[a.nu];
    for (int mu = 0; mu < a.D; ++mu) {
      if (mu == a.nu) continue;
      s += (int)(r % L.L[mu]) * L.stride[mu];
      r /= L.L[mu];
    }
    const long long e = a.kind == 0 ? u_index(L, a.nn, comp / a.nn, comp % a.nn, s) : f_index(L, a.d, comp, s);
    if (a.unpack) f[e] = b[i];
    else b[i] = f[e];
  }
}

// ---------------------------------------------------------------------------
// Counter-RNG field initialisation (bit-exact keys of the reference):
//   hot start  U = expi(alg_to_mat(sigma * gauss(key(1, s, mu, a))))  src/core/fields.hpp:25-34
//   momenta    P^a = gauss(key(stream, s, mu, a))                       src/core/fields.hpp:59-66
//   vectors    re = sigma gauss(key(stream, s, 2k)), im = sigma gauss(key(stream, s, 2k+1)) or 0
//                                                                       src/core/scalar_field.hpp:40-50
//   refresh streams key(0xC3|0xA1, traj) and key(0xD4, traj)           src/hmc/gauge_higgs_hmc.hpp:167-173
// ---------------------------------------------------------------------------
struct InitArgs {
  const Work* work;
  const LatDev* lats;
  void* U;
  void* P;
  void* vec;          // phi or pi
  int what;           // 0 hot start, 1 momentum refresh (trajectory keys), 2 vector gaussian
                      // 3 momentum with explicit stream, 4 cold links, 5 cold vector
  int pure;           // pure gauge keys (0xA1) for what == 1
  int real;
  int d;
  double sigma;
  unsigned long long stream;
};
// Gaussian draw for a field stored as R: the correctly rounded draw for FP64
// fields, the CUDA-libm draw for FP32 fields (identical after rounding to FP32
// but for ~1e-8 of draws).
template <typename R> __device__ __forceinline__ double gauss_r(uint64_t seed, uint64_t k) {
  return sizeof(R) == sizeof(double) ? ghrng::gauss(seed, k) : ghrng::gauss_md(seed, k);
}

template <int N, typename R>
__global__ void __launch_bounds__(KBLOCK) k_init(const InitArgs a) {
  pdl_enter();
  typedef typename Cmp<R>::t C;
  const Work w = a.work[blockIdx.x];
  if ((int)threadIdx.x >= w.n) return;
  const LatDev L = a.lats[w.lat];
  const int s = w.s0 + threadIdx.x;
  if (!active_site(L, s)) return;                 // halo sites come from the neighbours
  const long long gs = global_site(L, s);         // the RNG key's site
  constexpr int ng = N * N - 1;
  if (w.mu >= 0) {
    const int mu = w.mu;
    if (a.what == 0 || a.what == 4) {
      Mat<N, double> M;
      if (a.what == 0) {
        double v[ng];
#pragma unroll
        for (int g = 0; g < ng; ++g) v[g] = a.sigma * ghrng::gauss(L.seed, ghrng::key(1, gs, mu, g));
        M = expi<N>(alg_to_mat<N, double>(v));
      } else {
        set_ident(M);
      }
      st_link<N, double>((R*)a.U, L, mu, s, M);
    } else if (a.what == 1 || a.what == 3) {
      const unsigned long long st = (a.what == 1) ? ghrng::key(a.pure ? 0xA1 : 0xC3, L.traj) : a.stream;
      R* P = (R*)a.P;
      const long long pb = p_index(L, ng, mu, 0, s);
#pragma unroll
      for (int g = 0; g < ng; ++g) P[pb + g * ULANE] = (R)gauss_r<R>(L.seed, ghrng::key(st, gs, mu, g));
    }
    return;
  }
  // site items: vectors (pi on refresh, phi on gaussian / cold start)
  if (a.what == 1 && a.pure) return;
  if (a.what == 1 || a.what == 2) {
    const unsigned long long st = (a.what == 1) ? ghrng::key(0xD4, L.traj) : a.stream;
    const double sg = (a.what == 1) ? 1.0 : a.sigma;
    R* vec = (R*)a.vec;
    for (int k = 0; k < a.d; ++k) {
      const double re = sg * gauss_r<R>(L.seed, ghrng::key(st, gs, 2 * k));
      const double im = a.real ? 0.0 : sg * gauss_r<R>(L.seed, ghrng::key(st, gs, 2 * k + 1));
      stc<double>(vec, f_index(L, a.d, k, s), mk<double>(re, im));
    }
  } else if (a.what == 5) {
    R* vec = (R*)a.vec;
    for (int k = 0; k < a.d; ++k) stc<double>(vec, f_index(L, a.d, k, s), mk<double>(k == 0 ? a.sigma : 0.0, 0.0));
  }
}

// ---------------------------------------------------------------------------
// Polyakov loop (src/measure/observables.hpp:17-34): one thread per site with
// x_t = 0, product of the L_t links in direction t, FP64.
// ---------------------------------------------------------------------------
struct PolyArgs { const Work* work; const LatDev* lats; const void* U; int tdir; double* partials; };
template <int D, int N, typename R>
__global__ void __launch_bounds__(KBLOCK) k_polyakov(const PolyArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  double v = 0.0;
  if ((int)threadIdx.x < w.n) {
    const LatDev L = a.lats[w.lat];
    const int s = w.s0 + threadIdx.x;
    int x[D];
    coords<D>(L, s, x);
    if (x[a.tdir] == 0) {
      const int t = a.tdir;
      Mat<N, double> P = ld_link<N, double>((const R*)a.U, L, t, s);
      int cur = s, xt = 0;
      for (int k = 1; k < L.L[t]; ++k) {
        cur = nfwd(L, cur, xt, t);
        ++xt;
        P = mm(P, ld_link<N, double>((const R*)a.U, L, t, cur));
      }
      for (int i = 0; i < N; ++i) v += P.e[i * N + i].re;
    }
  }
  __shared__ double red[KBLOCK / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < KBLOCK / 32; ++q) t += red[q];
    a.partials[blockIdx.x] = t;
  }
}

// ---------------------------------------------------------------------------
// Loops traced in a probe irrep (src/measure/observables.hpp:36-101).
// Re chi_lambda(W) for an SU(N) matrix W and Young rows lambda (m rows): the Schur
// polynomial of W's eigenvalues by Jacobi-Trudi, s_lambda = det[h_{lambda_i - i + j}],
// with the complete symmetric polynomials h_k from the power sums p_k = Tr W^k by
// Newton's identities, k h_k = sum_{i=1}^{k} p_i h_{k-i}.  This is Tr D^(lambda)(W),
// the trace of the representation matrix, without forming it.
// ---------------------------------------------------------------------------
constexpr int CHAR_KMAX = 24;     // largest h index lambda_1 + m - 1
constexpr int CHAR_MMAX = 4;      // most Young rows

template <int N>
__device__ double re_character(const Mat<N, double>& W, const int* lam, int m) {
  const int K = lam[0] + m - 1;
  cx<double> p[CHAR_KMAX + 1], h[CHAR_KMAX + 1];
  Mat<N, double> Wk = W;
  for (int k = 1; k <= K; ++k) {
    if (k > 1) Wk = mm(Wk, W);
    cx<double> t = zero<double>();
    for (int i = 0; i < N; ++i) t = add(t, Wk.e[i * N + i]);
    p[k] = t;
  }
  h[0] = mk<double>(1.0, 0.0);
  for (int k = 1; k <= K; ++k) {
    cx<double> t = zero<double>();
    for (int i = 1; i <= k; ++i) t = cfma(t, p[i], h[k - i]);
    h[k] = scale(t, 1.0 / k);
  }
  cx<double> M[CHAR_MMAX * CHAR_MMAX];
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      const int k = lam[i] - i + j;
      M[i * m + j] = (k < 0) ? zero<double>() : h[k];
    }
  // determinant by elimination with partial pivoting (m <= 4)
  cx<double> det = mk<double>(1.0, 0.0);
  for (int c = 0; c < m; ++c) {
    int piv = c;
    for (int r = c + 1; r < m; ++r)
      if (norm2(M[r * m + c]) > norm2(M[piv * m + c])) piv = r;
    if (norm2(M[piv * m + c]) == 0.0) return 0.0;
    if (piv != c) {
      for (int j = 0; j < m; ++j) { const cx<double> t = M[c * m + j]; M[c * m + j] = M[piv * m + j]; M[piv * m + j] = t; }
      det = scale(det, -1.0);
    }
    det = mul(det, M[c * m + c]);
    const cx<double> inv = scale(conj(M[c * m + c]), 1.0 / norm2(M[c * m + c]));
    for (int r = c + 1; r < m; ++r) {
      const cx<double> f = mul(M[r * m + c], inv);
      for (int j = c; j < m; ++j) M[r * m + j] = sub(M[r * m + j], mul(f, M[c * m + j]));
    }
  }
  return det.re;
}

// mode 0: Polyakov line in direction tdir from every site with x_tdir = 0;
// mode 1: the Ra x Rb rectangle of every plane mu < nu based at every site
//         (path order of wilson_rect, src/measure/observables.hpp:36-46).
// Per block: sum over its sites of Re chi(loop), into partials (FP64).
struct LoopArgs {
  const Work* work; const LatDev* lats; const void* U; double* partials;
  int mode, tdir, Ra, Rb, m; int lam[CHAR_MMAX];
};
template <int D, int N, typename R>
__global__ void __launch_bounds__(KBLOCK) k_loops(const LoopArgs a) {
  pdl_enter();
  const Work w = a.work[blockIdx.x];
  double v = 0.0;
  if ((int)threadIdx.x < w.n) {
    const LatDev L = a.lats[w.lat];
    const int s = w.s0 + threadIdx.x;
    const R* U = (const R*)a.U;
    int x0[D];
    coords<D>(L, s, x0);
    if (a.mode == 0) {
      if (x0[a.tdir] == 0) {
        const int t = a.tdir;
        Mat<N, double> P = ld_link<N, double>(U, L, t, s);
        int cur = s, xt = 0;
        for (int k = 1; k < L.L[t]; ++k) {
          cur = nfwd(L, cur, xt, t);
          ++xt;
          P = mm(P, ld_link<N, double>(U, L, t, cur));
        }
        v = re_character<N>(P, a.lam, a.m);
      }
    } else {
      for (int mu = 0; mu < D; ++mu)
        for (int nu = mu + 1; nu < D; ++nu) {
          int x[D];
          for (int q = 0; q < D; ++q) x[q] = x0[q];
          int c = s;
          Mat<N, double> W = ld_link<N, double>(U, L, mu, c);
          c = nfwd(L, c, x[mu], mu); x[mu] = (x[mu] + 1 == L.L[mu]) ? 0 : x[mu] + 1;
          for (int i = 1; i < a.Ra; ++i) {
            W = mm(W, ld_link<N, double>(U, L, mu, c));
            c = nfwd(L, c, x[mu], mu); x[mu] = (x[mu] + 1 == L.L[mu]) ? 0 : x[mu] + 1;
          }
          for (int j = 0; j < a.Rb; ++j) {
            W = mm(W, ld_link<N, double>(U, L, nu, c));
            c = nfwd(L, c, x[nu], nu); x[nu] = (x[nu] + 1 == L.L[nu]) ? 0 : x[nu] + 1;
          }
          for (int i = 0; i < a.Ra; ++i) {
            c = nbwd(L, c, x[mu], mu); x[mu] = (x[mu] == 0) ? L.L[mu] - 1 : x[mu] - 1;
            W = mm_nd(W, ld_link<N, double>(U, L, mu, c));
          }
          for (int j = 0; j < a.Rb; ++j) {
            c = nbwd(L, c, x[nu], nu); x[nu] = (x[nu] == 0) ? L.L[nu] - 1 : x[nu] - 1;
            W = mm_nd(W, ld_link<N, double>(U, L, nu, c));
          }
          v += re_character<N>(W, a.lam, a.m);
        }
    }
  }
  __shared__ double red[KBLOCK / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < KBLOCK / 32; ++q) t += red[q];
    a.partials[blockIdx.x] = t;
  }
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference's AoS host arrays (FP64) and the
// device SoA planes (R).  kind: 0 links (N*N complex per (site,mu)),
// 1 momenta (ng reals per (site,mu)), 2 vectors (d complex per site).
// ---------------------------------------------------------------------------
struct XferArgs { const LatDev* lats; int lat; int kind; int D; int ncomp; double* host_aos; void* dev; int to_dev; };
template <typename R>
__global__ void k_xfer(const XferArgs a) {
  pdl_enter();
  const LatDev L = a.lats[a.lat];
  const long long per_site = (a.kind == 2) ? a.ncomp : (long long)a.D * a.ncomp;
  const long long total = (long long)L.V * per_site;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / per_site);
    const int r = (int)(e % per_site);
    if (a.kind == 1) {
      const long long di = p_index(L, a.ncomp, r / a.ncomp, r % a.ncomp, s);   // r = mu*ng + g
      R* P = (R*)a.dev;
      if (a.to_dev) P[di] = (R)a.host_aos[e]; else a.host_aos[e] = (double)P[di];
    } else {
      // r = mu*NN + c (links) or k (vectors)
      const long long di = (a.kind == 0) ? u_index(L, a.ncomp, r / a.ncomp, r % a.ncomp, s) : f_index(L, a.ncomp, r, s);
      if (a.to_dev) stc<double>((R*)a.dev, di, mk<double>(a.host_aos[2 * e], a.host_aos[2 * e + 1]));
      else { const cx<double> z = ldc_rw<double>((const R*)a.dev, di); a.host_aos[2 * e] = z.re; a.host_aos[2 * e + 1] = z.im; }
    }
  }
}

}  // namespace ghk
