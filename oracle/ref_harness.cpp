// ref_harness.cpp -- C entry points over the UNMODIFIED reference headers.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the reference
// source tree (its src/ directory, read-only) into oracle/_ref/libghref*.so.
// Nothing here restates the reference: every entry point constructs the
// reference's own objects (GaugeHiggsHMC, GaugeHMC, GaugeField, LinkMom,
// CVecField, FundamentalRep / AdjointRep / GeneralRep) and calls their methods,
// copying AoS arrays in and out.  Used to (1) pin the C restatement in
// oracle/gh_oracle.c, (2) generate tests/golden fixtures, (3) time the
// reference CPU path for bench.py's reference arm.
#include "hmc/gauge_higgs_hmc.hpp"
#include "hmc/hmc.hpp"
#include "measure/observables.hpp"
#include "rep/rep_fundamental.hpp"
#include "rep/rep_adjoint.hpp"
#include "rep/rep_general.hpp"
#include "action/scalar_invariants.hpp"
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace gh;

namespace {

// Representation factory with the reference driver's spec syntax
// (src/hmc_higgs.cpp:23-34), cached per (N, spec).
template <int N>
const Representation<N>* get_rep(const std::string& spec0) {
  static std::map<std::string, std::unique_ptr<Representation<N>>> cache;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(spec0);
  if (it != cache.end()) return it->second.get();
  std::unique_ptr<Representation<N>> r;
  std::string spec = spec0;
  if (spec == "fund") r = std::make_unique<FundamentalRep<N>>();
  else if (spec == "adj") r = std::make_unique<AdjointRep<N>>();
  else {
    bool real = false;
    const auto colon = spec.find(':');
    if (colon != std::string::npos) { real = (spec.substr(colon + 1) == "real"); spec = spec.substr(0, colon); }
    std::vector<int> rows; std::stringstream ss(spec); std::string tok;
    while (std::getline(ss, tok, ',')) if (!tok.empty()) rows.push_back(std::atoi(tok.c_str()));
    if (rows.empty()) return nullptr;
    r = std::make_unique<GeneralRep<N>>(rows, real ? GeneralRep<N>::RealType::Real : GeneralRep<N>::RealType::Complex);
  }
  const Representation<N>* p = r.get();
  cache[spec0] = std::move(r);
  return p;
}

template <int D> std::array<int, D> ext(const int* L) { std::array<int, D> e{}; for (int m = 0; m < D; ++m) e[m] = L[m]; return e; }

template <int N> void load_mat(Cmat<N>& M, const double* p) { for (int i = 0; i < N * N; ++i) M.a[i] = Complex(p[2 * i], p[2 * i + 1]); }
template <int N> void store_mat(const Cmat<N>& M, double* p) { for (int i = 0; i < N * N; ++i) { p[2 * i] = M.a[i].real(); p[2 * i + 1] = M.a[i].imag(); } }

template <int D, int N> void load_U(GaugeField<D, N>& U, const double* p) { for (std::size_t l = 0; l < U.u.size(); ++l) load_mat<N>(U.u[l], p + 2 * l * N * N); }
template <int D, int N> void store_U(const GaugeField<D, N>& U, double* p) { for (std::size_t l = 0; l < U.u.size(); ++l) store_mat<N>(U.u[l], p + 2 * l * N * N); }
template <int D, int N> void load_P(LinkMom<D, N>& P, const double* p) { for (std::size_t l = 0; l < P.p.size(); ++l) for (int a = 0; a < N * N - 1; ++a) P.p[l][a] = p[l * (N * N - 1) + a]; }
template <int D, int N> void store_P(const LinkMom<D, N>& P, double* p) { for (std::size_t l = 0; l < P.p.size(); ++l) for (int a = 0; a < N * N - 1; ++a) p[l * (N * N - 1) + a] = P.p[l][a]; }
template <int D> void load_V(CVecField<D>& f, const double* p) { for (std::size_t i = 0; i < f.data.size(); ++i) f.data[i] = Complex(p[2 * i], p[2 * i + 1]); }
template <int D> void store_V(const CVecField<D>& f, double* p) { for (std::size_t i = 0; i < f.data.size(); ++i) { p[2 * i] = f.data[i].real(); p[2 * i + 1] = f.data[i].imag(); } }

DVec load_dvec(int d, const double* p) { DVec v(d); for (int k = 0; k < d; ++k) v(k) = Complex(p[2 * k], p[2 * k + 1]); return v; }
void store_dvec(const DVec& v, double* p) { for (int k = 0; k < v.size(); ++k) { p[2 * k] = v(k).real(); p[2 * k + 1] = v(k).imag(); } }

}  // namespace

#define DISPATCH_N(N, CALL) \
  switch (N) { case 2: { constexpr int NN_ = 2; CALL(NN_); } case 3: { constexpr int NN_ = 3; CALL(NN_); } default: return -1; }
#define DISPATCH_DN(D, N, CALL) \
  if (D == 2 && N == 2) { CALL(2, 2); } else if (D == 3 && N == 2) { CALL(3, 2); } else if (D == 4 && N == 2) { CALL(4, 2); } \
  else if (D == 2 && N == 3) { CALL(2, 3); } else if (D == 3 && N == 3) { CALL(3, 3); } else if (D == 4 && N == 3) { CALL(4, 3); } \
  return -1;

extern "C" {

int ref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n; return 1;
#endif
}

uint64_t ref_key(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e) { return Rng::key(a, b, c, d, e); }
double ref_uniform(uint64_t seed, uint64_t k) { return Rng(seed).uniform(k); }
double ref_gauss(uint64_t seed, uint64_t k) { return Rng(seed).gauss(k); }
void ref_gauss_many(uint64_t seed, const uint64_t* keys, int64_t n, double* out) { Rng r(seed); for (int64_t i = 0; i < n; ++i) out[i] = r.gauss(keys[i]); }
void ref_uniform_many(uint64_t seed, const uint64_t* keys, int64_t n, double* out) { Rng r(seed); for (int64_t i = 0; i < n; ++i) out[i] = r.uniform(keys[i]); }

// ---- representation tables and per-link operations ----
int ref_rep_info(int N, const char* spec, int* d, int* real, int* nboxes, long* dimT, int* use_fast) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; *d = r->d; *real = r->real; \
    auto* g = dynamic_cast<const GeneralRep<NN>*>(r); *nboxes = g ? g->n : 0; *dimT = g ? g->dimT : 0; \
    *use_fast = g ? (int)g->use_fast : 0; return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
// T: [N^2-1][d][d] complex; W: [d][dimT] complex (general reps only; may be null)
int ref_rep_tables(int N, const char* spec, double* T, double* W) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; const int d = r->d; \
    for (int a = 0; a < NN * NN - 1; ++a) for (int i = 0; i < d * d; ++i) { \
      T[2 * ((size_t)a * d * d + i)] = r->T[a].a[i].real(); T[2 * ((size_t)a * d * d + i) + 1] = r->T[a].a[i].imag(); } \
    auto* g = dynamic_cast<const GeneralRep<NN>*>(r); \
    if (g && W) for (int l = 0; l < d; ++l) for (long i = 0; i < g->dimT; ++i) { \
      W[2 * ((size_t)l * g->dimT + i)] = g->W[l][i].real(); W[2 * ((size_t)l * g->dimT + i) + 1] = g->W[l][i].imag(); } \
    return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
int ref_rep_matrix(int N, const char* spec, const double* U, double* Dm) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; Cmat<NN> M; load_mat<NN>(M, U); \
    DMat R = r->rep_matrix(M); for (std::size_t i = 0; i < R.a.size(); ++i) { Dm[2 * i] = R.a[i].real(); Dm[2 * i + 1] = R.a[i].imag(); } return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
int ref_rep_rotate(int N, const char* spec, const double* U, const double* phi, double* out, int dag) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; Cmat<NN> M; load_mat<NN>(M, U); \
    DVec v = load_dvec(r->d, phi); store_dvec(dag ? r->rotate_dag(M, v) : r->rotate(M, v), out); return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
int ref_rep_hop(int N, const char* spec, const double* U, const double* phix, const double* phiy, double* g) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; Cmat<NN> M; load_mat<NN>(M, U); \
    auto gg = r->hop_link_g(M, load_dvec(r->d, phix), load_dvec(r->d, phiy)); for (int a = 0; a < NN * NN - 1; ++a) g[a] = gg[a]; return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}

// ---- group ----
int ref_expi(int N, const double* H, double* U) {
#define CALL(NN) { Cmat<NN> M; load_mat<NN>(M, H); store_mat<NN>(expi<NN>(M), U); return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
int ref_reunitarize(int N, double* U) {
#define CALL(NN) { Cmat<NN> M; load_mat<NN>(M, U); reunitarize<NN>(M); store_mat<NN>(M, U); return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
int ref_generators(int N, double* T) {
#define CALL(NN) { const auto& g = generators<NN>(); for (int a = 0; a < NN * NN - 1; ++a) store_mat<NN>(g.T[a], T + 2 * a * NN * NN); return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}

// ---- field initialisation ----
int ref_hot_start(int D, int N, const int* L, uint64_t seed, double sigma, double* U) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); G.hot(Rng(seed), sigma); store_U(G, U); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
int ref_mom_refresh(int D, int N, const int* L, uint64_t seed, uint64_t stream, double* P) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); LinkMom<DD, NN> M(lat); M.refresh(Rng(seed), stream); store_P(M, P); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
int ref_phi_gaussian(int D, const int* L, int d, uint64_t seed, uint64_t stream, int real, double sigma, double* phi) {
#define CALLD(DD) { Lattice<DD> lat(ext<DD>(L)); CVecField<DD> f(lat, d); f.gaussian(Rng(seed), stream, real != 0, sigma); store_V(f, phi); return 0; }
  if (D == 2) CALLD(2) else if (D == 3) CALLD(3) else if (D == 4) CALLD(4)
#undef CALLD
  return -1;
}

// ---- actions / forces / observables ----
double ref_gauge_action(int D, int N, const int* L, const double* U, double beta) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); return gauge_action<DD, NN>(G, beta); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
double ref_avg_plaquette(int D, int N, const int* L, const double* U) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); return avg_plaquette<DD, NN>(G); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
double ref_polyakov(int D, int N, const int* L, const double* U, int tdir) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); return polyakov_loop<DD, NN>(G, tdir); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
int ref_gauge_force(int D, int N, const int* L, const double* U, double beta, double* F) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); LinkMom<DD, NN> Fm(lat); Fm.zero(); \
    add_gauge_force<DD, NN>(G, beta, Fm); store_P(Fm, F); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
int ref_matter_force(int D, int N, const int* L, const char* spec, const double* U, const double* phi, double kappa, double* F) {
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    CVecField<DD> f(lat, r->d); load_V(f, phi); LinkMom<DD, NN> Fm(lat); Fm.zero(); \
    add_matter_link_force<DD, NN>(f, G, *r, kappa, Fm); store_P(Fm, F); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
int ref_scalar_force(int D, int N, const int* L, const char* spec, const double* U, const double* phi, double kappa, double lambda, double* Fphi) {
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    CVecField<DD> f(lat, r->d); load_V(f, phi); CVecField<DD> Fp(lat, r->d); \
    scalar_force<DD, NN>(f, G, *r, kappa, lambda, Fp); store_V(Fp, Fphi); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
double ref_scalar_action(int D, int N, const int* L, const char* spec, const double* U, const double* phi, double kappa, double lambda) {
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return 0.0 / 0.0; Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    CVecField<DD> f(lat, r->d); load_V(f, phi); return scalar_action<DD, NN>(f, G, *r, kappa, lambda); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
double ref_link_energy(int D, int N, const int* L, const char* spec, const double* U, const double* phi) {
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return 0.0 / 0.0; Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    CVecField<DD> f(lat, r->d); load_V(f, phi); return link_energy<DD, NN>(f, G, *r); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}

// ---- loops traced in a probe irrep (src/measure/observables.hpp:36-101) ----
double ref_wilson_loop(int D, int N, const int* L, const char* spec, const double* U, int Ra, int Rb) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    if (std::strcmp(spec, "fund0") == 0) return wilson_loop_fund<DD, NN>(G, Ra, Rb); \
    auto* r = get_rep<NN>(spec); if (!r) return 0.0 / 0.0; return wilson_loop_rep<DD, NN>(G, *r, Ra, Rb); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
double ref_polyakov_rep(int D, int N, const int* L, const char* spec, const double* U, int tdir) {
#define CALL(DD, NN) { Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    auto* r = get_rep<NN>(spec); if (!r) return 0.0 / 0.0; return polyakov_loop_rep<DD, NN>(G, *r, tdir); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}

// ---- multi-invariant onsite potential (src/action/scalar_invariants.hpp) ----
// Channels: the distinct adjoint-Casimir eigenvalues of R (x) Rbar, in the
// reference's order; returns their number (-1: bad N / spec).
int ref_casimir_channels(int N, const char* spec, double* c2, int cap) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; CasimirChannels<NN> ch(*r); \
    const int n = ch.n_channels(); for (int c = 0; c < n && c < cap; ++c) c2[c] = ch.lambda[c]; return n; }
  DISPATCH_N(N, CALL)
#undef CALL
}
// The combined superoperator sum_c 2 f_c P_c as built by MultiInvariantPotential:
// A[(p*d+q)*d*d + (i*d+j)] complex.
int ref_multi_superop(int N, const char* spec, const double* f, int nf, double mu2, double* A) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; CasimirChannels<NN> ch(*r); \
    if (nf != ch.n_channels()) return -3; MultiInvariantPotential<NN> pot(ch, std::vector<Real>(f, f + nf), mu2); \
    for (std::size_t k = 0; k < pot.Asuper.size(); ++k) { A[2 * k] = pot.Asuper[k].real(); A[2 * k + 1] = pot.Asuper[k].imag(); } \
    return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
// V(phi) and dV/dphibar of one d-vector.
int ref_multi_value_dV(int N, const char* spec, const double* f, int nf, double mu2, const double* phi, double* value, double* g) {
#define CALL(NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; CasimirChannels<NN> ch(*r); \
    if (nf != ch.n_channels()) return -3; MultiInvariantPotential<NN> pot(ch, std::vector<Real>(f, f + nf), mu2); \
    const DVec v = load_dvec(r->d, phi); *value = pot.value(v); store_dvec(pot.dV_dphibar(v), g); return 0; }
  DISPATCH_N(N, CALL)
#undef CALL
}
int ref_scalar_force_multi(int D, int N, const int* L, const char* spec, const double* U, const double* phi, double kappa,
                           const double* f, int nf, double mu2, double* Fphi) {
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return -2; CasimirChannels<NN> ch(*r); \
    if (nf != ch.n_channels()) return -3; MultiInvariantPotential<NN> pot(ch, std::vector<Real>(f, f + nf), mu2); \
    Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    CVecField<DD> fl(lat, r->d); load_V(fl, phi); CVecField<DD> Fp(lat, r->d); \
    scalar_force<DD, NN>(fl, G, *r, kappa, pot, Fp); store_V(Fp, Fphi); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}
double ref_scalar_action_multi(int D, int N, const int* L, const char* spec, const double* U, const double* phi, double kappa,
                               const double* f, int nf, double mu2) {
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return 0.0 / 0.0; CasimirChannels<NN> ch(*r); \
    if (nf != ch.n_channels()) return 0.0 / 0.0; MultiInvariantPotential<NN> pot(ch, std::vector<Real>(f, f + nf), mu2); \
    Lattice<DD> lat(ext<DD>(L)); GaugeField<DD, NN> G(lat); load_U(G, U); \
    CVecField<DD> fl(lat, r->d); load_V(fl, phi); return scalar_action<DD, NN>(fl, G, *r, kappa, pot); }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}

// ---- HMC state operations on caller buffers ----
// op: 0 kick(eps) 1 drift(eps) 2 md_evolve 3 hamiltonian 4 refresh_momenta 5 trajectory
//     6 reunitarize_all
// out[0] = H (op 3) / dH (op 5); out[1] = accepted (op 5); out[2] = new traj_count (op 5)
// spec == "none" selects the pure-gauge GaugeHMC (src/hmc/hmc.hpp).
int ref_hmc_op(int op, int D, int N, const int* L, const char* spec, uint64_t seed,
               double beta, double kappa, double lambda, double tau, int nmd, int integ,
               double eps, uint64_t traj_count, double* U, double* P, double* phi, double* pi, double* out) {
  const bool pure = std::strcmp(spec, "none") == 0;
#define CALL(DD, NN) { \
    if (pure) { GaugeHMC<DD, NN> h(ext<DD>(L), seed); h.beta = beta; h.tau = tau; h.nmd = nmd; \
      h.integ = integ == 0 ? Integrator::Leapfrog : Integrator::Omelyan2MN; h.traj_count = traj_count; \
      load_U(h.U, U); load_P(h.P, P); \
      switch (op) { case 0: h.kick(eps); break; case 1: h.drift(eps); break; case 2: h.md_evolve(); break; \
        case 3: out[0] = h.hamiltonian(); break; \
        case 4: h.P.refresh(h.rng, Rng::key(0xA1, h.traj_count)); break; \
        case 5: { bool a = h.trajectory(); out[0] = h.last_dH; out[1] = a; out[2] = (double)h.traj_count; break; } \
        case 6: h.U.reunitarize_all(); break; default: return -3; } \
      store_U(h.U, U); store_P(h.P, P); return 0; } \
    auto* r = get_rep<NN>(spec); if (!r) return -2; \
    GaugeHiggsHMC<DD, NN> h(ext<DD>(L), *r, seed); h.beta = beta; h.kappa = kappa; h.lambda = lambda; h.tau = tau; h.nmd = nmd; \
    h.integ = integ == 0 ? Integrator::Leapfrog : Integrator::Omelyan2MN; h.traj_count = traj_count; \
    load_U(h.U, U); load_P(h.P, P); load_V(h.phi, phi); load_V(h.pi, pi); \
    switch (op) { case 0: h.kick(eps); break; case 1: h.drift(eps); break; case 2: h.md_evolve(); break; \
      case 3: out[0] = h.hamiltonian(); break; case 4: h.refresh_momenta(); break; \
      case 5: { bool a = h.trajectory(); out[0] = h.last_dH; out[1] = a; out[2] = (double)h.traj_count; break; } \
      case 6: h.U.reunitarize_all(); break; default: return -3; } \
    store_U(h.U, U); store_P(h.P, P); store_V(h.phi, phi); store_V(h.pi, pi); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}

// Frozen-length scalar (GaugeHiggsHMC::frozen_phi = true): op 0 kick, 1 drift,
// 2 md_evolve, 3 hamiltonian, 4 refresh_momenta, 5 trajectory, 7 normalize_phi.
int ref_hmc_op_frozen(int op, int D, int N, const int* L, const char* spec, uint64_t seed,
                      double beta, double kappa, double lambda, double tau, int nmd, int integ,
                      double eps, uint64_t traj_count, double* U, double* P, double* phi, double* pi, double* out) {
#define CALL(DD, NN) { \
    auto* r = get_rep<NN>(spec); if (!r) return -2; \
    GaugeHiggsHMC<DD, NN> h(ext<DD>(L), *r, seed); h.beta = beta; h.kappa = kappa; h.lambda = lambda; h.tau = tau; h.nmd = nmd; \
    h.integ = integ == 0 ? Integrator::Leapfrog : Integrator::Omelyan2MN; h.traj_count = traj_count; h.frozen_phi = true; \
    load_U(h.U, U); load_P(h.P, P); load_V(h.phi, phi); load_V(h.pi, pi); \
    switch (op) { case 0: h.kick(eps); break; case 1: h.drift(eps); break; case 2: h.md_evolve(); break; \
      case 3: out[0] = h.hamiltonian(); break; case 4: h.refresh_momenta(); break; \
      case 5: { bool a = h.trajectory(); out[0] = h.last_dH; out[1] = a; out[2] = (double)h.traj_count; break; } \
      case 7: h.normalize_phi(); break; default: return -3; } \
    store_U(h.U, U); store_P(h.P, P); store_V(h.phi, phi); store_V(h.pi, pi); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}

// ---- the driver loop of src/hmc_higgs.cpp:64-87 / src/main.cpp:26-42 ----
// series: [nmeas][5] = plaquette, L_phi, L_link, Polyakov, dH (pure gauge: L_phi = L_link = 0)
// U0/phi0: optional start configuration (null => hot(hot_sigma) and gaussian(12345, phi_sigma))
int ref_run(int D, int N, const int* L, const char* spec, double beta, double kappa, double lambda,
            int ntherm, int nmeas, int nmd, double tau, uint64_t seed, int integ,
            double hot_sigma, double phi_sigma, double* series, double* acc) {
  const bool pure = std::strcmp(spec, "none") == 0;
#define CALL(DD, NN) { \
    if (pure) { GaugeHMC<DD, NN> h(ext<DD>(L), seed); h.beta = beta; h.tau = tau; h.nmd = nmd; \
      h.integ = integ == 0 ? Integrator::Leapfrog : Integrator::Omelyan2MN; h.U.hot(h.rng, hot_sigma); \
      for (int t = 0; t < ntherm; ++t) { h.trajectory(); } h.traj_count = 0; h.accept_count = 0; \
      for (int t = 0; t < nmeas; ++t) { h.trajectory(); double* o = series + 5 * t; o[0] = avg_plaquette<DD, NN>(h.U); \
        o[1] = 0; o[2] = 0; o[3] = polyakov_loop<DD, NN>(h.U); o[4] = h.last_dH; } \
      *acc = h.acceptance(); return 0; } \
    auto* r = get_rep<NN>(spec); if (!r) return -2; \
    GaugeHiggsHMC<DD, NN> h(ext<DD>(L), *r, seed); h.beta = beta; h.kappa = kappa; h.lambda = lambda; h.tau = tau; h.nmd = nmd; \
    h.integ = integ == 0 ? Integrator::Leapfrog : Integrator::Omelyan2MN; \
    h.U.hot(h.rng, hot_sigma); h.phi.gaussian(h.rng, 12345, r->real, phi_sigma); \
    for (int t = 0; t < ntherm; ++t) { h.trajectory(); } h.traj_count = 0; h.accept_count = 0; \
    for (int t = 0; t < nmeas; ++t) { h.trajectory(); double* o = series + 5 * t; o[0] = avg_plaquette<DD, NN>(h.U); \
      o[1] = higgs_length<DD>(h.phi); o[2] = link_energy<DD, NN>(h.phi, h.U, *r); o[3] = polyakov_loop<DD, NN>(h.U); o[4] = h.last_dH; } \
    *acc = h.acceptance(); return 0; }
  DISPATCH_DN(D, N, CALL)
#undef CALL
}

}  // extern "C"

// ---- a persistent reference HMC object: the reference driver's own loop of
// GaugeHiggsHMC::trajectory() (src/hmc_higgs.cpp:72-87), one call per step ----
struct RefSession {
  virtual ~RefSession() {}
  virtual int run(int ntraj, double* series) = 0;   // series: [ntraj][5] as ref_run
  virtual double acceptance() = 0;
  virtual int set_multi(const double* f, int nf, double mu2) = 0;   // nf must equal the channel count
  virtual void set_frozen(int on) = 0;                               // |phi_x| = 1, as GH_FROZEN
};
template <int DD, int NN>
struct RefSessionT : RefSession {
  const Representation<NN>* r;
  GaugeHiggsHMC<DD, NN> h;
  RefSessionT(const int* L, const Representation<NN>* rep, uint64_t seed) : r(rep), h(ext<DD>(L), *rep, seed) {}
  int run(int ntraj, double* series) override {
    for (int t = 0; t < ntraj; ++t) {
      h.trajectory();
      if (series) {
        double* o = series + 5 * t;
        o[0] = avg_plaquette<DD, NN>(h.U); o[1] = higgs_length<DD>(h.phi); o[2] = link_energy<DD, NN>(h.phi, h.U, *r);
        o[3] = polyakov_loop<DD, NN>(h.U); o[4] = h.last_dH;
      }
    }
    return 0;
  }
  double acceptance() override { return h.acceptance(); }
  // the reference driver's potential set-up (src/hmc_higgs_multi.cpp:51-80)
  std::unique_ptr<CasimirChannels<NN>> ch;
  std::unique_ptr<MultiInvariantPotential<NN>> pot;
  int set_multi(const double* f, int nf, double mu2) override {
    ch.reset(new CasimirChannels<NN>(*r));
    if (nf != ch->n_channels()) return -3;
    pot.reset(new MultiInvariantPotential<NN>(*ch, std::vector<Real>(f, f + nf), mu2));
    h.potential = pot.get();
    return 0;
  }
  // the driver's GH_FROZEN set-up (src/hmc_higgs_multi.cpp:81-82,90)
  void set_frozen(int on) override {
    h.frozen_phi = on != 0;
    if (on) h.normalize_phi();
  }
};

extern "C" {

void* ref_session_create(int D, int N, const int* L, const char* spec, double beta, double kappa, double lambda,
                         int nmd, double tau, uint64_t seed, int integ, double hot_sigma, double phi_sigma) {
  RefSession* s = nullptr;
#define CALL(DD, NN) { auto* r = get_rep<NN>(spec); if (!r) return nullptr; auto* t = new RefSessionT<DD, NN>(L, r, seed); \
    t->h.beta = beta; t->h.kappa = kappa; t->h.lambda = lambda; t->h.nmd = nmd; t->h.tau = tau; \
    t->h.integ = integ == 0 ? Integrator::Leapfrog : Integrator::Omelyan2MN; \
    t->h.U.hot(t->h.rng, hot_sigma); t->h.phi.gaussian(t->h.rng, 12345, r->real, phi_sigma); s = t; }
  if (D == 4 && N == 3) CALL(4, 3) else if (D == 4 && N == 2) CALL(4, 2) else if (D == 3 && N == 3) CALL(3, 3) else if (D == 3 && N == 2) CALL(3, 2)
#undef CALL
  return s;
}
int ref_session_run(void* s, int ntraj, double* series) { return s ? static_cast<RefSession*>(s)->run(ntraj, series) : -1; }
int ref_session_set_multi(void* s, const double* f, int nf, double mu2) {
  return s ? static_cast<RefSession*>(s)->set_multi(f, nf, mu2) : -1;
}
void ref_session_set_frozen(void* s, int on) { if (s) static_cast<RefSession*>(s)->set_frozen(on); }
double ref_session_acceptance(void* s) { return s ? static_cast<RefSession*>(s)->acceptance() : 0.0; }
void ref_session_destroy(void* s) { delete static_cast<RefSession*>(s); }

}  // extern "C"
