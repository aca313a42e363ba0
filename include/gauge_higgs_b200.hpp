// gauge_higgs_b200.hpp -- C++ host interface over the C ABI (gauge_higgs_b200.h).
//
// Mirrors the reference's host-side interface (hlammiv/gauge_higgs) so a driver
// written against it switches by changing includes and the namespace:
//   Representation objects   src/rep/representation.hpp:12-32 (FundamentalRep,
//                            AdjointRep, GeneralRep from Young rows, make_rep spec syntax
//                            of src/hmc_higgs.cpp:21-34)
//   GaugeHiggsHMC<D,N>       src/hmc/gauge_higgs_hmc.hpp:15-195: public couplings
//                            beta/kappa/lambda/tau/nmd/integ, traj_count/accept_count,
//                            last_dH; kick, drift, md_evolve, hamiltonian,
//                            refresh_momenta, trajectory, acceptance
//   GaugeHMC<D,N>            src/hmc/hmc.hpp:12-96 (pure gauge)
//   observables              avg_plaquette, higgs_length, link_energy, polyakov_loop
//   Stats                    src/measure/observables.hpp:104-145
//   CasimirChannels, MultiInvariantPotential   src/action/scalar_invariants.hpp:19-206
//   ReplicaTempering<D,N>    src/hmc/replica_tempering.hpp (parallel tempering in beta)
// Fields live on the GPU; U()/phi() copy them to host vectors in the reference's
// layouts.  Errors throw std::runtime_error, as the reference does.
#pragma once
#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <sstream>
#include <stdexcept>
#include <string>
#include <numeric>
#include <vector>
#include "gauge_higgs_b200.h"

namespace ghb {

inline void check(int rc, const gh_ctx* ctx) {
  if (rc != GH_OK) throw std::runtime_error(std::string("gauge_higgs_b200: ") + gh_last_error(ctx));
}

enum class Integrator { Leapfrog, Omelyan2MN };
enum class Precision { FP64 = GH_PREC_FP64, FP32_MD = GH_PREC_FP32_MD, FP32_ALL = GH_PREC_FP32_ALL };

// ---- representations ----
struct Representation {
  int kind = GH_REP_NONE, N = 0, d = 0, real = 0, n_boxes = 0, nality = 0;
  long dimT = 0;
  std::vector<double> T, W;   // complex interleaved (GENERAL only)
  std::vector<int> rows;      // Young rows of the irrep
  std::string repname;
  std::string name() const { return repname; }
  gh_rep_desc desc() const {
    gh_rep_desc r{};
    r.kind = kind; r.d = d; r.real = real; r.n_boxes = n_boxes; r.dimT = dimT;
    r.T = T.empty() ? nullptr : T.data();
    r.W = W.empty() ? nullptr : W.data();
    return r;
  }
};

template <int N> Representation FundamentalRep() {
  Representation r; r.kind = GH_REP_FUND; r.N = N; r.d = N; r.real = 0; r.nality = 1; r.repname = "fundamental";
  r.rows = {1};
  return r;
}
template <int N> Representation AdjointRep() {
  Representation r; r.kind = GH_REP_ADJ; r.N = N; r.d = N * N - 1; r.real = 1; r.nality = 0; r.repname = "adjoint";
  r.rows.assign((size_t)N - 1, 1);
  r.rows[0] = 2;
  return r;
}
// GeneralRep<N>(rows, real): the Young-symmetriser irrep (src/rep/rep_general.hpp:54-84)
template <int N> Representation GeneralRep(std::vector<int> rows, bool real = false) {
  Representation r;
  r.kind = GH_REP_GENERAL; r.N = N; r.real = real ? 1 : 0;
  long dimT = 0;
  check(gh_rep_general_info(N, rows.data(), (int)rows.size(), &r.d, &r.n_boxes, &dimT), nullptr);
  r.dimT = dimT;
  r.T.assign((size_t)(N * N - 1) * r.d * r.d * 2, 0.0);
  r.W.assign((size_t)r.d * dimT * 2, 0.0);
  check(gh_rep_general_build(N, rows.data(), (int)rows.size(), r.T.data(), r.W.data()), nullptr);
  r.nality = r.n_boxes % N;
  r.rows = rows;
  r.repname = "general[";
  for (size_t i = 0; i < rows.size(); ++i) r.repname += (i ? "," : "") + std::to_string(rows[i]);
  r.repname += "]";
  return r;
}
// src/hmc_higgs.cpp:23-34 spec syntax: "fund" | "adj" | "r1,r2,...[:real]"
template <int N> Representation make_rep(std::string spec) {
  if (spec == "fund") return FundamentalRep<N>();
  if (spec == "adj") return AdjointRep<N>();
  bool real = false;
  const auto colon = spec.find(':');
  if (colon != std::string::npos) { real = (spec.substr(colon + 1) == "real"); spec = spec.substr(0, colon); }
  std::vector<int> rows;
  std::stringstream ss(spec);
  std::string tok;
  while (std::getline(ss, tok, ',')) if (!tok.empty()) rows.push_back(std::atoi(tok.c_str()));
  if (rows.empty()) throw std::runtime_error("bad rep spec '" + spec + "'");
  return GeneralRep<N>(rows, real);
}

// ---- multi-invariant onsite potential (src/action/scalar_invariants.hpp) ----
// CasimirChannels<N>(rep): the quartic channels of R (x) Rbar, lambda = their
// adjoint-Casimir values, ascending (scalar_invariants.hpp:19-27).
template <int N> struct CasimirChannels {
  Representation rep;
  std::vector<double> lambda;
  explicit CasimirChannels(const Representation& R) : rep(R) {
    const gh_rep_desc d = rep.desc();
    int n = 0;
    check(gh_casimir_channels(N, &d, nullptr, 0, &n), nullptr);
    lambda.assign((size_t)n, 0.0);
    check(gh_casimir_channels(N, &d, lambda.data(), n, &n), nullptr);
  }
  int n_channels() const { return (int)lambda.size(); }
};
// MultiInvariantPotential<N>(channels, f, mu2): V = -mu2 phi^dag phi + sum_c f_c V_c
// (scalar_invariants.hpp:190-206); plug it in with hmc.potential = &pot.
template <int N> struct MultiInvariantPotential {
  const CasimirChannels<N>* ch = nullptr;
  std::vector<double> f;
  double mu2 = 0.0;
  MultiInvariantPotential(const CasimirChannels<N>& c, std::vector<double> ff, double m) : ch(&c), f(std::move(ff)), mu2(m) {
    if ((int)f.size() != c.n_channels())
      throw std::runtime_error("need " + std::to_string(c.n_channels()) + " couplings, got " + std::to_string(f.size()));
  }
};

// ---- HMC ----
template <int D, int N>
class GaugeHiggsHMC {
 public:
  // couplings and integrator: public members, as in the reference
  double beta = 2.3, kappa = 0.1, lambda = 0.5, tau = 1.0;
  int nmd = 20;
  Integrator integ = Integrator::Omelyan2MN;
  std::uint64_t traj_count = 0, accept_count = 0;
  double last_dH = 0.0;
  int64_t vol = 1;
  // optional onsite potential (src/hmc/gauge_higgs_hmc.hpp:25-27); nullptr = quartic in lambda
  const MultiInvariantPotential<N>* potential = nullptr;
  bool frozen_phi = false;   // |phi_x| = 1 scalar (src/hmc/gauge_higgs_hmc.hpp:38-40)

  GaugeHiggsHMC(const std::array<int, D>& extents, const Representation& R, std::uint64_t seed,
                Precision prec = Precision::FP64)
      : rep_(R), L_(extents) {
    for (int mu = 0; mu < D; ++mu) vol *= L_[mu];
    gh_rep_desc desc = rep_.desc();
    check(gh_ctx_create(D, N, 1, L_.data(), rep_.kind == GH_REP_NONE ? nullptr : &desc, (int)prec, &seed, &ctx_), nullptr);
  }
  GaugeHiggsHMC(const GaugeHiggsHMC&) = delete;
  GaugeHiggsHMC& operator=(const GaugeHiggsHMC&) = delete;
  ~GaugeHiggsHMC() { gh_ctx_destroy(ctx_); }

  gh_ctx* context() { sync_params(); return ctx_; }
  const Representation& rep() const { return rep_; }
  // how the device applies D(U): GH_PATH_REGISTER / GH_PATH_TENSOR / GH_PATH_CLOSED_FORM /
  // GH_PATH_PRODUCT / GH_PATH_PAIR (the closed form stands in for the reference's
  // GeneralRep::use_fast path; product and pair are exact re-expressions of the tensor apply)
  int rep_path() const { int p = 0; check(gh_rep_path(ctx_, &p), ctx_); return p; }
  // switch a general irrep between GH_PATH_PRODUCT / GH_PATH_PAIR and the path it takes
  // without them (an A/B of the same workload); throws for a path the irrep does not have
  void set_rep_path(int path) { check(gh_set_rep_path(ctx_, path), ctx_); }

  // initial fields (src/core/fields.hpp:25-34, src/core/scalar_field.hpp:34-50)
  void hot(double sigma = 1.0) { check(gh_hot_start(ctx_, sigma), ctx_); }
  void cold() { check(gh_cold_start(ctx_), ctx_); }
  void phi_gaussian(std::uint64_t stream, double sigma = 1.0) { check(gh_phi_gaussian(ctx_, stream, sigma), ctx_); }
  void phi_cold(double c = 1.0) { check(gh_phi_cold(ctx_, c), ctx_); }
  void normalize_phi() { check(gh_normalize_phi(ctx_), ctx_); }

  void kick(double eps) { sync_params(); check(gh_kick(ctx_, eps), ctx_); }
  void drift(double eps) { sync_params(); check(gh_drift(ctx_, eps), ctx_); }
  void md_evolve() { sync_params(); check(gh_md_evolve(ctx_), ctx_); }
  void refresh_momenta() { sync_params(); check(gh_refresh_momenta(ctx_), ctx_); }
  void reunitarize_all() { check(gh_reunitarize(ctx_), ctx_); }
  double hamiltonian() { return measure().H; }

  bool trajectory() {
    sync_params();
    double dH = 0.0;
    int acc = 0;
    check(gh_trajectory(ctx_, &dH, &acc), ctx_);
    last_dH = dH;
    pull_counters();
    return acc != 0;
  }
  // n trajectories without a host round trip in between; records of each
  std::vector<gh_traj_record> run(int n) {
    sync_params();
    std::vector<gh_traj_record> r((size_t)std::max(n, 0));
    check(gh_run_trajectories(ctx_, n, r.data()), ctx_);
    if (n > 0) last_dH = r.back().dH;
    pull_counters();
    return r;
  }
  double acceptance() const { return traj_count ? double(accept_count) / double(traj_count) : 0.0; }

  gh_obs measure() { sync_params(); gh_obs o; check(gh_measure(ctx_, 0, &o), ctx_); return o; }
  double avg_plaquette() { return measure().plaquette; }
  double higgs_length() { return measure().L_phi; }
  double link_energy() { return measure().L_link; }
  double polyakov_loop(int tdir = D - 1) { double p; check(gh_polyakov(ctx_, 0, tdir, &p), ctx_); return p; }
  // loops traced in a probe irrep (src/measure/observables.hpp:48-101)
  double wilson_loop_fund(int Ra, int Rb) { double w; check(gh_wilson_loop(ctx_, 0, Ra, Rb, nullptr, 0, &w), ctx_); return w; }
  double wilson_loop_rep(const Representation& R, int Ra, int Rb) {
    double w;
    check(gh_wilson_loop(ctx_, 0, Ra, Rb, R.rows.data(), (int)R.rows.size(), &w), ctx_);
    return w;
  }
  double polyakov_loop_rep(const Representation& R, int tdir = D - 1) {
    double p;
    check(gh_polyakov_rep(ctx_, 0, tdir, R.rows.data(), (int)R.rows.size(), &p), ctx_);
    return p;
  }

  // fields in the reference layouts (complex interleaved doubles)
  std::vector<double> U() { std::vector<double> u((size_t)vol * D * N * N * 2); check(gh_get_links(ctx_, 0, u.data()), ctx_); return u; }
  void set_U(const std::vector<double>& u) { check(gh_set_links(ctx_, 0, u.data()), ctx_); }
  std::vector<double> phi() { std::vector<double> p((size_t)vol * rep_.d * 2); check(gh_get_phi(ctx_, 0, p.data()), ctx_); return p; }
  void set_phi(const std::vector<double>& p) { check(gh_set_phi(ctx_, 0, p.data()), ctx_); }

  double max_unitarity_violation() {
    const std::vector<double> u = U();
    double worst = 0.0;
    for (size_t l = 0; l < u.size() / (2 * N * N); ++l) {
      const double* m = &u[l * 2 * N * N];
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
          double re = (i == j) ? -1.0 : 0.0, im = 0.0;
          for (int k = 0; k < N; ++k) {   // (U^dag U)_ij = sum_k conj(U_ki) U_kj
            const double ar = m[2 * (k * N + i)], ai = -m[2 * (k * N + i) + 1];
            const double br = m[2 * (k * N + j)], bi = m[2 * (k * N + j) + 1];
            re += ar * br - ai * bi;
            im += ar * bi + ai * br;
          }
          worst = std::max(worst, std::sqrt(re * re + im * im));
        }
    }
    return worst;
  }

 protected:
  void sync_params() {
    if (beta != pb_ || kappa != pk_ || lambda != pl_) {
      check(gh_set_couplings(ctx_, 0, beta, kappa, lambda), ctx_);
      pb_ = beta; pk_ = kappa; pl_ = lambda;
    }
    const int ig = integ == Integrator::Leapfrog ? GH_LEAPFROG : GH_OMELYAN;
    if (tau != pt_ || nmd != pn_ || ig != pi_) {
      check(gh_set_integrator(ctx_, ig, nmd, tau), ctx_);
      pt_ = tau; pn_ = nmd; pi_ = ig;
    }
    if (traj_count != ptc_ || accept_count != pac_) {
      check(gh_set_traj_count(ctx_, 0, traj_count, accept_count), ctx_);
      ptc_ = traj_count; pac_ = accept_count;
    }
    if (frozen_phi != pfz_) {
      check(gh_set_frozen_phi(ctx_, frozen_phi ? 1 : 0), ctx_);
      pfz_ = frozen_phi;
    }
    if (potential != ppot_) {
      if (potential) check(gh_set_potential_multi(ctx_, (int)potential->f.size(), potential->f.data(), potential->mu2), ctx_);
      else check(gh_set_potential_quartic(ctx_), ctx_);
      ppot_ = potential;
    }
  }
  void pull_counters() {
    std::uint64_t t, a, nf;
    check(gh_get_traj_count(ctx_, 0, &t, &a, &nf), ctx_);
    traj_count = ptc_ = t;
    accept_count = pac_ = a;
  }
  Representation rep_;
  std::array<int, D> L_;
  gh_ctx* ctx_ = nullptr;
  double pb_ = NAN, pk_ = NAN, pl_ = NAN, pt_ = NAN;
  int pn_ = -1, pi_ = -1;
  std::uint64_t ptc_ = 0, pac_ = 0;
  const MultiInvariantPotential<N>* ppot_ = nullptr;
  bool pfz_ = false;
};

template <int D, int N>
class GaugeHMC : public GaugeHiggsHMC<D, N> {
 public:
  GaugeHMC(const std::array<int, D>& extents, std::uint64_t seed, Precision prec = Precision::FP64)
      : GaugeHiggsHMC<D, N>(extents, Representation{}, seed, prec) {}
};

// ---- parallel tempering in beta (src/hmc/replica_tempering.hpp) ----
// Same interface as the reference's ReplicaTempering<D,N>: rung k holds beta_k; one
// step() runs n_sweep trajectories of every rung, then (if enabled) the even and odd
// swap passes.  All rungs live in one context and advance in the same launches; a
// swap exchanges the beta labels on the device, which is the reference's exchange of
// (U, phi) between rungs (each rung keeps its beta, the configurations migrate).
template <int D, int N>
class ReplicaTempering {
 public:
  std::vector<double> betas;
  bool enabled = true;
  int n_sweep = 1;

  ReplicaTempering(const std::array<int, D>& extents, const Representation& R, const std::vector<double>& beta_ladder,
                   std::uint64_t seed0, std::uint64_t seed_stride = 1000003ull, std::uint64_t swap_seed = 0x5A7AB1ECull,
                   Precision prec = Precision::FP64)
      : betas(beta_ladder), rep_(R), swap_seed_(swap_seed) {
    if (beta_ladder.size() < 2) throw std::runtime_error("ReplicaTempering: need >=2 replicas");
    for (size_t k = 1; k < beta_ladder.size(); ++k)
      if (!(beta_ladder[k] > beta_ladder[k - 1])) throw std::runtime_error("ReplicaTempering: beta-ladder must be strictly increasing");
    const int M = (int)beta_ladder.size();
    std::vector<int> L;
    std::vector<std::uint64_t> seeds;
    for (int k = 0; k < M; ++k) {
      L.insert(L.end(), extents.begin(), extents.end());
      seeds.push_back(seed0 + (std::uint64_t)k * seed_stride);
    }
    gh_rep_desc desc = rep_.desc();
    check(gh_ctx_create(D, N, M, L.data(), rep_.kind == GH_REP_NONE ? nullptr : &desc, (int)prec, seeds.data(), &ctx_), nullptr);
    for (int k = 0; k < M; ++k) check(gh_set_couplings(ctx_, k, beta_ladder[k], kappa_, lambda_), ctx_);
    rung_traj_.assign((size_t)M, 0);
    rung_acc_.assign((size_t)M, 0);
  }
  ReplicaTempering(const ReplicaTempering&) = delete;
  ReplicaTempering& operator=(const ReplicaTempering&) = delete;
  ~ReplicaTempering() { gh_ctx_destroy(ctx_); }

  std::size_t n_replicas() const { return betas.size(); }
  std::size_t n_pairs() const { return betas.size() - 1; }
  double beta(std::size_t k) const { return betas.at(k); }
  gh_ctx* context() { return ctx_; }

  void set_kappa(double kappa) { kappa_ = kappa; push_couplings(); }
  void set_lambda(double lambda) { lambda_ = lambda; push_couplings(); }
  void set_tau(double tau) { tau_ = tau; push_integrator(); }
  void set_nmd(int nmd) { nmd_ = nmd; push_integrator(); }
  void set_integrator(Integrator integ) { integ_ = integ; push_integrator(); }
  void set_potential(const MultiInvariantPotential<N>* pot) {
    if (pot) check(gh_set_potential_multi(ctx_, (int)pot->f.size(), pot->f.data(), pot->mu2), ctx_);
    else check(gh_set_potential_quartic(ctx_), ctx_);
  }
  void set_frozen_phi(bool f) {
    check(gh_set_frozen_phi(ctx_, f ? 1 : 0), ctx_);
    if (f) check(gh_normalize_phi(ctx_), ctx_);
  }
  // start configurations of every rung (each with its own seed)
  void hot(double sigma = 1.0) { check(gh_hot_start(ctx_, sigma), ctx_); }
  void phi_gaussian(std::uint64_t stream, double sigma = 1.0) { check(gh_phi_gaussian(ctx_, stream, sigma), ctx_); }

  // one cycle: n_sweep trajectories of every rung, then the swap passes (if enabled)
  std::vector<gh_traj_record> step() {
    if (enabled != pen_ || n_sweep != psw_) {
      check(gh_temper_enable(ctx_, enabled ? 2 : 0, swap_seed_), ctx_);
      check(gh_temper_interval(ctx_, n_sweep), ctx_);
      pen_ = enabled; psw_ = n_sweep;
    }
    std::vector<gh_traj_record> r((size_t)n_sweep * n_replicas());
    check(gh_run_trajectories(ctx_, n_sweep, r.data()), ctx_);
    for (const gh_traj_record& x : r) {
      const size_t k = rung_of(x.beta);
      ++rung_traj_[k];
      rung_acc_[k] += x.accepted ? 1 : 0;
    }
    return r;
  }

  std::uint64_t swap_attempts(std::size_t p) const { return stats().first.at(p); }
  std::uint64_t swap_accepts(std::size_t p) const { return stats().second.at(p); }
  double pair_acceptance(std::size_t p) const {
    const auto st = stats();
    return st.first.at(p) ? double(st.second.at(p)) / double(st.first.at(p)) : 0.0;
  }
  // HMC acceptance of the trajectories run at rung k's beta
  double hmc_acceptance(std::size_t k) const {
    return rung_traj_.at(k) ? double(rung_acc_.at(k)) / double(rung_traj_.at(k)) : 0.0;
  }
  // measurements of the configuration currently at rung k
  gh_obs measure(std::size_t k) {
    gh_obs o;
    check(gh_measure(ctx_, lattice_at(k), &o), ctx_);
    return o;
  }
  // GH_TEMPER: true unless unset or one of 0 / false / off / no (any case)
  static bool env_enabled() {
    const char* e = std::getenv("GH_TEMPER");
    if (!e) return false;
    std::string v(e);
    for (auto& c : v) c = (char)std::tolower((unsigned char)c);
    return !(v.empty() || v == "0" || v == "false" || v == "off" || v == "no");
  }

 private:
  size_t rung_of(double b) const {
    for (size_t k = 0; k < betas.size(); ++k)
      if (betas[k] == b) return k;
    throw std::runtime_error("ReplicaTempering: record with an unknown beta");
  }
  int lattice_at(std::size_t k) {
    for (int l = 0; l < (int)betas.size(); ++l) {
      double b, kp, lm;
      check(gh_get_couplings(ctx_, l, &b, &kp, &lm), ctx_);
      if (b == betas.at(k)) return l;
    }
    throw std::runtime_error("ReplicaTempering: rung not found");
  }
  void push_couplings() {
    for (int l = 0; l < (int)betas.size(); ++l) {
      double b, kp, lm;
      check(gh_get_couplings(ctx_, l, &b, &kp, &lm), ctx_);
      check(gh_set_couplings(ctx_, l, b, kappa_, lambda_), ctx_);
    }
  }
  void push_integrator() {
    check(gh_set_integrator(ctx_, integ_ == Integrator::Leapfrog ? GH_LEAPFROG : GH_OMELYAN, nmd_, tau_), ctx_);
  }
  std::pair<std::vector<std::uint64_t>, std::vector<std::uint64_t>> stats() const {
    std::vector<std::uint64_t> a(betas.size()), c(betas.size());
    check(gh_temper_stats(ctx_, a.data(), c.data(), nullptr), ctx_);
    return {a, c};
  }
  Representation rep_;
  std::uint64_t swap_seed_;
  gh_ctx* ctx_ = nullptr;
  double kappa_ = 0.1, lambda_ = 0.5, tau_ = 1.0;
  int nmd_ = 20;
  Integrator integ_ = Integrator::Omelyan2MN;
  bool pen_ = false;
  int psw_ = 0;
  std::vector<std::uint64_t> rung_traj_, rung_acc_;
};

// ---- time-series statistics (the quantities of src/measure/observables.hpp:104-145) ----
// Written from the definitions: population moments about the sample mean, chi = V Var,
// the Binder cumulant U4 = 1 - m4 / (3 m2^2), and the jackknife error of the mean over
// contiguous bins.  The bin rule is the reference's (it fixes the printed error bars):
// nbins bins of floor(n / nbins) samples from the start of the series (a remainder at
// the end is left out), nbins lowered to max(2, n / 2) for a series shorter than
// 2 nbins, and no error for n < 2.
struct Stats {
  std::vector<double> x;
  void add(double v) { x.push_back(v); }
  int n() const { return (int)x.size(); }
  double mean() const { return x.empty() ? 0.0 : std::accumulate(x.begin(), x.end(), 0.0) / (double)x.size(); }
  // k-th moment about the mean, 1/n normalisation
  double central_moment(int k) const {
    if (x.empty()) return 0.0;
    const double m = mean();
    double acc = 0.0;
    for (double v : x) acc += std::pow(v - m, k);
    return acc / (double)x.size();
  }
  double var() const { return central_moment(2); }
  double susceptibility(double volume) const { return volume * var(); }
  double binder() const {
    const double m2 = central_moment(2);
    return m2 > 0.0 ? 1.0 - central_moment(4) / (3.0 * m2 * m2) : 0.0;
  }
  double binned_error(int nbins = 16) const {
    const int total = n();
    if (total < 2) return 0.0;
    const int nb = total < 2 * nbins ? std::max(2, total / 2) : nbins;
    const int width = total / nb;
    // leave-one-bin-out means theta_b; error^2 = (nb - 1)/nb * sum_b (theta_b - <theta>)^2
    std::vector<double> bin_sum(nb, 0.0);
    for (int b = 0; b < nb; ++b)
      bin_sum[b] = std::accumulate(x.begin() + (size_t)b * width, x.begin() + (size_t)(b + 1) * width, 0.0);
    const double all = std::accumulate(bin_sum.begin(), bin_sum.end(), 0.0);
    std::vector<double> theta(nb);
    for (int b = 0; b < nb; ++b) theta[b] = (all - bin_sum[b]) / ((double)(nb - 1) * width);
    const double tbar = std::accumulate(theta.begin(), theta.end(), 0.0) / nb;
    double ss = 0.0;
    for (double t : theta) ss += (t - tbar) * (t - tbar);
    return std::sqrt((double)(nb - 1) / nb * ss);
  }
};

// ---- autocorrelation analysis (src/measure/autocorr.hpp) ----
// Madras-Sokal: autocovariance with 1/N normalisation, tau_int = 1/2 + sum_{t=1}^{W}
// rho(t) with the smallest window W >= 6 tau_int(W) (lags capped at 2000 and N-1);
// the error on the mean is sqrt(2 tau_int var / N).  A series with no fluctuations
// (variance <= 1e-24 <x^2>) has tau_int = 1/2 and error 0.
inline std::vector<double> autocovariance(const std::vector<double>& x, int maxlag) {
  const int n = (int)x.size();
  if (n == 0) return {};
  double m = 0.0;
  for (double v : x) m += v;
  m /= n;
  maxlag = std::min(maxlag < 0 ? n - 1 : maxlag, n - 1);
  std::vector<double> c((size_t)maxlag + 1, 0.0);
  for (int t = 0; t <= maxlag; ++t) {
    double s = 0.0;
    for (int i = 0; i + t < n; ++i) s += (x[i] - m) * (x[i + t] - m);
    c[t] = s / n;
  }
  return c;
}
inline bool no_fluctuations(const std::vector<double>& x, double c0) {
  double m2 = 0.0;
  for (double v : x) m2 += v * v;
  return c0 <= 1e-24 * (x.empty() ? 0.0 : m2 / x.size()) + 1e-300;
}
inline double tau_int(const std::vector<double>& x, int* window = nullptr) {
  const int n = (int)x.size();
  if (window) *window = 0;
  if (n < 2) return 0.5;
  const std::vector<double> c = autocovariance(x, std::min(n - 1, 2000));
  if (no_fluctuations(x, c[0])) return 0.5;
  double tau = 0.5;
  int W = (int)c.size() - 1;
  for (int M = 1; M < (int)c.size(); ++M) {
    tau += c[M] / c[0];
    if (M >= 6.0 * tau) { W = M; break; }
  }
  if (window) *window = W;
  return std::max(tau, 0.5);
}
inline double effective_sample_size(const std::vector<double>& x) {
  return x.empty() ? 0.0 : (double)x.size() / (2.0 * tau_int(x));
}
inline double autocorr_error(const std::vector<double>& x) {
  if (x.size() < 2) return 0.0;
  const double var = autocovariance(x, 0)[0];
  if (no_fluctuations(x, var)) return 0.0;
  return std::sqrt(2.0 * tau_int(x) * var / (double)x.size());
}

}  // namespace ghb
