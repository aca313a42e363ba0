// hmc_higgs_multi -- gauge + Higgs HMC with the multi-invariant onsite potential
//   V = -mu2 phi^dag phi + sum_c f_c V_c[phi]
// on the B200 engine.  Command line, environment switches and output lines are
// those of the reference driver (src/hmc_higgs_multi.cpp:1-125):
//   hmc_higgs_multi <rep> <L> <beta> <kappa> <mu2> <couplings|auto> [ntherm=80 nmeas=200 nmd=24 tau=1 seed=1 ts_outfile]
//     <couplings> = comma list f_0,f_1,... in the printed channel (C2) order, or "auto" (all 1)
//   Run with just <rep> to print the channels.  GH_COLD=1: ordered start (identity
//   links, phi = (1, 0, ...)) instead of hot.  GH_FROZEN=1: frozen-length scalar
//   |phi_x| = 1.  GH_PRECISION=fp32: FP32-MD mode.
// Compile-time D = NDIM, N = NCOL as in the reference build.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include "gauge_higgs_b200.hpp"

#ifndef NDIM
#define NDIM 4
#endif
#ifndef NCOL
#define NCOL 2
#endif
constexpr int kDim = NDIM, kN = NCOL;

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr,
      "usage: %s <rep> <L> <beta> <kappa> <mu2> <couplings|auto> [ntherm=80 nmeas=200 nmd=24 tau=1 seed=1 ts_outfile]\n"
      "  run with just <rep> to print the channel C2 values and the required #couplings.\n", argv[0]);
    return 1;
  }
  ghb::Representation rep;
  try { rep = ghb::make_rep<kN>(argv[1]); }
  catch (const std::exception& e) { std::fprintf(stderr, "rep error: %s\n", e.what()); return 1; }
  try {
    ghb::CasimirChannels<kN> ch(rep);
    std::printf("# rep=%s d=%d  %d quartic channels (C2): ", rep.name().c_str(), rep.d, ch.n_channels());
    for (double c : ch.lambda) std::printf("%.4g ", c);
    std::printf("\n");
    if (argc < 7) { std::printf("# provide %d couplings f_c (comma list) as arg 6 (or 'auto').\n", ch.n_channels()); return 0; }

    auto argf = [&](int i, double def) { return i < argc ? std::atof(argv[i]) : def; };
    auto argi = [&](int i, long def) { return i < argc ? std::atol(argv[i]) : def; };
    const int Lext = (int)argi(2, 8);
    const double beta = argf(3, 2.3), kappa = argf(4, 0.2), mu2 = argf(5, 1.0);
    const int ntherm = (int)argi(7, 80), nmeas = (int)argi(8, 200), nmd = (int)argi(9, 24);
    const double tau = argf(10, 1.0);
    const std::uint64_t seed = (std::uint64_t)argi(11, 1);
    const std::string ts_out = argc > 12 ? std::string(argv[12]) : std::string();
    std::vector<double> f;
    if (std::string(argv[6]) == "auto") f.assign((size_t)ch.n_channels(), 1.0);
    else { std::stringstream ss(argv[6]); std::string t; while (std::getline(ss, t, ',')) if (!t.empty()) f.push_back(std::atof(t.c_str())); }
    if ((int)f.size() != ch.n_channels()) {
      std::fprintf(stderr, "error: need %d couplings, got %zu\n", ch.n_channels(), f.size());
      return 1;
    }
    const bool frozen = std::getenv("GH_FROZEN") != nullptr;   // |phi_x| = 1 frozen-length scalar
    const char* pe = std::getenv("GH_PRECISION");
    const ghb::Precision prec = (pe && std::strcmp(pe, "fp32") == 0)       ? ghb::Precision::FP32_MD
                               : (pe && std::strcmp(pe, "fp32-all") == 0) ? ghb::Precision::FP32_ALL
                                                                          : ghb::Precision::FP64;
    ghb::MultiInvariantPotential<kN> pot(ch, f, mu2);

    std::array<int, kDim> L{};
    for (int mu = 0; mu < kDim; ++mu) L[mu] = Lext;
    ghb::GaugeHiggsHMC<kDim, kN> hmc(L, rep, seed, prec);
    hmc.beta = beta; hmc.kappa = kappa; hmc.tau = tau; hmc.nmd = nmd; hmc.potential = &pot;
    hmc.frozen_phi = frozen;
    std::printf("# D=%d SU(%d) L=%d^%d  beta=%.3f kappa=%.3f mu2=%.3f nmd=%d  potential=multi-invariant%s\n", kDim, kN,
                Lext, kDim, beta, kappa, mu2, nmd, frozen ? "  [FROZEN |phi|=1]" : "");
    if (std::getenv("GH_COLD")) { hmc.cold(); hmc.phi_cold(1.0); }
    else { hmc.hot(0.8); hmc.phi_gaussian(12345, 0.3); }
    if (frozen) hmc.normalize_phi();   // onto |phi_x| = 1 before thermalising
    hmc.run(ntherm);

    hmc.traj_count = 0; hmc.accept_count = 0;
    ghb::Stats plaq, Lphi, Llink;
    double sExp = 0.0;
    const double V = (double)hmc.vol;
    std::vector<double> ll, pl;
    const std::vector<gh_traj_record> rec = hmc.run(nmeas);
    for (const gh_traj_record& r : rec) {
      plaq.add(r.plaquette); Lphi.add(r.L_phi); Llink.add(r.L_link);
      pl.push_back(r.plaquette); ll.push_back(r.L_link);
      sExp += std::exp(-r.dH);
    }
    if (!ts_out.empty()) {
      std::ofstream out(ts_out);
      out << "# traj plaq L_link  (rep=" << rep.name() << " beta=" << beta << " kappa=" << kappa << " mu2=" << mu2
          << " nmd=" << nmd << ")\n";
      for (int t = 0; t < nmeas; ++t) out << t << ' ' << pl[t] << ' ' << ll[t] << '\n';
    }
    int W = 0;
    const double tau_ll = ghb::tau_int(ll, &W);
    std::printf("plaquette   = %.6f +/- %.6f\n", plaq.mean(), plaq.binned_error());
    std::printf("L_phi       = %.6f +/- %.6f\n", Lphi.mean(), Lphi.binned_error());
    std::printf("L_link      = %.6f +/- %.6f   chi_link=%.4f\n", Llink.mean(), ghb::autocorr_error(ll), Llink.susceptibility(V));
    std::printf("autocorr    = tau_int(L_link)=%.2f window=%d  N_eff=%.1f / %d meas\n", tau_ll, W,
                ghb::effective_sample_size(ll), nmeas);
    std::printf("acceptance  = %.4f   <exp(-dH)>=%.5f\n", hmc.acceptance(), nmeas > 0 ? sExp / nmeas : 0.0);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
