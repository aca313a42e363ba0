// hmc_higgs -- gauge + Higgs HMC driver on the B200 engine.  Command line, defaults
// and output lines are those of the reference driver (src/hmc_higgs.cpp:36-100):
//   hmc_higgs <rep> <L> <beta> <kappa> <lambda> [ntherm=80] [nmeas=200] [nmd=24] [tau=1.0] [seed=1]
//     <rep> = fund | adj | <Young rows e.g. 2,1> [':real']
// Compile-time D = NDIM, N = NCOL as in the reference build.  GH_PRECISION=fp32
// in the environment selects the FP32-MD mode (FP64 Hamiltonian).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include "gauge_higgs_b200.hpp"

#ifndef NDIM
#define NDIM 4
#endif
#ifndef NCOL
#define NCOL 2
#endif
constexpr int kDim = NDIM, kN = NCOL;

int main(int argc, char** argv) {
  if (argc < 6) {
    std::fprintf(stderr,
      "usage: %s <rep> <L> <beta> <kappa> <lambda> [ntherm=80] [nmeas=200] [nmd=24] [tau=1.0] [seed=1]\n"
      "  <rep> = fund | adj | <Young rows e.g. 2,1> [add ':real' for a real-scalar rep, e.g. 2,1:real]\n",
      argv[0]);
    return 1;
  }
  const char* repname = argv[1];
  auto argf = [&](int i, double def) { return i < argc ? std::atof(argv[i]) : def; };
  auto argi = [&](int i, long def) { return i < argc ? std::atol(argv[i]) : def; };
  const int Lext = (int)argi(2, 8);
  const double beta = argf(3, 2.3), kappa = argf(4, 0.2), lambda = argf(5, 0.5);
  const int ntherm = (int)argi(6, 80), nmeas = (int)argi(7, 200), nmd = (int)argi(8, 24);
  const double tau = argf(9, 1.0);
  const std::uint64_t seed = (std::uint64_t)argi(10, 1);
  const char* pe = std::getenv("GH_PRECISION");
  const ghb::Precision prec = (pe && std::strcmp(pe, "fp32") == 0)       ? ghb::Precision::FP32_MD
                               : (pe && std::strcmp(pe, "fp32-all") == 0) ? ghb::Precision::FP32_ALL
                                                                          : ghb::Precision::FP64;

  ghb::Representation rep;
  try { rep = ghb::make_rep<kN>(repname); }
  catch (const std::exception& e) { std::fprintf(stderr, "rep error: %s\n", e.what()); return 1; }

  std::array<int, kDim> L{};
  for (int mu = 0; mu < kDim; ++mu) L[mu] = Lext;
  try {
    ghb::GaugeHiggsHMC<kDim, kN> hmc(L, rep, seed, prec);
    hmc.beta = beta; hmc.kappa = kappa; hmc.lambda = lambda; hmc.tau = tau; hmc.nmd = nmd;
    std::printf("# Gauge+Higgs HMC: D=%d SU(%d) rep=%s d=%d N-ality=%d L=%d^%d vol=%lld\n", kDim, kN, rep.name().c_str(),
                rep.d, rep.nality, Lext, kDim, (long long)hmc.vol);
    std::printf("# beta=%.4f kappa=%.4f lambda=%.4f tau=%.3f nmd=%d  (kappa_c,free=1/(2D)=%.4f)\n", beta, kappa, lambda,
                tau, nmd, 1.0 / (2.0 * kDim));
    hmc.hot(0.8);
    hmc.phi_gaussian(12345, 0.3);
    hmc.run(ntherm);
    hmc.traj_count = 0; hmc.accept_count = 0;
    ghb::Stats plaq, Lphi, Llink, poly;
    double sExp = 0.0;
    const double V = (double)hmc.vol;
    for (int t = 0; t < nmeas; ++t) {
      const gh_traj_record r = hmc.run(1)[0];
      plaq.add(r.plaquette);
      Lphi.add(r.L_phi);
      Llink.add(r.L_link);
      poly.add(hmc.polyakov_loop());
      sExp += std::exp(-r.dH);
    }
    std::printf("plaquette   = %.6f +/- %.6f\n", plaq.mean(), plaq.binned_error());
    std::printf("L_phi       = %.6f +/- %.6f   (<phi^dag phi>)\n", Lphi.mean(), Lphi.binned_error());
    std::printf("L_link      = %.6f +/- %.6f   (gauge-inv hopping energy; transition locator)\n", Llink.mean(), Llink.binned_error());
    std::printf("Polyakov    = %.6f +/- %.6f\n", poly.mean(), poly.binned_error());
    std::printf("chi_link    = %.5f   (V*Var(L_link), susceptibility)\n", Llink.susceptibility(V));
    std::printf("Binder_link = %.5f   (U4 of L_link)\n", Llink.binder());
    std::printf("chi_phi     = %.5f   (V*Var(L_phi))\n", Lphi.susceptibility(V));
    std::printf("acceptance  = %.4f\n", hmc.acceptance());
    std::printf("<exp(-dH)>  = %.5f\n", sExp / nmeas);
    std::printf("max||UdU-I||= %.2e\n", hmc.max_unitarity_violation());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
