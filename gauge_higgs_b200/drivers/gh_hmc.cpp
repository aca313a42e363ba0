// gh_hmc -- pure-gauge HMC driver on the B200 engine.  Command line, defaults and
// output lines are those of the reference driver (src/main.cpp:11-51):
//   gh_hmc [L=8] [beta=2.3] [ntherm=50] [nmeas=100] [nmd=20] [tau=1.0] [seed=1]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "gauge_higgs_b200.hpp"

#ifndef NDIM
#define NDIM 4
#endif
#ifndef NCOL
#define NCOL 2
#endif
constexpr int kDim = NDIM, kN = NCOL;

int main(int argc, char** argv) {
  auto argf = [&](int i, double def) { return i < argc ? std::atof(argv[i]) : def; };
  auto argi = [&](int i, long def) { return i < argc ? std::atol(argv[i]) : def; };
  const int Lext = (int)argi(1, 8);
  const double beta = argf(2, 2.3);
  const int ntherm = (int)argi(3, 50), nmeas = (int)argi(4, 100), nmd = (int)argi(5, 20);
  const double tau = argf(6, 1.0);
  const std::uint64_t seed = (std::uint64_t)argi(7, 1);
  const char* pe = std::getenv("GH_PRECISION");
  const ghb::Precision prec = (pe && std::strcmp(pe, "fp32") == 0)       ? ghb::Precision::FP32_MD
                               : (pe && std::strcmp(pe, "fp32-all") == 0) ? ghb::Precision::FP32_ALL
                                                                          : ghb::Precision::FP64;
  std::array<int, kDim> L{};
  for (int mu = 0; mu < kDim; ++mu) L[mu] = Lext;
  try {
    ghb::GaugeHMC<kDim, kN> hmc(L, seed, prec);
    hmc.beta = beta; hmc.tau = tau; hmc.nmd = nmd;
    std::printf("# Pure-gauge HMC: D=%d  SU(%d)  L=%d^%d  vol=%lld  beta=%.4f  tau=%.3f  nmd=%d\n", kDim, kN, Lext, kDim,
                (long long)hmc.vol, beta, tau, nmd);
    hmc.hot(0.8);
    hmc.run(ntherm);
    std::printf("# thermalized %d trajectories; acceptance %.3f\n", ntherm, hmc.acceptance());
    hmc.traj_count = 0; hmc.accept_count = 0;
    double sP = 0.0, sP2 = 0.0, sExp = 0.0;
    const std::vector<gh_traj_record> rec = hmc.run(nmeas);
    for (const auto& r : rec) { sP += r.plaquette; sP2 += r.plaquette * r.plaquette; sExp += std::exp(-r.dH); }
    const double mP = sP / nmeas, varP = sP2 / nmeas - mP * mP;
    std::printf("# measured %d trajectories\n", nmeas);
    std::printf("plaquette       = %.6f +/- %.6f\n", mP, std::sqrt(std::max(0.0, varP) / nmeas));
    std::printf("acceptance      = %.4f\n", hmc.acceptance());
    std::printf("<exp(-dH)>      = %.5f  (should be ~1)\n", sExp / nmeas);
    std::printf("max ||U^dU-I||  = %.3e\n", hmc.max_unitarity_violation());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
