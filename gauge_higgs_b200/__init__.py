"""gauge_higgs_b200 -- B200-native molecular-dynamics engine for SU(N) gauge +
arbitrary-irrep Higgs Hybrid Monte Carlo.

The compute path is libgauge_higgs_b200.so (hand-written sm_100a CUDA behind the
C ABI in include/gauge_higgs_b200.h); this package is its host-side mirror of
the reference's C++ interface (GaugeHiggsHMC, GaugeHMC, the Representation
classes), plus batched ensembles with on-device kappa tempering.
"""
from ._lib import GaugeHiggsError, LIB_PATH  # noqa: F401  (raises ImportError if the library is missing)
from .hmc import (AdjointRep, CasimirChannels, Ensemble, FundamentalRep, GaugeHiggsHMC, GaugeHMC,  # noqa: F401
                  GeneralRep, LEAPFROG, MultiInvariantPotential, OMELYAN, Representation, make_rep)

