// Instantiates the kernels of SU(2) in double storage for D = 2, 3, 4 and every representation kind.
#include "gh_engine.cuh"
namespace ghk {
EngineBase* make_engine_n2_f64(int D, int rep) { return make_engine_NR<2, double>(D, rep); }
}  // namespace ghk
