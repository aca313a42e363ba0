// Instantiates the kernels of SU(3) in float storage for D = 2, 3, 4 and every representation kind.
#include "gh_engine.cuh"
namespace ghk {
EngineBase* make_engine_n3_f32(int D, int rep) { return make_engine_NR<3, float>(D, rep); }
}  // namespace ghk
