// k_force_2d.cu — 2-D instantiations of the fused pair sweep, FP64 (and neighbour counting).
// Compiled with -fmad=false (reference rounding of the FP64 parts).
#include "k_force_impl.cuh"

namespace gc {

GC_DEFINE_FORCE_TU(2, false, launch_force_2d_f64)

}  // namespace gc
