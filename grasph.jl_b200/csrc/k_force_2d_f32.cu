// k_force_2d_f32.cu — 2-D instantiations of the fused pair sweep, FP32-compensated.
// Compiled with -fmad=false (reference rounding of the FP64 parts).
#include "k_force_impl.cuh"

namespace gc {

GC_DEFINE_FORCE_TU(2, true, launch_force_2d_f32)

}  // namespace gc
