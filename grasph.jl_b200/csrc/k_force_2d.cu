// k_force_2d.cu — 2-D instantiations of the fused pair sweep.
// Compiled with -fmad=false (reference rounding).
#include "k_force_impl.cuh"

namespace gc {

int launch_force_f64_2d(const ForceArgs& A, bool count_only, cudaStream_t s) {
    if (A.kk == GC_KERNEL_CUBIC_SPLINE) return launch_nd<2, GC_KERNEL_CUBIC_SPLINE>(A, count_only, s);
    return launch_nd<2, GC_KERNEL_WENDLAND_C2>(A, count_only, s);
}

}  // namespace gc
