// gc_update.h — arguments of the elementwise integrator and updater kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gc_internal.h"

namespace gc {

struct StepArgs {
    int64_t N;
    int nd;
    const int32_t* inst_of;
    const SysInst* inst;
    double *x, *v, *rho, *dvdt, *drhodt, *q0v, *q0rho;
};

struct UpdArgs {
    int64_t N;
    int nd, ns, nvort;
    const int32_t* inst_of;
    const SysInst* inst;
    const UpdInst* u;   // per instance
    double dt;          // NaN: each instance's own dt
    double *rho, *p, *stress, *sr, *vort, *strain, *strainp, *dvdt, *drhodt;
};

void launch_halfstep(const StepArgs& a, cudaStream_t s);
void launch_fullstep(const StepArgs& a, cudaStream_t s);
void launch_update(const UpdArgs& a, cudaStream_t s);

}  // namespace gc
