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
    double *accv, *accrho;  // RK4 accumulators (nullptr for LeapFrog)
    double* vadj;           // v_adjustment when an XSPH functor is swept (else nullptr)
};

struct UpdArgs {
    int64_t N;
    int kind;           // GC_UPD_* of every instance (the model structure is shared)
    int nd, ns, nvort;
    const int32_t* inst_of;
    const SysInst* inst;
    const UpdInst* u;   // per instance
    double dt;          // NaN: each instance's own dt
    double *rho, *p, *stress, *sr, *vort, *strain, *strainp, *dvdt, *drhodt;
};

// One slot's FP32 sweep records (launch_pack32's arguments; xpk or pk may
// be nullptr).
struct PackArgs {
    int mode, nd, ns;
    int64_t N;
    const double *x, *v, *rho, *p, *stress;
    const int32_t* inst_of;
    const double* mass;
    double* xpk;
    float* pk;
};


void launch_halfstep(const StepArgs& a, cudaStream_t s);
// The half step fused with what follows it for the same particles before
// the first sweeps (src/TimeIntegration.jl:158, then _sweep_all_stages!'s
// stage-1 state updater :401-419): per particle the half step, the updater
// u (u.kind < 0: none; an elementwise kind), then (pk.pk or pk.xpk set) the
// FP32 records of the stage's first sweep.  One pass over the state instead
// of three.
void launch_halfstep_fused(const StepArgs& a, const UpdArgs& u, const PackArgs& pk, cudaStream_t s);
// Whether launch_halfstep_fused takes updater kind `kind` (the light,
// elementwise ones; the stress updaters keep their own launch).
bool halfstep_fuses(int kind);
void launch_fullstep(const StepArgs& a, cudaStream_t s);
// RK4 (src/TimeIntegration.jl:712-838): q0 snapshot, zero accumulators and
// dqdt reset; stage advance q = q0 + f·dt·dqdt (f = 0.5 or 1) and dqdt reset;
// damping and acc += w·dqdt after a stage's sweeps; q = q0 + dt·acc, zero
// XSPH pass and x += dt·v at the end.
void launch_rk4_begin(const StepArgs& a, cudaStream_t s);
void launch_rk4_advance(const StepArgs& a, double f, cudaStream_t s);
void launch_rk4_acc(const StepArgs& a, double w, cudaStream_t s);
void launch_rk4_final(const StepArgs& a, cudaStream_t s);
// src/TimeIntegration.jl:421-436, 684-685: with v_adjustment carried, the
// full step (or RK4 final) ends at v -= v_adjustment, v_adjustment = 0; after
// the XSPH sweeps this adds the new adjustment back and moves x by dt·v.
void launch_xsph_final(const StepArgs& a, cudaStream_t s);
void launch_update(const UpdArgs& a, cudaStream_t s);

// VirtualNormUpdater / PrescribedVelocityUpdater on a virtual system's
// source fields (src/StateUpdaters.jl:44-97).
struct VirtArgs {
    int64_t N;
    int nd, ns, kind;
    const int32_t* inst_of;
    const VirtInst* vi;  // per instance
    const UpdInst* u;    // per instance
    double *v, *rho, *p, *stress;
    const double* wsum;
};
void launch_virtual_update(const VirtArgs& a, cudaStream_t s);
// _update_virtual_positions! src/TimeIntegration.jl:389-397: x += prescribed_v·dt.
void launch_virtual_advance(double* x, int64_t N, int nd, const int32_t* inst_of, const SysInst* inst,
                            const VirtInst* vi, cudaStream_t s);

}  // namespace gc
