// gc_force.h — arguments of the fused pair-sweep kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gc_internal.h"

namespace gc {

constexpr int FORCE_TPB = 128;  // threads per block of the sweep
constexpr int FORCE_BUF = 64;   // staged-neighbour column of the counting sweep (shared memory)

// Launch configurations of the sweep: (min resident blocks, staged
// neighbours per thread, pair-loop unroll, chunk staging).  Chosen per
// (system, stage) by the tuner in gc_context.cu.
struct ForceCfg {
    int minb, buf, unroll;
    int stg;  // > 0: k_sweep_stg with chunks of stg candidates (policies that stage copies; k_sweep otherwise)
};
constexpr int NUM_FORCE_CFG = GC_NUM_SWEEP_CONFIGS;
constexpr ForceCfg FORCE_CFGS[NUM_FORCE_CFG] = {{4, 64, 1, 0}, {6, 64, 1, 0}, {5, 64, 1, 96}, {6, 64, 1, 96}};
constexpr int MAX_REFS = 8;     // interactions fused into one launch

// system_b kinds as seen by a functor (src/PairwiseFunctors.jl dispatch)
enum { BT_SELF = 0, BT_DYNAMIC = 1, BT_STATIC = 2, BT_GHOST = 3, BT_SYSTEM = 4 };

// per-particle divisor caches (one per slot, refreshed before each sweep)
enum { AUX_P_OVER_RHO2 = 0, AUX_INV_RHO2 = 1, AUX_MASS_OVER_RHO = 2 };

// Device-side functor code: FluidPfn with its two-sided (multiphase),
// fluid-solid and surface-tension forms enabled; the plain GC_PFN_FLUID code
// compiles them out of the pair loop.
constexpr int PFN_FLUID2 = 16;
template <int P>
__host__ __device__ constexpr bool fluid_pfn() {
    return P == GC_PFN_FLUID || P == PFN_FLUID2;
}

struct InterRef {
    int btype;
    const SysInst* bbox;  // per-instance bounding box of system_b (nullptr: never skip)
    const GridInst* gi;   // per instance
    const PfnInst* pi;    // per instance, this stage
    const int32_t* cs;    // packed CSR over system_b (global b indices)
    int64_t cs_cells;     // cells of cs that are valid (an instance beyond them is skipped)
    const double *bx, *bv, *brho, *bp, *bstress, *baux;
    const float* bfp;     // FP32 records of system_b (v, rho, aux, 1/rho, stress), pack_stride floats each
    const double* bxp;    // FP64 positions of system_b, pos_stride doubles each (FP32 sweep), or nullptr
    int64_t bN;           // planar stride of system_b's arrays
    int32_t* counts;      // optional per-particle accepted-pair counts
};

struct ForceArgs {
    int nd, ns, pfn, kk;
    int64_t aN;
    const int32_t* a_inst_of;
    const double *ax, *av, *arho, *aaux, *astress, *a_p;
    double *advdt, *adrhodt, *asr, *avort;
    const double* a_c;     // per-instance sound speed
    const double* a_mass;  // per-instance particle mass
    const float* a_cf;     // FP32 copies of the two above
    const float* a_massf;
    const float* afp;      // FP32 records of system_a (FP32-compensated precision)
    int prec;              // GC_PRECISION_*
    int* err;
    const int2* groups;        // warp groups (start, count) of system_a particles
    const int64_t* ngroups;    // device count of groups
    int num_sms;
    int cfg;                   // index into FORCE_CFGS
    int imask, iwsum;          // InterpolateFieldFn: fields (1<<GC_FIELD_*), accumulate w_sum into avort
    int nref;
    InterRef ref[MAX_REFS];
};

int launch_force_f64(const ForceArgs& A, bool count_only, cudaStream_t s);
void launch_groups_count(const GridInst* gi, int ninst, int nd, const int32_t* cs, int64_t ncols_cap,
                         int64_t cells_cap, int32_t* cnt, cudaStream_t s);
void launch_groups_fill(const GridInst* gi, int ninst, int nd, const int32_t* cs, const int32_t* off,
                        int64_t ncols_cap, int64_t cells_cap, int2* groups, int64_t* ngroups, cudaStream_t s);
void launch_aux(int mode, int64_t N, const int64_t* count, const double* rho, const double* p,
                const int32_t* inst_of, const double* mass, double* aux, cudaStream_t s);
// Per-particle records of the FP32-compensated sweep, one record per
// particle so a neighbour costs one or two sectors instead of one per field:
//   pk:  v[nd], rho, aux(mode), 1/rho, stress[ns], zero padding — pack_stride floats
//   xpk: x[nd] in FP64, zero padding — pos_stride doubles (the exact neighbour test)
// Either may be nullptr.  ns may be 0; stress may be nullptr (zeros).
__host__ __device__ constexpr int pack_stride(int nd, int ns) { return (nd + 3 + ns + 3) / 4 * 4; }
__host__ __device__ constexpr int pos_stride(int nd) { return nd == 2 ? 2 : 4; }
void launch_pack32(int mode, int64_t N, const int64_t* count, int nd, int ns, const double* x, const double* v,
                   const double* rho, const double* p, const double* stress, const int32_t* inst_of,
                   const double* mass, double* xpk, float* pk, cudaStream_t s);

}  // namespace gc
