// gc_internal.h — device-visible parameter structs and kernel launchers
// shared by the translation units of libgrasph_cuda.so.
//
// Layout in HBM: every system slot (one Grasph particle system, repeated
// across all instances of a context) is packed instance after instance.
// Per-particle fields are stored component-planar ("SoA"): component c of
// packed particle g lives at field[c*N + g], N = packed count of the slot.
// Particle indices are int32 (a context holds < 2^31 particles per slot).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/grasph_cuda.h"

namespace gc {

constexpr int MAXD = 3;   // spatial dimensions
constexpr int MAXS = 6;   // Voigt components
constexpr int MAX_STAGES = 8;
constexpr int MAX_INTER_PER_SYS = 16;

// Device error word bits (OR-ed by kernels, read by the host).
enum : int {
    ERR_NONFINITE = 1,      // NaN/Inf or out-of-range position in a key/cell
    ERR_CAPACITY = 2,       // a cell or ghost index beyond its buffer
    ERR_GRID_INCONS = 4,    // key order vs cell order disagreement (warning)
    ERR_TIMEOUT = 8,
    ERR_XSPH_GHOST = 16     // an XSPH write at a ghost index beyond the ghost's source system
};

// Per (system slot, instance) parameters; packed range [base, base+n).
struct SysInst {
    int64_t base, n;
    double mass, c, srcv[MAXD], srcrho;
    double sort_cutoff;  // 2·h_min of the instance (src/TimeIntegration.jl:612)
    double dt, half_dt, gamma_dt;
    // Written on the device each step:
    double bbmin[MAXD], bbmax[MAXD];  // bounding box (NaN-propagating min/max)
    int64_t kmin[MAXD], kext[MAXD];   // sort-key lattice box
    int64_t sort_cellbase, sort_ncells;
};

// Per (interaction, instance) grid and system_b parameters.
struct GridInst {
    double H, cell;                    // h, 2h
    // (2h)^2, then the FP32 copies of 1/h and of the kernel normalisation:
    // one 16-byte load in the FP32-compensated pair code
    alignas(16) double cutoff_sq;
    float f_invH, f_knorm;
    double knorm;                      // kernel normalisation
    double ming[MAXD];                 // grid origin (src/Interaction.jl:143)
    int64_t ng[MAXD];                  // cells per dimension (:179)
    int64_t ncells, cellbase;          // this instance's cells in the packed grid
    int64_t ncols, colbase;            // columns (all but the last dimension)
    double mina[MAXD], maxa[MAXD];     // system_a bounding box (coupled)
    // system_b wrapper parameters (src/BoundaryParticles.jl)
    double normal[MAXD], point[MAXD], beta, ljcut;
    double bmass, bc;                  // system_b mass and sound speed
    // FP32 copies for the FP32-compensated sweep
    float f_normal[MAXD], f_beta, f_ljcut, f_bmass, f_bc;
    int side_b;                        // 1 in the system_b-side copy of a two-sided interaction
};
static_assert(offsetof(GridInst, cutoff_sq) % 16 == 0 && offsetof(GridInst, f_invH) == offsetof(GridInst, cutoff_sq) + 8 &&
                  offsetof(GridInst, f_knorm) == offsetof(GridInst, cutoff_sq) + 12,
              "(2h)^2, 1/h and the kernel normalisation are read as one 16-byte load");

// Per (interaction, stage, instance) functor parameters.
struct PfnInst {
    double alpha, beta, h, delta, eps;
    // FP32 copies; h2eps = 0.01·h² (the first four 16-byte aligned: the pair
    // code reads them as one float4)
    alignas(16) float f_h;
    float f_h2eps, f_alpha, f_beta;
    float f_delta, f_eps;
    int S, has_delta, has_eps;
    int two;  // FluidPfn between two fluid systems, or FluidSolidPfn (both sides written)
    int fs;   // FluidSolidPfn: system_a's (the fluid's) pressure on both sides
};
static_assert(offsetof(PfnInst, f_h) % 16 == 0 && offsetof(PfnInst, f_h2eps) == offsetof(PfnInst, f_h) + 4 &&
                  offsetof(PfnInst, f_alpha) == offsetof(PfnInst, f_h) + 8 &&
                  offsetof(PfnInst, f_beta) == offsetof(PfnInst, f_h) + 12,
              "h, 0.01·h², α and β are read as one float4");

// Per (virtual system, instance) parameters.
struct VirtInst {
    double pv[MAXD];  // prescribed_v
};

// Per (ghost entry, instance) parameters.
struct GhostInst {
    double normals[GC_MAX_GHOST_PLANES][MAXD], points[GC_MAX_GHOST_PLANES][MAXD];
    double cutoff;
    int64_t src_base, src_n;   // source particles in the source slot
    int64_t cap_base, cap;     // capacity range in the packed ghost arrays
    int64_t base, n;           // current ghosts (written on the device)
    double mass, c;
};

// One per-particle field: ncomp planar components with stride N.
struct Field {
    double* p;
    int ncomp;
};

// Device pointers of one system slot (current buffers).
struct SlotPtrs {
    int64_t N;           // packed particle count (capacity for ghosts)
    int nd, ns, nvort, kind;
    double *x, *v, *rho, *dvdt, *drhodt, *p, *stress, *sr, *vort, *strain, *strainp, *vadj;
    double *q0v, *q0rho;
    int32_t* id;         // 1-based reference id
    int32_t* inst_of;    // instance of each packed particle
    SysInst* inst;       // per-instance parameters
    // ghosts only
    int32_t *io, *ib;    // 1-based source index / plane index
    double* normals;     // generation-order normals
    const int64_t* count;  // device count (ghosts) or nullptr
};

// Updater descriptor (per system, stage, chain position, instance).
struct UpdInst {
    int kind;
    double prm[GC_UPD_NPARAM];
    // precomputed on the host with the reference's expressions
    double pre;        // Tait: rho0*c*c/gamma
    int gamma_int;     // Tait: gamma is an integer that fits
    double D0, omn, om2n, a_phi, k_c, a_psi, apex_thr, apex;  // EP / Hooke
    uint32_t zmask;
};

#ifdef __CUDACC__
// Programmatic dependent launch.  In a captured step graph a kernel may be
// launched while the kernel it depends on is still running; every kernel's
// first act is therefore to wait until its predecessors have finished and
// their memory is visible (griddepcontrol.wait, which returns at once
// without such an edge), and only then does it let its own dependents
// launch, so that their launch overlaps its work.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#endif

}  // namespace gc
