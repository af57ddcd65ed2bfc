/*
 * grasph_cuda.h — C ABI of libgrasph_cuda.so, the sm_100a implementation of
 * Grasph.jl's per-timestep SPH hot path (sort → grid → ghosts → staged sweeps
 * → leapfrog update).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (GC_OK == 0).  A failed call leaves a message that
 * gc_last_error() returns.  Host arrays use the memory layout Julia gives a
 * `Vector{SVector{K,Float64}}`: particle-major, K consecutive doubles per
 * particle (`pointer(ps.x)` under `GC.@preserve`).  Integer fields (`id`,
 * ghost `idx_original`/`idx_boundary`) are int64 and 1-based as in Julia.
 *
 * Each declaration names the Grasph.jl function or constructor it replaces
 * (file:line in the Grasph.jl source tree).
 *
 * Objects live in a context (one CUDA device, one stream).  A context holds
 * one or more *instances*: independent simulations that share one model
 * structure (the same kinds of systems, interactions, functors and updaters
 * in the same order) but may differ in particle counts and parameters.  A
 * single-rank Grasph.jl run is one instance; batched runs pack many.
 */
#ifndef GRASPH_CUDA_H
#define GRASPH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    GC_OK = 0,
    GC_ERR_ARG = 1,               /* invalid argument (Julia ArgumentError)        */
    GC_ERR_OOM = 2,               /* device allocation failed / budget exceeded     */
    GC_ERR_CAPACITY = 3,          /* ghost, cell or neighbour capacity overflow     */
    GC_ERR_NONFINITE = 4,         /* NaN/Inf or out-of-Int64 position (InexactError)*/
    GC_ERR_GRID_INCONSISTENT = 5, /* sort-key order disagrees with grid-cell order  */
    GC_ERR_TIMEOUT = 6,           /* a bounded device wait ran out                  */
    GC_ERR_CUDA = 7,              /* CUDA runtime error                             */
    GC_ERR_STATE = 8,             /* call made in the wrong lifecycle state         */
    GC_ERR_UNSUPPORTED = 9        /* functor/system combination not implemented     */
};

/* ---------------------------------------------------------- system kinds */
/* src/Particles.jl:38 (Basic), :149 (Fluid), :245 (Stress), :351 (ElastoPlastic) */
enum {
    GC_SYS_BASIC = 0,
    GC_SYS_FLUID = 1,
    GC_SYS_STRESS = 2,
    GC_SYS_ELASTOPLASTIC = 3
};

/* ------------------------------------------------------------- field ids */
/* Per-particle arrays of src/Sorting.jl:15-26 plus ghost bookkeeping.      */
enum {
    GC_FIELD_X = 0,            /* ND doubles                                  */
    GC_FIELD_V = 1,            /* ND doubles                                  */
    GC_FIELD_RHO = 2,          /* 1 double                                    */
    GC_FIELD_DVDT = 3,         /* ND doubles                                  */
    GC_FIELD_DRHODT = 4,       /* 1 double                                    */
    GC_FIELD_P = 5,            /* 1 double   (Fluid, Stress, ElastoPlastic)   */
    GC_FIELD_STRESS = 6,       /* NS doubles (Stress, ElastoPlastic)          */
    GC_FIELD_STRAIN_RATE = 7,  /* NS doubles (Stress, ElastoPlastic)          */
    GC_FIELD_VORTICITY = 8,    /* 1 double in 2-D, 3 in 3-D (ElastoPlastic)   */
    GC_FIELD_STRAIN = 9,       /* NS doubles (ElastoPlastic)                  */
    GC_FIELD_STRAIN_P = 10,    /* NS doubles (ElastoPlastic)                  */
    GC_FIELD_ID = 11,          /* int64, 1-based                              */
    GC_FIELD_V_ADJUSTMENT = 12,/* ND doubles (always zero without XSPH)       */
    GC_FIELD_IDX_ORIGINAL = 13,/* ghosts: int64 source index, 1-based         */
    GC_FIELD_IDX_BOUNDARY = 14,/* ghosts: int64 plane index, 1-based          */
    GC_FIELD_NORMALS = 15,     /* ghosts: ND doubles                          */
    GC_FIELD_W_SUM = 16,       /* virtual systems, probes: 1 double, kernel-weight sum */
    GC_FIELD_COUNT = 17,       /* probes: 1 double, the NeighborCountFn extra   */
    GC_NFIELDS = 18
};

/* ------------------------------------------------------ boundary wrappers */
/* src/BoundaryParticles.jl:38 (StaticBoundarySystem), :68 (DynamicBoundarySystem) */
enum { GC_WRAP_DYNAMIC = 1, GC_WRAP_STATIC = 2 };

/* ---------------------------------------------------------- kernel kinds */
/* src/Kernels.jl:18 (CubicSplineKernel), :92 (WenlandC2Kernel)             */
enum { GC_KERNEL_CUBIC_SPLINE = 0, GC_KERNEL_WENDLAND_C2 = 1 };

/* ------------------------------------------------- pairwise functor kinds */
/* src/PairwiseFunctors.jl.  GC_PFN_COUNT is the counting functor the
 * reference's sweep tests use (test/test_interaction_sweep.jl:14-30): each
 * accepted pair adds 1 to dvdt[.][1] and drhodt of both endpoints.          */
enum {
    GC_PFN_NONE = 0,                    /* `nothing` stage                     */
    GC_PFN_FLUID = 1,                   /* FluidPfn :136                       */
    GC_PFN_CAUCHY_FLUID = 2,            /* CauchyFluidPfn :252                 */
    GC_PFN_STRAIN_RATE = 3,             /* StrainRatePfn :18                   */
    GC_PFN_STRAIN_RATE_VORTICITY = 4,   /* StrainRateVorticityPfn :78          */
    GC_PFN_COUNT = 5,
    GC_PFN_XSPH = 6,                    /* XSPHPfn :360-389; velocity-adjust functor only */
    GC_PFN_FLUID_SOLID = 7,             /* FluidSolidPfn :479-519 (system_b a real system) */
    GC_PFN_INTERPOLATE = 8,             /* InterpolateFieldFn :392-440, system_b a virtual
                                           system or a probe: [0] bitmask of 1<<GC_FIELD_* out
                                           of v, rho, stress  [1] accumulate_wsum (0 or 1)  */
    GC_PFN_NEIGHBOR_COUNT = 9           /* NeighborCountFn :442-460, system_b a probe:
                                           its GC_FIELD_COUNT extra += 1 per neighbour  */
};
/* Per-stage functor parameters, GC_PFN_NPARAM doubles each:
 *   [0] art_visc_alpha  [1] art_visc_beta  [2] h
 *   [3] sigma S (FluidPfn, FluidSolidPfn; 2 = Monaghan form)  [4] delta (NaN = nothing)
 *   [5] epsilon (NaN = nothing)                                            */
#define GC_PFN_NPARAM 6

/* ---------------------------------------------------------- updater kinds */
/* src/StateUpdaters.jl                                                     */
enum {
    GC_UPD_NONE = 0,          /* `nothing`                                  */
    GC_UPD_ZERO_FIELDS = 1,   /* ZeroFieldUpdater :30; param[0] = bitmask of 1<<GC_FIELD_* */
    GC_UPD_TAIT_EOS = 2,      /* TaitEOSUpdater :108; [0] rho0 [1] gamma    */
    GC_UPD_LINEAR_EOS = 3,    /* LinearEOSUpdater :131; [0] rho0            */
    GC_UPD_ELASTOPLASTIC = 4, /* ElastoPlasticStressUpdater :202; [0] E [1] nu [2] phi [3] psi [4] cohesion */
    GC_UPD_HOOKE = 5,         /* HookeLawStressUpdater :356; [0] E [1] nu   */
    GC_UPD_VISCOPLASTIC_MC = 6, /* ViscoPlasticMCStressUpdater :144-186, the stress part; its
                                  EOS is the chain entry before it. [0] friction angle
                                  (radians) [1] cohesion; NS = 3, 4 or 6    */
    GC_UPD_VIRTUAL_NORM = 7,  /* VirtualNormUpdater :44-76 (virtual systems): [0..2] v_mult,
                                 [3] bitmask of 1<<GC_FIELD_* out of v, rho, p, stress */
    GC_UPD_PRESCRIBED_V = 8   /* PrescribedVelocityUpdater :78-97 (virtual systems)    */
};
#define GC_UPD_NPARAM 6
/* At most this many updaters may be chained in one stage (a Julia tuple of
 * functors inside the per-stage tuple).                                    */
#define GC_UPD_MAX_CHAIN 4

/* ------------------------------------------------------- ghost copy modes */
/* src/GhostParticles.jl:53 (GhostCopier), :26 (HouseholderReflect)          */
enum { GC_COPY_PLAIN = 0, GC_COPY_HOUSEHOLDER = 1 };

/* ------------------------------------------------------------- precision */
enum {
    GC_PRECISION_FP64 = 0,             /* reference arithmetic, FP64 throughout    */
    GC_PRECISION_FP32_COMPENSATED = 1  /* FP32 pair sweep, Kahan sums, FP64 state  */
};

typedef struct gc_ctx gc_ctx;

typedef struct gc_stats {
    int64_t steps_done;          /* leapfrog steps completed in this context      */
    int64_t pairs_last_step;     /* accepted pairs of the last step, one stage:
                                    unordered self pairs + coupled (a,b) pairs   */
    int64_t grid_inconsistent;   /* cells where key order and cell order disagreed */
    int64_t kernel_launches;     /* device kernels launched by this context       */
    int64_t sweep_launches;      /* pair-sweep launches timed (profiling on)      */
    double sweep_ms;             /* summed device time of those launches          */
    int32_t last_status;         /* device error word of the last step            */
    int32_t pad;
    int64_t graph_steps;         /* steps run as replays of a captured step graph */
    int64_t rollbacks;           /* verified windows re-run exactly (a capacity
                                    was outgrown inside the window)              */
    int32_t sweep_cfg_chosen[4]; /* tuned (system, stage) sweeps per configuration */
    int64_t sorts_in_order;      /* system sorts whose cell keys were already in
                                    order, so the reorder was the identity
                                    (src/Sorting.jl:176-186)                     */
} gc_stats;

/* Launch configurations of the pair sweep (block residency, staged
 * neighbours per thread, prefetch of the next neighbour's data); all give
 * bit-identical results.                                                  */
#define GC_NUM_SWEEP_CONFIGS 4

/* ============================================================ lifecycle */
/* Create a context on `device`; `hbm_budget_bytes` caps device allocations
 * (0 = no cap).                                                           */
int gc_ctx_create(int device, size_t hbm_budget_bytes, gc_ctx** out);
int gc_ctx_destroy(gc_ctx* ctx);
const char* gc_last_error(gc_ctx* ctx);
const char* gc_status_string(int status);

/* Add an instance (an independent simulation).                            */
int gc_instance_add(gc_ctx* ctx, int* inst_out);

/* ====================================================== model building */
/* BasicParticleSystem / FluidParticleSystem / StressParticleSystem /
 * ElastoPlasticParticleSystem constructors, src/Particles.jl:61,173,272,381.
 * `ns` is ignored for Basic/Fluid.  Returns a handle in *sys_out.          */
int gc_add_system(gc_ctx* ctx, int inst, int kind, int64_t n, int ndims, int ns,
                  double mass, double c, const double* source_v, double source_rho,
                  int* sys_out);

/* DynamicBoundarySystem(inner, normal, point, beta) src/BoundaryParticles.jl:79
 * or StaticBoundarySystem(inner, lj_cutoff) :47.  `normal`/`point` are
 * ignored for the static kind.  Returns a handle usable as system_b.       */
int gc_add_boundary(gc_ctx* ctx, int inst, int sys, int kind, const double* normal,
                    const double* point, double beta_or_lj_cutoff, int* handle_out);

/* GhostParticleSystem(ps, copiers...) src/GhostParticles.jl:199 together with
 * GhostEntry(ghost, cutoff, (normal, point)...) :317.
 * Copier k (stage k+1) lists copier_nfields[k] (field, mode) entries, taken
 * consecutively from copier_fields/copier_modes; 0 entries = `nothing`.
 * `normals`/`points` hold nplanes×ndims doubles.  `capacity` bounds the ghost
 * count (0 = the source's particle count × nplanes).  At most
 * GC_MAX_GHOST_PLANES planes per entry (a 3-D box with its 6 faces, 12
 * edges and 8 corners takes 26).                                          */
#define GC_MAX_GHOST_PLANES 32
int gc_add_ghost(gc_ctx* ctx, int inst, int src_sys, int ncopiers,
                 const int* copier_nfields, const int* copier_fields, const int* copier_modes,
                 int nplanes, const double* normals, const double* points, double cutoff,
                 int64_t capacity, int* handle_out);

/* SystemInteraction(kernel, pfns, system_a[, system_b]) src/Interaction.jl:61,
 * with CubicSplineKernel(h; ndims) src/Kernels.jl:34 or WenlandC2Kernel :108.
 * b_handle = -1 for a self interaction.  pfn_params holds
 * nstages×GC_PFN_NPARAM doubles.  sys_a may be a ghost handle when every
 * stage is `nothing` or InterpolateFieldFn into a virtual system_b: the
 * ghosts' current arrays are interpolated (Trapdoor.jl's ghost_bottom).    */
int gc_add_interaction(gc_ctx* ctx, int inst, int sys_a, int b_handle, int kernel_kind,
                       double h, int nstages, const int* pfn_kinds, const double* pfn_params,
                       int* inter_out);

/* SystemInteraction(...; velocity_adjust_pairwise_fn) src/Interaction.jl:61-66:
 * kind GC_PFN_XSPH (XSPHPfn(epsilon)) or GC_PFN_NONE.  Swept by adjust_v!
 * (:309) in the step's XSPH correction, src/TimeIntegration.jl:421-436.
 * Every instance of a context must set the same kind on an interaction.   */
int gc_set_velocity_adjust(gc_ctx* ctx, int inst, int inter, int kind, double epsilon);

/* VirtualParticleSystem(source, name, n, ndims, mass, c; state_updater,
 * zero_fields, prescribed_v) src/Particles.jl:476-528, one of the
 * integrator's virtual_systems (src/TimeIntegration.jl:364-419, 683).
 * The source `src_sys` (a system handle) holds the virtual particles'
 * positions and fields; it is sorted with the virtual systems each step,
 * never integrated, and moved by prescribed_v·dt after each step.
 * zero_mask: bitmask of 1<<GC_FIELD_* zeroed, with w_sum, before each pass
 * of stage sweeps; prescribed_v: ndims doubles or NULL (zero).  The handle
 * serves as system_b and takes gc_set_updaters.                           */
int gc_add_virtual(gc_ctx* ctx, int inst, int src_sys, int zero_mask, const double* prescribed_v,
                   int* handle_out);

/* ProbeParticleSystem(name, positions | mirror_target; extras, state_updater,
 * prescribed_v) src/ProbeParticles.jl:23-102: n passive observers, measured
 * only by gc_measure_probes.  positions: n×ndims doubles, or NULL with
 * mirror_sys a system handle of n particles whose positions the probes take
 * at each measurement (-1: none).  extras_mask: bitmask of 1<<GC_FIELD_* out
 * of v, rho, p, stress (ns components) and count.  prescribed_v: ndims
 * doubles or NULL; probes move by prescribed_v·dt after each step.  The
 * handle takes gc_set_updaters (one stage) and gc_download_field (x, id,
 * w_sum and the extras, in probe order after a measurement).              */
int gc_add_probe(gc_ctx* ctx, int inst, int64_t n, int ndims, const double* positions, int mirror_sys,
                 int extras_mask, int ns, const double* prescribed_v, int* handle_out);

/* One of the integrator's probe_interactions: SystemInteraction(kernel,
 * pfn, system_a, probe) with pfn GC_PFN_INTERPOLATE or
 * GC_PFN_NEIGHBOR_COUNT (GC_PFN_NPARAM params), swept only by
 * gc_measure_probes.                                                       */
int gc_add_probe_interaction(gc_ctx* ctx, int inst, int sys_a, int probe, int kernel_kind, double h,
                             int pfn_kind, const double* pfn_params, int* inter_out);

/* _measure_probes! src/TimeIntegration.jl:454-502, for every instance: the
 * probe interactions' system_a re-sorted, mirrored probe positions taken,
 * probes sorted by cell, grids built, w_sum and extras zeroed, one sweep,
 * the probes' updaters, probes sorted back by id.                          */
int gc_measure_probes(gc_ctx* ctx);

/* The `state_updater` tuple of a system (src/Particles.jl:200): nstages
 * entries, each a chain of `chain_len[s]` updaters (kinds / GC_UPD_NPARAM
 * params taken consecutively).                                            */
int gc_set_updaters(gc_ctx* ctx, int inst, int sys, int nstages, const int* chain_len,
                    const int* kinds, const double* params);

/* LeapFrogTimeIntegrator(systems, interactions; ghosts, Γ)
 * src/TimeIntegration.jl:53.  The systems list is every system added to
 * the instance in order; the ghosts list every ghost handle.              */
int gc_set_integrator(gc_ctx* ctx, int inst, double damping_gamma);
/* The integrator's kind (the same for every instance of a context):
 * GC_INTEGRATOR_LEAPFROG (default) or GC_INTEGRATOR_RK4, RK4TimeIntegrator
 * src/TimeIntegration.jl:86 (one grid per step, four right-hand-side
 * evaluations, positions advanced once at the end).                       */
enum { GC_INTEGRATOR_LEAPFROG = 0, GC_INTEGRATOR_RK4 = 1 };
int gc_set_integrator_kind(gc_ctx* ctx, int inst, int kind);

/* Validate every instance against instance 0's structure and allocate the
 * device state.  Model-building calls are refused afterwards.              */
int gc_finalize(gc_ctx* ctx);

/* ============================================================ state I/O */
/* Copy one per-particle field between host (Julia AoS layout) and device.
 * `bytes` must equal n×components×8.  Ghost handles accept the ghost fields
 * (x, v, rho, p, stress, idx_original, idx_boundary, normals).              */
int gc_upload_field(gc_ctx* ctx, int inst, int handle, int field, const void* host, size_t bytes);
int gc_download_field(gc_ctx* ctx, int inst, int handle, int field, void* host, size_t bytes);
/* Many fields at once, one synchronisation for all of them (same layouts
 * and checks as the single-field calls; nothing is written when any entry
 * is invalid).                                                            */
typedef struct gc_field_io {
    int inst, handle, field;
    int32_t pad;
    void* host;
    size_t bytes;
} gc_field_io;
int gc_upload_fields(gc_ctx* ctx, int n, const gc_field_io* io);
int gc_download_fields(gc_ctx* ctx, int n, const gc_field_io* io);
/* Current particle count of a handle (ghost counts change every step).    */
int gc_get_count(gc_ctx* ctx, int inst, int handle, int64_t* n_out);

/* ============================================================ stepping */
int gc_set_precision(gc_ctx* ctx, int mode);

/* time_integrate!(::LeapFrogTimeIntegrator, nsteps, ...) loop body
 * src/TimeIntegration.jl:645-693 for every instance, dt = CFL·h_min/c_max
 * per instance (:598).  Printing and HDF5 output stay on the Julia side.   */
int gc_step(gc_ctx* ctx, int nsteps, double cfl);

int gc_get_stats(gc_ctx* ctx, gc_stats* out);

/* ======================================================== measurement */
/* The CUDA stream every kernel of the context is launched on (a
 * cudaStream_t), for callers that time work with CUDA events.            */
int gc_stream(gc_ctx* ctx, void** stream_out);
/* When on, every pair-sweep launch is bracketed by CUDA events on the
 * context's stream; gc_get_stats reports their summed time.  Resets the
 * sweep counters.                                                         */
int gc_set_profiling(gc_ctx* ctx, int on);
/* Step scheduling (no counterpart in the reference, whose loop is host
 * code).  on = 1 (default): after one exactly-sized step, gc_step captures
 * a step sized from buffer capacities as a CUDA graph (one per buffer
 * parity) and replays it, with no host round trip per step; every
 * `sync_every` steps (default 32) the host verifies the window, grows
 * capacities to `cap_margin` (>= 1, default 1.5; 0 keeps the current
 * value) times the largest plan seen, and re-runs the window exactly from
 * a device snapshot if a plan outgrew them.  Results are bit-identical to
 * on = 0 (every step sized by one host read of its plan).  The environment
 * variable GC_GRAPHS=0 forces on = 0.                                     */
int gc_set_graphs(gc_ctx* ctx, int on, int sync_every, double cap_margin);
/* cfg = -1 (default): autotune — the first steps of a context time every
 * sweep configuration once per (system, stage) sweep and keep the fastest.
 * 0 <= cfg < GC_NUM_SWEEP_CONFIGS: use that one everywhere.  The
 * environment variable GC_FORCE_CFG=<cfg> has the same effect.            */
int gc_set_sweep_config(gc_ctx* ctx, int cfg);
/* Measured FP64 FMA issue rate of the device in TFLOP/s (2 flops per FMA):
 * the compute ceiling of the FP64 pair sweep.                             */
int gc_measure_fp64_peak(gc_ctx* ctx, double* tflops_out);
/* Measured FP32 FMA issue rate of the device in TFLOP/s (2 flops per FMA):
 * the compute ceiling of the FP32-compensated pair sweep.                 */
int gc_measure_fp32_peak(gc_ctx* ctx, double* tflops_out);

/* ======================================================== phase hooks */
/* The same device kernels, one reference phase at a time (parity tests and
 * the per-phase Julia entry points).                                      */

/* sort_particles!(ps, cutoff, ...) src/Sorting.jl:157.  perm_out (may be
 * NULL) receives n 1-based source indices: new position k holds old
 * particle perm_out[k].                                                   */
int gc_sort_system(gc_ctx* ctx, int inst, int handle, double cutoff, int64_t* perm_out);

/* create_grid!(si) src/Interaction.jl:123.  Outputs (each may be NULL):
 * cell_start (1-based, length ncells+1, `cap` entries available),
 * mingridx (ND doubles), ngridx (ND int64), ncells.                        */
int gc_build_grid(gc_ctx* ctx, int inst, int inter, int64_t* cell_start_out, int64_t cap,
                  double* mingridx_out, int64_t* ngridx_out, int64_t* ncells_out);

/* generate_ghosts!(ge) src/GhostParticles.jl:344 (unsorted, generation order) */
int gc_generate_ghosts(gc_ctx* ctx, int inst, int ghost);
/* update_ghost_kinematics!(ge) src/GhostParticles.jl:404                  */
int gc_update_ghost_kinematics(gc_ctx* ctx, int inst, int ghost);
/* update_ghost!(ge, stage) src/GhostParticles.jl:277,423 (stage is 1-based) */
int gc_update_ghost(gc_ctx* ctx, int inst, int ghost, int stage);

/* sweep!(si, stage) src/Interaction.jl:292 — adds this interaction's pair
 * terms of `stage` (1-based) into the current accumulators.  Requires a
 * grid from gc_build_grid.                                                */
int gc_sweep(gc_ctx* ctx, int inst, int inter, int stage);

/* update_state!(ps, stage, dt) src/Particles.jl:542 (stage 1-based).     */
int gc_update_state(gc_ctx* ctx, int inst, int sys, int stage, double dt);

/* Accepted-pair count per system_a particle of an interaction, from the
 * grid of the last gc_build_grid / gc_step (n_a int32 values).             */
int gc_neighbor_counts(gc_ctx* ctx, int inst, int inter, int32_t* counts_out, int64_t n);

/* ============================================= allocation-free variant */
/* No counterpart in the reference.  The stable cell-key sort permutation of
 * gc_sort_system for callers that cannot call cudaMalloc — hosts whose
 * device memory is handed in full to their own pool allocator, and
 * latency-critical loops that cannot afford cudaMalloc/cudaFree's implicit
 * device synchronisation.  It allocates nothing: its scratch is a fixed
 * static device array (about 2 MB, held by every GPU that loads the library
 * until exit), so n is limited to 65536 particles and the key lattice's
 * bounding box to 131072 cells (GC_ERR_CAPACITY beyond either).
 * x_planar: device array, ndims×n doubles, component-major (x of all
 * particles, then y, ...).  perm_out: device array of n int32 receiving the
 * 0-based source index of each sorted position (the order of
 * `sort_particles!`, src/Sorting.jl:157, for keys floor(x_d/cutoff)).
 * stream: a cudaStream_t (NULL for the default stream); the call returns
 * after the stream has finished its work.  Each call resolves the scratch
 * array's device address on the current device (cudaGetSymbolAddress,
 * which allocates nothing).  Calls share the scratch array; calls that
 * overlap on the GPU race on it.                                           */
int gc_cell_sort_perm_noalloc(const double* x_planar, int64_t n, int ndims, double cutoff,
                              int32_t* perm_out, void* stream);

/* ============================================================= serving */
/* No counterpart in the reference (one simulation per Julia process).  A
 * server steps many simulations ("requests") on one device: requests are
 * admitted in arrival order while their estimated device memory fits
 * `hbm_budget_bytes`, simulations of one model structure are packed into
 * shared contexts ("batches") and stepped together, batches of different
 * structures run concurrently.  At every round boundary finished requests
 * leave, queued ones join, and each batch advances at most `round_steps`
 * steps (fewer when a request needs fewer to finish, so every request ends
 * exactly at its own step count).  A request's result is bit-identical to
 * the same simulation run alone in a context of the same precision.       */
typedef struct gc_server gc_server;
typedef struct gc_serve_stats {
    int64_t queued, running, batches;
    int64_t rounds, repacks;
    int64_t particle_steps;          /* moving particles × steps, all requests */
    int64_t device_bytes_reserved;   /* estimates of the admitted requests     */
    double repack_seconds;           /* host time spent rebuilding batches     */
    int64_t repack_instances;        /* requests placed by those rebuilds      */
    int64_t retries;                 /* requests run again alone, from their
                                        submitted state, after their batch's
                                        step failed                          */
} gc_serve_stats;
enum { GC_REQ_FAILED = -1, GC_REQ_QUEUED = 0, GC_REQ_RUNNING = 1, GC_REQ_DONE = 2 };

int gc_serve_create(int device, size_t hbm_budget_bytes, int round_steps, int precision, gc_server** out);
int gc_serve_destroy(gc_server* srv);
const char* gc_serve_last_error(gc_server* srv);
/* `model`: a context with one instance built by gc_instance_add/gc_add_*
 * and filled by gc_stage_field, not finalized.  The server owns it from
 * here on (released by gc_serve_release).  Runs `nsteps` steps at `cfl`.  */
int gc_serve_submit(gc_server* srv, gc_ctx* model, int nsteps, double cfl, int64_t* req_out);
/* One round: admit, repack, step every batch, retire finished requests
 * (their fields are copied to host memory).                              */
int gc_serve_pump(gc_server* srv, int* ncompleted);
/* state: GC_REQ_*; times in seconds since gc_serve_create (-1: not yet). */
int gc_serve_poll(gc_server* srv, int64_t req, int* state, int64_t* steps_done, double* t_submit,
                  double* t_admit, double* t_done);
/* A finished request's field, same layout as gc_download_field.          */
int gc_serve_download(gc_server* srv, int64_t req, int handle, int field, void* host, size_t bytes);
int gc_serve_release(gc_server* srv, int64_t req);
int gc_serve_get_stats(gc_server* srv, gc_serve_stats* out);

/* Before gc_finalize: keep a copy of a field in host memory; gc_finalize
 * (or a server admitting the request) uploads it.  Same layout and checks
 * as gc_upload_field.                                                     */
int gc_stage_field(gc_ctx* ctx, int inst, int handle, int field, const void* host, size_t bytes);

#ifdef __cplusplus
}
#endif
#endif /* GRASPH_CUDA_H */
