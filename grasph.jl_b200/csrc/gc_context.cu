// gc_context.cu — host runtime of libgrasph_cuda.so: model building, device
// memory, the per-step schedule and the C ABI of include/grasph_cuda.h.
//
// One step (src/TimeIntegration.jl:645-693) is issued as:
//   plan    bounding boxes → sort/grid/ghost plans → one host read of the
//           required cell counts (buffers grow here, before any mutation)
//   sort    stable counting sort of every moving system (key, histogram,
//           scan, scatter, per-cell fix-up, gather into the other buffer)
//   ghosts  flag → scan → fill (generation order) → sort
//   grids   cell histogram of every system_b → scan = CSR cell_start
//   half    v += dt/2·dvdt, rho += dt/2·drhodt, q0 snapshot, reset to source
//   stages  updaters → ghost copiers → one fused sweep per (system, stage)
//   full    damping, q = q0 + dt·dqdt, x += dt·v
// All launches go to the context's stream; the host reads device memory
// once per step (the plan) and once per gc_step call (the error word).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "gc_force.h"
#include "gc_internal.h"
#include "gc_kernels.h"
#include "gc_update.h"

using namespace gc;

namespace {

// ------------------------------------------------------------ host model
struct HUpd {
    int kind;
    double prm[GC_UPD_NPARAM];
};
struct HSys {
    int kind = 0, nd = 2, ns = 0, nvort = 0;
    int64_t n = 0;
    double mass = 0, c = 0, srcv[3] = {0, 0, 0}, srcrho = 0;
    bool upd_set = false;
    std::vector<std::vector<HUpd>> upd;
    bool vsrc = false;  // the source of a virtual system (not integrated)
    bool probe = false; // a probe's own arrays (the count extra lives in drhodt)
};
enum { H_SYS = 0, H_DYN = 1, H_STATIC = 2, H_GHOST = 3, H_VIRT = 4 };
// VirtualParticleSystem src/Particles.jl:476-528 over source system `src`
struct HVirt {
    int src = 0;
    int zmask = 0;
    double pv[3] = {0, 0, 0};
    bool upd_set = false;
    std::vector<std::vector<HUpd>> upd;
    bool probe = false;  // ProbeParticleSystem src/ProbeParticles.jl:23-102 (source = its own arrays)
    int mirror = -1;     // its mirror_target system, or -1
};
struct HHandle {
    int type = H_SYS, idx = 0;
    double normal[3] = {0, 0, 0}, point[3] = {0, 0, 0}, beta = 0, ljcut = 0;
};
struct HGhost {
    int src = 0;
    double cutoff = 0;
    int nplanes = 0;
    double normals[GC_MAX_GHOST_PLANES][3] = {}, points[GC_MAX_GHOST_PLANES][3] = {};
    std::vector<std::vector<std::pair<int, int>>> copiers;
    bool ex_p = false, ex_stress = false;
};
struct HInter {
    int a = 0, b = -1, kk = 0, nstages = 0;
    double H = 0;
    std::vector<int> pk;
    std::vector<std::array<double, GC_PFN_NPARAM>> pp;
    int vk = GC_PFN_NONE;  // velocity_adjust_pairwise_fn
    double veps = 0.0;
    bool probe = false;    // one of the integrator's probe_interactions
    int ag = -1;           // system_a is this ghost system (a = its source); InterpolateFieldFn only
};
struct HStaged {
    int handle, field;
    std::vector<char> bytes;  // the caller's layout, as gc_upload_field takes it
};
struct HInst {
    std::vector<HSys> sys;
    std::vector<HHandle> handles;
    std::vector<int> sys_handle;
    std::vector<HGhost> ghosts;
    std::vector<HInter> inters;
    std::vector<HVirt> virts;
    double gamma = 0;
    int integ = GC_INTEGRATOR_LEAPFROG;
    double cfl = NAN;              // own CFL number (serving); NaN: gc_step's
    std::vector<HStaged> staged;   // fields given before gc_finalize
};

// ---------------------------------------------------------- device state
enum { F_X = 0, F_V, F_RHO, F_DVDT, F_DRHODT, F_P, F_STRESS, F_SR, F_VORT, F_STRAIN, F_STRAINP, F_VADJ, NF };

struct DSlot {
    int64_t N = 0;
    int nd = 2, ns = 0, nvort = 0, kind = 0;
    int ncomp[NF] = {};
    double* f[2][NF] = {};
    int32_t* id[2] = {};
    int cur = 0;
    double *q0v = nullptr, *q0rho = nullptr, *aux = nullptr;
    double *accv = nullptr, *accrho = nullptr;  // RK4 accumulators (allocated on first use)
    int32_t* inst_of = nullptr;
    SysInst* d_inst = nullptr;
    std::vector<SysInst> h_inst;
    double *d_mass = nullptr, *d_c = nullptr;
    float *d_massf = nullptr, *d_cf = nullptr;
    float* fpk = nullptr;      // FP32 pack for the FP32-compensated sweep
    int64_t cap_fpk = 0;
    int64_t xpk_epoch = -1;    // pack_epoch the FP64 position copy was made in
    bool xpk_static = false;   // position copy of a system that does not move is current
    bool written = false;      // some functor writes this system
    bool moving = true;        // sorted and integrated every step
    bool vsrc = false;         // source of a virtual system: never integrated
    bool probe = false;        // a probe's arrays
    bool vmoves = false;       // a virtual system over it has a non-zero prescribed_v
    bool xmoves() const { return moving || vmoves; }  // positions change every step
    bool sorted_once = false;  // static systems: sorted since the last upload
    std::vector<int64_t> nonzero_kin;  // per instance: uploaded v/dvdt/drhodt nonzero
    // updaters: [stage][chain] -> per-instance UpdInst device array
    std::vector<std::vector<UpdInst*>> d_upd;
    std::vector<std::vector<int>> upd_kind;
    bool upd_set = false;
    int nupd = 0;
    // the fused half step of this pack_epoch already ran the stage-1
    // updaters and packed the stage-1 records (mode, record stress width)
    int64_t upd_fused_epoch = -1;
    int64_t pack_done_epoch = -1;
    int pack_done_stage = 0, pack_done_mode = -1, pack_done_ns = -1;
    // warp groups of this system's particles (one grid's columns)
    int2* groups = nullptr;
    int64_t* d_ngroups = nullptr;
    int32_t *gcnt = nullptr, *goff = nullptr;
    int64_t cap_gcols = 0;
    int64_t groups_key = -1, groups_ver = -1;
    double* F(int k) { return f[cur][k]; }
    double* A(int k) { return f[cur ^ 1][k]; }
};

struct DGhost {
    int src = 0, nplanes = 0, nd = 2, ns = 0;
    int64_t CAP = 0;
    // warp groups of the ghosts (system_b side of an XSPH sweep) and that
    // sweep's ghost-indexed sums before they are added to the source
    int2* groups = nullptr;
    int64_t* d_ngroups = nullptr;
    int32_t *gcnt = nullptr, *goff = nullptr;
    int64_t cap_gcols = 0;
    int64_t groups_key = -1, groups_ver = -1;
    double* gadj = nullptr;
    double* x[2] = {};
    int32_t *io[2] = {}, *ib[2] = {}, *ginst[2] = {};
    int cur = 0;
    double *normals = nullptr, *v = nullptr, *rho = nullptr, *p = nullptr, *stress = nullptr, *aux = nullptr;
    int32_t *flags = nullptr, *pos = nullptr;
    int64_t* d_count = nullptr;
    GhostInst* d_gh = nullptr;
    std::vector<GhostInst> h_gh;
    SysInst* d_inst = nullptr;
    std::vector<SysInst> h_inst;
    double *d_mass = nullptr, *d_c = nullptr;
    float* fpk = nullptr;
    int64_t cap_fpk = 0;
    int64_t xpk_epoch = -1;
    bool xpk_static = false;  // never set: ghosts are regenerated every step
    std::vector<std::vector<std::pair<int, int>>> copiers;
    bool ex_p = false, ex_stress = false;
    int64_t need_slot = -1;  // index into need[] for its sort cells
};

// A virtual system on the device: its w_sum over the source slot's packed
// particles, per-instance prescribed_v and updater chains.
struct DVirt {
    int src = 0;
    int zmask = 0;
    double* wsum = nullptr;
    VirtInst* d_vi = nullptr;
    bool moves = false;
    bool upd_set = false;
    int nupd = 0;
    std::vector<std::vector<UpdInst*>> d_upd;
    std::vector<std::vector<int>> upd_kind;
    bool probe = false;
    int mirror = -1;             // mirror_target slot of a probe
    double* wsum_alt = nullptr;  // a probe's w_sum, reordered by id at measurement
};

// system_b kinds of the host side; BT_VIRTUAL sweeps with the device's
// one-sided boundary forms (BT_GHOST) over the source slot's arrays
constexpr int BT_VIRTUAL = 5;

struct DInter {
    int a = 0, btype = BT_SELF, bslot = -1, bghost = -1, bvirt = -1, kk = 0, nstages = 0;
    bool two_sided = false;  // some stage writes system_b too (a second, system_b-side sweep)
    bool two_fluid = false;  // FluidPfn stages are the two-sided fluid x fluid form
    bool probe = false;      // a probe interaction: swept by gc_measure_probes only
    bool vadj = false;       // pk[nstages] is the velocity-adjust functor (XSPH)
    int ag = -1;             // system_a is this ghost system (a = its source slot)
    std::vector<int> pk;
    GridInst* d_gi = nullptr;
    GridInst* d_gi_b = nullptr;  // system_b side: system_a's mass and sound speed as the neighbour's
    std::vector<GridInst> h_gi;
    std::vector<PfnInst*> d_pi;
    int32_t* cs = nullptr;     // CSR over system_b
    int32_t* cs_a = nullptr;   // CSR over system_a (two-sided)
    int32_t* counts = nullptr; // per system_a particle
    int64_t cap_cells = 0;
    int64_t need_slot = -1;
    bool grid_valid = false;
    int64_t cells = 0;      // packed cells of the current grid
    int64_t grid_ver = -1;  // bumps at every rebuild
    int64_t csa_ver = -1;   // grid version cs_a was built for
    // one-sided against a system_b whose positions do not change: its CSR
    // stays current while the grid's geometry does, and a step's count and
    // scan are skipped on the device when the geometry is unchanged
    int* d_keep = nullptr;          // [0] cs is current for d_gi_prev, [1] this step's grid equals it
    GridInst* d_gi_prev = nullptr;  // geometry cs was last counted on, per instance
    int32_t* hist = nullptr;        // its own histogram (batched still grids): zero between uses
    int64_t cap_hist = 0;
};

// One captured step: valid for the buffer parities `pre` (cur of every slot,
// then of every ghost), leaves them at `post`.
struct StepGraph {
    std::vector<char> pre, post;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;  // kernels per replay
    // event-record nodes of the sweep timers: (node, pair index, 0 start / 1 end)
    std::vector<std::array<int64_t, 2>> ev_slots;
    std::vector<cudaGraphNode_t> ev_nodes;
};

// Copy of the carried state of a moving slot at the last verified step.
struct Snapshot {
    double* f[NF] = {};
    int32_t* id = nullptr;
    int cur = 0;
    int64_t n = 0;  // particles copied (capacity of the buffers)
};

}  // namespace

struct gc_ctx {
    int device = 0;
    size_t budget = 0, allocated = 0;
    cudaStream_t stream = nullptr;
    // device memory: cudaMalloc/cudaFree, or (contexts a server builds) a
    // stream-ordered pool that keeps freed memory for the next context, so
    // building and dropping a context neither maps memory nor waits on the
    // whole device
    cudaMemPool_t pool = nullptr;
    std::string err;
    std::vector<HInst> inst;
    bool finalized = false;
    int precision = GC_PRECISION_FP64;
    // structure
    std::vector<DSlot> slots;
    std::vector<DGhost> ghosts;
    std::vector<DInter> inters;
    std::vector<DVirt> virts;
    int nstages = 0;
    bool xsph = false;  // some interaction has a velocity-adjust functor: v_adjustment is carried
    // scratch
    int32_t *key = nullptr, *perm = nullptr, *hist = nullptr, *start = nullptr, *fill = nullptr, *scan_tmp = nullptr;
    int64_t cap_keyN = 0, cap_cells = 0, cap_scan = 0;
    unsigned long long* bbox_scratch = nullptr;
    int* d_err = nullptr;
    int* d_unsorted = nullptr;                     // a slot sort's keys were out of order
    unsigned long long* d_sorts_in_order = nullptr;  // slot sorts that found their keys in order
    unsigned long long* d_incons = nullptr;
    int64_t* d_need = nullptr;
    int64_t* h_need = nullptr;  // pinned
    int nneed = 0;
    int nplan = 0;  // entries of d_plan_args (the steps' interactions)
    int64_t* d_total_cells = nullptr;  // device copy of the current sort's cell total
    int64_t grid_version = 0;
    int num_sms = 148;
    int force_cfg = -1;  // fixed sweep configuration, -1: autotune
    // autotuning: per (slot, stage, functor) sweep, TUNE_ROUNDS timed
    // launches per configuration, then the fastest by its best launch
    static constexpr int TUNE_ROUNDS = 2;
    struct Tune {
        int best = -1, next = 0;
        double ms[NUM_FORCE_CFG] = {};
    };
    std::map<int64_t, Tune> tune;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tune_ev;
    std::vector<std::pair<int64_t, int>> tune_rec;  // (key, cfg) of each used tune_ev pair
    int64_t tune_version = 0;
    // host I/O staging (device side of AoS <-> planar transposes)
    double* staging = nullptr;
    int64_t cap_staging = 0;  // doubles
    int* d_ioflags = nullptr;  // per uploaded field: nonzero seen
    int cap_ioflags = 0;
    // stats / profiling
    int64_t steps_done = 0, resorts = 0;
    int last_status = 0;
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    size_t ev_used = 0;
    double sweep_ms = 0;
    int64_t sweep_launches = 0;
    unsigned long long* d_pairs = nullptr;
    // graph stepping: steps sized from capacities (no host read per step),
    // captured once per buffer parity and replayed; verified every
    // `sync_every` steps against a snapshot, rolled back and re-run exactly
    // when a capacity was exceeded
    bool graphs_on = true;
    int sync_every = 32;
    double cap_margin = 1.5;       // capacity = margin × largest need seen
    bool capmode = false;          // current step sized from capacities
    bool capturing = false;        // no allocation may happen
    bool exact_done = false;       // an exact step ran since the last change
    int64_t alloc_epoch = 0;       // bumps at every (re)allocation
    int64_t graphs_epoch = -1;     // alloc_epoch the graphs were captured at
    int graphs_key = -1;           // precision/config/profiling the graphs saw
    std::vector<StepGraph> graphs;
    std::vector<int64_t> need_max;  // per plan entry, largest need seen
    int64_t* d_need_max = nullptr;
    int64_t* h_need_max = nullptr;  // pinned
    int64_t* d_need_cap = nullptr;  // per plan entry, the cells capacity mode sizes for
    GridPlanArgs* d_plan_args = nullptr;  // grid plan arguments of every interaction
    std::vector<Snapshot> snaps;    // per slot (moving slots only)
    int64_t graph_steps = 0, rollbacks = 0;
    int64_t pack_epoch = 0;  // bumps at the start of every issued step (never rolled back)
    double params_cfl = NAN;  // CFL number the per-instance parameters were pushed for
    bool params_dirty = true;
};

namespace {

void drop_graphs(gc_ctx* ctx);
void invalidate_steps(gc_ctx* ctx);
struct DInter;
GridPlanArgs grid_plan_args(gc_ctx* ctx, DInter& D);

// ---------------------------------------------------------------- errors
int seterr(gc_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
    return code;
}

#define CU(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return seterr(ctx, GC_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                          __FILE__, __LINE__);                                                 \
    } while (0)

#define TRY(expr)            \
    do {                     \
        int st_ = (expr);    \
        if (st_) return st_; \
    } while (0)

// Host<->device copy ordered after everything already on the context's
// stream, complete on return.  (A plain cudaMemcpy runs on the legacy default
// stream, which does not wait for the context's non-blocking stream.)
int hcopy(gc_ctx* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    if (bytes == 0) return GC_OK;
    CU(cudaMemcpyAsync(dst, src, bytes, kind, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GC_OK;
}

template <class T>
int dalloc(gc_ctx* ctx, T** p, size_t count) {
    if (ctx->capturing) return seterr(ctx, GC_ERR_STATE, "allocation inside a step capture");
    ctx->alloc_epoch++;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    if (ctx->budget && ctx->allocated + bytes > ctx->budget)
        return seterr(ctx, GC_ERR_OOM, "device budget of %zu bytes exceeded", ctx->budget);
    void* q = nullptr;
    cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(&q, bytes, ctx->pool, ctx->stream) : cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return seterr(ctx, GC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    CU(cudaMemsetAsync(q, 0, bytes, ctx->stream));
    ctx->allocated += bytes;
    *p = (T*)q;
    return GC_OK;
}

// Device memory back to where it came from (stream-ordered into the pool).
void dev_free(gc_ctx* ctx, void* p) {
    if (!p) return;
    if (ctx->pool) cudaFreeAsync(p, ctx->stream);
    else cudaFree(p);
}

template <class T>
void dfree(gc_ctx* ctx, T*& p, size_t count) {
    if (p) {
        ctx->alloc_epoch++;
        dev_free(ctx, p);
        size_t bytes = count * sizeof(T);
        ctx->allocated -= std::min(ctx->allocated, bytes ? bytes : 16);
        p = nullptr;
    }
}

int sys_comps(const HSys& s, int field) {
    switch (field) {
        case GC_FIELD_X: case GC_FIELD_V: case GC_FIELD_DVDT: case GC_FIELD_V_ADJUSTMENT: return s.nd;
        case GC_FIELD_RHO: case GC_FIELD_DRHODT: case GC_FIELD_ID: return 1;
        case GC_FIELD_P: return s.kind >= GC_SYS_FLUID ? 1 : -1;
        case GC_FIELD_STRESS: case GC_FIELD_STRAIN_RATE: return s.kind >= GC_SYS_STRESS ? s.ns : -1;
        case GC_FIELD_VORTICITY: return s.kind == GC_SYS_ELASTOPLASTIC ? s.nvort : -1;
        case GC_FIELD_STRAIN: case GC_FIELD_STRAIN_P: return s.kind == GC_SYS_ELASTOPLASTIC ? s.ns : -1;
        case GC_FIELD_COUNT: return s.probe ? 1 : -1;
        default: return -1;
    }
}

int field_slot(int field) {
    switch (field) {
        case GC_FIELD_X: return F_X;
        case GC_FIELD_V: return F_V;
        case GC_FIELD_RHO: return F_RHO;
        case GC_FIELD_DVDT: return F_DVDT;
        case GC_FIELD_DRHODT: return F_DRHODT;
        case GC_FIELD_P: return F_P;
        case GC_FIELD_STRESS: return F_STRESS;
        case GC_FIELD_STRAIN_RATE: return F_SR;
        case GC_FIELD_VORTICITY: return F_VORT;
        case GC_FIELD_STRAIN: return F_STRAIN;
        case GC_FIELD_STRAIN_P: return F_STRAINP;
        case GC_FIELD_V_ADJUSTMENT: return F_VADJ;
        case GC_FIELD_COUNT: return F_DRHODT;  // a probe's count extra
        default: return -1;
    }
}

double kernel_norm(int kind, int nd, double H) {
    const double pi = 3.141592653589793;
    if (kind == GC_KERNEL_CUBIC_SPLINE) {
        if (nd == 1) return 2.0 / (3.0 * H);
        if (nd == 2) return 10.0 / ((7.0 * pi) * (H * H));
        return 1.0 / (pi * (H * H * H));
    }
    if (nd == 2) return 7.0 / ((64.0 * pi) * (H * H));
    return 21.0 / ((256.0 * pi) * (H * H * H));
}

// Does stage `stage` (1-based; nstages + 1 is the velocity-adjust functor)
// of an interaction also write system_b?  XSPHPfn's coupled form writes every
// system_b kind: a wrapper's system, or a ghost's source at the ghost index.
bool b_side_at(const DInter& D, int stage) {
    const int pk = D.pk[stage - 1];
    if (pk == GC_PFN_COUNT) return D.btype != BT_SELF && D.btype != BT_GHOST && D.bslot >= 0;
    if (pk == GC_PFN_XSPH) return D.btype != BT_SELF;
    if (pk == GC_PFN_FLUID_SOLID || pk == GC_PFN_INTERPOLATE || pk == GC_PFN_NEIGHBOR_COUNT) return true;
    return pk == GC_PFN_FLUID && D.two_fluid;
}

// Functor/system_b combinations implemented (the CPU oracle refuses the same).
int check_combo(gc_ctx* ctx, const HInst& I, const HInter& it, int pk) {
    const HSys& a = I.sys[it.a];
    if (pk == GC_PFN_NONE) return GC_OK;
    if (pk == GC_PFN_XSPH)
        return seterr(ctx, GC_ERR_UNSUPPORTED, "XSPHPfn is swept as velocity_adjust_pairwise_fn, not as a stage");
    if (pk < 0 || pk > GC_PFN_NEIGHBOR_COUNT) return seterr(ctx, GC_ERR_ARG, "bad functor kind %d", pk);
    if (it.ag >= 0) {
        // a ghost system_a (Trapdoor.jl's ghost_bottom): InterpolateFieldFn
        // into a virtual system, reading the ghosts' current arrays
        if (pk != GC_PFN_INTERPOLATE || it.b < 0 || I.handles[it.b].type != H_VIRT || I.virts[I.handles[it.b].idx].probe)
            return seterr(ctx, GC_ERR_UNSUPPORTED, "a ghost system_a sweeps only InterpolateFieldFn into a virtual system");
        const int m = (int)it.pp.back()[0];
        if ((m & (1 << GC_FIELD_STRESS)) && !I.ghosts[it.ag].ex_stress)
            return seterr(ctx, GC_ERR_UNSUPPORTED, "InterpolateFieldFn(:stress) from ghosts that carry no stress");
    }
    if (pk == GC_PFN_NEIGHBOR_COUNT) {  // the (real, probe) method, src/PairwiseFunctors.jl:455
        if (it.b < 0 || I.handles[it.b].type != H_VIRT || !I.virts[I.handles[it.b].idx].probe)
            return seterr(ctx, GC_ERR_UNSUPPORTED, "NeighborCountFn needs a probe as system_b");
        return GC_OK;
    }
    if (pk == GC_PFN_INTERPOLATE) {
        // the (real, virtual) method, src/PairwiseFunctors.jl:424; the fields exist on both sides
        if (it.b < 0 || I.handles[it.b].type != H_VIRT)
            return seterr(ctx, GC_ERR_UNSUPPORTED, "InterpolateFieldFn needs a virtual system as system_b");
        const HSys& s = I.sys[I.virts[I.handles[it.b].idx].src];
        const int m = (int)it.pp.back()[0];
        if (m & ~((1 << GC_FIELD_V) | (1 << GC_FIELD_RHO) | (1 << GC_FIELD_STRESS)))
            return seterr(ctx, GC_ERR_UNSUPPORTED, "InterpolateFieldFn: fields other than v, rho, stress");
        if ((m & (1 << GC_FIELD_STRESS)) && !(a.kind >= GC_SYS_STRESS && s.kind >= GC_SYS_STRESS && a.ns == s.ns))
            return seterr(ctx, GC_ERR_ARG, "InterpolateFieldFn(:stress) needs stress of one size on both systems");
        return GC_OK;
    }
    if (pk == GC_PFN_FLUID_SOLID) {
        // only the two-sided (system, system) method exists, src/PairwiseFunctors.jl:494
        if (a.kind < GC_SYS_FLUID) return seterr(ctx, GC_ERR_ARG, "FluidSolidPfn needs system_a's pressure");
        if (it.b < 0 || I.handles[it.b].type != H_SYS)
            return seterr(ctx, GC_ERR_UNSUPPORTED, "FluidSolidPfn needs a real system as system_b");
        return GC_OK;
    }
    if (pk == GC_PFN_FLUID && a.kind < GC_SYS_FLUID) return seterr(ctx, GC_ERR_ARG, "FluidPfn needs a pressure field");
    if ((pk == GC_PFN_CAUCHY_FLUID || pk == GC_PFN_STRAIN_RATE) && a.kind < GC_SYS_STRESS)
        return seterr(ctx, GC_ERR_ARG, "functor needs a stress system");
    if (pk == GC_PFN_STRAIN_RATE_VORTICITY && a.kind != GC_SYS_ELASTOPLASTIC)
        return seterr(ctx, GC_ERR_ARG, "StrainRateVorticityPfn needs an elasto-plastic system");
    if (pk == GC_PFN_CAUCHY_FLUID || pk == GC_PFN_STRAIN_RATE || pk == GC_PFN_STRAIN_RATE_VORTICITY) {
        if (a.nd == 2 && !(a.ns == 3 || a.ns == 4)) return seterr(ctx, GC_ERR_UNSUPPORTED, "2-D stress needs NS 3 or 4");
        if (a.nd == 3 && a.ns != 6) return seterr(ctx, GC_ERR_UNSUPPORTED, "3-D stress needs NS 6");
    }
    if (it.b < 0) return GC_OK;
    const HHandle& h = I.handles[it.b];
    if (h.type == H_VIRT) {
        // virtual system_b: the one-sided boundary forms (:193, :286, :37, :97)
        const HSys& s = I.sys[I.virts[h.idx].src];
        if (pk == GC_PFN_COUNT) return seterr(ctx, GC_ERR_UNSUPPORTED, "counting functor with a virtual system");
        if (pk == GC_PFN_FLUID && s.kind < GC_SYS_FLUID) return seterr(ctx, GC_ERR_ARG, "system_b has no pressure field");
        if (pk == GC_PFN_CAUCHY_FLUID && !(s.kind >= GC_SYS_STRESS && s.ns == a.ns))
            return seterr(ctx, GC_ERR_ARG, "system_b has no stress of system_a's size");
        return GC_OK;
    }
    if (pk == GC_PFN_COUNT) return h.type == H_GHOST ? seterr(ctx, GC_ERR_UNSUPPORTED, "counting functor with ghosts") : GC_OK;
    if (h.type == H_DYN || h.type == H_STATIC) return GC_OK;
    if (h.type == H_GHOST) {
        const HGhost& g = I.ghosts[h.idx];
        if (pk == GC_PFN_FLUID && !g.ex_p) return seterr(ctx, GC_ERR_UNSUPPORTED, "FluidPfn with ghosts needs a :p copier");
        if (pk == GC_PFN_CAUCHY_FLUID && !g.ex_stress)
            return seterr(ctx, GC_ERR_UNSUPPORTED, "CauchyFluidPfn with ghosts needs a :stress copier");
        return GC_OK;
    }
    const HSys& b = I.sys[h.idx];
    if (pk == GC_PFN_FLUID)  // two-sided between two fluid systems, one-sided otherwise
        return b.kind >= GC_SYS_FLUID ? GC_OK : seterr(ctx, GC_ERR_ARG, "system_b has no pressure field");
    if (pk == GC_PFN_CAUCHY_FLUID) return seterr(ctx, GC_ERR_UNSUPPORTED, "two-sided CauchyFluidPfn not implemented");
    return GC_OK;
}

// ------------------------------------------------------------- finalize
bool same_structure(const HInst& a, const HInst& b, std::string& why) {
    if (a.integ != b.integ) return why = "integrator kind", false;
    if (a.sys.size() != b.sys.size()) return why = "system count", false;
    if (a.virts.size() != b.virts.size()) return why = "virtual systems", false;
    for (size_t v = 0; v < a.virts.size(); ++v) {
        const HVirt &x = a.virts[v], &y = b.virts[v];
        if (x.src != y.src || x.zmask != y.zmask || x.upd_set != y.upd_set || x.upd.size() != y.upd.size() ||
            x.probe != y.probe || x.mirror != y.mirror)
            return why = "virtual systems or probes", false;
        for (size_t t = 0; t < x.upd.size(); ++t) {
            if (x.upd[t].size() != y.upd[t].size()) return why = "virtual updaters", false;
            for (size_t q = 0; q < x.upd[t].size(); ++q)
                if (x.upd[t][q].kind != y.upd[t][q].kind) return why = "virtual updaters", false;
        }
    }
    for (size_t s = 0; s < a.sys.size(); ++s) {
        const HSys &x = a.sys[s], &y = b.sys[s];
        if (x.kind != y.kind || x.nd != y.nd || x.ns != y.ns || x.vsrc != y.vsrc) return why = "system kinds", false;
        if (x.upd_set != y.upd_set || x.upd.size() != y.upd.size()) return why = "updater tuples", false;
        for (size_t t = 0; t < x.upd.size(); ++t) {
            if (x.upd[t].size() != y.upd[t].size()) return why = "updater chains", false;
            for (size_t q = 0; q < x.upd[t].size(); ++q)
                if (x.upd[t][q].kind != y.upd[t][q].kind) return why = "updater kinds", false;
        }
    }
    if (a.handles.size() != b.handles.size()) return why = "handles", false;
    for (size_t h = 0; h < a.handles.size(); ++h)
        if (a.handles[h].type != b.handles[h].type || a.handles[h].idx != b.handles[h].idx)
            return why = "wrapper/ghost handles", false;
    if (a.ghosts.size() != b.ghosts.size()) return why = "ghost entries", false;
    for (size_t g = 0; g < a.ghosts.size(); ++g) {
        const HGhost &x = a.ghosts[g], &y = b.ghosts[g];
        if (x.src != y.src || x.nplanes != y.nplanes || x.copiers != y.copiers) return why = "ghost entries", false;
    }
    if (a.inters.size() != b.inters.size()) return why = "interactions", false;
    for (size_t i = 0; i < a.inters.size(); ++i) {
        const HInter &x = a.inters[i], &y = b.inters[i];
        if (x.a != y.a || x.b != y.b || x.kk != y.kk || x.nstages != y.nstages || x.pk != y.pk || x.vk != y.vk ||
            x.probe != y.probe || x.ag != y.ag)
            return why = "interactions", false;
        for (int s = 0; s < x.nstages; ++s) {
            if (x.pp[s][3] != y.pp[s][3] || std::isnan(x.pp[s][4]) != std::isnan(y.pp[s][4]))
                return why = "functor variants", false;
            if (x.pk[s] == GC_PFN_INTERPOLATE && (x.pp[s][0] != y.pp[s][0] || x.pp[s][1] != y.pp[s][1]))
                return why = "interpolated fields", false;
        }
    }
    return true;
}

UpdInst make_upd(const HUpd& u, const HSys& s) {
    UpdInst d{};
    d.kind = u.kind;
    for (int q = 0; q < GC_UPD_NPARAM; ++q) d.prm[q] = u.prm[q];
    if (u.kind == GC_UPD_ZERO_FIELDS) d.zmask = (uint32_t)u.prm[0];
    if (u.kind == GC_UPD_TAIT_EOS) {
        double rho0 = u.prm[0], gam = u.prm[1];
        d.pre = rho0 * s.c * s.c / gam;
        d.gamma_int = (gam == std::trunc(gam) && std::fabs(gam) < 9.0e15) ? 1 : 0;
    }
    if (u.kind == GC_UPD_VISCOPLASTIC_MC) d.pre = std::tan(u.prm[0]);  // tan(φ), hoisted to the host
    if (u.kind == GC_UPD_ELASTOPLASTIC || u.kind == GC_UPD_HOOKE) {
        double E = u.prm[0], nu = u.prm[1], phi = u.prm[2], psi = u.prm[3], coh = u.prm[4];
        d.D0 = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
        d.omn = 1.0 - nu;
        d.om2n = 1.0 - 2.0 * nu;
        double sqrt3 = std::sqrt(3.0);
        double sphi = std::sin(phi), cphi = std::cos(phi), spsi = std::sin(psi);
        d.a_phi = 2.0 * sphi / (sqrt3 * (3.0 - sphi));
        d.k_c = 6.0 * coh * cphi / (sqrt3 * (3.0 - sphi));
        d.a_psi = 2.0 * spsi / (sqrt3 * (3.0 - spsi));
        d.apex_thr = d.k_c / d.a_phi;
        d.apex = d.k_c / d.a_phi / 3.0;
    }
    return d;
}

int finalize(gc_ctx* ctx) {
    if (ctx->inst.empty()) return seterr(ctx, GC_ERR_STATE, "no instance");
    const HInst& I0 = ctx->inst[0];
    if (I0.sys.empty()) return seterr(ctx, GC_ERR_ARG, "systems must not be empty");
    if (I0.inters.empty()) return seterr(ctx, GC_ERR_ARG, "interactions must not be empty");
    for (size_t k = 1; k < ctx->inst.size(); ++k) {
        std::string why;
        if (!same_structure(I0, ctx->inst[k], why))
            return seterr(ctx, GC_ERR_ARG, "instance %zu differs from instance 0 in %s", k, why.c_str());
    }
    CU(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
    ctx->nstages = 0;
    for (auto& it : I0.inters)
        if (!it.probe) {
            ctx->nstages = it.nstages;
            break;
        }
    if (ctx->nstages == 0) return seterr(ctx, GC_ERR_ARG, "interactions must not be empty");
    ctx->xsph = false;
    for (auto& it : I0.inters) ctx->xsph |= it.vk != GC_PFN_NONE;
    for (auto& it : I0.inters)
        if (!it.probe && it.nstages != ctx->nstages)
            return seterr(ctx, GC_ERR_ARG, "All interactions must have the same number of stages (pfns length)");
    if (ctx->nstages > MAX_STAGES) return seterr(ctx, GC_ERR_UNSUPPORTED, "too many stages");
    const int ninst = (int)ctx->inst.size();

    // per-instance dt inputs
    std::vector<double> hmin(ninst, 1e300), cmax(ninst, -1e300);
    for (int k = 0; k < ninst; ++k) {
        for (auto& it : ctx->inst[k].inters)
            if (!it.probe) hmin[k] = std::min(hmin[k], it.H);
        for (auto& s : ctx->inst[k].sys) cmax[k] = std::max(cmax[k], s.c);
    }

    // ---- system slots
    ctx->slots.resize(I0.sys.size());
    int64_t maxN = 0;
    for (size_t s = 0; s < I0.sys.size(); ++s) {
        DSlot& D = ctx->slots[s];
        const HSys& h0 = I0.sys[s];
        D.nd = h0.nd;
        D.ns = h0.ns;
        D.nvort = h0.nvort;
        D.kind = h0.kind;
        D.vsrc = h0.vsrc;
        D.probe = h0.probe;
        D.moving = !D.vsrc;
        D.h_inst.resize(ninst);
        D.nonzero_kin.assign(ninst, 0);
        int64_t base = 0;
        for (int k = 0; k < ninst; ++k) {
            const HSys& h = ctx->inst[k].sys[s];
            SysInst& S = D.h_inst[k];
            memset(&S, 0, sizeof S);
            S.base = base;
            S.n = h.n;
            S.mass = h.mass;
            S.c = h.c;
            for (int d = 0; d < 3; ++d) S.srcv[d] = h.srcv[d];
            S.srcrho = h.srcrho;
            S.sort_cutoff = 2.0 * hmin[k];
            base += h.n;
        }
        D.N = base;
        if (D.N >= (int64_t)1 << 31) return seterr(ctx, GC_ERR_CAPACITY, "more than 2^31 particles in one system slot");
        maxN = std::max(maxN, D.N);
        D.ncomp[F_X] = D.ncomp[F_V] = D.ncomp[F_DVDT] = D.nd;
        D.ncomp[F_RHO] = D.ncomp[F_DRHODT] = 1;
        D.ncomp[F_P] = D.kind >= GC_SYS_FLUID ? 1 : 0;
        D.ncomp[F_STRESS] = D.ncomp[F_SR] = D.kind >= GC_SYS_STRESS ? D.ns : 0;
        D.ncomp[F_VORT] = D.kind == GC_SYS_ELASTOPLASTIC ? D.nvort : 0;
        D.ncomp[F_STRAIN] = D.ncomp[F_STRAINP] = D.kind == GC_SYS_ELASTOPLASTIC ? D.ns : 0;
        D.ncomp[F_VADJ] = ctx->xsph ? D.nd : 0;
        for (int b = 0; b < 2; ++b) {
            for (int f = 0; f < NF; ++f)
                if (D.ncomp[f]) TRY(dalloc(ctx, &D.f[b][f], (size_t)D.ncomp[f] * D.N));
            TRY(dalloc(ctx, &D.id[b], (size_t)D.N));
        }
        TRY(dalloc(ctx, &D.q0v, (size_t)D.nd * D.N));
        TRY(dalloc(ctx, &D.q0rho, (size_t)D.N));
        TRY(dalloc(ctx, &D.aux, (size_t)D.N));
        TRY(dalloc(ctx, &D.inst_of, (size_t)D.N));
        TRY(dalloc(ctx, &D.groups, (size_t)D.N + 1));
        TRY(dalloc(ctx, &D.d_ngroups, 1));
        std::vector<int32_t> io(D.N);
        for (int k = 0; k < ninst; ++k)
            for (int64_t i = 0; i < D.h_inst[k].n; ++i) io[D.h_inst[k].base + i] = k;
        CU(cudaMemcpyAsync(D.inst_of, io.data(), io.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
        TRY(dalloc(ctx, &D.d_inst, (size_t)ninst));
        TRY(dalloc(ctx, &D.d_mass, (size_t)ninst));
        TRY(dalloc(ctx, &D.d_c, (size_t)ninst));
        std::vector<double> m(ninst), c(ninst);
        for (int k = 0; k < ninst; ++k) {
            m[k] = D.h_inst[k].mass;
            c[k] = D.h_inst[k].c;
        }
        CU(cudaMemcpyAsync(D.d_mass, m.data(), ninst * 8, cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(D.d_c, c.data(), ninst * 8, cudaMemcpyHostToDevice, ctx->stream));
        std::vector<float> mf(ninst), cf(ninst);
        for (int k = 0; k < ninst; ++k) {
            mf[k] = (float)m[k];
            cf[k] = (float)c[k];
        }
        TRY(dalloc(ctx, &D.d_massf, (size_t)ninst));
        TRY(dalloc(ctx, &D.d_cf, (size_t)ninst));
        CU(cudaMemcpyAsync(D.d_massf, mf.data(), ninst * 4, cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(D.d_cf, cf.data(), ninst * 4, cudaMemcpyHostToDevice, ctx->stream));
        // ids default to 1..n per instance
        std::vector<int32_t> ids(D.N);
        for (int k = 0; k < ninst; ++k)
            for (int64_t i = 0; i < D.h_inst[k].n; ++i) ids[D.h_inst[k].base + i] = (int32_t)(i + 1);
        CU(cudaMemcpyAsync(D.id[0], ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
        // updaters
        D.upd_set = h0.upd_set;
        D.nupd = (int)h0.upd.size();
        D.d_upd.resize(h0.upd.size());
        D.upd_kind.resize(h0.upd.size());
        for (size_t t = 0; t < h0.upd.size(); ++t) {
            for (size_t q = 0; q < h0.upd[t].size(); ++q) {
                std::vector<UpdInst> per(ninst);
                for (int k = 0; k < ninst; ++k) per[k] = make_upd(ctx->inst[k].sys[s].upd[t][q], ctx->inst[k].sys[s]);
                UpdInst* d = nullptr;
                TRY(dalloc(ctx, &d, (size_t)ninst));
                CU(cudaMemcpyAsync(d, per.data(), ninst * sizeof(UpdInst), cudaMemcpyHostToDevice, ctx->stream));
                D.d_upd[t].push_back(d);
                D.upd_kind[t].push_back(h0.upd[t][q].kind);
            }
        }
        // Host-side copies must outlive the async copies above.
        CU(cudaStreamSynchronize(ctx->stream));
    }

    // ---- virtual systems
    ctx->virts.resize(I0.virts.size());
    for (size_t v = 0; v < I0.virts.size(); ++v) {
        DVirt& V = ctx->virts[v];
        const HVirt& h0 = I0.virts[v];
        DSlot& S = ctx->slots[h0.src];
        V.src = h0.src;
        V.zmask = h0.zmask;
        V.upd_set = h0.upd_set;
        V.nupd = (int)h0.upd.size();
        V.probe = h0.probe;
        V.mirror = h0.mirror;
        if (V.probe) TRY(dalloc(ctx, &V.wsum_alt, (size_t)std::max<int64_t>(S.N, 1)));
        TRY(dalloc(ctx, &V.wsum, (size_t)std::max<int64_t>(S.N, 1)));
        CU(cudaMemsetAsync(V.wsum, 0, sizeof(double) * std::max<int64_t>(S.N, 1), ctx->stream));
        std::vector<VirtInst> vi(ninst);
        for (int k = 0; k < ninst; ++k) {
            const HVirt& h = ctx->inst[k].virts[v];
            for (int d = 0; d < MAXD; ++d) {
                vi[k].pv[d] = d < S.nd ? h.pv[d] : 0.0;
                V.moves |= vi[k].pv[d] != 0.0;
            }
        }
        S.vmoves |= V.moves;
        TRY(dalloc(ctx, &V.d_vi, (size_t)ninst));
        CU(cudaMemcpyAsync(V.d_vi, vi.data(), ninst * sizeof(VirtInst), cudaMemcpyHostToDevice, ctx->stream));
        V.d_upd.resize(h0.upd.size());
        V.upd_kind.resize(h0.upd.size());
        for (size_t t = 0; t < h0.upd.size(); ++t)
            for (size_t q = 0; q < h0.upd[t].size(); ++q) {
                std::vector<UpdInst> per(ninst);
                for (int k = 0; k < ninst; ++k)
                    per[k] = make_upd(ctx->inst[k].virts[v].upd[t][q], ctx->inst[k].sys[h0.src]);
                UpdInst* d = nullptr;
                TRY(dalloc(ctx, &d, (size_t)ninst));
                CU(cudaMemcpyAsync(d, per.data(), ninst * sizeof(UpdInst), cudaMemcpyHostToDevice, ctx->stream));
                V.d_upd[t].push_back(d);
                V.upd_kind[t].push_back(h0.upd[t][q].kind);
            }
        CU(cudaStreamSynchronize(ctx->stream));
    }

    // ---- ghosts
    ctx->ghosts.resize(I0.ghosts.size());
    for (size_t g = 0; g < I0.ghosts.size(); ++g) {
        DGhost& G = ctx->ghosts[g];
        const HGhost& h0 = I0.ghosts[g];
        DSlot& S = ctx->slots[h0.src];
        G.src = h0.src;
        G.nplanes = h0.nplanes;
        G.nd = S.nd;
        G.ns = S.ns;
        G.copiers = h0.copiers;
        G.ex_p = h0.ex_p;
        G.ex_stress = h0.ex_stress;
        G.CAP = S.N * G.nplanes;
        if (G.CAP >= (int64_t)1 << 31) return seterr(ctx, GC_ERR_CAPACITY, "ghost capacity beyond 2^31");
        maxN = std::max(maxN, G.CAP);
        for (int b = 0; b < 2; ++b) {
            TRY(dalloc(ctx, &G.x[b], (size_t)G.nd * G.CAP));
            TRY(dalloc(ctx, &G.io[b], (size_t)G.CAP));
            TRY(dalloc(ctx, &G.ib[b], (size_t)G.CAP));
            TRY(dalloc(ctx, &G.ginst[b], (size_t)G.CAP));
        }
        TRY(dalloc(ctx, &G.normals, (size_t)G.nd * G.CAP));
        TRY(dalloc(ctx, &G.v, (size_t)G.nd * G.CAP));
        TRY(dalloc(ctx, &G.rho, (size_t)G.CAP));
        TRY(dalloc(ctx, &G.aux, (size_t)G.CAP));
        if (G.ex_p) TRY(dalloc(ctx, &G.p, (size_t)G.CAP));
        if (G.ex_stress) TRY(dalloc(ctx, &G.stress, (size_t)G.ns * G.CAP));
        TRY(dalloc(ctx, &G.flags, (size_t)G.CAP));
        TRY(dalloc(ctx, &G.pos, (size_t)G.CAP + 1));
        TRY(dalloc(ctx, &G.d_count, 1));
        G.h_gh.resize(ninst);
        G.h_inst.resize(ninst);
        std::vector<double> m(ninst), c(ninst);
        for (int k = 0; k < ninst; ++k) {
            const HGhost& h = ctx->inst[k].ghosts[g];
            const HSys& src = ctx->inst[k].sys[h.src];
            GhostInst& H = G.h_gh[k];
            memset(&H, 0, sizeof H);
            for (int b = 0; b < h.nplanes; ++b)
                for (int d = 0; d < 3; ++d) {
                    H.normals[b][d] = h.normals[b][d];
                    H.points[b][d] = h.points[b][d];
                }
            H.cutoff = h.cutoff;
            H.src_base = S.h_inst[k].base;
            H.src_n = S.h_inst[k].n;
            H.mass = src.mass;
            H.c = src.c;
            SysInst& GI = G.h_inst[k];
            memset(&GI, 0, sizeof GI);
            GI.mass = src.mass;
            GI.c = src.c;
            GI.sort_cutoff = 2.0 * hmin[k];
            m[k] = src.mass;
            c[k] = src.c;
        }
        TRY(dalloc(ctx, &G.d_gh, (size_t)ninst));
        TRY(dalloc(ctx, &G.d_inst, (size_t)ninst));
        TRY(dalloc(ctx, &G.d_mass, (size_t)ninst));
        TRY(dalloc(ctx, &G.d_c, (size_t)ninst));
        CU(cudaMemcpyAsync(G.d_gh, G.h_gh.data(), ninst * sizeof(GhostInst), cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(G.d_inst, G.h_inst.data(), ninst * sizeof(SysInst), cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(G.d_mass, m.data(), ninst * 8, cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(G.d_c, c.data(), ninst * 8, cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
    }

    // ---- interactions
    ctx->inters.resize(I0.inters.size());
    for (size_t i = 0; i < I0.inters.size(); ++i) {
        DInter& D = ctx->inters[i];
        const HInter& h0 = I0.inters[i];
        D.a = h0.a;
        D.kk = h0.kk;
        D.nstages = h0.nstages;
        D.pk = h0.pk;
        D.probe = h0.probe;
        D.ag = h0.ag;
        D.vadj = h0.vk != GC_PFN_NONE;
        if (D.vadj) D.pk.push_back(h0.vk);  // the XSPH pass sweeps it as stage nstages + 1
        if (h0.b < 0) {
            D.btype = BT_SELF;
            D.bslot = h0.a;
        } else {
            const HHandle& hh = I0.handles[h0.b];
            if (hh.type == H_GHOST) {
                D.btype = BT_GHOST;
                D.bghost = hh.idx;
            } else if (hh.type == H_VIRT) {
                D.btype = BT_VIRTUAL;
                D.bvirt = hh.idx;
                D.bslot = I0.virts[hh.idx].src;
            } else {
                D.btype = hh.type == H_DYN ? BT_DYNAMIC : hh.type == H_STATIC ? BT_STATIC : BT_SYSTEM;
                D.bslot = hh.idx;
            }
        }
        D.two_fluid = D.btype == BT_SYSTEM && I0.sys[h0.a].kind == GC_SYS_FLUID &&
                      I0.sys[D.bslot].kind == GC_SYS_FLUID;
        for (int s = 0; s < (int)D.pk.size(); ++s)
            if (b_side_at(D, s + 1)) D.two_sided = true;
        D.h_gi.resize(ninst);
        for (int k = 0; k < ninst; ++k) {
            const HInst& I = ctx->inst[k];
            const HInter& h = I.inters[i];
            GridInst& G = D.h_gi[k];
            memset(&G, 0, sizeof G);
            G.H = h.H;
            G.cell = 2.0 * h.H;
            G.cutoff_sq = G.cell * G.cell;
            G.knorm = kernel_norm(h.kk, I.sys[h.a].nd, h.H);
            G.f_invH = (float)(1.0 / h.H);
            G.f_knorm = (float)G.knorm;
            if (h.b >= 0) {
                const HHandle& hh = I.handles[h.b];
                for (int d = 0; d < 3; ++d) {
                    G.normal[d] = hh.normal[d];
                    G.point[d] = hh.point[d];
                }
                G.beta = hh.beta;
                G.ljcut = hh.ljcut;
                for (int d = 0; d < 3; ++d) G.f_normal[d] = (float)hh.normal[d];
                G.f_beta = (float)hh.beta;
                G.f_ljcut = (float)hh.ljcut;
                if (hh.type == H_GHOST || hh.type == H_VIRT) {
                    const HSys& src = I.sys[hh.type == H_GHOST ? I.ghosts[hh.idx].src : I.virts[hh.idx].src];
                    G.bmass = src.mass;
                    G.bc = src.c;
                } else {
                    G.bmass = I.sys[hh.idx].mass;
                    G.bc = I.sys[hh.idx].c;
                }
                G.f_bmass = (float)G.bmass;
                G.f_bc = (float)G.bc;
            }
        }
        TRY(dalloc(ctx, &D.d_gi, (size_t)ninst));
        CU(cudaMemcpyAsync(D.d_gi, D.h_gi.data(), ninst * sizeof(GridInst), cudaMemcpyHostToDevice, ctx->stream));
        if (D.two_sided) {
            std::vector<GridInst> gb = D.h_gi;
            for (int k = 0; k < ninst; ++k) {
                const HSys& sa = ctx->inst[k].sys[ctx->inst[k].inters[i].a];
                gb[k].bmass = sa.mass;
                gb[k].bc = sa.c;
                gb[k].f_bmass = (float)sa.mass;
                gb[k].f_bc = (float)sa.c;
                gb[k].side_b = 1;
            }
            TRY(dalloc(ctx, &D.d_gi_b, (size_t)ninst));
            CU(cudaMemcpyAsync(D.d_gi_b, gb.data(), ninst * sizeof(GridInst), cudaMemcpyHostToDevice, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
        }
        D.d_pi.resize(D.nstages, nullptr);
        for (int s = 0; s < D.nstages; ++s) {
            std::vector<PfnInst> per(ninst);
            for (int k = 0; k < ninst; ++k) {
                const auto& p = ctx->inst[k].inters[i].pp[s];
                per[k].alpha = p[0];
                per[k].beta = p[1];
                per[k].h = p[2];
                per[k].S = (int)p[3];
                per[k].delta = std::isnan(p[4]) ? 0.0 : p[4];
                per[k].has_delta = std::isnan(p[4]) ? 0 : 1;
                per[k].f_alpha = (float)p[0];
                per[k].f_beta = (float)p[1];
                per[k].f_h = (float)p[2];
                per[k].f_h2eps = (float)(p[2] * p[2] * 0.01);
                per[k].f_delta = (float)per[k].delta;
                per[k].has_eps = std::isnan(p[5]) ? 0 : 1;
                per[k].eps = per[k].has_eps ? p[5] : 0.0;
                per[k].f_eps = (float)per[k].eps;
                per[k].two = (D.two_fluid && D.pk[s] == GC_PFN_FLUID) || D.pk[s] == GC_PFN_FLUID_SOLID;
                per[k].fs = D.pk[s] == GC_PFN_FLUID_SOLID;
            }
            TRY(dalloc(ctx, &D.d_pi[s], (size_t)ninst));
            CU(cudaMemcpyAsync(D.d_pi[s], per.data(), ninst * sizeof(PfnInst), cudaMemcpyHostToDevice, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
        }
        if (D.vadj) {
            // XSPHPfn(epsilon): epsilon in `alpha`
            std::vector<PfnInst> per(ninst);
            for (int k = 0; k < ninst; ++k) {
                memset(&per[k], 0, sizeof(PfnInst));
                per[k].alpha = ctx->inst[k].inters[i].veps;
                per[k].f_alpha = (float)per[k].alpha;
            }
            D.d_pi.push_back(nullptr);
            TRY(dalloc(ctx, &D.d_pi.back(), (size_t)ninst));
            CU(cudaMemcpyAsync(D.d_pi.back(), per.data(), ninst * sizeof(PfnInst), cudaMemcpyHostToDevice,
                               ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            if (D.btype == BT_GHOST) {
                // the ghosts' own warp groups and sums of the system_b side
                DGhost& G = ctx->ghosts[D.bghost];
                if (!G.gadj) {
                    TRY(dalloc(ctx, &G.groups, (size_t)G.CAP + 1));
                    TRY(dalloc(ctx, &G.d_ngroups, 1));
                    TRY(dalloc(ctx, &G.gadj, (size_t)G.nd * G.CAP));
                }
            }
        }
        TRY(dalloc(ctx, &D.counts, (size_t)(D.ag >= 0 ? ctx->ghosts[D.ag].CAP : ctx->slots[D.a].N)));
        if (!D.probe && D.ag < 0 && !D.two_sided && D.bslot >= 0 && D.btype != BT_SELF) {
            TRY(dalloc(ctx, &D.d_keep, 2));
            TRY(dalloc(ctx, &D.d_gi_prev, (size_t)ninst));
            CU(cudaMemsetAsync(D.d_keep, 0, 2 * sizeof(int), ctx->stream));
        }
        // writers
        bool writes = false;
        for (int s = 0; s < (int)D.pk.size(); ++s) writes |= D.pk[s] != GC_PFN_NONE;
        if (writes && D.ag < 0) ctx->slots[D.a].written = true;
        if (D.two_sided && D.bslot >= 0) ctx->slots[D.bslot].written = true;
        CU(cudaStreamSynchronize(ctx->stream));
    }

    // ---- shared scratch
    ctx->cap_keyN = std::max<int64_t>(maxN, 1);
    TRY(dalloc(ctx, &ctx->key, (size_t)ctx->cap_keyN));
    TRY(dalloc(ctx, &ctx->perm, (size_t)ctx->cap_keyN));
    TRY(dalloc(ctx, &ctx->bbox_scratch, (size_t)ninst * 2 * MAXD + 1));  // + block counter
    launch_bbox_reset(ctx->bbox_scratch, ninst, ctx->stream);
    TRY(dalloc(ctx, &ctx->d_err, 1));
    TRY(dalloc(ctx, &ctx->d_unsorted, 1));
    TRY(dalloc(ctx, &ctx->d_sorts_in_order, 1));
    TRY(dalloc(ctx, &ctx->d_incons, 1));
    TRY(dalloc(ctx, &ctx->d_total_cells, 1));
    ctx->nneed = (int)(ctx->slots.size() + ctx->ghosts.size() + ctx->inters.size());
    TRY(dalloc(ctx, &ctx->d_need, (size_t)ctx->nneed));
    CU(cudaMallocHost(&ctx->h_need, sizeof(int64_t) * ctx->nneed));
    TRY(dalloc(ctx, &ctx->d_need_max, (size_t)ctx->nneed));
    TRY(dalloc(ctx, &ctx->d_need_cap, (size_t)ctx->nneed));
    CU(cudaMallocHost(&ctx->h_need_max, sizeof(int64_t) * ctx->nneed));
    ctx->need_max.assign(ctx->nneed, 0);
    for (size_t g = 0; g < ctx->ghosts.size(); ++g) ctx->ghosts[g].need_slot = (int64_t)(ctx->slots.size() + g);
    for (size_t i = 0; i < ctx->inters.size(); ++i)
        ctx->inters[i].need_slot = (int64_t)(ctx->slots.size() + ctx->ghosts.size() + i);
    {
        std::vector<GridPlanArgs> pa;  // the steps' interactions; probe grids are planned at measurement
        for (auto& D : ctx->inters) {
            if (D.probe) continue;
            pa.push_back(grid_plan_args(ctx, D));
            // the keep check of a still system_b's CSR runs in its plan (the
            // only plan of such an interaction in a step)
            pa.back().prev = D.d_gi_prev;
            pa.back().keep = D.d_keep;
        }
        ctx->nplan = (int)pa.size();
        TRY(dalloc(ctx, &ctx->d_plan_args, pa.size()));
        TRY(hcopy(ctx, ctx->d_plan_args, pa.data(), pa.size() * sizeof(GridPlanArgs), cudaMemcpyHostToDevice));
    }
    ctx->finalized = true;
    return GC_OK;
}

// ------------------------------------------------------------- capacity
int ensure_cells(gc_ctx* ctx, int64_t cells) {
    if (cells + 1 > ctx->cap_cells) {
        int64_t cap = std::max<int64_t>(cells + 1 + cells / 4, 1024);
        CU(cudaStreamSynchronize(ctx->stream));  // in-flight kernels may use the old buffers
        dfree(ctx, ctx->hist, ctx->cap_cells);
        dfree(ctx, ctx->start, ctx->cap_cells);
        dfree(ctx, ctx->fill, ctx->cap_cells);
        TRY(dalloc(ctx, &ctx->hist, (size_t)cap));
        TRY(dalloc(ctx, &ctx->start, (size_t)cap));
        TRY(dalloc(ctx, &ctx->fill, (size_t)cap));
        ctx->cap_cells = cap;
    }
    int64_t st = scan_tmp_elems(ctx->cap_cells) + 16;
    if (st > ctx->cap_scan) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, ctx->scan_tmp, ctx->cap_scan);
        TRY(dalloc(ctx, &ctx->scan_tmp, (size_t)st));
        ctx->cap_scan = st;
    }
    return GC_OK;
}

int ensure_inter_cells(gc_ctx* ctx, DInter& D, int64_t cells) {
    if (cells + 1 > D.cap_cells) {
        int64_t cap = std::max<int64_t>(cells + 1 + cells / 4, 1024);
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, D.cs, D.cap_cells);
        dfree(ctx, D.cs_a, D.cap_cells);
        TRY(dalloc(ctx, &D.cs, (size_t)cap));
        if (D.btype != BT_SELF) TRY(dalloc(ctx, &D.cs_a, (size_t)cap));
        D.cap_cells = cap;
        if (D.d_keep) {
            // its own histogram for the batched still grids, zero between uses
            dfree(ctx, D.hist, D.cap_hist);
            D.cap_hist = still_hist_elems(cap);
            TRY(dalloc(ctx, &D.hist, (size_t)D.cap_hist));
            CU(cudaMemsetAsync(D.hist, 0, sizeof(int32_t) * D.cap_hist, ctx->stream));
            // new buffer: nothing counted (the step's plan may already have set keep[1])
            CU(cudaMemsetAsync(D.d_keep, 0, 2 * sizeof(int), ctx->stream));
        }
    }
    return ensure_cells(ctx, cells);
}

// ------------------------------------------------------------- phases
int check_launch(gc_ctx* ctx, const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return seterr(ctx, GC_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
    return GC_OK;
}

int ninst(gc_ctx* ctx) { return (int)ctx->inst.size(); }

int bbox_slot(gc_ctx* ctx, DSlot& S) {
    launch_bbox_fused(S.F(F_X), S.N, S.nd, S.inst_of, nullptr, S.d_inst, ctx->bbox_scratch, ninst(ctx), ctx->d_err,
                ctx->stream);
    return check_launch(ctx, "bbox");
}

// Conservative ghost extent before generation: the reflection of the source
// bounding box's corners across every plane, padded by one cell.
__global__ void k_ghost_bound(GhostInst* gh, const SysInst* src, SysInst* gi, int ninst, int nd, int nplanes) {
    pdl_enter();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ninst) return;
    const SysInst& S = src[k];
    double lo[MAXD], hi[MAXD];
    for (int d = 0; d < nd; ++d) {
        lo[d] = 1e300;
        hi[d] = -1e300;
    }
    int ncorner = 1 << nd;
    for (int b = 0; b < nplanes; ++b)
        for (int cI = 0; cI < ncorner; ++cI) {
            double x[MAXD], da = 0.0;
            for (int d = 0; d < nd; ++d) x[d] = (cI >> d) & 1 ? S.bbmax[d] : S.bbmin[d];
            for (int d = 0; d < nd; ++d) da += (x[d] - gh[k].points[b][d]) * gh[k].normals[b][d];
            for (int d = 0; d < nd; ++d) {
                double r = x[d] - 2.0 * da * gh[k].normals[b][d];
                lo[d] = fmin(lo[d], fmin(r, x[d]));
                hi[d] = fmax(hi[d], fmax(r, x[d]));
            }
        }
    double pad = 2.0 * S.sort_cutoff;
    for (int d = 0; d < nd; ++d) {
        gi[k].bbmin[d] = lo[d] - pad;
        gi[k].bbmax[d] = hi[d] + pad;
    }
    gi[k].n = S.n;  // upper bound on the count, used only for planning
}

// Stable counting sort of `S` (or of a ghost set when G != nullptr) over
// `cells` packed key cells (an upper bound on the planned total, which the
// device holds at `total`).
int sort_particles_slot(gc_ctx* ctx, DSlot* S, DGhost* G, int64_t cells, const int64_t* total) {
    const int ni = ninst(ctx);
    // The histogram and fill counters are zero on entry and left zero: the
    // scan clears what the keys counted, the fix-up what the scatter filled.
    TRY(ensure_cells(ctx, cells));
    GatherArgs ga{};
    if (S) {
        launch_sort_keys(S->F(F_X), S->N, S->nd, S->inst_of, nullptr, S->d_inst, ctx->key, ctx->hist, cells,
                         ctx->d_err, ctx->stream, ctx->d_unsorted);
        scan_exclusive_clear(ctx->hist, ctx->start, cells, ctx->scan_tmp, ctx->stream);
        launch_sort_scatter(ctx->key, S->N, nullptr, ctx->start, ctx->fill, ctx->perm, ctx->stream, ctx->d_unsorted);
        launch_sort_fixup_clear(ctx->start, cells, total, ctx->perm, ctx->fill, ctx->stream, ctx->d_unsorted,
                                ctx->d_sorts_in_order);
        for (int f = 0; f < NF; ++f)
            if (S->ncomp[f]) {
                ga.src[ga.nf] = S->F(f);
                ga.dst[ga.nf] = S->A(f);
                ga.ncomp[ga.nf++] = S->ncomp[f];
            }
        ga.isrc[0] = S->id[S->cur];
        ga.idst[0] = S->id[S->cur ^ 1];
        ga.ni = 1;
        ga.clear = ctx->d_unsorted;
        launch_gather_fields(ga, S->N, ctx->perm, nullptr, ctx->stream);
        S->cur ^= 1;
        S->xpk_static = false;
    } else {
        launch_sort_keys(G->x[G->cur], G->CAP, G->nd, G->ginst[G->cur], G->d_count, G->d_inst, ctx->key, ctx->hist,
                         cells, ctx->d_err, ctx->stream);
        scan_exclusive_clear(ctx->hist, ctx->start, cells, ctx->scan_tmp, ctx->stream);
        launch_sort_scatter(ctx->key, G->CAP, G->d_count, ctx->start, ctx->fill, ctx->perm, ctx->stream);
        launch_sort_fixup_clear(ctx->start, cells, total, ctx->perm, ctx->fill, ctx->stream);
        const int c = G->cur, a = c ^ 1;
        ga.src[0] = G->x[c];
        ga.dst[0] = G->x[a];
        ga.ncomp[0] = G->nd;
        ga.nf = 1;
        ga.isrc[0] = G->io[c];
        ga.idst[0] = G->io[a];
        ga.isrc[1] = G->ib[c];
        ga.idst[1] = G->ib[a];
        ga.isrc[2] = G->ginst[c];
        ga.idst[2] = G->ginst[a];
        ga.ni = 3;
        launch_gather_fields(ga, G->CAP, ctx->perm, G->d_count, ctx->stream);
        G->cur = a;
    }
    (void)ni;
    return check_launch(ctx, "sort");
}

int collect_profile(gc_ctx* ctx);

int read_need(gc_ctx* ctx) {
    CU(cudaMemcpyAsync(ctx->h_need, ctx->d_need, sizeof(int64_t) * ctx->nneed, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    TRY(collect_profile(ctx));
    int e = 0;
    TRY(hcopy(ctx, &e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e & ERR_NONFINITE) return seterr(ctx, GC_ERR_NONFINITE, "non-finite or out-of-range particle position");
    if (e & ERR_CAPACITY) return seterr(ctx, GC_ERR_CAPACITY, "grid or key range exceeds 2^31 cells");
    return GC_OK;
}

GridPlanArgs grid_plan_args(gc_ctx* ctx, DInter& D) {
    GridPlanArgs g{};
    g.gi = D.d_gi;
    g.gi_b = D.d_gi_b;
    g.ninst = ninst(ctx);
    g.nd = ctx->slots[D.a].nd;
    g.a = D.ag >= 0 ? ctx->ghosts[D.ag].d_inst : ctx->slots[D.a].d_inst;
    if (D.btype == BT_GHOST) g.b = ctx->ghosts[D.bghost].d_inst;
    else if (D.btype != BT_SELF) g.b = ctx->slots[D.bslot].d_inst;
    g.need = ctx->d_need + D.need_slot;
    g.err = ctx->d_err;
    return g;
}

// Ghost generation into the current buffers (generation order).
int generate_ghosts(gc_ctx* ctx, DGhost& G) {
    DSlot& S = ctx->slots[G.src];
    GhostGenArgs a{};
    a.src_x = S.F(F_X);
    a.Nsrc = S.N;
    a.src_inst_of = S.inst_of;
    a.gh = G.d_gh;
    a.ninst = ninst(ctx);
    a.nd = G.nd;
    a.nplanes = G.nplanes;
    a.flags = G.flags;
    a.pos = G.pos;
    a.gx = G.x[G.cur];
    a.gio = G.io[G.cur];
    a.gib = G.ib[G.cur];
    a.ginst = G.ginst[G.cur];
    a.gnormals = G.normals;
    a.count = G.d_count;
    a.ginst_params = G.d_inst;
    launch_ghost_flags(a, ctx->stream);
    int64_t n = G.CAP;
    int64_t st = scan_tmp_elems(n) + 16;
    if (st > ctx->cap_scan) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, ctx->scan_tmp, ctx->cap_scan);
        TRY(dalloc(ctx, &ctx->scan_tmp, (size_t)st));
        ctx->cap_scan = st;
    }
    scan_exclusive(G.flags, G.pos, n, ctx->scan_tmp, ctx->stream);
    launch_ghost_fill(a, ctx->stream);
    return check_launch(ctx, "ghost generation");
}

int ghost_bbox_and_plan(gc_ctx* ctx, DGhost& G) {
    launch_bbox_fused(G.x[G.cur], G.CAP, G.nd, G.ginst[G.cur], G.d_count, G.d_inst, ctx->bbox_scratch, ninst(ctx),
                ctx->d_err, ctx->stream);
    launch_sort_plan(G.d_inst, ninst(ctx), G.nd, ctx->d_need + G.need_slot, ctx->d_err, ctx->stream);
    return check_launch(ctx, "ghost plan");
}

// system_a's particles of an interaction: a system slot's arrays, or (a
// ghost system_a) the ghosts' current buffers up to the generated count
struct AParts {
    const double* x;
    int64_t N;
    const int32_t* inst_of;
    const int64_t* count;
};
AParts a_parts(gc_ctx* ctx, const DInter& D) {
    if (D.ag >= 0) {
        DGhost& G = ctx->ghosts[D.ag];
        return AParts{G.x[G.cur], G.CAP, G.ginst[G.cur], G.d_count};
    }
    DSlot& A = ctx->slots[D.a];
    return AParts{A.F(F_X), A.N, A.inst_of, nullptr};
}

// allow_keep: system_b's positions have not changed since its CSR was last
// counted, so an unchanged geometry keeps the CSR (decided on the device by
// the step's plan, keep[1]).
int build_grid(gc_ctx* ctx, DInter& D, int64_t cells, bool allow_keep = false) {
    TRY(ensure_inter_cells(ctx, D, cells));
    DSlot& A = ctx->slots[D.a];
    const int* skip = nullptr;
    if (D.d_keep) {
        if (allow_keep) skip = D.d_keep + 1;
        else CU(cudaMemsetAsync(D.d_keep, 0, sizeof(int), ctx->stream));  // counted on a geometry not recorded
    }
    const double* bx;
    const int32_t* binst;
    const int64_t* bcount = nullptr;
    int64_t bN;
    if (D.btype == BT_GHOST) {
        DGhost& G = ctx->ghosts[D.bghost];
        bx = G.x[G.cur];
        binst = G.ginst[G.cur];
        bcount = G.d_count;
        bN = G.CAP;
    } else {
        DSlot& B = ctx->slots[D.bslot];
        bx = B.F(F_X);
        binst = B.inst_of;
        bN = B.N;
    }
    launch_grid_count(bx, bN, A.nd, binst, bcount, D.d_gi, ctx->hist, cells, ctx->d_err, ctx->d_incons, ctx->stream,
                      skip);
    scan_exclusive_clear(ctx->hist, D.cs, cells, ctx->scan_tmp, ctx->stream, skip);
    if (D.two_sided) {
        const AParts ap = a_parts(ctx, D);
        launch_grid_count(ap.x, ap.N, A.nd, ap.inst_of, ap.count, D.d_gi, ctx->hist, cells, ctx->d_err,
                          ctx->d_incons, ctx->stream);
        scan_exclusive_clear(ctx->hist, D.cs_a, cells, ctx->scan_tmp, ctx->stream);
    }
    D.grid_valid = true;
    D.cells = cells;
    D.grid_ver = ++ctx->grid_version;
    D.csa_ver = D.two_sided ? D.grid_ver : -1;
    return check_launch(ctx, "grid");
}

// The grids of interactions against a system_b that does not move, built
// together: one count and one scan launch for all of them, each returning
// at once on the device while its grid's geometry is unchanged (keep[1]).
int build_still_grids(gc_ctx* ctx, const std::vector<DInter*>& L, const std::vector<int64_t>& need) {
    for (size_t i0 = 0; i0 < L.size(); i0 += STILL_MAX) {
        StillGridArgs a{};
        a.n = (int)std::min<size_t>(STILL_MAX, L.size() - i0);
        a.err = ctx->d_err;
        a.incons = ctx->d_incons;
        for (int i = 0; i < a.n; ++i) {
            DInter& D = *L[i0 + i];
            const int64_t cells = need[D.need_slot];
            TRY(ensure_inter_cells(ctx, D, cells));  // sizes the histogram with the CSR
            DSlot& B = ctx->slots[D.bslot];
            a.nd = ctx->slots[D.a].nd;
            a.g[i] = StillGrid{B.F(F_X), B.inst_of, B.N, D.d_gi, D.d_keep, D.hist, D.cs, cells};
            D.grid_valid = true;
            D.cells = cells;
            D.grid_ver = ++ctx->grid_version;
            D.csa_ver = -1;
        }
        launch_still_grids(a, ctx->stream);
    }
    return check_launch(ctx, "still grids");
}

// CSR of system_a's particles on a coupled interaction's grid.
int ensure_csa(gc_ctx* ctx, DInter& D) {
    if (D.btype == BT_SELF || D.csa_ver == D.grid_ver) return GC_OK;
    const AParts ap = a_parts(ctx, D);
    TRY(ensure_cells(ctx, D.cells));
    launch_grid_count(ap.x, ap.N, ctx->slots[D.a].nd, ap.inst_of, ap.count, D.d_gi, ctx->hist, D.cells, ctx->d_err,
                      ctx->d_incons, ctx->stream);
    scan_exclusive_clear(ctx->hist, D.cs_a, D.cells, ctx->scan_tmp, ctx->stream);
    D.csa_ver = D.grid_ver;
    return check_launch(ctx, "grid (system_a)");
}

// Warp groups of the particles of `cs` (a CSR on interaction D's grid) into
// the group tables of S (a system slot or a ghost system).
template <class St>
int build_groups(gc_ctx* ctx, St& S, DInter& D, int64_t key, const int32_t* cs) {
    if (S.groups_key == key && S.groups_ver == D.grid_ver) return GC_OK;
    const int64_t ncols_cap = D.cells;
    if (ncols_cap + 1 > S.cap_gcols) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, S.gcnt, S.cap_gcols);
        dfree(ctx, S.goff, S.cap_gcols);
        int64_t cap = ncols_cap + 1 + ncols_cap / 4;
        TRY(dalloc(ctx, &S.gcnt, (size_t)cap));
        TRY(dalloc(ctx, &S.goff, (size_t)cap));
        S.cap_gcols = cap;
    }
    TRY(ensure_cells(ctx, ncols_cap));  // scan scratch
    const int nd = ctx->slots[D.a].nd;
    launch_groups_count(D.d_gi, ninst(ctx), nd, cs, ncols_cap, D.cells, S.gcnt, ctx->stream);
    scan_exclusive(S.gcnt, S.goff, ncols_cap, ctx->scan_tmp, ctx->stream);
    launch_groups_fill(D.d_gi, ninst(ctx), nd, cs, S.goff, ncols_cap, D.cells, S.groups, S.d_ngroups, ctx->stream);
    S.groups_key = key;
    S.groups_ver = D.grid_ver;
    return check_launch(ctx, "groups");
}

// Warp groups of `slot`'s particles from the columns of interaction `id`'s
// grid: its system_b side when b_side, else its system_a side.
int ensure_groups(gc_ctx* ctx, int slot, int id, bool b_side) {
    DSlot& S = ctx->slots[slot];
    DInter& D = ctx->inters[id];
    const int64_t key = (int64_t)id * 2 + (b_side ? 1 : 0);
    if (S.groups_key == key && S.groups_ver == D.grid_ver) return GC_OK;
    const int32_t* cs;
    if (b_side || D.btype == BT_SELF) {
        cs = D.cs;
    } else {
        TRY(ensure_csa(ctx, D));
        cs = D.cs_a;
    }
    return build_groups(ctx, S, D, key, cs);
}

// Capacity mode: record the largest plans, and flag every plan that does
// not fit its buffers (the window is then rolled back and re-run exactly).
__global__ void k_need_max(const int64_t* need, int64_t* need_max, const int64_t* cap, int n, int* err) {
    pdl_enter();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (need[i] > need_max[i]) need_max[i] = need[i];
        if (need[i] > cap[i]) atomicOr(err, ERR_CAPACITY);
    }
}

// Cell bound for sorts and for interaction D's grid in capacity mode: the
// shared histogram and the interaction's CSR both have to hold it.
int64_t cap_sort_cells(gc_ctx* ctx) { return ctx->cap_cells - 1; }
int64_t cap_grid_cells(gc_ctx* ctx, const DInter& D) { return std::min(D.cap_cells, ctx->cap_cells) - 1; }

// Full prepare phase: sorts, ghosts and grids.  `sort_mask` selects which
// system slots are sorted.  Exact mode reads the planned cell counts back
// to size every buffer; capacity mode sizes from the buffers' capacities
// (no host read), and the kernels flag any plan that does not fit.
int prepare(gc_ctx* ctx, const std::vector<char>& sort_mask) {
    const int ni = ninst(ctx);
    CU(cudaMemsetAsync(ctx->d_need, 0, sizeof(int64_t) * ctx->nneed, ctx->stream));
    // bounding boxes of every real system (positions are current); a system
    // that does not move keeps the box computed after its last upload
    for (auto& S : ctx->slots)
        if (S.xmoves() || !S.sorted_once) TRY(bbox_slot(ctx, S));
    for (size_t s = 0; s < ctx->slots.size(); ++s)
        if (sort_mask[s])
            launch_sort_plan(ctx->slots[s].d_inst, ni, ctx->slots[s].nd, ctx->d_need + s, ctx->d_err, ctx->stream);
    for (auto& G : ctx->ghosts) {
        k_ghost_bound<<<(ni + 127) / 128, 128, 0, ctx->stream>>>(G.d_gh, ctx->slots[G.src].d_inst, G.d_inst, ni, G.nd,
                                                                 G.nplanes);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        launch_sort_plan(G.d_inst, ni, G.nd, ctx->d_need + G.need_slot, ctx->d_err, ctx->stream);
    }
    launch_grid_plan_all(ctx->d_plan_args, ctx->nplan, ctx->stream);
    TRY(check_launch(ctx, "plan"));
    std::vector<int64_t> need(ctx->nneed);
    if (ctx->capmode) {
        k_need_max<<<1, 128, 0, ctx->stream>>>(ctx->d_need, ctx->d_need_max, ctx->d_need_cap, ctx->nneed,
                                                ctx->d_err);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        for (size_t s = 0; s < ctx->slots.size(); ++s) need[s] = cap_sort_cells(ctx);
        for (auto& G : ctx->ghosts) need[G.need_slot] = cap_sort_cells(ctx);
        for (auto& D : ctx->inters) need[D.need_slot] = D.probe ? 0 : cap_grid_cells(ctx, D);
    } else {
        TRY(read_need(ctx));
        for (int i = 0; i < ctx->nneed; ++i) {
            need[i] = ctx->h_need[i];
            ctx->need_max[i] = std::max(ctx->need_max[i], need[i]);
        }
    }
    // sorts
    for (size_t s = 0; s < ctx->slots.size(); ++s)
        if (sort_mask[s]) TRY(sort_particles_slot(ctx, &ctx->slots[s], nullptr, need[s], ctx->d_need + s));
    // ghosts: generate, bound-checked plan, sort
    for (auto& G : ctx->ghosts) {
        TRY(generate_ghosts(ctx, G));
        TRY(ghost_bbox_and_plan(ctx, G));
        TRY(sort_particles_slot(ctx, nullptr, &G, need[G.need_slot], ctx->d_need + G.need_slot));
    }
    // grids (ghost-b plans are recomputed from the exact ghost boxes; the
    // cell count cannot exceed the planned bound)
    std::vector<DInter*> still;
    for (auto& D : ctx->inters) {
        if (D.probe) continue;
        if (D.btype == BT_GHOST || D.ag >= 0) launch_grid_plan(grid_plan_args(ctx, D), ctx->stream);
        const bool b_still = D.d_keep && !sort_mask[D.bslot] && !ctx->slots[D.bslot].xmoves();
        if (b_still && ctx->slots[D.bslot].N > 0 && need[D.need_slot] <= STILL_MAX_CELLS) {
            still.push_back(&D);
            continue;
        }
        TRY(build_grid(ctx, D, need[D.need_slot], b_still));
    }
    return build_still_grids(ctx, still, need);
}

StepArgs step_args(DSlot& S) {
    StepArgs a{};
    a.N = S.N;
    a.nd = S.nd;
    a.inst_of = S.inst_of;
    a.inst = S.d_inst;
    a.x = S.F(F_X);
    a.v = S.F(F_V);
    a.rho = S.F(F_RHO);
    a.dvdt = S.F(F_DVDT);
    a.drhodt = S.F(F_DRHODT);
    a.q0v = S.q0v;
    a.q0rho = S.q0rho;
    a.accv = S.accv;
    a.accrho = S.accrho;
    a.vadj = S.ncomp[F_VADJ] ? S.F(F_VADJ) : nullptr;
    return a;
}

UpdArgs upd_args(DSlot& S, int stage, size_t q, double dt_override) {
    UpdArgs a{};
    a.N = S.N;
    a.kind = S.upd_kind[stage - 1][q];
    a.nd = S.nd;
    a.ns = S.ns;
    a.nvort = S.nvort;
    a.inst_of = S.inst_of;
    a.inst = S.d_inst;
    a.u = S.d_upd[stage - 1][q];
    a.dt = dt_override;
    a.rho = S.F(F_RHO);
    a.p = S.F(F_P);
    a.stress = S.F(F_STRESS);
    a.sr = S.F(F_SR);
    a.vort = S.F(F_VORT);
    a.strain = S.F(F_STRAIN);
    a.strainp = S.F(F_STRAINP);
    a.dvdt = S.F(F_DVDT);
    a.drhodt = S.F(F_DRHODT);
    return a;
}

int run_updaters(gc_ctx* ctx, DSlot& S, int stage, double dt_override) {
    if (stage < 1 || stage > (int)S.d_upd.size()) return GC_OK;
    for (size_t q = 0; q < S.d_upd[stage - 1].size(); ++q) launch_update(upd_args(S, stage, q, dt_override), ctx->stream);
    return check_launch(ctx, "updater");
}

// A virtual system's updater chain for `stage` on its source's fields.
int run_virtual_updaters(gc_ctx* ctx, DVirt& V, int stage) {
    if (stage < 1 || stage > (int)V.d_upd.size()) return GC_OK;
    DSlot& S = ctx->slots[V.src];
    for (size_t q = 0; q < V.d_upd[stage - 1].size(); ++q) {
        const int kind = V.upd_kind[stage - 1][q];
        if (kind == GC_UPD_VIRTUAL_NORM || kind == GC_UPD_PRESCRIBED_V) {
            VirtArgs a{};
            a.N = S.N;
            a.nd = S.nd;
            a.ns = S.ns;
            a.kind = kind;
            a.inst_of = S.inst_of;
            a.vi = V.d_vi;
            a.u = V.d_upd[stage - 1][q];
            a.v = S.F(F_V);
            a.rho = S.F(F_RHO);
            a.p = S.ncomp[F_P] ? S.F(F_P) : nullptr;
            a.stress = S.ncomp[F_STRESS] ? S.F(F_STRESS) : nullptr;
            a.wsum = V.wsum;
            launch_virtual_update(a, ctx->stream);
        } else {
            UpdArgs a{};
            a.N = S.N;
            a.kind = kind;
            a.nd = S.nd;
            a.ns = S.ns;
            a.nvort = S.nvort;
            a.inst_of = S.inst_of;
            a.inst = S.d_inst;
            a.u = V.d_upd[stage - 1][q];
            a.dt = NAN;
            a.rho = S.F(F_RHO);
            a.p = S.F(F_P);
            a.stress = S.F(F_STRESS);
            a.sr = S.F(F_SR);
            a.vort = S.F(F_VORT);
            a.strain = S.F(F_STRAIN);
            a.strainp = S.F(F_STRAINP);
            a.dvdt = S.F(F_DVDT);
            a.drhodt = S.F(F_DRHODT);
            launch_update(a, ctx->stream);
        }
    }
    return check_launch(ctx, "virtual updater");
}

int ghost_kinematics(gc_ctx* ctx, DGhost& G) {
    DSlot& S = ctx->slots[G.src];
    launch_ghost_kinematics(G.CAP, G.d_count, G.nd, G.io[G.cur], G.ginst[G.cur], G.normals, G.d_gh, S.F(F_V),
                            S.F(F_RHO), S.N, G.v, G.rho, ctx->stream);
    return check_launch(ctx, "ghost kinematics");
}

int ghost_copy(gc_ctx* ctx, DGhost& G, int stage) {
    if (stage < 1 || stage > (int)G.copiers.size()) return GC_OK;
    DSlot& S = ctx->slots[G.src];
    for (auto& e : G.copiers[stage - 1]) {
        int field = e.first, mode = e.second;
        if (field == GC_FIELD_P)
            launch_ghost_copy(G.CAP, G.d_count, G.nd, 1, G.io[G.cur], G.ginst[G.cur], G.normals, G.d_gh, field, mode,
                              S.F(F_P), S.N, G.p, ctx->stream);
        else if (field == GC_FIELD_STRESS)
            launch_ghost_copy(G.CAP, G.d_count, G.nd, G.ns, G.io[G.cur], G.ginst[G.cur], G.normals, G.d_gh, field,
                              mode, S.F(F_STRESS), S.N, G.stress, ctx->stream);
    }
    return check_launch(ctx, "ghost copy");
}

// FP32-sweep buffers of a slot or ghost set: N FP64 positions (pos_stride
// each) followed by N FP32 records (pack_stride floats each).
template <class T>
int ensure_fpk(gc_ctx* ctx, T& X, int64_t N, int nd, int ns) {
    int64_t need = N * (2 * pos_stride(nd) + pack_stride(nd, ns));
    if (need > X.cap_fpk) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, X.fpk, X.cap_fpk);
        TRY(dalloc(ctx, &X.fpk, (size_t)need));
        X.cap_fpk = need;
        X.xpk_epoch = -1;  // the new buffer holds no positions yet
        X.xpk_static = false;
    }
    return GC_OK;
}

int aux_mode_for(int pfn) {
    if (pfn == GC_PFN_FLUID) return AUX_P_OVER_RHO2;
    if (pfn == GC_PFN_CAUCHY_FLUID) return AUX_INV_RHO2;
    return AUX_MASS_OVER_RHO;
}

// The ghosts' side of an XSPH sweep against ghost system_b (`A` holds the
// system_a launch): a gather over the ghosts through system_a's CSR into a
// ghost-indexed buffer, then added to the ghost SOURCE's v_adjustment at the
// ghost index, which is where the reference's `ps_b.v_adjustment[j]` lands
// (a ghost forwards that property to its source, src/GhostParticles.jl:226-236).
__global__ void k_xsph_ghost_add(const double* __restrict__ gadj, int64_t CAP, const int64_t* count, int nd,
                                 const int32_t* __restrict__ ginst, const GhostInst* __restrict__ gh,
                                 const SysInst* __restrict__ src, double* __restrict__ vadj, int64_t Ns, int* err) {
    pdl_enter();
    const int64_t n = *count;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        const int k = ginst[g];
        const int64_t local = g - gh[k].base;
        if (local >= src[k].n) {  // out of bounds in the reference
            atomicOr(err, ERR_XSPH_GHOST);
            continue;
        }
        const int64_t t = src[k].base + local;
        for (int d = 0; d < nd; ++d) vadj[d * Ns + t] = vadj[d * Ns + t] + gadj[d * CAP + g];
    }
}

int xsph_ghost_side(gc_ctx* ctx, const ForceArgs& A, int id, int stage) {
    DInter& D = ctx->inters[id];
    DGhost& G = ctx->ghosts[D.bghost];
    DSlot& S = ctx->slots[D.a];
    DSlot& src = ctx->slots[G.src];
    TRY(ensure_csa(ctx, D));
    TRY(build_groups(ctx, G, D, (int64_t)id * 2 + 1, D.cs));  // the ghosts' own CSR
    CU(cudaMemsetAsync(G.gadj, 0, sizeof(double) * G.nd * G.CAP, ctx->stream));
    ForceArgs R = A;
    R.groups = G.groups;
    R.ngroups = G.d_ngroups;
    R.nd = G.nd;
    R.ns = G.ns;
    R.aN = G.CAP;
    R.a_inst_of = G.ginst[G.cur];
    R.ax = G.x[G.cur];
    R.av = G.v;
    R.arho = G.rho;
    R.aaux = nullptr;
    R.astress = nullptr;
    R.a_p = nullptr;
    R.advdt = G.gadj;
    R.adrhodt = nullptr;
    R.asr = nullptr;
    R.avort = nullptr;
    R.a_c = G.d_c;
    R.a_mass = G.d_mass;
    R.a_cf = nullptr;
    R.a_massf = nullptr;
    R.afp = nullptr;
    R.prec = GC_PRECISION_FP64;
    R.nref = 1;
    InterRef& r = R.ref[0];
    r = InterRef{};
    r.btype = BT_SYSTEM;
    r.bbox = S.d_inst;
    r.gi = D.d_gi_b;
    r.pi = D.d_pi[stage - 1];
    r.cs = D.cs_a;
    r.cs_cells = D.cells;
    r.bx = S.F(F_X);
    r.bv = S.F(F_V);
    r.brho = S.F(F_RHO);
    r.bN = S.N;
    int st = launch_force_f64(R, false, ctx->stream);
    if (st) return seterr(ctx, st, "XSPH ghost side not implemented on the device");
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((G.CAP + 255) / 256, (int64_t)ctx->num_sms * 8));
    k_xsph_ghost_add<<<(unsigned)blocks, 256, 0, ctx->stream>>>(G.gadj, G.CAP, G.d_count, G.nd, G.ginst[G.cur],
                                                                 G.d_gh, src.d_inst, src.F(F_VADJ), src.N, ctx->d_err);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return check_launch(ctx, "sweep (XSPH ghost side)");
}

// InterpolateFieldFn stages (system_b virtual): nothing is written on the
// system_a side, so each interaction is one gather over the virtual system's
// source particles through system_a's CSR on the interaction's grid,
// accumulating into the source's fields and the virtual system's w_sum.
int interp_sweeps(gc_ctx* ctx, int a, const std::vector<int>& ids, int stage) {
    DSlot& S = ctx->slots[a];
    for (int id : ids) {
        DInter& D = ctx->inters[id];
        DSlot& B = ctx->slots[D.bslot];
        DVirt& V = ctx->virts[D.bvirt];
        if (!D.grid_valid) return seterr(ctx, GC_ERR_STATE, "sweep before create_grid");
        TRY(ensure_csa(ctx, D));
        TRY(ensure_groups(ctx, D.bslot, id, true));
        const auto& prm = ctx->inst[0].inters[id].pp[stage - 1];
        const bool count = D.pk[stage - 1] == GC_PFN_NEIGHBOR_COUNT;  // NeighborCountFn :455-460
        ForceArgs R{};
        R.nd = B.nd;
        R.ns = B.ns;
        R.pfn = GC_PFN_INTERPOLATE;
        R.kk = D.kk;
        R.aN = B.N;
        R.a_inst_of = B.inst_of;
        R.ax = B.F(F_X);
        R.av = B.F(F_V);
        R.arho = B.F(F_RHO);
        R.astress = B.F(F_STRESS);
        R.a_p = B.F(F_P);
        R.advdt = B.F(F_V);        // accumulation targets: v, rho, stress, w_sum
        R.adrhodt = B.F(F_RHO);
        R.asr = B.F(F_STRESS);
        R.avort = count ? B.F(F_DRHODT) : V.wsum;  // w_sum, or the count extra
        R.a_c = B.d_c;
        R.a_mass = B.d_mass;
        R.a_cf = B.d_cf;
        R.a_massf = B.d_massf;
        R.prec = GC_PRECISION_FP64;
        R.err = ctx->d_err;
        R.groups = B.groups;
        R.ngroups = B.d_ngroups;
        R.num_sms = ctx->num_sms;
        R.cfg = ctx->force_cfg >= 0 ? ctx->force_cfg : 0;
        R.imask = count ? 0 : (int)prm[0];
        R.iwsum = count ? 2 : (prm[1] != 0.0 ? 1 : 0);
        R.nref = 1;
        InterRef& r = R.ref[0];
        r.btype = BT_SYSTEM;
        r.bbox = S.d_inst;
        r.gi = D.d_gi_b;
        r.pi = D.d_pi[stage - 1];
        r.cs = D.cs_a;
        r.cs_cells = D.cells;
        if (D.ag >= 0) {
            // Trapdoor.jl's ghost_bottom: the ghosts' current arrays (stress
            // as the last GhostCopier left it), the source's mass in gi_b
            DGhost& Gh = ctx->ghosts[D.ag];
            r.bbox = Gh.d_inst;
            r.bx = Gh.x[Gh.cur];
            r.bv = Gh.v;
            r.brho = Gh.rho;
            r.bp = Gh.p;
            r.bstress = Gh.stress;
            r.bN = Gh.CAP;
        } else {
            r.bx = S.F(F_X);
            r.bv = S.F(F_V);
            r.brho = S.F(F_RHO);
            r.bp = S.F(F_P);
            r.bstress = S.F(F_STRESS);
            r.bN = S.N;
        }
        int st = launch_force_f64(R, false, ctx->stream);
        if (st) return seterr(ctx, st, "InterpolateFieldFn not implemented on the device for this system");
        TRY(check_launch(ctx, "sweep (interpolation)"));
    }
    return GC_OK;
}

// Fused sweep of the interactions `ids` (same system_a, same functor kind).
// How sweep_group treats system_a's state for a group of interactions of
// one functor kind: the functor the kernel runs, its per-particle divisor
// mode, whether the sweep is FP32-compensated and its record's stress width.
struct PackPlan {
    int pk0 = GC_PFN_NONE, pfn = GC_PFN_NONE, mode = 0, pk_ns = 0;
    bool interp = false, xsph = false, fp32 = false;
};

PackPlan pack_plan(gc_ctx* ctx, int a, const std::vector<int>& ids, int stage, bool count_only) {
    DSlot& S = ctx->slots[a];
    PackPlan pl;
    pl.pk0 = ctx->inters[ids[0]].pk[stage - 1];
    pl.interp = (pl.pk0 == GC_PFN_INTERPOLATE || pl.pk0 == GC_PFN_NEIGHBOR_COUNT) && !count_only;
    // FluidSolidPfn runs the FluidPfn kernel in its fluid-solid mode (PfnInst.fs)
    pl.pfn = pl.pk0 == GC_PFN_FLUID_SOLID ? GC_PFN_FLUID : pl.pk0;
    pl.mode = aux_mode_for(pl.pfn);
    pl.xsph = pl.pfn == GC_PFN_XSPH;  // writes v_adjustment; always FP64
    pl.fp32 = ctx->precision == GC_PRECISION_FP32_COMPENSATED && pl.pfn != GC_PFN_COUNT && !pl.xsph && !count_only;
    for (int id : ids)
        if (pl.pfn == GC_PFN_FLUID && ctx->inters[id].h_gi.size() && ctx->inst[0].inters[id].pp[stage - 1][3] == 1.0)
            pl.fp32 = false;  // the S = 1 (multiphase) pressure form stays in FP64
    pl.pk_ns = pl.pfn == GC_PFN_CAUCHY_FLUID ? S.ns : 0;
    return pl;
}

// The interaction groups a stage sweeps with system `a` as system_a, in
// launch order: grouped by functor kind in order of first appearance, at
// most MAX_REFS interactions per launch.
std::vector<std::vector<int>> stage_groups(gc_ctx* ctx, int a, int stage) {
    std::vector<int> kinds;
    for (size_t i = 0; i < ctx->inters.size(); ++i) {
        DInter& D = ctx->inters[i];
        if (D.probe) continue;
        int pk = D.pk[stage - 1];
        if (D.a != a || pk == GC_PFN_NONE) continue;
        if (std::find(kinds.begin(), kinds.end(), pk) == kinds.end()) kinds.push_back(pk);
    }
    std::vector<std::vector<int>> out;
    for (int pk : kinds) {
        std::vector<int> ids;
        for (size_t i = 0; i < ctx->inters.size(); ++i)
            if (!ctx->inters[i].probe && ctx->inters[i].a == a && ctx->inters[i].pk[stage - 1] == pk)
                ids.push_back((int)i);
        for (size_t off = 0; off < ids.size(); off += MAX_REFS)
            out.emplace_back(ids.begin() + off, ids.begin() + std::min(ids.size(), off + MAX_REFS));
    }
    return out;
}

int sweep_group(gc_ctx* ctx, int a, const std::vector<int>& ids, int stage, bool count_only) {
    DSlot& S = ctx->slots[a];
    const PackPlan pl = pack_plan(ctx, a, ids, stage, count_only);
    if (pl.interp) return interp_sweeps(ctx, a, ids, stage);
    const int pk0 = pl.pk0, pfn = pl.pfn, mode = pl.mode, pk_ns = pl.pk_ns;
    const bool xsph = pl.xsph, fp32 = pl.fp32;
    // FP32 sweep buffers: positions, then records (see ensure_fpk)
    auto xp_of = [](float* fpk) { return (double*)fpk; };
    auto pk_of = [](float* fpk, int64_t N, int nd) { return fpk + N * 2 * pos_stride(nd); };
    if (pfn != GC_PFN_COUNT && !xsph) {
        if (fp32) {
            TRY(ensure_fpk(ctx, S, S.N, S.nd, pk_ns));
            // the fused half step of this step may have packed these records
            const bool done = S.pack_done_epoch == ctx->pack_epoch && S.pack_done_stage == stage &&
                              S.pack_done_mode == mode && S.pack_done_ns == pk_ns;
            if (!done) {
                // positions do not change between the stages of a step
                const bool pos = S.xpk_epoch != ctx->pack_epoch;
                launch_pack32(mode, S.N, nullptr, S.nd, pk_ns, S.F(F_X), S.F(F_V), S.F(F_RHO), S.F(F_P),
                              S.F(F_STRESS), S.inst_of, S.d_mass, pos ? xp_of(S.fpk) : nullptr,
                              pk_of(S.fpk, S.N, S.nd), ctx->stream);
                S.xpk_epoch = ctx->pack_epoch;
            }
        } else {
            launch_aux(mode, S.N, nullptr, S.F(F_RHO), S.F(F_P), S.inst_of, S.d_mass, S.aux, ctx->stream);
        }
    }
    ForceArgs A{};
    A.nd = S.nd;
    A.ns = S.ns;
    A.pfn = pfn;
    if (pfn == GC_PFN_FLUID)  // a two-sided or fluid-solid reference needs the general fluid code
        for (int id : ids)
            if (pk0 == GC_PFN_FLUID_SOLID || ctx->inters[id].two_fluid) A.pfn = PFN_FLUID2;
    A.kk = ctx->inters[ids[0]].kk;
    A.aN = S.N;
    A.a_inst_of = S.inst_of;
    A.ax = S.F(F_X);
    A.av = S.F(F_V);
    A.arho = S.F(F_RHO);
    A.aaux = S.aux;
    A.astress = S.F(F_STRESS);
    A.a_p = S.F(F_P);
    A.advdt = xsph ? S.F(F_VADJ) : S.F(F_DVDT);
    A.adrhodt = S.F(F_DRHODT);
    A.asr = S.F(F_SR);
    A.avort = S.F(F_VORT);
    A.a_c = S.d_c;
    A.a_mass = S.d_mass;
    A.a_cf = S.d_cf;
    A.a_massf = S.d_massf;
    A.afp = fp32 ? pk_of(S.fpk, S.N, S.nd) : nullptr;
    A.prec = fp32 ? GC_PRECISION_FP32_COMPENSATED : GC_PRECISION_FP64;
    A.err = ctx->d_err;
    A.num_sms = ctx->num_sms;
    A.cfg = 0;
    int tune_slot = -1;
    if (ctx->force_cfg >= 0) {
        A.cfg = ctx->force_cfg;
    } else if (!count_only) {
        const int64_t key = ((int64_t)a * 16 + stage) * 8 + pk0;
        auto& t = ctx->tune[key];
        if (t.best >= 0) {
            A.cfg = t.best;
        } else if (ctx->steps_done > 0 && !ctx->capturing && t.next < gc_ctx::TUNE_ROUNDS * NUM_FORCE_CFG) {
            // time the configurations in turn (the first step, with its cold
            // sorts, is not timed)
            A.cfg = t.next++ % NUM_FORCE_CFG;
            if (ctx->tune_rec.size() == ctx->tune_ev.size()) {
                cudaEvent_t e0, e1;
                CU(cudaEventCreate(&e0));
                CU(cudaEventCreate(&e1));
                ctx->tune_ev.push_back({e0, e1});
            }
            tune_slot = (int)ctx->tune_rec.size();
            ctx->tune_rec.push_back({key, A.cfg});
        }
    }
    A.nref = 0;
    for (int id : ids)
        if (!ctx->inters[id].grid_valid) return seterr(ctx, GC_ERR_STATE, "sweep before create_grid");
    TRY(ensure_groups(ctx, a, ids[0], false));
    A.groups = S.groups;
    A.ngroups = S.d_ngroups;
    for (int id : ids) {
        DInter& D = ctx->inters[id];
        if (!D.grid_valid) return seterr(ctx, GC_ERR_STATE, "sweep before create_grid");
        if (A.nref == MAX_REFS) return seterr(ctx, GC_ERR_UNSUPPORTED, "too many interactions on one system");
        InterRef& r = A.ref[A.nref++];
        r.btype = D.btype == BT_VIRTUAL ? BT_GHOST : D.btype;  // virtual: the one-sided boundary forms
        r.gi = D.d_gi;
        r.pi = D.d_pi[stage - 1];
        r.cs = D.cs;
        r.cs_cells = D.cells;
        r.counts = D.counts;
        r.bbox = nullptr;
        if (D.btype == BT_GHOST) {
            DGhost& G = ctx->ghosts[D.bghost];
            r.bbox = G.d_inst;
            r.bx = G.x[G.cur];
            r.bv = G.v;
            r.brho = G.rho;
            r.bp = G.p;
            r.bstress = G.stress;
            r.bN = G.CAP;
            if (pfn != GC_PFN_COUNT && !xsph && !fp32)
                launch_aux(mode, G.CAP, G.d_count, G.rho, G.p, G.ginst[G.cur], G.d_mass, G.aux, ctx->stream);
            r.baux = G.aux;
            r.bfp = nullptr;
            r.bxp = nullptr;
            if (fp32) {
                TRY(ensure_fpk(ctx, G, G.CAP, G.nd, pk_ns));
                const bool pos = G.xpk_epoch != ctx->pack_epoch;
                launch_pack32(mode, G.CAP, G.d_count, G.nd, pk_ns, G.x[G.cur], G.v, G.rho, G.p, G.stress,
                              G.ginst[G.cur], G.d_mass, pos ? xp_of(G.fpk) : nullptr, pk_of(G.fpk, G.CAP, G.nd),
                              ctx->stream);
                G.xpk_epoch = ctx->pack_epoch;
                r.bfp = pk_of(G.fpk, G.CAP, G.nd);
                r.bxp = xp_of(G.fpk);
            }
        } else {
            DSlot& B = ctx->slots[D.bslot];
            if (D.btype != BT_SELF) r.bbox = B.d_inst;
            r.bx = B.F(F_X);
            r.bv = B.F(F_V);
            r.brho = B.F(F_RHO);
            r.bp = B.F(F_P);
            r.bstress = B.F(F_STRESS);
            r.bN = B.N;
            r.bfp = nullptr;
            r.bxp = nullptr;
            if (D.btype == BT_SELF) {
                r.baux = S.aux;
                if (fp32) {
                    r.bfp = pk_of(S.fpk, S.N, S.nd);
                    r.bxp = xp_of(S.fpk);
                }
            } else if ((D.btype == BT_SYSTEM || D.btype == BT_VIRTUAL) && pfn != GC_PFN_COUNT && !xsph && !fp32 &&
                       pk0 != GC_PFN_FLUID_SOLID) {
                launch_aux(mode, B.N, nullptr, B.F(F_RHO), B.F(F_P), B.inst_of, B.d_mass, B.aux, ctx->stream);
                r.baux = B.aux;
            } else {
                r.baux = B.aux;
            }
            if (fp32 && D.btype != BT_SELF) {
                // dynamic walls lend only their positions; other systems their records too
                const bool rec = D.btype == BT_SYSTEM || D.btype == BT_STATIC || D.btype == BT_VIRTUAL;
                TRY(ensure_fpk(ctx, B, B.N, B.nd, pk_ns));
                // positions: once per step, once for good for a system that does not move
                const bool pos = B.xmoves() ? B.xpk_epoch != ctx->pack_epoch : !B.xpk_static;
                launch_pack32(mode, B.N, nullptr, B.nd, pk_ns, B.F(F_X), B.F(F_V), B.F(F_RHO), B.F(F_P),
                              B.kind >= GC_SYS_STRESS ? B.F(F_STRESS) : nullptr, B.inst_of, B.d_mass,
                              pos ? xp_of(B.fpk) : nullptr, rec ? pk_of(B.fpk, B.N, B.nd) : nullptr, ctx->stream);
                B.xpk_epoch = ctx->pack_epoch;
                if (!B.xmoves()) B.xpk_static = true;
                r.bxp = xp_of(B.fpk);
                if (rec) {
                    r.bfp = pk_of(B.fpk, B.N, B.nd);
                    B.pack_done_epoch = -1;  // packed in this sweep's mode: B's own sweep packs again
                }
            }
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx->profiling && !count_only) {
        if (ctx->ev_used == ctx->ev_pool.size()) {
            cudaEvent_t a, b;
            CU(cudaEventCreate(&a));
            CU(cudaEventCreate(&b));
            ctx->ev_pool.push_back({a, b});
        }
        e0 = ctx->ev_pool[ctx->ev_used].first;
        e1 = ctx->ev_pool[ctx->ev_used].second;
        ctx->ev_used++;
        // inside a capture the record must become a node of the graph
        CU(cudaEventRecordWithFlags(e0, ctx->stream, ctx->capturing ? cudaEventRecordExternal : cudaEventRecordDefault));
    }
    if (tune_slot >= 0) CU(cudaEventRecord(ctx->tune_ev[tune_slot].first, ctx->stream));
    int st = launch_force_f64(A, count_only, ctx->stream);
    if (st) return seterr(ctx, st, "functor/system combination not implemented on the device");
    if (tune_slot >= 0) CU(cudaEventRecord(ctx->tune_ev[tune_slot].second, ctx->stream));
    if (e1)
        CU(cudaEventRecordWithFlags(e1, ctx->stream, ctx->capturing ? cudaEventRecordExternal : cudaEventRecordDefault));
    TRY(check_launch(ctx, "sweep"));
    // system_b side of two-sided interactions (counting functor; FluidPfn
    // between two fluid systems): a gather over system_b's particles through
    // system_a's CSR on the same grid, the functor's terms with the roles
    // swapped
    for (int id : ids) {
        DInter& D = ctx->inters[id];
        if (count_only || !b_side_at(D, stage)) continue;
        if (D.btype == BT_GHOST) {
            TRY(xsph_ghost_side(ctx, A, id, stage));
            continue;
        }
        DSlot& B = ctx->slots[D.bslot];
        TRY(ensure_groups(ctx, D.bslot, id, true));
        ForceArgs R = A;
        R.groups = B.groups;
        R.ngroups = B.d_ngroups;
        R.nd = B.nd;
        R.ns = B.ns;
        R.aN = B.N;
        R.a_inst_of = B.inst_of;
        R.ax = B.F(F_X);
        R.av = B.F(F_V);
        R.arho = B.F(F_RHO);
        R.aaux = B.aux;
        R.astress = B.F(F_STRESS);
        R.a_p = B.F(F_P);
        R.advdt = xsph ? B.F(F_VADJ) : B.F(F_DVDT);
        R.adrhodt = B.F(F_DRHODT);
        R.asr = B.F(F_SR);
        R.avort = B.F(F_VORT);
        R.a_c = B.d_c;
        R.a_mass = B.d_mass;
        R.a_cf = B.d_cf;
        R.a_massf = B.d_massf;
        R.afp = fp32 ? pk_of(B.fpk, B.N, B.nd) : nullptr;
        R.nref = 1;
        InterRef& r = R.ref[0];
        r.btype = BT_SYSTEM;
        r.bbox = S.d_inst;
        r.gi = D.d_gi_b;
        r.pi = D.d_pi[stage - 1];
        r.cs = D.cs_a;
        r.cs_cells = D.cells;
        r.counts = nullptr;
        r.bx = S.F(F_X);
        r.bv = S.F(F_V);
        r.brho = S.F(F_RHO);
        r.bp = S.F(F_P);
        r.bstress = S.F(F_STRESS);
        r.baux = S.aux;
        r.bN = S.N;
        r.bfp = fp32 ? pk_of(S.fpk, S.N, S.nd) : nullptr;
        r.bxp = fp32 ? xp_of(S.fpk) : nullptr;
        st = launch_force_f64(R, false, ctx->stream);
        if (st) return seterr(ctx, st, "two-sided functor not implemented on the device");
        TRY(check_launch(ctx, "sweep (system_b side)"));
    }
    return GC_OK;
}

int sweep_stage(gc_ctx* ctx, int stage) {
    for (size_t a = 0; a < ctx->slots.size(); ++a)
        for (auto& ids : stage_groups(ctx, (int)a, stage)) TRY(sweep_group(ctx, (int)a, ids, stage, false));
    return GC_OK;
}

void upload_inst_params(gc_ctx* ctx, double cfl) {
    const int ni = ninst(ctx);
    for (int k = 0; k < ni; ++k) {
        const HInst& I = ctx->inst[k];
        double h = 1e300, c = -1e300;
        for (auto& it : I.inters)
            if (!it.probe) h = std::min(h, it.H);
        for (auto& s : I.sys)
            if (!s.vsrc) c = std::max(c, s.c);  // the integrator's systems (src/TimeIntegration.jl:63)
        double dt = (std::isfinite(I.cfl) ? I.cfl : cfl) * h / c;
        for (auto& S : ctx->slots) {
            S.h_inst[k].dt = dt;
            S.h_inst[k].half_dt = dt / 2.0;
            S.h_inst[k].gamma_dt = I.gamma != 0.0 && dt > 0.0 ? I.gamma / dt : 0.0;  // dt = 0: a frozen instance
            S.h_inst[k].sort_cutoff = 2.0 * h;
        }
    }
}

int push_slot_params(gc_ctx* ctx, DSlot& S) {
    // Only the host-owned members; bbox/plan members are device-written.
    const int ni = ninst(ctx);
    std::vector<SysInst> cur(ni);
    TRY(hcopy(ctx, cur.data(), S.d_inst, ni * sizeof(SysInst), cudaMemcpyDeviceToHost));
    for (int k = 0; k < ni; ++k) {
        cur[k].base = S.h_inst[k].base;
        cur[k].n = S.h_inst[k].n;
        cur[k].mass = S.h_inst[k].mass;
        cur[k].c = S.h_inst[k].c;
        for (int d = 0; d < 3; ++d) cur[k].srcv[d] = S.h_inst[k].srcv[d];
        cur[k].srcrho = S.h_inst[k].srcrho;
        cur[k].sort_cutoff = S.h_inst[k].sort_cutoff;
        cur[k].dt = S.h_inst[k].dt;
        cur[k].half_dt = S.h_inst[k].half_dt;
        cur[k].gamma_dt = S.h_inst[k].gamma_dt;
    }
    TRY(hcopy(ctx, S.d_inst, cur.data(), ni * sizeof(SysInst), cudaMemcpyHostToDevice));
    return GC_OK;
}

// Returns true when some slot's motion changed (the step's structure with it).
bool decide_motion(gc_ctx* ctx) {
    bool changed = false;
    for (auto& S : ctx->slots) {
        bool src_zero = true;
        for (auto& h : S.h_inst) {
            for (int d = 0; d < S.nd; ++d) src_zero &= h.srcv[d] == 0.0;
            src_zero &= h.srcrho == 0.0;
        }
        bool kin_zero = true;
        for (auto v : S.nonzero_kin) kin_zero &= v == 0;
        // a virtual system's source is not one of the integrator's systems
        const bool m = !S.vsrc && (S.written || !src_zero || !kin_zero);
        changed |= m != S.moving;
        S.moving = m;
    }
    return changed;
}

int one_step_rk4(gc_ctx* ctx);

// _sweep_all_stages! src/TimeIntegration.jl:401-419: the virtual systems'
// w_sum and zero_fields cleared, then per stage the systems' updaters, the
// ghosts' copiers, the virtual systems' updaters and the sweeps.
int sweep_all_stages(gc_ctx* ctx) {
    for (auto& V : ctx->virts) {
        if (V.probe) continue;  // probes are cleared at measurement
        DSlot& S = ctx->slots[V.src];
        CU(cudaMemsetAsync(V.wsum, 0, sizeof(double) * S.N, ctx->stream));
        for (int f = 0; f < GC_NFIELDS; ++f) {
            if (!(V.zmask & (1 << f))) continue;
            const int k = field_slot(f);
            if (k >= 0 && S.ncomp[k]) CU(cudaMemsetAsync(S.F(k), 0, sizeof(double) * S.ncomp[k] * S.N, ctx->stream));
        }
    }
    for (int stage = 1; stage <= ctx->nstages; ++stage) {
        for (auto& S : ctx->slots)
            if (!S.vsrc && S.upd_set && S.nupd == ctx->nstages &&
                !(stage == 1 && S.upd_fused_epoch == ctx->pack_epoch))
                TRY(run_updaters(ctx, S, stage, NAN));
        for (auto& G : ctx->ghosts) TRY(ghost_copy(ctx, G, stage));
        for (auto& V : ctx->virts)
            if (!V.probe && V.upd_set && V.nupd == ctx->nstages) TRY(run_virtual_updaters(ctx, V, stage));
        TRY(sweep_stage(ctx, stage));
    }
    return GC_OK;
}

// _update_virtual_positions! :389-397, one virtual system after another
int advance_virtuals(gc_ctx* ctx) {
    for (auto& V : ctx->virts) {
        if (!V.moves) continue;  // x += 0·dt leaves x as it is
        DSlot& S = ctx->slots[V.src];
        launch_virtual_advance(S.F(F_X), S.N, S.nd, S.inst_of, S.d_inst, V.d_vi, ctx->stream);
    }
    return check_launch(ctx, "virtual positions");
}

// _xsph_correction! src/TimeIntegration.jl:421-436 after the full step has
// subtracted and zeroed v_adjustment: adjust_v! of every interaction with a
// velocity-adjust functor (stage nstages + 1, fused per system_a), then
// v += v_adjustment and the position update.
int xsph_pass(gc_ctx* ctx) {
    const int stage = ctx->nstages + 1;
    for (size_t a = 0; a < ctx->slots.size(); ++a) {
        std::vector<int> ids;
        for (size_t i = 0; i < ctx->inters.size(); ++i)
            if (ctx->inters[i].a == (int)a && ctx->inters[i].vadj) ids.push_back((int)i);
        for (size_t off = 0; off < ids.size(); off += MAX_REFS) {
            std::vector<int> chunk(ids.begin() + off, ids.begin() + std::min(ids.size(), off + MAX_REFS));
            TRY(sweep_group(ctx, (int)a, chunk, stage, false));
        }
    }
    for (auto& S : ctx->slots)
        if (S.moving) launch_xsph_final(step_args(S), ctx->stream);
    return check_launch(ctx, "XSPH correction");
}

// The LeapFrog half step of slot `a` fused with the stage-1 work that
// follows it for the same particles: its stage-1 updater when that is one
// light elementwise kind (moved here from _sweep_all_stages!, :401-419;
// nothing between the two reads or writes what it touches) and, for an
// FP32-compensated first sweep after it, that sweep's records
// (sweep_group then finds them packed).
int halfstep_stage1(gc_ctx* ctx, int a) {
    DSlot& S = ctx->slots[a];
    UpdArgs u{};
    u.kind = -1;
    // a stage-1 chain of at most one light updater moves into the half step
    const bool has1 = !S.vsrc && S.upd_set && S.nupd == ctx->nstages && ctx->nstages >= 1 && !S.d_upd.empty();
    const bool upd = has1 && S.d_upd[0].size() == 1 && halfstep_fuses(S.upd_kind[0][0]);
    if (upd) u = upd_args(S, 1, 0, NAN);
    PackArgs pk{};
    if (upd || !has1 || S.d_upd[0].empty()) {  // the pack follows the stage-1 updaters
        const auto groups = ctx->nstages >= 1 ? stage_groups(ctx, a, 1) : std::vector<std::vector<int>>{};
        if (!groups.empty()) {
            const PackPlan pl = pack_plan(ctx, a, groups[0], 1, false);
            if (pl.fp32 && !pl.interp && !pl.xsph && pl.pfn != GC_PFN_COUNT) {
                TRY(ensure_fpk(ctx, S, S.N, S.nd, pl.pk_ns));
                const bool pos = S.xpk_epoch != ctx->pack_epoch;
                pk = PackArgs{pl.mode, S.nd, pl.pk_ns, S.N, S.F(F_X), S.F(F_V), S.F(F_RHO), S.F(F_P), S.F(F_STRESS),
                              S.inst_of, S.d_mass, pos ? (double*)S.fpk : nullptr,
                              S.fpk + S.N * 2 * pos_stride(S.nd)};
                S.xpk_epoch = ctx->pack_epoch;
                S.pack_done_epoch = ctx->pack_epoch;
                S.pack_done_stage = 1;
                S.pack_done_mode = pl.mode;
                S.pack_done_ns = pl.pk_ns;
            }
        }
    }
    launch_halfstep_fused(step_args(S), u, pk, ctx->stream);
    if (upd) S.upd_fused_epoch = ctx->pack_epoch;
    return GC_OK;
}

int one_step(gc_ctx* ctx) {
    if (ctx->inst[0].integ == GC_INTEGRATOR_RK4) return one_step_rk4(ctx);
    ctx->pack_epoch++;
    std::vector<char> mask(ctx->slots.size());
    for (size_t s = 0; s < ctx->slots.size(); ++s) {
        DSlot& S = ctx->slots[s];
        mask[s] = !S.probe && (S.xmoves() || !S.sorted_once);  // probes: sorted at measurement
    }
    TRY(prepare(ctx, mask));
    for (size_t s = 0; s < ctx->slots.size(); ++s)
        if (mask[s]) ctx->slots[s].sorted_once = true;
    ctx->resorts += 1;
    for (size_t a = 0; a < ctx->slots.size(); ++a)
        if (ctx->slots[a].moving) TRY(halfstep_stage1(ctx, (int)a));
    TRY(check_launch(ctx, "half step"));
    for (auto& G : ctx->ghosts) TRY(ghost_kinematics(ctx, G));
    TRY(sweep_all_stages(ctx));
    for (auto& S : ctx->slots)
        if (S.moving) launch_fullstep(step_args(S), ctx->stream);
    TRY(check_launch(ctx, "full step"));
    if (ctx->xsph) TRY(xsph_pass(ctx));
    TRY(advance_virtuals(ctx));
    ctx->steps_done += 1;
    return GC_OK;
}

// src/TimeIntegration.jl:771-826: one grid per step, four right-hand-side
// evaluations from q0, q = q0 + dt·(k1/6 + k2/3 + k3/3 + k4/6), positions once.
int one_step_rk4(gc_ctx* ctx) {
    ctx->pack_epoch++;
    std::vector<char> mask(ctx->slots.size());
    for (size_t s = 0; s < ctx->slots.size(); ++s) {
        DSlot& S = ctx->slots[s];
        mask[s] = !S.probe && (S.xmoves() || !S.sorted_once);  // probes: sorted at measurement
        if (S.moving && !S.accv) {
            TRY(dalloc(ctx, &S.accv, (size_t)S.nd * S.N));
            TRY(dalloc(ctx, &S.accrho, (size_t)S.N));
        }
    }
    TRY(prepare(ctx, mask));
    for (size_t s = 0; s < ctx->slots.size(); ++s)
        if (mask[s]) ctx->slots[s].sorted_once = true;
    ctx->resorts += 1;
    // Julia's T(0.5), T(1.0) and T(1/6), T(1/3) (src/TimeIntegration.jl:742-743)
    const double advance[4] = {0.0, 0.5, 0.5, 1.0};
    const double weight[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    for (auto& S : ctx->slots)
        if (S.moving) launch_rk4_begin(step_args(S), ctx->stream);
    for (int it = 0; it < 4; ++it) {
        if (it > 0)
            for (auto& S : ctx->slots)
                if (S.moving) launch_rk4_advance(step_args(S), advance[it], ctx->stream);
        TRY(check_launch(ctx, "rk4 stage"));
        for (auto& G : ctx->ghosts) TRY(ghost_kinematics(ctx, G));
        TRY(sweep_all_stages(ctx));
        for (auto& S : ctx->slots)
            if (S.moving) launch_rk4_acc(step_args(S), weight[it], ctx->stream);
    }
    for (auto& S : ctx->slots)
        if (S.moving) launch_rk4_final(step_args(S), ctx->stream);
    TRY(check_launch(ctx, "rk4 final"));
    if (ctx->xsph) TRY(xsph_pass(ctx));
    TRY(advance_virtuals(ctx));
    ctx->steps_done += 1;
    return GC_OK;
}

int collect_profile(gc_ctx* ctx) {
    for (size_t i = 0; i < ctx->tune_rec.size(); ++i) {
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, ctx->tune_ev[i].first, ctx->tune_ev[i].second));
        auto& t = ctx->tune[ctx->tune_rec[i].first];
        double& m = t.ms[ctx->tune_rec[i].second];
        m = m > 0.0 ? std::min(m, (double)ms) : (double)ms;
        if (t.next == gc_ctx::TUNE_ROUNDS * NUM_FORCE_CFG && t.best < 0) {
            int b = 0;
            for (int c = 1; c < NUM_FORCE_CFG; ++c)
                if (t.ms[c] < t.ms[b]) b = c;
            t.best = b;
            ctx->tune_version++;
        }
    }
    ctx->tune_rec.clear();
    for (size_t i = 0; i < ctx->ev_used; ++i) {
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, ctx->ev_pool[i].first, ctx->ev_pool[i].second));
        ctx->sweep_ms += ms;
        ctx->sweep_launches += 1;
    }
    ctx->ev_used = 0;
    return GC_OK;
}

int finish_status(gc_ctx* ctx) {
    CU(cudaStreamSynchronize(ctx->stream));
    TRY(collect_profile(ctx));
    int e = 0;
    TRY(hcopy(ctx, &e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    ctx->last_status = e;
    if (e & ERR_NONFINITE) return seterr(ctx, GC_ERR_NONFINITE, "non-finite or out-of-range particle position");
    if (e & ERR_CAPACITY) return seterr(ctx, GC_ERR_CAPACITY, "a particle fell outside its grid or key range");
    if (e & ERR_XSPH_GHOST)
        return seterr(ctx, GC_ERR_UNSUPPORTED,
                      "XSPH against a ghost system wrote beyond the ghost source's length (out of bounds in the "
                      "reference)");
    return GC_OK;
}

bool valid_inst(gc_ctx* ctx, int inst) { return inst >= 0 && inst < (int)ctx->inst.size(); }
// ------------------------------------------------------- graph stepping
void drop_graphs(gc_ctx* ctx) {
    for (auto& g : ctx->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    ctx->graphs.clear();
}

// Any change of model state outside gc_step: the next step runs exactly
// (and sorts static systems again where asked), graphs are recaptured.
void invalidate_steps(gc_ctx* ctx) {
    drop_graphs(ctx);
    ctx->exact_done = false;
}

std::vector<char> parity(gc_ctx* ctx) {
    std::vector<char> p;
    for (auto& S : ctx->slots) p.push_back((char)S.cur);
    for (auto& G : ctx->ghosts) p.push_back((char)G.cur);
    return p;
}

void set_parity(gc_ctx* ctx, const std::vector<char>& p) {
    size_t i = 0;
    for (auto& S : ctx->slots) S.cur = p[i++];
    for (auto& G : ctx->ghosts) G.cur = p[i++];
}

int graph_key(gc_ctx* ctx) {
    return (int)(((ctx->precision * 64 + ctx->force_cfg + 1) * 2 + (ctx->profiling ? 1 : 0)) * 4096 +
                 ctx->tune_version % 4096);
}

// Steps stay exact (and timed) until every sweep has its configuration.
bool tuning(gc_ctx* ctx) {
    if (ctx->force_cfg >= 0) return false;
    if (ctx->tune.empty()) return true;
    for (auto& kv : ctx->tune)
        if (kv.second.best < 0) return true;
    return false;
}

template <class St>
int grow_gcols(gc_ctx* ctx, St& S, int64_t ncols) {
    if (ncols + 1 <= S.cap_gcols) return GC_OK;
    CU(cudaStreamSynchronize(ctx->stream));
    dfree(ctx, S.gcnt, S.cap_gcols);
    dfree(ctx, S.goff, S.cap_gcols);
    int64_t cap = ncols + 1 + ncols / 4;
    TRY(dalloc(ctx, &S.gcnt, (size_t)cap));
    TRY(dalloc(ctx, &S.goff, (size_t)cap));
    S.cap_gcols = cap;
    return GC_OK;
}

// Capacities for capacity-mode steps: every planned cell count seen so far,
// times the margin.  Growth happens here, at a verified point, never inside
// a captured step.
int size_capacities(gc_ctx* ctx) {
    const int n = ctx->nneed;
    CU(cudaMemcpyAsync(ctx->h_need_max, ctx->d_need_max, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < n; ++i) ctx->need_max[i] = std::max(ctx->need_max[i], ctx->h_need_max[i]);
    const double m = ctx->cap_margin;
    auto want = [&](int64_t need) { return (int64_t)((double)need * m) + 1024; };
    auto low = [&](int64_t need) { return (int64_t)((double)need * (1.0 + (m - 1.0) / 2.0)) + 512; };
    int64_t all = 0;
    for (int i = 0; i < n; ++i) all = std::max(all, ctx->need_max[i]);
    if (ctx->cap_cells - 1 < low(all)) TRY(ensure_cells(ctx, want(all)));
    for (auto& D : ctx->inters) {
        if (D.probe) continue;
        const int64_t nm = ctx->need_max[D.need_slot];
        if (D.cap_cells - 1 < low(nm)) TRY(ensure_inter_cells(ctx, D, want(nm)));
    }
    // scan scratch for ghost flags and for every capacity-sized scan
    int64_t scan_n = ctx->cap_cells;
    for (auto& G : ctx->ghosts) scan_n = std::max(scan_n, G.CAP);
    int64_t st = scan_tmp_elems(scan_n) + 16;
    if (st > ctx->cap_scan) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, ctx->scan_tmp, ctx->cap_scan);
        TRY(dalloc(ctx, &ctx->scan_tmp, (size_t)st));
        ctx->cap_scan = st;
    }
    // warp-group column tables of every system a grid groups
    for (auto& D : ctx->inters) {
        if (D.probe) continue;
        const int64_t cells = cap_grid_cells(ctx, D);
        TRY(grow_gcols(ctx, ctx->slots[D.a], cells));
        if (D.two_sided && D.bslot >= 0) TRY(grow_gcols(ctx, ctx->slots[D.bslot], cells));
        if (D.vadj && D.btype == BT_GHOST) TRY(grow_gcols(ctx, ctx->ghosts[D.bghost], cells));
    }
    // the bound each plan entry is checked against inside the steps
    std::vector<int64_t> cap(n);
    for (size_t s = 0; s < ctx->slots.size(); ++s) cap[s] = cap_sort_cells(ctx);
    for (auto& G : ctx->ghosts) cap[G.need_slot] = cap_sort_cells(ctx);
    for (auto& D : ctx->inters) cap[D.need_slot] = D.probe ? INT64_MAX : cap_grid_cells(ctx, D);
    TRY(hcopy(ctx, ctx->d_need_cap, cap.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice));
    return GC_OK;
}

// Snapshot of every moving slot's carried state (current buffers), the
// rollback point of a capacity-mode window.
int snapshot(gc_ctx* ctx, std::vector<char>& par) {
    ctx->snaps.resize(ctx->slots.size());
    for (size_t s = 0; s < ctx->slots.size(); ++s) {
        DSlot& S = ctx->slots[s];
        Snapshot& sn = ctx->snaps[s];
        if (!S.xmoves()) continue;
        if (sn.n != S.N) {
            for (int f = 0; f < NF; ++f) dfree(ctx, sn.f[f], (size_t)S.ncomp[f] * sn.n);
            dfree(ctx, sn.id, (size_t)sn.n);
            for (int f = 0; f < NF; ++f)
                if (S.ncomp[f]) TRY(dalloc(ctx, &sn.f[f], (size_t)S.ncomp[f] * S.N));
            TRY(dalloc(ctx, &sn.id, (size_t)S.N));
            sn.n = S.N;
        }
        for (int f = 0; f < NF; ++f)
            if (S.ncomp[f])
                CU(cudaMemcpyAsync(sn.f[f], S.F(f), sizeof(double) * S.ncomp[f] * S.N, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        CU(cudaMemcpyAsync(sn.id, S.id[S.cur], sizeof(int32_t) * S.N, cudaMemcpyDeviceToDevice, ctx->stream));
        sn.cur = S.cur;
    }
    par = parity(ctx);
    return GC_OK;
}

int restore(gc_ctx* ctx, const std::vector<char>& par) {
    set_parity(ctx, par);
    for (size_t s = 0; s < ctx->slots.size(); ++s) {
        DSlot& S = ctx->slots[s];
        Snapshot& sn = ctx->snaps[s];
        if (!S.xmoves()) continue;
        for (int f = 0; f < NF; ++f)
            if (S.ncomp[f])
                CU(cudaMemcpyAsync(S.F(f), sn.f[f], sizeof(double) * S.ncomp[f] * S.N, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        CU(cudaMemcpyAsync(S.id[S.cur], sn.id, sizeof(int32_t) * S.N, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return GC_OK;
}

int ev_pair(gc_ctx* ctx, size_t i) {
    while (ctx->ev_pool.size() <= i) {
        cudaEvent_t a, b;
        CU(cudaEventCreate(&a));
        CU(cudaEventCreate(&b));
        ctx->ev_pool.push_back({a, b});
    }
    return GC_OK;
}

// A copy of a captured step whose kernel-to-kernel edges are programmatic:
// a kernel may launch once every block of the kernel before it has passed
// pdl_enter (where each kernel first waits for its predecessors to finish),
// so the launches overlap the kernels before them.  Returns nullptr (the
// step keeps its plain edges) when GC_NO_PDL is set or the copy cannot be
// made and instantiated.
static cudaGraph_t programmatic_copy(cudaGraph_t graph) {
    static const bool off = [] {
        const char* e = getenv("GC_NO_PDL");
        return e && *e && *e != '0';
    }();
    if (off) return nullptr;
    size_t ne = 0;
    if (cudaGraphGetEdges_v2(graph, nullptr, nullptr, nullptr, &ne) != cudaSuccess || ne == 0) {
        cudaGetLastError();
        return nullptr;
    }
    std::vector<cudaGraphNode_t> from(ne), to(ne);
    std::vector<cudaGraphEdgeData> ed(ne);
    cudaGraph_t cl = nullptr;
    bool ok = cudaGraphGetEdges_v2(graph, from.data(), to.data(), ed.data(), &ne) == cudaSuccess &&
              cudaGraphClone(&cl, graph) == cudaSuccess;
    int converted = 0;
    for (size_t i = 0; ok && i < ne; ++i) {
        cudaGraphNodeType ta, tb;
        ok = cudaGraphNodeGetType(from[i], &ta) == cudaSuccess && cudaGraphNodeGetType(to[i], &tb) == cudaSuccess;
        if (!ok || ta != cudaGraphNodeTypeKernel || tb != cudaGraphNodeTypeKernel ||
            ed[i].type != cudaGraphDependencyTypeDefault)
            continue;
        cudaGraphNode_t a = nullptr, b = nullptr;
        ok = cudaGraphNodeFindInClone(&a, from[i], cl) == cudaSuccess &&
             cudaGraphNodeFindInClone(&b, to[i], cl) == cudaSuccess;
        cudaGraphEdgeData pe = ed[i];
        pe.from_port = cudaGraphKernelNodePortProgrammatic;
        pe.type = cudaGraphDependencyTypeProgrammatic;
        ok = ok && cudaGraphRemoveDependencies_v2(cl, &a, &b, &ed[i], 1) == cudaSuccess &&
             cudaGraphAddDependencies_v2(cl, &a, &b, &pe, 1) == cudaSuccess;
        converted += ok ? 1 : 0;
    }
    cudaGraphExec_t ex = nullptr;
    ok = ok && converted > 0 && cudaGraphInstantiate(&ex, cl, 0) == cudaSuccess;
    if (ex) cudaGraphExecDestroy(ex);
    if (!ok) {
        cudaGetLastError();
        if (cl) cudaGraphDestroy(cl);
        return nullptr;
    }
    return cl;
}

// Capture one capacity-mode step into `g` (nothing runs).
int capture_step(gc_ctx* ctx, StepGraph& g) {
    if (ctx->profiling) TRY(ev_pair(ctx, ctx->ev_used + 4 * ctx->slots.size() * (size_t)std::max(ctx->nstages, 1)));
    g.pre = parity(ctx);
    const size_t ev0 = ctx->ev_used;
    const long long l0 = g_launches.load();
    const int64_t steps0 = ctx->steps_done, resorts0 = ctx->resorts;
    CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->capturing = true;
    int st = one_step(ctx);
    ctx->capturing = false;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    g.launches = g_launches.load() - l0;
    g_launches.fetch_sub(g.launches);  // the capture launched nothing
    ctx->steps_done = steps0;
    ctx->resorts = resorts0;
    const size_t ev1 = ctx->ev_used;
    ctx->ev_used = ev0;
    if (st != GC_OK || e != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        set_parity(ctx, g.pre);
        if (st != GC_OK) return st;
        return seterr(ctx, GC_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
    }
    g.post = parity(ctx);
    set_parity(ctx, g.pre);
    if (cudaGraph_t pg = programmatic_copy(graph)) {
        cudaGraphDestroy(graph);
        graph = pg;
    }
    g.graph = graph;
    if (ev1 > ev0) {
        size_t nn = 0;
        CU(cudaGraphGetNodes(graph, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        CU(cudaGraphGetNodes(graph, nodes.data(), &nn));
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            CU(cudaGraphNodeGetType(nd, &t));
            if (t != cudaGraphNodeTypeEventRecord) continue;
            cudaEvent_t ev;
            CU(cudaGraphEventRecordNodeGetEvent(nd, &ev));
            for (size_t i = ev0; i < ev1; ++i) {
                if (ctx->ev_pool[i].first == ev || ctx->ev_pool[i].second == ev) {
                    g.ev_nodes.push_back(nd);
                    g.ev_slots.push_back({(int64_t)(i - ev0), ctx->ev_pool[i].first == ev ? 0 : 1});
                }
            }
        }
    }
    CU(cudaGraphInstantiate(&g.exec, graph, 0));
    return GC_OK;
}

int replay_step(gc_ctx* ctx, StepGraph& g) {
    if (!g.ev_nodes.empty()) {
        int64_t npairs = 0;
        for (auto& sl : g.ev_slots) npairs = std::max(npairs, sl[0] + 1);
        TRY(ev_pair(ctx, ctx->ev_used + (size_t)npairs));
        for (size_t q = 0; q < g.ev_nodes.size(); ++q) {
            auto& pr = ctx->ev_pool[ctx->ev_used + (size_t)g.ev_slots[q][0]];
            CU(cudaGraphExecEventRecordNodeSetEvent(g.exec, g.ev_nodes[q], g.ev_slots[q][1] ? pr.second : pr.first));
        }
        ctx->ev_used += (size_t)npairs;
    }
    CU(cudaGraphLaunch(g.exec, ctx->stream));
    set_parity(ctx, g.post);
    g_launches.fetch_add(g.launches);
    ctx->steps_done += 1;
    ctx->resorts += 1;
    ctx->graph_steps += 1;
    return GC_OK;
}

StepGraph* find_graph(gc_ctx* ctx) {
    const std::vector<char> p = parity(ctx);
    for (auto& g : ctx->graphs)
        if (g.pre == p) return &g;
    return nullptr;
}

// `nsteps` steps.  Without graphs (or for the first step after a change):
// exact steps, each sized by one host read of the plan.  Otherwise windows
// of up to `sync_every` captured capacity-mode steps, verified at the end of
// each window; a window whose plan outgrew a capacity is rolled back to its
// snapshot and re-run exactly.
int run_steps(gc_ctx* ctx, int nsteps) {
    static const bool env_off = [] {
        const char* e = getenv("GC_GRAPHS");
        return e && e[0] == '0';
    }();
    bool graphs = ctx->graphs_on && !env_off;
    int done = 0;
    while (done < nsteps) {
        if (!graphs || !ctx->exact_done || tuning(ctx)) {
            ctx->capmode = false;
            TRY(one_step(ctx));
            ctx->exact_done = true;
            ++done;
            continue;
        }
        TRY(size_capacities(ctx));
        const int W = std::min(ctx->sync_every, nsteps - done);
        // A one-step window needs no snapshot: the step's sort gathers every
        // moving system into its other buffers and leaves the current ones
        // untouched, so going back is a flip of the buffer parities.
        std::vector<char> par0;
        // a probe moved by prescribed_v is not re-sorted in the step, so only
        // a snapshot takes it back
        bool probe_moves = false;
        for (auto& S : ctx->slots) probe_moves |= S.probe && S.vmoves;
        const bool snap = W > 1 || probe_moves;
        if (!snap) par0 = parity(ctx);
        else TRY(snapshot(ctx, par0));
        if (ctx->alloc_epoch != ctx->graphs_epoch || graph_key(ctx) != ctx->graphs_key) {
            drop_graphs(ctx);
            ctx->graphs_epoch = ctx->alloc_epoch;
            ctx->graphs_key = graph_key(ctx);
        }
        int ran = 0;
        int cap_err = GC_OK;
        ctx->capmode = true;
        for (; ran < W; ++ran) {
            StepGraph* g = find_graph(ctx);
            if (!g) {
                ctx->graphs.emplace_back();
                cap_err = capture_step(ctx, ctx->graphs.back());
                if (cap_err != GC_OK) {
                    cudaGetLastError();  // the steps continue exactly
                    ctx->graphs.pop_back();
                    break;
                }
                g = &ctx->graphs.back();
            }
            TRY(replay_step(ctx, *g));
        }
        ctx->capmode = false;
        CU(cudaStreamSynchronize(ctx->stream));
        TRY(collect_profile(ctx));
        int e = 0;
        TRY(hcopy(ctx, &e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e & ERR_CAPACITY) {
            // a plan outgrew a capacity: back to the snapshot, then the same
            // steps exactly (which size every buffer from the plan)
            if (!snap) set_parity(ctx, par0);
            else TRY(restore(ctx, par0));
            ctx->steps_done -= ran;
            ctx->resorts -= ran;
            ctx->graph_steps -= ran;
            ctx->rollbacks += 1;
            for (auto& D : ctx->inters)  // a CSR counted inside the window may not have fitted
                if (D.d_keep) CU(cudaMemsetAsync(D.d_keep, 0, sizeof(int), ctx->stream));
            e &= ~ERR_CAPACITY;
            CU(cudaMemcpyAsync(ctx->d_err, &e, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            for (int w = 0; w < ran; ++w) TRY(one_step(ctx));
        } else if (e) {
            return GC_OK;  // finish_status reports it
        }
        done += ran;
        if (cap_err != GC_OK) graphs = false;  // this call continues exactly
    }
    return GC_OK;
}


}  // namespace

// ===================================================================== C ABI
extern "C" {

const char* gc_status_string(int st) {
    switch (st) {
        case GC_OK: return "GC_OK";
        case GC_ERR_ARG: return "GC_ERR_ARG";
        case GC_ERR_OOM: return "GC_ERR_OOM";
        case GC_ERR_CAPACITY: return "GC_ERR_CAPACITY";
        case GC_ERR_NONFINITE: return "GC_ERR_NONFINITE";
        case GC_ERR_GRID_INCONSISTENT: return "GC_ERR_GRID_INCONSISTENT";
        case GC_ERR_TIMEOUT: return "GC_ERR_TIMEOUT";
        case GC_ERR_CUDA: return "GC_ERR_CUDA";
        case GC_ERR_STATE: return "GC_ERR_STATE";
        case GC_ERR_UNSUPPORTED: return "GC_ERR_UNSUPPORTED";
    }
    return "unknown status";
}

int gc_ctx_create(int device, size_t hbm_budget_bytes, gc_ctx** out) {
    if (!out) return GC_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return GC_ERR_CUDA;
    if (device < 0 || device >= n) return GC_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GC_ERR_CUDA;
    gc_ctx* ctx = new gc_ctx();
    ctx->device = device;
    if (const char* e = getenv("GC_FORCE_CFG")) ctx->force_cfg = std::min(std::max(atoi(e), -1), NUM_FORCE_CFG - 1);
    ctx->budget = hbm_budget_bytes;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return GC_ERR_CUDA;
    }
    *out = ctx;
    return GC_OK;
}

int gc_ctx_destroy(gc_ctx* ctx) {
    if (!ctx) return GC_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& S : ctx->slots) {
        for (int b = 0; b < 2; ++b) {
            for (int f = 0; f < NF; ++f) dev_free(ctx, S.f[b][f]);
            dev_free(ctx, S.id[b]);
        }
        dev_free(ctx, S.q0v);
        dev_free(ctx, S.q0rho);
        dev_free(ctx, S.accv);
        dev_free(ctx, S.accrho);
        dev_free(ctx, S.aux);
        dev_free(ctx, S.inst_of);
        dev_free(ctx, S.groups);
        dev_free(ctx, S.d_ngroups);
        dev_free(ctx, S.gcnt);
        dev_free(ctx, S.goff);
        dev_free(ctx, S.d_inst);
        dev_free(ctx, S.d_mass);
        dev_free(ctx, S.d_c);
        dev_free(ctx, S.d_massf);
        dev_free(ctx, S.d_cf);
        dev_free(ctx, S.fpk);
        for (auto& ch : S.d_upd)
            for (auto* p : ch) dev_free(ctx, p);
    }
    for (auto& G : ctx->ghosts) {
        for (int b = 0; b < 2; ++b) {
            dev_free(ctx, G.x[b]);
            dev_free(ctx, G.io[b]);
            dev_free(ctx, G.ib[b]);
            dev_free(ctx, G.ginst[b]);
        }
        dev_free(ctx, G.normals);
        dev_free(ctx, G.v);
        dev_free(ctx, G.rho);
        dev_free(ctx, G.p);
        dev_free(ctx, G.stress);
        dev_free(ctx, G.aux);
        dev_free(ctx, G.flags);
        dev_free(ctx, G.pos);
        dev_free(ctx, G.d_count);
        dev_free(ctx, G.d_gh);
        dev_free(ctx, G.d_inst);
        dev_free(ctx, G.d_mass);
        dev_free(ctx, G.d_c);
        dev_free(ctx, G.fpk);
        dev_free(ctx, G.groups);
        dev_free(ctx, G.d_ngroups);
        dev_free(ctx, G.gcnt);
        dev_free(ctx, G.goff);
        dev_free(ctx, G.gadj);
    }
    for (auto& V : ctx->virts) {
        dev_free(ctx, V.wsum);
        dev_free(ctx, V.wsum_alt);
        dev_free(ctx, V.d_vi);
        for (auto& chain : V.d_upd)
            for (auto* p : chain) dev_free(ctx, p);
    }
    for (auto& D : ctx->inters) {
        dev_free(ctx, D.d_gi);
        dev_free(ctx, D.d_gi_b);
        for (auto* p : D.d_pi) dev_free(ctx, p);
        dev_free(ctx, D.cs);
        dev_free(ctx, D.cs_a);
        dev_free(ctx, D.counts);
        dev_free(ctx, D.d_keep);
        dev_free(ctx, D.d_gi_prev);
        dev_free(ctx, D.hist);
    }
    dev_free(ctx, ctx->key);
    dev_free(ctx, ctx->perm);
    dev_free(ctx, ctx->hist);
    dev_free(ctx, ctx->start);
    dev_free(ctx, ctx->fill);
    dev_free(ctx, ctx->scan_tmp);
    dev_free(ctx, ctx->bbox_scratch);
    dev_free(ctx, ctx->d_err);
    dev_free(ctx, ctx->d_unsorted);
    dev_free(ctx, ctx->d_sorts_in_order);
    dev_free(ctx, ctx->d_incons);
    dev_free(ctx, ctx->d_need);
    dev_free(ctx, ctx->d_total_cells);
    if (ctx->h_need) cudaFreeHost(ctx->h_need);
    dev_free(ctx, ctx->d_need_max);
    dev_free(ctx, ctx->d_need_cap);
    dev_free(ctx, ctx->d_plan_args);
    if (ctx->h_need_max) cudaFreeHost(ctx->h_need_max);
    drop_graphs(ctx);
    for (auto& sn : ctx->snaps) {
        for (int f = 0; f < NF; ++f) dev_free(ctx, sn.f[f]);
        dev_free(ctx, sn.id);
    }
    dev_free(ctx, ctx->staging);
    dev_free(ctx, ctx->d_ioflags);
    dev_free(ctx, ctx->d_pairs);
    for (auto& e : ctx->ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    for (auto& e : ctx->tune_ev) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (ctx->pool) cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return GC_OK;
}

const char* gc_last_error(gc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int gc_instance_add(gc_ctx* ctx, int* inst_out) {
    if (!ctx || !inst_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    ctx->inst.emplace_back();
    *inst_out = (int)ctx->inst.size() - 1;
    return GC_OK;
}

int gc_add_system(gc_ctx* ctx, int inst, int kind, int64_t n, int ndims, int ns, double mass, double c,
                  const double* source_v, double source_rho, int* sys_out) {
    if (!ctx || !sys_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance %d", inst);
    if (n <= 0) return seterr(ctx, GC_ERR_ARG, "n must be positive, got %lld", (long long)n);
    if (ndims < 2 || ndims > 3) return seterr(ctx, GC_ERR_UNSUPPORTED, "ndims must be 2 or 3, got %d", ndims);
    if (kind < GC_SYS_BASIC || kind > GC_SYS_ELASTOPLASTIC) return seterr(ctx, GC_ERR_ARG, "bad system kind");
    if (kind >= GC_SYS_STRESS && !(ns == 3 || ns == 4 || ns == 6))
        return seterr(ctx, GC_ERR_ARG, "ns must be 3, 4, or 6, got %d", ns);
    HInst& I = ctx->inst[inst];
    HSys s;
    s.kind = kind;
    s.n = n;
    s.nd = ndims;
    s.ns = kind >= GC_SYS_STRESS ? ns : 0;
    s.nvort = kind == GC_SYS_ELASTOPLASTIC ? (ndims == 2 ? 1 : 3) : 0;
    s.mass = mass;
    s.c = c;
    for (int d = 0; d < ndims; ++d) s.srcv[d] = source_v ? source_v[d] : 0.0;
    s.srcrho = source_rho;
    I.sys.push_back(s);
    HHandle h;
    h.type = H_SYS;
    h.idx = (int)I.sys.size() - 1;
    I.handles.push_back(h);
    I.sys_handle.push_back((int)I.handles.size() - 1);
    *sys_out = (int)I.handles.size() - 1;
    return GC_OK;
}

static int sys_of(gc_ctx* ctx, int inst, int handle) {
    if (!valid_inst(ctx, inst)) return -1;
    HInst& I = ctx->inst[inst];
    if (handle < 0 || handle >= (int)I.handles.size() || I.handles[handle].type != H_SYS) return -1;
    return I.handles[handle].idx;
}

int gc_add_boundary(gc_ctx* ctx, int inst, int sys, int kind, const double* normal, const double* point,
                    double beta_or_lj_cutoff, int* handle_out) {
    if (!ctx || !handle_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    int si = sys_of(ctx, inst, sys);
    if (si < 0) return seterr(ctx, GC_ERR_ARG, "boundary inner must be a system handle");
    HInst& I = ctx->inst[inst];
    HHandle h;
    h.idx = si;
    const int nd = I.sys[si].nd;
    if (kind == GC_WRAP_DYNAMIC) {
        if (!normal || !point) return seterr(ctx, GC_ERR_ARG, "dynamic boundary needs normal and point");
        h.type = H_DYN;
        for (int d = 0; d < nd; ++d) {
            h.normal[d] = normal[d];
            h.point[d] = point[d];
        }
        h.beta = beta_or_lj_cutoff;
    } else if (kind == GC_WRAP_STATIC) {
        h.type = H_STATIC;
        h.ljcut = beta_or_lj_cutoff;
    } else {
        return seterr(ctx, GC_ERR_ARG, "bad boundary kind %d", kind);
    }
    I.handles.push_back(h);
    *handle_out = (int)I.handles.size() - 1;
    return GC_OK;
}

int gc_add_ghost(gc_ctx* ctx, int inst, int src_sys, int ncopiers, const int* copier_nfields,
                 const int* copier_fields, const int* copier_modes, int nplanes, const double* normals,
                 const double* points, double cutoff, int64_t capacity, int* handle_out) {
    if (!ctx || !handle_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    int si = sys_of(ctx, inst, src_sys);
    if (si < 0) return seterr(ctx, GC_ERR_ARG, "ghost source must be a system handle");
    if (nplanes < 1) return seterr(ctx, GC_ERR_ARG, "at least one boundary (normal, point) pair is required");
    if (nplanes > GC_MAX_GHOST_PLANES)
        return seterr(ctx, GC_ERR_UNSUPPORTED, "at most %d planes per ghost entry", GC_MAX_GHOST_PLANES);
    HInst& I = ctx->inst[inst];
    const HSys& s = I.sys[si];
    HGhost g;
    g.src = si;
    g.cutoff = cutoff;
    g.nplanes = nplanes;
    for (int b = 0; b < nplanes; ++b)
        for (int d = 0; d < s.nd; ++d) {
            g.normals[b][d] = normals[b * s.nd + d];
            g.points[b][d] = points[b * s.nd + d];
        }
    int pos = 0;
    for (int k = 0; k < ncopiers; ++k) {
        std::vector<std::pair<int, int>> cp;
        for (int e = 0; e < copier_nfields[k]; ++e, ++pos) {
            int fld = copier_fields[pos], mode = copier_modes[pos];
            if (fld == GC_FIELD_P) {
                if (s.kind < GC_SYS_FLUID) return seterr(ctx, GC_ERR_ARG, "copier field p missing on source");
                g.ex_p = true;
            } else if (fld == GC_FIELD_STRESS) {
                if (s.kind < GC_SYS_STRESS) return seterr(ctx, GC_ERR_ARG, "copier field stress missing on source");
                g.ex_stress = true;
            } else if (fld != GC_FIELD_RHO) {
                return seterr(ctx, GC_ERR_UNSUPPORTED, "copier field %d not supported", fld);
            }
            cp.push_back({fld, mode});
        }
        g.copiers.push_back(cp);
    }
    (void)capacity;
    I.ghosts.push_back(g);
    HHandle h;
    h.type = H_GHOST;
    h.idx = (int)I.ghosts.size() - 1;
    I.handles.push_back(h);
    *handle_out = (int)I.handles.size() - 1;
    return GC_OK;
}

int gc_add_interaction(gc_ctx* ctx, int inst, int sys_a, int b_handle, int kernel_kind, double h, int nstages,
                       const int* pfn_kinds, const double* pfn_params, int* inter_out) {
    if (!ctx || !inter_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    int si = sys_of(ctx, inst, sys_a);
    int ag = -1;
    if (si < 0 && valid_inst(ctx, inst) && sys_a >= 0 && sys_a < (int)ctx->inst[inst].handles.size() &&
        ctx->inst[inst].handles[sys_a].type == H_GHOST) {
        ag = ctx->inst[inst].handles[sys_a].idx;
        si = ctx->inst[inst].ghosts[ag].src;
    }
    if (si < 0) return seterr(ctx, GC_ERR_ARG, "system_a must be a system handle");
    HInst& I = ctx->inst[inst];
    if (b_handle >= (int)I.handles.size()) return seterr(ctx, GC_ERR_ARG, "bad system_b handle");
    if (nstages < 1 || nstages > MAX_STAGES) return seterr(ctx, GC_ERR_ARG, "bad stage count");
    if (kernel_kind != GC_KERNEL_CUBIC_SPLINE && kernel_kind != GC_KERNEL_WENDLAND_C2)
        return seterr(ctx, GC_ERR_ARG, "bad kernel kind");
    HInter it;
    it.a = si;
    it.ag = ag;
    it.b = b_handle;
    it.kk = kernel_kind;
    it.H = h;
    it.nstages = nstages;
    for (int s = 0; s < nstages; ++s) {
        it.pk.push_back(pfn_kinds[s]);
        std::array<double, GC_PFN_NPARAM> a;
        for (int k = 0; k < GC_PFN_NPARAM; ++k) a[k] = pfn_params[s * GC_PFN_NPARAM + k];
        if ((pfn_kinds[s] == GC_PFN_FLUID || pfn_kinds[s] == GC_PFN_FLUID_SOLID) && !(a[3] == 1.0 || a[3] == 2.0))
            return seterr(ctx, GC_ERR_UNSUPPORTED, "FluidPfn/FluidSolidPfn sigma must be 1 or 2");
        it.pp.push_back(a);
        int st = check_combo(ctx, I, it, pfn_kinds[s]);
        if (st) return st;
    }
    I.inters.push_back(it);
    *inter_out = (int)I.inters.size() - 1;
    return GC_OK;
}

int gc_add_virtual(gc_ctx* ctx, int inst, int src_sys, int zero_mask, const double* prescribed_v,
                   int* handle_out) {
    if (!ctx || !handle_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    int si = sys_of(ctx, inst, src_sys);
    if (si < 0) return seterr(ctx, GC_ERR_ARG, "a virtual system needs a source system handle");
    HInst& I = ctx->inst[inst];
    const int allowed = (1 << GC_FIELD_V) | (1 << GC_FIELD_RHO) | (1 << GC_FIELD_P) | (1 << GC_FIELD_STRESS) |
                        (1 << GC_FIELD_DVDT) | (1 << GC_FIELD_DRHODT) | (1 << GC_FIELD_STRAIN_RATE);
    if (zero_mask & ~allowed) return seterr(ctx, GC_ERR_UNSUPPORTED, "zero_fields outside v, rho, p, stress, rates");
    HVirt v;
    v.src = si;
    v.zmask = zero_mask;
    if (prescribed_v)
        for (int d = 0; d < I.sys[si].nd; ++d) v.pv[d] = prescribed_v[d];
    I.sys[si].vsrc = true;
    I.virts.push_back(v);
    HHandle h;
    h.type = H_VIRT;
    h.idx = (int)I.virts.size() - 1;
    I.handles.push_back(h);
    *handle_out = (int)I.handles.size() - 1;
    return GC_OK;
}

int gc_add_probe(gc_ctx* ctx, int inst, int64_t n, int ndims, const double* positions, int mirror_sys,
                 int extras_mask, int ns, const double* prescribed_v, int* handle_out) {
    if (!ctx || !handle_out) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance");
    if (n <= 0) return seterr(ctx, GC_ERR_ARG, "positions must not be empty");
    if (ndims < 2 || ndims > 3) return seterr(ctx, GC_ERR_UNSUPPORTED, "ndims must be 2 or 3, got %d", ndims);
    HInst& I = ctx->inst[inst];
    int mi = -1;
    if (mirror_sys >= 0) {
        mi = sys_of(ctx, inst, mirror_sys);
        if (mi < 0 || I.sys[mi].n != n || I.sys[mi].nd != ndims)
            return seterr(ctx, GC_ERR_ARG, "mirror target must be a system of n particles");
    } else if (!positions) {
        return seterr(ctx, GC_ERR_ARG, "probe positions or a mirror target are required");
    }
    const int allowed = (1 << GC_FIELD_V) | (1 << GC_FIELD_RHO) | (1 << GC_FIELD_P) | (1 << GC_FIELD_STRESS) |
                        (1 << GC_FIELD_COUNT);
    if (extras_mask & ~allowed) return seterr(ctx, GC_ERR_UNSUPPORTED, "probe extras outside v, rho, p, stress, count");
    const bool st = extras_mask & (1 << GC_FIELD_STRESS);
    if (st && !(ns == 3 || ns == 4 || ns == 6)) return seterr(ctx, GC_ERR_ARG, "ns must be 3, 4, or 6");
    HSys s;
    s.kind = st ? GC_SYS_STRESS : (extras_mask & (1 << GC_FIELD_P)) ? GC_SYS_FLUID : GC_SYS_BASIC;
    s.nd = ndims;
    s.ns = st ? ns : 0;
    s.n = n;
    s.vsrc = true;
    s.probe = true;
    I.sys.push_back(s);
    HVirt v;
    v.src = (int)I.sys.size() - 1;
    v.probe = true;
    v.mirror = mi;
    if (prescribed_v)
        for (int d = 0; d < ndims; ++d) v.pv[d] = prescribed_v[d];
    I.virts.push_back(v);
    HHandle h;
    h.type = H_VIRT;
    h.idx = (int)I.virts.size() - 1;
    I.handles.push_back(h);
    *handle_out = (int)I.handles.size() - 1;
    if (positions)
        TRY(gc_stage_field(ctx, inst, *handle_out, GC_FIELD_X, positions, (size_t)(n * ndims * 8)));
    return GC_OK;
}

int gc_add_probe_interaction(gc_ctx* ctx, int inst, int sys_a, int probe, int kernel_kind, double h,
                             int pfn_kind, const double* pfn_params, int* inter_out) {
    if (!ctx || !inter_out || !pfn_params) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    int si = sys_of(ctx, inst, sys_a);
    if (si < 0) return seterr(ctx, GC_ERR_ARG, "system_a must be a system handle");
    HInst& I = ctx->inst[inst];
    if (probe < 0 || probe >= (int)I.handles.size() || I.handles[probe].type != H_VIRT ||
        !I.virts[I.handles[probe].idx].probe)
        return seterr(ctx, GC_ERR_ARG, "system_b must be a probe");
    if (pfn_kind != GC_PFN_INTERPOLATE && pfn_kind != GC_PFN_NEIGHBOR_COUNT)
        return seterr(ctx, GC_ERR_UNSUPPORTED, "probe interactions take InterpolateFieldFn or NeighborCountFn");
    if (kernel_kind != GC_KERNEL_CUBIC_SPLINE && kernel_kind != GC_KERNEL_WENDLAND_C2)
        return seterr(ctx, GC_ERR_ARG, "bad kernel kind");
    HInter it;
    it.a = si;
    it.b = probe;
    it.kk = kernel_kind;
    it.H = h;
    it.nstages = 1;
    it.probe = true;
    it.pk.push_back(pfn_kind);
    std::array<double, GC_PFN_NPARAM> a;
    for (int k = 0; k < GC_PFN_NPARAM; ++k) a[k] = pfn_params[k];
    it.pp.push_back(a);
    TRY(check_combo(ctx, I, it, pfn_kind));
    I.inters.push_back(it);
    *inter_out = (int)I.inters.size() - 1;
    return GC_OK;
}

// mirror_target positions into probe slots, x_p[id_src[i]] = x_src[i] (the
// probes are in id order between measurements)
__global__ void k_probe_mirror(double* __restrict__ xp, int64_t Np, const SysInst* __restrict__ pinst,
                               const double* __restrict__ xs, int64_t Ns, const int32_t* __restrict__ sid,
                               const int32_t* __restrict__ sinst_of, int nd) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < Ns; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = pinst[sinst_of[g]].base + sid[g] - 1;
        for (int d = 0; d < nd; ++d) xp[d * Np + t] = xs[d * Ns + g];
    }
}

// perm[base + id - 1] = position: the gather that puts a slot back in id order
__global__ void k_perm_by_id(const int32_t* __restrict__ id, const int32_t* __restrict__ inst_of,
                             const SysInst* __restrict__ inst, int64_t N, int32_t* __restrict__ perm) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x)
        perm[inst[inst_of[g]].base + id[g] - 1] = (int32_t)g;
}

// sort_particles! of one slot at measurement: its box, its plan, its sort
static int resort_slot(gc_ctx* ctx, int s) {
    DSlot& S = ctx->slots[s];
    TRY(bbox_slot(ctx, S));
    launch_sort_plan(S.d_inst, ninst(ctx), S.nd, ctx->d_need + s, ctx->d_err, ctx->stream);
    TRY(read_need(ctx));
    TRY(sort_particles_slot(ctx, &S, nullptr, ctx->h_need[s], ctx->d_need + s));
    S.xpk_static = false;
    S.xpk_epoch = -1;
    return check_launch(ctx, "measurement sort");
}

int gc_measure_probes(gc_ctx* ctx) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    if (!ctx->finalized) return seterr(ctx, GC_ERR_STATE, "call gc_finalize first");
    const unsigned nb = (unsigned)std::max(1, ctx->num_sms * 8);
    CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CU(cudaMemsetAsync(ctx->d_need, 0, sizeof(int64_t) * ctx->nneed, ctx->stream));
    // the probe interactions' system_a, re-sorted: positions moved since the step's sort
    std::vector<char> done(ctx->slots.size(), 0);
    for (auto& D : ctx->inters)
        if (D.probe && !done[D.a]) {
            done[D.a] = 1;
            TRY(resort_slot(ctx, D.a));
        }
    for (auto& V : ctx->virts) {
        if (!V.probe || V.mirror < 0) continue;
        DSlot& P = ctx->slots[V.src];
        DSlot& M = ctx->slots[V.mirror];
        k_probe_mirror<<<nb, 256, 0, ctx->stream>>>(P.F(F_X), P.N, P.d_inst, M.F(F_X), M.N, M.id[M.cur], M.inst_of,
                                                    P.nd);
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    for (auto& V : ctx->virts)
        if (V.probe) TRY(resort_slot(ctx, V.src));
    for (auto& D : ctx->inters) {
        if (!D.probe) continue;
        launch_grid_plan(grid_plan_args(ctx, D), ctx->stream);
        TRY(read_need(ctx));
        TRY(build_grid(ctx, D, ctx->h_need[D.need_slot]));
    }
    // auto_zero_probe! src/ProbeParticles.jl:117-124: w_sum and every extra
    for (auto& V : ctx->virts) {
        if (!V.probe) continue;
        DSlot& P = ctx->slots[V.src];
        CU(cudaMemsetAsync(V.wsum, 0, sizeof(double) * P.N, ctx->stream));
        for (int f : {F_V, F_RHO, F_P, F_STRESS, F_DRHODT})
            if (P.ncomp[f]) CU(cudaMemsetAsync(P.F(f), 0, sizeof(double) * P.ncomp[f] * P.N, ctx->stream));
    }
    for (size_t i = 0; i < ctx->inters.size(); ++i)
        if (ctx->inters[i].probe) TRY(interp_sweeps(ctx, ctx->inters[i].a, {(int)i}, 1));
    for (auto& V : ctx->virts)  // update_state!(probe): stage 1
        if (V.probe && V.nupd >= 1) TRY(run_virtual_updaters(ctx, V, 1));
    // _sort_probe_by_id! src/ProbeParticles.jl:129-143
    for (auto& V : ctx->virts) {
        if (!V.probe) continue;
        DSlot& P = ctx->slots[V.src];
        k_perm_by_id<<<nb, 256, 0, ctx->stream>>>(P.id[P.cur], P.inst_of, P.d_inst, P.N, ctx->perm);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        GatherArgs ga{};
        for (int f = 0; f < NF; ++f)
            if (P.ncomp[f]) {
                ga.src[ga.nf] = P.F(f);
                ga.dst[ga.nf] = P.A(f);
                ga.ncomp[ga.nf++] = P.ncomp[f];
            }
        ga.src[ga.nf] = V.wsum;
        ga.dst[ga.nf] = V.wsum_alt;
        ga.ncomp[ga.nf++] = 1;
        ga.isrc[0] = P.id[P.cur];
        ga.idst[0] = P.id[P.cur ^ 1];
        ga.ni = 1;
        launch_gather_fields(ga, P.N, ctx->perm, nullptr, ctx->stream);
        P.cur ^= 1;
        std::swap(V.wsum, V.wsum_alt);
    }
    TRY(check_launch(ctx, "probe measurement"));
    return finish_status(ctx);
}

int gc_set_velocity_adjust(gc_ctx* ctx, int inst, int inter, int kind, double epsilon) {
    if (!ctx) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance");
    HInst& I = ctx->inst[inst];
    if (inter < 0 || inter >= (int)I.inters.size()) return seterr(ctx, GC_ERR_ARG, "bad interaction");
    if (kind != GC_PFN_NONE && kind != GC_PFN_XSPH)
        return seterr(ctx, GC_ERR_UNSUPPORTED, "velocity-adjust functor kind %d has no device implementation", kind);
    if (kind != GC_PFN_NONE && I.inters[inter].ag >= 0)
        return seterr(ctx, GC_ERR_UNSUPPORTED, "no velocity-adjust functor on a ghost system_a");
    I.inters[inter].vk = kind;
    I.inters[inter].veps = epsilon;
    return GC_OK;
}

int gc_set_updaters(gc_ctx* ctx, int inst, int sys, int nstages, const int* chain_len, const int* kinds,
                    const double* params) {
    if (!ctx) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    if (valid_inst(ctx, inst) && sys >= 0 && sys < (int)ctx->inst[inst].handles.size() &&
        ctx->inst[inst].handles[sys].type == H_VIRT) {
        HVirt& vp = ctx->inst[inst].virts[ctx->inst[inst].handles[sys].idx];
        vp.upd.clear();
        vp.upd_set = true;
        int pos = 0;
        for (int st = 0; st < nstages; ++st) {
            if (chain_len[st] > GC_UPD_MAX_CHAIN) return seterr(ctx, GC_ERR_UNSUPPORTED, "updater chain too long");
            std::vector<HUpd> chain;
            for (int k = 0; k < chain_len[st]; ++k, ++pos) {
                HUpd u;
                u.kind = kinds[pos];
                for (int q = 0; q < GC_UPD_NPARAM; ++q) u.prm[q] = params[pos * GC_UPD_NPARAM + q];
                if (u.kind != GC_UPD_NONE && u.kind != GC_UPD_ZERO_FIELDS && u.kind != GC_UPD_VIRTUAL_NORM &&
                    u.kind != GC_UPD_PRESCRIBED_V)
                    return seterr(ctx, GC_ERR_UNSUPPORTED, "updater kind %d on a virtual system", u.kind);
                if (u.kind != GC_UPD_NONE) chain.push_back(u);
            }
            vp.upd.push_back(chain);
        }
        return GC_OK;
    }
    int si = sys_of(ctx, inst, sys);
    if (si < 0) return seterr(ctx, GC_ERR_ARG, "updaters need a system handle");
    HSys& s = ctx->inst[inst].sys[si];
    s.upd.clear();
    s.upd_set = true;
    int pos = 0;
    for (int st = 0; st < nstages; ++st) {
        if (chain_len[st] > GC_UPD_MAX_CHAIN) return seterr(ctx, GC_ERR_UNSUPPORTED, "updater chain too long");
        std::vector<HUpd> chain;
        for (int k = 0; k < chain_len[st]; ++k, ++pos) {
            HUpd u;
            u.kind = kinds[pos];
            for (int q = 0; q < GC_UPD_NPARAM; ++q) u.prm[q] = params[pos * GC_UPD_NPARAM + q];
            if ((u.kind == GC_UPD_ELASTOPLASTIC || u.kind == GC_UPD_HOOKE) &&
                !(s.kind == GC_SYS_ELASTOPLASTIC && s.ns == 4))
                return seterr(ctx, GC_ERR_ARG, "ElastoPlasticStressUpdater requires NS=4 (plane-strain Voigt)");
            if ((u.kind == GC_UPD_TAIT_EOS || u.kind == GC_UPD_LINEAR_EOS) && s.kind < GC_SYS_FLUID)
                return seterr(ctx, GC_ERR_ARG, "EOS updater needs a pressure field");
            if (u.kind == GC_UPD_VISCOPLASTIC_MC && (s.kind < GC_SYS_STRESS || (s.ns != 3 && s.ns != 4 && s.ns != 6)))
                return seterr(ctx, GC_ERR_ARG, "ViscoPlasticMCStressUpdater needs stress with NS = 3, 4 or 6");
            if (u.kind == GC_UPD_VIRTUAL_NORM || u.kind == GC_UPD_PRESCRIBED_V)
                return seterr(ctx, GC_ERR_ARG, "this updater acts on a virtual system");
            if (u.kind < GC_UPD_NONE || u.kind > GC_UPD_VISCOPLASTIC_MC) return seterr(ctx, GC_ERR_ARG, "bad updater kind");
            if (u.kind != GC_UPD_NONE) chain.push_back(u);
        }
        s.upd.push_back(chain);
    }
    return GC_OK;
}

int gc_set_integrator(gc_ctx* ctx, int inst, double damping_gamma) {
    if (!ctx) return GC_ERR_ARG;
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance");
    ctx->inst[inst].gamma = damping_gamma;
    return GC_OK;
}

int gc_set_integrator_kind(gc_ctx* ctx, int inst, int kind) {
    if (!ctx) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance");
    if (kind != GC_INTEGRATOR_LEAPFROG && kind != GC_INTEGRATOR_RK4)
        return seterr(ctx, GC_ERR_ARG, "unknown integrator kind %d", kind);
    ctx->inst[inst].integ = kind;
    return GC_OK;
}

int gc_finalize(gc_ctx* ctx) {
    if (!ctx) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized");
    cudaSetDevice(ctx->device);
    int st = finalize(ctx);
    if (st) return st;
    upload_inst_params(ctx, 0.0);
    for (auto& S : ctx->slots) TRY(push_slot_params(ctx, S));
    for (size_t k = 0; k < ctx->inst.size(); ++k) {
        std::vector<HStaged> staged;
        staged.swap(ctx->inst[k].staged);
        for (auto& f : staged)
            TRY(gc_upload_field(ctx, (int)k, f.handle, f.field, f.bytes.data(), f.bytes.size()));
    }
    return GC_OK;
}

int gc_stage_field(gc_ctx* ctx, int inst, int handle, int field, const void* host, size_t bytes) {
    if (!ctx || (!host && bytes)) return GC_ERR_ARG;
    if (ctx->finalized) return seterr(ctx, GC_ERR_STATE, "context already finalized: use gc_upload_field");
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance");
    HInst& I = ctx->inst[inst];
    if (handle < 0 || handle >= (int)I.handles.size() || I.handles[handle].type == H_GHOST ||
        (I.handles[handle].type == H_VIRT && !I.virts[I.handles[handle].idx].probe))
        return seterr(ctx, GC_ERR_ARG, "bad system handle");
    const HHandle& hh = I.handles[handle];
    const HSys& hs = I.sys[hh.type == H_VIRT ? I.virts[hh.idx].src : hh.idx];
    const int comps = sys_comps(hs, field);
    if (comps < 0 && field != GC_FIELD_V_ADJUSTMENT)
        return seterr(ctx, GC_ERR_ARG, "field %d not present on this system", field);
    const int width = field == GC_FIELD_V_ADJUSTMENT ? hs.nd : comps;
    if (bytes != (size_t)(hs.n * width * 8)) return seterr(ctx, GC_ERR_ARG, "byte count mismatch (%zu)", bytes);
    for (auto& f : I.staged)
        if (f.handle == handle && f.field == field) {
            f.bytes.assign((const char*)host, (const char*)host + bytes);
            return GC_OK;
        }
    I.staged.push_back({handle, field, std::vector<char>((const char*)host, (const char*)host + bytes)});
    return GC_OK;
}

// ---------------------------------------------------------------- state I/O
static int ensure_staging(gc_ctx* ctx, int64_t doubles) {
    if (doubles > ctx->cap_staging) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, ctx->staging, ctx->cap_staging);
        int64_t cap = std::max<int64_t>(doubles, 1 << 16);
        TRY(dalloc(ctx, &ctx->staging, (size_t)cap));
        ctx->cap_staging = cap;
    }
    return GC_OK;
}

static int ghost_field_io(gc_ctx* ctx, int inst, DGhost& G, int field, void* host, size_t bytes) {
    const GhostInst* hg = nullptr;
    std::vector<GhostInst> gh(ninst(ctx));
    TRY(hcopy(ctx, gh.data(), G.d_gh, gh.size() * sizeof(GhostInst), cudaMemcpyDeviceToHost));
    hg = &gh[inst];
    const int64_t n = hg->n, base = hg->base;
    auto get_planar = [&](const double* src, int ncomp, int64_t stride) -> int {
        if (bytes != (size_t)(n * ncomp * 8)) return seterr(ctx, GC_ERR_ARG, "byte count mismatch (%zu)", bytes);
        std::vector<double> tmp((size_t)ncomp * n);
        for (int c = 0; c < ncomp; ++c)
            if (n) TRY(hcopy(ctx, &tmp[(size_t)c * n], src + c * stride + base, n * 8, cudaMemcpyDeviceToHost));
        double* out = (double*)host;
        for (int64_t i = 0; i < n; ++i)
            for (int c = 0; c < ncomp; ++c) out[i * ncomp + c] = tmp[(size_t)c * n + i];
        return GC_OK;
    };
    auto get_i32 = [&](const int32_t* src) -> int {
        if (bytes != (size_t)(n * 8)) return seterr(ctx, GC_ERR_ARG, "byte count mismatch (%zu)", bytes);
        std::vector<int32_t> tmp(n);
        if (n) TRY(hcopy(ctx, tmp.data(), src + base, n * 4, cudaMemcpyDeviceToHost));
        int64_t* out = (int64_t*)host;
        for (int64_t i = 0; i < n; ++i) out[i] = tmp[i];
        return GC_OK;
    };
    switch (field) {
        case GC_FIELD_X: return get_planar(G.x[G.cur], G.nd, G.CAP);
        case GC_FIELD_V: return get_planar(G.v, G.nd, G.CAP);
        case GC_FIELD_RHO: return get_planar(G.rho, 1, G.CAP);
        case GC_FIELD_NORMALS: return get_planar(G.normals, G.nd, G.CAP);
        case GC_FIELD_P:
            if (!G.ex_p) return seterr(ctx, GC_ERR_ARG, "ghost has no p");
            return get_planar(G.p, 1, G.CAP);
        case GC_FIELD_STRESS:
            if (!G.ex_stress) return seterr(ctx, GC_ERR_ARG, "ghost has no stress");
            return get_planar(G.stress, G.ns, G.CAP);
        case GC_FIELD_IDX_ORIGINAL: return get_i32(G.io[G.cur]);
        case GC_FIELD_IDX_BOUNDARY: return get_i32(G.ib[G.cur]);
    }
    return seterr(ctx, GC_ERR_ARG, "field not present on ghosts");
}

struct HandleRef {
    DSlot* slot = nullptr;
    DGhost* ghost = nullptr;
    DVirt* virt = nullptr;
    int sys = -1;
};

static int resolve(gc_ctx* ctx, int inst, int handle, HandleRef* r) {
    if (!ctx->finalized) return seterr(ctx, GC_ERR_STATE, "call gc_finalize first");
    if (!valid_inst(ctx, inst)) return seterr(ctx, GC_ERR_ARG, "bad instance");
    HInst& I = ctx->inst[inst];
    if (handle < 0 || handle >= (int)I.handles.size()) return seterr(ctx, GC_ERR_ARG, "bad handle");
    const HHandle& h = I.handles[handle];
    if (h.type == H_GHOST) {
        r->ghost = &ctx->ghosts[h.idx];
    } else if (h.type == H_VIRT) {
        r->virt = &ctx->virts[h.idx];
        r->sys = ctx->virts[h.idx].src;
        if (r->virt->probe) r->slot = &ctx->slots[r->sys];  // a probe's fields are its own
    } else {
        r->slot = &ctx->slots[h.idx];
        r->sys = h.idx;
    }
    return GC_OK;
}

// Nonzero test of uploaded kinematics (and of v_adjustment, which must be
// zero) on the device: flag[k] = 1 when any of the n doubles is nonzero.
__global__ void k_any_nonzero(const double* __restrict__ a, int64_t n, int* flag) {
    pdl_enter();
    bool nz = false;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        nz |= a[i] != 0.0;
    if (__any_sync(0xffffffffu, nz) && (threadIdx.x & 31) == 0) *flag = 1;
}

static int ensure_ioflags(gc_ctx* ctx, int n) {
    if (n > ctx->cap_ioflags) {
        CU(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, ctx->d_ioflags, (size_t)ctx->cap_ioflags);
        const int cap = std::max(n, 64);
        TRY(dalloc(ctx, &ctx->d_ioflags, (size_t)cap));
        ctx->cap_ioflags = cap;
    }
    return GC_OK;
}

int gc_upload_fields(gc_ctx* ctx, int nio, const gc_field_io* io) {
    if (!ctx || nio < 0 || (nio && !io)) return GC_ERR_ARG;
    // validate everything first: nothing is written on a bad request
    std::vector<HandleRef> ref(nio);
    std::vector<int> comps(nio);
    int64_t total = 0;
    for (int q = 0; q < nio; ++q) {
        const gc_field_io& f = io[q];
        if (!f.host) return seterr(ctx, GC_ERR_ARG, "null host buffer");
        TRY(resolve(ctx, f.inst, f.handle, &ref[q]));
        if (ref[q].ghost) return seterr(ctx, GC_ERR_ARG, "ghost fields are generated on the device");
        if (ref[q].virt && !ref[q].slot) return seterr(ctx, GC_ERR_ARG, "a virtual system's fields are its source's");
        const HSys& hs = ctx->inst[f.inst].sys[ref[q].sys];
        comps[q] = sys_comps(hs, f.field);
        if (comps[q] < 0) return seterr(ctx, GC_ERR_ARG, "field %d not present on this system", f.field);
        if (f.bytes != (size_t)(hs.n * comps[q] * 8))
            return seterr(ctx, GC_ERR_ARG, "byte count mismatch (%zu)", f.bytes);
        total += hs.n * comps[q];
    }
    TRY(ensure_staging(ctx, std::max<int64_t>(total, 1)));
    TRY(ensure_ioflags(ctx, nio));
    CU(cudaMemsetAsync(ctx->d_ioflags, 0, sizeof(int) * std::max(nio, 1), ctx->stream));
    int64_t off = 0;
    for (int q = 0; q < nio; ++q) {
        const gc_field_io& f = io[q];
        DSlot& S = *ref[q].slot;
        const int64_t n = ctx->inst[f.inst].sys[ref[q].sys].n, base = S.h_inst[f.inst].base;
        double* st = ctx->staging + off;
        off += n * comps[q];
        if (n == 0) continue;
        CU(cudaMemcpyAsync(st, f.host, f.bytes, cudaMemcpyHostToDevice, ctx->stream));
        const bool check = f.field == GC_FIELD_V || f.field == GC_FIELD_DVDT || f.field == GC_FIELD_DRHODT ||
                           f.field == GC_FIELD_V_ADJUSTMENT;
        if (check) {
            k_any_nonzero<<<(unsigned)std::min<int64_t>((n * comps[q] + 255) / 256, 1024), 256, 0, ctx->stream>>>(
                st, n * comps[q], ctx->d_ioflags + q);
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
        if (f.field == GC_FIELD_V_ADJUSTMENT && !S.ncomp[F_VADJ]) continue;  // not carried: must be zero
        if (f.field == GC_FIELD_ID) launch_i64_to_i32((const int64_t*)st, S.id[S.cur] + base, n, ctx->stream);
        else launch_aos_to_planar(st, S.F(field_slot(f.field)), n, comps[q], S.N, base, ctx->stream);
    }
    std::vector<int> flags(std::max(nio, 1));
    CU(cudaMemcpyAsync(flags.data(), ctx->d_ioflags, sizeof(int) * std::max(nio, 1), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    TRY(check_launch(ctx, "upload"));
    bool structural = false;
    for (int q = 0; q < nio; ++q) {
        const gc_field_io& f = io[q];
        DSlot& S = *ref[q].slot;
        if (f.field == GC_FIELD_V_ADJUSTMENT && flags[q] && !S.ncomp[F_VADJ])
            return seterr(ctx, GC_ERR_UNSUPPORTED,
                          "non-zero v_adjustment needs a velocity-adjust functor (it is not carried without one)");
        if (f.field == GC_FIELD_X) {
            // a system that is not sorted every step is sorted again
            if (!S.moving) structural = true;
            S.sorted_once = false;
            S.xpk_static = false;
            S.xpk_epoch = -1;
        }
        if (f.field == GC_FIELD_V || f.field == GC_FIELD_DVDT || f.field == GC_FIELD_DRHODT ||
            f.field == GC_FIELD_V_ADJUSTMENT) {
            int64_t bit = f.field == GC_FIELD_V ? 1 : f.field == GC_FIELD_DVDT ? 2 : f.field == GC_FIELD_DRHODT ? 4 : 8;
            if (flags[q]) S.nonzero_kin[f.inst] |= bit;
            else S.nonzero_kin[f.inst] &= ~bit;
        }
    }
    for (auto& D : ctx->inters) D.grid_valid = false;
    if (structural) invalidate_steps(ctx);
    return GC_OK;
}

int gc_upload_field(gc_ctx* ctx, int inst, int handle, int field, const void* host, size_t bytes) {
    if (!ctx || !host) return GC_ERR_ARG;
    gc_field_io f{inst, handle, field, 0, const_cast<void*>(host), bytes};
    return gc_upload_fields(ctx, 1, &f);
}

int gc_download_fields(gc_ctx* ctx, int nio, const gc_field_io* io) {
    if (!ctx || nio < 0 || (nio && !io)) return GC_ERR_ARG;
    std::vector<HandleRef> ref(nio);
    std::vector<int> comps(nio);
    int64_t total = 0;
    for (int q = 0; q < nio; ++q) {
        const gc_field_io& f = io[q];
        if (!f.host) return seterr(ctx, GC_ERR_ARG, "null host buffer");
        TRY(resolve(ctx, f.inst, f.handle, &ref[q]));
        if (ref[q].ghost) continue;
        const HSys& hs = ctx->inst[f.inst].sys[ref[q].sys];
        if (ref[q].virt && (f.field == GC_FIELD_W_SUM || !ref[q].slot)) {
            // a virtual system holds only w_sum; its fields are its source's (a probe's are its own)
            if (f.field != GC_FIELD_W_SUM) return seterr(ctx, GC_ERR_ARG, "a virtual system's fields are its source's");
            if (f.bytes != (size_t)(hs.n * 8)) return seterr(ctx, GC_ERR_ARG, "byte count mismatch (%zu)", f.bytes);
            comps[q] = 1;
            total += hs.n;
            continue;
        }
        comps[q] = sys_comps(hs, f.field);
        if (comps[q] < 0) return seterr(ctx, GC_ERR_ARG, "field %d not present on this system", f.field);
        if (f.bytes != (size_t)(hs.n * comps[q] * 8))
            return seterr(ctx, GC_ERR_ARG, "byte count mismatch (%zu)", f.bytes);
        total += hs.n * comps[q];
    }
    TRY(ensure_staging(ctx, std::max<int64_t>(total, 1)));
    int64_t off = 0;
    for (int q = 0; q < nio; ++q) {
        const gc_field_io& f = io[q];
        if (ref[q].ghost) continue;
        DSlot& S = ref[q].virt ? ctx->slots[ref[q].virt->src] : *ref[q].slot;
        const int64_t n = ctx->inst[f.inst].sys[ref[q].sys].n, base = S.h_inst[f.inst].base;
        double* st = ctx->staging + off;
        off += n * comps[q];
        if (ref[q].virt && f.field == GC_FIELD_W_SUM) {
            if (n) CU(cudaMemcpyAsync(f.host, ref[q].virt->wsum + base, f.bytes, cudaMemcpyDeviceToHost, ctx->stream));
            continue;
        }
        if (f.field == GC_FIELD_V_ADJUSTMENT && !S.ncomp[F_VADJ]) {  // not carried: zero
            memset(f.host, 0, f.bytes);
            continue;
        }
        if (n == 0) continue;
        if (f.field == GC_FIELD_ID) launch_i32_to_i64(S.id[S.cur] + base, (int64_t*)st, n, ctx->stream);
        else launch_planar_to_aos(S.F(field_slot(f.field)), st, n, comps[q], S.N, base, ctx->stream);
        CU(cudaMemcpyAsync(f.host, st, f.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    TRY(check_launch(ctx, "download"));
    for (int q = 0; q < nio; ++q)
        if (ref[q].ghost) TRY(ghost_field_io(ctx, io[q].inst, *ref[q].ghost, io[q].field, io[q].host, io[q].bytes));
    return GC_OK;
}

int gc_download_field(gc_ctx* ctx, int inst, int handle, int field, void* host, size_t bytes) {
    if (!ctx || !host) return GC_ERR_ARG;
    gc_field_io f{inst, handle, field, 0, host, bytes};
    return gc_download_fields(ctx, 1, &f);
}

int gc_get_count(gc_ctx* ctx, int inst, int handle, int64_t* n_out) {
    if (!ctx || !n_out) return GC_ERR_ARG;
    HandleRef r;
    TRY(resolve(ctx, inst, handle, &r));
    if (r.ghost) {
        std::vector<GhostInst> gh(ninst(ctx));
        CU(cudaStreamSynchronize(ctx->stream));
        TRY(hcopy(ctx, gh.data(), r.ghost->d_gh, gh.size() * sizeof(GhostInst), cudaMemcpyDeviceToHost));
        *n_out = gh[inst].n;
    } else {
        *n_out = ctx->inst[inst].sys[r.sys].n;  // a virtual system: its source's count
    }
    return GC_OK;
}

int gc_set_precision(gc_ctx* ctx, int mode) {
    if (!ctx) return GC_ERR_ARG;
    if (mode != GC_PRECISION_FP64 && mode != GC_PRECISION_FP32_COMPENSATED)
        return seterr(ctx, GC_ERR_ARG, "bad precision mode");
    ctx->precision = mode;
    return GC_OK;
}

int gc_step(gc_ctx* ctx, int nsteps, double cfl) {
    if (!ctx) return GC_ERR_ARG;
    if (!ctx->finalized) return seterr(ctx, GC_ERR_STATE, "call gc_finalize first");
    if (nsteps < 0) return seterr(ctx, GC_ERR_ARG, "negative step count");
    cudaSetDevice(ctx->device);
    // per-instance step parameters change only with the CFL number (or when
    // a phase hook or the serving loop has edited them)
    if (ctx->params_dirty || !(cfl == ctx->params_cfl)) {
        upload_inst_params(ctx, cfl);
        for (auto& S : ctx->slots) TRY(push_slot_params(ctx, S));
        ctx->params_cfl = cfl;
        ctx->params_dirty = false;
    }
    if (decide_motion(ctx)) invalidate_steps(ctx);
    CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    TRY(run_steps(ctx, nsteps));
    return finish_status(ctx);
}

int gc_get_stats(gc_ctx* ctx, gc_stats* out) {
    if (!ctx || !out) return GC_ERR_ARG;
    memset(out, 0, sizeof *out);
    out->steps_done = ctx->steps_done;
    out->last_status = ctx->last_status;
    out->kernel_launches = (int64_t)g_launches.load();
    out->sweep_launches = ctx->sweep_launches;
    out->sweep_ms = ctx->sweep_ms;
    out->graph_steps = ctx->graph_steps;
    out->rollbacks = ctx->rollbacks;
    for (auto& kv : ctx->tune)
        if (kv.second.best >= 0 && kv.second.best < 4) out->sweep_cfg_chosen[kv.second.best] += 1;
    if (ctx->finalized && ctx->steps_done > 0) {
        if (!ctx->d_pairs) TRY(dalloc(ctx, &ctx->d_pairs, 1));
        int64_t pairs = 0;
        for (auto& D : ctx->inters) {
            if (D.probe) continue;
            // InterpolateFieldFn stages gather on the system_b side and count nothing
            bool active = false;
            for (int p : D.pk) active |= p != GC_PFN_NONE && p != GC_PFN_INTERPOLATE && p != GC_PFN_NEIGHBOR_COUNT;
            if (!active) continue;
            CU(cudaMemsetAsync(ctx->d_pairs, 0, 8, ctx->stream));
            launch_sum_counts(D.counts, ctx->slots[D.a].N, ctx->d_pairs, ctx->stream);
            unsigned long long v = 0;
            CU(cudaMemcpyAsync(&v, ctx->d_pairs, 8, cudaMemcpyDeviceToHost, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            pairs += D.btype == BT_SELF ? (int64_t)(v / 2) : (int64_t)v;
        }
        out->pairs_last_step = pairs;
    }
    if (ctx->d_incons) {
        unsigned long long v = 0;
        TRY(hcopy(ctx, &v, ctx->d_incons, sizeof v, cudaMemcpyDeviceToHost));
        out->grid_inconsistent = (int64_t)v;
    }
    if (ctx->d_sorts_in_order) {
        unsigned long long v = 0;
        TRY(hcopy(ctx, &v, ctx->d_sorts_in_order, sizeof v, cudaMemcpyDeviceToHost));
        out->sorts_in_order = (int64_t)v;
    }
    return GC_OK;
}

// ------------------------------------------------------------- phase hooks
int gc_sort_system(gc_ctx* ctx, int inst, int handle, double cutoff, int64_t* perm_out) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    HandleRef r;
    TRY(resolve(ctx, inst, handle, &r));
    const int ni = ninst(ctx);
    CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CU(cudaMemsetAsync(ctx->d_need, 0, sizeof(int64_t) * ctx->nneed, ctx->stream));
    if (r.ghost) {
        DGhost& G = *r.ghost;
        std::vector<SysInst> gi(ni);
        TRY(hcopy(ctx, gi.data(), G.d_inst, ni * sizeof(SysInst), cudaMemcpyDeviceToHost));
        for (auto& g : gi) g.sort_cutoff = cutoff;
        TRY(hcopy(ctx, G.d_inst, gi.data(), ni * sizeof(SysInst), cudaMemcpyHostToDevice));
        TRY(ghost_bbox_and_plan(ctx, G));
        TRY(read_need(ctx));
        TRY(sort_particles_slot(ctx, nullptr, &G, ctx->h_need[G.need_slot], ctx->d_need + G.need_slot));
        TRY(finish_status(ctx));  // host reads below must follow the stream's kernels
        if (perm_out) {
            TRY(hcopy(ctx, gi.data(), G.d_inst, ni * sizeof(SysInst), cudaMemcpyDeviceToHost));
            const int64_t n = gi[inst].n, base = gi[inst].base;
            std::vector<int32_t> p(n);
            if (n) TRY(hcopy(ctx, p.data(), ctx->perm + base, n * 4, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < n; ++i) perm_out[i] = p[i] - base + 1;
        }
        return finish_status(ctx);
    }
    DSlot& S = *r.slot;
    for (auto& h : S.h_inst) h.sort_cutoff = cutoff;
    ctx->params_dirty = true;  // the next gc_step restores its own cutoff
    TRY(push_slot_params(ctx, S));
    TRY(bbox_slot(ctx, S));
    launch_sort_plan(S.d_inst, ni, S.nd, ctx->d_need + r.sys, ctx->d_err, ctx->stream);
    TRY(read_need(ctx));
    TRY(sort_particles_slot(ctx, &S, nullptr, ctx->h_need[r.sys], ctx->d_need + r.sys));
    TRY(finish_status(ctx));  // host reads below must follow the stream's kernels
    if (perm_out) {
        const int64_t n = S.h_inst[inst].n, base = S.h_inst[inst].base;
        std::vector<int32_t> p(n);
        TRY(hcopy(ctx, p.data(), ctx->perm + base, n * 4, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i) perm_out[i] = p[i] - base + 1;
    }
    for (auto& D : ctx->inters) D.grid_valid = false;
    return finish_status(ctx);
}

int gc_build_grid(gc_ctx* ctx, int inst, int inter, int64_t* cell_start_out, int64_t cap, double* mingridx_out,
                  int64_t* ngridx_out, int64_t* ncells_out) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    if (!ctx->finalized) return seterr(ctx, GC_ERR_STATE, "call gc_finalize first");
    if (!valid_inst(ctx, inst) || inter < 0 || inter >= (int)ctx->inters.size())
        return seterr(ctx, GC_ERR_ARG, "bad interaction");
    DInter& D = ctx->inters[inter];
    CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CU(cudaMemsetAsync(ctx->d_need, 0, sizeof(int64_t) * ctx->nneed, ctx->stream));
    if (D.ag >= 0) {
        DGhost& G = ctx->ghosts[D.ag];
        launch_bbox_fused(G.x[G.cur], G.CAP, G.nd, G.ginst[G.cur], G.d_count, G.d_inst, ctx->bbox_scratch, ninst(ctx),
                          ctx->d_err, ctx->stream);
    } else {
        TRY(bbox_slot(ctx, ctx->slots[D.a]));
    }
    if (D.btype == BT_GHOST) {
        DGhost& G = ctx->ghosts[D.bghost];
        launch_bbox_fused(G.x[G.cur], G.CAP, G.nd, G.ginst[G.cur], G.d_count, G.d_inst, ctx->bbox_scratch, ninst(ctx),
                    ctx->d_err, ctx->stream);
    } else if (D.btype != BT_SELF) {
        TRY(bbox_slot(ctx, ctx->slots[D.bslot]));
    }
    launch_grid_plan(grid_plan_args(ctx, D), ctx->stream);
    TRY(read_need(ctx));
    TRY(build_grid(ctx, D, ctx->h_need[D.need_slot]));
    TRY(finish_status(ctx));
    std::vector<GridInst> gi(ninst(ctx));
    TRY(hcopy(ctx, gi.data(), D.d_gi, gi.size() * sizeof(GridInst), cudaMemcpyDeviceToHost));
    const GridInst& G = gi[inst];
    const int nd = ctx->slots[D.a].nd;
    if (ncells_out) *ncells_out = G.ncells;
    if (mingridx_out)
        for (int d = 0; d < nd; ++d) mingridx_out[d] = G.ming[d];
    if (ngridx_out)
        for (int d = 0; d < nd; ++d) ngridx_out[d] = G.ng[d];
    if (cell_start_out) {
        if (cap < G.ncells + 1) return seterr(ctx, GC_ERR_CAPACITY, "cell_start buffer too small");
        std::vector<int32_t> cs(G.ncells + 1);
        TRY(hcopy(ctx, cs.data(), D.cs + G.cellbase, cs.size() * 4, cudaMemcpyDeviceToHost));
        int64_t bbase;
        if (D.btype == BT_GHOST) {
            std::vector<GhostInst> gh(ninst(ctx));
            TRY(hcopy(ctx, gh.data(), ctx->ghosts[D.bghost].d_gh, gh.size() * sizeof(GhostInst), cudaMemcpyDeviceToHost));
            bbase = gh[inst].base;
        } else {
            bbase = ctx->slots[D.bslot].h_inst[inst].base;
        }
        for (int64_t c = 0; c <= G.ncells; ++c) cell_start_out[c] = cs[c] - bbase + 1;
    }
    return GC_OK;
}

int gc_generate_ghosts(gc_ctx* ctx, int inst, int ghost) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    HandleRef r;
    TRY(resolve(ctx, inst, ghost, &r));
    if (!r.ghost) return seterr(ctx, GC_ERR_ARG, "not a ghost handle");
    CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    TRY(generate_ghosts(ctx, *r.ghost));
    for (auto& D : ctx->inters) D.grid_valid = false;
    return finish_status(ctx);
}

int gc_update_ghost_kinematics(gc_ctx* ctx, int inst, int ghost) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    HandleRef r;
    TRY(resolve(ctx, inst, ghost, &r));
    if (!r.ghost) return seterr(ctx, GC_ERR_ARG, "not a ghost handle");
    TRY(ghost_kinematics(ctx, *r.ghost));
    return finish_status(ctx);
}

int gc_update_ghost(gc_ctx* ctx, int inst, int ghost, int stage) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    HandleRef r;
    TRY(resolve(ctx, inst, ghost, &r));
    if (!r.ghost) return seterr(ctx, GC_ERR_ARG, "not a ghost handle");
    TRY(ghost_copy(ctx, *r.ghost, stage));
    return finish_status(ctx);
}

int gc_sweep(gc_ctx* ctx, int inst, int inter, int stage) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    if (!ctx->finalized) return seterr(ctx, GC_ERR_STATE, "call gc_finalize first");
    if (!valid_inst(ctx, inst) || inter < 0 || inter >= (int)ctx->inters.size())
        return seterr(ctx, GC_ERR_ARG, "bad interaction");
    DInter& D = ctx->inters[inter];
    if (stage < 1 || stage > D.nstages || D.pk[stage - 1] == GC_PFN_NONE) return GC_OK;
    CU(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    TRY(sweep_group(ctx, D.a, std::vector<int>{inter}, stage, false));
    return finish_status(ctx);
}

int gc_update_state(gc_ctx* ctx, int inst, int sys, int stage, double dt) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx) return GC_ERR_ARG;
    HandleRef r;
    TRY(resolve(ctx, inst, sys, &r));
    if (r.virt) {
        TRY(run_virtual_updaters(ctx, *r.virt, stage));
        return finish_status(ctx);
    }
    if (!r.slot) return seterr(ctx, GC_ERR_ARG, "not a system handle");
    TRY(run_updaters(ctx, *r.slot, stage, dt));
    return finish_status(ctx);
}

int gc_neighbor_counts(gc_ctx* ctx, int inst, int inter, int32_t* counts_out, int64_t n) {
    if (ctx) invalidate_steps(ctx);
    if (!ctx || !counts_out) return GC_ERR_ARG;
    if (!ctx->finalized) return seterr(ctx, GC_ERR_STATE, "call gc_finalize first");
    if (!valid_inst(ctx, inst) || inter < 0 || inter >= (int)ctx->inters.size())
        return seterr(ctx, GC_ERR_ARG, "bad interaction");
    DInter& D = ctx->inters[inter];
    DSlot& S = ctx->slots[D.a];
    if (D.ag >= 0) return seterr(ctx, GC_ERR_UNSUPPORTED, "neighbour counts of a ghost system_a");
    if (n != S.h_inst[inst].n) return seterr(ctx, GC_ERR_ARG, "count buffer length mismatch");
    // A counting sweep: the first non-`nothing` stage's functor kind decides
    // the launch; counts do not depend on it.
    int stage = 1;
    for (int s = 1; s <= D.nstages; ++s)
        if (D.pk[s - 1] != GC_PFN_NONE) {
            stage = s;
            break;
        }
    std::vector<int> ids{inter};
    std::vector<int> saved = D.pk;
    for (auto& p : D.pk) p = GC_PFN_COUNT;
    int st = sweep_group(ctx, D.a, ids, stage, true);
    D.pk = saved;
    TRY(st);
    TRY(finish_status(ctx));
    TRY(hcopy(ctx, counts_out, D.counts + S.h_inst[inst].base, n * 4, cudaMemcpyDeviceToHost));
    return GC_OK;
}

int gc_stream(gc_ctx* ctx, void** stream_out) {
    if (!ctx || !stream_out) return GC_ERR_ARG;
    *stream_out = (void*)ctx->stream;
    return GC_OK;
}

int gc_set_profiling(gc_ctx* ctx, int on) {
    if (!ctx) return GC_ERR_ARG;
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->ev_used = 0;
    ctx->profiling = on != 0;
    ctx->sweep_ms = 0;
    ctx->sweep_launches = 0;
    return GC_OK;
}

int gc_set_sweep_config(gc_ctx* ctx, int cfg) {
    if (!ctx) return GC_ERR_ARG;
    if (cfg < -1 || cfg >= NUM_FORCE_CFG) return seterr(ctx, GC_ERR_ARG, "sweep configuration out of range");
    ctx->force_cfg = cfg;
    invalidate_steps(ctx);
    return GC_OK;
}

int gc_set_graphs(gc_ctx* ctx, int on, int sync_every, double cap_margin) {
    if (!ctx) return GC_ERR_ARG;
    if (sync_every < 1) return seterr(ctx, GC_ERR_ARG, "sync_every must be at least 1");
    if (cap_margin != 0.0 && !(cap_margin >= 1.0 && cap_margin <= 16.0))
        return seterr(ctx, GC_ERR_ARG, "cap_margin must be 0 or in [1, 16]");
    ctx->graphs_on = on != 0;
    ctx->sync_every = sync_every;
    if (cap_margin != 0.0) ctx->cap_margin = cap_margin;
    invalidate_steps(ctx);
    return GC_OK;
}

int gc_measure_fp64_peak(gc_ctx* ctx, double* tflops_out) {
    if (!ctx || !tflops_out) return GC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    double* out = nullptr;
    TRY(dalloc(ctx, &out, 1));
    const int threads = 256, blocks = sms * 8, iters = 1 << 16;
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    launch_fp64_peak(out, blocks, threads, 1024, ctx->stream);  // warm-up
    CU(cudaEventRecord(a, ctx->stream));
    launch_fp64_peak(out, blocks, threads, iters, ctx->stream);
    CU(cudaEventRecord(b, ctx->stream));
    CU(cudaEventSynchronize(b));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    dfree(ctx, out, 1);
    double flops = 2.0 * 8.0 * (double)iters * threads * blocks;
    *tflops_out = flops / (ms * 1e-3) / 1e12;
    return GC_OK;
}

int gc_measure_fp32_peak(gc_ctx* ctx, double* tflops_out) {
    if (!ctx || !tflops_out) return GC_ERR_ARG;
    cudaSetDevice(ctx->device);
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    float* out = nullptr;
    TRY(dalloc(ctx, &out, 1));
    const int threads = 256, blocks = sms * 8, iters = 1 << 17;
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    launch_fp32_peak(out, blocks, threads, 1024, ctx->stream);  // warm-up
    CU(cudaEventRecord(a, ctx->stream));
    launch_fp32_peak(out, blocks, threads, iters, ctx->stream);
    CU(cudaEventRecord(b, ctx->stream));
    CU(cudaEventSynchronize(b));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    dfree(ctx, out, 1);
    double flops = 2.0 * 8.0 * (double)iters * threads * blocks;
    *tflops_out = flops / (ms * 1e-3) / 1e12;
    return GC_OK;
}

}  // extern "C"

// ============================================================ packing
// Runtime support of the serving loop (gc_serve.cu): contexts are rebuilt
// with a new set of instances, each copied from a running context (device
// state) or from a model context (staged host fields).
namespace gc {

struct PackSeg {
    const void* src;
    int64_t src_stride, src_base, dst_base, n;
};

template <class T>
__global__ void k_pack(const PackSeg* __restrict__ seg, int ncomp, T* __restrict__ dst, int64_t dst_stride) {
    pdl_enter();
    const PackSeg S = seg[blockIdx.y];
    const T* src = (const T*)S.src;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < ncomp; ++c) dst[c * dst_stride + S.dst_base + i] = src[c * S.src_stride + S.src_base + i];
}

bool ctx_same_structure(gc_ctx* a, int ia, gc_ctx* b, int ib) {
    std::string why;
    return same_structure(a->inst[ia], b->inst[ib], why);
}

bool ctx_finalized(gc_ctx* c) { return c->finalized; }

// Move a context to a new stream of the given priority (highest: true),
// once its queued work is done.  Blocks of a higher-priority stream are
// dispatched before pending blocks of others, so a context being built while
// other contexts step does not wait behind their kernels at every sync.
int ctx_set_priority(gc_ctx* ctx, bool highest) {
    gc_ctx* c = ctx;
    int least = 0, greatest = 0;
    CU(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    cudaStream_t ns = nullptr;
    CU(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, highest ? greatest : least));
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
    c->stream = ns;
    return GC_OK;
}
int ctx_ninst(gc_ctx* c) { return (int)c->inst.size(); }

int ctx_set_cfl(gc_ctx* c, int inst, double cfl) {
    if (!valid_inst(c, inst)) return GC_ERR_ARG;
    c->inst[inst].cfl = cfl;
    c->params_dirty = true;
    return GC_OK;
}

int64_t ctx_particles(gc_ctx* c, int inst) {
    int64_t n = 0;
    for (auto& s : c->inst[inst].sys) n += s.n;
    return n;
}

// Particles whose positions move (the serving throughput counts these).
int64_t ctx_moving_particles(gc_ctx* c, int inst) {
    const HInst& I = c->inst[inst];
    std::vector<char> w(I.sys.size(), 0);
    for (auto& it : I.inters)
        for (int p : it.pk)
            if (p != GC_PFN_NONE) w[it.a] = 1;
    int64_t n = 0;
    for (size_t s = 0; s < I.sys.size(); ++s)
        if (w[s]) n += I.sys[s].n;
    return n;
}

// Device bytes one instance of `m` needs in a packed context: its carried
// fields (two buffers and the rollback snapshot), step temporaries, ghost
// capacity and the grids over the staged positions' box (doubled for
// runout), with a quarter on top.
int64_t ctx_estimate_bytes(gc_ctx* m, int inst) {
    const HInst& I = m->inst[inst];
    int64_t b = 0;
    for (auto& s : I.sys) {
        int comps = 0;
        for (int f = 0; f < GC_NFIELDS; ++f) {
            if (f == GC_FIELD_ID || f == GC_FIELD_V_ADJUSTMENT) continue;
            const int c = sys_comps(s, f);
            if (c > 0) comps += c;
        }
        b += s.n * (comps * 8 * 3 + (s.nd + 2) * 8 + 4 * 4 + 8 + 4 * (s.nd + 3 + s.ns) + 8 + 4 * 4);
    }
    for (auto& g : I.ghosts) {
        const HSys& src = I.sys[g.src];
        const int64_t cap = src.n * g.nplanes;
        b += cap * (src.nd * 8 * 4 + 4 * 8 + 8 * 3 + src.ns * 8 + 4 * (src.nd + 3 + src.ns));
    }
    // grid cells from the staged positions' bounding box
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    int nd = I.sys.empty() ? 2 : I.sys[0].nd;
    bool any = false;
    for (auto& f : I.staged) {
        if (f.field != GC_FIELD_X) continue;
        const double* x = (const double*)f.bytes.data();
        const int64_t n = (int64_t)f.bytes.size() / 8 / nd;
        for (int64_t i = 0; i < n; ++i)
            for (int d = 0; d < nd; ++d) {
                lo[d] = std::min(lo[d], x[i * nd + d]);
                hi[d] = std::max(hi[d], x[i * nd + d]);
                any = true;
            }
    }
    double hmin = 1e300;
    for (auto& it : I.inters) hmin = std::min(hmin, it.H);
    if (any && hmin < 1e300) {
        double cells = 1;
        for (int d = 0; d < nd; ++d) cells *= (hi[d] - lo[d]) / (2.0 * hmin) * 2.0 + 8.0;
        b += (int64_t)(cells * (double)I.inters.size() * 4 * 2 * 1.5) + (int64_t)(cells * 4 * 3 * 1.5);
    }
    return b + b / 4;
}

// An instance's model without its staged field bytes (they can be hundreds
// of MB of host memory and are read from the source where needed).
HInst model_of(HInst& from) {
    std::vector<HStaged> keep;
    keep.swap(from.staged);
    HInst out = from;
    from.staged.swap(keep);
    return out;
}

// A context with no device state holding one instance's model (no staged
// fields): the structure a batch of the serving loop is keyed by.
int ctx_model_copy(gc_ctx* m, int inst, gc_ctx** out) {
    gc_ctx* c = nullptr;
    TRY(gc_ctx_create(m->device, 0, &c));
    c->inst.push_back(model_of(m->inst[inst]));
    *out = c;
    return GC_OK;
}

// A repack in two parts.  ctx_pack_plan (on the caller's thread) copies what
// the new context needs from the sources: every instance's model, the
// sources of their state, and the sweep configurations a running context
// of this structure tuned.  ctx_pack_build then makes and finalizes the new
// context and uploads the staged fields of instances that come from model
// contexts; it reads only the plan and those models, so it may run while
// the running sources step.  ctx_pack_fill copies the running instances'
// device state once their sources have stopped.
struct PackJob {
    int precision = GC_PRECISION_FP64;
    std::vector<HInst> models;
    std::vector<std::pair<gc_ctx*, int>> src;  // per new instance: its source and instance there
    std::map<int64_t, gc_ctx::Tune> tune;
};

PackJob* ctx_pack_plan(int precision, const std::vector<std::pair<gc_ctx*, int>>& src) {
    PackJob* J = new PackJob;
    J->precision = precision;
    J->src = src;
    for (auto& p : src) J->models.push_back(model_of(p.first->inst[p.second]));
    // the sweep configurations a running context of this structure tuned
    // carry over (the structure, and so the tuner's keys, are the same)
    for (auto& p : src)
        if (p.first->finalized && p.first->precision == precision && p.first->force_cfg < 0) {
            for (auto& kv : p.first->tune)
                if (kv.second.best >= 0) J->tune[kv.first] = kv.second;
            break;
        }
    return J;
}

void ctx_pack_free(PackJob* J) { delete J; }

int ctx_pack_build(PackJob* J, int device, cudaMemPool_t pool, gc_ctx** out, std::string* err) {
    *out = nullptr;
    gc_ctx* ctx = nullptr;
    TRY(gc_ctx_create(device, 0, &ctx));
    ctx->pool = pool;
    if (pool) TRY(ctx_set_priority(ctx, true));
    auto fail = [&](int st) {
        if (err) *err = ctx->err;
        gc_ctx_destroy(ctx);
        return st;
    };
    ctx->inst = J->models;
    int st = gc_finalize(ctx);
    if (st) return fail(st);
    st = gc_set_precision(ctx, J->precision);
    if (st) return fail(st);
    for (auto& kv : J->tune) ctx->tune[kv.first] = kv.second;
    // instances that come from model contexts: their staged fields
    for (size_t k = 0; k < J->src.size(); ++k) {
        gc_ctx* sc = J->src[k].first;
        if (sc->finalized) continue;
        for (auto& f : sc->inst[J->src[k].second].staged) {
            st = gc_upload_field(ctx, (int)k, f.handle, f.field, f.bytes.data(), f.bytes.size());
            if (st) return fail(st);
        }
    }
    CU(cudaStreamSynchronize(ctx->stream));
    *out = ctx;
    return GC_OK;
}

int ctx_pack_fill(PackJob* J, gc_ctx* ctx, std::string* err) {
    auto fail = [&](int st) {
        if (err) *err = ctx->err;
        return st;
    };
    const auto& src = J->src;
    for (auto& p : src)
        if (p.first->finalized) cudaStreamSynchronize(p.first->stream);
    // every (slot, field) segment table in one upload, then the copies
    std::vector<PackSeg> tab;
    struct Launch {
        size_t off, n;
        int64_t nmax;
        int slot, field;
    };
    std::vector<Launch> launches;
    for (size_t s = 0; s < ctx->slots.size(); ++s) {
        DSlot& D = ctx->slots[s];
        for (int f = -1; f < NF; ++f) {  // -1: ids
            if (f >= 0 && !D.ncomp[f]) continue;
            const size_t off = tab.size();
            int64_t nmax = 0;
            for (size_t k = 0; k < src.size(); ++k) {
                gc_ctx* sc = src[k].first;
                if (!sc->finalized) continue;
                DSlot& S = sc->slots[s];
                const int si = src[k].second;
                PackSeg g;
                g.src = f < 0 ? (const void*)S.id[S.cur] : (const void*)S.F(f);
                g.src_stride = S.N;
                g.src_base = S.h_inst[si].base;
                g.dst_base = D.h_inst[k].base;
                g.n = S.h_inst[si].n;
                nmax = std::max(nmax, g.n);
                tab.push_back(g);
            }
            if (tab.size() == off || nmax == 0) {
                tab.resize(off);
                continue;
            }
            launches.push_back({off, tab.size() - off, nmax, (int)s, f});
        }
        for (size_t k = 0; k < src.size(); ++k)
            if (src[k].first->finalized) D.nonzero_kin[k] = src[k].first->slots[s].nonzero_kin[src[k].second];
    }
    if (!tab.empty()) {
        PackSeg* d_seg = nullptr;
        if (dalloc(ctx, &d_seg, tab.size()) != GC_OK) return fail(GC_ERR_OOM);
        if (cudaMemcpyAsync(d_seg, tab.data(), sizeof(PackSeg) * tab.size(), cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess) {
            dfree(ctx, d_seg, tab.size());
            return fail(seterr(ctx, GC_ERR_CUDA, "pack table upload"));
        }
        for (const Launch& L : launches) {
            DSlot& D = ctx->slots[L.slot];
            dim3 grid((unsigned)std::min<int64_t>((L.nmax + 255) / 256, 64), (unsigned)L.n);
            if (L.field < 0) k_pack<int32_t><<<grid, 256, 0, ctx->stream>>>(d_seg + L.off, 1, D.id[D.cur], D.N);
            else k_pack<double><<<grid, 256, 0, ctx->stream>>>(d_seg + L.off, D.ncomp[L.field], D.F(L.field), D.N);
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
        // the host table lives until the copy has run
        cudaStreamSynchronize(ctx->stream);
        dfree(ctx, d_seg, tab.size());
    }
    int st = check_launch(ctx, "pack");
    if (st) return fail(st);
    CU(cudaStreamSynchronize(ctx->stream));
    return GC_OK;
}

// (handle, field, bytes) of every result field of one instance's systems.
void ctx_result_fields(gc_ctx* c, int inst, std::vector<std::array<int64_t, 3>>& out) {
    out.clear();
    const HInst& I = c->inst[inst];
    for (size_t h = 0; h < I.handles.size(); ++h) {
        if (I.handles[h].type != H_SYS) continue;
        const HSys& s = I.sys[I.handles[h].idx];
        for (int f = 0; f < GC_NFIELDS; ++f) {
            const int comps = sys_comps(s, f);
            if (comps <= 0) continue;
            out.push_back({(int64_t)h, (int64_t)f, s.n * comps * 8});
        }
    }
}

const char* ctx_error(gc_ctx* c) { return c->err.c_str(); }

}  // namespace gc
