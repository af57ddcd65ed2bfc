// gc_kernels.h — host-callable launchers of the device kernels.
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "gc_internal.h"

namespace gc {

// ---------------------------------------------------------------- scan
// Exclusive prefix sum of n int32 counts into out[0..n] (out[n] = total).
// `tmp` must hold scan_tmp_elems(n) int32.
int64_t scan_tmp_elems(int64_t n);
// clear_in: the last pass also zeroes in[0..n) (histograms left ready for
// their next use, no separate memset).
void scan_exclusive(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t s);
// skip: optional device flag; when set, the launches return at once.
void scan_exclusive_clear(int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t s,
                          const int* skip = nullptr);

// ---------------------------------------------------------- bounding box
// Per-instance min/max of a slot's positions into inst[k].bbmin/bbmax.
// `count` (nullable) bounds the packed range for ghost slots.
void launch_bbox(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count, SysInst* inst,
                 unsigned long long* scratch, int ninst, int* err, cudaStream_t s);
// One launch; `scratch` (ninst·2·MAXD + 1 words) must have been reset once
// with launch_bbox_reset and is left reset.
void launch_bbox_reset(unsigned long long* scratch, int ninst, cudaStream_t s);
void launch_bbox_fused(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count,
                       SysInst* inst, unsigned long long* scratch, int ninst, int* err, cudaStream_t s);

// ------------------------------------------------------------------ sort
// Per-instance key lattice from the bbox; writes total cells to *need.
void launch_sort_plan(SysInst* inst, int ninst, int nd, int64_t* need, int* err, cudaStream_t s);
// Flat sort key per particle + histogram.
// `unsorted` (optional): a device flag, zero on entry, that the keys
// kernel sets when the keys are not already non-decreasing; given to the
// scatter and the clearing fix-up, a flag left zero makes the sort the
// identity without the fill counters (src/Sorting.jl:176-186).  The gather
// that follows clears it (GatherArgs::clear).
void launch_sort_keys(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count,
                      const SysInst* inst, int32_t* key, int32_t* hist, int64_t cells_cap, int* err, cudaStream_t s,
                      int* unsorted = nullptr);
void launch_sort_scatter(const int32_t* key, int64_t N, const int64_t* count, const int32_t* start, int32_t* fill,
                         int32_t* perm, cudaStream_t s, const int* unsorted = nullptr);
void launch_sort_fixup(const int32_t* start, int64_t ncells_cap, const int64_t* total_cells, int32_t* perm,
                       cudaStream_t s);
void launch_gather(const double* src, double* dst, int ncomp, int64_t N, const int32_t* perm, const int64_t* count,
                   cudaStream_t s);
void launch_gather_i32(const int32_t* src, int32_t* dst, int64_t N, const int32_t* perm, const int64_t* count,
                       cudaStream_t s);
// fixup that also zeroes the per-cell fill counters it has consumed
// (with `unsorted` left zero it only counts the in-order sort)
void launch_sort_fixup_clear(const int32_t* start, int64_t ncells_cap, const int64_t* total_cells, int32_t* perm,
                             int32_t* fill, cudaStream_t s, const int* unsorted = nullptr,
                             unsigned long long* in_order_count = nullptr);
// Every carried field of a slot in one launch.
constexpr int GATHER_MAX = 16;
struct GatherArgs {
    int nf, ni;
    const double* src[GATHER_MAX];
    double* dst[GATHER_MAX];
    int ncomp[GATHER_MAX];
    const int32_t* isrc[4];
    int32_t* idst[4];
    int* clear;  // optional: a sort's order flag, zeroed by the gather
};
void launch_gather_fields(const GatherArgs& a, int64_t N, const int32_t* perm, const int64_t* count,
                          cudaStream_t s);

// ------------------------------------------------------------------ grid
struct GridPlanArgs {
    GridInst* gi;
    GridInst* gi_b;        // system_b-side copy (two-sided interactions): geometry mirrored, or nullptr
    int ninst, nd;
    const SysInst* a;      // system_a per-instance bbox
    const SysInst* b;      // system_b per-instance bbox (nullptr for self)
    const int64_t* bn;     // ghost-b counts per instance (nullptr otherwise)
    int64_t* need;         // total cells
    int* err;
    // interactions whose system_b does not move (nullptr otherwise): after
    // the plan, keep[1] = (every instance's grid equals prev) && keep[0],
    // prev = the grid, keep[0] = 1.  keep[0] says the CSR is current for
    // prev; keep[1] lets this step's count and scan return at once.
    GridInst* prev;
    int* keep;
};
void launch_grid_plan(const GridPlanArgs& a, cudaStream_t s);
// The plans of n interactions (device array of arguments), one block each.
void launch_grid_plan_all(const GridPlanArgs* d_args, int n, cudaStream_t s);
// cell histogram of the particles of one slot on an interaction's grid
// (skip: optional device flag; when set, the launch returns at once).
void launch_grid_count(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count,
                       const GridInst* gi, int32_t* hist, int64_t cells_cap, int* err,
                       unsigned long long* incons, cudaStream_t s, const int* skip = nullptr);
// The grids of the interactions whose system_b does not move, counted and
// scanned in one launch each: entry y of the table is interaction y's CSR,
// counted into its own histogram (zero between uses; the scan clears it)
// and skipped on the device while keep[1] is set.  cells <= STILL_MAX_CELLS.
constexpr int STILL_MAX = 16;
constexpr int64_t STILL_MAX_CELLS = 2048LL * 2048LL;
struct StillGrid {
    const double* x;
    const int32_t* inst_of;
    int64_t N;      // system_b's particles
    const GridInst* gi;
    const int* keep;
    int32_t* hist;  // cells entries, then the scan's tile sums
    int32_t* cs;    // CSR, cells + 1 entries
    int64_t cells;
};
struct StillGridArgs {
    StillGrid g[STILL_MAX];
    int n, nd;
    int* err;
    unsigned long long* incons;
};
// Tile sums after the histogram's cells: entries of hist beyond cells.
int64_t still_hist_elems(int64_t cells);
void launch_still_grids(const StillGridArgs& a, cudaStream_t s);

// ---------------------------------------------------------------- ghosts
struct GhostGenArgs {
    const double* src_x;   // source slot positions
    int64_t Nsrc;
    const int32_t* src_inst_of;
    GhostInst* gh;
    int ninst, nd, nplanes;
    int32_t* flags;        // nplanes*Nsrc
    int32_t* pos;          // nplanes*Nsrc + 1
    // raw (generation-order) ghost arrays, capacity nplanes*Nsrc
    double* gx;
    int32_t *gio, *gib, *ginst;
    double* gnormals;
    int64_t* count;        // total ghosts (device)
    SysInst* ginst_params; // ghost sort parameters per instance
};
void launch_ghost_flags(const GhostGenArgs& a, cudaStream_t s);
void launch_ghost_fill(const GhostGenArgs& a, cudaStream_t s);
void launch_ghost_kinematics(int64_t cap, const int64_t* count, int nd, const int32_t* io, const int32_t* ginst,
                             const double* normals, const GhostInst* gh, const double* src_v, const double* src_rho,
                             int64_t Nsrc, double* gv, double* grho, cudaStream_t s);
void launch_ghost_copy(int64_t cap, const int64_t* count, int nd, int ns, const int32_t* io, const int32_t* ginst,
                       const double* normals, const GhostInst* gh, int field, int mode, const double* src,
                       int64_t Nsrc, double* dst, cudaStream_t s);

// --------------------------------------------------------------- host I/O
void launch_aos_to_planar(const double* src, double* dst, int64_t n, int comps, int64_t N, int64_t base,
                          cudaStream_t s);
void launch_planar_to_aos(const double* src, double* dst, int64_t n, int comps, int64_t N, int64_t base,
                          cudaStream_t s);
void launch_i64_to_i32(const int64_t* src, int32_t* dst, int64_t n, cudaStream_t s);
void launch_i32_to_i64(const int32_t* src, int64_t* dst, int64_t n, cudaStream_t s);

// ------------------------------------------------------------ measurement
void launch_sum_counts(const int32_t* c, int64_t n, unsigned long long* out, cudaStream_t s);
void launch_fp64_peak(double* out, int blocks, int threads, int iters, cudaStream_t s);
void launch_fp32_peak(float* out, int blocks, int threads, int iters, cudaStream_t s);
extern std::atomic<long long> g_launches;

}  // namespace gc
