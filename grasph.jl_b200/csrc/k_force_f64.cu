// k_force_f64.cu — dispatch of the fused pair sweep, warp-group lists and
// per-particle divisor caches.  Compiled with -fmad=false.
#include <cstdio>

#include "gc_device.cuh"
#include "gc_force.h"
#include "gc_kernels.h"
#include "gc_pack.cuh"

namespace gc {

int launch_force_2d_f64(const ForceArgs& A, bool count_only, cudaStream_t s);
int launch_force_3d_f64(const ForceArgs& A, bool count_only, cudaStream_t s);
int launch_force_2d_f32(const ForceArgs& A, bool count_only, cudaStream_t s);
int launch_force_3d_f32(const ForceArgs& A, bool count_only, cudaStream_t s);

int launch_force_f64(const ForceArgs& A, bool count_only, cudaStream_t s) {
    if (A.aN <= 0 || A.nref == 0) return 0;
    const bool f32 = A.prec == GC_PRECISION_FP32_COMPENSATED && !count_only && A.pfn != GC_PFN_COUNT;
    if (A.nd == 2) return f32 ? launch_force_2d_f32(A, count_only, s) : launch_force_2d_f64(A, count_only, s);
    return f32 ? launch_force_3d_f32(A, count_only, s) : launch_force_3d_f64(A, count_only, s);
}

// --------------------------------------------------------------- groups
// Columns of the primary grid → warp groups of ≤ 32 consecutive particles.
__device__ __forceinline__ int find_inst(const GridInst* gi, int ninst, int64_t col) {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (gi[mid].colbase <= col) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// `cells_cap`: cells of `cs` that are valid (cs holds cells_cap + 1
// entries); an instance whose grid reaches beyond them contributes nothing
// (the grid build has flagged the overflow).
__global__ void k_groups_count(const GridInst* __restrict__ gi, int ninst, int nd, const int32_t* __restrict__ cs,
                               int64_t ncols_cap, int64_t cells_cap, int32_t* __restrict__ cnt) {
    pdl_enter();
    const int64_t T = gi[ninst - 1].colbase + gi[ninst - 1].ncols;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncols_cap;
         c += (int64_t)gridDim.x * blockDim.x) {
        if (c >= T) {
            cnt[c] = 0;
            continue;
        }
        const GridInst& G = gi[find_inst(gi, ninst, c)];
        const int64_t ngl = G.ng[nd - 1];
        const int64_t local = c - G.colbase;
        const int64_t b = G.cellbase + local * ngl;
        if (G.cellbase + G.ncells > cells_cap) {
            cnt[c] = 0;
            continue;
        }
        const int32_t n = cs[b + ngl] - cs[b];
        cnt[c] = (n + 31) / 32;
    }
}

__global__ void k_groups_fill(const GridInst* __restrict__ gi, int ninst, int nd, const int32_t* __restrict__ cs,
                              const int32_t* __restrict__ off, int64_t ncols_cap, int64_t cells_cap,
                              int2* __restrict__ groups, int64_t* ngroups) {
    pdl_enter();
    const int64_t T = gi[ninst - 1].colbase + gi[ninst - 1].ncols;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < T && c < ncols_cap;
         c += (int64_t)gridDim.x * blockDim.x) {
        const GridInst& G = gi[find_inst(gi, ninst, c)];
        if (G.cellbase + G.ncells > cells_cap) continue;
        const int64_t ngl = G.ng[nd - 1];
        const int64_t local = c - G.colbase;
        const int64_t b = G.cellbase + local * ngl;
        const int32_t s0 = cs[b], n = cs[b + ngl] - s0;
        int32_t o = off[c];
        for (int32_t q = 0; q < n; q += 32) groups[o++] = make_int2(s0 + q, n - q < 32 ? n - q : 32);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *ngroups = off[ncols_cap];
}

void launch_groups_count(const GridInst* gi, int ninst, int nd, const int32_t* cs, int64_t ncols_cap,
                         int64_t cells_cap, int32_t* cnt, cudaStream_t s) {
    int64_t b = (ncols_cap + 255) / 256;
    if (b < 1) b = 1;
    k_groups_count<<<(int)b, 256, 0, s>>>(gi, ninst, nd, cs, ncols_cap, cells_cap, cnt);
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_groups_fill(const GridInst* gi, int ninst, int nd, const int32_t* cs, const int32_t* off,
                        int64_t ncols_cap, int64_t cells_cap, int2* groups, int64_t* ngroups, cudaStream_t s) {
    int64_t b = (ncols_cap + 255) / 256;
    if (b < 1) b = 1;
    k_groups_fill<<<(int)b, 256, 0, s>>>(gi, ninst, nd, cs, off, ncols_cap, cells_cap, groups, ngroups);
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

// Per-particle factors the functors divide by, computed once per stage
// with the reference's expressions so pair terms stay bit-identical.
__global__ void k_aux(int mode, int64_t N, const int64_t* count, const double* __restrict__ rho,
                      const double* __restrict__ p, const int32_t* __restrict__ inst_of, const double* mass,
                      double* __restrict__ aux) {
    pdl_enter();
    int64_t n = count ? *count : N;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        double r = rho[g];
        if (mode == AUX_P_OVER_RHO2) aux[g] = p[g] / (r * r);
        else if (mode == AUX_INV_RHO2) aux[g] = 1.0 / (r * r);
        else aux[g] = mass[inst_of[g]] / r;
    }
}

__global__ void k_pack32(PackArgs a, const int64_t* count) {
    pdl_enter();
    const int64_t n = count ? *count : a.N;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x)
        pack_one(a, g);
}

void launch_pack32(int mode, int64_t N, const int64_t* count, int nd, int ns, const double* x, const double* v,
                   const double* rho, const double* p, const double* stress, const int32_t* inst_of,
                   const double* mass, double* xpk, float* pk, cudaStream_t s) {
    if (N <= 0 || (!xpk && !pk)) return;
    int64_t blocks = (N + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    PackArgs a{mode, nd, ns, N, x, v, rho, p, stress, inst_of, mass, xpk, pk};
    k_pack32<<<(int)blocks, 256, 0, s>>>(a, count);
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_aux(int mode, int64_t N, const int64_t* count, const double* rho, const double* p,
                const int32_t* inst_of, const double* mass, double* aux, cudaStream_t s) {
    if (N <= 0) return;
    int blocks = (int)((N + 255) / 256);
    k_aux<<<blocks, 256, 0, s>>>(mode, N, count, rho, p, inst_of, mass, aux);
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

}  // namespace gc
