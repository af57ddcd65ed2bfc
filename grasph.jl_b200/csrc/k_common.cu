// k_common.cu — scan, bounding boxes, stable counting sort, grid CSR and
// ghost generation kernels.  All HBM-bound integer/byte work plus the FP64
// key/cell arithmetic, which follows the reference bit for bit:
//   key  = floor(x_d / cutoff)                    src/Sorting.jl:122-124
//   cell = floor((x_d - mingridx_d) / cell_size)  src/Interaction.jl:197-206
// Compiled with -fmad=false.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "gc_device.cuh"
#include "gc_kernels.h"

namespace gc {

std::atomic<long long> g_launches{0};

constexpr int TPB = 256;

static inline int nblk(int64_t n, int tpb = TPB) {
    int64_t b = (n + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > 2147483647LL) b = 2147483647LL;
    return (int)b;
}

// Every launcher adds the number of kernels it enqueued.
#define COUNTED(n) (g_launches.fetch_add((n), std::memory_order_relaxed))

// Warp-aggregated counter increment: every lane of the warp calls it; each
// valid lane adds 1 to ctr[k] and receives a distinct slot of the counter's
// old value + its rank among the warp's lanes with the same k (in lane
// order).  Sorted or nearly sorted keys give one atomic per distinct key per
// warp instead of one per particle.
__device__ __forceinline__ int32_t warp_agg_inc(int32_t* ctr, int32_t k, bool valid) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned grp = __match_any_sync(FULL, valid ? k : INT32_MIN);
    const int leader = __ffs(grp) - 1;
    int32_t base = 0;
    if (valid && lane == leader) base = atomicAdd(&ctr[k], __popc(grp));
    base = __shfl_sync(FULL, base, leader);
    return base + __popc(grp & ((1u << lane) - 1u));
}

// ================================================================== scan
constexpr int SCAN_T = 512, SCAN_I = 4, SCAN_TILE = SCAN_T * SCAN_I;

__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t* total) {
    __shared__ int32_t warp_sums[SCAN_T / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int32_t w = lane < SCAN_T / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_T / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    int32_t base = wid > 0 ? warp_sums[wid - 1] : 0;
    *total = warp_sums[SCAN_T / 32 - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void k_scan_reduce(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ bsum,
                              const int* skip) {
    pdl_enter();
    if (skip && *skip) return;
    int64_t t0 = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k)
        if (t0 + k < n) s += in[t0 + k];
    int32_t total;
    (void)block_excl_scan(s, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int64_t n, const int32_t* __restrict__ boff,
                             int32_t* __restrict__ out, int32_t* clear, const int* skip) {
    pdl_enter();
    if (skip && *skip) return;
    int64_t t0 = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
    int32_t v[SCAN_I];
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        v[k] = t0 + k < n ? in[t0 + k] : 0;
        s += v[k];
    }
    if (clear) {
#pragma unroll
        for (int k = 0; k < SCAN_I; ++k)
            if (t0 + k < n) clear[t0 + k] = 0;
    }
    int32_t total;
    int32_t run = block_excl_scan(s, &total) + (boff ? boff[blockIdx.x] : 0);
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        if (t0 + k < n) out[t0 + k] = run;
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = (boff ? boff[blockIdx.x] : 0) + total;
}

int64_t scan_tmp_elems(int64_t n) {
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb <= 1) return 0;
    return nb + (nb + 1) + scan_tmp_elems(nb);
}

// Second pass for up to SCAN_TILE tiles: each block adds up the sums of the
// tiles before it itself (at most SCAN_TILE values), so the scan of the tile
// sums needs no launch of its own.
__global__ void k_scan_apply_sums(const int32_t* __restrict__ in, int64_t n, const int32_t* __restrict__ bsum,
                                  int32_t* __restrict__ out, int32_t* clear, const int* skip) {
    pdl_enter();
    if (skip && *skip) return;
    __shared__ int32_t off;
    {
        int32_t s = 0;
        for (int64_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) s += bsum[b];
        int32_t total;
        (void)block_excl_scan(s, &total);
        if (threadIdx.x == 0) off = total;
        __syncthreads();
    }
    int64_t t0 = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
    int32_t v[SCAN_I];
    int32_t sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        v[k] = t0 + k < n ? in[t0 + k] : 0;
        sum += v[k];
    }
    if (clear) {
#pragma unroll
        for (int k = 0; k < SCAN_I; ++k)
            if (t0 + k < n) clear[t0 + k] = 0;
    }
    int32_t total;
    int32_t run = block_excl_scan(sum, &total) + off;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        if (t0 + k < n) out[t0 + k] = run;
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = off + total;
}

// skip: when non-null and *skip is set on the device, every launch returns
// at once (the output is already current).
static void scan_impl(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp, int32_t* clear, cudaStream_t s,
                      const int* skip) {
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb > 1 && nb <= SCAN_TILE) {
        k_scan_reduce<<<(unsigned)nb, SCAN_T, 0, s>>>(in, n, tmp, skip);
        k_scan_apply_sums<<<(unsigned)nb, SCAN_T, 0, s>>>(in, n, tmp, out, clear, skip);
        COUNTED(2);
        return;
    }
    if (nb <= 1) {
        k_scan_apply<<<1, SCAN_T, 0, s>>>(in, n, nullptr, out, clear, skip);
        COUNTED(1);
        return;
    }
    int32_t* bsum = tmp;
    int32_t* boff = tmp + nb;
    k_scan_reduce<<<(unsigned)nb, SCAN_T, 0, s>>>(in, n, bsum, skip);
    scan_impl(bsum, boff, nb, tmp + nb + nb + 1, nullptr, s, skip);
    k_scan_apply<<<(unsigned)nb, SCAN_T, 0, s>>>(in, n, boff, out, clear, skip);
    COUNTED(2);
}

void scan_exclusive(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t s) {
    scan_impl(in, out, n, tmp, nullptr, s, nullptr);
}

void scan_exclusive_clear(int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t s, const int* skip) {
    scan_impl(in, out, n, tmp, in, s, skip);
}

// Particle g's coordinates, every load issued before any value is used
// (a loop over a run-time dimension count would otherwise wait out one
// memory round trip per coordinate).
__device__ __forceinline__ void load_pos(const double* __restrict__ x, int64_t N, int64_t g, int nd, double* v) {
#pragma unroll
    for (int d = 0; d < MAXD; ++d) v[d] = d < nd ? x[d * N + g] : 0.0;
}

// ========================================================== bounding box
__global__ void k_bbox_reset(unsigned long long* scratch, int ninst) {
    pdl_enter();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ninst) return;
    for (int d = 0; d < MAXD; ++d) {
        scratch[(k * 2 + 0) * MAXD + d] = ~0ull;
        scratch[(k * 2 + 1) * MAXD + d] = 0ull;
    }
}

__global__ void k_bbox(const double* __restrict__ x, int64_t N, int nd, const int32_t* __restrict__ inst_of,
                       const int64_t* count, unsigned long long* scratch, int* err) {
    pdl_enter();
    int64_t n = count ? *count : N;
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = g < n;
    int k = valid ? inst_of[g] : -1;
    unsigned long long mn[MAXD], mx[MAXD];
    bool bad = false;
    for (int d = 0; d < MAXD; ++d) {
        mn[d] = ~0ull;
        mx[d] = 0ull;
    }
    if (valid) {
        for (int d = 0; d < nd; ++d) {
            double v = x[d * N + g];
            if (!isfinite(v)) bad = true;
            mn[d] = mx[d] = ord_key(v);
        }
    }
    if (bad) atomicOr(err, ERR_NONFINITE);
    __shared__ int k0;
    if (threadIdx.x == 0) k0 = k;
    __syncthreads();
    int uniform = __syncthreads_and(!valid || k == k0);
    if (uniform && k0 >= 0) {
        // block-uniform instance: reduce then one atomic per dimension
        __shared__ unsigned long long smn[TPB / 32][MAXD], smx[TPB / 32][MAXD];
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int d = 0; d < nd; ++d) {
            unsigned long long a = mn[d], b = mx[d];
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long a2 = __shfl_down_sync(0xffffffffu, a, o);
                unsigned long long b2 = __shfl_down_sync(0xffffffffu, b, o);
                a = a2 < a ? a2 : a;
                b = b2 > b ? b2 : b;
            }
            if (lane == 0) {
                smn[wid][d] = a;
                smx[wid][d] = b;
            }
        }
        __syncthreads();
        if (threadIdx.x < nd) {
            int d = threadIdx.x;
            unsigned long long a = ~0ull, b = 0ull;
            for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
                a = smn[w][d] < a ? smn[w][d] : a;
                b = smx[w][d] > b ? smx[w][d] : b;
            }
            atomicMin(&scratch[(k0 * 2 + 0) * MAXD + d], a);
            atomicMax(&scratch[(k0 * 2 + 1) * MAXD + d], b);
        }
    } else if (valid) {
        for (int d = 0; d < nd; ++d) {
            atomicMin(&scratch[(k * 2 + 0) * MAXD + d], mn[d]);
            atomicMax(&scratch[(k * 2 + 1) * MAXD + d], mx[d]);
        }
    }
}

__global__ void k_bbox_finish(const unsigned long long* scratch, SysInst* inst, int ninst, int nd) {
    pdl_enter();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ninst) return;
    for (int d = 0; d < nd; ++d) {
        unsigned long long a = scratch[(k * 2 + 0) * MAXD + d], b = scratch[(k * 2 + 1) * MAXD + d];
        inst[k].bbmin[d] = a == ~0ull ? 0.0 : ord_val(a);
        inst[k].bbmax[d] = b == 0ull ? 0.0 : ord_val(b);
    }
}

void launch_bbox_reset(unsigned long long* scratch, int ninst, cudaStream_t s) {
    k_bbox_reset<<<nblk(ninst), TPB, 0, s>>>(scratch, ninst);
    COUNTED(1);
}

// One-launch bounding box: block reductions into the per-instance scratch,
// then the last block to finish writes the boxes and resets the scratch
// (and the block counter after it) for the next launch.
__global__ void k_bbox_fused(const double* __restrict__ x, int64_t N, int nd, const int32_t* __restrict__ inst_of,
                             const int64_t* count, unsigned long long* scratch, SysInst* inst, int ninst, int* err,
                             int64_t tiles_per_block) {
    pdl_enter();
    // each block reduces a contiguous run of 256-particle tiles: every thread
    // keeps the running min/max of its particles while they belong to one
    // instance (flushing with atomics when the instance changes), and the
    // block reduces them once at the end, so one block makes 2·nd atomics,
    // not 2·nd per tile (ordered keys: min/max is exact in any order)
    const int64_t n = count ? *count : N;
    int krun = -1;
    unsigned long long amn[MAXD], amx[MAXD];
    for (int d = 0; d < MAXD; ++d) {
        amn[d] = ~0ull;
        amx[d] = 0ull;
    }
    bool bad = false;
    for (int64_t tile = (int64_t)blockIdx.x * tiles_per_block;
         tile < (int64_t)(blockIdx.x + 1) * tiles_per_block && tile * blockDim.x < n; ++tile) {
        const int64_t g = tile * blockDim.x + threadIdx.x;
        if (g >= n) continue;
        double xv[MAXD];
        load_pos(x, N, g, nd, xv);
        const int k = inst_of[g];
        if (k != krun) {
            if (krun >= 0)
                #pragma unroll
                for (int d = 0; d < MAXD; ++d) {
                    if (d >= nd) break;
                    atomicMin(&scratch[(krun * 2 + 0) * MAXD + d], amn[d]);
                    atomicMax(&scratch[(krun * 2 + 1) * MAXD + d], amx[d]);
                }
            krun = k;
            for (int d = 0; d < MAXD; ++d) {
                amn[d] = ~0ull;
                amx[d] = 0ull;
            }
        }
        #pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= nd) break;
            const double v = xv[d];
            if (!isfinite(v)) bad = true;
            const unsigned long long key = ord_key(v);
            amn[d] = key < amn[d] ? key : amn[d];
            amx[d] = key > amx[d] ? key : amx[d];
        }
    }
    if (bad) atomicOr(err, ERR_NONFINITE);
    // thread 0 holds the block's first particle, so its instance is the
    // block's whenever the block has any
    __shared__ int k0;
    if (threadIdx.x == 0) k0 = krun;
    __syncthreads();
    const int uniform = __syncthreads_and(krun < 0 || krun == k0);
    if (uniform && k0 >= 0) {
        __shared__ unsigned long long smn[TPB / 32][MAXD], smx[TPB / 32][MAXD];
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        #pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= nd) break;
            unsigned long long a = amn[d], b = amx[d];
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long a2 = __shfl_down_sync(0xffffffffu, a, o);
                unsigned long long b2 = __shfl_down_sync(0xffffffffu, b, o);
                a = a2 < a ? a2 : a;
                b = b2 > b ? b2 : b;
            }
            if (lane == 0) {
                smn[wid][d] = a;
                smx[wid][d] = b;
            }
        }
        __syncthreads();
        if (threadIdx.x < nd) {
            const int d = threadIdx.x;
            unsigned long long a = ~0ull, b = 0ull;
            for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
                a = smn[w][d] < a ? smn[w][d] : a;
                b = smx[w][d] > b ? smx[w][d] : b;
            }
            atomicMin(&scratch[(k0 * 2 + 0) * MAXD + d], a);
            atomicMax(&scratch[(k0 * 2 + 1) * MAXD + d], b);
        }
    } else if (krun >= 0) {
        #pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= nd) break;
            atomicMin(&scratch[(krun * 2 + 0) * MAXD + d], amn[d]);
            atomicMax(&scratch[(krun * 2 + 1) * MAXD + d], amx[d]);
        }
    }
    unsigned long long* counter = scratch + (size_t)ninst * 2 * MAXD;
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1ull) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int k = threadIdx.x; k < ninst; k += blockDim.x) {
        #pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= nd) break;
            unsigned long long a = atomicExch(&scratch[(k * 2 + 0) * MAXD + d], ~0ull);
            unsigned long long b = atomicExch(&scratch[(k * 2 + 1) * MAXD + d], 0ull);
            inst[k].bbmin[d] = a == ~0ull ? 0.0 : ord_val(a);
            inst[k].bbmax[d] = b == 0ull ? 0.0 : ord_val(b);
        }
    }
    if (threadIdx.x == 0) atomicExch(counter, 0ull);
}

void launch_bbox_fused(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count,
                       SysInst* inst, unsigned long long* scratch, int ninst, int* err, cudaStream_t s) {
    const int64_t tiles = std::max<int64_t>((N + TPB - 1) / TPB, 1);
    const int64_t per = std::max<int64_t>((tiles + 1183) / 1184, 1);  // about 8 blocks per SM
    const int blocks = (int)((tiles + per - 1) / per);
    k_bbox_fused<<<blocks, TPB, 0, s>>>(x, N, nd, inst_of, count, scratch, inst, ninst, err, per);
    COUNTED(1);
}

void launch_bbox(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count, SysInst* inst,
                 unsigned long long* scratch, int ninst, int* err, cudaStream_t s) {
    k_bbox_reset<<<nblk(ninst), TPB, 0, s>>>(scratch, ninst);
    if (N > 0) k_bbox<<<nblk(N), TPB, 0, s>>>(x, N, nd, inst_of, count, scratch, err);
    k_bbox_finish<<<nblk(ninst), TPB, 0, s>>>(scratch, inst, ninst, nd);
    COUNTED(N > 0 ? 3 : 2);
}

// ================================================================== sort
__global__ void k_sort_plan(SysInst* inst, int ninst, int nd, int64_t* need, int* err) {
    pdl_enter();
    for (int k = threadIdx.x; k < ninst; k += blockDim.x) {
        SysInst& S = inst[k];
        int64_t cells = S.n > 0 ? 1 : 0;
        for (int d = 0; d < nd && S.n > 0; ++d) {
            int64_t lo, hi;
            bool ok = floor_i64(S.bbmin[d] / S.sort_cutoff, &lo) && floor_i64(S.bbmax[d] / S.sort_cutoff, &hi);
            if (!ok) {
                atomicOr(err, ERR_NONFINITE);
                lo = hi = 0;
            }
            S.kmin[d] = lo;
            S.kext[d] = hi - lo + 1;
            cells *= S.kext[d];
            if (cells > (1LL << 31)) {
                atomicOr(err, ERR_CAPACITY);
                cells = 1LL << 31;
            }
        }
        S.sort_ncells = cells;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t base = 0;
        for (int k = 0; k < ninst; ++k) {
            inst[k].sort_cellbase = base;
            base += inst[k].sort_ncells;
        }
        *need = base;
    }
}

void launch_sort_plan(SysInst* inst, int ninst, int nd, int64_t* need, int* err, cudaStream_t s) {
    k_sort_plan<<<1, 1024, 0, s>>>(inst, ninst, nd, need, err);
    COUNTED(1);
}

// The packed cell key of particle g (src/Sorting.jl:157-175): -1 with
// `bad` set to the error bit when a coordinate is not finite or falls
// outside the planned cells.
__device__ __forceinline__ int32_t sort_key_of(const double* __restrict__ x, int64_t N, int nd,
                                               const int32_t* __restrict__ inst_of, const SysInst* __restrict__ inst,
                                               int64_t g, int64_t cells_cap, int* bad) {
    double xv[MAXD];
    load_pos(x, N, g, nd, xv);
    const SysInst& S = inst[inst_of[g]];
    int64_t flat = 0;
    bool ok = true;
    #pragma unroll
    for (int d = 0; d < MAXD; ++d) {
        if (d >= nd) break;
        int64_t kd;
        if (!floor_i64(xv[d] / S.sort_cutoff, &kd)) {
            ok = false;
            break;
        }
        int64_t rel = kd - S.kmin[d];
        if (rel < 0 || rel >= S.kext[d]) ok = false;
        flat = flat * S.kext[d] + rel;
    }
    flat += S.sort_cellbase;
    if (!ok || flat < 0 || flat >= cells_cap) {
        *bad = ok ? ERR_CAPACITY : ERR_NONFINITE;
        return -1;
    }
    *bad = 0;
    return (int32_t)flat;
}

__global__ void k_sort_keys(const double* __restrict__ x, int64_t N, int nd, const int32_t* __restrict__ inst_of,
                            const int64_t* count, const SysInst* __restrict__ inst, int32_t* __restrict__ key,
                            int32_t* __restrict__ hist, int64_t cells_cap, int* err, int* unsorted) {
    pdl_enter();
    int64_t n = count ? *count : N;
    const int lane = threadIdx.x & 31;
    // whole warps iterate together (warp-aggregated histogram)
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x; g0 < n; g0 += stride) {
        const int64_t g = g0 + threadIdx.x;
        bool valid = g < n;
        int32_t kk = -1;
        int bad = 0;
        if (valid) {
            kk = sort_key_of(x, N, nd, inst_of, inst, g, cells_cap, &bad);
            if (bad) {
                atomicOr(err, bad);
                valid = false;
            }
            key[g] = kk;
        }
        warp_agg_inc(hist, kk, valid);
        if (unsorted) {
            // keys already non-decreasing (src/Sorting.jl:176-186): each
            // thread compares with the key before it, from the lane below,
            // the previous warp's last lane (shared memory) or, for the
            // block's first thread, recomputed; an invalid key counts as out
            // of order
            __shared__ int32_t wlast[TPB / 32];
            const int wid = threadIdx.x >> 5;
            int32_t prev = __shfl_up_sync(0xffffffffu, kk, 1);
            if (lane == 31) wlast[wid] = kk;
            __syncthreads();
            if (lane == 0) {
                if (wid > 0) {
                    prev = wlast[wid - 1];
                } else if (g > 0 && g < n) {
                    int pb = 0;
                    prev = sort_key_of(x, N, nd, inst_of, inst, g - 1, cells_cap, &pb);
                }
            }
            __syncthreads();  // wlast is rewritten by the next tile
            const bool order_broken = g < n && (bad || (g > 0 && prev > kk));
            if (__any_sync(0xffffffffu, order_broken) && lane == 0) atomicOr(unsorted, 1);
        }
    }
}

void launch_sort_keys(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count,
                      const SysInst* inst, int32_t* key, int32_t* hist, int64_t cells_cap, int* err, cudaStream_t s,
                      int* unsorted) {
    if (N <= 0) return;
    k_sort_keys<<<nblk(N), TPB, 0, s>>>(x, N, nd, inst_of, count, inst, key, hist, cells_cap, err,
                                        unsorted);  // blockDim == TPB, a multiple of 32
    COUNTED(1);
}

__global__ void k_sort_scatter(const int32_t* __restrict__ key, int64_t N, const int64_t* count,
                               const int32_t* __restrict__ start, int32_t* __restrict__ fill,
                               int32_t* __restrict__ perm, const int* unsorted) {
    pdl_enter();
    int64_t n = count ? *count : N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    if (unsorted && *unsorted == 0) {
        // keys in order: the stable sort is the identity
        for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += stride) perm[g] = (int32_t)g;
        return;
    }
    // whole warps iterate together (warp-aggregated fill counters); the
    // order inside a cell is restored by the fix-up
    for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x; g0 < n; g0 += stride) {
        const int64_t g = g0 + threadIdx.x;
        const int32_t k = g < n ? key[g] : -1;
        const bool valid = k >= 0;
        const int32_t slot = warp_agg_inc(fill, k, valid);
        if (valid) perm[start[k] + slot] = (int32_t)g;
    }
}

void launch_sort_scatter(const int32_t* key, int64_t N, const int64_t* count, const int32_t* start, int32_t* fill,
                         int32_t* perm, cudaStream_t s, const int* unsorted) {
    if (N <= 0) return;
    k_sort_scatter<<<nblk(N), TPB, 0, s>>>(key, N, count, start, fill, perm, unsorted);
    COUNTED(1);
}

// Atomic placement leaves each cell's members in arbitrary order; sorting
// each cell's segment by source index restores the stable order of
// Julia's sortperm (equal keys keep ascending original index).
__global__ void k_sort_fixup(const int32_t* __restrict__ start, int64_t ncells_cap, const int64_t* total_cells,
                             int32_t* __restrict__ perm) {
    pdl_enter();
    int64_t nc = *total_cells;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc && c < ncells_cap;
         c += (int64_t)gridDim.x * blockDim.x) {
        int32_t s = start[c], e = start[c + 1];
        for (int32_t i = s + 1; i < e; ++i) {
            int32_t v = perm[i];
            int32_t j = i - 1;
            while (j >= s && perm[j] > v) {
                perm[j + 1] = perm[j];
                --j;
            }
            perm[j + 1] = v;
        }
    }
}

// Sort W values in registers (a bitonic network: no data-dependent
// branches, every index known at compile time, so v stays in registers).
template <int W>
__device__ __forceinline__ void reg_sort(int32_t* v) {
#pragma unroll
    for (int k = 2; k <= W; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < W; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const int32_t a = v[i], b = v[l];
                    const bool up = (i & k) == 0;
                    v[i] = up ? min(a, b) : max(a, b);
                    v[l] = up ? max(a, b) : min(a, b);
                }
            }
}

// One cell's segment perm[s, s + m) with m <= W sorted ascending in
// registers (padding INT32_MAX), unless it already is.
template <int W>
__device__ __forceinline__ void sort_segment(int32_t* __restrict__ perm, int32_t s, int32_t m) {
    int32_t v[W];
    bool sorted = true;
#pragma unroll
    for (int q = 0; q < W; ++q) {
        v[q] = q < m ? perm[s + q] : INT32_MAX;
        if (q > 0 && v[q] < v[q - 1]) sorted = false;
    }
    if (sorted) return;
    reg_sort<W>(v);
#pragma unroll
    for (int q = 0; q < W; ++q)
        if (q < m) perm[s + q] = v[q];
}

// One thread per cell: the fill counter cleared, then the cell's segment
// sorted by source index in registers (segments of up to 32 members; a
// larger one by an insertion sort in place).
__global__ void k_sort_fixup_clear(const int32_t* __restrict__ start, int64_t ncells_cap, const int64_t* total_cells,
                                   int32_t* __restrict__ perm, int32_t* __restrict__ fill, const int* unsorted,
                                   unsigned long long* in_order_count) {
    pdl_enter();
    if (unsorted && *unsorted == 0) {
        // the scatter placed nothing through the fill counters
        if (in_order_count && blockIdx.x == 0 && threadIdx.x == 0) *in_order_count += 1ull;
        return;
    }
    int64_t nc = *total_cells;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc && c < ncells_cap;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = start[c], e = start[c + 1];
        fill[c] = 0;
        const int32_t m = e - s;
        if (m <= 1) continue;
        if (m <= 8) {
            sort_segment<8>(perm, s, m);
        } else if (m <= 16) {
            sort_segment<16>(perm, s, m);
        } else if (m <= 32) {
            sort_segment<32>(perm, s, m);
        } else {
            for (int32_t i = s + 1; i < e; ++i) {
                int32_t v = perm[i];
                int32_t j = i - 1;
                while (j >= s && perm[j] > v) {
                    perm[j + 1] = perm[j];
                    --j;
                }
                perm[j + 1] = v;
            }
        }
    }
}

void launch_sort_fixup_clear(const int32_t* start, int64_t ncells_cap, const int64_t* total_cells, int32_t* perm,
                             int32_t* fill, cudaStream_t s, const int* unsorted, unsigned long long* in_order_count) {
    if (ncells_cap <= 0) return;
    k_sort_fixup_clear<<<nblk(ncells_cap), TPB, 0, s>>>(start, ncells_cap, total_cells, perm, fill, unsorted,
                                                        in_order_count);
    COUNTED(1);
}

void launch_sort_fixup(const int32_t* start, int64_t ncells_cap, const int64_t* total_cells, int32_t* perm,
                       cudaStream_t s) {
    if (ncells_cap <= 0) return;
    k_sort_fixup<<<nblk(ncells_cap), TPB, 0, s>>>(start, ncells_cap, total_cells, perm);
    COUNTED(1);
}

__global__ void k_gather(const double* __restrict__ src, double* __restrict__ dst, int ncomp, int64_t N,
                         const int32_t* __restrict__ perm, const int64_t* count) {
    pdl_enter();
    int64_t n = count ? *count : N;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = perm[g];
        // a permutation left incomplete by a flagged key overflow may hold
        // stale entries: keep every read inside the array
        if ((uint64_t)o >= (uint64_t)N) o = g;
        for (int c = 0; c < ncomp; ++c) dst[c * N + g] = src[c * N + o];
    }
}

__global__ void k_gather_i32(const int32_t* __restrict__ src, int32_t* __restrict__ dst, int64_t N,
                             const int32_t* __restrict__ perm, const int64_t* count) {
    pdl_enter();
    int64_t n = count ? *count : N;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = perm[g];
        if ((uint64_t)o >= (uint64_t)N) o = g;
        dst[g] = src[o];
    }
}

// blockIdx.y picks the field (the int32 fields after the double ones), so
// every thread has one independent gather per component.
__global__ void k_gather_fields(GatherArgs a, int64_t N, const int32_t* __restrict__ perm, const int64_t* count) {
    pdl_enter();
    const int64_t n = count ? *count : N;
    const int f = blockIdx.y;
    // the sort's order flag, read by the scatter and fix-up launched
    // before this gather, is cleared for the next sort
    if (a.clear && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *a.clear = 0;
    // two elements per thread (g and g + blockDim.x), their loads issued
    // together
    const int64_t step = (int64_t)gridDim.x * blockDim.x * 2;
    for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x * 2 + threadIdx.x; g0 < n; g0 += step) {
        int64_t gs[2] = {g0, g0 + blockDim.x};
        int64_t o[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            o[e] = gs[e] < n ? perm[gs[e]] : gs[e];
            if ((uint64_t)o[e] >= (uint64_t)N) o[e] = gs[e];
        }
        if (f < a.nf) {
            const double* __restrict__ src = a.src[f];
            double* __restrict__ dst = a.dst[f];
            const int nc = a.ncomp[f];
            double v[2][MAXS];
#pragma unroll
            for (int e = 0; e < 2; ++e)
#pragma unroll
                for (int c = 0; c < MAXS; ++c)
                    if (c < nc && gs[e] < n) v[e][c] = __ldg(src + c * N + o[e]);
#pragma unroll
            for (int e = 0; e < 2; ++e)
#pragma unroll
                for (int c = 0; c < MAXS; ++c)
                    if (c < nc && gs[e] < n) dst[c * N + gs[e]] = v[e][c];
        } else {
            int32_t iv[2];
#pragma unroll
            for (int e = 0; e < 2; ++e)
                if (gs[e] < n) iv[e] = __ldg(a.isrc[f - a.nf] + o[e]);
#pragma unroll
            for (int e = 0; e < 2; ++e)
                if (gs[e] < n) a.idst[f - a.nf][gs[e]] = iv[e];
        }
    }
}

void launch_gather_fields(const GatherArgs& a, int64_t N, const int32_t* perm, const int64_t* count,
                          cudaStream_t s) {
    if (N <= 0 || (a.nf == 0 && a.ni == 0)) return;
    dim3 grid((unsigned)nblk((N + 1) / 2), (unsigned)(a.nf + a.ni));
    k_gather_fields<<<grid, TPB, 0, s>>>(a, N, perm, count);
    COUNTED(1);
}

void launch_gather(const double* src, double* dst, int ncomp, int64_t N, const int32_t* perm, const int64_t* count,
                   cudaStream_t s) {
    if (N <= 0 || ncomp <= 0) return;
    k_gather<<<nblk(N), TPB, 0, s>>>(src, dst, ncomp, N, perm, count);
    COUNTED(1);
}

void launch_gather_i32(const int32_t* src, int32_t* dst, int64_t N, const int32_t* perm, const int64_t* count,
                       cudaStream_t s) {
    if (N <= 0) return;
    k_gather_i32<<<nblk(N), TPB, 0, s>>>(src, dst, N, perm, count);
    COUNTED(1);
}

// ================================================================== grid
// src/Interaction.jl:131-193: origin snapped to a multiple of the cell
// size below min−2h, ngridx = floor((max+2h − origin)/h2) + 1.
__device__ void grid_plan_block(const GridPlanArgs& a);
__global__ void k_grid_plan(GridPlanArgs a) {
    pdl_enter(); grid_plan_block(a); }
__global__ void k_grid_plan_all(const GridPlanArgs* __restrict__ args) {
    pdl_enter(); grid_plan_block(args[blockIdx.x]); }

void launch_grid_plan_all(const GridPlanArgs* d_args, int n, cudaStream_t s) {
    if (n <= 0) return;
    k_grid_plan_all<<<n, 1024, 0, s>>>(d_args);
    COUNTED(1);
}

__device__ void grid_plan_block(const GridPlanArgs& a) {
    for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) {
        GridInst& G = a.gi[k];
        const SysInst& A = a.a[k];
        double mn[MAXD], mx[MAXD];
        #pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= a.nd) break;
            mn[d] = A.bbmin[d];
            mx[d] = A.bbmax[d];
            G.mina[d] = mn[d];
            G.maxa[d] = mx[d];
        }
        if (a.b) {
            const SysInst& B = a.b[k];
            if (B.n > 0)
                #pragma unroll
                for (int d = 0; d < MAXD; ++d) {
                    if (d >= a.nd) break;
                    mn[d] = jmin(mn[d], B.bbmin[d]);
                    mx[d] = jmax(mx[d], B.bbmax[d]);
                }
        }
        const double c = G.cell;
        int64_t cells = 1;
        #pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= a.nd) break;
            double raw = mn[d] - 2.0 * c;
            G.ming[d] = floor(raw / c) * c;
            double maxg = mx[d] + 2.0 * c;
            int64_t ngd;
            if (!floor_i64((maxg - G.ming[d]) / c, &ngd)) {
                atomicOr(a.err, ERR_NONFINITE);
                ngd = 0;
            }
            G.ng[d] = ngd + 1;
            cells *= G.ng[d];
            if (cells > (1LL << 31)) {
                atomicOr(a.err, ERR_CAPACITY);
                cells = 1LL << 31;
            }
        }
        G.ncells = cells;
        G.ncols = cells / G.ng[a.nd - 1];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t base = 0, cb = 0;
        for (int k = 0; k < a.ninst; ++k) {
            a.gi[k].cellbase = base;
            a.gi[k].colbase = cb;
            base += a.gi[k].ncells;
            cb += a.gi[k].ncols;
        }
        *a.need = base;
    }
    if (a.gi_b) {
        // the system_b-side copy keeps its own neighbour mass and sound speed
        __syncthreads();
        for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) {
            GridInst& B = a.gi_b[k];
            const double bm = B.bmass, bc = B.bc;
            const float fbm = B.f_bmass, fbc = B.f_bc;
            const int sb = B.side_b;
            B = a.gi[k];
            B.bmass = bm;
            B.bc = bc;
            B.side_b = sb;
            B.f_bmass = fbm;
            B.f_bc = fbc;
        }
    }
    if (a.keep) {
        // is every instance's grid the one the CSR was last counted on?
        __shared__ int same;
        __syncthreads();
        if (threadIdx.x == 0) same = a.keep[0];
        __syncthreads();
        for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) {
            const GridInst& g = a.gi[k];
            const GridInst& p = a.prev[k];
            bool eq = g.cellbase == p.cellbase && g.ncells == p.ncells;
            for (int d = 0; d < a.nd; ++d)
                eq = eq && g.ng[d] == p.ng[d] && __double_as_longlong(g.ming[d]) == __double_as_longlong(p.ming[d]);
            if (!eq) atomicAnd(&same, 0);
        }
        __syncthreads();
        for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) a.prev[k] = a.gi[k];
        if (threadIdx.x == 0) {
            a.keep[1] = same;
            a.keep[0] = 1;
        }
    }
}

void launch_grid_plan(const GridPlanArgs& a, cudaStream_t s) {
    k_grid_plan<<<1, 1024, 0, s>>>(a);
    COUNTED(1);
}

__device__ __forceinline__ bool cell_flat(const double* __restrict__ x, int64_t N, int64_t g, int nd,
                                          const GridInst& G, int64_t* flat) {
    double xv[MAXD];
    load_pos(x, N, g, nd, xv);
    int64_t f = 0;
    #pragma unroll
    for (int d = 0; d < MAXD; ++d) {
        if (d >= nd) break;
        int64_t cd;
        if (!floor_i64((xv[d] - G.ming[d]) / G.cell, &cd)) return false;
        if (cd < 0 || cd >= G.ng[d]) return false;
        f = f * G.ng[d] + cd;
    }
    *flat = f;
    return true;
}

// Blocks bid, bid + nblocks, ... of a grid-stride pass over the particles.
__device__ __forceinline__ void grid_count_blocks(const double* __restrict__ x, int64_t N, int nd,
                                                  const int32_t* __restrict__ inst_of, const int64_t* count,
                                                  const GridInst* __restrict__ gi, int32_t* __restrict__ hist,
                                                  int64_t cells_cap, int* err, unsigned long long* incons,
                                                  int64_t bid, int64_t nblocks) {
    int64_t n = count ? *count : N;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // whole warps iterate together (warp-aggregated histogram; the previous
    // particle's cell comes from the neighbouring lane)
    const int64_t stride = nblocks * blockDim.x;
    for (int64_t g0 = bid * blockDim.x; g0 < n; g0 += stride) {
        const int64_t g = g0 + threadIdx.x;
        bool valid = g < n;
        int k = -1;
        int64_t f = -1;
        if (valid) {
            k = inst_of[g];
            const GridInst& G = gi[k];
            if (!cell_flat(x, N, g, nd, G, &f) || G.cellbase + f >= cells_cap) {
                atomicOr(err, ERR_CAPACITY);
                valid = false;
                f = -1;
            }
        }
        const int32_t cell = valid ? (int32_t)(gi[k].cellbase + f) : -1;
        warp_agg_inc(hist, cell, valid);
        // src/Interaction.jl:214-236 assumes the sort order makes cells
        // non-decreasing; count the places where it does not.
        int64_t fp = __shfl_up_sync(FULL, f, 1);
        int kp = __shfl_up_sync(FULL, k, 1);
        bool have = lane > 0;
        if (lane == 0 && valid && g > 0) {
            kp = inst_of[g - 1];
            have = kp == k && cell_flat(x, N, g - 1, nd, gi[k], &fp);
        }
        if (valid && have && kp == k && fp > f) {
            atomicAdd(incons, 1ull);
            atomicOr(err, ERR_GRID_INCONS);
        }
    }
}

__global__ void k_grid_count(const double* __restrict__ x, int64_t N, int nd, const int32_t* __restrict__ inst_of,
                             const int64_t* count, const GridInst* __restrict__ gi, int32_t* __restrict__ hist,
                             int64_t cells_cap, int* err, unsigned long long* incons, const int* skip) {
    pdl_enter();
    if (skip && *skip) return;
    grid_count_blocks(x, N, nd, inst_of, count, gi, hist, cells_cap, err, incons, blockIdx.x, gridDim.x);
}

void launch_grid_count(const double* x, int64_t N, int nd, const int32_t* inst_of, const int64_t* count,
                       const GridInst* gi, int32_t* hist, int64_t cells_cap, int* err, unsigned long long* incons,
                       cudaStream_t s, const int* skip) {
    if (N <= 0) return;
    k_grid_count<<<nblk(N), TPB, 0, s>>>(x, N, nd, inst_of, count, gi, hist, cells_cap, err, incons, skip);
    COUNTED(1);
}

// ------------------------------------------------ still grids, batched
// Every interaction whose system_b does not move recounts its CSR only when
// its grid's geometry changed (keep[1], set by the plan).  Their counts and
// scans run as one launch each over a table of interactions (blockIdx.y),
// with a few blocks per interaction striding over the work: on the usual
// step every block returns at once, and separate launches of one block per
// tile would cost more in launch latency than the work they skip.
int64_t still_hist_elems(int64_t cells) { return cells + (cells + SCAN_TILE - 1) / SCAN_TILE + 1; }

__global__ void k_still_count(const __grid_constant__ StillGridArgs a) {
    pdl_enter();
    const StillGrid& g = a.g[blockIdx.y];
    if (g.keep[1]) return;
    grid_count_blocks(g.x, g.N, a.nd, g.inst_of, nullptr, g.gi, g.hist, g.cells, a.err, a.incons, blockIdx.x,
                      gridDim.x);
}

// Tile sums of each histogram, after its cells.
__global__ void k_still_scan_reduce(const __grid_constant__ StillGridArgs a) {
    pdl_enter();
    const StillGrid& g = a.g[blockIdx.y];
    if (g.keep[1]) return;
    const int64_t nb = (g.cells + SCAN_TILE - 1) / SCAN_TILE;
    int32_t* bsum = g.hist + g.cells;
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const int64_t t0 = b * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
        int32_t s = 0;
#pragma unroll
        for (int k = 0; k < SCAN_I; ++k)
            if (t0 + k < g.cells) s += g.hist[t0 + k];
        int32_t total;
        (void)block_excl_scan(s, &total);
        if (threadIdx.x == 0) bsum[b] = total;
    }
}

// Exclusive scan of each histogram into its CSR (cells + 1 entries), the
// histogram cleared as it is read; each tile adds up the sums before it.
__global__ void k_still_scan_apply(const __grid_constant__ StillGridArgs a) {
    pdl_enter();
    const StillGrid& g = a.g[blockIdx.y];
    if (g.keep[1]) return;
    const int64_t n = g.cells;
    const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    const int32_t* bsum = g.hist + n;
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        int32_t off;
        {
            int32_t s = 0;
            for (int64_t t = threadIdx.x; t < b; t += blockDim.x) s += bsum[t];
            (void)block_excl_scan(s, &off);
        }
        const int64_t t0 = b * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
        int32_t v[SCAN_I];
        int32_t sum = 0;
#pragma unroll
        for (int k = 0; k < SCAN_I; ++k) {
            v[k] = t0 + k < n ? g.hist[t0 + k] : 0;
            sum += v[k];
        }
#pragma unroll
        for (int k = 0; k < SCAN_I; ++k)
            if (t0 + k < n) g.hist[t0 + k] = 0;
        int32_t total;
        int32_t run = block_excl_scan(sum, &total) + off;
#pragma unroll
        for (int k = 0; k < SCAN_I; ++k) {
            if (t0 + k < n) g.cs[t0 + k] = run;
            run += v[k];
        }
        if (b == nb - 1 && threadIdx.x == 0) g.cs[n] = off + total;
    }
}

void launch_still_grids(const StillGridArgs& a, cudaStream_t s) {
    if (a.n <= 0) return;
    int64_t maxN = 1, maxnb = 1;
    for (int i = 0; i < a.n; ++i) {
        maxN = std::max(maxN, a.g[i].N);
        maxnb = std::max(maxnb, (a.g[i].cells + SCAN_TILE - 1) / SCAN_TILE);
    }
    const unsigned bc = (unsigned)std::min<int64_t>(nblk(maxN), 2 * 148);
    const unsigned bs = (unsigned)std::min<int64_t>(maxnb, 148);
    k_still_count<<<dim3(bc, a.n), TPB, 0, s>>>(a);
    k_still_scan_reduce<<<dim3(bs, a.n), SCAN_T, 0, s>>>(a);
    k_still_scan_apply<<<dim3(bs, a.n), SCAN_T, 0, s>>>(a);
    COUNTED(3);
}

// ================================================================ ghosts
// src/GhostParticles.jl:344-392: a source particle within `cutoff` of a
// plane (0 < da <= cutoff) gets a mirror image; ghosts are ordered
// instance-major, then plane-major, then by source index.
template <int ND>
__device__ __forceinline__ double plane_da(const double* __restrict__ x, int64_t N, int64_t g, const double* pt,
                                           const double* nrm) {
    double t[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) t[d] = x[d * N + g] - pt[d];
    return dotv<ND>(t, nrm);
}

template <int ND>
__global__ void k_ghost_flags(GhostGenArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.Nsrc;
         g += (int64_t)gridDim.x * blockDim.x) {
        const GhostInst& H = a.gh[a.src_inst_of[g]];
        int64_t local = g - H.src_base;
        for (int b = 0; b < a.nplanes; ++b) {
            double da = plane_da<ND>(a.src_x, a.Nsrc, g, H.points[b], H.normals[b]);
            int64_t v = H.src_base * a.nplanes + b * H.src_n + local;
            a.flags[v] = (fabs(da) <= H.cutoff && da > 0.0) ? 1 : 0;
        }
    }
}

template <int ND>
__global__ void k_ghost_fill(GhostGenArgs a) {
    pdl_enter();
    const int64_t CAP = a.Nsrc * a.nplanes;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.Nsrc;
         g += (int64_t)gridDim.x * blockDim.x) {
        int k = a.src_inst_of[g];
        const GhostInst& H = a.gh[k];
        int64_t local = g - H.src_base;
        for (int b = 0; b < a.nplanes; ++b) {
            int64_t v = H.src_base * a.nplanes + b * H.src_n + local;
            if (!a.flags[v]) continue;
            double da = plane_da<ND>(a.src_x, a.Nsrc, g, H.points[b], H.normals[b]);
            int64_t p = a.pos[v];
            double s = 2.0 * da;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                a.gx[d * CAP + p] = a.src_x[d * a.Nsrc + g] - s * H.normals[b][d];
                a.gnormals[d * CAP + p] = H.normals[b][d];
            }
            a.gio[p] = (int32_t)(local + 1);
            a.gib[p] = b + 1;
            a.ginst[p] = k;
        }
    }
}

__global__ void k_ghost_ranges(GhostGenArgs a) {
    pdl_enter();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.ninst; k += gridDim.x * blockDim.x) {
        GhostInst& H = a.gh[k];
        int64_t v0 = H.src_base * a.nplanes, v1 = (H.src_base + H.src_n) * a.nplanes;
        H.base = a.pos[v0];
        H.n = a.pos[v1] - a.pos[v0];
        a.ginst_params[k].base = H.base;
        a.ginst_params[k].n = H.n;
        if (k == a.ninst - 1) *a.count = a.pos[a.Nsrc * a.nplanes];
    }
}

void launch_ghost_flags(const GhostGenArgs& a, cudaStream_t s) {
    if (a.nd == 2) k_ghost_flags<2><<<nblk(a.Nsrc), TPB, 0, s>>>(a);
    else k_ghost_flags<3><<<nblk(a.Nsrc), TPB, 0, s>>>(a);
    COUNTED(1);
}

void launch_ghost_fill(const GhostGenArgs& a, cudaStream_t s) {
    if (a.nd == 2) k_ghost_fill<2><<<nblk(a.Nsrc), TPB, 0, s>>>(a);
    else k_ghost_fill<3><<<nblk(a.Nsrc), TPB, 0, s>>>(a);
    k_ghost_ranges<<<nblk(a.ninst), TPB, 0, s>>>(a);
    COUNTED(2);
}

// src/GhostParticles.jl:404-421.  `normals` is read at the sorted position
// k: the reference's ghost sort does not permute the cached normals.
template <int ND>
__global__ void k_ghost_kin(int64_t cap, const int64_t* count, const int32_t* __restrict__ io,
                            const int32_t* __restrict__ ginst, const double* __restrict__ normals,
                            const GhostInst* __restrict__ gh, const double* __restrict__ src_v,
                            const double* __restrict__ src_rho, int64_t Nsrc, double* __restrict__ gv,
                            double* __restrict__ grho) {
    pdl_enter();
    int64_t n = *count;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = gh[ginst[k]].src_base + io[k] - 1;
        double nrm[ND], vr[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            nrm[d] = normals[d * cap + k];
            vr[d] = src_v[d * Nsrc + o];
        }
        double s = 2.0 * dotv<ND>(vr, nrm);
#pragma unroll
        for (int d = 0; d < ND; ++d) gv[d * cap + k] = vr[d] - s * nrm[d];
        grho[k] = src_rho[o];
    }
}

void launch_ghost_kinematics(int64_t cap, const int64_t* count, int nd, const int32_t* io, const int32_t* ginst,
                             const double* normals, const GhostInst* gh, const double* src_v, const double* src_rho,
                             int64_t Nsrc, double* gv, double* grho, cudaStream_t s) {
    if (cap <= 0) return;
    if (nd == 2) k_ghost_kin<2><<<nblk(cap), TPB, 0, s>>>(cap, count, io, ginst, normals, gh, src_v, src_rho, Nsrc, gv, grho);
    else k_ghost_kin<3><<<nblk(cap), TPB, 0, s>>>(cap, count, io, ginst, normals, gh, src_v, src_rho, Nsrc, gv, grho);
    COUNTED(1);
}

// src/GhostParticles.jl:66-129
__global__ void k_ghost_copy(int64_t cap, const int64_t* count, int nd, int ns, const int32_t* __restrict__ io,
                             const int32_t* __restrict__ ginst, const double* __restrict__ normals,
                             const GhostInst* __restrict__ gh, int field, int mode, const double* __restrict__ src,
                             int64_t Nsrc, double* __restrict__ dst) {
    pdl_enter();
    int64_t n = *count;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = gh[ginst[k]].src_base + io[k] - 1;
        if (field == GC_FIELD_P) {
            dst[k] = src[o];
            continue;
        }
        // loops over the compile-time bound keep sg and out in registers
        double sg[MAXS];
#pragma unroll
        for (int q = 0; q < MAXS; ++q) sg[q] = q < ns ? src[q * Nsrc + o] : 0.0;
        if (mode != GC_COPY_HOUSEHOLDER) {
#pragma unroll
            for (int q = 0; q < MAXS; ++q)
                if (q < ns) dst[q * cap + k] = sg[q];
            continue;
        }
        double out[MAXS];
        if (ns == 3 || ns == 4) {
            double nx = normals[k], ny = normals[cap + k];
            int xy = ns == 3 ? 2 : 3;
            double tx = sg[0] * nx + sg[xy] * ny;
            double ty = sg[xy] * nx + sg[1] * ny;
            double sc = tx * nx + ty * ny;
            out[0] = sg[0] - 4.0 * tx * nx + 4.0 * sc * nx * nx;
            out[1] = sg[1] - 4.0 * ty * ny + 4.0 * sc * ny * ny;
            if (ns == 4) out[2] = sg[2];
            out[xy] = sg[xy] - 2.0 * (tx * ny + nx * ty) + 4.0 * sc * nx * ny;
        } else {
            double nx = normals[k], ny = normals[cap + k], nz = normals[2 * cap + k];
            double tx = sg[0] * nx + sg[3] * ny + sg[4] * nz;
            double ty = sg[3] * nx + sg[1] * ny + sg[5] * nz;
            double tz = sg[4] * nx + sg[5] * ny + sg[2] * nz;
            double sc = tx * nx + ty * ny + tz * nz;
            out[0] = sg[0] - 4.0 * tx * nx + 4.0 * sc * nx * nx;
            out[1] = sg[1] - 4.0 * ty * ny + 4.0 * sc * ny * ny;
            out[2] = sg[2] - 4.0 * tz * nz + 4.0 * sc * nz * nz;
            out[3] = sg[3] - 2.0 * (tx * ny + nx * ty) + 4.0 * sc * nx * ny;
            out[4] = sg[4] - 2.0 * (tx * nz + nx * tz) + 4.0 * sc * nx * nz;
            out[5] = sg[5] - 2.0 * (ty * nz + ny * tz) + 4.0 * sc * ny * nz;
        }
#pragma unroll
        for (int q = 0; q < MAXS; ++q)
            if (q < ns) dst[q * cap + k] = out[q];
        (void)nd;
    }
}

void launch_ghost_copy(int64_t cap, const int64_t* count, int nd, int ns, const int32_t* io, const int32_t* ginst,
                       const double* normals, const GhostInst* gh, int field, int mode, const double* src,
                       int64_t Nsrc, double* dst, cudaStream_t s) {
    if (cap <= 0) return;
    k_ghost_copy<<<nblk(cap), TPB, 0, s>>>(cap, count, nd, ns, io, ginst, normals, gh, field, mode, src, Nsrc, dst);
    COUNTED(1);
}

// ============================================================ host I/O
// Julia's AoS layout (K doubles per particle) <-> planar device fields.
__global__ void k_aos_to_planar(const double* __restrict__ src, double* __restrict__ dst, int64_t n, int comps,
                                int64_t N, int64_t base) {
    pdl_enter();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * comps;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = t / comps;
        int c = (int)(t - i * comps);
        dst[c * N + base + i] = src[t];
    }
}
__global__ void k_planar_to_aos(const double* __restrict__ src, double* __restrict__ dst, int64_t n, int comps,
                                int64_t N, int64_t base) {
    pdl_enter();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * comps;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = t / comps;
        int c = (int)(t - i * comps);
        dst[t] = src[c * N + base + i];
    }
}
__global__ void k_i64_to_i32(const int64_t* __restrict__ src, int32_t* __restrict__ dst, int64_t n) {
    pdl_enter();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        dst[t] = (int32_t)src[t];
}
__global__ void k_i32_to_i64(const int32_t* __restrict__ src, int64_t* __restrict__ dst, int64_t n) {
    pdl_enter();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        dst[t] = (int64_t)src[t];
}

void launch_aos_to_planar(const double* src, double* dst, int64_t n, int comps, int64_t N, int64_t base,
                          cudaStream_t s) {
    if (n <= 0) return;
    int b = nblk(n * comps);
    if (b > 148 * 32) b = 148 * 32;
    k_aos_to_planar<<<b, TPB, 0, s>>>(src, dst, n, comps, N, base);
    COUNTED(1);
}
void launch_planar_to_aos(const double* src, double* dst, int64_t n, int comps, int64_t N, int64_t base,
                          cudaStream_t s) {
    if (n <= 0) return;
    int b = nblk(n * comps);
    if (b > 148 * 32) b = 148 * 32;
    k_planar_to_aos<<<b, TPB, 0, s>>>(src, dst, n, comps, N, base);
    COUNTED(1);
}
void launch_i64_to_i32(const int64_t* src, int32_t* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_i64_to_i32<<<nblk(n), TPB, 0, s>>>(src, dst, n);
    COUNTED(1);
}
void launch_i32_to_i64(const int32_t* src, int64_t* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_i32_to_i64<<<nblk(n), TPB, 0, s>>>(src, dst, n);
    COUNTED(1);
}

// ===================================================== measurement helpers
__global__ void k_sum_counts(const int32_t* __restrict__ c, int64_t n, unsigned long long* out) {
    pdl_enter();
    unsigned long long s = 0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        s += (unsigned long long)c[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}
void launch_sum_counts(const int32_t* c, int64_t n, unsigned long long* out, cudaStream_t s) {
    if (n <= 0) return;
    int b = nblk(n);
    if (b > 148 * 8) b = 148 * 8;
    k_sum_counts<<<b, TPB, 0, s>>>(c, n, out);
    COUNTED(1);
}

// FP64 FMA issue rate: eight independent dependent chains per thread.
__global__ void k_fp64_peak(double* out, int iters, double a, double b) {
    pdl_enter();
    double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
           x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b);
        x1 = fma(x1, a, b);
        x2 = fma(x2, a, b);
        x3 = fma(x3, a, b);
        x4 = fma(x4, a, b);
        x5 = fma(x5, a, b);
        x6 = fma(x6, a, b);
        x7 = fma(x7, a, b);
    }
    double r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (r == 12345.678) out[0] = r;  // keeps the chains live
}
void launch_fp64_peak(double* out, int blocks, int threads, int iters, cudaStream_t s) {
    k_fp64_peak<<<blocks, threads, 0, s>>>(out, iters, 0.9999999, 1e-9);
    COUNTED(1);
}

// FP32 FMA issue rate: eight independent dependent chains per thread.
__global__ void k_fp32_peak(float* out, int iters, float a, float b) {
    pdl_enter();
    float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
          x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fmaf(x0, a, b);
        x1 = fmaf(x1, a, b);
        x2 = fmaf(x2, a, b);
        x3 = fmaf(x3, a, b);
        x4 = fmaf(x4, a, b);
        x5 = fmaf(x5, a, b);
        x6 = fmaf(x6, a, b);
        x7 = fmaf(x7, a, b);
    }
    float r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (r == 12345.678f) out[0] = r;  // keeps the chains live
}
void launch_fp32_peak(float* out, int blocks, int threads, int iters, cudaStream_t s) {
    k_fp32_peak<<<blocks, threads, 0, s>>>(out, iters, 0.9999999f, 1e-9f);
    COUNTED(1);
}

}  // namespace gc
