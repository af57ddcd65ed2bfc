// k_noalloc.cu — the stable cell-key sort permutation without any device
// allocation, for callers that cannot call cudaMalloc: hosts whose device
// memory is handed in full to their own pool allocator (where a stray
// cudaMalloc can fail or fragment the pool), and latency-critical loops in
// which the implicit device synchronisation of cudaMalloc/cudaFree is not
// acceptable.
//
// All scratch (keys, cell histogram, cell starts, per-cell fill counters,
// scan blocks, the bounding box and an error word) lives in one file-scope
// `__device__` array of fixed size, so the limits below are hard limits.
// Every GPU that loads the library holds this array until the process exits.
// Calls share it and it keeps the last call's contents: each call clears the
// parts that must start at zero, and calls that overlap on the GPU (two
// streams, or two host threads) race on it.
//
// Host code only ever sees a stand-in for the array's name; every call
// resolves the array's device address with cudaGetSymbolAddress (which
// allocates nothing) on the caller's current device, so the address is
// right for the device and context of that call, also after a
// cudaDeviceReset has re-created the context.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "gc_kernels.h"

namespace gc {
namespace {

constexpr int64_t NA_MAX_N = 1 << 16;      // particles per call
constexpr int64_t NA_MAX_CELLS = 1 << 17;  // cells of the key lattice's bounding box

// scratch layout in 32-bit words
constexpr int64_t NA_KEY = 0;                                  // int32[MAX_N]
constexpr int64_t NA_INST = NA_KEY + NA_MAX_N;                 // int32[MAX_N] (all zero: one instance)
constexpr int64_t NA_HIST = NA_INST + NA_MAX_N;                // int32[MAX_CELLS+1]
constexpr int64_t NA_START = NA_HIST + NA_MAX_CELLS + 1;       // int32[MAX_CELLS+1]
constexpr int64_t NA_FILL = NA_START + NA_MAX_CELLS + 1;       // int32[MAX_CELLS+1]
constexpr int64_t NA_SCAN = NA_FILL + NA_MAX_CELLS + 1;        // scan blocks
constexpr int64_t NA_SCAN_WORDS = 1024;                        // ≥ scan_tmp_elems(MAX_CELLS)
constexpr int64_t NA_TAIL = (NA_SCAN + NA_SCAN_WORDS + 63) / 64 * 64;  // 256-byte aligned tail
// tail (in bytes from NA_TAIL*4): SysInst, bbox ull[2*MAXD], int64 cells, int err
constexpr int64_t NA_TAIL_BYTES = 1024;
constexpr int64_t NA_WORDS = NA_TAIL + NA_TAIL_BYTES / 4;

__device__ __align__(256) int32_t g_noalloc_scratch[NA_WORDS];

__global__ void k_na_init(SysInst* S, int64_t n, double cutoff, int64_t* cells, int* err) {
    pdl_enter();
    SysInst s{};
    s.base = 0;
    s.n = n;
    s.sort_cutoff = cutoff;
    *S = s;
    *cells = 0;
    *err = 0;
}

}  // namespace
}  // namespace gc

extern "C" int gc_cell_sort_perm_noalloc(const double* x_planar, int64_t n, int ndims, double cutoff,
                                         int32_t* perm_out, void* stream) {
    using namespace gc;
    if (n < 0 || n > NA_MAX_N) return GC_ERR_CAPACITY;  // at most 65536 particles per call
    if (ndims < 2 || ndims > 3 || !(cutoff > 0.0) || !std::isfinite(cutoff)) return GC_ERR_ARG;
    if (n > 0 && (!x_planar || !perm_out)) return GC_ERR_ARG;
    if (n == 0) return GC_OK;
    // the scratch array's address on the current device
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return GC_ERR_CUDA;
    if (scan_tmp_elems(NA_MAX_CELLS) > NA_SCAN_WORDS) return GC_ERR_CAPACITY;
    cudaStream_t s = (cudaStream_t)stream;
    int32_t* base = (int32_t*)addr;
    int32_t* key = base + NA_KEY;
    int32_t* inst_of = base + NA_INST;
    int32_t* hist = base + NA_HIST;
    int32_t* start = base + NA_START;
    int32_t* fill = base + NA_FILL;
    int32_t* scan = base + NA_SCAN;
    char* tail = (char*)(base + NA_TAIL);
    SysInst* S = (SysInst*)tail;
    unsigned long long* bbox = (unsigned long long*)(tail + ((sizeof(SysInst) + 15) / 16) * 16);
    int64_t* cells = (int64_t*)(bbox + 2 * MAXD);
    int* err = (int*)(cells + 1);

    k_na_init<<<1, 1, 0, s>>>(S, n, cutoff, cells, err);
    if (cudaMemsetAsync(inst_of, 0, n * sizeof(int32_t), s) != cudaSuccess) return GC_ERR_CUDA;
    if (cudaMemsetAsync(hist, 0, (NA_MAX_CELLS + 1) * sizeof(int32_t), s) != cudaSuccess) return GC_ERR_CUDA;
    if (cudaMemsetAsync(fill, 0, (NA_MAX_CELLS + 1) * sizeof(int32_t), s) != cudaSuccess) return GC_ERR_CUDA;
    launch_bbox(x_planar, n, ndims, inst_of, nullptr, S, bbox, 1, err, s);
    launch_sort_plan(S, 1, ndims, cells, err, s);
    launch_sort_keys(x_planar, n, ndims, inst_of, nullptr, S, key, hist, NA_MAX_CELLS, err, s);
    scan_exclusive(hist, start, NA_MAX_CELLS, scan, s);
    launch_sort_scatter(key, n, nullptr, start, fill, perm_out, s);
    launch_sort_fixup(start, NA_MAX_CELLS, cells, perm_out, s);
    if (cudaGetLastError() != cudaSuccess) return GC_ERR_CUDA;
    int h_err = 0;
    if (cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return GC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return GC_ERR_CUDA;
    if (h_err & ERR_NONFINITE) return GC_ERR_NONFINITE;
    if (h_err & ERR_CAPACITY) return GC_ERR_CAPACITY;  // key lattice beyond 131072 cells
    return GC_OK;
}
