// k_force_impl.cuh — the fused pair sweep in the reference's FP64 arithmetic.
//
// Gather formulation of src/Interaction.jl:393-732: one thread owns one
// system_a particle and sums its side of every accepted pair of every
// interaction of the current stage, in registers, then writes once.  The
// reference's coloured half-shell writes both endpoints; every functor on
// this path is exactly antisymmetric (or symmetric) under i↔j, so each
// side's term is bit-identical to the one the reference adds — only the
// order of the additions differs.
//
// Candidate enumeration walks the same 3-cell strips of the CSR grid as the
// reference (3 strips in 2-D, 9 in 3-D) and applies the same acceptance
// test r² < (2h)² on the same FP64 dx, so the neighbour sets are
// bit-identical.  Accepted neighbour indices are staged in a per-thread
// column of shared memory and processed in batches: the expensive pair
// physics runs with every lane busy instead of diverging on rejections.
//
// Compiled with -fmad=false (reference rounding).
#pragma once
#include <cstdio>

#include "gc_device.cuh"
#include "gc_force.h"
#include "gc_kernels.h"

namespace gc {

// psi / rho for psi == +0 (δ-SPH off): +0 for a positive density, and the
// literal quotient otherwise.
__device__ __forceinline__ double zero_over(double r) {
    if (r > 0.0) return 0.0;
    return 0.0 / r;
}

template <int ND>
struct OwnState {
    double x[ND], v[ND];
    double rho, aux;
};

// ------------------------------------------------------- pair physics
// One accepted pair (i owned, j neighbour), returns the i-side increment.
template <int ND, int NS, int PFN, int KK>
struct Pair {
    static __device__ __forceinline__ void geom(const double* dx, double rr, double H, double knorm, double* gx) {
        double r = sqrt(rr);
        double q = r / H;
        double gc = kernel_dw_dq<KK>(knorm, q) / (r * H);
#pragma unroll
        for (int d = 0; d < ND; ++d) gx[d] = gc * dx[d];
    }
};

template <int ND, int NS>
__device__ __forceinline__ void cauchy_f(const double* si, const double* sj, double ci, double cj, const double* g,
                                         double* out) {
    if (ND == 2) {
        constexpr int XY = NS == 3 ? 2 : 3;
        out[0] = (si[0] * g[0] + si[XY] * g[1]) * ci + (sj[0] * g[0] + sj[XY] * g[1]) * cj;
        out[1] = (si[XY] * g[0] + si[1] * g[1]) * ci + (sj[XY] * g[0] + sj[1] * g[1]) * cj;
    } else {
        out[0] = (si[0] * g[0] + si[3] * g[1] + si[4] * g[2]) * ci + (sj[0] * g[0] + sj[3] * g[1] + sj[4] * g[2]) * cj;
        out[1] = (si[3] * g[0] + si[1] * g[1] + si[5] * g[2]) * ci + (sj[3] * g[0] + sj[1] * g[1] + sj[5] * g[2]) * cj;
        out[2] = (si[4] * g[0] + si[5] * g[1] + si[2] * g[2]) * ci + (sj[4] * g[0] + sj[5] * g[1] + sj[2] * g[2]) * cj;
    }
}

template <int ND, int NS>
__device__ __forceinline__ void strain_rate_f(const double* dv, const double* g, double* sr) {
    if (ND == 2) {
        sr[0] = dv[0] * g[0];
        sr[1] = dv[1] * g[1];
        if (NS == 4) {
            sr[2] = 0.0;
            sr[3] = 0.5 * (dv[0] * g[1] + dv[1] * g[0]);
        } else {
            sr[2] = 0.5 * (dv[0] * g[1] + dv[1] * g[0]);
        }
    } else {
        sr[0] = dv[0] * g[0];
        sr[1] = dv[1] * g[1];
        sr[2] = dv[2] * g[2];
        sr[3] = 0.5 * (dv[0] * g[1] + dv[1] * g[0]);
        sr[4] = 0.5 * (dv[0] * g[2] + dv[2] * g[0]);
        sr[5] = 0.5 * (dv[1] * g[2] + dv[2] * g[1]);
    }
}

template <int ND>
__device__ __forceinline__ void vorticity_f(const double* dv, const double* g, double* w) {
    w[0] = 0.5 * (dv[0] * g[1] - dv[1] * g[0]);
    if (ND == 3) {
        w[1] = 0.5 * (dv[0] * g[2] - dv[2] * g[0]);
        w[2] = 0.5 * (dv[1] * g[2] - dv[2] * g[1]);
    }
}

template <int ND, int NS>
struct Acc {
    double dv[ND];
    double dr;
    double sr[NS > 0 ? NS : 1];
    double w[ND == 2 ? 1 : 3];
};

// One staged candidate j of reference r for owned particle i: the exact
// reference test r² < (2h)² (src/Interaction.jl:546-548) on the FP64
// positions, then the functor's i-side term.  Returns 1 when accepted.
template <int ND, int NS, int PFN, int KK>
__device__ __forceinline__ int process_pair(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                            const PfnInst& P, int64_t gi, int k, const OwnState<ND>& o,
                                            const double* osig, double da, int32_t j, Acc<ND, NS>& acc) {
    const int64_t Nb = r.bN;
    double dx[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) dx[d] = o.x[d] - r.bx[d * Nb + j];
    double rr = dotv<ND>(dx, dx);
    if (!(rr < G.cutoff_sq)) return 0;
    if (PFN == GC_PFN_COUNT) {
        acc.dv[0] += 1.0;
        acc.dr += 1.0;
        return 1;
    }
    double gx[ND];
    Pair<ND, NS, PFN, KK>::geom(dx, rr, G.H, G.knorm, gx);
    const double ca = A.a_c[k];
    const double mass_a = A.a_mass[k];

    if (r.btype == BT_DYNAMIC) {
        // src/PairwiseFunctors.jl:53,111,222,334
        double t[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) t[d] = r.bx[d * Nb + j] - G.point[d];
        double db = dotv<ND>(t, G.normal);
        double m = -jmin(G.beta, fabs(db / da));
        double vj[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) vj[d] = m * o.v[d];
        if (PFN == GC_PFN_FLUID || PFN == GC_PFN_CAUCHY_FLUID) {
            double dv[ND];
#pragma unroll
            for (int d = 0; d < ND; ++d) dv[d] = o.v[d] - vj[d];
            double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, o.rho, P.alpha, P.beta, ca, ca);
            if (PFN == GC_PFN_FLUID) {
                double dh = P.S == 1 ? -(A.a_p[gi] + A.a_p[gi]) / (o.rho * o.rho) : -(o.aux + o.aux);
                double s = mass_a * (dh - piv);
#pragma unroll
                for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + s * gx[d];
            } else {
                double hv[ND];
                cauchy_f<ND, NS>(osig, osig, o.aux, o.aux, gx, hv);
#pragma unroll
                for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + mass_a * (hv[d] - piv * gx[d]);
            }
            double dr = dotv<ND>(dv, gx);
            double tail;
            if (P.has_delta) {
                double psi = diffusion<ND>(dx, rr, o.rho, o.rho, ca, ca, P.h, P.h, gx, P.delta);
                tail = psi / o.rho;
            } else {
                tail = zero_over(o.rho);
            }
            double cdc = (PFN == GC_PFN_FLUID && P.S == 1) ? o.rho / o.rho : 1.0;
            acc.dr = acc.dr + mass_a * ((PFN == GC_PFN_FLUID ? dr * cdc : dr) + tail);
        } else {  // strain rate (+ vorticity)
            double dv[ND];
#pragma unroll
            for (int d = 0; d < ND; ++d) dv[d] = vj[d] - o.v[d];
            double sr[NS > 0 ? NS : 1];
            strain_rate_f<ND, NS>(dv, gx, sr);
            const double f = o.aux;  // mass_a / rho_i
#pragma unroll
            for (int q = 0; q < NS; ++q) acc.sr[q] = acc.sr[q] + sr[q] * f;
            if (PFN == GC_PFN_STRAIN_RATE_VORTICITY) {
                double w[ND == 2 ? 1 : 3];
                vorticity_f<ND>(dv, gx, w);
#pragma unroll
                for (int q = 0; q < (ND == 2 ? 1 : 3); ++q) acc.w[q] = acc.w[q] + w[q] * f;
            }
        }
        return 1;
    }

    // neighbour state
    double vj[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) vj[d] = r.bv[d * Nb + j];
    const double rhoj = r.brho[j];

    if (r.btype == BT_STATIC && (PFN == GC_PFN_FLUID || PFN == GC_PFN_CAUCHY_FLUID)) {
        // src/PairwiseFunctors.jl:210-219, :322-331
        double dv[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dv[d] = o.v[d] - vj[d];
        double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, rhoj, P.alpha, P.beta, ca, ca);
        double rf = lennard_jones<ND>(dx, rr, G.ljcut, ca);
        double s = (-G.bmass) * piv;
#pragma unroll
        for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + (s * gx[d] + rf * dx[d]);
        return 1;
    }

    if (PFN == GC_PFN_FLUID) {
        double dv[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dv[d] = o.v[d] - vj[d];
        double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, rhoj, P.alpha, P.beta, ca, ca);
        double auxj = r.baux[j];
        double dh = P.S == 1 ? -(A.a_p[gi] + r.bp[j]) / (o.rho * rhoj) : -(o.aux + auxj);
        double mj = r.btype == BT_SELF ? mass_a : G.bmass;
        double s = mj * (dh - piv);
#pragma unroll
        for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + s * gx[d];
        double dr = dotv<ND>(dv, gx);
        double tail;
        if (P.has_delta) {
            double psi = diffusion<ND>(dx, rr, o.rho, rhoj, ca, ca, P.h, P.h, gx, P.delta);
            tail = psi / rhoj;
        } else {
            tail = zero_over(rhoj);
        }
        double cdc = P.S == 1 ? o.rho / rhoj : 1.0;
        acc.dr = acc.dr + mj * (dr * cdc + tail);
    } else if (PFN == GC_PFN_CAUCHY_FLUID) {
        // self :265 / ghost one-sided :286
        double dv[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dv[d] = o.v[d] - vj[d];
        const bool self = r.btype == BT_SELF;
        double cb = self ? ca : G.bc;
        double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, rhoj, P.alpha, P.beta, ca, cb);
        double sj[NS > 0 ? NS : 1];
#pragma unroll
        for (int q = 0; q < NS; ++q) sj[q] = r.bstress[q * Nb + j];
        double hv[ND];
        cauchy_f<ND, NS>(osig, sj, o.aux, r.baux[j], gx, hv);
        double mj = self ? mass_a : G.bmass;
#pragma unroll
        for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + mj * (hv[d] - piv * gx[d]);
        double dr = dotv<ND>(dv, gx);
        double tail;
        if (P.has_delta) {
            double psi = diffusion<ND>(dx, rr, o.rho, rhoj, ca, ca, P.h, P.h, gx, P.delta);
            tail = psi / rhoj;
        } else {
            tail = zero_over(rhoj);
        }
        acc.dr = acc.dr + mj * (dr + tail);
    } else {
        // strain rate (+vorticity): self :20/:80, generic one-sided :37/:97
        double dv[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dv[d] = vj[d] - o.v[d];
        double sr[NS > 0 ? NS : 1];
        strain_rate_f<ND, NS>(dv, gx, sr);
        const double f = r.baux[j];  // mass_j / rho_j
#pragma unroll
        for (int q = 0; q < NS; ++q) acc.sr[q] = acc.sr[q] + sr[q] * f;
        if (PFN == GC_PFN_STRAIN_RATE_VORTICITY) {
            double w[ND == 2 ? 1 : 3];
            vorticity_f<ND>(dv, gx, w);
#pragma unroll
            for (int q = 0; q < (ND == 2 ? 1 : 3); ++q) acc.w[q] = acc.w[q] + w[q] * f;
        }
    }
    (void)gi;
    return 1;
}

// ---------------------------------------------------------------- kernel
// One warp owns one group: up to 32 consecutive (sorted) system_a particles
// of one grid column (all cell coordinates but the last equal).  For each
// 3-cell strip of the reference stencil the warp walks the union of its
// lanes' candidate ranges — contiguous in the CSR because cells along the
// last dimension are consecutive — loading 32 candidates at a time with one
// coalesced load and broadcasting them by shuffles.  A lane accepts a
// candidate only inside its own strip range [cs[z-1], cs[z+2]) and with
// r² < (2h)², which is exactly the reference's pair test.  Accepted indices
// go to the lane's shared-memory column; when any lane's column is nearly
// full the whole warp evaluates its staged pairs, so the FP64 pair physics
// runs on converged warps.
template <int ND, int NS, int PFN, int KK, bool COUNT_ONLY, int UNROLL>
__device__ __forceinline__ int flush_all(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                         const PfnInst& P, int64_t gi, int k, const OwnState<ND>& o,
                                         const double* osig, double da, int nbuf, const int32_t* col, int BT,
                                         Acc<ND, NS>& acc) {
    int acc_n = 0;
    int t = 0;
    if (UNROLL == 2) {
        // two independent pair evaluations in flight; their sums enter acc in order
        for (; t + 1 < nbuf; t += 2) {
            const int32_t j0 = col[t * BT], j1 = col[(t + 1) * BT];
            acc_n += process_pair<ND, NS, (COUNT_ONLY ? GC_PFN_COUNT : PFN), KK>(A, r, G, P, gi, k, o, osig, da, j0, acc);
            acc_n += process_pair<ND, NS, (COUNT_ONLY ? GC_PFN_COUNT : PFN), KK>(A, r, G, P, gi, k, o, osig, da, j1, acc);
        }
    }
    for (; t < nbuf; ++t)
        acc_n += process_pair<ND, NS, (COUNT_ONLY ? GC_PFN_COUNT : PFN), KK>(A, r, G, P, gi, k, o, osig, da,
                                                                            col[t * BT], acc);
    return acc_n;
}

template <int ND, int NS, int PFN, int KK, bool COUNT_ONLY, int MINB, int BUF, int UNROLL>
__global__ void __launch_bounds__(FORCE_TPB, MINB) k_force(ForceArgs A) {
    extern __shared__ int32_t sbuf[];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x;
    const int BT = blockDim.x;
    int32_t* col = sbuf + tid;
    const int64_t ngroups = *A.ngroups;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t N = A.aN;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ngroups; w += nwarps) {
        const int2 grp = A.groups[w];
        const bool active = lane < grp.y;
        const int64_t gi = (int64_t)grp.x + (active ? lane : 0);
        const int k = A.a_inst_of[gi];

        OwnState<ND> o;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            o.x[d] = A.ax[d * N + gi];
            o.v[d] = A.av[d * N + gi];
        }
        o.rho = A.arho[gi];
        o.aux = A.aaux ? A.aaux[gi] : 0.0;
        double osig[NS > 0 ? NS : 1];
#pragma unroll
        for (int q = 0; q < NS; ++q) osig[q] = (PFN == GC_PFN_CAUCHY_FLUID) ? A.astress[q * N + gi] : 0.0;

        Acc<ND, NS> acc;
#pragma unroll
        for (int d = 0; d < ND; ++d) acc.dv[d] = 0.0;
        acc.dr = 0.0;
        if (!COUNT_ONLY) {
            if (PFN == GC_PFN_FLUID || PFN == GC_PFN_CAUCHY_FLUID || PFN == GC_PFN_COUNT) {
#pragma unroll
                for (int d = 0; d < ND; ++d) acc.dv[d] = A.advdt[d * N + gi];
                acc.dr = A.adrhodt[gi];
            } else {
#pragma unroll
                for (int q = 0; q < NS; ++q) acc.sr[q] = A.asr[q * N + gi];
                if (PFN == GC_PFN_STRAIN_RATE_VORTICITY) {
#pragma unroll
                    for (int q = 0; q < (ND == 2 ? 1 : 3); ++q) acc.w[q] = A.avort[q * N + gi];
                }
            }
        }

        for (int ri = 0; ri < A.nref; ++ri) {
            const InterRef& r = A.ref[ri];
            const GridInst& G = r.gi[k];
            const PfnInst& P = r.pi[k];
            if (r.bbox) {
                // No system_b particle can be within the cutoff of any lane:
                // skip (the box test has a 0.1% margin, so no pair is lost).
                const SysInst& B = r.bbox[k];
                bool near = B.n > 0;
                const double m = 1.001 * G.cell;
#pragma unroll
                for (int d = 0; d < ND; ++d) near = near && o.x[d] >= B.bbmin[d] - m && o.x[d] <= B.bbmax[d] + m;
                if (!__any_sync(FULL, active && near)) {
                    if (active && r.counts) r.counts[gi] = 0;
                    continue;
                }
            }
            int64_t c[ND];
            bool ok = true;
#pragma unroll
            for (int d = 0; d < ND; ++d)
                if (!floor_i64((o.x[d] - G.ming[d]) / G.cell, &c[d]) || c[d] < 1 || c[d] >= G.ng[d] - 1) ok = false;
            if (active && !ok) atomicOr(A.err, ERR_CAPACITY);
            double da = 0.0;
            if (r.btype == BT_DYNAMIC) {
                double t[ND];
#pragma unroll
                for (int d = 0; d < ND; ++d) t[d] = o.x[d] - G.point[d];
                da = dotv<ND>(t, G.normal);
            }
            const int64_t Nb = r.bN;
            const bool self = r.btype == BT_SELF;
            int nbuf = 0;
            int32_t accepted = 0;
            // column of lane 0; the cooperative walk needs every active lane in it
            int64_t c0 = __shfl_sync(FULL, c[0], 0);
            int64_t c1 = ND == 3 ? __shfl_sync(FULL, c[1], 0) : 0;
            bool same = ok && c[0] == c0 && (ND == 2 || c[1] == c1);
            const bool coop = __all_sync(FULL, !active || same);
            if (coop) {
                constexpr int L = ND - 1;  // last dimension
                int64_t zlo = active ? c[L] : INT64_MAX, zhi = active ? c[L] : INT64_MIN;
#pragma unroll
                for (int o2 = 16; o2 > 0; o2 >>= 1) {
                    int64_t a2 = __shfl_xor_sync(FULL, zlo, o2), b2 = __shfl_xor_sync(FULL, zhi, o2);
                    zlo = a2 < zlo ? a2 : zlo;
                    zhi = b2 > zhi ? b2 : zhi;
                }
                // Conservative FP32 prefilter in coordinates relative to lane 0:
                // |rel| spans a few cells, so single-precision rounding moves r²
                // by < 1e-5 relative; the 1e-3 margin keeps every true pair.
                double xref[ND];
                float xi_f[ND];
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    xref[d] = __shfl_sync(FULL, o.x[d], 0);
                    xi_f[d] = (float)(o.x[d] - xref[d]);
                }
                const float cut_f = (float)(G.cutoff_sq * 1.001);
                const int64_t ngl = G.ng[L];
                const int nstrips = ND == 2 ? 3 : 9;
                for (int sidx = 0; sidx < nstrips; ++sidx) {
                    int64_t colflat;
                    if (ND == 2) colflat = c0 + sidx - 1;
                    else colflat = (c0 + sidx / 3 - 1) * G.ng[1] + (c1 + sidx % 3 - 1);
                    const int64_t base = G.cellbase + colflat * ngl;
                    const int32_t u0 = r.cs[base + zlo - 1], u1 = r.cs[base + zhi + 2];
                    const int32_t lo = r.cs[base + c[L] - 1], hi = r.cs[base + c[L] + 2];
                    for (int32_t ch = u0; ch < u1; ch += 32) {
                        if (__any_sync(FULL, nbuf > BUF - 32)) {
                            accepted += flush_all<ND, NS, PFN, KK, COUNT_ONLY, UNROLL>(A, r, G, P, gi, k, o, osig, da,
                                                                                      nbuf, col, BT, acc);
                            nbuf = 0;
                            __syncwarp();
                        }
                        const int32_t jl = ch + lane;
                        float xj[ND];
#pragma unroll
                        for (int d = 0; d < ND; ++d) xj[d] = jl < u1 ? (float)(r.bx[d * Nb + jl] - xref[d]) : 0.0f;
                        const int m = u1 - ch < 32 ? (int)(u1 - ch) : 32;
                        for (int t = 0; t < m; ++t) {
                            float rr = 0.0f;
#pragma unroll
                            for (int d = 0; d < ND; ++d) {
                                float dd = xi_f[d] - __shfl_sync(FULL, xj[d], t);
                                rr += dd * dd;
                            }
                            const int32_t jt = ch + t;
                            if (active && jt >= lo && jt < hi && !(self && jt == gi) && rr < cut_f)
                                col[(nbuf++) * BT] = jt;
                        }
                    }
                }
                accepted += flush_all<ND, NS, PFN, KK, COUNT_ONLY, UNROLL>(A, r, G, P, gi, k, o, osig, da, nbuf,
                                                                          col, BT, acc);
                nbuf = 0;
                __syncwarp();
            } else if (active && ok) {
                // rare: lanes disagree on the column in this grid; walk own strips
                const int nstrips = ND == 2 ? 3 : 9;
                for (int sidx = 0; sidx < nstrips; ++sidx) {
                    int64_t base;
                    if (ND == 2) base = G.cellbase + (c[0] + sidx - 1) * G.ng[1] + (c[1] - 1);
                    else base = G.cellbase + ((c[0] + sidx / 3 - 1) * G.ng[1] + (c[1] + sidx % 3 - 1)) * G.ng[2] + (c[2] - 1);
                    const int32_t s0 = r.cs[base], e0 = r.cs[base + 3];
                    for (int32_t j = s0; j < e0; ++j) {
                        if (self && j == gi) continue;
                        col[(nbuf++) * BT] = j;
                        if (nbuf == BUF) {
                            accepted += flush_all<ND, NS, PFN, KK, COUNT_ONLY, UNROLL>(A, r, G, P, gi, k, o, osig, da,
                                                                                      nbuf, col, BT, acc);
                            nbuf = 0;
                        }
                    }
                }
                accepted += flush_all<ND, NS, PFN, KK, COUNT_ONLY, UNROLL>(A, r, G, P, gi, k, o, osig, da, nbuf, col,
                                                                          BT, acc);
                nbuf = 0;
            }
            __syncwarp();
            if (active && r.counts) r.counts[gi] = accepted;
        }

        if (!COUNT_ONLY && active) {
            if (PFN == GC_PFN_FLUID || PFN == GC_PFN_CAUCHY_FLUID || PFN == GC_PFN_COUNT) {
#pragma unroll
                for (int d = 0; d < ND; ++d) A.advdt[d * N + gi] = acc.dv[d];
                A.adrhodt[gi] = acc.dr;
            } else {
#pragma unroll
                for (int q = 0; q < NS; ++q) A.asr[q * N + gi] = acc.sr[q];
                if (PFN == GC_PFN_STRAIN_RATE_VORTICITY) {
#pragma unroll
                    for (int q = 0; q < (ND == 2 ? 1 : 3); ++q) A.avort[q * N + gi] = acc.w[q];
                }
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ dispatch
template <int ND, int NS, int PFN, int KK, int C>
static void launch_c(const ForceArgs& A, cudaStream_t s) {
    constexpr ForceCfg cf = FORCE_CFGS[C];
    int64_t warps = A.aN;
    int64_t blocks = (warps * 32 + FORCE_TPB - 1) / FORCE_TPB;
    if (blocks > (int64_t)A.num_sms * cf.minb * 4) blocks = (int64_t)A.num_sms * cf.minb * 4;
    if (blocks < 1) blocks = 1;
    size_t smem = (size_t)cf.buf * FORCE_TPB * sizeof(int32_t);
    k_force<ND, NS, PFN, KK, false, cf.minb, cf.buf, cf.unroll><<<(int)blocks, FORCE_TPB, smem, s>>>(A);
}

template <int ND, int NS, int PFN, int KK>
static void launch_t(const ForceArgs& A, bool count_only, cudaStream_t s) {
    // grid-stride over groups; at most one group per particle
    if (count_only) {
        int64_t blocks = (A.aN * 32 + FORCE_TPB - 1) / FORCE_TPB;
        if (blocks > (int64_t)A.num_sms * 16) blocks = (int64_t)A.num_sms * 16;
        if (blocks < 1) blocks = 1;
        size_t smem = (size_t)FORCE_BUF * FORCE_TPB * sizeof(int32_t);
        k_force<ND, NS, PFN, KK, true, 4, FORCE_BUF, 1><<<(int)blocks, FORCE_TPB, smem, s>>>(A);
    } else if (KK != GC_KERNEL_CUBIC_SPLINE || PFN == GC_PFN_COUNT) {
        launch_c<ND, NS, PFN, KK, 0>(A, s);
    } else {
        switch (A.cfg) {
            case 1: launch_c<ND, NS, PFN, KK, 1>(A, s); break;
            case 2: launch_c<ND, NS, PFN, KK, 2>(A, s); break;
            case 3: launch_c<ND, NS, PFN, KK, 3>(A, s); break;
            default: launch_c<ND, NS, PFN, KK, 0>(A, s); break;
        }
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

template <int ND, int NS, int KK>
static int launch_pfn(const ForceArgs& A, bool count_only, cudaStream_t s) {
    switch (A.pfn) {
        case GC_PFN_FLUID: launch_t<ND, NS, GC_PFN_FLUID, KK>(A, count_only, s); return 0;
        case GC_PFN_COUNT: launch_t<ND, NS, GC_PFN_COUNT, KK>(A, count_only, s); return 0;
        case GC_PFN_CAUCHY_FLUID:
            if (NS == 0) return GC_ERR_UNSUPPORTED;
            launch_t<ND, NS, GC_PFN_CAUCHY_FLUID, KK>(A, count_only, s);
            return 0;
        case GC_PFN_STRAIN_RATE:
            if (NS == 0) return GC_ERR_UNSUPPORTED;
            launch_t<ND, NS, GC_PFN_STRAIN_RATE, KK>(A, count_only, s);
            return 0;
        case GC_PFN_STRAIN_RATE_VORTICITY:
            if (NS == 0) return GC_ERR_UNSUPPORTED;
            launch_t<ND, NS, GC_PFN_STRAIN_RATE_VORTICITY, KK>(A, count_only, s);
            return 0;
    }
    return GC_ERR_UNSUPPORTED;
}

template <int ND, int KK>
static int launch_nd(const ForceArgs& A, bool count_only, cudaStream_t s) {
    const bool stress_pfn = A.pfn == GC_PFN_CAUCHY_FLUID || A.pfn == GC_PFN_STRAIN_RATE ||
                            A.pfn == GC_PFN_STRAIN_RATE_VORTICITY;
    if (!stress_pfn) return launch_pfn<ND, 0, KK>(A, count_only, s);
    if (ND == 2) {
        if (A.ns == 3) return launch_pfn<ND, 3, KK>(A, count_only, s);
        if (A.ns == 4) return launch_pfn<ND, 4, KK>(A, count_only, s);
        return GC_ERR_UNSUPPORTED;
    }
    if (A.ns == 6) return launch_pfn<ND, 6, KK>(A, count_only, s);
    return GC_ERR_UNSUPPORTED;
}

}  // namespace gc
