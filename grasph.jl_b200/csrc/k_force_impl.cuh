// k_force_impl.cuh — the fused pair sweep (FP64 reference arithmetic and FP32-compensated).
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
// The FP64 policy relies on -fmad=false; the FP32 policy uses explicit
// __dmul_rn/__dadd_rn for the exact acceptance test.
#pragma once
#include <type_traits>
#include <cstdio>
#include <cuda_pipeline.h>

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

// Neighbour j's FP64 state, read from system_b's planar arrays ...
struct NbGlobal {
    const InterRef& r;
    int64_t j;
    __device__ __forceinline__ double x(int d) const { return r.bx[d * r.bN + j]; }
    __device__ __forceinline__ double v(int d) const { return r.bv[d * r.bN + j]; }
    __device__ __forceinline__ double rho() const { return r.brho[j]; }
    __device__ __forceinline__ double aux() const { return r.baux[j]; }
    __device__ __forceinline__ double p() const { return r.bp[j]; }
    __device__ __forceinline__ double stress(int q) const { return r.bstress[q * r.bN + j]; }
};

// ... or from its copy staged in shared memory by PhysF64::issue: 16-byte
// chunks q*BT of the slot, the position's components in pairs, then
// [v, ρ, aux, p] in pairs (the functors staged there read no stress).
template <int ND>
struct NbSlot {
    static constexpr int XQ = (ND + 1) / 2;
    const float4* slot;
    int BT;
    __device__ __forceinline__ double x(int d) const {
        return reinterpret_cast<const double*>(&slot[(d >> 1) * BT])[d & 1];
    }
    __device__ __forceinline__ double rec(int e) const {
        return reinterpret_cast<const double*>(&slot[(XQ + (e >> 1)) * BT])[e & 1];
    }
    __device__ __forceinline__ double v(int d) const { return rec(d); }
    __device__ __forceinline__ double rho() const { return rec(ND); }
    __device__ __forceinline__ double aux() const { return rec(ND + 1); }
    __device__ __forceinline__ double p() const { return rec(ND + 2); }
    __device__ __forceinline__ double stress(int) const { return 0.0; }
};

// One candidate j (source nb) of reference r for owned particle i: the
// exact reference test r² < (2h)² (src/Interaction.jl:546-548) on the FP64
// positions, then the functor's i-side term.  Returns 1 when accepted.
// BTK: the system_b kind when known at compile time (-1: r.btype).
template <int ND, int NS, int PFN, int KK, int BTK = -1, class Nb>
__device__ __forceinline__ int process_pair(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                            const PfnInst& P, int64_t gi, int k, const OwnState<ND>& o,
                                            const double* osig, double da, const Nb& nb, Acc<ND, NS>& acc,
                                            const double2* cam = nullptr) {
    // system_a's sound speed and mass: the warp's shared copy (cam) or the
    // per-instance arrays
    auto sound_a = [&]() { return cam ? cam->x : A.a_c[k]; };
    auto mass_of_a = [&]() { return cam ? cam->y : A.a_mass[k]; };
    const int btype = BTK >= 0 ? BTK : r.btype;
    double dx[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) dx[d] = o.x[d] - nb.x(d);
    double rr = dotv<ND>(dx, dx);
    if (!(rr < G.cutoff_sq)) return 0;
    if (PFN == GC_PFN_COUNT) {
        acc.dv[0] += 1.0;
        acc.dr += 1.0;
        return 1;
    }
    if (PFN == GC_PFN_INTERPOLATE) {
        // InterpolateFieldFn(ps_a, ps_b::VirtualParticleSystem)
        // src/PairwiseFunctors.jl:424-428 from the virtual particle's side:
        // kw = w·(m_a/ρ_a[i]); f[j] += kw·f_a[i]; w_sum[j] += kw
        const double q = sqrt(rr) / G.H;
        const double kw = kernel_w<KK>(G.knorm, q) * (G.bmass / nb.rho());
        if (A.imask & (1 << GC_FIELD_V)) {
#pragma unroll
            for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + kw * nb.v(d);
        }
        if (A.imask & (1 << GC_FIELD_RHO)) acc.dr = acc.dr + kw * nb.rho();
        if (A.imask & (1 << GC_FIELD_STRESS)) {
#pragma unroll
            for (int q2 = 0; q2 < NS; ++q2) acc.sr[q2] = acc.sr[q2] + kw * nb.stress(q2);
        }
        if (A.iwsum) acc.w[0] = acc.w[0] + (A.iwsum == 2 ? 1.0 : kw);  // 2: NeighborCountFn's count
        return 1;
    }
    if (PFN == GC_PFN_XSPH) {
        // XSPHPfn src/PairwiseFunctors.jl:364-389, xsph_veladjust
        // src/PairwisePhysics.jl:268-270: du = ((-ε·dv)·w)/(ρ_i + ρ_j),
        // v_adjustment_i += du·m_j.  Every system_b kind contributes its stored
        // velocity and density (a boundary wrapper forwards to its system);
        // the system_b side is this same term with the roles swapped.
        const double q = sqrt(rr) / G.H;
        const double wk = kernel_w<KK>(G.knorm, q);
        const double den = o.rho + nb.rho();
        const double mj = btype == BT_SELF ? mass_of_a() : G.bmass;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const double du = (((-P.alpha) * (o.v[d] - nb.v(d))) * wk) / den;
            acc.dv[d] = acc.dv[d] + du * mj;
        }
        return 1;
    }
    double gx[ND];
    Pair<ND, NS, PFN, KK>::geom(dx, rr, G.H, G.knorm, gx);
    const double ca = sound_a();
    const double mass_a = mass_of_a();

    if (btype == BT_DYNAMIC) {
        // src/PairwiseFunctors.jl:53,111,222,334
        double t[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) t[d] = nb.x(d) - G.point[d];
        double db = dotv<ND>(t, G.normal);
        double m = -jmin(G.beta, fabs(db / da));
        double vj[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) vj[d] = m * o.v[d];
        if (fluid_pfn<PFN>() || PFN == GC_PFN_CAUCHY_FLUID) {
            double dv[ND];
#pragma unroll
            for (int d = 0; d < ND; ++d) dv[d] = o.v[d] - vj[d];
            double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, o.rho, P.alpha, P.beta, ca, ca);
            if (fluid_pfn<PFN>()) {
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
            double cdc = (fluid_pfn<PFN>() && P.S == 1) ? o.rho / o.rho : 1.0;
            acc.dr = acc.dr + mass_a * ((fluid_pfn<PFN>() ? dr * cdc : dr) + tail);
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
    for (int d = 0; d < ND; ++d) vj[d] = nb.v(d);
    const double rhoj = nb.rho();

    if (btype == BT_STATIC && (fluid_pfn<PFN>() || PFN == GC_PFN_CAUCHY_FLUID)) {
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

    if (fluid_pfn<PFN>()) {
        double dv[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dv[d] = o.v[d] - vj[d];
        // two-sided fluid x fluid :173 uses both sound speeds, one-sided :193 its own twice
        const bool two = PFN == PFN_FLUID2 && P.two;  // multiphase / fluid-solid variant only
        const double cb = two ? G.bc : ca;
        double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, rhoj, P.alpha, P.beta, ca, cb);
        double dh;
        if (PFN == PFN_FLUID2 && P.fs) {
            // FluidSolidPfn :494-519: the fluid's pressure on both sides; the
            // fluid is the neighbour on the system_b side
            if (G.side_b) {
                const double pf = nb.p();
                dh = P.S == 1 ? -(pf + pf) / (o.rho * rhoj) : -(nb.aux() + pf / (o.rho * o.rho));
            } else {
                const double pf = A.a_p[gi];
                dh = P.S == 1 ? -(pf + pf) / (o.rho * rhoj) : -(o.aux + pf / (rhoj * rhoj));
            }
        } else {
            dh = P.S == 1 ? -(A.a_p[gi] + nb.p()) / (o.rho * rhoj) : -(o.aux + nb.aux());
        }
        double mj = btype == BT_SELF ? mass_a : G.bmass;
        if (two) {
            // dv_tmp = (dh + ast - piv)·gx, then mass_j·dv_tmp; the system_b side
            // runs this same code with the roles swapped (every factor is
            // symmetric or flips sign exactly with dx, dv and gx)
            double c = dh;
            if (P.has_eps) c = c + P.eps * (-(fabs(A.a_p[gi]) + fabs(nb.p())) / (o.rho * rhoj));
            c = c - piv;
#pragma unroll
            for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + mj * (c * gx[d]);
        } else {
            double s = mj * (dh - piv);
#pragma unroll
            for (int d = 0; d < ND; ++d) acc.dv[d] = acc.dv[d] + s * gx[d];
        }
        double dr = dotv<ND>(dv, gx);
        double tail;
        if (P.has_delta) {
            double psi = diffusion<ND>(dx, rr, o.rho, rhoj, ca, cb, P.h, P.h, gx, P.delta);
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
        const bool self = btype == BT_SELF;
        double cb = self ? ca : G.bc;
        double piv = art_visc<ND>(dx, dv, rr, P.h, o.rho, rhoj, P.alpha, P.beta, ca, cb);
        double sj[NS > 0 ? NS : 1];
#pragma unroll
        for (int q = 0; q < NS; ++q) sj[q] = nb.stress(q);
        double hv[ND];
        cauchy_f<ND, NS>(osig, sj, o.aux, nb.aux(), gx, hv);
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
        const double f = nb.aux();  // mass_j / rho_j
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

// ------------------------------------------------------------ policies
// The candidate walk below is shared by two physics policies:
//   PhysF64  the reference's FP64 expression trees (bit-identical pair terms)
//   PhysF32  FP32 pair physics with Kahan-compensated per-particle sums
// Both apply the exact FP64 acceptance test, so neighbour sets are identical.

template <int ND, int NS, int PFN, int KK>
struct PhysF64 {
    static constexpr bool BLOCKED = false;  // plain FP64 sums: nothing to merge at strip ends
    struct Own {
        OwnState<ND> o;
        double sig[NS > 0 ? NS : 1];
    };
    using AccT = Acc<ND, NS>;
    static constexpr int NSUM = 1;  // (plain FP64 sums live in AccT)
    template <class Sum>
    static __device__ __forceinline__ void flush(AccT&, Sum&) {}
    template <class Sum>
    static __device__ __forceinline__ void init_sum(Sum&) {}
    template <class Sum>
    static __device__ __forceinline__ void store_sum(const ForceArgs& A, int64_t gi, const AccT& acc, Sum&) {
        store(A, gi, acc);
    }
    static __device__ __forceinline__ void load(const ForceArgs& A, int64_t gi, Own& w) {
        const int64_t N = A.aN;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            w.o.x[d] = A.ax[d * N + gi];
            w.o.v[d] = A.av[d * N + gi];
        }
        w.o.rho = A.arho[gi];
        w.o.aux = A.aaux ? A.aaux[gi] : 0.0;
#pragma unroll
        for (int q = 0; q < NS; ++q) w.sig[q] = (PFN == GC_PFN_CAUCHY_FLUID) ? A.astress[q * N + gi] : 0.0;
    }
    static __device__ __forceinline__ const double* xpos(const Own& w) { return w.o.x; }
    static __device__ __forceinline__ void init(const ForceArgs& A, int64_t gi, AccT& acc, bool from_memory) {
        const int64_t N = A.aN;
#pragma unroll
        for (int d = 0; d < ND; ++d) acc.dv[d] = 0.0;
        acc.dr = 0.0;
        if (!from_memory) return;
        if (PFN == GC_PFN_INTERPOLATE) {
            // targets: v (advdt), rho (adrhodt), stress (asr), w_sum (avort)
            if (A.imask & (1 << GC_FIELD_V)) {
#pragma unroll
                for (int d = 0; d < ND; ++d) acc.dv[d] = A.advdt[d * N + gi];
            }
            if (A.imask & (1 << GC_FIELD_RHO)) acc.dr = A.adrhodt[gi];
            if (A.imask & (1 << GC_FIELD_STRESS)) {
#pragma unroll
                for (int q = 0; q < NS; ++q) acc.sr[q] = A.asr[q * N + gi];
            }
            acc.w[0] = A.iwsum ? A.avort[gi] : 0.0;
        } else if (PFN == GC_PFN_XSPH) {  // advdt is the v_adjustment array here
#pragma unroll
            for (int d = 0; d < ND; ++d) acc.dv[d] = A.advdt[d * N + gi];
        } else if (fluid_pfn<PFN>() || PFN == GC_PFN_CAUCHY_FLUID || PFN == GC_PFN_COUNT) {
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
    static __device__ __forceinline__ void store(const ForceArgs& A, int64_t gi, const AccT& acc) {
        const int64_t N = A.aN;
        if (PFN == GC_PFN_INTERPOLATE) {
            if (A.imask & (1 << GC_FIELD_V)) {
#pragma unroll
                for (int d = 0; d < ND; ++d) A.advdt[d * N + gi] = acc.dv[d];
            }
            if (A.imask & (1 << GC_FIELD_RHO)) A.adrhodt[gi] = acc.dr;
            if (A.imask & (1 << GC_FIELD_STRESS)) {
#pragma unroll
                for (int q = 0; q < NS; ++q) A.asr[q * N + gi] = acc.sr[q];
            }
            if (A.iwsum) A.avort[gi] = acc.w[0];
        } else if (PFN == GC_PFN_XSPH) {
#pragma unroll
            for (int d = 0; d < ND; ++d) A.advdt[d * N + gi] = acc.dv[d];
        } else if (fluid_pfn<PFN>() || PFN == GC_PFN_CAUCHY_FLUID || PFN == GC_PFN_COUNT) {
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
    static __device__ __forceinline__ double plane_da(const Own& w, const GridInst& G) {
        double t[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) t[d] = w.o.x[d] - G.point[d];
        return dotv<ND>(t, G.normal);
    }
    template <int P2>
    static __device__ __forceinline__ int pair(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                               const PfnInst& P, int64_t gi, int k, const Own& w, double da,
                                               int32_t j, AccT& acc) {
        return process_pair<ND, NS, P2, KK>(A, r, G, P, gi, k, w.o, w.sig, da, NbGlobal{r, j}, acc);
    }

    // Chunk staging (k_sweep_stg) for the fluid functors: a neighbour's FP64
    // position, then its [v, ρ, aux, p] (NbSlot's layout), copied from the
    // planar arrays by 8-byte asynchronous copies; a dynamic boundary's
    // term reads only the position, and p is copied only for the functor
    // forms that read it.  The pair terms are the same expression trees on
    // the same values as k_sweep's, so both kernels give the same bits.
    static constexpr int NQP = (ND + 1) / 2, NQR = 3;
    static constexpr int NQ = fluid_pfn<PFN>() ? NQP + NQR : 0;
    static __device__ __forceinline__ void issue(const InterRef& r, const PfnInst& P, int32_t j, float4* slot,
                                                 int BT) {
        auto cp = [&](int e, const double* src) {  // double e of the slot
            __pipeline_memcpy_async(reinterpret_cast<double*>(&slot[(e >> 1) * BT]) + (e & 1), src, 8);
        };
        const int64_t N = r.bN;
#pragma unroll
        for (int d = 0; d < ND; ++d) cp(d, r.bx + d * N + j);
        if (r.btype == BT_DYNAMIC) return;
        constexpr int E = 2 * NQP;  // first double of the record
#pragma unroll
        for (int d = 0; d < ND; ++d) cp(E + d, r.bv + d * N + j);
        cp(E + ND, r.brho + j);
        if (r.baux) cp(E + ND + 1, r.baux + j);
        // p: the multiphase pressure form, FluidSolidPfn's fluid side and the
        // two-sided form's ε term
        if (P.S == 1 || (PFN == PFN_FLUID2 && (P.fs || P.has_eps))) cp(E + ND + 2, r.bp + j);
    }
    template <int P2, int BTK = -1>
    static __device__ __forceinline__ int pair_slot(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                                    const PfnInst& P, int64_t gi, int k, const Own& w, double da,
                                                    const float4* slot, int BT, const float2* cam, AccT& acc) {
        return process_pair<ND, NS, P2, KK, BTK>(A, r, G, P, gi, k, w.o, w.sig, da, NbSlot<ND>{slot, BT}, acc,
                                                 reinterpret_cast<const double2*>(cam));
    }
    // system_a's sound speed and mass of instance k into the warp's 16-byte slot
    static __device__ __forceinline__ void stage_cam(const ForceArgs& A, int k, float2* cam) {
        if (A.a_c && A.a_mass) *reinterpret_cast<double2*>(cam) = make_double2(A.a_c[k], A.a_mass[k]);
    }
};

// ---------------------------------------------------------------- FP32
__device__ __forceinline__ void kadd(float& s, float& c, float x) {
    // Kahan (compensated) summation: c carries the rounding error of s.
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

// x added to a strip's partial sum when `on`.  An explicit round-to-nearest
// add: the compiler may not fuse it with the product that made x, which it
// would otherwise do differently in the two sweeps (and so change bits
// between launch configurations).
__device__ __forceinline__ void padd_if(float& p, float x, bool on) {
    const float t = __fadd_rn(p, x);
    p = on ? t : p;
}

// A particle's compensated sums (N components: sum s_j, compensation c_j),
// in registers or in the warp's shared memory ([2N][32], one column per
// lane, so a warp's accesses hit 32 different banks).
template <int N>
struct SumRegs {
    float s[N], c[N];
    __device__ __forceinline__ float& S(int j) { return s[j]; }
    __device__ __forceinline__ float& C(int j) { return c[j]; }
};
template <int N>
struct SumSmem {
    float* b;
    int lane;
    __device__ __forceinline__ float& S(int j) { return b[j * 32 + lane]; }
    __device__ __forceinline__ float& C(int j) { return b[(N + j) * 32 + lane]; }
};


template <int ND>
__device__ __forceinline__ double dot_exact(const double* a, const double* b) {
    double s = __dmul_rn(a[0], b[0]);
#pragma unroll
    for (int d = 1; d < ND; ++d) s = __dadd_rn(s, __dmul_rn(a[d], b[d]));
    return s;
}

template <int ND>
__device__ __forceinline__ float dotf(const float* a, const float* b) {
    float s = a[0] * b[0];
#pragma unroll
    for (int d = 1; d < ND; ++d) s += a[d] * b[d];
    return s;
}

template <int KK>
__device__ __forceinline__ float kernel_dw_dq_f(float norm, float q) {
    if (KK == GC_KERNEL_CUBIC_SPLINE) {
        float a = fmaxf(0.f, 2.f - q), b = fmaxf(0.f, 1.f - q);
        return norm * (-3.f * (0.25f * (a * a) - (b * b)));
    } else {
        float a = fmaxf(0.f, 2.f - q);
        return ((-norm * 10.f) * q) * (a * a * a);
    }
}

template <int ND, int NS, int PFN, int KK>
struct PhysF32 {
    // record layout of the FP32 pack (pack_stride floats per particle)
    static constexpr int NSP = PFN == GC_PFN_CAUCHY_FLUID ? NS : 0;
    static constexpr int R = pack_stride(ND, NSP);
    static constexpr int XD = pos_stride(ND);
    struct Own {
        double x[ND];
        float v[ND];
        float rho, aux, irho;
        float sig[NS > 0 ? NS : 1];
    };
    // one record by 16-byte loads
    static __device__ __forceinline__ void rec_load(const float* __restrict__ pk, int64_t j, float* f) {
        const float4* p = reinterpret_cast<const float4*>(pk + j * R);
#pragma unroll
        for (int q = 0; q < R / 4; ++q) {
            const float4 t = p[q];
            f[4 * q] = t.x;
            f[4 * q + 1] = t.y;
            f[4 * q + 2] = t.z;
            f[4 * q + 3] = t.w;
        }
    }
    static __device__ __forceinline__ void pos_load(const InterRef& r, int64_t j, double* x) {
        if (r.bxp) {
            const double2* p = reinterpret_cast<const double2*>(r.bxp + j * XD);
            const double2 a = p[0];
            x[0] = a.x;
            x[1] = a.y;
            if (ND == 3) x[ND - 1] = p[1].x;
        } else {
#pragma unroll
            for (int d = 0; d < ND; ++d) x[d] = r.bx[d * r.bN + j];
        }
    }
    // Per-particle sums s with Kahan compensation c, fed strip by strip: a
    // pair's term goes into the plain FP32 partial p of its strip (AccT, in
    // registers), and at the end of each strip p is added to s with
    // compensation (the sums: registers in k_sweep, shared memory in
    // k_sweep_stg).  Both sweeps evaluate a particle's pairs of a strip in
    // the same order and merge at the same strip ends, so every launch
    // configuration gives the same bits.  Components: dv/dt then dρ/dt
    // (fluid, Cauchy and counting functors), or the strain rate then the
    // vorticity.
    static constexpr bool BLOCKED = true;
    static constexpr bool FLUIDLIKE = fluid_pfn<PFN>() || PFN == GC_PFN_CAUCHY_FLUID || PFN == GC_PFN_COUNT;
    static constexpr int NSX = NS > 0 ? NS : 1;
    static constexpr int NVORT = ND == 2 ? 1 : 3;
    static constexpr int NSUM = FLUIDLIKE ? ND + 1 : NSX + (PFN == GC_PFN_STRAIN_RATE_VORTICITY ? NVORT : 0);
    static constexpr int IDR = ND;   // dρ/dt's component (fluid-like)
    static constexpr int IW = NSX;   // the first vorticity component
    struct AccT {
        float p[NSUM];
    };
    // A zero partial is skipped (a compensated add of 0 would fold c into
    // s), so a strip a sweep does not visit merges exactly like an empty one.
    template <class Sum>
    static __device__ __forceinline__ void flush(AccT& acc, Sum& sum) {
#pragma unroll
        for (int j = 0; j < NSUM; ++j) {
            if (acc.p[j] != 0.f) kadd(sum.S(j), sum.C(j), acc.p[j]);
            acc.p[j] = 0.f;
        }
    }
    template <class Sum>
    static __device__ __forceinline__ void init_sum(Sum& sum) {
#pragma unroll
        for (int j = 0; j < NSUM; ++j) sum.S(j) = sum.C(j) = 0.f;
    }
    static __device__ __forceinline__ void load(const ForceArgs& A, int64_t gi, Own& w) {
        const int64_t N = A.aN;
        float f[R];
        rec_load(A.afp, gi, f);
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            w.x[d] = A.ax[d * N + gi];
            w.v[d] = f[d];
        }
        w.rho = f[ND];
        w.aux = f[ND + 1];
        w.irho = f[ND + 2];
#pragma unroll
        for (int q = 0; q < NS; ++q) w.sig[q] = (PFN == GC_PFN_CAUCHY_FLUID) ? f[ND + 3 + q] : 0.f;
    }
    static __device__ __forceinline__ const double* xpos(const Own& w) { return w.x; }
    static __device__ __forceinline__ void init(const ForceArgs&, int64_t, AccT& acc, bool) {
#pragma unroll
        for (int j = 0; j < NSUM; ++j) acc.p[j] = 0.f;
    }
    // (the sweeps merge every strip's partials before storing)
    template <class Sum>
    static __device__ __forceinline__ void store_sum(const ForceArgs& A, int64_t gi, const AccT&, Sum& sum) {
        // FP64 state += compensated FP32 sum (s − c)
        const int64_t N = A.aN;
        if (FLUIDLIKE) {
#pragma unroll
            for (int d = 0; d < ND; ++d)
                A.advdt[d * N + gi] = A.advdt[d * N + gi] + ((double)sum.S(d) - (double)sum.C(d));
            A.adrhodt[gi] = A.adrhodt[gi] + ((double)sum.S(IDR) - (double)sum.C(IDR));
        } else {
#pragma unroll
            for (int q = 0; q < NS; ++q) A.asr[q * N + gi] = A.asr[q * N + gi] + ((double)sum.S(q) - (double)sum.C(q));
            if (PFN == GC_PFN_STRAIN_RATE_VORTICITY) {
#pragma unroll
                for (int q = 0; q < NVORT; ++q)
                    A.avort[q * N + gi] = A.avort[q * N + gi] + ((double)sum.S(IW + q) - (double)sum.C(IW + q));
            }
        }
    }
    static __device__ __forceinline__ double plane_da(const Own& w, const GridInst& G) {
        double t[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) t[d] = w.x[d] - G.point[d];
        return dotv<ND>(t, G.normal);
    }
    template <int P2>
    static __device__ __forceinline__ int pair(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                               const PfnInst& P, int64_t gi, int k, const Own& w, double da,
                                               int32_t j, AccT& acc) {
        double xj[ND];
        pos_load(r, j, xj);
        return pair_data<P2>(A, r, G, P, gi, k, w, da, xj, SrcGlobal{r.bfp, j}, make_float2(A.a_cf[k], A.a_massf[k]),
                             acc);
    }

    // Where a neighbour's record comes from: global memory (k_sweep) or a
    // staged shared-memory slot (k_sweep_stg).
    struct SrcGlobal {
        const float* pk;
        int64_t j;
        __device__ __forceinline__ void get(float* f) const { rec_load(pk, j, f); }
    };
    struct SrcSlot {
        const float4* slot;
        int BT;
        __device__ __forceinline__ void get(float* f) const {
#pragma unroll
            for (int q = 0; q < R / 4; ++q) {
                const float4 t = slot[(XD / 2 + q) * BT];
                f[4 * q] = t.x;
                f[4 * q + 1] = t.y;
                f[4 * q + 2] = t.z;
                f[4 * q + 3] = t.w;
            }
        }
    };

    // Copy of a neighbour's position and record into a shared-memory slot
    // (16-byte asynchronous copies), chunk q at slot[q*BT]; pair_slot reads it.
    static constexpr int NQP = XD / 2, NQR = R / 4, NQ = NQP + NQR;
    static __device__ __forceinline__ void issue(const InterRef& r, const PfnInst&, int32_t j, float4* slot,
                                                 int BT) {
        const float4* px = reinterpret_cast<const float4*>(r.bxp + (int64_t)j * XD);
#pragma unroll
        for (int q = 0; q < NQP; ++q) __pipeline_memcpy_async(&slot[q * BT], &px[q], 16);
        if (r.btype != BT_DYNAMIC) {
            const float4* pr = reinterpret_cast<const float4*>(r.bfp + (int64_t)j * R);
#pragma unroll
            for (int q = 0; q < NQR; ++q) __pipeline_memcpy_async(&slot[(NQP + q) * BT], &pr[q], 16);
        }
    }
    // system_a's FP32 sound speed and mass of instance k into the warp's slot
    static __device__ __forceinline__ void stage_cam(const ForceArgs& A, int k, float2* cam) {
        if (A.a_cf) *cam = make_float2(A.a_cf[k], A.a_massf[k]);
    }
    // cam: system_a's (FP32) sound speed and mass of this instance; BTK: the
    // system_b kind when known at compile time (-1: r.btype)
    template <int P2, int BTK = -1>
    static __device__ __forceinline__ int pair_slot(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                                    const PfnInst& P, int64_t gi, int k, const Own& w, double da,
                                                    const float4* slot, int BT, const float2* cam, AccT& acc) {
        double xj[ND];
#pragma unroll
        for (int q = 0; q < NQP; ++q) {
            const double2 t = *reinterpret_cast<const double2*>(&slot[q * BT]);
            if (2 * q < ND) xj[2 * q] = t.x;
            if (2 * q + 1 < ND) xj[2 * q + 1] = t.y;
        }
        return pair_data<P2, BTK>(A, r, G, P, gi, k, w, da, xj, SrcSlot{slot, BT}, *cam, acc);
    }

    template <int P2, int BTK = -1, class Src>
    static __device__ __forceinline__ int pair_data(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                                    const PfnInst& P, int64_t gi, int k, const Own& w, double da,
                                                    const double* xj, const Src& src, float2 cam, AccT& acc) {
        const int bt = BTK >= 0 ? BTK : r.btype;
        double dx[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dx[d] = __dsub_rn(w.x[d], xj[d]);
        const double rr = dot_exact<ND>(dx, dx);
        // (2h)^2, 1/h and the kernel normalisation: one 16-byte load
        const int4 gq = *reinterpret_cast<const int4*>(&G.cutoff_sq);
        // the exact test decides, without a branch, whether the pair's terms
        // are added (the pair's arithmetic stays one straight-line block)
        const bool in = rr < __hiloint2double(gq.y, gq.x);
        if (P2 == GC_PFN_COUNT) {
            if (!in) return 0;
            if constexpr (FLUIDLIKE) {
                acc.p[0] += 1.f;
                acc.p[IDR] += 1.f;
            }
            return 1;
        }
        float dxf[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) dxf[d] = (float)dx[d];
        const float rrf = (float)rr;
        const float rinv = rsqrtf(rrf);
        const float rf = rrf * rinv;
        // h, 0.01·h², α and β: one vector load
        const float4 pv = *reinterpret_cast<const float4*>(&P.f_h);
        const float invh = __int_as_float(gq.z);
        const float q = rf * invh;
        const float gc = kernel_dw_dq_f<KK>(__int_as_float(gq.w), q) * invh * rinv;
        float gx[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) gx[d] = gc * dxf[d];
        const float ca = cam.x, ma = cam.y;

        float vj[ND], rhoj, auxj, irhoj;
        float fj[R];
        if (bt == BT_DYNAMIC) {
            // src/PairwiseFunctors.jl:53,111,222,334: mirrored velocity, own density
            float db = (float)da;
#pragma unroll
            for (int d = 0; d < ND; ++d) db -= dxf[d] * G.f_normal[d];
            const float m = -fminf(G.f_beta, fabsf(__fdividef(db, (float)da)));
#pragma unroll
            for (int d = 0; d < ND; ++d) vj[d] = m * w.v[d];
            rhoj = w.rho;
            auxj = w.aux;
            irhoj = w.irho;
        } else {
            src.get(fj);
#pragma unroll
            for (int d = 0; d < ND; ++d) vj[d] = fj[d];
            rhoj = fj[ND];
            auxj = fj[ND + 1];
            irhoj = fj[ND + 2];
        }
        if constexpr (P2 == GC_PFN_STRAIN_RATE || P2 == GC_PFN_STRAIN_RATE_VORTICITY) {
            float dv[ND];
#pragma unroll
            for (int d = 0; d < ND; ++d) dv[d] = vj[d] - w.v[d];
            const float f = bt == BT_DYNAMIC ? w.aux : auxj;  // mass / rho
            float sr[NS > 0 ? NS : 1];
            if (ND == 2) {
                sr[0] = dv[0] * gx[0];
                sr[1] = dv[1] * gx[1];
                if (NS == 4) {
                    sr[2] = 0.f;
                    sr[3] = 0.5f * (dv[0] * gx[1] + dv[1] * gx[0]);
                } else {
                    sr[2] = 0.5f * (dv[0] * gx[1] + dv[1] * gx[0]);
                }
            } else {
                sr[0] = dv[0] * gx[0];
                sr[1] = dv[1] * gx[1];
                sr[2] = dv[2] * gx[2];
                sr[3] = 0.5f * (dv[0] * gx[1] + dv[1] * gx[0]);
                sr[4] = 0.5f * (dv[0] * gx[2] + dv[2] * gx[0]);
                sr[5] = 0.5f * (dv[1] * gx[2] + dv[2] * gx[1]);
            }
            if constexpr (!FLUIDLIKE) {
#pragma unroll
                for (int q2 = 0; q2 < NS; ++q2) padd_if(acc.p[q2], sr[q2] * f, in);
                if constexpr (P2 == GC_PFN_STRAIN_RATE_VORTICITY && PFN == GC_PFN_STRAIN_RATE_VORTICITY) {
                    padd_if(acc.p[IW], 0.5f * (dv[0] * gx[1] - dv[1] * gx[0]) * f, in);
                    if (ND == 3) {
                        padd_if(acc.p[IW + 1], 0.5f * (dv[0] * gx[2] - dv[2] * gx[0]) * f, in);
                        padd_if(acc.p[IW + 2], 0.5f * (dv[1] * gx[2] - dv[2] * gx[1]) * f, in);
                    }
                }
            }
            return in ? 1 : 0;
        } else {
            // momentum + continuity (FluidPfn, CauchyFluidPfn)
            float dv[ND];
#pragma unroll
            for (int d = 0; d < ND; ++d) dv[d] = w.v[d] - vj[d];
            const bool self = bt == BT_SELF, dyn = bt == BT_DYNAMIC;
            const bool two = P2 == PFN_FLUID2 && P.two;  // multiphase / fluid-solid variant only
            const float cb = ((P2 == GC_PFN_CAUCHY_FLUID && bt == BT_GHOST) || two) ? G.f_bc : ca;
            float piv = 0.f;
            const float vr = dotf<ND>(dxf, dv);
            if (vr < 0.f) {
                const float muv = __fdividef(pv.x * vr, rrf + pv.y);
                const float mc = 0.5f * (ca + cb);
                piv = (pv.w * muv - pv.z * mc) * muv * 2.f * w.irho * irhoj;
            }
            if (bt == BT_STATIC) {
                const float x = G.f_ljcut * rinv, x2 = x * x, x6 = x2 * x2 * x2;
                const float lj = rf < G.f_ljcut ? (x6 * x6 - x6) / rrf : 0.f;
                const float rfj = (0.01f * ca) * ca * lj;
                const float s = -G.f_bmass * piv;
                if constexpr (FLUIDLIKE)
#pragma unroll
                    for (int d = 0; d < ND; ++d) padd_if(acc.p[d], s * gx[d] + rfj * dxf[d], in);
                return in ? 1 : 0;
            }
            const float mj = (self || dyn) ? ma : G.f_bmass;
            if (fluid_pfn<P2>()) {
                float dh;
                if (two && P.fs) {  // the fluid's pressure p = (p/ρ²)·ρ² on both sides
                    if (G.side_b) dh = -(auxj + (auxj * rhoj * rhoj) * w.irho * w.irho);
                    else dh = -(w.aux + (w.aux * w.rho * w.rho) * irhoj * irhoj);
                } else {
                    dh = -(w.aux + auxj);
                }
                // artificial surface tension ε·(−(|p_i| + |p_j|)/(ρ_i ρ_j)), with
                // |p| = |p/ρ²|·ρ² from the record
                if (two && P.has_eps) dh -= P.f_eps * (fabsf(w.aux) * w.rho * irhoj + fabsf(auxj) * rhoj * w.irho);
                const float s = mj * (dh - piv);
                if constexpr (FLUIDLIKE)
#pragma unroll
                    for (int d = 0; d < ND; ++d) padd_if(acc.p[d], s * gx[d], in);
            } else {
                // Cauchy stress divergence: stress_j is the own stress on a dynamic boundary
                float sj[NS > 0 ? NS : 1];
#pragma unroll
                for (int q2 = 0; q2 < NS; ++q2) sj[q2] = dyn ? w.sig[q2] : fj[ND + 3 + q2];
                const float ci = w.aux, cj = auxj;
                float hv[ND];
                if (ND == 2) {
                    constexpr int XY = NS == 3 ? 2 : 3;
                    hv[0] = (w.sig[0] * gx[0] + w.sig[XY] * gx[1]) * ci + (sj[0] * gx[0] + sj[XY] * gx[1]) * cj;
                    hv[1] = (w.sig[XY] * gx[0] + w.sig[1] * gx[1]) * ci + (sj[XY] * gx[0] + sj[1] * gx[1]) * cj;
                } else {
                    hv[0] = (w.sig[0] * gx[0] + w.sig[3] * gx[1] + w.sig[4] * gx[2]) * ci +
                            (sj[0] * gx[0] + sj[3] * gx[1] + sj[4] * gx[2]) * cj;
                    hv[1] = (w.sig[3] * gx[0] + w.sig[1] * gx[1] + w.sig[5] * gx[2]) * ci +
                            (sj[3] * gx[0] + sj[1] * gx[1] + sj[5] * gx[2]) * cj;
                    hv[2] = (w.sig[4] * gx[0] + w.sig[5] * gx[1] + w.sig[2] * gx[2]) * ci +
                            (sj[4] * gx[0] + sj[5] * gx[1] + sj[2] * gx[2]) * cj;
                }
                if constexpr (FLUIDLIKE)
#pragma unroll
                    for (int d = 0; d < ND; ++d) padd_if(acc.p[d], mj * (hv[d] - piv * gx[d]), in);
            }
            float tail = 0.f;
            if (P.has_delta) {
                const float cd = two ? 0.5f * (ca + cb) : ca;
                const float psi = 2.f * P.f_delta * cd * pv.x * (w.rho - rhoj) * dotf<ND>(dxf, gx) / rrf;
                tail = psi * irhoj;
            }
            if constexpr (FLUIDLIKE) padd_if(acc.p[IDR], mj * (dotf<ND>(dv, gx) + tail), in);
            (void)gi;
            return in ? 1 : 0;
        }
    }
};

// ------------------------------------------------ shared sweep pieces
// Per (warp, interaction) set-up of both sweeps.  Returns false when the
// warp has nothing to do with this interaction: system_b's box is out of
// reach of every lane (the box test has a 0.1% margin, so no pair is lost)
// or the instance's grid did not fit its buffer (flagged, nothing read).
// Otherwise c holds each lane's cell coordinates (ok: inside the grid, with
// a flagged error when not), c0/c1 lane 0's first two, and coop whether all
// active lanes share lane 0's grid column.
template <int ND>
__device__ __forceinline__ bool ref_cells(const ForceArgs& A, const InterRef& r, const GridInst& G, int k,
                                          const double* ox, bool active, int lane, int32_t gi, int32_t* c,
                                          bool& ok, int32_t& c0, int32_t& c1, bool& coop) {
    const unsigned FULL = 0xffffffffu;
    if (r.bbox) {
        const SysInst& B = r.bbox[k];
        bool near = B.n > 0;
        const double m = 1.001 * G.cell;
#pragma unroll
        for (int d = 0; d < ND; ++d) near = near && ox[d] >= B.bbmin[d] - m && ox[d] <= B.bbmax[d] + m;
        if (!__any_sync(FULL, active && near)) {
            if (active && r.counts) r.counts[gi] = 0;
            return false;
        }
    }
    if (G.cellbase + G.ncells > r.cs_cells) {
        if (lane == 0) atomicOr(A.err, ERR_CAPACITY);
        if (active && r.counts) r.counts[gi] = 0;
        return false;
    }
    // cell coordinates (a grid has < 2^31 cells, so they fit int32)
    ok = true;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        int64_t cd;
        if (!floor_i64(__dsub_rn(ox[d], G.ming[d]) / G.cell, &cd) || cd < 1 || cd >= G.ng[d] - 1) {
            ok = false;
            cd = 1;
        }
        c[d] = (int32_t)cd;
    }
    if (active && !ok) atomicOr(A.err, ERR_CAPACITY);
    c0 = __shfl_sync(FULL, c[0], 0);
    c1 = ND == 3 ? __shfl_sync(FULL, c[1], 0) : 0;
    const bool same = ok && c[0] == c0 && (ND == 2 || c[1] == c1);
    coop = __all_sync(FULL, !active || same);
    return true;
}

// The warp's range [zlo, zhi] of last-dimension cells over its active lanes.
template <int ND>
__device__ __forceinline__ void warp_zrange(const int32_t* c, bool active, int32_t& zlo, int32_t& zhi) {
    const unsigned FULL = 0xffffffffu;
    zlo = active ? c[ND - 1] : INT32_MAX;
    zhi = active ? c[ND - 1] : INT32_MIN;
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
        const int32_t a2 = __shfl_xor_sync(FULL, zlo, o2), b2 = __shfl_xor_sync(FULL, zhi, o2);
        zlo = a2 < zlo ? a2 : zlo;
        zhi = b2 > zhi ? b2 : zhi;
    }
}

// Conservative FP32 prefilter of a batch of mb <= 32 candidates against this
// lane (coordinates relative to lane 0; rows of the batch `stride` floats
// apart, entries past mb far away): bit t set when candidate t may be within
// the cutoff.  Two candidates per packed FP32x2 instruction.  The chain
// starts from −cut, so it ends at r² − cut and its sign bit is the hit: one
// funnel shift per candidate moves it into the mask (candidates pushed from
// last to first).  A NaN result is not guaranteed a clear sign bit, so the
// callers mask out inactive lanes.  V4: 16-byte loads of four candidates'
// coordinates (rows and the base 16-byte aligned).
template <int ND, bool V4 = false>
__device__ __forceinline__ unsigned batch_hits(const float* cb, int stride, int mb, const float* xi, float cut_f) {
    const float2 neg1 = make_float2(-1.0f, -1.0f);
    const float2 ncut = make_float2(-cut_f, -cut_f);
    unsigned hits = 0;
#pragma unroll
    for (int t0 = 0; t0 < 32; t0 += 8) {
        if (t0 >= mb) break;  // warp-uniform
        unsigned h8 = 0;
#pragma unroll
        for (int t = 4; t >= 0; t -= 4) {
            float2 ra = ncut, rb = ncut;  // candidates t, t+1 and t+2, t+3
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const float* row = cb + d * stride + t0 + t;
                float2 xa, xb;
                if (V4) {
                    const float4 q = *reinterpret_cast<const float4*>(row);
                    xa = make_float2(q.x, q.y);
                    xb = make_float2(q.z, q.w);
                } else {
                    xa = *reinterpret_cast<const float2*>(row);
                    xb = *reinterpret_cast<const float2*>(row + 2);
                }
                const float2 xo = make_float2(xi[d], xi[d]);
                const float2 da = __ffma2_rn(xa, neg1, xo), db = __ffma2_rn(xb, neg1, xo);
                ra = __ffma2_rn(da, da, ra);
                rb = __ffma2_rn(db, db, rb);
            }
            h8 = __funnelshift_l(__float_as_uint(rb.y), h8, 1);
            h8 = __funnelshift_l(__float_as_uint(rb.x), h8, 1);
            h8 = __funnelshift_l(__float_as_uint(ra.y), h8, 1);
            h8 = __funnelshift_l(__float_as_uint(ra.x), h8, 1);
        }
        hits |= h8 << t0;
    }
    return hits;
}

// This lane's own strip range [lo, hi) and the self pair as a mask over the
// batch of 32 candidates starting at index jb.
__device__ __forceinline__ unsigned own_allow(int32_t lo, int32_t hi, int32_t jb, bool self, int32_t gi) {
    const int32_t tlo = lo - jb, thi = hi - jb;
    unsigned allow = tlo <= 0 ? 0xffffffffu : (tlo >= 32 ? 0u : 0xffffffffu << tlo);
    allow &= thi >= 32 ? 0xffffffffu : (thi <= 0 ? 0u : 0xffffffffu >> (32 - thi));
    if (self) {
        const int32_t ts = gi - jb;
        if (ts >= 0 && ts < 32) allow &= ~(1u << ts);
    }
    return allow;
}

// Per-warp copies of an interaction's grid and functor parameters (the pair
// loops read these: loop-invariant values the register budget would
// otherwise re-load from global memory for every pair).
constexpr int SWEEP_GI_BYTES = ((int)sizeof(GridInst) + 15) / 16 * 16;
constexpr int SWEEP_PI_BYTES = ((int)sizeof(PfnInst) + 15) / 16 * 16;
constexpr int SWEEP_PARAM_BYTES = SWEEP_GI_BYTES + SWEEP_PI_BYTES;

// Copy of a parameter block into a warp's shared memory, 4 bytes per lane.
template <class T>
__device__ __forceinline__ void warp_copy(T* dst, const T& src, int lane) {
    static_assert(sizeof(T) % 4 == 0, "4-byte words");
    const int* s = reinterpret_cast<const int*>(&src);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = lane; i < (int)(sizeof(T) / 4); i += 32) d[i] = s[i];
}

// Shared memory of one block of k_sweep: the staged-neighbour columns, the
// per-warp candidate coordinates (ND rows of 32, then lane 0's position) and
// the per-warp parameter copies.
template <int ND>
__host__ __device__ constexpr int sweep_smem_bytes(int buf) {
    return (buf * FORCE_TPB * 4 + (FORCE_TPB / 32) * ND * 34 * 4 + 15) / 16 * 16 + (FORCE_TPB / 32) * SWEEP_PARAM_BYTES;
}

// ---------------------------------------------------------------- kernel
// One warp owns one group: up to 32 consecutive (sorted) system_a particles
// of one grid column (all cell coordinates but the last equal).  For each
// 3-cell strip of the reference stencil the warp walks the union of its
// lanes' candidate ranges — contiguous in the CSR because cells along the
// last dimension are consecutive — loading 32 candidates at a time with one
// coalesced load and broadcasting them by shuffles.  A lane keeps a
// candidate only inside its own strip range [cs[z-1], cs[z+2]) and when a
// conservative FP32 distance test passes; the policy's pair() then applies
// the exact reference test r² < (2h)² on FP64 positions.  Staged indices go
// to the lane's shared-memory column; when any column is nearly full the
// whole warp evaluates its staged pairs, so the pair physics runs on
// converged warps.
template <class Phys, bool COUNT_ONLY, int UNROLL, int PFN>
__device__ __forceinline__ int flush_all(const ForceArgs& A, const InterRef& r, const GridInst& G,
                                         const PfnInst& P, int64_t gi, int k, const typename Phys::Own& w,
                                         double da, int nbuf, const int32_t* col, int BT, typename Phys::AccT& acc) {
    constexpr int P2 = COUNT_ONLY ? GC_PFN_COUNT : PFN;
    int acc_n = 0;
    int t = 0;
    if (UNROLL == 2) {
        for (; t + 1 < nbuf; t += 2) {
            const int32_t j0 = col[t * BT], j1 = col[(t + 1) * BT];
            acc_n += Phys::template pair<P2>(A, r, G, P, gi, k, w, da, j0, acc);
            acc_n += Phys::template pair<P2>(A, r, G, P, gi, k, w, da, j1, acc);
        }
    }
    for (; t < nbuf; ++t) acc_n += Phys::template pair<P2>(A, r, G, P, gi, k, w, da, col[t * BT], acc);
    return acc_n;
}

template <class Phys, int ND, int PFN, bool COUNT_ONLY, int MINB, int BUF, int UNROLL>
__global__ void __launch_bounds__(FORCE_TPB, MINB) k_sweep(ForceArgs A) {
    pdl_enter();
    extern __shared__ int32_t sbuf[];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x;
    const int BT = blockDim.x;
    int32_t* col = sbuf + tid;
    // per-warp candidate coordinates, ND rows of 32 floats, after the columns
    // per warp: ND rows of 32 candidate coordinates, then ND doubles (lane 0's position)
    float* cand = reinterpret_cast<float*>(sbuf + BUF * FORCE_TPB) + (tid >> 5) * (ND * 34);
    char* pbase = reinterpret_cast<char*>(sbuf) + (BUF * FORCE_TPB * 4 + (FORCE_TPB / 32) * ND * 34 * 4 + 15) / 16 * 16 +
                  (tid >> 5) * SWEEP_PARAM_BYTES;
    GridInst* gsm = reinterpret_cast<GridInst*>(pbase);
    PfnInst* psm = reinterpret_cast<PfnInst*>(pbase + SWEEP_GI_BYTES);
    const int64_t ngroups = *A.ngroups;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t wg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wg < ngroups; wg += nwarps) {
        const int2 grp = A.groups[wg];
        const bool active = lane < grp.y;
        const int32_t gi = grp.x + (active ? lane : 0);  // packed indices fit int32
        const int k = A.a_inst_of[gi];
        typename Phys::Own w;
        Phys::load(A, gi, w);
        const double* ox = Phys::xpos(w);
        typename Phys::AccT acc;
        Phys::init(A, gi, acc, !COUNT_ONLY);
        SumRegs<Phys::NSUM> sum;
        Phys::init_sum(sum);

        for (int ri = 0; ri < A.nref; ++ri) {
            const InterRef& r = A.ref[ri];
            const GridInst& G = r.gi[k];
            const PfnInst& P = r.pi[k];
            int32_t c[ND], c0, c1;
            bool ok, coop;
            if (!ref_cells<ND>(A, r, G, k, ox, active, lane, gi, c, ok, c0, c1, coop)) continue;
            const double da = r.btype == BT_DYNAMIC ? Phys::plane_da(w, G) : 0.0;
            warp_copy(gsm, G, lane);
            warp_copy(psm, P, lane);
            __syncwarp();
            const GridInst& Gs = *gsm;
            const PfnInst& Ps = *psm;
            const int64_t Nb = r.bN;
            const bool self = r.btype == BT_SELF;
            int nbuf = 0;
            int32_t accepted = 0;
            if (coop) {
                constexpr int L = ND - 1;  // last dimension
                int32_t zlo, zhi;
                warp_zrange<ND>(c, active, zlo, zhi);
                // Conservative FP32 prefilter in coordinates relative to lane 0:
                // |rel| spans a few cells, so single-precision rounding moves r²
                // by < 1e-5 relative; the 1e-3 margin keeps every true pair.
                // Inactive lanes have an empty own range and accept nothing.
                // lane 0's position, the origin of the relative coordinates,
                // kept in the warp's shared memory rather than in registers
                double* xref = reinterpret_cast<double*>(cand + ND * 32);
                float xi[ND];
                if (lane == 0) {
#pragma unroll
                    for (int d = 0; d < ND; ++d) xref[d] = ox[d];
                }
                __syncwarp();
#pragma unroll
                for (int d = 0; d < ND; ++d) xi[d] = active ? (float)(ox[d] - xref[d]) : 0.f;
                const float cut_f = (float)(G.cutoff_sq * 1.001);
                const int64_t ngl = G.ng[L];
                const int nstrips = ND == 2 ? 3 : 9;
                for (int sidx = 0; sidx < nstrips; ++sidx) {
                    int64_t colflat;
                    if (ND == 2) colflat = c0 + sidx - 1;
                    else colflat = (c0 + sidx / 3 - 1) * G.ng[1] + (c1 + sidx % 3 - 1);
                    const int64_t base = G.cellbase + colflat * ngl;
                    const int32_t u0 = r.cs[base + zlo - 1], u1 = r.cs[base + zhi + 2];
                    const int32_t lo = active ? r.cs[base + c[L] - 1] : 0, hi = active ? r.cs[base + c[L] + 2] : 0;
                    for (int32_t ch = u0; ch < u1; ch += 32) {
                        if (__any_sync(FULL, nbuf > BUF - 32)) {
                            accepted += flush_all<Phys, COUNT_ONLY, UNROLL, PFN>(A, r, Gs, Ps, gi, k, w, da, nbuf, col,
                                                                                 BT, acc);
                            nbuf = 0;
                            __syncwarp();
                        }
                        // 32 candidates, coordinates relative to lane 0, staged in
                        // shared memory (beyond the range: far away)
                        const int32_t jl = ch + lane;
#pragma unroll
                        for (int d = 0; d < ND; ++d)
                            cand[d * 32 + lane] = jl < u1 ? (float)(r.bx[d * Nb + jl] - xref[d]) : 1e30f;
                        __syncwarp();
                        const int m = u1 - ch < 32 ? (int)(u1 - ch) : 32;
                        unsigned hits = batch_hits<ND>(cand, 32, m, xi, cut_f) & own_allow(lo, hi, ch, self, gi);
                        while (hits) {
                            const int t = __ffs(hits) - 1;
                            hits &= hits - 1;
                            col[(nbuf++) * BT] = ch + t;
                        }
                        __syncwarp();
                    }
                    if (Phys::BLOCKED) {
                        // the strip's pairs, then its partial sums merged
                        accepted += flush_all<Phys, COUNT_ONLY, UNROLL, PFN>(A, r, Gs, Ps, gi, k, w, da, nbuf, col,
                                                                             BT, acc);
                        nbuf = 0;
                        __syncwarp();
                        Phys::flush(acc, sum);
                    }
                }
                accepted += flush_all<Phys, COUNT_ONLY, UNROLL, PFN>(A, r, Gs, Ps, gi, k, w, da, nbuf, col, BT, acc);
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
                            accepted += flush_all<Phys, COUNT_ONLY, UNROLL, PFN>(A, r, Gs, Ps, gi, k, w, da, nbuf, col,
                                                                                 BT, acc);
                            nbuf = 0;
                        }
                    }
                    if (Phys::BLOCKED) {
                        accepted += flush_all<Phys, COUNT_ONLY, UNROLL, PFN>(A, r, Gs, Ps, gi, k, w, da, nbuf, col,
                                                                             BT, acc);
                        nbuf = 0;
                        Phys::flush(acc, sum);
                    }
                }
                accepted += flush_all<Phys, COUNT_ONLY, UNROLL, PFN>(A, r, Gs, Ps, gi, k, w, da, nbuf, col, BT, acc);
                nbuf = 0;
            }
            __syncwarp();
            if (active && r.counts) r.counts[gi] = accepted;
        }
        if (!COUNT_ONLY && active) Phys::store_sum(A, gi, acc, sum);
        __syncwarp();
    }
}

// ------------------------------------------------- staged FP32 sweep
// Shared memory of one warp of k_sweep_stg: the staged copies of a chunk of
// CH candidates ([NQ][CH] 16-byte chunks: FP64 position, then FP32 record),
// lane 0's position (the origin of the prefilter), the candidates' FP32
// coordinates relative to it ([ND][CH]), and copies of the interaction's
// grid and functor parameters for this warp's instance.
constexpr int STG_GI_BYTES = SWEEP_GI_BYTES;
constexpr int STG_PI_BYTES = SWEEP_PI_BYTES;
template <int ND, int NQ, int CH, int NSUM>
__host__ __device__ constexpr int stg_warp_bytes() {
    return NQ * CH * 16 + 32 + (ND * CH * 4 + 15) / 16 * 16 + STG_GI_BYTES + STG_PI_BYTES + 16 + NSUM * 2 * 32 * 4;
}


// The FP32-compensated sweep with chunk staging.  The walk is k_sweep's (one
// warp per group of one grid column, the union of its lanes' candidate
// ranges strip by strip), but the warp copies each chunk of up to CH
// consecutive candidates of a strip into its shared memory once (16-byte
// asynchronous copies, one round trip per chunk), tests them against every
// lane with the FP32 prefilter, and then evaluates each lane's accepted
// candidates of the chunk from the staged copies.  No pair waits on a
// global load; the exact cutoff test and the pair arithmetic are the
// policy's pair_data, as in k_sweep.
template <class Phys, int ND, int PFN, int MINB, int CH>
__global__ void __launch_bounds__(FORCE_TPB, MINB) k_sweep_stg(ForceArgs A) {
    pdl_enter();
    static_assert(CH % 32 == 0 && CH >= 32 && CH <= 128, "chunk of 1 to 4 batches of 32");
    constexpr int NB = CH / 32;
    constexpr int NQ = Phys::NQ;
    constexpr int WB = stg_warp_bytes<ND, NQ, CH, Phys::NSUM>();
    extern __shared__ float4 sstg[];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    char* wbase = reinterpret_cast<char*>(sstg) + (threadIdx.x >> 5) * WB;
    float4* slots = reinterpret_cast<float4*>(wbase);
    double* xref = reinterpret_cast<double*>(wbase + NQ * CH * 16);
    float* cand = reinterpret_cast<float*>(wbase + NQ * CH * 16 + 32);
    // the pair loop reads the interaction's parameters from these copies
    // (loop-invariant loads the register budget would otherwise re-issue
    // from global memory for every pair)
    GridInst* gsm = reinterpret_cast<GridInst*>(wbase + NQ * CH * 16 + 32 + (ND * CH * 4 + 15) / 16 * 16);
    PfnInst* psm = reinterpret_cast<PfnInst*>(reinterpret_cast<char*>(gsm) + STG_GI_BYTES);
    float2* camsm = reinterpret_cast<float2*>(reinterpret_cast<char*>(psm) + STG_PI_BYTES);
    // this lane's compensated sums (touched only at strip ends)
    SumSmem<Phys::NSUM> sum{reinterpret_cast<float*>(reinterpret_cast<char*>(camsm) + 16), lane};
    const int64_t ngroups = *A.ngroups;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t wg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wg < ngroups; wg += nwarps) {
        const int2 grp = A.groups[wg];
        const bool active = lane < grp.y;
        const int32_t gi = grp.x + (active ? lane : 0);  // packed indices fit int32
        const int k = A.a_inst_of[gi];
        typename Phys::Own w;
        Phys::load(A, gi, w);
        const double* ox = Phys::xpos(w);
        typename Phys::AccT acc;
        Phys::init(A, gi, acc, true);
        Phys::init_sum(sum);

        for (int ri = 0; ri < A.nref; ++ri) {
            const InterRef& r = A.ref[ri];
            const GridInst& G = r.gi[k];
            const PfnInst& P = r.pi[k];
            int32_t c[ND], c0, c1;
            bool ok, coop;
            if (!ref_cells<ND>(A, r, G, k, ox, active, lane, gi, c, ok, c0, c1, coop)) continue;
            const double da = r.btype == BT_DYNAMIC ? Phys::plane_da(w, G) : 0.0;
            const bool self = r.btype == BT_SELF;
            int32_t accepted = 0;
            const int nstrips = ND == 2 ? 3 : 9;
            warp_copy(gsm, G, lane);
            warp_copy(psm, P, lane);
            if (lane == 0) Phys::stage_cam(A, k, camsm);
            __syncwarp();
            const GridInst& Gs = *gsm;
            const PfnInst& Ps = *psm;
            if (coop) {
                constexpr int L = ND - 1;
                int32_t zlo, zhi;
                warp_zrange<ND>(c, active, zlo, zhi);
                if (lane == 0) {
#pragma unroll
                    for (int d = 0; d < ND; ++d) xref[d] = ox[d];
                }
                __syncwarp();
                // conservative FP32 prefilter relative to lane 0 (k_sweep's);
                // inactive lanes have an empty own range and accept nothing
                float xi[ND];
#pragma unroll
                for (int d = 0; d < ND; ++d) xi[d] = active ? (float)(ox[d] - xref[d]) : 0.f;
                const float cut_f = (float)(G.cutoff_sq * 1.001);
                const int64_t ngl = G.ng[L];
                auto strip_base = [&](int s2) -> int64_t {
                    int64_t colflat;
                    if (ND == 2) colflat = c0 + s2 - 1;
                    else colflat = (c0 + s2 / 3 - 1) * G.ng[1] + (c1 + s2 % 3 - 1);
                    return G.cellbase + colflat * ngl;
                };
                // every strip's warp-wide candidate range, lane s holding strip s's
                int32_t su0 = 0, su1 = 0;
                if (lane < nstrips) {
                    const int64_t b2 = strip_base(lane);
                    su0 = r.cs[b2 + zlo - 1];
                    su1 = r.cs[b2 + zhi + 2];
                }
                // the strips, with the pair code specialised for a self
                // interaction (the dominant kind) and generic otherwise
                auto strips = [&](auto btk) {
                    constexpr int BTK = decltype(btk)::value;
                    for (int sidx = 0; sidx < nstrips; ++sidx) {
                        const int32_t u0 = __shfl_sync(FULL, su0, sidx), u1 = __shfl_sync(FULL, su1, sidx);
                        if (u0 >= u1) continue;  // warp-uniform
                        const int64_t base = strip_base(sidx);
                        // this lane's own strip range [cs[z-1], cs[z+2]) (empty when inactive)
                        const int32_t lo = active ? r.cs[base + c[L] - 1] : 0;
                        const int32_t hi = active ? r.cs[base + c[L] + 2] : 0;
                        for (int32_t ch = u0; ch < u1; ch += CH) {
                            const int n = u1 - ch < CH ? (int)(u1 - ch) : CH;
                            for (int i = lane; i < n; i += 32) Phys::issue(r, Ps, ch + i, slots + i, CH);
                            __pipeline_commit();
                            __pipeline_wait_prior(0);
                            // this lane's staged positions -> relative FP32 coordinates
#pragma unroll
                            for (int i0 = 0; i0 < CH; i0 += 32) {
                                const int i = i0 + lane;
#pragma unroll
                                for (int d = 0; d < ND; ++d) {
                                    float v = 1e30f;  // beyond the chunk: far away
                                    if (i < n) {
                                        const double2 t = *reinterpret_cast<const double2*>(&slots[(d >> 1) * CH + i]);
                                        v = (float)(((d & 1) ? t.y : t.x) - xref[d]);
                                    }
                                    cand[d * CH + i] = v;
                                }
                            }
                            __syncwarp();
                            // accepted candidates of the chunk, one mask per batch of 32
                            unsigned msk[NB];
#pragma unroll
                            for (int b = 0; b < NB; ++b) {
                                msk[b] = 0u;
                                if (32 * b < n) {
                                    const int mb = n - 32 * b < 32 ? n - 32 * b : 32;
                                    msk[b] = batch_hits<ND, true>(cand + 32 * b, CH, mb, xi, cut_f) &
                                             own_allow(lo, hi, ch + 32 * b, self, gi);
                                }
                            }
                            // this lane's accepted candidates, from the staged copies, in
                            // increasing order: msk[0] is the current batch's mask, and an
                            // empty one shifts the later batches down
                            int mbase = 0;
                            while (true) {
                                if (msk[0] == 0u) {
#pragma unroll
                                    for (int s2 = 1; s2 < NB; ++s2) {
                                        if (msk[0] == 0u) {
#pragma unroll
                                            for (int b = 0; b + 1 < NB; ++b) msk[b] = msk[b + 1];
                                            msk[NB - 1] = 0u;
                                            mbase += 32;
                                        }
                                    }
                                    if (msk[0] == 0u) break;
                                }
                                const int t = mbase + __ffs(msk[0]) - 1;
                                msk[0] &= msk[0] - 1;
                                accepted += Phys::template pair_slot<PFN, BTK>(A, r, Gs, Ps, gi, k, w, da, slots + t, CH, camsm, acc);
                            }
                            __syncwarp();  // every lane is done with the chunk before the next one lands
                        }
                        Phys::flush(acc, sum);  // the strip's partial sums
                    }
                };
                if (self) strips(std::integral_constant<int, BT_SELF>{});
                else strips(std::integral_constant<int, -1>{});
            } else if (active && ok) {
                // rare: lanes disagree on the column in this grid; walk own strips
                for (int sidx = 0; sidx < nstrips; ++sidx) {
                    int64_t base;
                    if (ND == 2) base = G.cellbase + (c[0] + sidx - 1) * G.ng[1] + (c[1] - 1);
                    else base = G.cellbase + ((c[0] + sidx / 3 - 1) * G.ng[1] + (c[1] + sidx % 3 - 1)) * G.ng[2] + (c[2] - 1);
                    const int32_t s0 = r.cs[base], e0 = r.cs[base + 3];
                    for (int32_t j = s0; j < e0; ++j) {
                        if (self && j == gi) continue;
                        accepted += Phys::template pair<PFN>(A, r, G, P, gi, k, w, da, j, acc);
                    }
                    Phys::flush(acc, sum);
                }
            }
            __syncwarp();
            if (active && r.counts) r.counts[gi] = accepted;
        }
        if (active) Phys::store_sum(A, gi, acc, sum);
        __syncwarp();
    }
}

// ------------------------------------------------------------ dispatch
template <class Phys, int ND, int PFN, int C>
static void launch_c(const ForceArgs& A, cudaStream_t s) {
    constexpr ForceCfg cf = FORCE_CFGS[C];
    int64_t warps = A.aN;
    int64_t blocks = (warps * 32 + FORCE_TPB - 1) / FORCE_TPB;
    if (blocks > (int64_t)A.num_sms * cf.minb * 4) blocks = (int64_t)A.num_sms * cf.minb * 4;
    if (blocks < 1) blocks = 1;
    if constexpr (cf.stg > 0 && Phys::NQ > 0) {
        constexpr size_t smem = (size_t)(FORCE_TPB / 32) * stg_warp_bytes<ND, Phys::NQ, cf.stg, Phys::NSUM>();
        auto kern = k_sweep_stg<Phys, ND, PFN, cf.minb, cf.stg>;
        if (smem > 48 * 1024) {
            static bool opted = false;
            if (!opted) {
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                opted = true;
            }
        }
        kern<<<(int)blocks, FORCE_TPB, smem, s>>>(A);
    } else {
        const size_t smem = (size_t)sweep_smem_bytes<ND>(cf.buf);
        auto kern = k_sweep<Phys, ND, PFN, false, cf.minb, cf.buf, cf.unroll>;
        if (smem > 48 * 1024) {
            // beyond the default dynamic shared-memory limit: opt in once per kernel
            static bool opted = false;
            if (!opted) {
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                opted = true;
            }
        }
        kern<<<(int)blocks, FORCE_TPB, smem, s>>>(A);
    }
}

template <class Phys, int ND, int PFN>
static void launch_cfg(const ForceArgs& A, cudaStream_t s) {
    switch (A.cfg) {
        case 1: launch_c<Phys, ND, PFN, 1>(A, s); break;
        case 2: launch_c<Phys, ND, PFN, 2>(A, s); break;
        case 3: launch_c<Phys, ND, PFN, 3>(A, s); break;
        default: launch_c<Phys, ND, PFN, 0>(A, s); break;
    }
}

// F32: this translation unit's precision (the FP32-compensated launches and
// the FP64 ones are compiled separately).
template <int ND, int NS, int PFN, int KK, bool F32>
static void launch_t(const ForceArgs& A, bool count_only, cudaStream_t s) {
    if constexpr (F32) {
        if constexpr (PFN != GC_PFN_COUNT && PFN != GC_PFN_XSPH && PFN != GC_PFN_INTERPOLATE)
            launch_cfg<PhysF32<ND, NS, PFN, KK>, ND, PFN>(A, s);
    } else {
        using P64 = PhysF64<ND, NS, PFN, KK>;
        if (count_only) {
            int64_t blocks = (A.aN * 32 + FORCE_TPB - 1) / FORCE_TPB;
            if (blocks > (int64_t)A.num_sms * 16) blocks = (int64_t)A.num_sms * 16;
            if (blocks < 1) blocks = 1;
            const size_t smem = (size_t)sweep_smem_bytes<ND>(FORCE_BUF);
            k_sweep<P64, ND, PFN, true, 4, FORCE_BUF, 1><<<(int)blocks, FORCE_TPB, smem, s>>>(A);
        } else {
            launch_cfg<P64, ND, PFN>(A, s);
        }
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

template <int ND, int NS, int KK, bool F32>
static int launch_pfn(const ForceArgs& A, bool count_only, cudaStream_t s) {
    switch (A.pfn) {
        case GC_PFN_FLUID: launch_t<ND, NS, GC_PFN_FLUID, KK, F32>(A, count_only, s); return 0;
        case PFN_FLUID2: launch_t<ND, NS, PFN_FLUID2, KK, F32>(A, count_only, s); return 0;
        case GC_PFN_COUNT: launch_t<ND, NS, GC_PFN_COUNT, KK, F32>(A, count_only, s); return 0;
        case GC_PFN_INTERPOLATE:  // FP64 only
            if constexpr (F32) {
                return GC_ERR_UNSUPPORTED;
            } else {
                launch_t<ND, NS, GC_PFN_INTERPOLATE, KK, F32>(A, count_only, s);
                return 0;
            }
        case GC_PFN_XSPH:  // FP64 only (a cheap, memory-bound functor)
            if constexpr (F32) {
                return GC_ERR_UNSUPPORTED;
            } else {
                launch_t<ND, NS, GC_PFN_XSPH, KK, F32>(A, count_only, s);
                return 0;
            }
        case GC_PFN_CAUCHY_FLUID:
            if (NS == 0) return GC_ERR_UNSUPPORTED;
            launch_t<ND, NS, GC_PFN_CAUCHY_FLUID, KK, F32>(A, count_only, s);
            return 0;
        case GC_PFN_STRAIN_RATE:
            if (NS == 0) return GC_ERR_UNSUPPORTED;
            launch_t<ND, NS, GC_PFN_STRAIN_RATE, KK, F32>(A, count_only, s);
            return 0;
        case GC_PFN_STRAIN_RATE_VORTICITY:
            if (NS == 0) return GC_ERR_UNSUPPORTED;
            launch_t<ND, NS, GC_PFN_STRAIN_RATE_VORTICITY, KK, F32>(A, count_only, s);
            return 0;
    }
    return GC_ERR_UNSUPPORTED;
}

template <int ND, int KK, bool F32>
static int launch_nd(const ForceArgs& A, bool count_only, cudaStream_t s) {
    const bool stress_pfn = A.pfn == GC_PFN_CAUCHY_FLUID || A.pfn == GC_PFN_STRAIN_RATE ||
                            A.pfn == GC_PFN_STRAIN_RATE_VORTICITY ||
                            (A.pfn == GC_PFN_INTERPOLATE && (A.imask & (1 << GC_FIELD_STRESS)));
    if (!stress_pfn) return launch_pfn<ND, 0, KK, F32>(A, count_only, s);
    if (ND == 2) {
        if (A.ns == 3) return launch_pfn<ND, 3, KK, F32>(A, count_only, s);
        if (A.ns == 4) return launch_pfn<ND, 4, KK, F32>(A, count_only, s);
        return GC_ERR_UNSUPPORTED;
    }
    if (A.ns == 6) return launch_pfn<ND, 6, KK, F32>(A, count_only, s);
    return GC_ERR_UNSUPPORTED;
}

// One translation unit per (dimension, precision): defines
// launch_force_<ND>d_<f32|f64>.
#define GC_DEFINE_FORCE_TU(NDIM, F32, NAME)                                               \
    int NAME(const ForceArgs& A, bool count_only, cudaStream_t s) {                      \
        if (A.kk == GC_KERNEL_CUBIC_SPLINE)                                               \
            return launch_nd<NDIM, GC_KERNEL_CUBIC_SPLINE, F32>(A, count_only, s);        \
        return launch_nd<NDIM, GC_KERNEL_WENDLAND_C2, F32>(A, count_only, s);             \
    }

}  // namespace gc
