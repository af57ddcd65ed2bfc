// gc_pack.cuh — one particle's FP32 sweep record and FP64 position copy
// (the layout of pack_stride / pos_stride in gc_force.h), shared by the pack
// kernel and the fused half step.
#pragma once

#include "gc_force.h"
#include "gc_update.h"

namespace gc {

// One FP32 record of ND dimensions and NS stress components: with both
// known at compile time the record stays in registers.
template <int ND, int NS>
__device__ __forceinline__ void pack_rec(const PackArgs& a, int64_t g) {
    constexpr int R = pack_stride(ND, NS);
    const int64_t N = a.N;
    float rec[R];
    const double r = a.rho[g];
#pragma unroll
    for (int d = 0; d < ND; ++d) rec[d] = (float)a.v[d * N + g];
    rec[ND] = (float)r;
    double aux;
    if (a.mode == AUX_P_OVER_RHO2) aux = a.p ? a.p[g] / (r * r) : 0.0;  // boundaries may have no pressure
    else if (a.mode == AUX_INV_RHO2) aux = 1.0 / (r * r);
    else aux = a.mass[a.inst_of[g]] / r;
    rec[ND + 1] = (float)aux;
    rec[ND + 2] = (float)(1.0 / r);
#pragma unroll
    for (int q = 0; q < NS; ++q) rec[ND + 3 + q] = a.stress ? (float)a.stress[q * N + g] : 0.0f;
#pragma unroll
    for (int q = ND + 3 + NS; q < R; ++q) rec[q] = 0.0f;
    float4* o = reinterpret_cast<float4*>(a.pk + g * R);
#pragma unroll
    for (int q = 0; q < R / 4; ++q) o[q] = make_float4(rec[4 * q], rec[4 * q + 1], rec[4 * q + 2], rec[4 * q + 3]);
}

// Any other shape (the stress systems' checks admit none): run-time sizes.
__device__ __forceinline__ void pack_rec_any(const PackArgs& a, int64_t g) {
    const int64_t N = a.N;
    const int nd = a.nd, ns = a.ns;
    const int R = pack_stride(nd, ns);
    float rec[16];
    const double r = a.rho[g];
    for (int d = 0; d < nd; ++d) rec[d] = (float)a.v[d * N + g];
    rec[nd] = (float)r;
    double aux;
    if (a.mode == AUX_P_OVER_RHO2) aux = a.p ? a.p[g] / (r * r) : 0.0;
    else if (a.mode == AUX_INV_RHO2) aux = 1.0 / (r * r);
    else aux = a.mass[a.inst_of[g]] / r;
    rec[nd + 1] = (float)aux;
    rec[nd + 2] = (float)(1.0 / r);
    for (int q = 0; q < ns; ++q) rec[nd + 3 + q] = a.stress ? (float)a.stress[q * N + g] : 0.0f;
    for (int q = nd + 3 + ns; q < R; ++q) rec[q] = 0.0f;
    float4* o = reinterpret_cast<float4*>(a.pk + g * R);
    for (int q = 0; q < R / 4; ++q) o[q] = make_float4(rec[4 * q], rec[4 * q + 1], rec[4 * q + 2], rec[4 * q + 3]);
}

__device__ __forceinline__ void pack_one(const PackArgs& a, int64_t g) {
    const int64_t N = a.N;
    const int nd = a.nd, ns = a.ns;
    if (a.xpk) {
        // 16-byte stores: (x, y) then (z, 0) in 3-D
        double2* o = reinterpret_cast<double2*>(a.xpk + g * pos_stride(nd));
        o[0] = make_double2(a.x[g], a.x[N + g]);
        if (nd == 3) o[1] = make_double2(a.x[2 * N + g], 0.0);
    }
    if (!a.pk) return;
    // the records' shapes: no stress, or a Cauchy functor's stress (Voigt
    // 3 or 4 in 2-D, 6 in 3-D)
    if (nd == 3 && ns == 6) pack_rec<3, 6>(a, g);
    else if (nd == 3 && ns == 0) pack_rec<3, 0>(a, g);
    else if (nd == 2 && ns == 3) pack_rec<2, 3>(a, g);
    else if (nd == 2 && ns == 4) pack_rec<2, 4>(a, g);
    else if (nd == 2 && ns == 0) pack_rec<2, 0>(a, g);
    else pack_rec_any(a, g);
}

}  // namespace gc
