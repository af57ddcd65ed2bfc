// gc_pack.cuh — one particle's FP32 sweep record and FP64 position copy
// (the layout of pack_stride / pos_stride in gc_force.h), shared by the pack
// kernel and the fused half step.
#pragma once

#include "gc_force.h"
#include "gc_update.h"

namespace gc {

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
    const int R = pack_stride(nd, ns);
    float rec[16];
    const double r = a.rho[g];
    for (int d = 0; d < nd; ++d) rec[d] = (float)a.v[d * N + g];
    rec[nd] = (float)r;
    double aux;
    if (a.mode == AUX_P_OVER_RHO2) aux = a.p ? a.p[g] / (r * r) : 0.0;  // boundaries may have no pressure
    else if (a.mode == AUX_INV_RHO2) aux = 1.0 / (r * r);
    else aux = a.mass[a.inst_of[g]] / r;
    rec[nd + 1] = (float)aux;
    rec[nd + 2] = (float)(1.0 / r);
    for (int q = 0; q < ns; ++q) rec[nd + 3 + q] = a.stress ? (float)a.stress[q * N + g] : 0.0f;
    for (int q = nd + 3 + ns; q < R; ++q) rec[q] = 0.0f;
    float4* o = reinterpret_cast<float4*>(a.pk + g * R);
    for (int q = 0; q < R / 4; ++q) o[q] = make_float4(rec[4 * q], rec[4 * q + 1], rec[4 * q + 2], rec[4 * q + 3]);
}

}  // namespace gc
