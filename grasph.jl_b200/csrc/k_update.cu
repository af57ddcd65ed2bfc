// k_update.cu — leapfrog half/full step and per-particle state updaters.
//
// Rounding follows the reference: `@fastmath` axpy on scalar fields
// (src/Utils.jl:19-29) is a fused multiply-add; on SVector fields the
// FastMath operators fall back to plain `*` and `+`, two roundings.
// Compiled with -fmad=false; fused operations are explicit fma().
#include "gc_device.cuh"
#include "gc_kernels.h"
#include "gc_update.h"
#include "gc_pack.cuh"

namespace gc {

constexpr int UTPB = 256;

static inline int ublk(int64_t n) {
    int64_t b = (n + UTPB - 1) / UTPB;
    return (int)(b < 1 ? 1 : b);
}

// src/TimeIntegration.jl:158 (_halfstep_ps!) with the q0 snapshot of :220.
// Every load comes before the first store: the fields are separate arrays,
// but the compiler cannot know that, and would otherwise wait out a memory
// round trip per component.
__device__ __forceinline__ void halfstep_one(const StepArgs& a, int64_t g) {
    double v[MAXD], dv[MAXD];
#pragma unroll
    for (int d = 0; d < MAXD; ++d)
        if (d < a.nd) {
            v[d] = a.v[d * a.N + g];
            dv[d] = a.dvdt[d * a.N + g];
        }
    const double r = a.rho[g], dr = a.drhodt[g];
    const SysInst& S = a.inst[a.inst_of[g]];
    const double h = S.half_dt;
#pragma unroll
    for (int d = 0; d < MAXD; ++d)
        if (d < a.nd) {
            a.q0v[d * a.N + g] = v[d];
            a.v[d * a.N + g] = v[d] + h * dv[d];
            a.dvdt[d * a.N + g] = S.srcv[d];
        }
    a.q0rho[g] = r;
    a.rho[g] = fma(h, dr, r);
    a.drhodt[g] = S.srcrho;
}

__global__ void k_halfstep(StepArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x)
        halfstep_one(a, g);
}

template <int KIND>
__device__ __forceinline__ void update_one(const UpdArgs& a, int64_t g);

// KIND: the updater's GC_UPD_* kind, or -1 for none
template <int KIND>
__global__ void k_halfstep_fused(StepArgs a, UpdArgs u, PackArgs pk) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        halfstep_one(a, g);
        if (KIND >= 0) update_one<KIND>(u, g);
        if (pk.pk || pk.xpk) pack_one(pk, g);
    }
}

// src/TimeIntegration.jl:673-682: damping, full step, zero XSPH pass, x += dt·v
// (every load before the first store, as in halfstep_one).
__global__ void k_fullstep(StepArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        const SysInst& S = a.inst[a.inst_of[g]];
        const double dt = S.dt;
        const bool damp = S.gamma_dt != 0.0;
        double dvl[MAXD], q0[MAXD], vo[MAXD], xa[MAXD];  // xa: x, or v_adjustment with XSPH
#pragma unroll
        for (int d = 0; d < MAXD; ++d)
            if (d < a.nd) {
                dvl[d] = a.dvdt[d * a.N + g];
                q0[d] = a.q0v[d * a.N + g];
                vo[d] = damp ? a.v[d * a.N + g] : 0.0;
                xa[d] = a.vadj ? a.vadj[d * a.N + g] : a.x[d * a.N + g];
            }
        const double q0r = a.q0rho[g], dr = a.drhodt[g];
#pragma unroll
        for (int d = 0; d < MAXD; ++d) {
            if (d >= a.nd) continue;
            double dv = dvl[d];
            if (damp) {
                dv = dv - S.gamma_dt * vo[d];
                a.dvdt[d * a.N + g] = dv;
            }
            double v = q0[d] + dt * dv;
            if (a.vadj) {
                // XSPH correction first half; positions move after the sweeps
                v = v + (-1.0 * xa[d]);
                a.vadj[d * a.N + g] = 0.0;
                a.v[d * a.N + g] = v;
            } else {
                v = (v + (-1.0 * 0.0)) + 1.0 * 0.0;
                a.v[d * a.N + g] = v;
                a.x[d * a.N + g] = xa[d] + dt * v;
            }
        }
        a.rho[g] = fma(dt, dr, q0r);
    }
}

// :434 and :684-685: v += v_adjustment, then x += dt·v.
__global__ void k_xsph_final(StepArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        const double dt = a.inst[a.inst_of[g]].dt;
        for (int d = 0; d < a.nd; ++d) {
            const double v = a.v[d * a.N + g] + 1.0 * a.vadj[d * a.N + g];
            a.v[d * a.N + g] = v;
            a.x[d * a.N + g] = a.x[d * a.N + g] + dt * v;
        }
    }
}

// ------------------------------------------------------------------ RK4
// src/TimeIntegration.jl:783-791 (_save_q0_all!, _zero_acc_all!) and, for
// the first stage, :800 (_reset_dqdt_all!).
__global__ void k_rk4_begin(StepArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        const SysInst& S = a.inst[a.inst_of[g]];
        for (int d = 0; d < a.nd; ++d) {
            a.q0v[d * a.N + g] = a.v[d * a.N + g];
            a.accv[d * a.N + g] = 0.0;
            a.dvdt[d * a.N + g] = S.srcv[d];
        }
        a.q0rho[g] = a.rho[g];
        a.accrho[g] = 0.0;
        a.drhodt[g] = S.srcrho;
    }
}

// :802 (_rk4_advance_all!): q = q0 + (f·dt)·dqdt, then dqdt <- source.
__global__ void k_rk4_advance(StepArgs a, double f) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        const SysInst& S = a.inst[a.inst_of[g]];
        const double c = f * S.dt;
        for (int d = 0; d < a.nd; ++d) {
            a.v[d * a.N + g] = a.q0v[d * a.N + g] + c * a.dvdt[d * a.N + g];
            a.dvdt[d * a.N + g] = S.srcv[d];
        }
        a.rho[g] = fma(c, a.drhodt[g], a.q0rho[g]);
        a.drhodt[g] = S.srcrho;
    }
}

// :814-816: damping (dvdt -= Γ/dt·v), then acc += w·dqdt.
__global__ void k_rk4_acc(StepArgs a, double w) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        const SysInst& S = a.inst[a.inst_of[g]];
        for (int d = 0; d < a.nd; ++d) {
            double dv = a.dvdt[d * a.N + g];
            if (S.gamma_dt != 0.0) {
                dv = dv - S.gamma_dt * a.v[d * a.N + g];
                a.dvdt[d * a.N + g] = dv;
            }
            a.accv[d * a.N + g] = a.accv[d * a.N + g] + w * dv;
        }
        a.accrho[g] = fma(w, a.drhodt[g], a.accrho[g]);
    }
}

// :820-826: q = q0 + dt·acc, zero XSPH pass, x += dt·v.
__global__ void k_rk4_final(StepArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x) {
        const SysInst& S = a.inst[a.inst_of[g]];
        const double dt = S.dt;
        for (int d = 0; d < a.nd; ++d) {
            double v = a.q0v[d * a.N + g] + dt * a.accv[d * a.N + g];
            if (a.vadj) {
                v = v + (-1.0 * a.vadj[d * a.N + g]);
                a.vadj[d * a.N + g] = 0.0;
                a.v[d * a.N + g] = v;
            } else {
                v = (v + (-1.0 * 0.0)) + 1.0 * 0.0;
                a.v[d * a.N + g] = v;
                a.x[d * a.N + g] = a.x[d * a.N + g] + dt * v;
            }
        }
        a.rho[g] = fma(dt, a.accrho[g], a.q0rho[g]);
    }
}

void launch_rk4_begin(const StepArgs& a, cudaStream_t s) {
    if (a.N > 0) k_rk4_begin<<<ublk(a.N), UTPB, 0, s>>>(a);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}
void launch_rk4_advance(const StepArgs& a, double f, cudaStream_t s) {
    if (a.N > 0) k_rk4_advance<<<ublk(a.N), UTPB, 0, s>>>(a, f);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}
void launch_rk4_acc(const StepArgs& a, double w, cudaStream_t s) {
    if (a.N > 0) k_rk4_acc<<<ublk(a.N), UTPB, 0, s>>>(a, w);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}
void launch_rk4_final(const StepArgs& a, cudaStream_t s) {
    if (a.N > 0) k_rk4_final<<<ublk(a.N), UTPB, 0, s>>>(a);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}

void launch_xsph_final(const StepArgs& a, cudaStream_t s) {
    if (a.N > 0) k_xsph_final<<<ublk(a.N), UTPB, 0, s>>>(a);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}

void launch_halfstep(const StepArgs& a, cudaStream_t s) {
    if (a.N > 0) k_halfstep<<<ublk(a.N), UTPB, 0, s>>>(a);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}
void launch_halfstep_fused(const StepArgs& a, const UpdArgs& u, const PackArgs& pk, cudaStream_t s) {
    if (a.N <= 0) return;
    switch (u.kind) {
        case GC_UPD_ZERO_FIELDS: k_halfstep_fused<GC_UPD_ZERO_FIELDS><<<ublk(a.N), UTPB, 0, s>>>(a, u, pk); break;
        case GC_UPD_TAIT_EOS: k_halfstep_fused<GC_UPD_TAIT_EOS><<<ublk(a.N), UTPB, 0, s>>>(a, u, pk); break;
        case GC_UPD_LINEAR_EOS: k_halfstep_fused<GC_UPD_LINEAR_EOS><<<ublk(a.N), UTPB, 0, s>>>(a, u, pk); break;
        default: k_halfstep_fused<-1><<<ublk(a.N), UTPB, 0, s>>>(a, u, pk); break;
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_fullstep(const StepArgs& a, cudaStream_t s) {
    if (a.N > 0) k_fullstep<<<ublk(a.N), UTPB, 0, s>>>(a);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}

// ------------------------------------------------------------- updaters
// src/StateUpdaters.jl:202-335 (ElastoPlasticStressUpdater, NS = 4)
__device__ __forceinline__ void ep_update(const UpdInst& u, double dt, double* s, const double* er, double w,
                                          double* e, double* ep) {
    const double nu = u.prm[1];
    const double D0 = u.D0, omn = u.omn, om2n = u.om2n;
    double sxx = s[0], syy = s[1], szz = s[2], sxy = s[3];
    double dexx = er[0] * dt, deyy = er[1] * dt, dezz = er[2] * dt, dexy = er[3] * dt;
    double dsxx = D0 * (omn * dexx + nu * deyy + nu * dezz);
    double dsyy = D0 * (nu * dexx + omn * deyy + nu * dezz);
    double dszz = D0 * (nu * dexx + nu * deyy + omn * dezz);
    double dsxy = D0 * om2n * dexy;
    double wdt = w * dt;
    dsxx = dsxx - 2.0 * sxy * wdt;
    dsyy = dsyy + 2.0 * sxy * wdt;
    dsxy = dsxy + (sxx - syy) * wdt;
    double txx = sxx + dsxx, tyy = syy + dsyy, tzz = szz + dszz, txy = sxy + dsxy;
    double I1 = txx + tyy + tzz;
    double p3 = I1 / 3.0;
    double s_xx = txx - p3, s_yy = tyy - p3, s_zz = tzz - p3, s_xy = txy;
    double J2 = 0.5 * (s_xx * s_xx + s_yy * s_yy + s_zz * s_zz + 2.0 * (s_xy * s_xy));
    double sqJ2 = sqrt(J2);
    double f = u.a_phi * I1 + sqJ2 - u.k_c;
    double depxx = 0.0, depyy = 0.0, depzz = 0.0, depxy = 0.0;
    if (f > 0.0) {
        double inv2 = 1.0 / (2.0 * sqJ2);
        double dfxx = u.a_phi + s_xx * inv2, dfyy = u.a_phi + s_yy * inv2, dfzz = u.a_phi + s_zz * inv2;
        double dfxy = s_xy * inv2;
        double dgxx = u.a_psi + s_xx * inv2, dgyy = u.a_psi + s_yy * inv2, dgzz = u.a_psi + s_zz * inv2;
        double dgxy = s_xy * inv2;
        double Dxx = D0 * (omn * dgxx + nu * dgyy + nu * dgzz);
        double Dyy = D0 * (nu * dgxx + omn * dgyy + nu * dgzz);
        double Dzz = D0 * (nu * dgxx + nu * dgyy + omn * dgzz);
        double Dxy = D0 * om2n * dgxy;
        double denom = dfxx * Dxx + dfyy * Dyy + dfzz * Dzz + 2.0 * dfxy * Dxy;
        double dl = f / denom;
        depxx = dl * dgxx;
        depyy = dl * dgyy;
        depzz = dl * dgzz;
        depxy = dl * dgxy;
        dsxx = dsxx - D0 * (omn * depxx + nu * depyy + nu * depzz);
        dsyy = dsyy - D0 * (nu * depxx + omn * depyy + nu * depzz);
        dszz = dszz - D0 * (nu * depxx + nu * depyy + omn * depzz);
        dsxy = dsxy - D0 * om2n * depxy;
    }
    s[0] = sxx + dsxx;
    s[1] = syy + dsyy;
    s[2] = szz + dszz;
    s[3] = sxy + dsxy;
    if (sxx + dsxx + syy + dsyy + szz + dszz > u.apex_thr) {
        s[0] = u.apex;
        s[1] = u.apex;
        s[2] = u.apex;
        s[3] = 0.0;
    }
    e[0] = e[0] + dexx;
    e[1] = e[1] + deyy;
    e[2] = e[2] + dezz;
    e[3] = e[3] + dexy;
    ep[0] = ep[0] + depxx;
    ep[1] = ep[1] + depyy;
    ep[2] = ep[2] + depzz;
    ep[3] = ep[3] + depxy;
}

// One kernel per updater kind, so the light equation-of-state kinds are not
// held to the registers of the stress return mappings.
template <int KIND>
__global__ void k_update(UpdArgs a) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.N; g += (int64_t)gridDim.x * blockDim.x)
        update_one<KIND>(a, g);
}

// One particle's updater of kind KIND (src/StateUpdaters.jl), the body of
// k_update.
template <int KIND>
__device__ __forceinline__ void update_one(const UpdArgs& a, int64_t g) {
    const int64_t N = a.N;
    {
        const int k = a.inst_of[g];
        const UpdInst& u = a.u[k];
        const double dt = isnan(a.dt) ? a.inst[k].dt : a.dt;
        switch (KIND) {
            case GC_UPD_ZERO_FIELDS:
                if ((u.zmask >> GC_FIELD_STRAIN_RATE) & 1u)
                    for (int q = 0; q < a.ns; ++q) a.sr[q * N + g] = 0.0;
                if ((u.zmask >> GC_FIELD_VORTICITY) & 1u)
                    for (int q = 0; q < a.nvort; ++q) a.vort[q * N + g] = 0.0;
                if ((u.zmask >> GC_FIELD_P) & 1u) a.p[g] = 0.0;
                if ((u.zmask >> GC_FIELD_STRESS) & 1u)
                    for (int q = 0; q < a.ns; ++q) a.stress[q * N + g] = 0.0;
                if ((u.zmask >> GC_FIELD_DVDT) & 1u)
                    for (int d = 0; d < a.nd; ++d) a.dvdt[d * N + g] = 0.0;
                if ((u.zmask >> GC_FIELD_DRHODT) & 1u) a.drhodt[g] = 0.0;
                break;
            case GC_UPD_TAIT_EOS: {
                // src/StateUpdaters.jl:114-118
                double ratio = a.rho[g] / u.prm[0];
                double pw = u.gamma_int ? comp_powi(ratio, (int64_t)u.prm[1]) : pow(ratio, u.prm[1]);
                a.p[g] = u.pre * (pw - 1.0);
                break;
            }
            case GC_UPD_LINEAR_EOS: {
                double c = a.inst[k].c;
                a.p[g] = c * c * (a.rho[g] - u.prm[0]);
                break;
            }
            case GC_UPD_ELASTOPLASTIC: {
                double s[4], er[4], e[4], ep[4];
                for (int q = 0; q < 4; ++q) {
                    s[q] = a.stress[q * N + g];
                    er[q] = a.sr[q * N + g];
                    e[q] = a.strain[q * N + g];
                    ep[q] = a.strainp[q * N + g];
                }
                ep_update(u, dt, s, er, a.vort[g], e, ep);
                for (int q = 0; q < 4; ++q) {
                    a.stress[q * N + g] = s[q];
                    a.strain[q * N + g] = e[q];
                    a.strainp[q * N + g] = ep[q];
                }
                break;
            }
            case GC_UPD_VISCOPLASTIC_MC: {
                // src/StateUpdaters.jl:155-186 after the EOS: rigid-plastic
                // Mohr–Coulomb stress along the strain rate, minus p, apex clamp
                const int ns = a.ns;
                double sr[MAXS];
                for (int q = 0; q < ns; ++q) sr[q] = a.sr[q * N + g];
                double m;
                if (ns == 3) m = sr[0] * sr[0] + sr[1] * sr[1] + 2.0 * (sr[2] * sr[2]);
                else if (ns == 4) m = sr[0] * sr[0] + sr[1] * sr[1] + 2.0 * (sr[3] * sr[3]);
                else
                    m = sr[0] * sr[0] + sr[1] * sr[1] + sr[2] * sr[2] +
                        2.0 * (sr[3] * sr[3] + sr[4] * sr[4] + sr[5] * sr[5]);
                m = jmax(sqrt(m), 2.220446049250313e-16);  // eps(Float64)
                const double p = a.p[g];
                const double sc = 2.0 * (u.prm[1] + p * u.pre);
                const int nn = ns == 3 ? 2 : 3;  // normal components
                double st[MAXS], tr = 0.0;
                for (int q = 0; q < ns; ++q) {
                    st[q] = (sc * sr[q]) / m;
                    st[q] = st[q] - (q < nn ? p : 0.0);
                }
                for (int q = 0; q < nn; ++q) tr = q == 0 ? st[0] : tr + st[q];
                const bool apex = tr > 0.0;
                for (int q = 0; q < ns; ++q) a.stress[q * N + g] = apex ? 0.0 : st[q];
                break;
            }
            case GC_UPD_HOOKE: {
                // src/StateUpdaters.jl:366-405
                const double nu = u.prm[1], D0 = u.D0, omn = u.omn, om2n = u.om2n;
                double sxx = a.stress[g], syy = a.stress[N + g], szz = a.stress[2 * N + g], sxy = a.stress[3 * N + g];
                double dexx = a.sr[g] * dt, deyy = a.sr[N + g] * dt, dezz = a.sr[2 * N + g] * dt,
                       dexy = a.sr[3 * N + g] * dt;
                double dsxx = D0 * (omn * dexx + nu * deyy + nu * dezz);
                double dsyy = D0 * (nu * dexx + omn * deyy + nu * dezz);
                double dszz = D0 * (nu * dexx + nu * deyy + omn * dezz);
                double dsxy = D0 * om2n * dexy;
                double wdt = a.vort[g] * dt;
                dsxx = dsxx - 2.0 * sxy * wdt;
                dsyy = dsyy + 2.0 * sxy * wdt;
                dsxy = dsxy + (sxx - syy) * wdt;
                double nxx = sxx + dsxx, nyy = syy + dsyy, nzz = szz + dszz, nxy = sxy + dsxy;
                a.stress[g] = nxx;
                a.stress[N + g] = nyy;
                a.stress[2 * N + g] = nzz;
                a.stress[3 * N + g] = nxy;
                a.p[g] = -(nxx + nyy + nzz) / 3.0;
                break;
            }
            default:
                break;
        }
    }
}

void launch_update(const UpdArgs& a, cudaStream_t s) {
    if (a.N <= 0) return;
    switch (a.kind) {
        case GC_UPD_ZERO_FIELDS: k_update<GC_UPD_ZERO_FIELDS><<<ublk(a.N), UTPB, 0, s>>>(a); break;
        case GC_UPD_TAIT_EOS: k_update<GC_UPD_TAIT_EOS><<<ublk(a.N), UTPB, 0, s>>>(a); break;
        case GC_UPD_LINEAR_EOS: k_update<GC_UPD_LINEAR_EOS><<<ublk(a.N), UTPB, 0, s>>>(a); break;
        case GC_UPD_ELASTOPLASTIC: k_update<GC_UPD_ELASTOPLASTIC><<<ublk(a.N), UTPB, 0, s>>>(a); break;
        case GC_UPD_VISCOPLASTIC_MC: k_update<GC_UPD_VISCOPLASTIC_MC><<<ublk(a.N), UTPB, 0, s>>>(a); break;
        case GC_UPD_HOOKE: k_update<GC_UPD_HOOKE><<<ublk(a.N), UTPB, 0, s>>>(a); break;
        default: return;  // no per-particle work
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

bool halfstep_fuses(int kind) {
    return kind == GC_UPD_ZERO_FIELDS || kind == GC_UPD_TAIT_EOS || kind == GC_UPD_LINEAR_EOS;
}

// ----------------------------------------------------------- virtual systems
// VirtualNormUpdater (src/StateUpdaters.jl:65-76): each listed field divided
// by w_sum (zero where w_sum is zero), then v = v·v_mult + prescribed_v, two
// roundings (a fused broadcast, no contraction); PrescribedVelocityUpdater
// (:95-97): v += prescribed_v.
__global__ void k_virtual_update(VirtArgs a) {
    pdl_enter();
    const int64_t N = a.N;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
        const int k = a.inst_of[g];
        const double* pv = a.vi[k].pv;
        if (a.kind == GC_UPD_PRESCRIBED_V) {
            for (int d = 0; d < a.nd; ++d) a.v[d * N + g] = a.v[d * N + g] + pv[d];
            continue;
        }
        const UpdInst& u = a.u[k];
        const int m = (int)u.prm[3];
        const double w = a.wsum[g];
        if (m & (1 << GC_FIELD_V))
            for (int d = 0; d < a.nd; ++d) {
                const double val = w == 0.0 ? 0.0 : a.v[d * N + g] / w;
                a.v[d * N + g] = val * u.prm[d] + pv[d];
            }
        if (m & (1 << GC_FIELD_RHO)) a.rho[g] = w == 0.0 ? 0.0 : a.rho[g] / w;
        if ((m & (1 << GC_FIELD_P)) && a.p) a.p[g] = w == 0.0 ? 0.0 : a.p[g] / w;
        if ((m & (1 << GC_FIELD_STRESS)) && a.stress)
            for (int q = 0; q < a.ns; ++q) a.stress[q * N + g] = w == 0.0 ? 0.0 : a.stress[q * N + g] / w;
    }
}

void launch_virtual_update(const VirtArgs& a, cudaStream_t s) {
    if (a.N > 0) k_virtual_update<<<ublk(a.N), UTPB, 0, s>>>(a);
    g_launches.fetch_add(a.N > 0, std::memory_order_relaxed);
}

__global__ void k_virtual_advance(double* __restrict__ x, int64_t N, int nd, const int32_t* __restrict__ inst_of,
                                  const SysInst* __restrict__ inst, const VirtInst* __restrict__ vi) {
    pdl_enter();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
        const int k = inst_of[g];
        const double dt = inst[k].dt;
        for (int d = 0; d < nd; ++d) x[d * N + g] = x[d * N + g] + vi[k].pv[d] * dt;
    }
}

void launch_virtual_advance(double* x, int64_t N, int nd, const int32_t* inst_of, const SysInst* inst,
                            const VirtInst* vi, cudaStream_t s) {
    if (N > 0) k_virtual_advance<<<ublk(N), UTPB, 0, s>>>(x, N, nd, inst_of, inst, vi);
    g_launches.fetch_add(N > 0, std::memory_order_relaxed);
}

}  // namespace gc
