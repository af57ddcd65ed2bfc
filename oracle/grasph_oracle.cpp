// grasph_oracle.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A plain C++17 restatement of Grasph.jl's per-timestep SPH path, used as the
// parity checker for libgrasph_cuda.so.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load it.  The product library never
// links, loads or falls back to it.
//
// Every routine follows the reference's own loop order and expression trees
// (file:line cited per function), compiled with -ffp-contract=off and no
// fast-math so the FP64 arithmetic is the reference's arithmetic:
//   * SVector operations are per component, dot products are left-to-right
//     sums of products (StaticArrays 1.9 `_vecdot`);
//   * `x^3` is x*x*x (Julia literal_pow), `x^2` is x*x;
//   * `@fastmath` axpy on scalar fields (src/Utils.jl:19-29) is taken as a
//     fused multiply-add, on SVector fields as separate multiply and add
//     (Base.FastMath falls back to plain operators for non-scalar types);
//   * `x^y` with an integer-valued Float64 y and `x^n` with an Int n use a
//     compensated power-by-squaring (Graillat, Langlois & Louvet, "Algorithms
//     for accurate, validated and fast polynomial evaluation", 2009 — the
//     compensated-power scheme), which is the method Julia 1.12 applies to
//     these cases; other real powers call std::pow.
// The coloured sweeps can run on OpenMP threads; colours make every thread's
// writes disjoint, so threaded results equal serial results bit for bit.
//
// Parity status: the sort, grid, neighbour sets and per-pair arithmetic are
// pinned by the reference's known-answer tests (ported under tests/).  Tait
// EOS, artificial-viscosity, Lennard-Jones, dynamic-boundary and continuity
// magnitudes have no known-answer test in the reference and are pinned only
// by this restatement (Julia is not available to run the reference itself).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <array>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/grasph_cuda.h"

namespace {

// ------------------------------------------------------------------ helpers

// Julia `min`/`max` on Float64: NaN propagates; min(-0.0, 0.0) == -0.0.
inline double jmin(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return a - b;  // NaN
    if (a < b) return a;
    if (b < a) return b;
    return std::signbit(a) ? a : b;
}
inline double jmax(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return a - b;
    if (a > b) return a;
    if (b > a) return b;
    return std::signbit(a) ? b : a;
}

// Julia floor(Int, v): InexactError when v is not representable.
inline bool floor_int(double v, int64_t* out) {
    double f = std::floor(v);
    if (!(f >= -9.2233720368547758e18 && f < 9.2233720368547758e18)) return false;
    *out = (int64_t)f;
    return true;
}

// Error-free product a*b = p + e (exact with a correctly rounded fma).
inline void two_prod(double a, double b, double* p, double* e) {
    *p = a * b;
    *e = std::fma(a, b, -*p);
}

// Compensated x^n for integer n (power by squaring with the rounding error of
// each product carried in a second word).
double comp_powi(double x, int64_t n) {
    if (n == 0) return 1.0;
    if (n == 3) return x * x * x;
    double xl = 0.0;
    if (n < 0) {
        double rx = 1.0 / x;
        if (n == -2) return rx * rx;
        if (std::isfinite(x)) xl = -std::fma(x, rx, -1.0) * rx;
        x = rx;
        n = -n;
    }
    double y = 1.0, yl = 0.0;
    while (n > 1) {
        if (n & 1) {
            double err = y * xl + x * yl;
            double p, e;
            two_prod(x, y, &p, &e);
            y = p;
            yl = e + err;
        }
        double err = x * 2.0 * xl;
        double p, e;
        two_prod(x, x, &p, &e);
        x = p;
        xl = e + err;
        n >>= 1;
    }
    double err = y * xl + x * yl;
    if (std::isfinite(x) && std::isfinite(err)) return std::fma(x, y, err);
    return x * y;
}

double jpow(double x, double y) {
    if (y == std::trunc(y) && std::fabs(y) < 9.0e15) return comp_powi(x, (int64_t)y);
    return std::pow(x, y);
}

// ------------------------------------------------------------------ model

struct Upd {
    int kind;
    double prm[GC_UPD_NPARAM];
};

struct Sys {
    int kind = GC_SYS_BASIC, nd = 2, ns = 0, nvort = 0;
    int64_t n = 0;
    double mass = 0, c = 0, srcv[3] = {0, 0, 0}, srcrho = 0;
    std::vector<double> x, v, vadj, rho, dvdt, drhodt, p, stress, sr, vort, strain, strainp;
    std::vector<int64_t> id;
    bool upd_set = false;
    std::vector<std::vector<Upd>> upd;  // one chain per updater-tuple entry
    std::vector<double> q0v, q0rho;
    std::vector<double> accv, accrho;  // RK4 accumulators
    // Magnitude shadows of the rate fields (test infrastructure, track_mag):
    // |value| when the field is set (reset to its source term, zeroed,
    // uploaded), then + |term| for every pair term and damping term added
    // to it.  Permuted with the particles.
    std::vector<double> mdvdt, mdrhodt, msr, mvort;
    // Integrated-state shadows (track_mag): Σ over steps of each increment's
    // magnitude, dt·M(dv/dt) for v, dt·M(dρ/dt) for ρ, dt·max(|v|, M(v)) for
    // x; zero when the field is set.  The scale of a trajectory's error.
    std::vector<double> mvi, mrhoi, mxi, accmv, accmrho;
    // Elasto-plastic and Hooke systems (track_mag): Σ over steps of the
    // stress increment's magnitude, dt·|D|·M(ε̇) + 2·dt·|σ|·M(ω) per
    // component, and of the strain increment's, dt·M(ε̇).
    std::vector<double> mstr, mstrain;
    bool vsrc = false;  // the source of a virtual system: not one of the integrator's systems
    bool probe = false; // a probe's own arrays (count extra in drhodt)
    bool has_p() const { return kind >= GC_SYS_FLUID; }
    bool has_stress() const { return kind >= GC_SYS_STRESS; }
    bool is_ep() const { return kind == GC_SYS_ELASTOPLASTIC; }
};

struct Copier {
    std::vector<std::pair<int, int>> entries;  // (field, mode)
};

struct Ghost {
    int src = 0;
    double cutoff = 0;
    int nplanes = 0;
    std::vector<double> pn, pp;
    std::vector<Copier> copiers;
    bool ex_p = false, ex_stress = false;
    int64_t n = 0;
    std::vector<double> x, v, rho, normals, p, stress;
    std::vector<int64_t> io, ib;
};

enum { H_SYS = 0, H_DYN = 1, H_STATIC = 2, H_GHOST = 3, H_VIRT = 4 };

// VirtualParticleSystem src/Particles.jl:476-528: every per-particle field is
// the source system's; w_sum, the updaters and prescribed_v are its own.
struct Virt {
    int src = 0;
    int zmask = 0;  // zero_fields as 1<<GC_FIELD_*
    double pv[3] = {0, 0, 0};
    std::vector<double> wsum;
    bool upd_set = false;
    std::vector<std::vector<Upd>> upd;
    bool probe = false;  // ProbeParticleSystem src/ProbeParticles.jl:23-102 (source = its own arrays)
    int mirror = -1;     // its mirror_target system, or -1
};
struct Handle {
    int type = H_SYS;
    int idx = 0;  // system index (H_SYS, wrappers) or ghost index
    double normal[3] = {0, 0, 0}, point[3] = {0, 0, 0};
    double beta = 0, ljcut = 0;
};

struct Inter {
    int a = 0;      // system index
    int b = -1;     // handle index or -1
    int kk = GC_KERNEL_CUBIC_SPLINE;
    double H = 0;
    int nstages = 0;
    std::vector<int> pk;
    std::vector<std::array<double, GC_PFN_NPARAM>> pp;
    double cell = 0;
    double ming[3] = {0, 0, 0};
    int64_t ng[3] = {1, 1, 1};
    std::vector<int64_t> cs, csa;
    double mina[3] = {0, 0, 0}, maxa[3] = {0, 0, 0};
    bool grid = false;
    bool probe = false;  // one of the integrator's probe_interactions (swept at measurement only)
    int ag = -1;         // system_a is this ghost system (a = its source); InterpolateFieldFn only
    Sys proxy;           // the ghost's current arrays as a system (system_a of such an interaction)
    int vk = GC_PFN_NONE;  // velocity_adjust_pairwise_fn (XSPHPfn or nothing)
    double veps = 0.0;     // its epsilon
};

}  // namespace

struct oracle_ctx {
    std::vector<Sys> sys;
    std::vector<Ghost> ghosts;
    std::vector<Handle> handles;
    std::vector<int> sys_handle;  // handle of each system
    std::vector<Inter> inters;
    std::vector<Virt> virts;
    double gamma = 0;
    int integ = GC_INTEGRATOR_LEAPFROG;
    int threads = 1;
    int track_mag = 0;  // magnitude shadows: 0 off, 1 over the terms, 2 over the inputs
    int64_t steps = 0;
    std::string err;
};

namespace {

int fail(oracle_ctx* c, int code, const char* msg) {
    c->err = msg;
    return code;
}

// ------------------------------------------------------------------ kernels
// src/Kernels.jl:42-81 (cubic spline), :116-153 (Wendland C2)
struct Kern {
    int kind, nd;
    double H, norm;
};

Kern make_kernel(int kind, int nd, double H) {
    Kern k{kind, nd, H, 0.0};
    const double pi = 3.141592653589793;
    if (kind == GC_KERNEL_CUBIC_SPLINE) {
        if (nd == 1) k.norm = 2.0 / (3.0 * H);
        else if (nd == 2) k.norm = 10.0 / ((7.0 * pi) * (H * H));
        else k.norm = 1.0 / (pi * (H * H * H));
    } else {
        if (nd == 2) k.norm = 7.0 / ((64.0 * pi) * (H * H));
        else k.norm = 21.0 / ((256.0 * pi) * (H * H * H));
    }
    return k;
}

inline double kernel_w(const Kern& k, double q) {
    if (k.kind == GC_KERNEL_CUBIC_SPLINE) {
        double a = jmax(0.0, 2.0 - q), b = jmax(0.0, 1.0 - q);
        return k.norm * (0.25 * (a * a * a) - (b * b * b));
    }
    double a = jmax(0.0, 2.0 - q);
    double a2 = a * a;
    return (k.norm * (a2 * a2)) * (2.0 * q + 1.0);
}

inline double kernel_dw_dq(const Kern& k, double q) {
    if (k.kind == GC_KERNEL_CUBIC_SPLINE) {
        double a = jmax(0.0, 2.0 - q), b = jmax(0.0, 1.0 - q);
        return k.norm * (-3.0 * (0.25 * (a * a) - (b * b)));
    }
    double a = jmax(0.0, 2.0 - q);
    return ((-k.norm * 10.0) * q) * (a * a * a);
}

// ------------------------------------------------------------- primitives
// src/PairwisePhysics.jl

// Test infrastructure: set (read-only) during a magnitude pass over the
// inputs (track_mag 2).  Every difference or signed sum a pair term is built
// from -- velocities, densities, pressures, stresses, gradient components --
// is then taken as the sum of the magnitudes, so the shadow bounds how far
// the term moves when its inputs carry relative errors (a trajectory that
// drifted by a few ulps, or inputs rounded to FP32).  Zero otherwise.
int g_mag_inputs = 0;

template <int ND>
inline void vdiff(const double* a, const double* b, double* out) {
    for (int d = 0; d < ND; ++d) out[d] = g_mag_inputs ? std::fabs(a[d]) + std::fabs(b[d]) : a[d] - b[d];
}

template <int ND>
inline double dot(const double* a, const double* b) {
    double s = a[0] * b[0];
    for (int d = 1; d < ND; ++d) s = s + a[d] * b[d];
    return s;
}

template <int ND>
inline double dot_abs(const double* a, const double* b) {
    double s = 0.0;
    for (int d = 0; d < ND; ++d) s += std::fabs(a[d]) * std::fabs(b[d]);
    return s;
}

// :29-34
template <int ND>
inline double art_visc(const double* dx, const double* dv, double h, double ri, double rj,
                       double alpha, double beta, double ci, double cj) {
    double vr = g_mag_inputs ? -dot_abs<ND>(dx, dv) : jmin(dot<ND>(dx, dv), 0.0);
    double muv = (h * vr) / (dot<ND>(dx, dx) + (h * h) * 0.01);
    double mc = 0.5 * (ci + cj);
    return ((beta * muv - alpha * mc) * muv) / ((0.5 * ri) * rj);
}

// :58-69
inline double pressure_coeff(double pi_, double pj, double ri, double rj, int S) {
    if (g_mag_inputs) {
        pi_ = std::fabs(pi_);
        pj = std::fabs(pj);
    }
    if (S == 1) return -(pi_ + pj) / (ri * rj);
    return -(pi_ / (ri * ri) + pj / (rj * rj));
}

// :99-105
inline double cont_coeff(double ri, double rj, int S) { return S == 1 ? ri / rj : 1.0; }

// :238-243 (the nine-argument form every functor calls)
template <int ND>
inline double diffusion(const double* dx, double ri, double rj, double ci, double cj, double hi,
                        double hj, const double* gx, double delta, bool on) {
    if (!on) return 0.0;
    double rr = dot<ND>(dx, dx);
    double c = 0.5 * (ci + cj);
    double h = 0.5 * (hi + hj);
    const double drho = g_mag_inputs ? std::fabs(ri) + std::fabs(rj) : ri - rj;
    return (((((2.0 * delta) * c) * h) * drho) * dot<ND>(dx, gx)) / rr;
}

// :258-263
template <int ND>
inline double lennard_jones(const double* dx, double cutoff, double c) {
    double rr = dot<ND>(dx, dx);
    double r = std::sqrt(rr);
    double ind = r < cutoff ? 1.0 : 0.0;
    double f = (ind * (comp_powi(cutoff / r, 12) - comp_powi(cutoff / r, 6))) / rr;
    return ((0.01 * c) * c) * f;
}

// :125-151; out has ND components
template <int ND>
inline void cauchy(const double* si_, const double* sj_, int ns, double ri, double rj, const double* g,
                   double* out) {
    double ci = 1.0 / (ri * ri);
    double cj = 1.0 / (rj * rj);
    double ai[6], aj[6];
    const double* si = si_;
    const double* sj = sj_;
    if (g_mag_inputs) {
        for (int q = 0; q < ns; ++q) {
            ai[q] = std::fabs(si_[q]);
            aj[q] = std::fabs(sj_[q]);
        }
        si = ai;
        sj = aj;
    }
    if (ND == 2) {
        int xy = ns == 3 ? 2 : 3;
        out[0] = (si[0] * g[0] + si[xy] * g[1]) * ci + (sj[0] * g[0] + sj[xy] * g[1]) * cj;
        out[1] = (si[xy] * g[0] + si[1] * g[1]) * ci + (sj[xy] * g[0] + sj[1] * g[1]) * cj;
    } else {
        out[0] = (si[0] * g[0] + si[3] * g[1] + si[4] * g[2]) * ci +
                 (sj[0] * g[0] + sj[3] * g[1] + sj[4] * g[2]) * cj;
        out[1] = (si[3] * g[0] + si[1] * g[1] + si[5] * g[2]) * ci +
                 (sj[3] * g[0] + sj[1] * g[1] + sj[5] * g[2]) * cj;
        out[2] = (si[4] * g[0] + si[5] * g[1] + si[2] * g[2]) * ci +
                 (sj[4] * g[0] + sj[5] * g[1] + sj[2] * g[2]) * cj;
    }
}

// :169-195
template <int ND>
inline void strain_rate_t(const double* dv, const double* g, int ns, double* sr) {
    if (ND == 2) {
        sr[0] = dv[0] * g[0];
        sr[1] = dv[1] * g[1];
        if (ns == 4) {
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

// :210-220
template <int ND>
inline void vorticity_t(const double* dv, const double* g, double* w) {
    if (g_mag_inputs) {
        w[0] = 0.5 * (dv[0] * g[1] + dv[1] * g[0]);
        if (ND == 3) {
            w[1] = 0.5 * (dv[0] * g[2] + dv[2] * g[0]);
            w[2] = 0.5 * (dv[1] * g[2] + dv[2] * g[1]);
        }
        return;
    }
    if (ND == 2) {
        w[0] = 0.5 * (dv[0] * g[1] - dv[1] * g[0]);
    } else {
        w[0] = 0.5 * (dv[0] * g[1] - dv[1] * g[0]);
        w[1] = 0.5 * (dv[0] * g[2] - dv[2] * g[0]);
        w[2] = 0.5 * (dv[1] * g[2] - dv[2] * g[1]);
    }
}

// ---------------------------------------------------------------- b views

struct BView {
    int type;  // H_SYS / H_DYN / H_STATIC / H_GHOST
    int64_t n;
    const double* x;
    const double* v;
    const double* rho;
    const double* p;
    const double* stress;
    double mass, c;
    int ns;
    Sys* sys;  // backing system for two-sided writes (H_SYS and wrappers)
    Virt* virt;  // H_VIRT: the virtual system (w_sum)
    const double* normal;
    const double* point;
    double beta, ljcut;
};

struct Pfn {
    int kind;
    double alpha, beta, h;
    int S;
    double delta;
    bool has_delta;
    double eps;  // artificial surface tension (two-sided FluidPfn only)
    bool has_eps;
    int imask;   // InterpolateFieldFn: fields (1<<GC_FIELD_*)
    bool iwsum;  // InterpolateFieldFn: accumulate w_sum
    bool mag = false;  // magnitude pass: rate accumulators sum |term| (see track_mag)
};

// One pair term added to (acc) or subtracted from (dec) a rate accumulator,
// rounded as the reference's `a += t` / `a -= t`.  In a magnitude pass the
// accumulator is a magnitude shadow and receives |t|: the per-particle
// Σ|terms| that scales a summation-order difference.
inline void acc(const Pfn& f, double& x, double t) { x = f.mag ? x + std::fabs(t) : x + t; }
inline void dec(const Pfn& f, double& x, double t) { x = f.mag ? x + std::fabs(t) : x - t; }

Pfn make_pfn(int kind, const double* prm) {
    Pfn f;
    f.kind = kind;
    f.alpha = prm[0];
    f.beta = prm[1];
    f.h = prm[2];
    f.S = (int)prm[3];
    f.delta = prm[4];
    f.has_delta = !std::isnan(prm[4]);
    f.eps = prm[5];
    f.has_eps = !std::isnan(prm[5]);
    f.imask = kind == GC_PFN_INTERPOLATE ? (int)prm[0] : 0;
    f.iwsum = kind == GC_PFN_INTERPOLATE && prm[1] != 0.0;
    return f;
}

// --------------------------------------------------------- self functors
// src/PairwiseFunctors.jl :20 (SR), :80 (SRV), :151 (Fluid), :265 (Cauchy)
template <int ND>
void pfn_self(const Pfn& f, Sys& ps, int64_t i, int64_t j, const double* dx, const double* gx, double w) {
    const int ns = ps.ns;
    switch (f.kind) {
        case GC_PFN_FLUID: {
            const double* vi = &ps.v[i * ND];
            const double* vj = &ps.v[j * ND];
            double ri = ps.rho[i], rj = ps.rho[j], pi_ = ps.p[i], pj = ps.p[j];
            double mass = ps.mass;
            double dv[ND];
            vdiff<ND>(vi, vj, dv);
            double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, ps.c, ps.c);
            double dh = pressure_coeff(pi_, pj, ri, rj, f.S);
            double s = mass * (dh - piv);
            for (int d = 0; d < ND; ++d) {
                double t = s * gx[d];
                acc(f, ps.dvdt[i * ND + d], t);
                dec(f, ps.dvdt[j * ND + d], t);
            }
            double dr = dot<ND>(dv, gx);
            double psi = diffusion<ND>(dx, ri, rj, ps.c, ps.c, f.h, f.h, gx, f.delta, f.has_delta);
            acc(f, ps.drhodt[i], mass * (dr * cont_coeff(ri, rj, f.S) + psi / rj));
            acc(f, ps.drhodt[j], mass * (dr * cont_coeff(rj, ri, f.S) - psi / ri));
            break;
        }
        case GC_PFN_CAUCHY_FLUID: {
            const double* vi = &ps.v[i * ND];
            const double* vj = &ps.v[j * ND];
            double ri = ps.rho[i], rj = ps.rho[j];
            double mass = ps.mass;
            double dv[ND], hv[ND];
            vdiff<ND>(vi, vj, dv);
            double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, ps.c, ps.c);
            cauchy<ND>(&ps.stress[i * ns], &ps.stress[j * ns], ns, ri, rj, gx, hv);
            for (int d = 0; d < ND; ++d) {
                double t = mass * (hv[d] - piv * gx[d]);
                acc(f, ps.dvdt[i * ND + d], t);
                dec(f, ps.dvdt[j * ND + d], t);
            }
            double dr = dot<ND>(dv, gx);
            double psi = diffusion<ND>(dx, ri, rj, ps.c, ps.c, f.h, f.h, gx, f.delta, f.has_delta);
            acc(f, ps.drhodt[i], mass * (dr + psi / rj));
            acc(f, ps.drhodt[j], mass * (dr - psi / ri));
            break;
        }
        case GC_PFN_STRAIN_RATE:
        case GC_PFN_STRAIN_RATE_VORTICITY: {
            double ri = ps.rho[i], rj = ps.rho[j];
            double mass = ps.mass;
            double dv[ND], sr[6], w[3];
            vdiff<ND>(&ps.v[j * ND], &ps.v[i * ND], dv);
            strain_rate_t<ND>(dv, gx, ns, sr);
            double fi = mass / rj, fj = mass / ri;
            for (int k = 0; k < ns; ++k) {
                acc(f, ps.sr[i * ns + k], sr[k] * fi);
                acc(f, ps.sr[j * ns + k], sr[k] * fj);
            }
            if (f.kind == GC_PFN_STRAIN_RATE_VORTICITY) {
                vorticity_t<ND>(dv, gx, w);
                const int nv = ps.nvort;
                for (int k = 0; k < nv; ++k) {
                    acc(f, ps.vort[i * nv + k], w[k] * fi);
                    acc(f, ps.vort[j * nv + k], w[k] * fj);
                }
            }
            break;
        }
        case GC_PFN_COUNT: {
            ps.dvdt[i * ND] += 1.0;
            ps.dvdt[j * ND] += 1.0;
            ps.drhodt[i] += 1.0;
            ps.drhodt[j] += 1.0;
            break;
        }
        case GC_PFN_XSPH: {  // :364-375 with xsph_veladjust src/PairwisePhysics.jl:268-270
            double ri = ps.rho[i], rj = ps.rho[j], den = ri + rj;
            for (int d = 0; d < ND; ++d) {
                double du = (((-f.alpha) * (ps.v[i * ND + d] - ps.v[j * ND + d])) * w) / den;
                ps.vadj[i * ND + d] = ps.vadj[i * ND + d] + du * ps.mass;
                ps.vadj[j * ND + d] = ps.vadj[j * ND + d] - du * ps.mass;
            }
            break;
        }
        default:
            break;
    }
}

// ------------------------------------------------------ coupled functors
// src/PairwiseFunctors.jl: generic one-sided :37/:97/:193; dynamic
// :53/:111/:222/:334; static :210/:322; ghost Cauchy :286; counting (tests).
template <int ND>
void pfn_coupled(const Pfn& f, Sys& a, const BView& b, int64_t i, int64_t j, const double* dx,
                 const double* gx, double w, int* err) {
    const int ns = a.ns;
    const double* vi = &a.v[i * ND];
    if (f.kind == GC_PFN_NEIGHBOR_COUNT) {  // NeighborCountFn :455-460 (count extra)
        b.sys->drhodt[j] += 1.0;
        return;
    }
    if (f.kind == GC_PFN_INTERPOLATE) {
        // InterpolateFieldFn(ps_a, ps_b::VirtualParticleSystem) :424-428:
        // f_b[j] += kw·f_a[i] with kw = w·(m_a/ρ_a[i]); w_sum[j] += kw
        Sys& bs = *b.sys;
        const double kw = w * (a.mass / a.rho[i]);
        if (f.imask & (1 << GC_FIELD_V))
            for (int d = 0; d < ND; ++d) bs.v[j * ND + d] = bs.v[j * ND + d] + kw * a.v[i * ND + d];
        if (f.imask & (1 << GC_FIELD_RHO)) bs.rho[j] = bs.rho[j] + kw * a.rho[i];
        if (f.imask & (1 << GC_FIELD_STRESS))
            for (int q = 0; q < ns; ++q) bs.stress[j * ns + q] = bs.stress[j * ns + q] + kw * a.stress[i * ns + q];
        if (f.iwsum) b.virt->wsum[j] = b.virt->wsum[j] + kw;
        return;
    }
    if (f.kind == GC_PFN_XSPH) {
        // generic coupled XSPHPfn :378-389 for every system_b: its stored v and
        // rho (a wrapper forwards to the wrapped system), and the write goes to
        // ps_b.v_adjustment[j] -- for a ghost system that property is the
        // SOURCE's array (src/GhostParticles.jl:226-236), indexed by the ghost
        // index j; beyond the source's length the reference writes out of bounds
        double ri = a.rho[i], rj = b.rho[j], den = ri + rj;
        double* adj_b = nullptr;
        if (b.type == H_GHOST) {
            if (j >= b.sys->n) {
                *err = 1;
                return;
            }
        }
        adj_b = b.sys->vadj.data();
        for (int d = 0; d < ND; ++d) {
            double du = (((-f.alpha) * (vi[d] - b.v[j * ND + d])) * w) / den;
            a.vadj[i * ND + d] = a.vadj[i * ND + d] + du * b.mass;
            adj_b[j * ND + d] = adj_b[j * ND + d] - du * a.mass;
        }
        return;
    }
    if (f.kind == GC_PFN_COUNT) {
        a.dvdt[i * ND] += 1.0;
        a.drhodt[i] += 1.0;
        b.sys->dvdt[j * ND] += 1.0;
        b.sys->drhodt[j] += 1.0;
        return;
    }
    if (b.type == H_DYN) {
        double tmp[ND];
        for (int d = 0; d < ND; ++d) tmp[d] = a.x[i * ND + d] - b.point[d];
        double da = dot<ND>(tmp, b.normal);
        for (int d = 0; d < ND; ++d) tmp[d] = b.x[j * ND + d] - b.point[d];
        double db = dot<ND>(tmp, b.normal);
        double m = -jmin(b.beta, std::fabs(db / da));
        double vj[ND];
        for (int d = 0; d < ND; ++d) vj[d] = m * vi[d];
        double ri = a.rho[i];
        double mass = a.mass;
        switch (f.kind) {
            case GC_PFN_FLUID: {
                double pi_ = a.p[i];
                double dv[ND];
                vdiff<ND>(vi, vj, dv);
                double piv = art_visc<ND>(dx, dv, f.h, ri, ri, f.alpha, f.beta, a.c, a.c);
                double dh = pressure_coeff(pi_, pi_, ri, ri, f.S);
                double s = mass * (dh - piv);
                for (int d = 0; d < ND; ++d) acc(f, a.dvdt[i * ND + d], s * gx[d]);
                double dr = dot<ND>(dv, gx);
                double psi = diffusion<ND>(dx, ri, ri, a.c, a.c, f.h, f.h, gx, f.delta, f.has_delta);
                acc(f, a.drhodt[i], mass * (dr * cont_coeff(ri, ri, f.S) + psi / ri));
                break;
            }
            case GC_PFN_CAUCHY_FLUID: {
                double dv[ND], hv[ND];
                vdiff<ND>(vi, vj, dv);
                double piv = art_visc<ND>(dx, dv, f.h, ri, ri, f.alpha, f.beta, a.c, a.c);
                const double* si = &a.stress[i * ns];
                cauchy<ND>(si, si, ns, ri, ri, gx, hv);
                for (int d = 0; d < ND; ++d)
                    acc(f, a.dvdt[i * ND + d], mass * (hv[d] - piv * gx[d]));
                double dr = dot<ND>(dv, gx);
                double psi = diffusion<ND>(dx, ri, ri, a.c, a.c, f.h, f.h, gx, f.delta, f.has_delta);
                acc(f, a.drhodt[i], mass * (dr + psi / ri));
                break;
            }
            case GC_PFN_STRAIN_RATE:
            case GC_PFN_STRAIN_RATE_VORTICITY: {
                double dv[ND], sr[6], w[3];
                vdiff<ND>(vj, vi, dv);
                strain_rate_t<ND>(dv, gx, ns, sr);
                double fi = mass / ri;
                for (int k = 0; k < ns; ++k) acc(f, a.sr[i * ns + k], sr[k] * fi);
                if (f.kind == GC_PFN_STRAIN_RATE_VORTICITY) {
                    vorticity_t<ND>(dv, gx, w);
                    for (int k = 0; k < a.nvort; ++k)
                        acc(f, a.vort[i * a.nvort + k], w[k] * fi);
                }
                break;
            }
        }
        return;
    }
    const double* vj = &b.v[j * ND];
    double ri = a.rho[i], rj = b.rho[j];
    if (b.type == H_STATIC && (f.kind == GC_PFN_FLUID || f.kind == GC_PFN_CAUCHY_FLUID)) {
        double dv[ND];
        vdiff<ND>(vi, vj, dv);
        double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, a.c, a.c);
        double rf = lennard_jones<ND>(dx, b.ljcut, a.c);
        double s = (-b.mass) * piv;
        for (int d = 0; d < ND; ++d) acc(f, a.dvdt[i * ND + d], (s * gx[d] + rf * dx[d]));
        return;
    }
    if (f.kind == GC_PFN_FLUID_SOLID) {
        // FluidSolidPfn :494-519: the two-sided fluid form with the fluid's
        // pressure p_i on both sides of the pressure term, no surface tension
        Sys& bs = *b.sys;
        double pi_ = a.p[i];
        double dv[ND];
        vdiff<ND>(vi, vj, dv);
        double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, a.c, bs.c);
        double dh = pressure_coeff(pi_, pi_, ri, rj, f.S);
        double c = dh - piv;
        for (int d = 0; d < ND; ++d) {
            double t = c * gx[d];
            acc(f, a.dvdt[i * ND + d], b.mass * t);
            dec(f, bs.dvdt[j * ND + d], a.mass * t);
        }
        double dr = dot<ND>(dv, gx);
        double psi = diffusion<ND>(dx, ri, rj, a.c, bs.c, f.h, f.h, gx, f.delta, f.has_delta);
        acc(f, a.drhodt[i], b.mass * (dr * cont_coeff(ri, rj, f.S) + psi / rj));
        acc(f, bs.drhodt[j], a.mass * (dr * cont_coeff(rj, ri, f.S) - psi / ri));
        return;
    }
    if (f.kind == GC_PFN_FLUID && b.type == H_SYS && a.kind == GC_SYS_FLUID && b.sys->kind == GC_SYS_FLUID) {
        // two-sided fluid x fluid (multiphase) :173-190: both systems' rates,
        // each side weighted by the other side's mass, mean sound speed
        Sys& bs = *b.sys;
        double pi_ = a.p[i], pj = b.p[j];
        double dv[ND];
        vdiff<ND>(vi, vj, dv);
        double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, a.c, bs.c);
        double dh = pressure_coeff(pi_, pj, ri, rj, f.S);
        // artificial_surface_tension_coeff src/PairwisePhysics.jl:286-290
        double ast = f.has_eps ? f.eps * pressure_coeff(std::fabs(pi_), std::fabs(pj), ri, rj, 1) : 0.0;
        double c = dh + ast - piv;
        for (int d = 0; d < ND; ++d) {
            double t = c * gx[d];
            acc(f, a.dvdt[i * ND + d], b.mass * t);
            dec(f, bs.dvdt[j * ND + d], a.mass * t);
        }
        double dr = dot<ND>(dv, gx);
        double psi = diffusion<ND>(dx, ri, rj, a.c, bs.c, f.h, f.h, gx, f.delta, f.has_delta);
        acc(f, a.drhodt[i], b.mass * (dr * cont_coeff(ri, rj, f.S) + psi / rj));
        acc(f, bs.drhodt[j], a.mass * (dr * cont_coeff(rj, ri, f.S) - psi / ri));
        return;
    }
    switch (f.kind) {
        case GC_PFN_FLUID: {  // generic one-sided :193
            double pi_ = a.p[i], pj = b.p[j];
            double dv[ND];
            vdiff<ND>(vi, vj, dv);
            double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, a.c, a.c);
            double dh = pressure_coeff(pi_, pj, ri, rj, f.S);
            double s = b.mass * (dh - piv);
            for (int d = 0; d < ND; ++d) acc(f, a.dvdt[i * ND + d], s * gx[d]);
            double dr = dot<ND>(dv, gx);
            double psi = diffusion<ND>(dx, ri, rj, a.c, a.c, f.h, f.h, gx, f.delta, f.has_delta);
            acc(f, a.drhodt[i], b.mass * (dr * cont_coeff(ri, rj, f.S) + psi / rj));
            break;
        }
        case GC_PFN_CAUCHY_FLUID: {  // ghost one-sided :286
            double dv[ND], hv[ND];
            vdiff<ND>(vi, vj, dv);
            double piv = art_visc<ND>(dx, dv, f.h, ri, rj, f.alpha, f.beta, a.c, b.c);
            cauchy<ND>(&a.stress[i * ns], &b.stress[j * ns], ns, ri, rj, gx, hv);
            for (int d = 0; d < ND; ++d)
                acc(f, a.dvdt[i * ND + d], b.mass * (hv[d] - piv * gx[d]));
            double dr = dot<ND>(dv, gx);
            double psi = diffusion<ND>(dx, ri, rj, a.c, a.c, f.h, f.h, gx, f.delta, f.has_delta);
            acc(f, a.drhodt[i], b.mass * (dr + psi / rj));
            break;
        }
        case GC_PFN_STRAIN_RATE:
        case GC_PFN_STRAIN_RATE_VORTICITY: {  // generic one-sided :37/:97
            double dv[ND], sr[6], w[3];
            vdiff<ND>(vj, vi, dv);
            strain_rate_t<ND>(dv, gx, ns, sr);
            double fi = b.mass / rj;
            for (int k = 0; k < ns; ++k) acc(f, a.sr[i * ns + k], sr[k] * fi);
            if (f.kind == GC_PFN_STRAIN_RATE_VORTICITY) {
                vorticity_t<ND>(dv, gx, w);
                for (int k = 0; k < a.nvort; ++k)
                    acc(f, a.vort[i * a.nvort + k], w[k] * fi);
            }
            break;
        }
    }
}

// ----------------------------------------------------------------- pairs
// src/Interaction.jl:543-557 (_pair_self!) and :717-732 (_pair_coupled!)
template <int ND>
inline void pair_self(const Pfn& f, const Kern& k, Sys& ps, int64_t i, int64_t j, double h,
                      double cutoff_sq) {
    double dx[ND];
    for (int d = 0; d < ND; ++d) dx[d] = ps.x[i * ND + d] - ps.x[j * ND + d];
    double r_sq = dot<ND>(dx, dx);
    if (r_sq < cutoff_sq) {
        double r = std::sqrt(r_sq);
        double q = r / h;
        double gc = kernel_dw_dq(k, q) / (r * h);
        double w = f.kind == GC_PFN_XSPH ? kernel_w(k, q) : 0.0;
        double gx[ND];
        for (int d = 0; d < ND; ++d) gx[d] = g_mag_inputs ? std::fabs(gc * dx[d]) : gc * dx[d];
        pfn_self<ND>(f, ps, i, j, dx, gx, w);
    }
}

template <int ND>
inline void pair_coupled(const Pfn& f, const Kern& k, Sys& a, const BView& b, int64_t i, int64_t j,
                         double h, double cutoff_sq, int* err) {
    double dx[ND];
    for (int d = 0; d < ND; ++d) dx[d] = a.x[i * ND + d] - b.x[j * ND + d];
    double r_sq = dot<ND>(dx, dx);
    if (r_sq < cutoff_sq) {
        double r = std::sqrt(r_sq);
        double q = r / h;
        double gc = kernel_dw_dq(k, q) / (r * h);
        double w = (f.kind == GC_PFN_XSPH || f.kind == GC_PFN_INTERPOLATE) ? kernel_w(k, q) : 0.0;
        double gx[ND];
        for (int d = 0; d < ND; ++d) gx[d] = g_mag_inputs ? std::fabs(gc * dx[d]) : gc * dx[d];
        pfn_coupled<ND>(f, a, b, i, j, dx, gx, w, err);
    }
}

// Cell-range helper: cs is 1-based CSR (cs[c] for c in 1..ncells+1 stored at cs[c-1]).
inline int64_t CS(const std::vector<int64_t>& cs, int64_t c1) { return cs[(size_t)(c1 - 1)]; }

// ---------------------------------------------------------------- sweeps
// src/Interaction.jl:393-439 (2-D self, 6 colours), :477-541 (3-D, 18 colours)
template <int ND>
void sweep_self(oracle_ctx* ctx, Inter& it, const Pfn& f) {
    Sys& ps = ctx->sys[it.a];
    Kern k = make_kernel(it.kk, ND, it.H);
    const double h = it.H;
    const double cutoff_sq = it.cell * it.cell;
    const std::vector<int64_t>& cs = it.cs;
    if (ND == 2) {
        const int64_t ny = it.ng[1], nx = it.ng[0];
        for (int colour = 0; colour < 6; ++colour) {
            int64_t bx = colour / 3 + 2, by = colour % 3 + 2;
            int64_t nax = bx <= nx - 1 ? (nx - 1 - bx) / 2 + 1 : 0;
            int64_t nay = by <= ny - 1 ? (ny - 1 - by) / 3 + 1 : 0;
            int64_t total = nax * nay;
#pragma omp parallel for schedule(static) num_threads(ctx->threads)
            for (int64_t flat = 1; flat <= total; ++flat) {
                int64_t sx = (flat - 1) / nay, sy = (flat - 1) % nay;
                int64_t cx = bx + sx * 2, cy = by + sy * 3;
                int64_t cell = (cx - 1) * ny + cy;
                int64_t pstart = CS(cs, cell), pend_same = CS(cs, cell + 1), pend_next = CS(cs, cell + 2);
                int64_t nb = cell + ny - 1;
                int64_t nps = CS(cs, nb), npe = CS(cs, nb + 3);
                for (int64_t pi_ = pstart; pi_ <= pend_same - 1; ++pi_) {
                    for (int64_t pj = pi_ + 1; pj <= pend_next - 1; ++pj)
                        pair_self<ND>(f, k, ps, pi_ - 1, pj - 1, h, cutoff_sq);
                    for (int64_t pj = nps; pj <= npe - 1; ++pj)
                        pair_self<ND>(f, k, ps, pi_ - 1, pj - 1, h, cutoff_sq);
                }
            }
        }
    } else {
        const int64_t nz = it.ng[2], ny = it.ng[1], nx = it.ng[0], nyz = ny * nz;
        const int64_t off[4] = {nz - 1, nyz - nz - 1, nyz - 1, nyz + nz - 1};
        for (int colour = 0; colour < 18; ++colour) {
            int64_t bx = colour / 9 + 2, by = (colour % 9) / 3 + 2, bz = colour % 3 + 2;
            int64_t nax = bx <= nx - 1 ? (nx - 1 - bx) / 2 + 1 : 0;
            int64_t nay = by <= ny - 1 ? (ny - 1 - by) / 3 + 1 : 0;
            int64_t naz = bz <= nz - 1 ? (nz - 1 - bz) / 3 + 1 : 0;
            int64_t nayz = nay * naz, total = nax * nayz;
#pragma omp parallel for schedule(static) num_threads(ctx->threads)
            for (int64_t flat = 1; flat <= total; ++flat) {
                int64_t sx = (flat - 1) / nayz, rem = (flat - 1) % nayz;
                int64_t sy = rem / naz, sz = rem % naz;
                int64_t cx = bx + sx * 2, cy = by + sy * 3, cz = bz + sz * 3;
                int64_t cell = (cx - 1) * nyz + (cy - 1) * nz + cz;
                int64_t pstart = CS(cs, cell), pend = CS(cs, cell + 1), pend_next = CS(cs, cell + 2);
                for (int64_t pi_ = pstart; pi_ <= pend - 1; ++pi_)
                    for (int64_t pj = pi_ + 1; pj <= pend_next - 1; ++pj)
                        pair_self<ND>(f, k, ps, pi_ - 1, pj - 1, h, cutoff_sq);
                for (int dir = 0; dir < 4; ++dir) {
                    int64_t nb = cell + off[dir];
                    int64_t nps = CS(cs, nb), npe = CS(cs, nb + 3);
                    for (int64_t pi_ = pstart; pi_ <= pend - 1; ++pi_)
                        for (int64_t pj = nps; pj <= npe - 1; ++pj)
                            pair_self<ND>(f, k, ps, pi_ - 1, pj - 1, h, cutoff_sq);
                }
            }
        }
    }
}

int make_view(oracle_ctx* ctx, int handle, BView* out);

// system_a of an interaction: a system, or (InterpolateFieldFn from ghosts,
// Trapdoor.jl's ghost_bottom) a ghost system's current arrays with its
// source's mass and sound speed
Sys& system_a(oracle_ctx* ctx, Inter& it) {
    if (it.ag < 0) return ctx->sys[it.a];
    const Ghost& g = ctx->ghosts[it.ag];
    const Sys& src = ctx->sys[g.src];
    Sys& p = it.proxy;
    p.kind = src.kind;
    p.nd = src.nd;
    p.ns = src.ns;
    p.n = g.n;
    p.mass = src.mass;
    p.c = src.c;
    const size_t n = (size_t)g.n, nd = (size_t)src.nd, ns = (size_t)src.ns;
    p.x.assign(g.x.begin(), g.x.begin() + n * nd);
    p.v.assign(g.v.begin(), g.v.begin() + n * nd);
    p.rho.assign(g.rho.begin(), g.rho.begin() + n);
    if (g.ex_stress) p.stress.assign(g.stress.begin(), g.stress.begin() + n * ns);
    else p.stress.assign(n * ns, 0.0);
    if (g.ex_p) p.p.assign(g.p.begin(), g.p.begin() + n);
    else p.p.assign(n, 0.0);
    return p;
}

// src/Interaction.jl:600-645 (2-D coupled, 9 colours), :660-715 (3-D, 27 colours)
template <int ND>
int sweep_coupled(oracle_ctx* ctx, Inter& it, const Pfn& f, const BView& b) {
    Sys& a = system_a(ctx, it);
    int err = 0;
    // a ghost's XSPH writes land in its source's array at ghost indices, which
    // a-side writes of other cells of the colour may also touch: one thread
    const int threads = (f.kind == GC_PFN_XSPH && b.type == H_GHOST) ? 1 : ctx->threads;
    Kern k = make_kernel(it.kk, ND, it.H);
    const double h = it.H, cutoff = it.cell;
    const double cutoff_sq = it.cell * it.cell;
    const std::vector<int64_t>& cs = it.cs;
    const std::vector<int64_t>& csa = it.csa;
    int64_t cmin[3], cmax[3];
    for (int d = 0; d < ND; ++d) {
        floor_int((it.mina[d] - it.ming[d]) / cutoff, &cmin[d]);
        floor_int((it.maxa[d] - it.ming[d]) / cutoff, &cmax[d]);
        cmin[d] += 1;
        cmax[d] += 1;
    }
    if (ND == 2) {
        const int64_t ny = it.ng[1];
        for (int colour = 0; colour < 9; ++colour) {
            int64_t bx = colour / 3 + cmin[0], by = colour % 3 + cmin[1];
            int64_t nax = bx <= cmax[0] ? (cmax[0] - bx) / 3 + 1 : 0;
            int64_t nay = by <= cmax[1] ? (cmax[1] - by) / 3 + 1 : 0;
            int64_t total = nax * nay;
#pragma omp parallel for schedule(static) num_threads(threads)
            for (int64_t flat = 1; flat <= total; ++flat) {
                int64_t sx = (flat - 1) / nay, sy = (flat - 1) % nay;
                int64_t cx = bx + sx * 3, cy = by + sy * 3;
                int64_t cell = (cx - 1) * ny + cy;
                int64_t as = CS(csa, cell), ae = CS(csa, cell + 1);
                for (int64_t pi_ = as; pi_ <= ae - 1; ++pi_)
                    for (int64_t dcx = -1; dcx <= 1; ++dcx) {
                        int64_t nb = cell + dcx * ny - 1;
                        int64_t bs = CS(cs, nb), be = CS(cs, nb + 3);
                        for (int64_t pj = bs; pj <= be - 1; ++pj)
                            pair_coupled<ND>(f, k, a, b, pi_ - 1, pj - 1, h, cutoff_sq, &err);
                    }
            }
        }
    } else {
        const int64_t nz = it.ng[2], ny = it.ng[1], nyz = ny * nz;
        for (int colour = 0; colour < 27; ++colour) {
            int64_t bx = colour / 9 + cmin[0], by = (colour % 9) / 3 + cmin[1], bz = colour % 3 + cmin[2];
            int64_t nax = bx <= cmax[0] ? (cmax[0] - bx) / 3 + 1 : 0;
            int64_t nay = by <= cmax[1] ? (cmax[1] - by) / 3 + 1 : 0;
            int64_t naz = bz <= cmax[2] ? (cmax[2] - bz) / 3 + 1 : 0;
            int64_t nayz = nay * naz, total = nax * nayz;
#pragma omp parallel for schedule(static) num_threads(threads)
            for (int64_t flat = 1; flat <= total; ++flat) {
                int64_t sx = (flat - 1) / nayz, rem = (flat - 1) % nayz;
                int64_t sy = rem / naz, sz = rem % naz;
                int64_t cx = bx + sx * 3, cy = by + sy * 3, cz = bz + sz * 3;
                int64_t cell = (cx - 1) * nyz + (cy - 1) * nz + cz;
                int64_t as = CS(csa, cell), ae = CS(csa, cell + 1);
                for (int64_t pi_ = as; pi_ <= ae - 1; ++pi_)
                    for (int64_t dcx = -1; dcx <= 1; ++dcx)
                        for (int64_t dcy = -1; dcy <= 1; ++dcy) {
                            int64_t nb = cell + dcx * nyz + dcy * nz - 1;
                            int64_t bs = CS(cs, nb), be = CS(cs, nb + 3);
                            for (int64_t pj = bs; pj <= be - 1; ++pj)
                                pair_coupled<ND>(f, k, a, b, pi_ - 1, pj - 1, h, cutoff_sq, &err);
                        }
            }
        }
    }
    return err ? GC_ERR_CAPACITY : GC_OK;
}

// ------------------------------------------------------------------- grid
// src/Interaction.jl:131-251
int cell_1idx(const double* x, int nd, const double* ming, double dcell, const int64_t* ng,
              int64_t* out) {
    int64_t flat = 0, stride = 1;
    for (int d = nd - 1; d >= 0; --d) {
        int64_t cd;
        if (!floor_int((x[d] - ming[d]) / dcell, &cd)) return GC_ERR_NONFINITE;
        flat += cd * stride;
        stride *= ng[d];
    }
    *out = flat + 1;
    return GC_OK;
}

int populate_sorted(std::vector<int64_t>& cs, const double* x, int64_t n, int nd, const double* ming,
                    double cutoff, const int64_t* ng) {
    int64_t ncells = (int64_t)cs.size() - 1;
    int64_t prev = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t cell;
        int st = cell_1idx(&x[i * nd], nd, ming, cutoff, ng, &cell);
        if (st) return st;
        if (cell != prev) {
            if (cell < 1 || cell > ncells) return GC_ERR_CAPACITY;
            cs[(size_t)(cell - 1)] = i + 1;
            prev = cell;
        }
    }
    cs[(size_t)ncells] = n + 1;
    for (int64_t c = ncells; c >= 1; --c)
        if (cs[(size_t)(c - 1)] == 0) cs[(size_t)(c - 1)] = cs[(size_t)c];
    return GC_OK;
}

void bbox(const double* x, int64_t n, int nd, double* mn, double* mx, bool init) {
    int64_t start = 0;
    if (init) {
        for (int d = 0; d < nd; ++d) mn[d] = mx[d] = x[d];
        start = 1;
    }
    for (int64_t i = start; i < n; ++i)
        for (int d = 0; d < nd; ++d) {
            mn[d] = jmin(mn[d], x[i * nd + d]);
            mx[d] = jmax(mx[d], x[i * nd + d]);
        }
}

int create_grid(oracle_ctx* ctx, Inter& it) {
    Sys& a = system_a(ctx, it);
    const int nd = a.nd;
    const double cutoff = it.cell;
    double mn[3], mx[3];
    bbox(a.x.data(), a.n, nd, mn, mx, true);
    BView b{};
    if (it.b >= 0) {
        int st = make_view(ctx, it.b, &b);
        if (st) return st;
        for (int d = 0; d < nd; ++d) {
            it.mina[d] = mn[d];
            it.maxa[d] = mx[d];
        }
        bbox(b.x, b.n, nd, mn, mx, false);
    }
    for (int d = 0; d < nd; ++d) {
        double raw = mn[d] - 2.0 * cutoff;
        it.ming[d] = std::floor(raw / cutoff) * cutoff;
        double maxg = mx[d] + 2.0 * cutoff;
        int64_t ngd;
        if (!floor_int((maxg - it.ming[d]) / cutoff, &ngd)) return fail(ctx, GC_ERR_NONFINITE, "non-finite grid extent");
        it.ng[d] = ngd + 1;
    }
    int64_t ncells = 1;
    for (int d = 0; d < nd; ++d) ncells *= it.ng[d];
    if (ncells > (int64_t)1 << 34) return fail(ctx, GC_ERR_CAPACITY, "grid too large");
    it.cs.assign((size_t)ncells + 1, 0);
    int st;
    if (it.b < 0) {
        st = populate_sorted(it.cs, a.x.data(), a.n, nd, it.ming, cutoff, it.ng);
    } else {
        it.csa.assign((size_t)ncells + 1, 0);
        st = populate_sorted(it.csa, a.x.data(), a.n, nd, it.ming, cutoff, it.ng);
        if (!st) st = populate_sorted(it.cs, b.x, b.n, nd, it.ming, cutoff, it.ng);
    }
    if (st) return fail(ctx, st, "grid population failed (non-finite position or cell outside grid)");
    it.grid = true;
    return GC_OK;
}

// ------------------------------------------------------------------- sort
// src/Sorting.jl:157-195; stable lexicographic order of floor(x/cutoff).
int sort_keys(const double* x, int64_t n, int nd, double cutoff, std::vector<int64_t>& keys) {
    keys.resize((size_t)n * nd);
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < nd; ++d)
            if (!floor_int(x[i * nd + d] / cutoff, &keys[(size_t)(i * nd + d)])) return GC_ERR_NONFINITE;
    return GC_OK;
}

inline bool lt_key(const int64_t* a, const int64_t* b, int nd) {
    for (int d = 0; d < nd; ++d)
        if (a[d] != b[d]) return a[d] < b[d];
    return false;
}

template <class T>
void apply_perm(std::vector<T>& arr, const std::vector<int64_t>& perm, int comps) {
    if (arr.empty() || comps == 0) return;
    std::vector<T> scratch(arr.size());
    int64_t n = (int64_t)perm.size();
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < comps; ++k) scratch[(size_t)(i * comps + k)] = arr[(size_t)(perm[i] * comps + k)];
    for (int64_t i = 0; i < n * comps; ++i) arr[(size_t)i] = scratch[(size_t)i];
}

// Returns 1 if a permutation was applied, 0 for the fast path; <0 on error.
int sort_order(const double* x, int64_t n, int nd, double cutoff, std::vector<int64_t>& perm) {
    perm.resize((size_t)n);
    std::iota(perm.begin(), perm.end(), 0);
    if (n <= 1) return 0;
    std::vector<int64_t> keys;
    if (sort_keys(x, n, nd, cutoff, keys)) return -GC_ERR_NONFINITE;
    bool sorted = true;
    for (int64_t i = 0; i + 1 < n; ++i)
        if (lt_key(&keys[(size_t)((i + 1) * nd)], &keys[(size_t)(i * nd)], nd)) {
            sorted = false;
            break;
        }
    if (sorted) return 0;
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t p, int64_t q) {
        return lt_key(&keys[(size_t)(p * nd)], &keys[(size_t)(q * nd)], nd);
    });
    return 1;
}

// ------------------------------------------------- magnitude shadows
// Test infrastructure, not part of the reference: with track_mag on, each
// rate field (dvdt, drhodt, strain rate, vorticity) has a shadow holding
// |initial value| + Σ|every term added since|, the per-particle scale on
// which a result summed in another order is compared.
void mag_set(const std::vector<double>& f, std::vector<double>& m) {
    m.resize(f.size());
    for (size_t k = 0; k < f.size(); ++k) m[k] = std::fabs(f[k]);
}

void mag_ensure(Sys& s) {
    if (s.mstr.size() != s.stress.size()) s.mstr.assign(s.stress.size(), 0.0);
    if (s.mstrain.size() != s.strain.size()) s.mstrain.assign(s.strain.size(), 0.0);
    if (s.mvi.size() != s.v.size()) s.mvi.assign(s.v.size(), 0.0);
    if (s.mrhoi.size() != s.rho.size()) s.mrhoi.assign(s.rho.size(), 0.0);
    if (s.mxi.size() != s.x.size()) s.mxi.assign(s.x.size(), 0.0);
    if (s.mdvdt.size() != s.dvdt.size()) mag_set(s.dvdt, s.mdvdt);
    if (s.mdrhodt.size() != s.drhodt.size()) mag_set(s.drhodt, s.mdrhodt);
    if (s.msr.size() != s.sr.size()) mag_set(s.sr, s.msr);
    if (s.mvort.size() != s.vort.size()) mag_set(s.vort, s.mvort);
}

void mag_swap(Sys& s) {
    s.dvdt.swap(s.mdvdt);
    s.drhodt.swap(s.mdrhodt);
    s.sr.swap(s.msr);
    s.vort.swap(s.mvort);
}

void mag_permute(Sys& s, const std::vector<int64_t>& perm);

void permute_system(Sys& s, const std::vector<int64_t>& perm) {
    const int nd = s.nd, ns = s.ns;
    apply_perm(s.x, perm, nd);
    apply_perm(s.id, perm, 1);
    apply_perm(s.v, perm, nd);
    apply_perm(s.vadj, perm, nd);
    apply_perm(s.rho, perm, 1);
    apply_perm(s.dvdt, perm, nd);
    apply_perm(s.drhodt, perm, 1);
    if (s.has_p()) apply_perm(s.p, perm, 1);
    if (s.has_stress()) {
        apply_perm(s.stress, perm, ns);
        apply_perm(s.sr, perm, ns);
    }
    if (s.is_ep()) {
        apply_perm(s.vort, perm, s.nvort);
        apply_perm(s.strain, perm, ns);
        apply_perm(s.strainp, perm, ns);
    }
    mag_permute(s, perm);
}

void mag_permute(Sys& s, const std::vector<int64_t>& perm) {
    if (s.mstr.size() == s.stress.size() && !s.mstr.empty()) apply_perm(s.mstr, perm, s.ns);
    if (s.mstrain.size() == s.strain.size() && !s.mstrain.empty()) apply_perm(s.mstrain, perm, s.ns);
    if (s.mvi.size() == s.v.size() && !s.mvi.empty()) apply_perm(s.mvi, perm, s.nd);
    if (s.mrhoi.size() == s.rho.size() && !s.mrhoi.empty()) apply_perm(s.mrhoi, perm, 1);
    if (s.mxi.size() == s.x.size() && !s.mxi.empty()) apply_perm(s.mxi, perm, s.nd);
    if (s.mdvdt.size() == s.dvdt.size() && !s.mdvdt.empty()) apply_perm(s.mdvdt, perm, s.nd);
    if (s.mdrhodt.size() == s.drhodt.size() && !s.mdrhodt.empty()) apply_perm(s.mdrhodt, perm, 1);
    if (s.msr.size() == s.sr.size() && !s.msr.empty()) apply_perm(s.msr, perm, s.ns);
    if (s.mvort.size() == s.vort.size() && !s.mvort.empty()) apply_perm(s.mvort, perm, s.nvort);
}

int sort_system(Sys& s, double cutoff, std::vector<int64_t>* perm_out) {
    std::vector<int64_t> perm;
    int r = sort_order(s.x.data(), s.n, s.nd, cutoff, perm);
    if (r < 0) return -r;
    if (r == 1) {
        const int nd = s.nd, ns = s.ns;
        apply_perm(s.x, perm, nd);
        apply_perm(s.id, perm, 1);
        apply_perm(s.v, perm, nd);
        apply_perm(s.vadj, perm, nd);
        apply_perm(s.rho, perm, 1);
        apply_perm(s.dvdt, perm, nd);
        apply_perm(s.drhodt, perm, 1);
        if (s.has_p()) apply_perm(s.p, perm, 1);
        if (s.has_stress()) {
            apply_perm(s.stress, perm, ns);
            apply_perm(s.sr, perm, ns);
        }
        if (s.is_ep()) {
            apply_perm(s.vort, perm, s.nvort);
            apply_perm(s.strain, perm, ns);
            apply_perm(s.strainp, perm, ns);
        }
        mag_permute(s, perm);
    }
    if (perm_out) *perm_out = perm;
    return GC_OK;
}

// Ghost sort: permutes (x, v, rho, idx_original, idx_boundary, extras); the
// cached normals are not in the reference's permuted-array list
// (src/Sorting.jl:33-40) and stay in generation order.
int sort_ghost(Ghost& g, int nd, int ns, double cutoff, std::vector<int64_t>* perm_out) {
    std::vector<int64_t> perm;
    int r = sort_order(g.x.data(), g.n, nd, cutoff, perm);
    if (r < 0) return -r;
    if (r == 1) {
        apply_perm(g.x, perm, nd);
        apply_perm(g.v, perm, nd);
        apply_perm(g.rho, perm, 1);
        apply_perm(g.io, perm, 1);
        apply_perm(g.ib, perm, 1);
        if (g.ex_p) apply_perm(g.p, perm, 1);
        if (g.ex_stress) apply_perm(g.stress, perm, ns);
    }
    if (perm_out) *perm_out = perm;
    return GC_OK;
}

// ----------------------------------------------------------------- ghosts
// src/GhostParticles.jl:344-392
void generate_ghosts(oracle_ctx* ctx, Ghost& g) {
    Sys& ps = ctx->sys[g.src];
    const int nd = ps.nd;
    int64_t total = 0;
    for (int b = 0; b < g.nplanes; ++b)
        for (int64_t i = 0; i < ps.n; ++i) {
            double tmp[3];
            for (int d = 0; d < nd; ++d) tmp[d] = ps.x[i * nd + d] - g.pp[b * nd + d];
            double da = nd == 2 ? dot<2>(tmp, &g.pn[b * nd]) : dot<3>(tmp, &g.pn[b * nd]);
            if (std::fabs(da) <= g.cutoff && da > 0.0) ++total;
        }
    g.n = total;
    g.x.assign((size_t)total * nd, 0.0);
    g.v.resize((size_t)total * nd);
    g.rho.resize((size_t)total);
    g.io.assign((size_t)total, 0);
    g.ib.assign((size_t)total, 0);
    g.normals.assign((size_t)total * nd, 0.0);
    if (g.ex_p) g.p.resize((size_t)total);
    if (g.ex_stress) g.stress.resize((size_t)total * ps.ns);
    int64_t cur = 0;
    for (int b = 0; b < g.nplanes; ++b)
        for (int64_t i = 0; i < ps.n; ++i) {
            double tmp[3];
            for (int d = 0; d < nd; ++d) tmp[d] = ps.x[i * nd + d] - g.pp[b * nd + d];
            double da = nd == 2 ? dot<2>(tmp, &g.pn[b * nd]) : dot<3>(tmp, &g.pn[b * nd]);
            if (std::fabs(da) <= g.cutoff && da > 0.0) {
                for (int d = 0; d < nd; ++d) g.x[cur * nd + d] = ps.x[i * nd + d] - (2.0 * da) * g.pn[b * nd + d];
                g.io[cur] = i + 1;
                g.ib[cur] = b + 1;
                for (int d = 0; d < nd; ++d) g.normals[cur * nd + d] = g.pn[b * nd + d];
                ++cur;
            }
        }
}

// src/GhostParticles.jl:404-421
void ghost_kinematics(oracle_ctx* ctx, Ghost& g) {
    Sys& ps = ctx->sys[g.src];
    const int nd = ps.nd;
    for (int64_t k = 0; k < g.n; ++k) {
        const double* nrm = &g.normals[k * nd];
        int64_t o = g.io[k] - 1;
        const double* vr = &ps.v[o * nd];
        double dvn = nd == 2 ? dot<2>(vr, nrm) : dot<3>(vr, nrm);
        double s = 2.0 * dvn;
        for (int d = 0; d < nd; ++d) g.v[k * nd + d] = vr[d] - s * nrm[d];
        g.rho[k] = ps.rho[o];
    }
}

// src/GhostParticles.jl:66-110
void householder(const double* s, int ns, const double* n, int nd, double* out) {
    if (ns == 3 || ns == 4) {
        double nx = n[0], ny = n[1];
        int xy = ns == 3 ? 2 : 3;
        double tx = s[0] * nx + s[xy] * ny;
        double ty = s[xy] * nx + s[1] * ny;
        double sc = tx * nx + ty * ny;
        out[0] = s[0] - 4.0 * tx * nx + 4.0 * sc * nx * nx;
        out[1] = s[1] - 4.0 * ty * ny + 4.0 * sc * ny * ny;
        if (ns == 4) out[2] = s[2];
        out[xy] = s[xy] - 2.0 * (tx * ny + nx * ty) + 4.0 * sc * nx * ny;
    } else {
        double nx = n[0], ny = n[1], nz = n[2];
        double tx = s[0] * nx + s[3] * ny + s[4] * nz;
        double ty = s[3] * nx + s[1] * ny + s[5] * nz;
        double tz = s[4] * nx + s[5] * ny + s[2] * nz;
        double sc = tx * nx + ty * ny + tz * nz;
        out[0] = s[0] - 4.0 * tx * nx + 4.0 * sc * nx * nx;
        out[1] = s[1] - 4.0 * ty * ny + 4.0 * sc * ny * ny;
        out[2] = s[2] - 4.0 * tz * nz + 4.0 * sc * nz * nz;
        out[3] = s[3] - 2.0 * (tx * ny + nx * ty) + 4.0 * sc * nx * ny;
        out[4] = s[4] - 2.0 * (tx * nz + nx * tz) + 4.0 * sc * nx * nz;
        out[5] = s[5] - 2.0 * (ty * nz + ny * tz) + 4.0 * sc * ny * nz;
    }
    (void)nd;
}

// src/GhostParticles.jl:112-129,261-278
void update_ghost(oracle_ctx* ctx, Ghost& g, int stage) {
    if (stage < 1 || stage > (int)g.copiers.size()) return;
    Sys& ps = ctx->sys[g.src];
    const int nd = ps.nd, ns = ps.ns;
    for (auto& e : g.copiers[stage - 1].entries) {
        int field = e.first, mode = e.second;
        for (int64_t k = 0; k < g.n; ++k) {
            int64_t o = g.io[k] - 1;
            if (field == GC_FIELD_P) {
                g.p[k] = ps.p[o];
            } else if (field == GC_FIELD_STRESS) {
                if (mode == GC_COPY_HOUSEHOLDER)
                    householder(&ps.stress[o * ns], ns, &g.normals[k * nd], nd, &g.stress[k * ns]);
                else
                    for (int q = 0; q < ns; ++q) g.stress[k * ns + q] = ps.stress[o * ns + q];
            }
            // A :rho copier writes the extras copy, which the first-class rho shadows.
        }
    }
}

// --------------------------------------------------------------- updaters
// src/StateUpdaters.jl
// The magnitude shadows of a plane-strain stress update from the strain
// rate and vorticity shadows (test infrastructure; a no-op unless the
// shadows are kept).
void mag_stress_increment(Sys& ps, int64_t i, double E, double nu, double dt) {
    if (ps.mstr.size() != ps.stress.size() || ps.msr.size() != ps.sr.size() || ps.mvort.size() != ps.vort.size())
        return;
    const double* m = &ps.msr[i * 4];
    const double* s = &ps.stress[i * 4];
    const double D0 = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mxx = m[0] * dt, myy = m[1] * dt, mzz = m[2] * dt, mxy = m[3] * dt;
    const double mw = ps.mvort[i * ps.nvort] * dt;
    double* o = &ps.mstr[i * 4];
    o[0] += D0 * ((1.0 - nu) * mxx + nu * myy + nu * mzz) + 2.0 * std::fabs(s[3]) * mw;
    o[1] += D0 * (nu * mxx + (1.0 - nu) * myy + nu * mzz) + 2.0 * std::fabs(s[3]) * mw;
    o[2] += D0 * (nu * mxx + nu * myy + (1.0 - nu) * mzz);
    o[3] += D0 * (1.0 - 2.0 * nu) * mxy + (std::fabs(s[0]) + std::fabs(s[1])) * mw;
    if (ps.mstrain.size() == ps.strain.size())
        for (int q = 0; q < 4; ++q) ps.mstrain[i * 4 + q] += m[q] * dt;
}

void ep_update(Sys& ps, int64_t i, const Upd& u, double dt) {
    const double E = u.prm[0], nu = u.prm[1], phi = u.prm[2], psi = u.prm[3], coh = u.prm[4];
    mag_stress_increment(ps, i, E, nu, dt);
    double* s = &ps.stress[i * 4];
    const double* er = &ps.sr[i * 4];
    double w = ps.vort[i * ps.nvort];
    double sxx = s[0], syy = s[1], szz = s[2], sxy = s[3];
    double dexx = er[0] * dt, deyy = er[1] * dt, dezz = er[2] * dt, dexy = er[3] * dt;
    double D0 = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double dsxx = D0 * ((1.0 - nu) * dexx + nu * deyy + nu * dezz);
    double dsyy = D0 * (nu * dexx + (1.0 - nu) * deyy + nu * dezz);
    double dszz = D0 * (nu * dexx + nu * deyy + (1.0 - nu) * dezz);
    double dsxy = D0 * (1.0 - 2.0 * nu) * dexy;
    double wdt = w * dt;
    dsxx = dsxx - 2.0 * sxy * wdt;
    dsyy = dsyy + 2.0 * sxy * wdt;
    dsxy = dsxy + (sxx - syy) * wdt;
    double txx = sxx + dsxx, tyy = syy + dsyy, tzz = szz + dszz, txy = sxy + dsxy;
    double sqrt3 = std::sqrt(3.0);
    double sphi = std::sin(phi), cphi = std::cos(phi);
    double a_phi = 2.0 * sphi / (sqrt3 * (3.0 - sphi));
    double k_c = 6.0 * coh * cphi / (sqrt3 * (3.0 - sphi));
    double I1 = txx + tyy + tzz;
    double p3 = I1 / 3.0;
    double s_xx = txx - p3, s_yy = tyy - p3, s_zz = tzz - p3, s_xy = txy;
    double J2 = 0.5 * (s_xx * s_xx + s_yy * s_yy + s_zz * s_zz + 2.0 * (s_xy * s_xy));
    double sqJ2 = std::sqrt(J2);
    double f = a_phi * I1 + sqJ2 - k_c;
    double depxx = 0.0, depyy = 0.0, depzz = 0.0, depxy = 0.0;
    if (f > 0.0) {
        double spsi = std::sin(psi);
        double a_psi = 2.0 * spsi / (sqrt3 * (3.0 - spsi));
        double inv2 = 1.0 / (2.0 * sqJ2);
        double dfxx = a_phi + s_xx * inv2, dfyy = a_phi + s_yy * inv2, dfzz = a_phi + s_zz * inv2;
        double dfxy = s_xy * inv2;
        double dgxx = a_psi + s_xx * inv2, dgyy = a_psi + s_yy * inv2, dgzz = a_psi + s_zz * inv2;
        double dgxy = s_xy * inv2;
        double Dxx = D0 * ((1.0 - nu) * dgxx + nu * dgyy + nu * dgzz);
        double Dyy = D0 * (nu * dgxx + (1.0 - nu) * dgyy + nu * dgzz);
        double Dzz = D0 * (nu * dgxx + nu * dgyy + (1.0 - nu) * dgzz);
        double Dxy = D0 * (1.0 - 2.0 * nu) * dgxy;
        double denom = dfxx * Dxx + dfyy * Dyy + dfzz * Dzz + 2.0 * dfxy * Dxy;
        double dl = f / denom;
        depxx = dl * dgxx;
        depyy = dl * dgyy;
        depzz = dl * dgzz;
        depxy = dl * dgxy;
        dsxx = dsxx - D0 * ((1.0 - nu) * depxx + nu * depyy + nu * depzz);
        dsyy = dsyy - D0 * (nu * depxx + (1.0 - nu) * depyy + nu * depzz);
        dszz = dszz - D0 * (nu * depxx + nu * depyy + (1.0 - nu) * depzz);
        dsxy = dsxy - D0 * (1.0 - 2.0 * nu) * depxy;
    }
    s[0] = sxx + dsxx;
    s[1] = syy + dsyy;
    s[2] = szz + dszz;
    s[3] = sxy + dsxy;
    if (sxx + dsxx + syy + dsyy + szz + dszz > k_c / a_phi) {
        double apex = k_c / a_phi / 3.0;
        s[0] = apex;
        s[1] = apex;
        s[2] = apex;
        s[3] = 0.0;
    }
    double* e = &ps.strain[i * 4];
    double* ep = &ps.strainp[i * 4];
    e[0] = e[0] + dexx;
    e[1] = e[1] + deyy;
    e[2] = e[2] + dezz;
    e[3] = e[3] + dexy;
    ep[0] = ep[0] + depxx;
    ep[1] = ep[1] + depyy;
    ep[2] = ep[2] + depzz;
    ep[3] = ep[3] + depxy;
}

void hooke_update(Sys& ps, int64_t i, const Upd& u, double dt) {
    const double E = u.prm[0], nu = u.prm[1];
    mag_stress_increment(ps, i, E, nu, dt);
    double* s = &ps.stress[i * 4];
    const double* er = &ps.sr[i * 4];
    double w = ps.vort[i * ps.nvort];
    double sxx = s[0], syy = s[1], szz = s[2], sxy = s[3];
    double dexx = er[0] * dt, deyy = er[1] * dt, dezz = er[2] * dt, dexy = er[3] * dt;
    double D0 = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double dsxx = D0 * ((1.0 - nu) * dexx + nu * deyy + nu * dezz);
    double dsyy = D0 * (nu * dexx + (1.0 - nu) * deyy + nu * dezz);
    double dszz = D0 * (nu * dexx + nu * deyy + (1.0 - nu) * dezz);
    double dsxy = D0 * (1.0 - 2.0 * nu) * dexy;
    double wdt = w * dt;
    dsxx = dsxx - 2.0 * sxy * wdt;
    dsyy = dsyy + 2.0 * sxy * wdt;
    dsxy = dsxy + (sxx - syy) * wdt;
    double nxx = sxx + dsxx, nyy = syy + dsyy, nzz = szz + dszz, nxy = sxy + dsxy;
    s[0] = nxx;
    s[1] = nyy;
    s[2] = nzz;
    s[3] = nxy;
    ps.p[i] = -(nxx + nyy + nzz) / 3.0;
}

void apply_updater(Sys& ps, const Upd& u, double dt) {
    const int64_t n = ps.n;
    switch (u.kind) {
        case GC_UPD_ZERO_FIELDS: {
            uint64_t mask = (uint64_t)u.prm[0];
            for (int64_t i = 0; i < n; ++i) {
                if (mask & (1u << GC_FIELD_STRAIN_RATE))
                    for (int k = 0; k < ps.ns; ++k) ps.sr[i * ps.ns + k] = 0.0;
                if (mask & (1u << GC_FIELD_VORTICITY))
                    for (int k = 0; k < ps.nvort; ++k) ps.vort[i * ps.nvort + k] = 0.0;
                if (mask & (1u << GC_FIELD_P)) ps.p[i] = 0.0;
                if (mask & (1u << GC_FIELD_STRESS))
                    for (int k = 0; k < ps.ns; ++k) ps.stress[i * ps.ns + k] = 0.0;
                if (mask & (1u << GC_FIELD_DVDT))
                    for (int d = 0; d < ps.nd; ++d) ps.dvdt[i * ps.nd + d] = 0.0;
                if (mask & (1u << GC_FIELD_DRHODT)) ps.drhodt[i] = 0.0;
            }
            if (mask & (1u << GC_FIELD_STRAIN_RATE)) std::fill(ps.msr.begin(), ps.msr.end(), 0.0);
            if (mask & (1u << GC_FIELD_VORTICITY)) std::fill(ps.mvort.begin(), ps.mvort.end(), 0.0);
            if (mask & (1u << GC_FIELD_DVDT)) std::fill(ps.mdvdt.begin(), ps.mdvdt.end(), 0.0);
            if (mask & (1u << GC_FIELD_DRHODT)) std::fill(ps.mdrhodt.begin(), ps.mdrhodt.end(), 0.0);
            break;
        }
        case GC_UPD_TAIT_EOS: {
            const double rho0 = u.prm[0], gam = u.prm[1];
            const double pre = rho0 * ps.c * ps.c / gam;
            for (int64_t i = 0; i < n; ++i) ps.p[i] = pre * (jpow(ps.rho[i] / rho0, gam) - 1.0);
            break;
        }
        case GC_UPD_LINEAR_EOS: {
            const double rho0 = u.prm[0];
            for (int64_t i = 0; i < n; ++i) ps.p[i] = ps.c * ps.c * (ps.rho[i] - rho0);
            break;
        }
        case GC_UPD_ELASTOPLASTIC:
            for (int64_t i = 0; i < n; ++i) ep_update(ps, i, u, dt);
            break;
        case GC_UPD_HOOKE:
            for (int64_t i = 0; i < n; ++i) hooke_update(ps, i, u, dt);
            break;
        case GC_UPD_VISCOPLASTIC_MC: {
            // src/StateUpdaters.jl:155-186 (after the EOS entry before it)
            const double tphi = std::tan(u.prm[0]), coh = u.prm[1];
            const int ns = ps.ns, nn = ns == 3 ? 2 : 3;
            for (int64_t i = 0; i < n; ++i) {
                const double* sr = &ps.sr[i * ns];
                double m;
                if (ns == 3) m = sr[0] * sr[0] + sr[1] * sr[1] + 2.0 * (sr[2] * sr[2]);
                else if (ns == 4) m = sr[0] * sr[0] + sr[1] * sr[1] + 2.0 * (sr[3] * sr[3]);
                else
                    m = sr[0] * sr[0] + sr[1] * sr[1] + sr[2] * sr[2] +
                        2.0 * (sr[3] * sr[3] + sr[4] * sr[4] + sr[5] * sr[5]);
                m = jmax(std::sqrt(m), 2.220446049250313e-16);  // eps(Float64)
                const double p = ps.p[i];
                const double sc = 2.0 * (coh + p * tphi);
                double st[6];
                for (int q = 0; q < ns; ++q) st[q] = (sc * sr[q]) / m - (q < nn ? p : 0.0);
                double tr = st[0];
                for (int q = 1; q < nn; ++q) tr = tr + st[q];
                for (int q = 0; q < ns; ++q) ps.stress[i * ns + q] = tr > 0.0 ? 0.0 : st[q];
            }
            break;
        }
        default:
            break;
    }
}

// src/Particles.jl:542-570
void update_state(Sys& ps, int stage, double dt) {
    if (stage < 1 || stage > (int)ps.upd.size()) return;
    for (const Upd& u : ps.upd[stage - 1]) apply_updater(ps, u, dt);
}

// ------------------------------------------------------------------ views
int make_view(oracle_ctx* ctx, int handle, BView* out) {
    if (handle < 0 || handle >= (int)ctx->handles.size()) return GC_ERR_ARG;
    const Handle& h = ctx->handles[handle];
    BView b{};
    b.type = h.type;
    if (h.type == H_VIRT) {
        Virt& vp = ctx->virts[h.idx];
        Sys& s = ctx->sys[vp.src];
        b.n = s.n;
        b.x = s.x.data();
        b.v = s.v.data();
        b.rho = s.rho.data();
        b.p = s.has_p() ? s.p.data() : nullptr;
        b.stress = s.has_stress() ? s.stress.data() : nullptr;
        b.mass = s.mass;
        b.c = s.c;
        b.ns = s.ns;
        b.sys = &s;
        b.virt = &vp;
    } else if (h.type == H_GHOST) {
        Ghost& g = ctx->ghosts[h.idx];
        Sys& src = ctx->sys[g.src];
        b.n = g.n;
        b.x = g.x.data();
        b.v = g.v.data();
        b.rho = g.rho.data();
        b.p = g.ex_p ? g.p.data() : nullptr;
        b.stress = g.ex_stress ? g.stress.data() : nullptr;
        b.mass = src.mass;
        b.c = src.c;
        b.ns = src.ns;
        b.sys = &src;  // the ghost's forwarded properties (v_adjustment) are the source's
    } else {
        Sys& s = ctx->sys[h.idx];
        b.n = s.n;
        b.x = s.x.data();
        b.v = s.v.data();
        b.rho = s.rho.data();
        b.p = s.has_p() ? s.p.data() : nullptr;
        b.stress = s.has_stress() ? s.stress.data() : nullptr;
        b.mass = s.mass;
        b.c = s.c;
        b.ns = s.ns;
        b.sys = &s;
        b.normal = h.normal;
        b.point = h.point;
        b.beta = h.beta;
        b.ljcut = h.ljcut;
    }
    *out = b;
    return GC_OK;
}

// Which functor/system_b combinations the restatement (and the device
// library) implement; the rest are refused instead of guessed.
int check_combo(oracle_ctx* ctx, const Inter& it, int pk) {
    const Sys& a = ctx->sys[it.a];
    if (pk == GC_PFN_NONE) return GC_OK;
    if (pk == GC_PFN_XSPH || pk < 0 || pk > GC_PFN_NEIGHBOR_COUNT) return GC_ERR_UNSUPPORTED;  // XSPH: velocity-adjust only
    if (it.ag >= 0) {
        // a ghost system_a: only InterpolateFieldFn into a virtual system
        if (pk != GC_PFN_INTERPOLATE || it.b < 0 || ctx->handles[it.b].type != H_VIRT ||
            ctx->virts[ctx->handles[it.b].idx].probe)
            return GC_ERR_UNSUPPORTED;
        const int m = (int)it.pp.back()[0];
        if ((m & (1 << GC_FIELD_STRESS)) && !ctx->ghosts[it.ag].ex_stress) return GC_ERR_UNSUPPORTED;
    }
    if (pk == GC_PFN_NEIGHBOR_COUNT) {  // the (real, probe) method :455
        if (it.b < 0 || ctx->handles[it.b].type != H_VIRT || !ctx->virts[ctx->handles[it.b].idx].probe)
            return GC_ERR_UNSUPPORTED;
        return GC_OK;
    }
    if (pk == GC_PFN_INTERPOLATE) {
        // the (real, virtual) method :424; the fields exist on both sides
        if (it.b < 0 || ctx->handles[it.b].type != H_VIRT) return GC_ERR_UNSUPPORTED;
        const Sys& s = ctx->sys[ctx->virts[ctx->handles[it.b].idx].src];
        const int m = (int)it.pp.back()[0];
        if (m & ~((1 << GC_FIELD_V) | (1 << GC_FIELD_RHO) | (1 << GC_FIELD_STRESS))) return GC_ERR_UNSUPPORTED;
        if ((m & (1 << GC_FIELD_STRESS)) && !(a.has_stress() && s.has_stress() && a.ns == s.ns)) return GC_ERR_ARG;
        return GC_OK;
    }
    if (pk == GC_PFN_FLUID_SOLID) {
        // only the two-sided (system, system) method exists (:494)
        if (!a.has_p()) return GC_ERR_ARG;
        if (it.b < 0 || ctx->handles[it.b].type != H_SYS) return GC_ERR_UNSUPPORTED;
        return GC_OK;
    }
    if (pk == GC_PFN_FLUID && !a.has_p()) return GC_ERR_ARG;
    if ((pk == GC_PFN_CAUCHY_FLUID || pk == GC_PFN_STRAIN_RATE) && !a.has_stress()) return GC_ERR_ARG;
    if (pk == GC_PFN_STRAIN_RATE_VORTICITY && !a.is_ep()) return GC_ERR_ARG;
    if ((pk == GC_PFN_CAUCHY_FLUID || pk == GC_PFN_STRAIN_RATE || pk == GC_PFN_STRAIN_RATE_VORTICITY)) {
        if (a.nd == 2 && !(a.ns == 3 || a.ns == 4)) return GC_ERR_UNSUPPORTED;
        if (a.nd == 3 && a.ns != 6) return GC_ERR_UNSUPPORTED;
    }
    if (it.b < 0) return GC_OK;
    const Handle& h = ctx->handles[it.b];
    if (h.type == H_VIRT) {
        // virtual system_b: the one-sided boundary forms (:193, :286, :37, :97)
        const Sys& s = ctx->sys[ctx->virts[h.idx].src];
        if (pk == GC_PFN_COUNT) return GC_ERR_UNSUPPORTED;
        if (pk == GC_PFN_FLUID) return s.has_p() ? GC_OK : GC_ERR_ARG;
        if (pk == GC_PFN_CAUCHY_FLUID) return s.has_stress() && s.ns == a.ns ? GC_OK : GC_ERR_ARG;
        return GC_OK;
    }
    if (pk == GC_PFN_COUNT) return h.type == H_GHOST ? GC_ERR_UNSUPPORTED : GC_OK;
    if (h.type == H_DYN) return GC_OK;
    if (h.type == H_STATIC) return GC_OK;
    if (h.type == H_GHOST) {
        const Ghost& g = ctx->ghosts[h.idx];
        if (pk == GC_PFN_FLUID && !g.ex_p) return GC_ERR_UNSUPPORTED;
        if (pk == GC_PFN_CAUCHY_FLUID && !g.ex_stress) return GC_ERR_UNSUPPORTED;
        return GC_OK;
    }
    // plain real system_b: FluidPfn is two-sided between two fluid systems,
    // one-sided otherwise
    const Sys& b = ctx->sys[h.idx];
    if (pk == GC_PFN_FLUID) {
        return b.has_p() ? GC_OK : GC_ERR_ARG;
    }
    if (pk == GC_PFN_CAUCHY_FLUID) return GC_ERR_UNSUPPORTED;  // two-sided real-real
    return GC_OK;
}

// mag: the magnitude pass of track_mag (rate fields swapped with their
// shadows by the caller); functors that write no rate field are skipped.
int sweep(oracle_ctx* ctx, Inter& it, int stage, bool mag = false) {
    if (stage < 1 || stage > it.nstages) return GC_OK;
    int pk = it.pk[stage - 1];
    if (pk == GC_PFN_NONE) return GC_OK;
    if (mag && (pk == GC_PFN_INTERPOLATE || pk == GC_PFN_NEIGHBOR_COUNT || pk == GC_PFN_XSPH)) return GC_OK;
    if (!it.grid) return fail(ctx, GC_ERR_STATE, "sweep before create_grid");
    Pfn f = make_pfn(pk, it.pp[stage - 1].data());
    f.mag = mag;
    const int nd = ctx->sys[it.a].nd;
    if (it.b < 0) {
        if (nd == 2) sweep_self<2>(ctx, it, f);
        else sweep_self<3>(ctx, it, f);
    } else {
        BView b;
        int st = make_view(ctx, it.b, &b);
        if (st) return st;
        st = nd == 2 ? sweep_coupled<2>(ctx, it, f, b) : sweep_coupled<3>(ctx, it, f, b);
        if (st) return fail(ctx, st, "XSPH: a ghost index beyond its source system's length");
    }
    return GC_OK;
}

// adjust_v! src/Interaction.jl:309: one sweep of the velocity-adjust functor
int adjust_v(oracle_ctx* ctx, Inter& it) {
    if (it.vk == GC_PFN_NONE) return GC_OK;
    if (!it.grid) return fail(ctx, GC_ERR_STATE, "adjust_v before create_grid");
    std::array<double, GC_PFN_NPARAM> prm{};
    prm[0] = it.veps;
    prm[4] = prm[5] = std::nan("");
    Pfn f = make_pfn(it.vk, prm.data());
    const int nd = ctx->sys[it.a].nd;
    if (it.b < 0) {
        if (nd == 2) sweep_self<2>(ctx, it, f);
        else sweep_self<3>(ctx, it, f);
        return GC_OK;
    }
    BView b;
    int st = make_view(ctx, it.b, &b);
    if (st) return st;
    st = nd == 2 ? sweep_coupled<2>(ctx, it, f, b) : sweep_coupled<3>(ctx, it, f, b);
    if (st) return fail(ctx, st, "XSPH: a ghost index beyond its source system's length");
    return GC_OK;
}

// _xsph_correction! src/TimeIntegration.jl:421-436: v -= v_adjustment, zero
// it, re-run every interaction's velocity-adjust functor, v += v_adjustment
// (both axpys as separate multiply and add, the SVector form)
int xsph_correction(oracle_ctx* ctx) {
    for (auto& s : ctx->sys)
        if (!s.vsrc)
            for (int64_t i = 0; i < s.n * s.nd; ++i) s.v[i] = s.v[i] + (-1.0 * s.vadj[i]);
    for (auto& s : ctx->sys)
        if (!s.vsrc) std::fill(s.vadj.begin(), s.vadj.end(), 0.0);
    for (auto& it : ctx->inters) {
        int st = adjust_v(ctx, it);
        if (st) return st;
    }
    for (auto& s : ctx->sys)
        if (!s.vsrc)
            for (int64_t i = 0; i < s.n * s.nd; ++i) s.v[i] = s.v[i] + 1.0 * s.vadj[i];
    return GC_OK;
}

// ------------------------------------------------------------- integrator
// src/TimeIntegration.jl:580-697 (LeapFrog)
int num_stages(oracle_ctx* ctx) {
    for (auto& it : ctx->inters)
        if (!it.probe) return it.nstages;
    return 0;
}

// Virtual systems (src/Particles.jl:476-528, src/TimeIntegration.jl:364-419)
void zero_field(Sys& s, int field) {
    switch (field) {
        case GC_FIELD_V: std::fill(s.v.begin(), s.v.end(), 0.0); break;
        case GC_FIELD_RHO: std::fill(s.rho.begin(), s.rho.end(), 0.0); break;
        case GC_FIELD_DVDT:
            std::fill(s.dvdt.begin(), s.dvdt.end(), 0.0);
            std::fill(s.mdvdt.begin(), s.mdvdt.end(), 0.0);
            break;
        case GC_FIELD_DRHODT:
            std::fill(s.drhodt.begin(), s.drhodt.end(), 0.0);
            std::fill(s.mdrhodt.begin(), s.mdrhodt.end(), 0.0);
            break;
        case GC_FIELD_P: std::fill(s.p.begin(), s.p.end(), 0.0); break;
        case GC_FIELD_STRESS: std::fill(s.stress.begin(), s.stress.end(), 0.0); break;
        case GC_FIELD_STRAIN_RATE:
            std::fill(s.sr.begin(), s.sr.end(), 0.0);
            std::fill(s.msr.begin(), s.msr.end(), 0.0);
            break;
        default: break;
    }
}

// auto_zero_virtual! :510-514: w_sum and the zero_fields
void auto_zero_virtual(oracle_ctx* ctx, Virt& vp) {
    std::fill(vp.wsum.begin(), vp.wsum.end(), 0.0);
    for (int f = 0; f < GC_NFIELDS; ++f)
        if (vp.zmask & (1 << f)) zero_field(ctx->sys[vp.src], f);
}

// VirtualNormUpdater src/StateUpdaters.jl:65-76, PrescribedVelocityUpdater
// :95-97; other updaters act on the source's fields
void apply_virtual_updater(Sys& s, Virt& vp, const Upd& u, double dt) {
    const int64_t n = s.n;
    const int nd = s.nd, ns = s.ns;
    if (u.kind == GC_UPD_VIRTUAL_NORM) {
        const int m = (int)u.prm[3];
        for (int64_t i = 0; i < n; ++i) {
            const double w = vp.wsum[i];
            if (m & (1 << GC_FIELD_V))
                for (int d = 0; d < nd; ++d) {
                    const double val = w == 0.0 ? 0.0 : s.v[i * nd + d] / w;
                    s.v[i * nd + d] = val * u.prm[d] + vp.pv[d];
                }
            if (m & (1 << GC_FIELD_RHO)) s.rho[i] = w == 0.0 ? 0.0 : s.rho[i] / w;
            if (m & (1 << GC_FIELD_P)) s.p[i] = w == 0.0 ? 0.0 : s.p[i] / w;
            if (m & (1 << GC_FIELD_STRESS))
                for (int q = 0; q < ns; ++q) s.stress[i * ns + q] = w == 0.0 ? 0.0 : s.stress[i * ns + q] / w;
        }
    } else if (u.kind == GC_UPD_PRESCRIBED_V) {
        for (int64_t i = 0; i < n; ++i)
            for (int d = 0; d < nd; ++d) s.v[i * nd + d] = s.v[i * nd + d] + vp.pv[d];
    } else {
        apply_updater(s, u, dt);
    }
}

// _sweep_all_stages! :401-419: auto-zero the virtuals, then per stage the
// systems' updaters, the ghosts' copiers, the virtuals' updaters and every
// interaction's sweep
int sweep_all_stages(oracle_ctx* ctx, int nst, double dt) {
    for (auto& vp : ctx->virts)
        if (!vp.probe) auto_zero_virtual(ctx, vp);
    for (int stage = 1; stage <= nst; ++stage) {
        for (auto& s : ctx->sys)
            if (!s.vsrc && s.upd_set && (int)s.upd.size() == nst) update_state(s, stage, dt);
        for (auto& g : ctx->ghosts) update_ghost(ctx, g, stage);
        for (auto& vp : ctx->virts)
            if (!vp.probe && vp.upd_set && (int)vp.upd.size() == nst)
                for (const Upd& u : vp.upd[stage - 1]) apply_virtual_updater(ctx->sys[vp.src], vp, u, dt);
        for (auto& it : ctx->inters) {
            if (it.probe) continue;
            int st = sweep(ctx, it, stage);
            if (st) return st;
        }
        if (ctx->track_mag) {  // the same sweeps again, summing |term| into the shadows
            for (auto& s : ctx->sys) {
                mag_ensure(s);
                mag_swap(s);
            }
            g_mag_inputs = ctx->track_mag == 2;
            int st = GC_OK;
            for (auto& it : ctx->inters) {
                if (it.probe) continue;
                st = sweep(ctx, it, stage, true);
                if (st) break;
            }
            g_mag_inputs = 0;
            for (auto& s : ctx->sys) mag_swap(s);
            if (st) return st;
        }
    }
    return GC_OK;
}

// Shadows of the rate fields just reset to their source terms.
void mag_reset_rates(oracle_ctx* ctx, Sys& s) {
    if (!ctx->track_mag) return;
    mag_set(s.dvdt, s.mdvdt);
    mag_set(s.drhodt, s.mdrhodt);
}

// Damping's term -(Γ/dt)·v added to the shadow of dvdt.
void mag_damping(oracle_ctx* ctx, Sys& s, double gdt) {
    if (!ctx->track_mag) return;
    mag_ensure(s);
    for (int64_t i = 0; i < s.n * s.nd; ++i) s.mdvdt[i] = s.mdvdt[i] + std::fabs(gdt * s.v[i]);
}

// The integrated-state shadows after a step's full update q = q0 + dt·rate
// (LeapFrog: the rates' shadows; RK4: the weighted sum of its four).
void mag_integrate(oracle_ctx* ctx, Sys& s, double dt, const std::vector<double>& mv,
                   const std::vector<double>& mrho) {
    if (!ctx->track_mag) return;
    mag_ensure(s);
    for (int64_t i = 0; i < s.n * s.nd; ++i) s.mvi[i] = s.mvi[i] + dt * mv[i];
    for (int64_t i = 0; i < s.n; ++i) s.mrhoi[i] = s.mrhoi[i] + dt * mrho[i];
}

// XSPH's velocity adjustment added to the v shadow; the position update
// x += dt·v added to the x shadow with v's scale max(|v|, M(v)).
void mag_positions(oracle_ctx* ctx, Sys& s, double dt, bool xsph) {
    if (!ctx->track_mag) return;
    mag_ensure(s);
    if (xsph)
        for (int64_t i = 0; i < s.n * s.nd; ++i) s.mvi[i] = s.mvi[i] + std::fabs(s.vadj[i]);
    for (int64_t i = 0; i < s.n * s.nd; ++i)
        s.mxi[i] = s.mxi[i] + dt * std::max(std::fabs(s.v[i]), s.mvi[i]);
}

bool any_xsph(oracle_ctx* ctx) {
    for (auto& it : ctx->inters)
        if (it.vk != GC_PFN_NONE) return true;
    return false;
}

// _prepare_grids! :364-379: ghosts, ghost sort, virtual (source) sort, grids
int prepare_grids(oracle_ctx* ctx, double sort_cutoff) {
    for (auto& g : ctx->ghosts) generate_ghosts(ctx, g);
    for (auto& g : ctx->ghosts) {
        const Sys& src = ctx->sys[g.src];
        int st = sort_ghost(g, src.nd, src.ns, sort_cutoff, nullptr);
        if (st) return fail(ctx, st, "ghost sort: non-finite position");
    }
    for (auto& vp : ctx->virts) {
        if (vp.probe) continue;  // probes are sorted at measurement
        int st = sort_system(ctx->sys[vp.src], sort_cutoff, nullptr);
        if (st) return fail(ctx, st, "virtual sort: non-finite position");
    }
    for (auto& it : ctx->inters) {
        if (it.probe) continue;
        int st = create_grid(ctx, it);
        if (st) return st;
    }
    return GC_OK;
}

// _measure_probes! src/TimeIntegration.jl:454-502
int measure_probes(oracle_ctx* ctx) {
    double hmin = 1e300;
    for (auto& it : ctx->inters)
        if (!it.probe) hmin = std::min(hmin, it.H);
    const double cutoff = 2.0 * hmin;
    // the probe interactions' system_a, re-sorted (positions moved since the step's sort)
    std::vector<char> done(ctx->sys.size(), 0);
    for (auto& it : ctx->inters) {
        if (!it.probe || done[it.a]) continue;
        done[it.a] = 1;
        int st = sort_system(ctx->sys[it.a], cutoff, nullptr);
        if (st) return fail(ctx, st, "sort: non-finite position");
    }
    // mirrored positions: x[id_src[i]] = x_src[i] (probe ids are 1..n here)
    for (auto& vp : ctx->virts) {
        if (!vp.probe || vp.mirror < 0) continue;
        Sys& p = ctx->sys[vp.src];
        const Sys& m = ctx->sys[vp.mirror];
        for (int64_t i = 0; i < m.n; ++i)
            for (int d = 0; d < p.nd; ++d) p.x[(size_t)((m.id[i] - 1) * p.nd + d)] = m.x[(size_t)(i * m.nd + d)];
    }
    for (auto& vp : ctx->virts) {
        if (!vp.probe) continue;
        int st = sort_system(ctx->sys[vp.src], cutoff, nullptr);
        if (st) return fail(ctx, st, "probe sort: non-finite position");
    }
    for (auto& it : ctx->inters) {
        if (!it.probe) continue;
        int st = create_grid(ctx, it);
        if (st) return st;
    }
    // auto_zero_probe! src/ProbeParticles.jl:117-124: w_sum and every extra
    for (auto& vp : ctx->virts) {
        if (!vp.probe) continue;
        Sys& p = ctx->sys[vp.src];
        std::fill(vp.wsum.begin(), vp.wsum.end(), 0.0);
        for (int f : {GC_FIELD_V, GC_FIELD_RHO, GC_FIELD_P, GC_FIELD_STRESS, GC_FIELD_DRHODT}) zero_field(p, f);
    }
    for (auto& it : ctx->inters) {
        if (!it.probe) continue;
        int st = sweep(ctx, it, 1);
        if (st) return st;
    }
    for (auto& vp : ctx->virts)  // update_state!(probe): stage 1, dt = 0
        if (vp.probe && !vp.upd.empty())
            for (const Upd& u : vp.upd[0]) apply_virtual_updater(ctx->sys[vp.src], vp, u, 0.0);
    // _sort_probe_by_id! :129-143
    for (auto& vp : ctx->virts) {
        if (!vp.probe) continue;
        Sys& p = ctx->sys[vp.src];
        std::vector<int64_t> perm((size_t)p.n);
        for (int64_t i = 0; i < p.n; ++i) perm[(size_t)(p.id[i] - 1)] = i;
        permute_system(p, perm);
        apply_perm(vp.wsum, perm, 1);
    }
    return GC_OK;
}

// _update_virtual_positions! :389-397: x += prescribed_v·dt, per virtual system
void update_virtual_positions(oracle_ctx* ctx, double dt) {
    for (auto& vp : ctx->virts) {
        Sys& s = ctx->sys[vp.src];
        double step[3];
        for (int d = 0; d < s.nd; ++d) step[d] = vp.pv[d] * dt;
        for (int64_t i = 0; i < s.n; ++i)
            for (int d = 0; d < s.nd; ++d) s.x[i * s.nd + d] = s.x[i * s.nd + d] + step[d];
    }
}

int step_once(oracle_ctx* ctx, double dt) {
    const int nst = num_stages(ctx);
    double hmin = 1e300;
    for (auto& it : ctx->inters) hmin = std::min(hmin, it.H);
    const double sort_cutoff = 2.0 * hmin;
    // 1. sort every real system (a virtual's source is sorted with the virtuals)
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        int st = sort_system(s, sort_cutoff, nullptr);
        if (st) return fail(ctx, st, "sort: non-finite position");
    }
    // 2. save q0
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        s.q0v = s.v;
        s.q0rho = s.rho;
    }
    // 3-5. ghosts, ghost sort, virtual sort, grids
    {
        int st = prepare_grids(ctx, sort_cutoff);
        if (st) return st;
    }
    // 6. half-step: q += dt/2 * dqdt, dqdt <- source
    const double half = dt / 2.0;
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        const int nd = s.nd;
        for (int64_t i = 0; i < s.n * nd; ++i) s.v[i] = s.v[i] + half * s.dvdt[i];
        for (int64_t i = 0; i < s.n; ++i) s.rho[i] = std::fma(half, s.drhodt[i], s.rho[i]);
        for (int64_t i = 0; i < s.n; ++i)
            for (int d = 0; d < nd; ++d) s.dvdt[i * nd + d] = s.srcv[d];
        for (int64_t i = 0; i < s.n; ++i) s.drhodt[i] = s.srcrho;
        mag_reset_rates(ctx, s);
    }
    // 7. ghost kinematics
    for (auto& g : ctx->ghosts) ghost_kinematics(ctx, g);
    // 8. stages
    {
        int st = sweep_all_stages(ctx, nst, dt);
        if (st) return st;
    }
    // 8b. damping
    if (ctx->gamma != 0.0) {
        const double gdt = ctx->gamma / dt;
        for (auto& s : ctx->sys)
            if (!s.vsrc) {
                for (int64_t i = 0; i < s.n * s.nd; ++i) s.dvdt[i] = s.dvdt[i] - gdt * s.v[i];
                mag_damping(ctx, s, gdt);
            }
    }
    // 9. full step: q = q0 + dt * dqdt
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        for (int64_t i = 0; i < s.n * s.nd; ++i) s.v[i] = s.q0v[i] + dt * s.dvdt[i];
        for (int64_t i = 0; i < s.n; ++i) s.rho[i] = std::fma(dt, s.drhodt[i], s.q0rho[i]);
        if (ctx->track_mag) {
            mag_ensure(s);
            mag_integrate(ctx, s, dt, s.mdvdt, s.mdrhodt);
        }
    }
    // 10. XSPH correction
    {
        int st = xsph_correction(ctx);
        if (st) return st;
    }
    // 11. positions, then the virtual systems'
    const bool xs = any_xsph(ctx);
    for (auto& s : ctx->sys)
        if (!s.vsrc) {
            for (int64_t i = 0; i < s.n * s.nd; ++i) s.x[i] = s.x[i] + dt * s.v[i];
            mag_positions(ctx, s, dt, xs);
        }
    update_virtual_positions(ctx, dt);
    ctx->steps += 1;
    return GC_OK;
}

// src/TimeIntegration.jl:712-838 (RK4): one grid per step, four right-hand
// side evaluations from q0, q = q0 + dt·acc, positions once at the end.
// Rounding as for LeapFrog: `@fastmath` axpy fuses on scalar fields (rho)
// and rounds twice on SVector fields (v).
int step_rk4(oracle_ctx* ctx, double dt) {
    const int nst = num_stages(ctx);
    double hmin = 1e300;
    for (auto& it : ctx->inters) hmin = std::min(hmin, it.H);
    const double sort_cutoff = 2.0 * hmin;
    // 1. sort every real system
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        int st = sort_system(s, sort_cutoff, nullptr);
        if (st) return fail(ctx, st, "sort: non-finite position");
    }
    // 2. save q0, zero the accumulators (:783-784)
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        s.q0v = s.v;
        s.q0rho = s.rho;
        s.accv.assign(s.v.size(), 0.0);
        s.accrho.assign(s.rho.size(), 0.0);
        if (ctx->track_mag) {
            s.accmv.assign(s.v.size(), 0.0);
            s.accmrho.assign(s.rho.size(), 0.0);
        }
    }
    // 3-5. ghosts, ghost sort, virtual sort, grids (:787-788)
    {
        int st = prepare_grids(ctx, sort_cutoff);
        if (st) return st;
    }
    // T(0.5), T(1.0), T(1/6), T(1/3) (:742-743)
    const double advance[4] = {0.0, 0.5, 0.5, 1.0};
    const double weight[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    for (int rk = 0; rk < 4; ++rk) {
        // 6. reset dqdt (first stage) or q = q0 + (f·dt)·dqdt then reset (:797-803)
        const double c = advance[rk] * dt;
        for (auto& s : ctx->sys) {
            if (s.vsrc) continue;
            const int nd = s.nd;
            if (rk > 0) {
                for (int64_t i = 0; i < s.n * nd; ++i) s.v[i] = s.q0v[i] + c * s.dvdt[i];
                for (int64_t i = 0; i < s.n; ++i) s.rho[i] = std::fma(c, s.drhodt[i], s.q0rho[i]);
            }
            for (int64_t i = 0; i < s.n; ++i)
                for (int d = 0; d < nd; ++d) s.dvdt[i * nd + d] = s.srcv[d];
            for (int64_t i = 0; i < s.n; ++i) s.drhodt[i] = s.srcrho;
            mag_reset_rates(ctx, s);
        }
        // 7. ghost kinematics (:805-807)
        for (auto& g : ctx->ghosts) ghost_kinematics(ctx, g);
        // 8. stages (:809-810)
        {
            int st = sweep_all_stages(ctx, nst, dt);
            if (st) return st;
        }
        // damping and acc += w·dqdt (:812-814)
        if (ctx->gamma != 0.0) {
            const double gdt = ctx->gamma / dt;
            for (auto& s : ctx->sys)
                if (!s.vsrc) {
                    for (int64_t i = 0; i < s.n * s.nd; ++i) s.dvdt[i] = s.dvdt[i] - gdt * s.v[i];
                    mag_damping(ctx, s, gdt);
                }
        }
        for (auto& s : ctx->sys) {
            if (s.vsrc) continue;
            for (int64_t i = 0; i < s.n * s.nd; ++i) s.accv[i] = s.accv[i] + weight[rk] * s.dvdt[i];
            for (int64_t i = 0; i < s.n; ++i) s.accrho[i] = std::fma(weight[rk], s.drhodt[i], s.accrho[i]);
            if (ctx->track_mag) {
                mag_ensure(s);
                for (int64_t i = 0; i < s.n * s.nd; ++i) s.accmv[i] = s.accmv[i] + weight[rk] * s.mdvdt[i];
                for (int64_t i = 0; i < s.n; ++i) s.accmrho[i] = s.accmrho[i] + weight[rk] * s.mdrhodt[i];
            }
        }
    }
    // 9. q = q0 + dt·acc (:818)
    for (auto& s : ctx->sys) {
        if (s.vsrc) continue;
        for (int64_t i = 0; i < s.n * s.nd; ++i) s.v[i] = s.q0v[i] + dt * s.accv[i];
        for (int64_t i = 0; i < s.n; ++i) s.rho[i] = std::fma(dt, s.accrho[i], s.q0rho[i]);
        mag_integrate(ctx, s, dt, s.accmv, s.accmrho);
    }
    // 10. XSPH correction (:821)
    {
        int st = xsph_correction(ctx);
        if (st) return st;
    }
    // 11. positions (:824), then the virtual systems' (:825)
    const bool xs = any_xsph(ctx);
    for (auto& s : ctx->sys)
        if (!s.vsrc) {
            for (int64_t i = 0; i < s.n * s.nd; ++i) s.x[i] = s.x[i] + dt * s.v[i];
            mag_positions(ctx, s, dt, xs);
        }
    update_virtual_positions(ctx, dt);
    ctx->steps += 1;
    return GC_OK;
}

double compute_dt(oracle_ctx* ctx, double cfl) {
    double c = -1e300, h = 1e300;
    for (auto& s : ctx->sys)
        if (!s.vsrc) c = std::max(c, s.c);  // the integrator's systems (:108)
    for (auto& it : ctx->inters)
        if (!it.probe) h = std::min(h, it.H);
    return cfl * h / c;
}

// field access
int field_comps(const Sys& s, int field) {
    switch (field) {
        case GC_FIELD_X: case GC_FIELD_V: case GC_FIELD_DVDT: case GC_FIELD_V_ADJUSTMENT: return s.nd;
        case GC_FIELD_RHO: case GC_FIELD_DRHODT: case GC_FIELD_ID: return 1;
        case GC_FIELD_P: return s.has_p() ? 1 : -1;
        case GC_FIELD_STRESS: case GC_FIELD_STRAIN_RATE: return s.has_stress() ? s.ns : -1;
        case GC_FIELD_VORTICITY: return s.is_ep() ? s.nvort : -1;
        case GC_FIELD_STRAIN: case GC_FIELD_STRAIN_P: return s.is_ep() ? s.ns : -1;
        default: return -1;
    }
}

std::vector<double>* field_vec(Sys& s, int field) {
    switch (field) {
        case GC_FIELD_X: return &s.x;
        case GC_FIELD_V: return &s.v;
        case GC_FIELD_RHO: return &s.rho;
        case GC_FIELD_DVDT: return &s.dvdt;
        case GC_FIELD_DRHODT: return &s.drhodt;
        case GC_FIELD_P: return &s.p;
        case GC_FIELD_STRESS: return &s.stress;
        case GC_FIELD_STRAIN_RATE: return &s.sr;
        case GC_FIELD_VORTICITY: return &s.vort;
        case GC_FIELD_STRAIN: return &s.strain;
        case GC_FIELD_STRAIN_P: return &s.strainp;
        case GC_FIELD_V_ADJUSTMENT: return &s.vadj;
        default: return nullptr;
    }
}

}  // namespace

// =================================================================== C API
extern "C" {

int oracle_create(oracle_ctx** out) {
    *out = new oracle_ctx();
    return GC_OK;
}

int oracle_destroy(oracle_ctx* ctx) {
    delete ctx;
    return GC_OK;
}

const char* oracle_last_error(oracle_ctx* ctx) { return ctx->err.c_str(); }

int oracle_set_threads(oracle_ctx* ctx, int threads) {
    ctx->threads = threads < 1 ? 1 : threads;
    return GC_OK;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int oracle_add_system(oracle_ctx* ctx, int kind, int64_t n, int nd, int ns, double mass, double c,
                      const double* source_v, double source_rho, int* sys_out) {
    if (n <= 0) return fail(ctx, GC_ERR_ARG, "n must be positive");
    if (nd < 2 || nd > 3) return fail(ctx, GC_ERR_UNSUPPORTED, "ndims must be 2 or 3");
    if (kind < GC_SYS_BASIC || kind > GC_SYS_ELASTOPLASTIC) return fail(ctx, GC_ERR_ARG, "bad system kind");
    Sys s;
    s.kind = kind;
    s.n = n;
    s.nd = nd;
    s.ns = kind >= GC_SYS_STRESS ? ns : 0;
    if (kind >= GC_SYS_STRESS && !(ns == 3 || ns == 4 || ns == 6)) return fail(ctx, GC_ERR_ARG, "ns must be 3, 4, or 6");
    s.nvort = kind == GC_SYS_ELASTOPLASTIC ? (nd == 2 ? 1 : 3) : 0;
    s.mass = mass;
    s.c = c;
    for (int d = 0; d < nd; ++d) s.srcv[d] = source_v ? source_v[d] : 0.0;
    s.srcrho = source_rho;
    s.x.assign((size_t)n * nd, 0.0);
    s.v.assign((size_t)n * nd, 0.0);
    s.vadj.assign((size_t)n * nd, 0.0);
    s.rho.assign((size_t)n, 0.0);
    s.dvdt.assign((size_t)n * nd, 0.0);
    s.drhodt.assign((size_t)n, 0.0);
    s.id.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) s.id[i] = i + 1;
    if (s.has_p()) s.p.assign((size_t)n, 0.0);
    if (s.has_stress()) {
        s.stress.assign((size_t)n * s.ns, 0.0);
        s.sr.assign((size_t)n * s.ns, 0.0);
    }
    if (s.is_ep()) {
        s.vort.assign((size_t)n * s.nvort, 0.0);
        s.strain.assign((size_t)n * s.ns, 0.0);
        s.strainp.assign((size_t)n * s.ns, 0.0);
    }
    ctx->sys.push_back(std::move(s));
    Handle h;
    h.type = H_SYS;
    h.idx = (int)ctx->sys.size() - 1;
    ctx->handles.push_back(h);
    ctx->sys_handle.push_back((int)ctx->handles.size() - 1);
    *sys_out = (int)ctx->handles.size() - 1;
    return GC_OK;
}

static int sys_index(oracle_ctx* ctx, int handle) {
    if (handle < 0 || handle >= (int)ctx->handles.size()) return -1;
    if (ctx->handles[handle].type != H_SYS) return -1;
    return ctx->handles[handle].idx;
}

int oracle_add_boundary(oracle_ctx* ctx, int sys, int kind, const double* normal, const double* point,
                        double beta_or_lj, int* handle_out) {
    int si = sys_index(ctx, sys);
    if (si < 0) return fail(ctx, GC_ERR_ARG, "boundary inner must be a system");
    Handle h;
    h.type = kind == GC_WRAP_DYNAMIC ? H_DYN : H_STATIC;
    h.idx = si;
    const int nd = ctx->sys[si].nd;
    if (kind == GC_WRAP_DYNAMIC) {
        for (int d = 0; d < nd; ++d) {
            h.normal[d] = normal[d];
            h.point[d] = point[d];
        }
        h.beta = beta_or_lj;
    } else if (kind == GC_WRAP_STATIC) {
        h.ljcut = beta_or_lj;
    } else {
        return fail(ctx, GC_ERR_ARG, "bad boundary kind");
    }
    ctx->handles.push_back(h);
    *handle_out = (int)ctx->handles.size() - 1;
    return GC_OK;
}

int oracle_add_ghost(oracle_ctx* ctx, int src_sys, int ncopiers, const int* copier_nfields,
                     const int* copier_fields, const int* copier_modes, int nplanes, const double* normals,
                     const double* points, double cutoff, int* handle_out) {
    int si = sys_index(ctx, src_sys);
    if (si < 0) return fail(ctx, GC_ERR_ARG, "ghost source must be a system");
    if (nplanes < 1) return fail(ctx, GC_ERR_ARG, "at least one boundary (normal, point) pair is required");
    const Sys& s = ctx->sys[si];
    Ghost g;
    g.src = si;
    g.cutoff = cutoff;
    g.nplanes = nplanes;
    g.pn.assign(normals, normals + nplanes * s.nd);
    g.pp.assign(points, points + nplanes * s.nd);
    int pos = 0;
    for (int k = 0; k < ncopiers; ++k) {
        Copier cp;
        for (int e = 0; e < copier_nfields[k]; ++e, ++pos) {
            int fld = copier_fields[pos], mode = copier_modes[pos];
            if (fld == GC_FIELD_P) {
                if (!s.has_p()) return fail(ctx, GC_ERR_ARG, "copier field p missing on source");
                g.ex_p = true;
            } else if (fld == GC_FIELD_STRESS) {
                if (!s.has_stress()) return fail(ctx, GC_ERR_ARG, "copier field stress missing on source");
                g.ex_stress = true;
            } else if (fld != GC_FIELD_RHO) {
                return fail(ctx, GC_ERR_UNSUPPORTED, "copier field not supported");
            }
            cp.entries.push_back({fld, mode});
        }
        g.copiers.push_back(cp);
    }
    ctx->ghosts.push_back(std::move(g));
    Handle h;
    h.type = H_GHOST;
    h.idx = (int)ctx->ghosts.size() - 1;
    ctx->handles.push_back(h);
    *handle_out = (int)ctx->handles.size() - 1;
    return GC_OK;
}

int oracle_add_interaction(oracle_ctx* ctx, int sys_a, int b_handle, int kernel_kind, double h, int nstages,
                           const int* pfn_kinds, const double* pfn_params, int* inter_out) {
    int si = sys_index(ctx, sys_a);
    int ag = -1;
    if (si < 0 && sys_a >= 0 && sys_a < (int)ctx->handles.size() && ctx->handles[sys_a].type == H_GHOST) {
        ag = ctx->handles[sys_a].idx;
        si = ctx->ghosts[ag].src;
    }
    if (si < 0) return fail(ctx, GC_ERR_ARG, "system_a must be a system");
    if (b_handle >= (int)ctx->handles.size()) return fail(ctx, GC_ERR_ARG, "bad system_b handle");
    Inter it;
    it.a = si;
    it.ag = ag;
    it.b = b_handle;
    it.kk = kernel_kind;
    it.H = h;
    it.nstages = nstages;
    it.cell = 2.0 * h;
    for (int s = 0; s < nstages; ++s) {
        it.pk.push_back(pfn_kinds[s]);
        std::array<double, GC_PFN_NPARAM> a;
        for (int k = 0; k < GC_PFN_NPARAM; ++k) a[k] = pfn_params[s * GC_PFN_NPARAM + k];
        it.pp.push_back(a);
        int st = check_combo(ctx, it, pfn_kinds[s]);
        if (st) return fail(ctx, st, "unsupported pairwise functor / system combination");
    }
    ctx->inters.push_back(std::move(it));
    *inter_out = (int)ctx->inters.size() - 1;
    return GC_OK;
}

int oracle_add_probe(oracle_ctx* ctx, int64_t n, int nd, const double* positions, int mirror_sys, int extras_mask,
                     int ns, const double* prescribed_v, int* handle_out) {
    if (n <= 0) return fail(ctx, GC_ERR_ARG, "positions must not be empty");
    if (nd < 2 || nd > 3) return fail(ctx, GC_ERR_UNSUPPORTED, "ndims must be 2 or 3");
    int mi = -1;
    if (mirror_sys >= 0) {
        mi = sys_index(ctx, mirror_sys);
        if (mi < 0 || ctx->sys[mi].n != n || ctx->sys[mi].nd != nd)
            return fail(ctx, GC_ERR_ARG, "mirror target must be a system of n particles");
    } else if (!positions) {
        return fail(ctx, GC_ERR_ARG, "probe positions or a mirror target are required");
    }
    const bool st = extras_mask & (1 << GC_FIELD_STRESS);
    if (st && !(ns == 3 || ns == 4 || ns == 6)) return fail(ctx, GC_ERR_ARG, "ns must be 3, 4, or 6");
    Sys s;
    s.kind = st ? GC_SYS_STRESS : (extras_mask & (1 << GC_FIELD_P)) ? GC_SYS_FLUID : GC_SYS_BASIC;
    s.n = n;
    s.nd = nd;
    s.ns = st ? ns : 0;
    s.x.assign((size_t)n * nd, 0.0);
    if (positions) std::memcpy(s.x.data(), positions, sizeof(double) * n * nd);
    else s.x = ctx->sys[mi].x;
    s.v.assign((size_t)n * nd, 0.0);
    s.vadj.assign((size_t)n * nd, 0.0);
    s.rho.assign((size_t)n, 0.0);
    s.dvdt.assign((size_t)n * nd, 0.0);
    s.drhodt.assign((size_t)n, 0.0);
    s.id.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) s.id[i] = i + 1;
    if (s.has_p()) s.p.assign((size_t)n, 0.0);
    if (s.has_stress()) {
        s.stress.assign((size_t)n * s.ns, 0.0);
        s.sr.assign((size_t)n * s.ns, 0.0);
    }
    s.vsrc = true;
    s.probe = true;
    ctx->sys.push_back(std::move(s));
    Virt vp;
    vp.src = (int)ctx->sys.size() - 1;
    vp.probe = true;
    vp.mirror = mi;
    if (prescribed_v)
        for (int d = 0; d < nd; ++d) vp.pv[d] = prescribed_v[d];
    vp.wsum.assign((size_t)n, 0.0);
    ctx->virts.push_back(vp);
    Handle h;
    h.type = H_VIRT;
    h.idx = (int)ctx->virts.size() - 1;
    ctx->handles.push_back(h);
    *handle_out = (int)ctx->handles.size() - 1;
    return GC_OK;
}

int oracle_add_probe_interaction(oracle_ctx* ctx, int sys_a, int probe, int kernel_kind, double h, int pfn_kind,
                                 const double* pfn_params, int* inter_out) {
    int si = sys_index(ctx, sys_a);
    if (si < 0) return fail(ctx, GC_ERR_ARG, "system_a must be a system");
    if (probe < 0 || probe >= (int)ctx->handles.size() || ctx->handles[probe].type != H_VIRT ||
        !ctx->virts[ctx->handles[probe].idx].probe)
        return fail(ctx, GC_ERR_ARG, "system_b must be a probe");
    if (pfn_kind != GC_PFN_INTERPOLATE && pfn_kind != GC_PFN_NEIGHBOR_COUNT)
        return fail(ctx, GC_ERR_UNSUPPORTED, "probe interactions take InterpolateFieldFn or NeighborCountFn");
    Inter it;
    it.a = si;
    it.b = probe;
    it.kk = kernel_kind;
    it.H = h;
    it.nstages = 1;
    it.cell = 2.0 * h;
    it.probe = true;
    it.pk.push_back(pfn_kind);
    std::array<double, GC_PFN_NPARAM> a;
    for (int k = 0; k < GC_PFN_NPARAM; ++k) a[k] = pfn_params[k];
    it.pp.push_back(a);
    int st = check_combo(ctx, it, pfn_kind);
    if (st) return fail(ctx, st, "unsupported probe functor / system combination");
    ctx->inters.push_back(std::move(it));
    *inter_out = (int)ctx->inters.size() - 1;
    return GC_OK;
}

int oracle_measure_probes(oracle_ctx* ctx) { return measure_probes(ctx); }

int oracle_add_virtual(oracle_ctx* ctx, int src_sys, int zero_mask, const double* prescribed_v, int* handle_out) {
    int si = sys_index(ctx, src_sys);
    if (si < 0) return fail(ctx, GC_ERR_ARG, "a virtual system needs a source system");
    Virt vp;
    vp.src = si;
    vp.zmask = zero_mask;
    Sys& s = ctx->sys[si];
    if (prescribed_v)
        for (int d = 0; d < s.nd; ++d) vp.pv[d] = prescribed_v[d];
    vp.wsum.assign((size_t)s.n, 0.0);
    s.vsrc = true;
    ctx->virts.push_back(vp);
    Handle h;
    h.type = H_VIRT;
    h.idx = (int)ctx->virts.size() - 1;
    ctx->handles.push_back(h);
    *handle_out = (int)ctx->handles.size() - 1;
    return GC_OK;
}

int oracle_set_updaters(oracle_ctx* ctx, int sys, int nstages, const int* chain_len, const int* kinds,
                        const double* params) {
    if (sys >= 0 && sys < (int)ctx->handles.size() && ctx->handles[sys].type == H_VIRT) {
        Virt& vp = ctx->virts[ctx->handles[sys].idx];
        vp.upd.clear();
        vp.upd_set = true;
        int pos = 0;
        for (int st = 0; st < nstages; ++st) {
            std::vector<Upd> chain;
            for (int k = 0; k < chain_len[st]; ++k, ++pos) {
                Upd u;
                u.kind = kinds[pos];
                for (int q = 0; q < GC_UPD_NPARAM; ++q) u.prm[q] = params[pos * GC_UPD_NPARAM + q];
                if (u.kind != GC_UPD_ZERO_FIELDS && u.kind != GC_UPD_VIRTUAL_NORM && u.kind != GC_UPD_PRESCRIBED_V)
                    return fail(ctx, GC_ERR_UNSUPPORTED, "updater kind on a virtual system");
                chain.push_back(u);
            }
            vp.upd.push_back(chain);
        }
        return GC_OK;
    }
    int si = sys_index(ctx, sys);
    if (si < 0) return fail(ctx, GC_ERR_ARG, "updaters need a system");
    Sys& s = ctx->sys[si];
    s.upd.clear();
    s.upd_set = true;
    int pos = 0;
    for (int st = 0; st < nstages; ++st) {
        std::vector<Upd> chain;
        for (int k = 0; k < chain_len[st]; ++k, ++pos) {
            Upd u;
            u.kind = kinds[pos];
            for (int q = 0; q < GC_UPD_NPARAM; ++q) u.prm[q] = params[pos * GC_UPD_NPARAM + q];
            if ((u.kind == GC_UPD_ELASTOPLASTIC || u.kind == GC_UPD_HOOKE) && !(s.is_ep() && s.ns == 4))
                return fail(ctx, GC_ERR_ARG, "ElastoPlasticStressUpdater requires NS=4 (plane-strain Voigt)");
            if ((u.kind == GC_UPD_TAIT_EOS || u.kind == GC_UPD_LINEAR_EOS) && !s.has_p())
                return fail(ctx, GC_ERR_ARG, "EOS updater needs a pressure field");
            if (u.kind == GC_UPD_VISCOPLASTIC_MC && (!s.has_stress() || (s.ns != 3 && s.ns != 4 && s.ns != 6)))
                return fail(ctx, GC_ERR_ARG, "ViscoPlasticMCStressUpdater needs stress with NS = 3, 4 or 6");
            if (u.kind == GC_UPD_VIRTUAL_NORM || u.kind == GC_UPD_PRESCRIBED_V)
                return fail(ctx, GC_ERR_ARG, "this updater acts on a virtual system");
            chain.push_back(u);
        }
        s.upd.push_back(chain);
    }
    return GC_OK;
}

int oracle_set_velocity_adjust(oracle_ctx* ctx, int inter, int kind, double epsilon) {
    if (!ctx || inter < 0 || inter >= (int)ctx->inters.size()) return GC_ERR_ARG;
    if (kind != GC_PFN_NONE && kind != GC_PFN_XSPH) return fail(ctx, GC_ERR_ARG, "velocity-adjust functor kind");
    if (kind != GC_PFN_NONE && ctx->inters[inter].ag >= 0)
        return fail(ctx, GC_ERR_UNSUPPORTED, "no velocity-adjust functor on a ghost system_a");
    ctx->inters[inter].vk = kind;
    ctx->inters[inter].veps = epsilon;
    return GC_OK;
}

int oracle_set_integrator_kind(oracle_ctx* ctx, int kind) {
    if (kind != GC_INTEGRATOR_LEAPFROG && kind != GC_INTEGRATOR_RK4) return GC_ERR_ARG;
    ctx->integ = kind;
    return GC_OK;
}

int oracle_set_integrator(oracle_ctx* ctx, double gamma) {
    ctx->gamma = gamma;
    return GC_OK;
}

int oracle_set_field(oracle_ctx* ctx, int handle, int field, const void* host, size_t bytes) {
    if (handle < 0 || handle >= (int)ctx->handles.size()) return fail(ctx, GC_ERR_ARG, "bad handle");
    const Handle& h = ctx->handles[handle];
    if (h.type == H_GHOST) return fail(ctx, GC_ERR_ARG, "ghost fields are generated, not set");
    if (h.type == H_VIRT && !ctx->virts[h.idx].probe)
        return fail(ctx, GC_ERR_ARG, "a virtual system's fields are its source's");
    Sys& s = ctx->sys[h.type == H_VIRT ? ctx->virts[h.idx].src : h.idx];
    int comps = field_comps(s, field);
    if (comps < 0) return fail(ctx, GC_ERR_ARG, "field not present on this system");
    if (bytes != (size_t)s.n * comps * 8) return fail(ctx, GC_ERR_ARG, "byte count mismatch");
    if (field == GC_FIELD_ID) {
        std::memcpy(s.id.data(), host, bytes);
        return GC_OK;
    }
    std::vector<double>* vec = field_vec(s, field);
    std::memcpy(vec->data(), host, bytes);
    if (ctx->track_mag) {
        mag_ensure(s);
        if (field == GC_FIELD_V) std::fill(s.mvi.begin(), s.mvi.end(), 0.0);
        if (field == GC_FIELD_RHO) std::fill(s.mrhoi.begin(), s.mrhoi.end(), 0.0);
        if (field == GC_FIELD_X) std::fill(s.mxi.begin(), s.mxi.end(), 0.0);
        if (field == GC_FIELD_STRESS) std::fill(s.mstr.begin(), s.mstr.end(), 0.0);
        if (field == GC_FIELD_STRAIN) std::fill(s.mstrain.begin(), s.mstrain.end(), 0.0);
        if (field == GC_FIELD_DVDT) mag_set(s.dvdt, s.mdvdt);
        if (field == GC_FIELD_DRHODT) mag_set(s.drhodt, s.mdrhodt);
        if (field == GC_FIELD_STRAIN_RATE) mag_set(s.sr, s.msr);
        if (field == GC_FIELD_VORTICITY) mag_set(s.vort, s.mvort);
    }
    return GC_OK;
}

// Test infrastructure: keep the rate fields' magnitude shadows, summing
// each pair term's magnitude (mode 1) or the magnitude it takes with every
// difference of its inputs replaced by the sum of their magnitudes (mode 2);
// 0 turns them off.  Switching on sets every shadow to |field| (rates) or 0
// (integrated fields).
int oracle_set_track_magnitude(oracle_ctx* ctx, int on) {
    if (on < 0 || on > 2) return fail(ctx, GC_ERR_ARG, "magnitude mode is 0, 1 or 2");
    ctx->track_mag = on;
    for (auto& s : ctx->sys) {
        if (ctx->track_mag) {
            mag_set(s.dvdt, s.mdvdt);
            mag_set(s.drhodt, s.mdrhodt);
            mag_set(s.sr, s.msr);
            mag_set(s.vort, s.mvort);
            s.mvi.assign(s.v.size(), 0.0);
            s.mrhoi.assign(s.rho.size(), 0.0);
            s.mxi.assign(s.x.size(), 0.0);
            s.mstr.assign(s.stress.size(), 0.0);
            s.mstrain.assign(s.strain.size(), 0.0);
        } else {
            s.mstr.clear();
            s.mstrain.clear();
            s.mvi.clear();
            s.mrhoi.clear();
            s.mxi.clear();
            s.mdvdt.clear();
            s.mdrhodt.clear();
            s.msr.clear();
            s.mvort.clear();
        }
    }
    return GC_OK;
}

// The magnitude shadow of a rate field (dvdt, drhodt, strain rate,
// vorticity) or of an integrated field (v, rho, x, stress, strain: the
// summed increments' magnitudes) of a system, in the layout of
// oracle_get_field.
int oracle_get_magnitude(oracle_ctx* ctx, int handle, int field, void* host, size_t bytes) {
    if (!ctx->track_mag) return fail(ctx, GC_ERR_STATE, "magnitude tracking is off");
    if (handle < 0 || handle >= (int)ctx->handles.size()) return fail(ctx, GC_ERR_ARG, "bad handle");
    const Handle& h = ctx->handles[handle];
    if (h.type != H_SYS) return fail(ctx, GC_ERR_ARG, "magnitudes are kept for systems only");
    Sys& s = ctx->sys[h.idx];
    mag_ensure(s);
    const std::vector<double>* m = field == GC_FIELD_DVDT          ? &s.mdvdt
                                   : field == GC_FIELD_DRHODT      ? &s.mdrhodt
                                   : field == GC_FIELD_STRAIN_RATE ? &s.msr
                                   : field == GC_FIELD_VORTICITY   ? &s.mvort
                                   : field == GC_FIELD_V           ? &s.mvi
                                   : field == GC_FIELD_RHO         ? &s.mrhoi
                                   : field == GC_FIELD_X           ? &s.mxi
                                   : field == GC_FIELD_STRESS      ? &s.mstr
                                   : field == GC_FIELD_STRAIN      ? &s.mstrain
                                                                   : nullptr;
    if (!m) return fail(ctx, GC_ERR_ARG, "no magnitude shadow for this field");
    if (bytes != m->size() * 8) return fail(ctx, GC_ERR_ARG, "byte count mismatch");
    if (bytes) std::memcpy(host, m->data(), bytes);
    return GC_OK;
}

int oracle_get_count(oracle_ctx* ctx, int handle, int64_t* n_out) {
    if (handle < 0 || handle >= (int)ctx->handles.size()) return fail(ctx, GC_ERR_ARG, "bad handle");
    const Handle& h = ctx->handles[handle];
    *n_out = h.type == H_GHOST  ? ctx->ghosts[h.idx].n
             : h.type == H_VIRT ? ctx->sys[ctx->virts[h.idx].src].n
                                : ctx->sys[h.idx].n;
    return GC_OK;
}

int oracle_get_field(oracle_ctx* ctx, int handle, int field, void* host, size_t bytes) {
    if (handle < 0 || handle >= (int)ctx->handles.size()) return fail(ctx, GC_ERR_ARG, "bad handle");
    const Handle& h = ctx->handles[handle];
    if (h.type == H_VIRT) {
        const Virt& vp = ctx->virts[h.idx];
        if (field == GC_FIELD_W_SUM) {
            if (bytes != vp.wsum.size() * 8) return fail(ctx, GC_ERR_ARG, "byte count mismatch");
            if (bytes) std::memcpy(host, vp.wsum.data(), bytes);
            return GC_OK;
        }
        if (!vp.probe) return fail(ctx, GC_ERR_ARG, "a virtual system's fields are its source's");
        Sys& p = ctx->sys[vp.src];
        const int comps = field == GC_FIELD_COUNT ? 1 : field_comps(p, field);
        if (comps < 0) return fail(ctx, GC_ERR_ARG, "field not present on this probe");
        if (bytes != (size_t)p.n * comps * 8) return fail(ctx, GC_ERR_ARG, "byte count mismatch");
        if (field == GC_FIELD_ID) std::memcpy(host, p.id.data(), bytes);
        else std::memcpy(host, (field == GC_FIELD_COUNT ? &p.drhodt : field_vec(p, field))->data(), bytes);
        return GC_OK;
    }
    if (h.type == H_GHOST) {
        Ghost& g = ctx->ghosts[h.idx];
        const Sys& s = ctx->sys[g.src];
        const void* src = nullptr;
        size_t need = 0;
        switch (field) {
            case GC_FIELD_X: src = g.x.data(); need = g.n * s.nd * 8; break;
            case GC_FIELD_V: src = g.v.data(); need = g.n * s.nd * 8; break;
            case GC_FIELD_RHO: src = g.rho.data(); need = g.n * 8; break;
            case GC_FIELD_P: if (!g.ex_p) return fail(ctx, GC_ERR_ARG, "ghost has no p"); src = g.p.data(); need = g.n * 8; break;
            case GC_FIELD_STRESS: if (!g.ex_stress) return fail(ctx, GC_ERR_ARG, "ghost has no stress"); src = g.stress.data(); need = g.n * s.ns * 8; break;
            case GC_FIELD_IDX_ORIGINAL: src = g.io.data(); need = g.n * 8; break;
            case GC_FIELD_IDX_BOUNDARY: src = g.ib.data(); need = g.n * 8; break;
            case GC_FIELD_NORMALS: src = g.normals.data(); need = g.n * s.nd * 8; break;
            default: return fail(ctx, GC_ERR_ARG, "field not present on ghosts");
        }
        if (bytes != need) return fail(ctx, GC_ERR_ARG, "byte count mismatch");
        if (need) std::memcpy(host, src, need);
        return GC_OK;
    }
    Sys& s = ctx->sys[h.idx];
    int comps = field_comps(s, field);
    if (comps < 0) return fail(ctx, GC_ERR_ARG, "field not present on this system");
    if (bytes != (size_t)s.n * comps * 8) return fail(ctx, GC_ERR_ARG, "byte count mismatch");
    if (field == GC_FIELD_ID) {
        std::memcpy(host, s.id.data(), bytes);
        return GC_OK;
    }
    std::memcpy(host, field_vec(s, field)->data(), bytes);
    return GC_OK;
}

int oracle_step(oracle_ctx* ctx, int nsteps, double cfl) {
    if (ctx->inters.empty()) return fail(ctx, GC_ERR_ARG, "interactions must not be empty");
    const int nst = num_stages(ctx);
    for (auto& it : ctx->inters)
        if (!it.probe && it.nstages != nst)
            return fail(ctx, GC_ERR_ARG, "All interactions must have the same number of stages");
    double dt = compute_dt(ctx, cfl);
    for (int s = 0; s < nsteps; ++s) {
        int st = ctx->integ == GC_INTEGRATOR_RK4 ? step_rk4(ctx, dt) : step_once(ctx, dt);
        if (st) return st;
    }
    return GC_OK;
}

int oracle_sort_system(oracle_ctx* ctx, int handle, double cutoff, int64_t* perm_out) {
    if (handle < 0 || handle >= (int)ctx->handles.size()) return fail(ctx, GC_ERR_ARG, "bad handle");
    const Handle& h = ctx->handles[handle];
    std::vector<int64_t> perm;
    int st;
    int64_t n;
    if (h.type == H_GHOST) {
        Ghost& g = ctx->ghosts[h.idx];
        st = sort_ghost(g, ctx->sys[g.src].nd, ctx->sys[g.src].ns, cutoff, &perm);
        n = g.n;
    } else {
        st = sort_system(ctx->sys[h.idx], cutoff, &perm);
        n = ctx->sys[h.idx].n;
    }
    if (st) return fail(ctx, st, "sort failed: non-finite position");
    if (perm_out)
        for (int64_t i = 0; i < n; ++i) perm_out[i] = perm[i] + 1;
    return GC_OK;
}

int oracle_build_grid(oracle_ctx* ctx, int inter, int64_t* cell_start_out, int64_t cap, double* mingridx_out,
                      int64_t* ngridx_out, int64_t* ncells_out) {
    if (inter < 0 || inter >= (int)ctx->inters.size()) return fail(ctx, GC_ERR_ARG, "bad interaction");
    Inter& it = ctx->inters[inter];
    int st = create_grid(ctx, it);
    if (st) return st;
    const int nd = ctx->sys[it.a].nd;
    int64_t ncells = (int64_t)it.cs.size() - 1;
    if (ncells_out) *ncells_out = ncells;
    if (mingridx_out)
        for (int d = 0; d < nd; ++d) mingridx_out[d] = it.ming[d];
    if (ngridx_out)
        for (int d = 0; d < nd; ++d) ngridx_out[d] = it.ng[d];
    if (cell_start_out) {
        if (cap < ncells + 1) return fail(ctx, GC_ERR_CAPACITY, "cell_start buffer too small");
        std::memcpy(cell_start_out, it.cs.data(), (size_t)(ncells + 1) * 8);
    }
    return GC_OK;
}

// Coupled grids also carry system_a's CSR (src/Interaction.jl:168-172).
int oracle_grid_cell_start_a(oracle_ctx* ctx, int inter, int64_t* out, int64_t cap) {
    Inter& it = ctx->inters[inter];
    if (it.csa.empty()) return fail(ctx, GC_ERR_STATE, "no system_a grid");
    if (cap < (int64_t)it.csa.size()) return fail(ctx, GC_ERR_CAPACITY, "buffer too small");
    std::memcpy(out, it.csa.data(), it.csa.size() * 8);
    return GC_OK;
}

int oracle_generate_ghosts(oracle_ctx* ctx, int ghost) {
    if (ghost < 0 || ghost >= (int)ctx->handles.size() || ctx->handles[ghost].type != H_GHOST)
        return fail(ctx, GC_ERR_ARG, "not a ghost handle");
    generate_ghosts(ctx, ctx->ghosts[ctx->handles[ghost].idx]);
    return GC_OK;
}

int oracle_update_ghost_kinematics(oracle_ctx* ctx, int ghost) {
    if (ghost < 0 || ghost >= (int)ctx->handles.size() || ctx->handles[ghost].type != H_GHOST)
        return fail(ctx, GC_ERR_ARG, "not a ghost handle");
    ghost_kinematics(ctx, ctx->ghosts[ctx->handles[ghost].idx]);
    return GC_OK;
}

int oracle_update_ghost(oracle_ctx* ctx, int ghost, int stage) {
    if (ghost < 0 || ghost >= (int)ctx->handles.size() || ctx->handles[ghost].type != H_GHOST)
        return fail(ctx, GC_ERR_ARG, "not a ghost handle");
    update_ghost(ctx, ctx->ghosts[ctx->handles[ghost].idx], stage);
    return GC_OK;
}

int oracle_sweep(oracle_ctx* ctx, int inter, int stage) {
    if (inter < 0 || inter >= (int)ctx->inters.size()) return fail(ctx, GC_ERR_ARG, "bad interaction");
    return sweep(ctx, ctx->inters[inter], stage);
}

int oracle_update_state(oracle_ctx* ctx, int sys, int stage, double dt) {
    if (sys >= 0 && sys < (int)ctx->handles.size() && ctx->handles[sys].type == H_VIRT) {
        Virt& vp = ctx->virts[ctx->handles[sys].idx];
        if (stage >= 1 && stage <= (int)vp.upd.size())
            for (const Upd& u : vp.upd[stage - 1]) apply_virtual_updater(ctx->sys[vp.src], vp, u, dt);
        return GC_OK;
    }
    int si = sys_index(ctx, sys);
    if (si < 0) return fail(ctx, GC_ERR_ARG, "not a system handle");
    update_state(ctx->sys[si], stage, dt);
    return GC_OK;
}

// Kernel primitives for the known-answer tests (src/Kernels.jl).
double oracle_kernel_norm(int kind, int nd, double H) { return make_kernel(kind, nd, H).norm; }
double oracle_kernel_w(int kind, int nd, double H, double q) { return kernel_w(make_kernel(kind, nd, H), q); }
double oracle_kernel_dw_dq(int kind, int nd, double H, double q) {
    return kernel_dw_dq(make_kernel(kind, nd, H), q);
}
double oracle_powi(double x, int64_t n) { return comp_powi(x, n); }

// Number of leapfrog steps done.
int64_t oracle_steps(oracle_ctx* ctx) { return ctx->steps; }

}  // extern "C"
