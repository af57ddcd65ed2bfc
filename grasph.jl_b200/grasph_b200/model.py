"""Host-side mirror of Grasph.jl's model API.

The classes below keep the names, constructor arguments, validation and
error behaviour of the Julia API on the hot path, so code (and tests)
written against Grasph.jl translate line for line.  They hold host state in
numpy arrays shaped like Julia's ``Vector{SVector{K,Float64}}`` (``(n, K)``,
row-major, i.e. the same bytes as Julia's AoS layout).  Numerical work is
never done here: `grasph_b200.engine` ships the model to libgrasph_cuda.so.

Reference counterparts (Grasph.jl source tree):
  particle systems   src/Particles.jl:38,149,245,351
  boundary wrappers  src/BoundaryParticles.jl:38,68
  ghosts             src/GhostParticles.jl:53,174,300
  kernels            src/Kernels.jl:18,92
  pair functors      src/PairwiseFunctors.jl:18,78,136,252
  state updaters     src/StateUpdaters.jl:30,108,131,202,356
  interaction        src/Interaction.jl:23,61
  integrator         src/TimeIntegration.jl:29,53
"""
from __future__ import annotations

import math
from typing import Iterable, Sequence

import numpy as np

from . import consts as C


class ArgumentError(ValueError):
    """Mirror of Julia's ``ArgumentError`` for invalid constructor input."""


# ------------------------------------------------------------ element types
#
# A particle system's element type T is Float64 (default) or Float32
# (src/Particles.jl:67,78).  Its arrays, mass and c are stored in T; kernels,
# functors and updaters built from float32 values are specialised on
# Float32.  The device library computes every system in the session's
# precision from the values widened to Float64 and rounds the results back
# to T on download.

_JULIA_NAME = {np.dtype(np.float32): "Float32", np.dtype(np.float64): "Float64"}


def _elt(dtype):
    """`dtype` as a numpy float type (Float32 or Float64)."""
    try:
        d = np.dtype(dtype)
    except TypeError:
        d = None
    if d not in _JULIA_NAME:
        raise ArgumentError(f"dtype must be Float32 or Float64, got {dtype}")
    return d.type


def _promote(*vals):
    """The float type Julia's `promote(float.(vals)...)` gives: Float32 when
    every value is a float32, Float64 once any is not (integers and Python
    floats promote to Float64)."""
    vs = [v for v in vals if v is not None]
    if vs and all(isinstance(v, np.float32) for v in vs):
        return np.float32
    return np.float64


def _scalar(t, v):
    """A T-typed scalar: a Python float for Float64, np.float32 for Float32."""
    return float(v) if t is np.float64 else np.float32(v)


def float_type(functor):
    """The AbstractFloat type parameter a functor is specialised on, or None
    for an unparameterised one (a function, ``nothing``, a tuple)."""
    return getattr(functor, "_elt", None)


def _check_functors_eltype(functors, T, label):
    """src/Utils.jl:59-78: a functor specialised on a float type other than
    the target's raises ArgumentError."""
    for f in functors:
        P = float_type(f)
        if P is not None and P is not T:
            raise ArgumentError(
                f"{label} {type(f).__name__} is specialised on {_JULIA_NAME[np.dtype(P)]} "
                f"but target expects {_JULIA_NAME[np.dtype(T)]}; construct it with "
                f"{_JULIA_NAME[np.dtype(T)]} values")


# ---------------------------------------------------------------- systems

class AbstractParticleSystem:
    """Common base; concrete types mirror src/Particles.jl."""

    kind = C.GC_SYS_BASIC
    has_p = False
    has_stress = False
    is_ep = False

    def __init__(self, name: str, n: int, ndims: int, mass: float, c: float, *,
                 ns: int = 0, dtype=np.float64, source_v=None, source_rho: float = 0.0,
                 state_updater=()):
        n = int(n)
        ndims = int(ndims)
        if n <= 0:
            raise ArgumentError(f"n must be positive, got {n}")
        if ndims <= 0:
            raise ArgumentError(f"ndims must be positive, got {ndims}")
        T = _elt(dtype)
        if source_v is None:
            source_v = np.zeros(ndims)
        source_v = np.asarray(source_v, dtype=T)
        if source_v.shape != (ndims,):
            raise ArgumentError(
                f"length(source_v) = {source_v.size} must equal ndims = {ndims}")
        ups = state_updater if isinstance(state_updater, tuple) else (state_updater,)
        _check_functors_eltype(ups, T, "state updater")
        self.dtype = np.dtype(T)
        self.name = str(name)
        self.n = n
        self.ndims = ndims
        self.ns = int(ns)
        self.mass = _scalar(T, mass)
        self.c = _scalar(T, c)
        self.source_v = source_v
        self.source_rho = _scalar(T, source_rho)
        self.id = np.arange(1, n + 1, dtype=np.int64)
        self.x = np.zeros((n, ndims), T)
        self.v = np.zeros((n, ndims), T)
        self.v_adjustment = np.zeros((n, ndims), T)
        self.rho = np.zeros(n, T)
        self.dvdt = np.zeros((n, ndims), T)
        self.drhodt = np.zeros(n, T)
        self.state_updater = ups

    # Fields in the order of src/Sorting.jl:15-26 (the arrays a sort permutes).
    def particle_fields(self):
        f = [("x", C.GC_FIELD_X), ("id", C.GC_FIELD_ID), ("v", C.GC_FIELD_V),
             ("v_adjustment", C.GC_FIELD_V_ADJUSTMENT), ("rho", C.GC_FIELD_RHO),
             ("dvdt", C.GC_FIELD_DVDT), ("drhodt", C.GC_FIELD_DRHODT)]
        if self.has_p:
            f.append(("p", C.GC_FIELD_P))
        if self.has_stress:
            f += [("stress", C.GC_FIELD_STRESS), ("strain_rate", C.GC_FIELD_STRAIN_RATE)]
        if self.is_ep:
            f += [("vorticity", C.GC_FIELD_VORTICITY), ("strain", C.GC_FIELD_STRAIN),
                  ("strain_p", C.GC_FIELD_STRAIN_P)]
        return f

    def __repr__(self):
        return f"{type(self).__name__}({self.name!r}, n={self.n}, ndims={self.ndims})"


class BasicParticleSystem(AbstractParticleSystem):
    """src/Particles.jl:38-101."""

    kind = C.GC_SYS_BASIC

    def __init__(self, name, n, ndims, mass, c, **kw):
        super().__init__(name, n, ndims, mass, c, **kw)


class FluidParticleSystem(AbstractParticleSystem):
    """src/Particles.jl:149-214 (Basic fields plus pressure ``p``)."""

    kind = C.GC_SYS_FLUID
    has_p = True

    def __init__(self, name, n, ndims, mass, c, **kw):
        super().__init__(name, n, ndims, mass, c, **kw)
        self.p = np.zeros(self.n, self.dtype)


class StressParticleSystem(AbstractParticleSystem):
    """src/Particles.jl:245-317 (Fluid fields plus Voigt ``stress``, ``strain_rate``)."""

    kind = C.GC_SYS_STRESS
    has_p = True
    has_stress = True

    def __init__(self, name, n, ndims, ns, mass, c, **kw):
        ns = int(ns)
        if ns not in (3, 4, 6):
            raise ArgumentError(f"ns must be 3, 4, or 6, got {ns}")
        super().__init__(name, n, ndims, mass, c, ns=ns, **kw)
        self.p = np.zeros(self.n, self.dtype)
        self.stress = np.zeros((self.n, ns), self.dtype)
        self.strain_rate = np.zeros((self.n, ns), self.dtype)


class ElastoPlasticParticleSystem(StressParticleSystem):
    """src/Particles.jl:351-430 (Stress fields plus vorticity, strain, strain_p).

    2-D vorticity is a scalar per particle, 3-D a 3-vector (:401)."""

    kind = C.GC_SYS_ELASTOPLASTIC
    is_ep = True

    def __init__(self, name, n, ndims, ns, mass, c, **kw):
        super().__init__(name, n, ndims, ns, mass, c, **kw)
        T = self.dtype
        self.vorticity = np.zeros(self.n, T) if self.ndims == 2 else np.zeros((self.n, 3), T)
        self.strain = np.zeros((self.n, self.ns), T)
        self.strain_p = np.zeros((self.n, self.ns), T)


# --------------------------------------------------------------- wrappers

class AbstractBoundarySystem:
    """Wrapper that forwards every field to ``inner`` (src/BoundaryParticles.jl:13-20)."""

    wrap_kind = 0

    def __getattr__(self, item):
        return getattr(self.__dict__["inner"], item)


class StaticBoundarySystem(AbstractBoundarySystem):
    """Lennard-Jones repulsion boundary, src/BoundaryParticles.jl:38-49."""

    wrap_kind = C.GC_WRAP_STATIC

    def __init__(self, inner: AbstractParticleSystem, lj_cutoff: float):
        self.inner = inner
        self.lj_cutoff = float(lj_cutoff)


class DynamicBoundarySystem(AbstractBoundarySystem):
    """Distance-ratio velocity boundary, src/BoundaryParticles.jl:68-86."""

    wrap_kind = C.GC_WRAP_DYNAMIC

    def __init__(self, inner: AbstractParticleSystem, normal, point, beta: float):
        nd = inner.ndims
        self.inner = inner
        self.boundary_normal = np.asarray(normal, dtype=np.float64).reshape(nd)
        self.boundary_point = np.asarray(point, dtype=np.float64).reshape(nd)
        self.boundary_beta = float(beta)


# ----------------------------------------------------------------- ghosts

class HouseholderReflect:
    """Marker: reflect a Voigt tensor by H σ H (src/GhostParticles.jl:26)."""


_FIELD_BY_NAME = {"p": C.GC_FIELD_P, "stress": C.GC_FIELD_STRESS, "rho": C.GC_FIELD_RHO}


class GhostCopier:
    """Per-stage field copier, src/GhostParticles.jl:53-59.

    Entries are field names, or ``(name, HouseholderReflect())`` pairs."""

    def __init__(self, *entries):
        self.entries = []
        for e in entries:
            if isinstance(e, tuple):
                name, mode = e
                if not isinstance(mode, HouseholderReflect):
                    raise ArgumentError("copy mode must be HouseholderReflect()")
                m = C.GC_COPY_HOUSEHOLDER
            else:
                name, m = e, C.GC_COPY_PLAIN
            name = str(name).lstrip(":")
            if name not in _FIELD_BY_NAME:
                raise ArgumentError(f"unsupported ghost copier field :{name}")
            self.entries.append((name, m))

    @property
    def fields(self):
        return tuple(n for n, _ in self.entries)


class GhostParticleSystem:
    """Mirror particles owned per step, src/GhostParticles.jl:174-220."""

    def __init__(self, ps: AbstractParticleSystem, *updaters, name=None):
        for u in updaters:
            if u is not None and not isinstance(u, GhostCopier):
                raise ArgumentError("ghost updaters must be GhostCopier or nothing")
        self.source = ps
        self.name = f"ghost({ps.name})" if name is None else str(name)
        self.updaters = tuple(updaters)
        seen = []
        for u in self.updaters:
            if u is None:
                continue
            for f in u.fields:
                if f not in seen:
                    seen.append(f)
        self.extras_fields = tuple(seen)
        nd = ps.ndims
        self.x = np.zeros((0, nd))
        self.v = np.zeros((0, nd))
        self.rho = np.zeros(0)
        self.idx_original = np.zeros(0, dtype=np.int64)
        self.idx_boundary = np.zeros(0, dtype=np.int64)
        self.normals = np.zeros((0, nd))
        self.extras = {f: (np.zeros(0) if f != "stress" else np.zeros((0, ps.ns)))
                       for f in self.extras_fields}

    @property
    def n(self):
        return self.x.shape[0]

    @property
    def ndims(self):
        return self.source.ndims

    @property
    def mass(self):
        return self.source.mass

    @property
    def c(self):
        return self.source.c

    def __getattr__(self, item):
        ex = self.__dict__.get("extras", {})
        if item in ex:
            return ex[item]
        return getattr(self.__dict__["source"], item)


class GhostEntry:
    """A ghost system plus its boundary planes, src/GhostParticles.jl:300-329."""

    def __init__(self, ghost: GhostParticleSystem, cutoff: float, *boundary_pairs,
                 capacity: int = 0):
        if not boundary_pairs:
            raise ArgumentError("at least one boundary (normal, point) pair is required")
        nd = ghost.ndims
        self.ghost = ghost
        self.cutoff = float(cutoff)
        self.normals = np.array([np.asarray(nrm, dtype=np.float64).reshape(nd)
                                 for nrm, _ in boundary_pairs])
        self.points = np.array([np.asarray(pt, dtype=np.float64).reshape(nd)
                                for _, pt in boundary_pairs])
        self.capacity = int(capacity)

    @property
    def boundaries(self):
        return list(zip(self.normals, self.points))


# ---------------------------------------------------------------- kernels

class AbstractKernel:
    """Kernel of element type T = typeof(h) (src/Kernels.jl:33): h,
    norm_coeff and interaction_length are T values."""

    kind = C.GC_KERNEL_CUBIC_SPLINE

    def __init__(self, h: float, ndims: int = 3):
        self._elt = _promote(h)
        self.h = _scalar(self._elt, h)
        self.ndims = int(ndims)

    @property
    def interaction_length(self):
        return _scalar(self._elt, 2.0 * self.h)

    def _norm(self, v):
        return _scalar(self._elt, v)

    def _hpow(self, k):
        """H^k in T, as Julia's literal power: H*H, H*H*H."""
        H = self._elt(self.h)
        r = H
        for _ in range(k - 1):
            r = r * H
        return float(r)


class CubicSplineKernel(AbstractKernel):
    """src/Kernels.jl:18-81."""

    kind = C.GC_KERNEL_CUBIC_SPLINE

    @property
    def norm_coeff(self):
        H = float(self.h)
        if self.ndims == 1:
            return self._norm(2.0 / (3.0 * H))
        if self.ndims == 2:
            return self._norm(10.0 / ((7.0 * math.pi) * self._hpow(2)))
        return self._norm(1.0 / (math.pi * self._hpow(3)))


class WenlandC2Kernel(AbstractKernel):
    """src/Kernels.jl:92-153."""

    kind = C.GC_KERNEL_WENDLAND_C2

    @property
    def norm_coeff(self):
        if self.ndims == 2:
            return self._norm(7.0 / ((64.0 * math.pi) * self._hpow(2)))
        return self._norm(21.0 / ((256.0 * math.pi) * self._hpow(3)))


# ----------------------------------------------------------- pair functors

class _Pfn:
    kind = C.GC_PFN_NONE

    def params(self):
        p = np.zeros(C.GC_PFN_NPARAM)
        p[4] = np.nan
        p[5] = np.nan
        return p


class FluidPfn(_Pfn):
    """Weakly-compressible momentum + continuity, src/PairwiseFunctors.jl:136-242."""

    kind = C.GC_PFN_FLUID

    def __init__(self, alpha, beta, h, *, sigma=2, delta=None, epsilon=None):
        T = self._elt = _promote(alpha, beta, h)
        self.art_visc_alpha = _scalar(T, alpha)
        self.art_visc_beta = _scalar(T, beta)
        self.h = _scalar(T, h)
        self.sigma = int(sigma)
        if self.sigma not in (1, 2):
            raise ArgumentError("FluidPfn sigma must be 1 or 2 on the device path")
        self.delta = None if delta is None else _scalar(T, delta)
        # artificial surface tension: used by the two-sided fluid x fluid form only
        self.epsilon = None if epsilon is None else _scalar(T, epsilon)

    def params(self):
        p = super().params()
        p[0], p[1], p[2], p[3] = self.art_visc_alpha, self.art_visc_beta, self.h, self.sigma
        if self.delta is not None:
            p[4] = self.delta
        if self.epsilon is not None:
            p[5] = self.epsilon
        return p


class FluidSolidPfn(_Pfn):
    """Fluid against a linear-elastic solid, src/PairwiseFunctors.jl:463-519:
    the two-sided fluid form with the fluid's (system_a's) pressure on both
    sides.  Only the (system, system) method exists."""

    kind = C.GC_PFN_FLUID_SOLID

    def __init__(self, alpha, beta, h, *, sigma=2, delta=None):
        T = self._elt = _promote(alpha, beta, h)
        self.art_visc_alpha = _scalar(T, alpha)
        self.art_visc_beta = _scalar(T, beta)
        self.h = _scalar(T, h)
        self.sigma = int(sigma)
        if self.sigma not in (1, 2):
            raise ArgumentError("FluidSolidPfn sigma must be 1 or 2 on the device path")
        self.delta = None if delta is None else _scalar(T, delta)

    def params(self):
        p = super().params()
        p[0], p[1], p[2], p[3] = self.art_visc_alpha, self.art_visc_beta, self.h, self.sigma
        if self.delta is not None:
            p[4] = self.delta
        return p


class CauchyFluidPfn(_Pfn):
    """Cauchy-stress momentum + continuity, src/PairwiseFunctors.jl:252-355."""

    kind = C.GC_PFN_CAUCHY_FLUID

    def __init__(self, alpha, beta, h, *, delta=None):
        T = self._elt = _promote(alpha, beta, h)
        self.art_visc_alpha = _scalar(T, alpha)
        self.art_visc_beta = _scalar(T, beta)
        self.h = _scalar(T, h)
        self.delta = None if delta is None else _scalar(T, delta)

    def params(self):
        p = super().params()
        p[0], p[1], p[2], p[3] = self.art_visc_alpha, self.art_visc_beta, self.h, 2
        if self.delta is not None:
            p[4] = self.delta
        return p


class StrainRatePfn(_Pfn):
    """src/PairwiseFunctors.jl:18-70."""

    kind = C.GC_PFN_STRAIN_RATE


class StrainRateVorticityPfn(_Pfn):
    """src/PairwiseFunctors.jl:78-126."""

    kind = C.GC_PFN_STRAIN_RATE_VORTICITY


class CountingPfn(_Pfn):
    """Adds 1 to ``dvdt[:,0]`` and ``drhodt`` of both pair endpoints: the
    counting functor of the reference's sweep tests
    (test/test_interaction_sweep.jl:14-30)."""

    kind = C.GC_PFN_COUNT


_INTERP_FIELDS = {"v": C.GC_FIELD_V, "rho": C.GC_FIELD_RHO, "stress": C.GC_FIELD_STRESS}


class InterpolateFieldFn(_Pfn):
    """SPH interpolation f_j += (m_i/ρ_i)·f_i·W_ij from real system_a particles
    into a VirtualParticleSystem system_b, src/PairwiseFunctors.jl:392-428."""

    kind = C.GC_PFN_INTERPOLATE

    def __init__(self, *fields, accumulate_wsum=True):
        names = [str(f).lstrip(":") for f in fields]
        if not names:
            raise ArgumentError("InterpolateFieldFn needs at least one field")
        for n in names:
            if n not in _INTERP_FIELDS:
                raise ArgumentError(f"InterpolateFieldFn: field :{n} has no device implementation")
        self.fields = tuple(names)
        self.accumulate_wsum = bool(accumulate_wsum)

    def params(self):
        p = super().params()
        p[0] = float(sum(1 << _INTERP_FIELDS[n] for n in self.fields))
        p[1] = 1.0 if self.accumulate_wsum else 0.0
        return p


class NeighborCountFn(_Pfn):
    """probe.field[j] += 1 per neighbour, src/PairwiseFunctors.jl:442-460."""

    kind = C.GC_PFN_NEIGHBOR_COUNT

    def __init__(self, field):
        self.field = str(field).lstrip(":")


class XSPHPfn(_Pfn):
    """XSPH velocity smoothing, src/PairwiseFunctors.jl:357-389; only as a
    `velocity_adjust_pairwise_fn` (swept by adjust_v! in the step's XSPH
    correction, src/TimeIntegration.jl:421-436)."""

    kind = C.GC_PFN_XSPH

    def __init__(self, epsilon):
        T = self._elt = _promote(epsilon)
        self.epsilon = _scalar(T, epsilon)


def _pfn_kind(p):
    return C.GC_PFN_NONE if p is None else p.kind


def _pfn_params(p):
    return _Pfn().params() if p is None else p.params()


# ---------------------------------------------------------- state updaters

class _Updater:
    kind = C.GC_UPD_NONE

    def params(self):
        return np.zeros(C.GC_UPD_NPARAM)

    def entries(self):
        """(kind, params) chain entries this updater compiles to."""
        return [(self.kind, self.params())]


class ZeroFieldUpdater(_Updater):
    """src/StateUpdaters.jl:30-42."""

    kind = C.GC_UPD_ZERO_FIELDS
    _ok = {"strain_rate": C.GC_FIELD_STRAIN_RATE, "vorticity": C.GC_FIELD_VORTICITY,
           "p": C.GC_FIELD_P, "stress": C.GC_FIELD_STRESS, "dvdt": C.GC_FIELD_DVDT,
           "drhodt": C.GC_FIELD_DRHODT}

    def __init__(self, *fields):
        names = [str(f).lstrip(":") for f in fields]
        for n in names:
            if n not in self._ok:
                raise ArgumentError(f"ZeroFieldUpdater: unsupported field :{n}")
        self.fields = tuple(names)

    def params(self):
        p = super().params()
        mask = 0
        for n in self.fields:
            mask |= 1 << self._ok[n]
        p[0] = float(mask)
        return p


class TaitEOSUpdater(_Updater):
    """p = ρ0 c²/γ ((ρ/ρ0)^γ − 1), src/StateUpdaters.jl:108-118."""

    kind = C.GC_UPD_TAIT_EOS

    def __init__(self, rho0, gamma=None):
        T = self._elt = _promote(rho0)
        self.rho0 = _scalar(T, rho0)
        self.gamma = _scalar(T, 7.0 if gamma is None else gamma)

    def params(self):
        p = super().params()
        p[0], p[1] = self.rho0, self.gamma
        return p


class LinearEOSUpdater(_Updater):
    """p = c² (ρ − ρ0), src/StateUpdaters.jl:131-140."""

    kind = C.GC_UPD_LINEAR_EOS

    def __init__(self, rho0):
        T = self._elt = _promote(rho0)
        self.rho0 = _scalar(T, rho0)

    def params(self):
        p = super().params()
        p[0] = self.rho0
        return p


class ElastoPlasticStressUpdater(_Updater):
    """Jaumann + Drucker–Prager return mapping, src/StateUpdaters.jl:202-335."""

    kind = C.GC_UPD_ELASTOPLASTIC

    def __init__(self, E, nu, phi, psi, cohesion):
        T = self._elt = _promote(E, nu, phi, psi, cohesion)
        self.E, self.nu, self.phi, self.psi, self.cohesion = (_scalar(T, v) for v in (E, nu, phi, psi, cohesion))

    def params(self):
        p = super().params()
        p[:5] = [self.E, self.nu, self.phi, self.psi, self.cohesion]
        return p


class VirtualNormUpdater(_Updater):
    """Normalise the listed fields of a VirtualParticleSystem by its w_sum
    and apply the velocity multiplier, src/StateUpdaters.jl:44-76."""

    kind = C.GC_UPD_VIRTUAL_NORM
    _ok = {"v": C.GC_FIELD_V, "rho": C.GC_FIELD_RHO, "p": C.GC_FIELD_P, "stress": C.GC_FIELD_STRESS}

    def __init__(self, v_mult, *fields):
        vm = np.asarray(v_mult)
        self._elt = np.float32 if vm.dtype == np.float32 else np.float64
        self.v_mult = vm.astype(self._elt).ravel()
        names = [str(f).lstrip(":") for f in fields]
        for n in names:
            if n not in self._ok:
                raise ArgumentError(f"VirtualNormUpdater: field :{n} has no device implementation")
        self.fields = tuple(names)

    def params(self):
        p = super().params()
        p[:self.v_mult.size] = self.v_mult
        p[3] = float(sum(1 << self._ok[n] for n in self.fields))
        return p


class PrescribedVelocityUpdater(_Updater):
    """v += prescribed_v on a VirtualParticleSystem, src/StateUpdaters.jl:78-97."""

    kind = C.GC_UPD_PRESCRIBED_V


class HookeLawStressUpdater(_Updater):
    """Plane-strain Hooke update, src/StateUpdaters.jl:356-405."""

    kind = C.GC_UPD_HOOKE

    def __init__(self, E, nu):
        T = self._elt = _promote(E, nu)
        self.E, self.nu = _scalar(T, E), _scalar(T, nu)

    def params(self):
        p = super().params()
        p[0], p[1] = self.E, self.nu
        return p


class ViscoPlasticMCStressUpdater(_Updater):
    """Rigid-plastic Mohr–Coulomb stress along the strain rate after an EOS
    update, src/StateUpdaters.jl:144-186.  Compiles to two chain entries:
    the EOS, then the stress part."""

    kind = C.GC_UPD_VISCOPLASTIC_MC

    def __init__(self, eos, friction_angle, cohesion):
        if not isinstance(eos, (TaitEOSUpdater, LinearEOSUpdater)):
            raise ArgumentError("ViscoPlasticMCStressUpdater: eos must be an EOS updater")
        self.eos = eos
        T = self._elt = _promote(friction_angle, cohesion)
        self.friction_angle = _scalar(T, friction_angle)
        self.cohesion = _scalar(T, cohesion)

    def params(self):
        p = super().params()
        p[0], p[1] = self.friction_angle, self.cohesion
        return p

    def entries(self):
        return self.eos.entries() + [(self.kind, self.params())]


def updater_chains(ps: AbstractParticleSystem):
    """The state_updater tuple as per-stage chains of (kind, params)."""
    chains = []
    for entry in ps.state_updater:
        if entry is None:
            chains.append([])
        elif isinstance(entry, tuple):
            chains.append([e for u in entry if u is not None for e in u.entries()])
        elif isinstance(entry, _Updater):
            chains.append(entry.entries())
        else:
            raise ArgumentError(f"unsupported state updater {type(entry).__name__}")
    return chains


# ------------------------------------------------------------ interaction

class SystemInteraction:
    """src/Interaction.jl:23-92."""

    def __init__(self, kernel: AbstractKernel, pairwise_fn, system_a, system_b=None, *,
                 velocity_adjust_pairwise_fn=None):
        nd = system_a.ndims
        if kernel.ndims != nd:
            raise ArgumentError(f"kernel.ndims ({kernel.ndims}) must match system_a.ndims ({nd})")
        if system_b is not None and system_b.ndims != nd:
            raise ArgumentError(
                f"system_b.ndims ({system_b.ndims}) must match system_a.ndims ({nd})")
        if not isinstance(system_a, (AbstractParticleSystem, GhostParticleSystem)):
            raise ArgumentError("system_a must be a particle system")
        vpf = velocity_adjust_pairwise_fn
        if vpf is not None and not isinstance(vpf, XSPHPfn):
            raise ArgumentError(f"velocity-adjust functor {type(vpf).__name__} has no device implementation")
        self.kernel = kernel
        self.pfns = pairwise_fn if isinstance(pairwise_fn, tuple) else (pairwise_fn,)
        _check_functors_eltype(self.pfns, system_a.dtype.type, "pairwise functor")
        for f in self.pfns:
            if isinstance(f, XSPHPfn):
                raise ArgumentError("XSPHPfn is a velocity-adjust functor, not a stage functor")
        self.vadjust_pfn = vpf
        self.system_a = system_a
        self.system_b = system_b
        self.ndims = nd
        self._cell_size = 2.0 * kernel.h

    def is_coupled(self):
        return self.system_b is not None


def is_coupled(si: SystemInteraction) -> bool:
    return si.is_coupled()


# ------------------------------------------------------------- integrator

class VirtualParticleSystem:
    """A source system seen through SPH interpolation, src/Particles.jl:476-528.

    Every per-particle field is the source's (the same arrays); `w_sum`, the
    state updaters and `prescribed_v` are its own.  The source is not one of
    the integrator's systems: it is sorted with the virtual systems, never
    integrated, and moved by prescribed_v·dt after each step."""

    def __init__(self, ps: AbstractParticleSystem, name, n, ndims, mass, c, *, dtype=np.float64,
                 state_updater=(), zero_fields=(), prescribed_v=None):
        if int(ndims) != ps.ndims:
            raise ArgumentError(f"ndims={ndims} does not match source ndims={ps.ndims}")
        if int(n) != ps.n:
            raise ArgumentError(f"n={n} does not match source n={ps.n}")
        self.name = str(name)
        self.source = ps
        self.w_sum = np.zeros(ps.n)
        ups = state_updater if isinstance(state_updater, tuple) else (state_updater,)
        self.state_updater = ups
        zf = [str(f).lstrip(":") for f in zero_fields]
        for f in zf:
            if f not in ("v", "rho", "p", "stress", "dvdt", "drhodt", "strain_rate"):
                raise ArgumentError(f"zero_fields: :{f} has no device implementation")
        self.zero_fields = tuple(zf)
        pv = np.zeros(ps.ndims) if prescribed_v is None else np.asarray(prescribed_v, dtype=np.float64).ravel()
        if pv.shape != (ps.ndims,):
            raise ArgumentError("prescribed_v must have ndims components")
        self.prescribed_v = pv

    def __getattr__(self, name):
        # forwarded to the source (only reached for attributes not set above)
        if name == "source":
            raise AttributeError(name)
        return getattr(self.source, name)

    @property
    def zero_mask(self):
        ids = {"v": C.GC_FIELD_V, "rho": C.GC_FIELD_RHO, "p": C.GC_FIELD_P, "stress": C.GC_FIELD_STRESS,
               "dvdt": C.GC_FIELD_DVDT, "drhodt": C.GC_FIELD_DRHODT, "strain_rate": C.GC_FIELD_STRAIN_RATE}
        return sum(1 << ids[f] for f in self.zero_fields)


class ProbeParticleSystem:
    """Passive observers measured only at save cadence,
    src/ProbeParticles.jl:23-102.

    `ProbeParticleSystem(name, positions, ...)` or
    `ProbeParticleSystem(name, mirror_target, ...)` (positions taken from
    that system at each measurement).  `extras` maps names to per-probe
    arrays: v, rho, p, stress take InterpolateFieldFn sums, one integer
    array takes a NeighborCountFn count."""

    _fields = {"v": C.GC_FIELD_V, "rho": C.GC_FIELD_RHO, "p": C.GC_FIELD_P, "stress": C.GC_FIELD_STRESS}

    def __init__(self, name, positions_or_target, *, extras=None, state_updater=(), prescribed_v=None,
                 dtype=np.float64):
        if np.dtype(dtype) != np.float64:
            raise ArgumentError("only Float64 probes are supported by the device library")
        self.name = str(name)
        if isinstance(positions_or_target, AbstractParticleSystem):
            self.mirror_target = positions_or_target
            self.x = np.array(positions_or_target.x, dtype=np.float64)
        else:
            self.mirror_target = None
            self.x = np.array(positions_or_target, dtype=np.float64)
            if self.x.size == 0:
                raise ArgumentError("positions must not be empty")
        if self.x.ndim != 2:
            raise ArgumentError("positions must be n×ndims")
        self.n, self.ndims = self.x.shape
        self.id = np.arange(1, self.n + 1, dtype=np.int64)
        self.w_sum = np.zeros(self.n)
        self.extras = {}
        self.count_field = None
        for k, arr in (extras or {}).items():
            a = np.array(arr)
            if a.shape[0] != self.n:
                raise ArgumentError(f"extras.{k} has length {a.shape[0]} but n={self.n}")
            if k not in self._fields:
                if not np.issubdtype(a.dtype, np.integer) or self.count_field is not None:
                    raise ArgumentError(f"extras.{k}: only v, rho, p, stress and one integer count are supported")
                self.count_field = k
            self.extras[k] = a.astype(np.int64 if k == self.count_field else np.float64)
        ups = state_updater if isinstance(state_updater, tuple) else (state_updater,)
        self.state_updater = ups
        pv = np.zeros(self.ndims) if prescribed_v is None else np.asarray(prescribed_v, dtype=np.float64).ravel()
        if pv.shape != (self.ndims,):
            raise ArgumentError("prescribed_v must have ndims components")
        self.prescribed_v = pv

    def __getattr__(self, name):
        extras = self.__dict__.get("extras", {})
        if name in extras:
            return extras[name]
        mt = self.__dict__.get("mirror_target")
        if mt is not None:
            return getattr(mt, name)
        raise AttributeError(f"ProbeParticleSystem has no field {name}")

    @property
    def extras_mask(self):
        m = sum(1 << self._fields[k] for k in self.extras if k in self._fields)
        if self.count_field is not None:
            m |= 1 << C.GC_FIELD_COUNT
        return m

    @property
    def ns(self):
        return self.extras["stress"].shape[1] if "stress" in self.extras else 0


class LeapFrogTimeIntegrator:
    """src/TimeIntegration.jl:29-67."""

    kind = C.GC_INTEGRATOR_LEAPFROG

    def __init__(self, systems, interactions, *, ghosts=(), gamma=0.0, virtual_systems=(), probes=(),
                 probe_interactions=(), **kw):
        if "Γ" in kw:
            gamma = kw.pop("Γ")
        if kw:
            raise ArgumentError(f"unsupported integrator options {sorted(kw)}")
        sys_ = (systems,) if isinstance(systems, AbstractParticleSystem) else tuple(systems)
        ints = (interactions,) if isinstance(interactions, SystemInteraction) else tuple(interactions)
        gsts = (ghosts,) if isinstance(ghosts, GhostEntry) else tuple(ghosts)
        if not sys_:
            raise ArgumentError("systems must not be empty")
        if not ints:
            raise ArgumentError("interactions must not be empty")
        self.systems = sys_
        self.interactions = ints
        self.ghosts = gsts
        vs = (virtual_systems,) if isinstance(virtual_systems, VirtualParticleSystem) else tuple(virtual_systems)
        for v in vs:
            if not isinstance(v, VirtualParticleSystem):
                raise ArgumentError("virtual_systems must be VirtualParticleSystems")
        self.virtual_systems = vs
        self.probes = (probes,) if isinstance(probes, ProbeParticleSystem) else tuple(probes)
        self.probe_interactions = ((probe_interactions,) if isinstance(probe_interactions, SystemInteraction)
                                   else tuple(probe_interactions))
        for p in self.probes:
            if not isinstance(p, ProbeParticleSystem):
                raise ArgumentError("probes must be ProbeParticleSystems")
        for si in self.probe_interactions:
            if not any(si.system_b is p for p in self.probes):
                raise ArgumentError("a probe interaction's system_b must be one of `probes`")
        T = sys_[0].dtype.type
        self.c = _scalar(T, max(ps.c for ps in sys_))
        self.h = _scalar(T, min(it.kernel.h for it in ints))
        self.gamma = _scalar(T, gamma)
        self._device = None


class RK4TimeIntegrator(LeapFrogTimeIntegrator):
    """src/TimeIntegration.jl:86-113: classical fourth-order Runge-Kutta, one
    neighbour grid per step, positions advanced once at the end."""

    kind = C.GC_INTEGRATOR_RK4
