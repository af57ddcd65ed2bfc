"""Two-sided FluidPfn between two fluid systems (multiphase) and the
bubble scenarios (bubble.jl, bubble2.jl, bubble3.jl with its XSPH).

The reference has no tests for this functor.  The known answers restate
src/PairwiseFunctors.jl:173-190 with src/PairwisePhysics.jl:29-34 (artificial
viscosity with both sound speeds), :58-64 (pressure coefficient, sigma 1 and
2), :99-105 (continuity coefficient), :238-243 (density diffusion) and
:286-288 (artificial surface tension) for one pair, and check both systems'
rates.  The device path is then held to the oracle on the bubble layouts:
eight ghost planes (walls and diagonal corners), RK4 and LeapFrog, sigma 1
and 2, with and without surface tension.
"""
import math

import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
import parity
from gc_helpers import BACKENDS, make_backend, session


def _pair_case(sigma, eps, delta):
    h = 0.1
    a = G.FluidParticleSystem("a", 1, 2, 2.5, 30.0)
    b = G.FluidParticleSystem("b", 1, 2, 0.75, 45.0)
    a.x[0], b.x[0] = [0.0, 0.0], [0.07, 0.04]
    a.v[0], b.v[0] = [0.3, -0.1], [-0.2, 0.25]
    a.rho[0], b.rho[0] = 1010.0, 480.0
    a.p[0], b.p[0] = 1500.0, -200.0
    pfn = G.FluidPfn(0.05, 0.02, h, sigma=sigma, delta=delta, epsilon=eps)
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), pfn, a, b)
    return a, b, si, h


def _expected(a, b, h, sigma, eps, delta, alpha=0.05, beta=0.02):
    k = G.CubicSplineKernel(h, ndims=2)
    dx = a.x[0] - b.x[0]
    rr = dx[0] * dx[0] + dx[1] * dx[1]
    r = math.sqrt(rr)
    q = r / h
    t2, t1 = max(0.0, 2 - q), max(0.0, 1 - q)
    gx = k.norm_coeff * (-3.0 * (0.25 * t2 * t2 - t1 * t1)) / (r * h) * dx
    dv = a.v[0] - b.v[0]
    ri, rj, pi_, pj = a.rho[0], b.rho[0], a.p[0], b.p[0]
    vr = min(dx[0] * dv[0] + dx[1] * dv[1], 0.0)
    muv = h * vr / (rr + h * h * 0.01)
    mc = 0.5 * (a.c + b.c)
    piv = (beta * muv - alpha * mc) * muv / (0.5 * ri * rj)
    if sigma == 1:
        dh = -(pi_ + pj) / (ri * rj)
    else:
        dh = -(pi_ / (ri * ri) + pj / (rj * rj))
    ast = 0.0 if eps is None else eps * (-(abs(pi_) + abs(pj)) / (ri * rj))
    tmp = (dh + ast - piv) * gx
    dr = dv[0] * gx[0] + dv[1] * gx[1]
    psi = 0.0
    if delta is not None:
        psi = 2.0 * delta * (0.5 * (a.c + b.c)) * h * (ri - rj) * (dx[0] * gx[0] + dx[1] * gx[1]) / rr
    ci, cj = (ri / rj, rj / ri) if sigma == 1 else (1.0, 1.0)
    return (b.mass * tmp, -a.mass * tmp,
            b.mass * (dr * ci + psi / rj), a.mass * (dr * cj - psi / ri))


@pytest.mark.parametrize("be", BACKENDS)
@pytest.mark.parametrize("sigma,eps,delta", [(2, None, None), (1, None, None), (2, 0.1, 0.1), (1, 0.1, None)])
def test_two_sided_fluid_pair(be, sigma, eps, delta):
    a, b, si, h = _pair_case(sigma, eps, delta)
    lf, s = session(be, [a, b], [si])
    s.create_grid(si)
    s.sweep(si, 1)
    s.pull()
    dva, dvb, dra, drb = _expected(a, b, h, sigma, eps, delta)
    np.testing.assert_allclose(a.dvdt[0], dva, rtol=1e-12)
    np.testing.assert_allclose(b.dvdt[0], dvb, rtol=1e-12)
    assert math.isclose(a.drhodt[0], dra, rel_tol=1e-12)
    assert math.isclose(b.drhodt[0], drb, rel_tol=1e-12)
    # momentum exchanged between the phases sums to zero
    np.testing.assert_allclose(a.mass * a.dvdt[0] + b.mass * b.dvdt[0], 0.0, atol=1e-12 * np.abs(a.mass * dva).max())


@pytest.mark.parametrize("be", BACKENDS)
def test_fluid_against_stress_system_stays_one_sided(be):
    h = 0.1
    a = G.FluidParticleSystem("a", 1, 2, 2.5, 30.0)
    b = G.StressParticleSystem("b", 1, 2, 3, 0.75, 45.0)
    a.x[0], b.x[0] = [0.0, 0.0], [0.07, 0.04]
    a.rho[0], b.rho[0] = 1000.0, 1000.0
    a.p[0], b.p[0] = 10.0, 20.0
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.FluidPfn(0.05, 0.0, h), a, b)
    lf, s = session(be, [a, b], [si])
    s.create_grid(si)
    s.sweep(si, 1)
    s.pull()
    assert np.any(a.dvdt[0] != 0.0)
    assert np.all(b.dvdt[0] == 0.0) and b.drhodt[0] == 0.0


@pytest.mark.parametrize("variant", list(scenarios.BUBBLE_VARIANTS))
def test_bubble_layout(variant):
    lf, meta = scenarios.bubble(variant, dx=0.2)
    fx, fy = lf.systems
    assert fx.n + fy.n == 30 * 50 and fy.n > 0
    assert np.all(fy.x[:, 0] ** 2 + fy.x[:, 1] ** 2 < 1.0)
    assert len(lf.ghosts[0].normals) == 8
    # hydrostatic: density falls with height in each phase
    for ps in (fx, fy):
        order = np.argsort(ps.x[:, 1])
        assert np.all(np.diff(ps.rho[order]) <= 1e-9)


def _run(lf, be, nsteps, cfl, prec=None, graphs=None):
    kw = {} if prec is None else dict(precision=prec)
    s = G.Session([lf], backend=make_backend(be), **kw)
    if graphs is not None:
        s.backend.set_graphs(graphs, 16)
    s.push()
    s.step(nsteps, cfl)
    s.pull()
    return s




def test_bubble_oracle_runs_and_conserves_mass():
    lf, meta = scenarios.bubble("bubble3", dx=0.2)
    _run(lf, "oracle", 3, meta["cfl"])
    for ps in lf.systems:
        assert np.all(np.isfinite(ps.x)) and np.all(np.isfinite(ps.rho))
    assert np.any(lf.systems[1].dvdt != 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", list(scenarios.BUBBLE_VARIANTS))
@pytest.mark.parametrize("integ", ["rk4", "leapfrog"])
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
def test_bubble_parity_fp64(variant, integ, nsteps, tol):
    # the scripts' Courant number 1.5 is an RK4 one; LeapFrog needs a smaller step
    cfl = 1.5 if integ == "rk4" else 0.2
    parity.run_and_compare(lambda: scenarios.bubble(variant, dx=0.1, integrator=integ, cfl=cfl), nsteps, cfl, tol)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["bubble", "bubble3"])
def test_bubble_parity_fp32c(variant):
    _, meta = scenarios.bubble(variant, dx=0.1)
    parity.run_and_compare(lambda: scenarios.bubble(variant, dx=0.1), 20, meta["cfl"], 1e-4,
                           precision=G.PRECISION_FP32_COMPENSATED)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [G.PRECISION_FP64, G.PRECISION_FP32_COMPENSATED])
def test_bubble_graph_steps_bit_identical(prec):
    out = []
    for graphs in (False, True):
        lf, meta = scenarios.bubble("bubble", dx=0.1)
        st = _run(lf, "cuda", 40, meta["cfl"], prec=prec, graphs=graphs).stats()
        out.append((lf, st))
    (le, _), (lg, st) = out
    assert st["graph_steps"] > 0
    for se, sg in zip(le.systems, lg.systems):
        for name, _ in se.particle_fields():
            assert np.array_equal(getattr(se, name), getattr(sg, name)), f"{se.name}.{name}"


# ------------------------------------------------------------ FluidSolidPfn
# src/PairwiseFunctors.jl:463-519: FluidPfn's two-sided form with the
# fluid's (system_a's) pressure on both sides and no surface tension.

def _fs_expected(a, b, h, sigma, delta, alpha=0.05, beta=0.02):
    k = G.CubicSplineKernel(h, ndims=2)
    dx = a.x[0] - b.x[0]
    rr = dx[0] * dx[0] + dx[1] * dx[1]
    r = math.sqrt(rr)
    q = r / h
    t2, t1 = max(0.0, 2 - q), max(0.0, 1 - q)
    gx = k.norm_coeff * (-3.0 * (0.25 * t2 * t2 - t1 * t1)) / (r * h) * dx
    dv = a.v[0] - b.v[0]
    ri, rj, pf = a.rho[0], b.rho[0], a.p[0]
    vr = min(dx[0] * dv[0] + dx[1] * dv[1], 0.0)
    muv = h * vr / (rr + h * h * 0.01)
    piv = (beta * muv - alpha * 0.5 * (a.c + b.c)) * muv / (0.5 * ri * rj)
    dh = -(pf + pf) / (ri * rj) if sigma == 1 else -(pf / (ri * ri) + pf / (rj * rj))
    tmp = (dh - piv) * gx
    dr = dv[0] * gx[0] + dv[1] * gx[1]
    psi = 0.0
    if delta is not None:
        psi = 2.0 * delta * (0.5 * (a.c + b.c)) * h * (ri - rj) * (dx[0] * gx[0] + dx[1] * gx[1]) / rr
    ci, cj = (ri / rj, rj / ri) if sigma == 1 else (1.0, 1.0)
    return (b.mass * tmp, -a.mass * tmp, b.mass * (dr * ci + psi / rj), a.mass * (dr * cj - psi / ri))


@pytest.mark.parametrize("be", BACKENDS)
@pytest.mark.parametrize("sigma,delta", [(2, None), (1, None), (2, 0.1)])
def test_fluid_solid_pair(be, sigma, delta):
    h = 0.1
    a = G.FluidParticleSystem("water", 1, 2, 2.5, 30.0)
    b = G.ElastoPlasticParticleSystem("wall", 1, 2, 4, 6.0, 480.0)
    a.x[0], b.x[0] = [0.0, 0.0], [0.07, 0.04]
    a.v[0], b.v[0] = [0.3, -0.1], [-0.02, 0.01]
    a.rho[0], b.rho[0] = 1010.0, 2400.0
    a.p[0], b.p[0] = 1500.0, -9.0e5  # the wall's own pressure plays no part
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.FluidSolidPfn(0.05, 0.02, h, sigma=sigma, delta=delta),
                             a, b)
    lf, s = session(be, [a, b], [si])
    s.create_grid(si)
    s.sweep(si, 1)
    s.pull()
    dva, dvb, dra, drb = _fs_expected(a, b, h, sigma, delta)
    np.testing.assert_allclose(a.dvdt[0], dva, rtol=1e-12)
    np.testing.assert_allclose(b.dvdt[0], dvb, rtol=1e-12)
    assert math.isclose(a.drhodt[0], dra, rel_tol=1e-12)
    assert math.isclose(b.drhodt[0], drb, rel_tol=1e-12)


@pytest.mark.parametrize("be", BACKENDS)
def test_fluid_solid_needs_a_real_system_b(be):
    h = 0.1
    a = G.FluidParticleSystem("water", 1, 2, 2.5, 30.0)
    w = G.BasicParticleSystem("w", 1, 2, 1.0, 30.0)
    dyn = G.DynamicBoundarySystem(w, (0.0, 1.0), (0.0, 0.0), 3.0)
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.FluidSolidPfn(0.05, 0.0, h), a, dyn)
    with pytest.raises(Exception):
        session(be, [a, w], [si])


def test_dambreak_wall_layout():
    lf, meta = scenarios.dambreak_wall()
    assert [p.n for p in lf.systems] == [2500, 60, 468, 240, 240, 468]


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
@pytest.mark.parametrize("x_wall", [60.0, 25.0])
def test_dambreak_wall_parity(nsteps, tol, x_wall):
    _, meta = scenarios.dambreak_wall(x_wall=x_wall)
    parity.run_and_compare(lambda: scenarios.dambreak_wall(x_wall=x_wall), nsteps, meta["cfl"], tol)


@pytest.mark.gpu
def test_dambreak_wall_fp32c():
    _, meta = scenarios.dambreak_wall(x_wall=25.0)
    parity.run_and_compare(lambda: scenarios.dambreak_wall(x_wall=25.0), 20, meta["cfl"],
                           {"*": 1e-4, "strain": 1e-2, "strain_p": 1e-2}, precision=G.PRECISION_FP32_COMPENSATED)
