"""XSPH velocity correction: XSPHPfn (src/PairwiseFunctors.jl:357-389) swept
by adjust_v! (src/Interaction.jl:309) in _xsph_correction!
(src/TimeIntegration.jl:421-436), between the full step and the position
update.

The reference has no XSPH tests.  The known answers below take particles
with no stage functor and no source term, so one LeapFrog step leaves v
unchanged until the correction: v_adjustment_i = sum over neighbours of
((-eps (v_i - v_j)) w) / (rho_i + rho_j) * m_j, then v += v_adjustment and
x += dt v.  A ghost system_b forwards `v_adjustment` to its source
(src/GhostParticles.jl:226-236), so the system_b-side write of a ghost pair
lands in the SOURCE's array at the GHOST's index; the ghost test places that
index on a particle that has no neighbour at all and checks that it moves.
"""
import math

import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
import parity
from gc_helpers import BACKENDS, make_backend


def _w(h, r):
    k = G.CubicSplineKernel(h, ndims=2)
    q = r / h
    a, b = max(0.0, 2.0 - q), max(0.0, 1.0 - q)
    return k.norm_coeff * (0.25 * a ** 3 - b ** 3)


def _step(be, lf, cfl):
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    s.step(1, cfl)
    s.pull()
    return s


def _by_id(ps, field):
    return np.asarray(getattr(ps, field))[np.argsort(ps.id)]


@pytest.mark.parametrize("be", BACKENDS)
def test_xsph_self_pair(be):
    h, eps, c, m = 0.1, 0.5, 10.0, 2.0
    ps = G.BasicParticleSystem("p", 2, 2, m, c)
    ps.x[:] = [[0.5, 0.5], [0.56, 0.53]]
    ps.v[:] = [[0.3, -0.1], [-0.2, 0.4]]
    ps.rho[:] = [1000.0, 990.0]
    x0, v0, rho = ps.x.copy(), ps.v.copy(), ps.rho.copy()
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), None, ps,
                             velocity_adjust_pairwise_fn=G.XSPHPfn(eps))
    lf = G.LeapFrogTimeIntegrator([ps], [si])
    _step(be, lf, 0.2)
    dt = 0.2 * h / c
    w = _w(h, np.linalg.norm(x0[0] - x0[1]))
    du = ((-eps * (v0[0] - v0[1])) * w) / (rho[0] + rho[1])
    adj = np.array([du * m, -du * m])
    np.testing.assert_allclose(_by_id(ps, "v_adjustment"), adj, rtol=1e-12)
    np.testing.assert_allclose(_by_id(ps, "v"), v0 + adj, rtol=1e-12)
    np.testing.assert_allclose(_by_id(ps, "x"), x0 + dt * (v0 + adj), rtol=1e-12)


@pytest.mark.parametrize("be", BACKENDS)
def test_xsph_coupled_writes_both_systems(be):
    h, eps, c = 0.1, 0.3, 10.0
    a = G.BasicParticleSystem("a", 1, 2, 2.0, c)
    b = G.BasicParticleSystem("b", 1, 2, 0.5, c)
    a.x[0], b.x[0] = [0.5, 0.5], [0.45, 0.58]
    a.v[0], b.v[0] = [0.1, 0.2], [-0.3, 0.05]
    a.rho[0], b.rho[0] = 1000.0, 500.0
    va, vb = a.v[0].copy(), b.v[0].copy()
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), None, a, b,
                             velocity_adjust_pairwise_fn=G.XSPHPfn(eps))
    lf = G.LeapFrogTimeIntegrator([a, b], [si])
    _step(be, lf, 0.2)
    w = _w(h, math.hypot(0.05, 0.08))
    du = ((-eps * (va - vb)) * w) / 1500.0
    np.testing.assert_allclose(a.v_adjustment[0], du * 0.5, rtol=1e-12)
    np.testing.assert_allclose(b.v_adjustment[0], -du * 2.0, rtol=1e-12)
    np.testing.assert_allclose(a.v[0], va + du * 0.5, rtol=1e-12)
    np.testing.assert_allclose(b.v[0], vb - du * 2.0, rtol=1e-12)


@pytest.mark.parametrize("be", BACKENDS)
def test_xsph_ghost_side_lands_at_the_ghost_index(be):
    h, eps, c, m = 0.1, 0.5, 10.0, 1.5
    ps = G.BasicParticleSystem("p", 2, 2, m, c)
    # B far from everything; A near the floor y = 0 (mirrored there).  The
    # sort puts B first (smaller x cell), so the ghost of A has index 1 and
    # its system_b-side term lands on B.
    ps.x[:] = [[0.9, 0.05], [0.1, 0.6]]
    ps.v[:] = [[0.3, -0.2], [0.0, 0.0]]
    ps.rho[:] = 1000.0
    ghost = G.GhostParticleSystem(ps, None)
    ge = G.GhostEntry(ghost, 0.2, ((0.0, 1.0), (0.0, 0.0)))
    kern = G.CubicSplineKernel(h, ndims=2)
    si = G.SystemInteraction(kern, None, ps, ghost, velocity_adjust_pairwise_fn=G.XSPHPfn(eps))
    lf = G.LeapFrogTimeIntegrator([ps], [si], ghosts=(ge,))
    _step(be, lf, 0.2)
    vA = np.array([0.3, -0.2])
    vg = np.array([0.3, 0.2])  # mirrored velocity of the ghost
    w = _w(h, 0.1)
    du = ((-eps * (vA - vg)) * w) / 2000.0
    adj = _by_id(ps, "v_adjustment")
    np.testing.assert_allclose(adj[0], du * m, rtol=1e-12)   # A: a-side
    np.testing.assert_allclose(adj[1], -du * m, rtol=1e-12)  # B: the ghost index
    np.testing.assert_allclose(_by_id(ps, "v")[1], -du * m, rtol=1e-12)


@pytest.mark.parametrize("be", BACKENDS)
def test_xsph_as_stage_functor_is_refused(be):
    ps = G.BasicParticleSystem("p", 2, 2, 1.0, 1.0)
    with pytest.raises(G.ArgumentError):
        G.SystemInteraction(G.CubicSplineKernel(0.1, ndims=2), G.XSPHPfn(0.5), ps)




def _run(lf, be, nsteps, cfl, prec=None, graphs=None):
    kw = {} if prec is None else dict(precision=prec)
    s = G.Session([lf], backend=make_backend(be), **kw)
    if graphs is not None:
        s.backend.set_graphs(graphs, 16)
    s.push()
    s.step(nsteps, cfl)
    s.pull()
    return s


def _dambreak_xsph(**kw):
    lf, meta = scenarios.dambreak_2d(nx=20, ny=40, dx=0.05, tank=(2.0, 2.5))
    for it in lf.interactions:
        it.vadjust_pfn = G.XSPHPfn(0.5)
    return lf, meta


def test_bubble3_oracle_xsph_moves_the_adjustment():
    lf, meta = scenarios.bubble("bubble3", dx=0.2)
    _run(lf, "oracle", 2, meta["cfl"])
    assert np.any(lf.systems[0].v_adjustment != 0.0) and np.any(lf.systems[1].v_adjustment != 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("integ", ["rk4", "leapfrog"])
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
def test_bubble3_xsph_parity(integ, nsteps, tol):
    cfl = 1.5 if integ == "rk4" else 0.2
    parity.run_and_compare(lambda: scenarios.bubble("bubble3", dx=0.1, integrator=integ, cfl=cfl), nsteps, cfl, tol)


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
def test_dambreak_xsph_with_dynamic_walls_parity(nsteps, tol):
    # XSPH against a DynamicBoundarySystem uses the wall's stored v and rho and
    # writes the wall's own v_adjustment, so the walls move
    _, meta = _dambreak_xsph()
    parity.run_and_compare(_dambreak_xsph, nsteps, meta["cfl"], tol)


@pytest.mark.gpu
def test_bubble3_xsph_fp32c():
    _, meta = scenarios.bubble("bubble3", dx=0.1)
    parity.run_and_compare(lambda: scenarios.bubble("bubble3", dx=0.1), 20, meta["cfl"], 1e-4,
                           precision=G.PRECISION_FP32_COMPENSATED)


@pytest.mark.gpu
def test_xsph_graph_steps_bit_identical():
    out = []
    for graphs in (False, True):
        lf, meta = scenarios.bubble("bubble3", dx=0.1)
        st = _run(lf, "cuda", 40, meta["cfl"], graphs=graphs).stats()
        out.append((lf, st))
    (le, _), (lg, st) = out
    assert st["graph_steps"] > 0
    for se, sg in zip(le.systems, lg.systems):
        for name, _ in se.particle_fields():
            assert np.array_equal(getattr(se, name), getattr(sg, name)), f"{se.name}.{name}"
