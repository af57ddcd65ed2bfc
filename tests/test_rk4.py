"""RK4TimeIntegrator (src/TimeIntegration.jl:86-113, 712-838).

The reference has no RK4 tests; the known answers here follow from the
algorithm: a particle with no neighbours and a constant source term gets
k1 = k2 = k3 = k4 = source, so v = v0 + dt·acc with acc accumulated in the
reference's order and rounding, and x = x0 + dt·v with the new velocity.
The device path is then checked against the oracle's restatement on the
three scenario kinds on the per-particle scale (FP64 one step within
1e-10, 20 steps within 1e-8),
and captured RK4 steps against exact ones bit for bit.
"""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
from gc_helpers import BACKENDS, basic, kernel, make_backend
import parity


def _rk4(lf):
    return G.RK4TimeIntegrator(lf.systems, lf.interactions, ghosts=lf.ghosts, gamma=lf.gamma)


@pytest.mark.parametrize("be", BACKENDS)
def test_rk4_free_particle(be):
    ps = basic(n=1, c=10.0, source_v=[0.0, -1.0])
    ps.x[0] = [0.5, 0.5]
    ps.v[0] = [0.25, 0.0]
    ps.rho[:] = 1000.0
    lf = G.RK4TimeIntegrator([ps], [G.SystemInteraction(kernel(), None, ps)])
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    s.step(3, 0.5)
    s.pull()
    dt = 0.5 * 0.1 / 10.0
    x = np.array([0.5, 0.5])
    v = np.array([0.25, 0.0])
    g = np.array([0.0, -1.0])
    for _ in range(3):
        acc = np.zeros(2)
        for w in (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0):
            acc = acc + w * g
        v = v + dt * acc
        x = x + dt * v
    assert np.array_equal(ps.v[0], v)
    assert np.array_equal(ps.x[0], x)
    assert np.array_equal(ps.dvdt[0], g)
    assert np.all(ps.rho == 1000.0)


CASES = {
    "dambreak_2d": (scenarios.dambreak_2d, dict(nx=20, ny=40, dx=0.05, tank=(2.0, 2.5))),
    "dambreak_3d": (scenarios.dambreak_3d, dict(nx=8, ny=6, nz=12, dx=0.05, tank=(1.0, 0.5, 1.0))),
    "column": (scenarios.column_collapse, dict(nx=40, ny=20, dx=0.005)),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
def test_rk4_parity(case, nsteps, tol):
    """Per-particle scale of tests/parity.py; after 20 steps the state on
    its integrated scale, then one further step from the device's state at
    1e-10."""
    builder, kw = CASES[case]
    lf_g, meta = builder(**kw)
    lf_c, _ = builder(**kw)
    lf_g, lf_c = _rk4(lf_g), _rk4(lf_c)
    g = G.Session([lf_g], backend=make_backend("cuda"))
    # an RK4 step's later right-hand sides start from states that already
    # carry the earlier ones' summation order: shadows over the inputs
    c = G.Session([lf_c], backend=make_backend("oracle", track=parity.INPUTS))
    for s in (g, c):
        s.push()
        s.step(nsteps, meta["cfl"])
        s.pull()
    if nsteps == 1:
        parity.compare_integrators(lf_g, lf_c, c, tol)
    else:
        parity.compare_integrators(lf_g, lf_c, c, tol, exact_ids=False, skip=parity.RATES)
        parity.one_step_from_device_state(lf_g, lf_c, g, c, meta["cfl"], 1e-10, mode=parity.INPUTS)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [G.PRECISION_FP64, G.PRECISION_FP32_COMPENSATED])
def test_rk4_graph_steps_bit_identical(prec):
    builder, kw = CASES["column"]
    out = []
    for graphs in (False, True):
        lf, meta = builder(**kw)
        lf = _rk4(lf)
        s = G.Session([lf], backend=make_backend("cuda"), precision=prec)
        s.backend.set_graphs(graphs, 16)
        s.push()
        s.step(40, meta["cfl"])
        s.pull()
        out.append((lf, s.stats()))
    (le, _), (lg, st) = out
    assert st["graph_steps"] > 0
    for se, sg in zip(le.systems, lg.systems):
        for name, _ in se.particle_fields():
            assert np.array_equal(getattr(se, name), getattr(sg, name)), f"{se.name}.{name}"
