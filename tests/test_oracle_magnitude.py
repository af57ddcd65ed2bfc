"""The oracle's magnitude shadows, the per-particle scale of the parity
tests (tests/parity.py): keeping them changes no result, every shadow
bounds its field, and a one-pair case gives the pair term's magnitude."""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
from gc_helpers import make_backend
import parity

CASES = {
    "dambreak_2d": (scenarios.dambreak_2d, dict(nx=12, ny=20, dx=0.05, tank=(1.5, 1.5))),
    "column": (scenarios.column_collapse, dict(nx=24, ny=12, dx=0.005)),
    "dambreak_lj_2d": (scenarios.dambreak_lj_2d, dict(nfx=10, nfy=10, nbx=30, nby=16)),
    "granular": (scenarios.granular_column, dict(nfx=24, nfy=12, dx=0.005)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_tracking_changes_nothing_and_bounds_fields(case):
    builder, kw = CASES[case]
    runs = []
    for track in (False, True):
        lf, meta = builder(**kw)
        s = G.Session([lf], backend=make_backend("oracle", track=track, threads=2))
        s.push()
        s.step(3, meta["cfl"])
        s.pull()
        runs.append((lf, s))
    (l0, _), (l1, s1) = runs
    for a, b in zip(l0.systems, l1.systems):
        for name, _ in a.particle_fields():
            assert np.array_equal(getattr(a, name), getattr(b, name)), f"{a.name}.{name}"
    mags = parity.oracle_magnitudes(s1, l1)
    for ps in l1.systems:
        for name, m in mags[id(ps)].items():
            if name in parity.RATES:
                assert (m >= np.abs(getattr(ps, name))).all(), f"{ps.name}.{name}"
            else:
                assert (m >= 0.0).all(), f"{ps.name}.{name}"
    # a system compared with itself has no error on any scale
    parity.compare_integrators(l1, l1, s1, 0.0)


def test_one_pair_magnitude_is_the_term():
    """Two fluid particles: dv/dt = g + t and -t for the pair term t; the
    shadow holds |g| + |t| on both."""
    ps = G.FluidParticleSystem("f", 2, 2, 1.0, 10.0, source_v=[0.0, -9.81])
    ps.x[:] = [[0.0, 0.0], [0.07, 0.02]]
    ps.rho[:] = [1000.0, 1001.0]
    ps.p[:] = [500.0, 800.0]
    k = G.CubicSplineKernel(0.05, ndims=2)
    si = G.SystemInteraction(k, G.FluidPfn(0.1, 0.0, 0.05), ps)
    lf = G.LeapFrogTimeIntegrator([ps], [si])
    s = G.Session([lf], backend=make_backend("oracle", track=True))
    s.push()
    s.step(1, 0.1)
    s.pull()
    mag = parity.oracle_magnitudes(s, lf)[id(ps)]
    g = np.array([0.0, -9.81])
    t0 = ps.dvdt[0] - g
    t1 = ps.dvdt[1] - g
    assert np.allclose(t0, -t1, rtol=1e-14, atol=0)
    assert np.allclose(mag["dvdt"][0], np.abs(g) + np.abs(t0), rtol=1e-14, atol=0)
    assert np.allclose(mag["dvdt"][1], np.abs(g) + np.abs(t1), rtol=1e-14, atol=0)
