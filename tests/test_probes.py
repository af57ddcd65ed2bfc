"""Probes at save cadence: ProbeParticleSystem (src/ProbeParticles.jl:23-143),
NeighborCountFn and InterpolateFieldFn into probes
(src/PairwiseFunctors.jl:436-460), _measure_probes! and
_advance_probe_positions! (src/TimeIntegration.jl:440-502).

Restates test/test_probe_particles.jl:269-450 and :547-570 (the
measurements the reference reads back from its HDF5 snapshot are read here
after `Session.measure_probes`, which is the save-time measurement without
the file), on the oracle and on the device, and then holds the device to
the oracle on a probe grid over the EP column.
"""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
from gc_helpers import BACKENDS, make_backend


def _line_fluid(n=8, dx=0.1, rho0=1000.0, c=100.0):
    h = 1.2 * dx
    ps = G.FluidParticleSystem("fluid", n, 2, rho0 * dx * dx, c, state_updater=G.TaitEOSUpdater(rho0))
    ps.x[:, 0] = np.arange(n) * dx
    ps.rho[:] = rho0
    return ps, G.CubicSplineKernel(h, ndims=2), h


def _session(be, ps, kernel, h, probe, pfn):
    si_self = G.SystemInteraction(kernel, G.FluidPfn(0.1, 0.0, h), ps)
    si_probe = G.SystemInteraction(kernel, pfn, ps, probe)
    lf = G.LeapFrogTimeIntegrator([ps], [si_self], probes=(probe,), probe_interactions=(si_probe,))
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    return lf, s


@pytest.mark.parametrize("be", BACKENDS)
def test_neighbor_counts_on_a_line(be):
    ps, kernel, h = _line_fluid(n=8)
    probe = G.ProbeParticleSystem("probe", ps, extras={"nbr": np.zeros(8, dtype=int)})
    lf, s = _session(be, ps, kernel, h, probe, G.NeighborCountFn("nbr"))
    s.step(1, 0.1)
    s.measure_probes()
    nbr = probe.nbr
    assert nbr[0] < nbr[3] and nbr[7] < nbr[3]
    assert nbr.max() in (nbr[3], nbr[4])


@pytest.mark.parametrize("be", BACKENDS)
def test_neighbor_counts_symmetric(be):
    ps, kernel, h = _line_fluid(n=5)
    probe = G.ProbeParticleSystem("probe", ps, extras={"nbr": np.zeros(5, dtype=int)})
    lf, s = _session(be, ps, kernel, h, probe, G.NeighborCountFn("nbr"))
    s.step(1, 0.1)
    s.measure_probes()
    nbr = probe.nbr
    assert nbr[0] == nbr[4] and nbr[1] == nbr[3] and nbr[2] >= nbr[1]


@pytest.mark.parametrize("be", BACKENDS)
def test_constant_field_recovered_at_probes(be):
    ps, kernel, h = _line_fluid(n=8)
    ps.v[:] = [1.0, 0.5]
    probe = G.ProbeParticleSystem("probe", [[0.35, 0.0], [0.45, 0.0], [0.55, 0.0]],
                                  extras={"v": np.zeros((3, 2))},
                                  state_updater=G.VirtualNormUpdater((1.0, 1.0), "v"))
    lf, s = _session(be, ps, kernel, h, probe, G.InterpolateFieldFn("v"))
    s.step(1, 0.1)
    s.measure_probes()
    assert np.all(np.abs(probe.v[:, 0] - 1.0) < 0.01) and np.all(np.abs(probe.v[:, 1] - 0.5) < 0.01)


@pytest.mark.parametrize("be", BACKENDS)
def test_scalar_field_recovered_at_probes(be):
    ps, kernel, h = _line_fluid(n=6)
    ps.rho[:] = 1234.0
    probe = G.ProbeParticleSystem("probe", [[0.2, 0.0], [0.3, 0.0]], extras={"rho": np.zeros(2)},
                                  state_updater=G.VirtualNormUpdater((1.0, 1.0), "rho"))
    lf, s = _session(be, ps, kernel, h, probe, G.InterpolateFieldFn("rho"))
    s.step(1, 0.1)
    s.measure_probes()
    assert np.all(np.abs(probe.rho - 1234.0) < 10.0)


@pytest.mark.parametrize("be", BACKENDS)
def test_prescribed_v_advances_probes_every_step(be):
    ps, kernel, h = _line_fluid(n=4)
    probe = G.ProbeParticleSystem("probe", [[0.0, 0.0]], extras={"cnt": np.zeros(1, dtype=int)},
                                  prescribed_v=(1.0, 0.0))
    lf, s = _session(be, ps, kernel, h, probe, G.NeighborCountFn("cnt"))
    dt = 0.1 * h / lf.c
    s.step(3, 0.1)
    s.pull()
    x = 0.0
    for _ in range(3):
        x = x + 1.0 * dt
    np.testing.assert_allclose(probe.x[0], [x, 0.0], rtol=0, atol=1e-12)


@pytest.mark.parametrize("be", BACKENDS)
def test_mirrored_probes_are_in_id_order(be):
    ps, kernel, h = _line_fluid(n=4)
    ps.v[:] = [0.5, 0.0]
    probe = G.ProbeParticleSystem("probe", ps, extras={"cnt": np.zeros(4, dtype=int)})
    lf, s = _session(be, ps, kernel, h, probe, G.NeighborCountFn("cnt"))
    s.step(5, 0.1)
    s.measure_probes()
    s.pull()
    assert np.array_equal(probe.id, np.arange(1, 5))
    np.testing.assert_array_equal(probe.x, ps.x[np.argsort(ps.id)])


def _crossing(be):
    ps = G.FluidParticleSystem("fluid", 2, 2, 1000.0, 1.0, state_updater=G.TaitEOSUpdater(1000.0))
    ps.x[:] = [[0.0, 0.0], [1.0, 0.0]]
    ps.rho[:] = 1000.0
    ps.v[:] = [[20.0, 0.0], [-20.0, 0.0]]
    kernel = G.CubicSplineKernel(0.25, ndims=2)
    probe = G.ProbeParticleSystem("probe", ps, extras={"cnt": np.zeros(2, dtype=int)})
    si_self = G.SystemInteraction(kernel, None, ps)
    si_probe = G.SystemInteraction(kernel, G.NeighborCountFn("cnt"), ps, probe)
    lf = G.LeapFrogTimeIntegrator([ps], [si_self], probes=(probe,), probe_interactions=(si_probe,))
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    return s, probe


@pytest.mark.parametrize("be", BACKENDS)
def test_measurement_uses_freshly_sorted_sources(be):
    s, probe = _crossing(be)
    s.step(1, 1.0)
    s.measure_probes()
    assert list(probe.cnt) == [1, 1]


@pytest.mark.parametrize("be", BACKENDS)
def test_mirrored_probes_follow_source_identity(be):
    s, probe = _crossing(be)
    s.step(2, 1.0)
    s.measure_probes()
    np.testing.assert_allclose(probe.x[:, 0], [10.0, -9.0])


def _column_probes(stress_probe=True):
    lf, meta = scenarios.ep_column_virtual(dx=0.004, geostatic=True)
    fluid = lf.systems[0]
    kernel = lf.interactions[0].kernel
    gx, gy = np.meshgrid(np.linspace(0.01, 0.19, 10), np.linspace(0.005, 0.095, 6), indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel()], axis=1)
    grid = G.ProbeParticleSystem("grid", pts, extras={"stress": np.zeros((len(pts), 4)), "rho": np.zeros(len(pts))},
                                 state_updater=G.VirtualNormUpdater((1.0, 1.0), "stress", "rho"),
                                 prescribed_v=(0.0, -0.01))
    mirror = G.ProbeParticleSystem("mirror", fluid, extras={"nbr": np.zeros(fluid.n, dtype=int)})
    pints = (G.SystemInteraction(kernel, G.InterpolateFieldFn("stress", "rho"), fluid, grid),
             G.SystemInteraction(kernel, G.NeighborCountFn("nbr"), fluid, mirror))
    lf2 = G.LeapFrogTimeIntegrator(lf.systems, lf.interactions, virtual_systems=lf.virtual_systems,
                                   probes=(grid, mirror), probe_interactions=pints)
    return lf2, meta, grid, mirror


@pytest.mark.gpu
def test_probe_parity_on_ep_column():
    out = []
    for be in ("cuda", "oracle"):
        lf, meta, grid, mirror = _column_probes()
        s = G.Session([lf], backend=make_backend(be))
        s.push()
        for _ in range(3):
            s.step(5, meta["cfl"])
            s.measure_probes()
        s.pull()
        out.append((grid, mirror))
    (gg, mg), (gc, mc) = out
    assert np.array_equal(mg.nbr, mc.nbr) and np.array_equal(mg.id, mc.id)
    np.testing.assert_allclose(mg.x, mc.x, rtol=0, atol=1e-12)
    np.testing.assert_allclose(gg.x, gc.x, rtol=0, atol=1e-15)
    for name in ("stress", "rho"):
        a, b = getattr(gg, name), getattr(gc, name)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), name
    assert np.abs(gg.w_sum - gc.w_sum).max() <= 1e-10 * np.abs(gc.w_sum).max()
