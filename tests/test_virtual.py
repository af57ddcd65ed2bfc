"""Virtual-particle boundaries: VirtualParticleSystem (src/Particles.jl:476-528),
InterpolateFieldFn (src/PairwiseFunctors.jl:392-428), VirtualNormUpdater and
PrescribedVelocityUpdater (src/StateUpdaters.jl:44-97) and the integrator's
handling of virtual systems (src/TimeIntegration.jl:364-419, 683).

The reference has no tests for these.  The known answers restate the
interpolation for one real/virtual pair (f_j += kw f_i, w_sum_j += kw with
kw = W(r) m_i/rho_i), the normalisation (f/w_sum, v·v_mult + prescribed_v,
zero where w_sum is zero) and the position update of a moving virtual
system; the device is then held to the oracle on the EP_ColumnCollapse2.jl
layout (four stages, no-slip bottom, free-slip left wall).
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


def _pair(pv=None, v_mult=(-1.0, 1.0)):
    h = 0.1
    real = G.StressParticleSystem("soil", 1, 2, 4, 2.0, 20.0)
    real.x[0] = [0.5, 0.5]
    real.v[0] = [0.3, -0.2]
    real.rho[0] = 1800.0
    real.stress[0] = [-10.0, -20.0, -15.0, 3.0]
    src = G.StressParticleSystem("wall", 2, 2, 4, 2.0, 20.0)
    src.x[:] = [[0.56, 0.45], [2.0, 2.0]]  # the second is out of reach: w_sum stays 0
    src.rho[:] = 1800.0
    src.v[:] = 7.0
    virt = G.VirtualParticleSystem(src, "wall_virt", 2, 2, 2.0, 20.0, zero_fields=("v", "rho", "stress"),
                                   prescribed_v=pv,
                                   state_updater=(G.VirtualNormUpdater(v_mult, "v", "rho", "stress"),))
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2),
                             G.InterpolateFieldFn("v", "rho", "stress"), real, virt)
    lf = G.LeapFrogTimeIntegrator([real], [si], virtual_systems=(virt,))
    return real, src, virt, si, lf, h


@pytest.mark.parametrize("be", BACKENDS)
def test_interpolate_and_normalise_pair(be):
    real, src, virt, si, lf, h = _pair(pv=(0.0, -0.5))
    s = G.Session([lf], backend=make_backend(be))
    # zero_fields act at the start of a step's stage loop; here the sweep runs alone
    src.v[:] = 0.0
    src.rho[:] = 0.0
    s.push()
    s.create_grid(si)
    s.sweep(si, 1)
    s.pull()
    kw = _w(h, math.hypot(0.06, 0.05)) * (2.0 / 1800.0)
    j = int(np.argmax(virt.w_sum))
    assert math.isclose(virt.w_sum[j], kw, rel_tol=1e-12) and virt.w_sum[1 - j] == 0.0
    np.testing.assert_allclose(src.v[j], kw * real.v[0], rtol=1e-12)
    assert math.isclose(src.rho[j], kw * 1800.0, rel_tol=1e-12)
    np.testing.assert_allclose(src.stress[j], kw * real.stress[0], rtol=1e-12)
    s.update_state(virt, 1, 0.0)
    s.pull()
    np.testing.assert_allclose(src.v[j], (kw * real.v[0] / kw) * np.array([-1.0, 1.0]) + [0.0, -0.5], rtol=1e-12)
    np.testing.assert_allclose(src.stress[j], kw * real.stress[0] / kw, rtol=1e-12)
    # w_sum = 0: every listed field is zero, v then gets prescribed_v
    assert src.rho[1 - j] == 0.0 and np.all(src.stress[1 - j] == 0.0)
    np.testing.assert_allclose(src.v[1 - j], [0.0, -0.5])


@pytest.mark.parametrize("be", BACKENDS)
def test_virtual_source_moves_with_prescribed_v_and_is_not_integrated(be):
    real, src, virt, si, lf, h = _pair(pv=(0.0, -0.5))
    real.source_v[:] = [0.0, -9.81]
    x0 = src.x.copy()
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    s.step(3, 0.2)
    s.pull()
    dt = 0.2 * h / 20.0
    xs = x0.copy()
    for _ in range(3):
        xs = xs + np.array([0.0, -0.5]) * dt
    order = np.argsort(src.id)
    np.testing.assert_allclose(src.x[order], xs, rtol=0, atol=1e-15)
    assert np.all(src.dvdt == 0.0)  # never integrated


def test_virtual_source_in_systems_is_refused():
    real, src, virt, si, lf, h = _pair()
    lf2 = G.LeapFrogTimeIntegrator([real, src], [si], virtual_systems=(virt,))
    with pytest.raises(G.ArgumentError):
        G.Session([lf2], backend=make_backend("oracle"))


def test_ep_column_virtual_layout():
    lf, meta = scenarios.ep_column_virtual()
    assert (meta["n_fluid"], meta["n_bottom"], meta["n_left"]) == (5000, 759, 150)
    assert len(lf.virtual_systems) == 2


def _run(lf, be, nsteps, cfl, prec=None, graphs=None):
    kw = {} if prec is None else dict(precision=prec)
    mode = parity.one_step_mode(lf, G.PRECISION_FP64 if prec is None else prec) if nsteps == 1 else parity.INPUTS
    s = G.Session([lf], backend=make_backend(be, track=mode if be == "oracle" else False), **kw)
    if graphs is not None:
        s.backend.set_graphs(graphs, 16)
    s.push()
    s.step(nsteps, cfl)
    s.pull()
    return s


def _systems(lf):
    return list(lf.systems) + [v.source for v in lf.virtual_systems]


def _cmp(lf_g, lf_c, sess_c, nsteps, tol, rate_tol=None):
    """The integrator's systems on the per-particle scale of tests/parity.py
    (after several steps: the state on its integrated scale).  The virtual
    systems' interpolated fields and w_sum (and the probes) are
    normalised weighted averages of the soil's fields, compared on each
    field's own scale."""
    if nsteps == 1:
        parity.compare_integrators(lf_g, lf_c, sess_c, tol, rate_tol)
    else:
        parity.compare_integrators(lf_g, lf_c, sess_c, tol, exact_ids=False, skip=parity.RATES)
    tol = tol["*"] if isinstance(tol, dict) else tol
    for vg, vc in zip(lf_g.virtual_systems, lf_c.virtual_systems):
        sg, sc = vg.source, vc.source
        ig, ic = np.argsort(sg.id), np.argsort(sc.id)
        for name, _ in sg.particle_fields():
            if name == "id":
                continue
            a = np.asarray(getattr(sg, name), dtype=float)[ig]
            b = np.asarray(getattr(sc, name), dtype=float)[ic]
            scale = max(np.abs(b).max(), 1e-300)
            err = np.abs(a - b).max() / scale
            assert err <= tol, f"{sg.name}.{name}: {err:.3e} > {tol}"
        scale = max(np.abs(vc.w_sum).max(), 1e-300)
        err = np.abs(vg.w_sum[ig] - vc.w_sum[ic]).max() / scale
        assert err <= tol, f"{vg.name}.w_sum: {err:.3e} > {tol}"


def test_ep_column_virtual_oracle_fills_the_walls():
    lf, meta = scenarios.ep_column_virtual(dx=0.004)
    _run(lf, "oracle", 3, meta["cfl"])
    b, l = lf.virtual_systems
    assert (b.w_sum > 0).sum() > 0 and (l.w_sum > 0).sum() > 0
    assert np.any(l.source.stress != 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
@pytest.mark.parametrize("bottom_v", [None, (0.0, -0.05)])
def test_ep_column_virtual_parity(nsteps, tol, bottom_v):
    lf_g, meta = scenarios.ep_column_virtual(bottom_v=bottom_v, geostatic=True)
    lf_c, _ = scenarios.ep_column_virtual(bottom_v=bottom_v, geostatic=True)
    _run(lf_g, "cuda", nsteps, meta["cfl"])
    c = _run(lf_c, "oracle", nsteps, meta["cfl"])
    _cmp(lf_g, lf_c, c, nsteps, tol)


@pytest.mark.gpu
def test_ep_column_virtual_fp32c():
    lf_g, meta = scenarios.ep_column_virtual(geostatic=True)
    lf_c, _ = scenarios.ep_column_virtual(geostatic=True)
    _run(lf_g, "cuda", 20, meta["cfl"], prec=G.PRECISION_FP32_COMPENSATED)
    c = _run(lf_c, "oracle", 20, meta["cfl"])
    _cmp(lf_g, lf_c, c, 20, {"*": 1e-3, "strain": 1e-2, "strain_p": 1e-2})


@pytest.mark.gpu
@pytest.mark.parametrize("bottom_v", [None, (0.0, -0.05)])
def test_ep_column_virtual_graph_steps_bit_identical(bottom_v):
    out = []
    for graphs in (False, True):
        lf, meta = scenarios.ep_column_virtual(bottom_v=bottom_v)
        st = _run(lf, "cuda", 40, meta["cfl"], graphs=graphs).stats()
        out.append((lf, st))
    (le, _), (lg, st) = out
    assert st["graph_steps"] > 0
    for se, sg in zip(_systems(le), _systems(lg)):
        for name, _ in se.particle_fields():
            assert np.array_equal(getattr(se, name), getattr(sg, name)), f"{se.name}.{name}"
    for ve, vg in zip(le.virtual_systems, lg.virtual_systems):
        assert np.array_equal(ve.w_sum, vg.w_sum)
