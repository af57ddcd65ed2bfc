"""Trapdoor.jl: InterpolateFieldFn with a ghost system as system_a
(`ghost_bottom = SystemInteraction(kernel, (interp_rho, nothing, interp_str,
nothing), walls_ghost, bottom_virt)`), the (real, virtual) method of
src/PairwiseFunctors.jl:424-428 reading a GhostParticleSystem's own arrays
(src/GhostParticles.jl:174-236: x, v, rho and the copied extras; mass from
the source), and the whole Trapdoor.jl layout: EP soil with four stages,
free-slip wall ghosts copying Householder-reflected stress at stage 3, a
static bottom and a trapdoor as virtual systems sharing the stage
updaters, and stress probes over the trapdoor.

The known answer restates one ghost/virtual pair: the ghost of a particle
at (0.05, 0.5) behind the wall x = 0 sits at (-0.05, 0.5) with v_x negated
and σ_xy negated (the copier), and a virtual particle receives kw·f_ghost
with kw = W(r)·m/ρ_ghost.  The device is then held to the oracle on a
reduced trapdoor in both of the script's integrators (settling with damping
Γ, and the moving trapdoor).
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


def _ghost_pair():
    h = 0.1
    real = G.StressParticleSystem("soil", 1, 2, 4, 2.0, 20.0)
    real.x[0] = [0.05, 0.5]
    real.v[0] = [0.3, -0.2]
    real.rho[0] = 1800.0
    real.stress[0] = [-10.0, -20.0, -15.0, 3.0]
    ghost = G.GhostParticleSystem(real, G.GhostCopier(("stress", G.HouseholderReflect())))
    ge = G.GhostEntry(ghost, 3.0 * h, ((1.0, 0.0), (0.0, 0.0)))
    src = G.StressParticleSystem("wall", 2, 2, 4, 2.0, 20.0)
    src.x[:] = [[-0.08, 0.45], [-2.0, 2.0]]  # the second is out of reach
    virt = G.VirtualParticleSystem(src, "wall_virt", 2, 2, 2.0, 20.0, zero_fields=("v", "rho", "stress"),
                                   state_updater=(G.VirtualNormUpdater((1.0, 1.0), "v", "rho", "stress"),))
    si = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.InterpolateFieldFn("v", "rho", "stress"),
                             ghost, virt)
    lf = G.LeapFrogTimeIntegrator([real], [si], ghosts=(ge,), virtual_systems=(virt,))
    return real, ghost, ge, src, virt, si, lf, h


@pytest.mark.parametrize("be", BACKENDS)
def test_interpolate_from_ghosts_pair(be):
    real, ghost, ge, src, virt, si, lf, h = _ghost_pair()
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    s.generate_ghosts(ge)
    s.update_ghost_kinematics(ge)
    s.update_ghost(ge, 1)
    s.create_grid(si)
    s.sweep(si, 1)
    s.pull()
    s.pull_ghost(ge)
    assert ghost.n == 1
    np.testing.assert_allclose(ghost.x[0], [-0.05, 0.5], rtol=0, atol=1e-15)
    np.testing.assert_allclose(ghost.v[0], [-0.3, -0.2], rtol=0, atol=1e-15)
    np.testing.assert_allclose(ghost.stress[0], [-10.0, -20.0, -15.0, -3.0], rtol=0, atol=1e-12)
    kw = _w(h, math.hypot(0.03, 0.05)) * (2.0 / 1800.0)
    j = int(np.argmax(virt.w_sum))
    assert math.isclose(virt.w_sum[j], kw, rel_tol=1e-12) and virt.w_sum[1 - j] == 0.0
    np.testing.assert_allclose(src.v[j], kw * np.array([-0.3, -0.2]), rtol=1e-12)
    assert math.isclose(src.rho[j], kw * 1800.0, rel_tol=1e-12)
    np.testing.assert_allclose(src.stress[j], kw * np.array([-10.0, -20.0, -15.0, -3.0]), rtol=1e-12)
    assert np.all(src.v[1 - j] == 0.0) and src.rho[1 - j] == 0.0


@pytest.mark.parametrize("be", BACKENDS)
def test_ghost_system_a_takes_only_interpolation(be):
    real, ghost, ge, src, virt, si, lf, h = _ghost_pair()
    bad = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.StrainRateVorticityPfn(), ghost, virt)
    lf2 = G.LeapFrogTimeIntegrator([real], [bad], ghosts=(ge,), virtual_systems=(virt,))
    with pytest.raises(Exception):
        G.Session([lf2], backend=make_backend(be))


def test_ghost_system_a_needs_copied_stress():
    real, ghost, ge, src, virt, si, lf, h = _ghost_pair()
    bare = G.GhostParticleSystem(real)
    ge2 = G.GhostEntry(bare, 3.0 * h, ((1.0, 0.0), (0.0, 0.0)))
    it = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.InterpolateFieldFn("stress"), bare, virt)
    lf2 = G.LeapFrogTimeIntegrator([real], [it], ghosts=(ge2,), virtual_systems=(virt,))
    with pytest.raises(Exception):
        G.Session([lf2], backend=make_backend("oracle"))


def test_trapdoor_layout():
    lf, meta = scenarios.trapdoor()
    assert (meta["n_soil"], meta["n_bottom"], meta["n_trapdoor"]) == (26400, 2340, 400)
    assert len(lf.virtual_systems) == 2 and len(lf.ghosts) == 1 and len(lf.probes) == 1
    assert isinstance(lf.interactions[2].system_a, G.GhostParticleSystem)
    assert lf.gamma == 0.002
    lf2, _ = scenarios.trapdoor(moving=True)
    assert lf2.gamma == 0.0 and tuple(lf2.virtual_systems[1].prescribed_v) == (0.0, -0.005)


def _small(moving):
    return scenarios.trapdoor(nx=48, ny=20, ntd_x=12, n_layers=4, moving=moving, geostatic=True)


def test_trapdoor_oracle_ghosts_reach_the_bottom():
    out = []
    for drop in (False, True):
        lf, meta = _small(False)
        if drop:
            inters = [it for k, it in enumerate(lf.interactions) if k != 2]
            lf = G.LeapFrogTimeIntegrator(lf.systems, inters, ghosts=lf.ghosts, virtual_systems=lf.virtual_systems)
        s = G.Session([lf], backend=make_backend("oracle"))
        s.push()
        s.step(1, meta["cfl"])
        s.pull()
        b = lf.virtual_systems[0]
        o = np.argsort(b.source.id)
        out.append((b.w_sum[o].copy(), b.source.x[o].copy()))
    (w_all, x), (w_soil, _) = out
    diff = w_all != w_soil
    assert diff.any()
    # only bottom particles within 2h of a ghost (x within 3h + 2h of a wall) change
    L = 48 * 0.05
    near = (x[:, 0] < 5 * 0.06) | (x[:, 0] > L - 5 * 0.06)
    assert np.all(near[diff]) and np.all(w_all[diff] > w_soil[diff])


def _run(lf, be, nsteps, cfl, prec=None, graphs=None):
    kw = {} if prec is None else dict(precision=prec)
    mode = parity.one_step_mode(lf, G.PRECISION_FP64 if prec is None else prec) if nsteps == 1 else parity.INPUTS
    s = G.Session([lf], backend=make_backend(be, track=mode if be == "oracle" else False), **kw)
    if graphs is not None:
        s.backend.set_graphs(graphs, 16)
    s.push()
    s.step(nsteps, cfl)
    s.measure_probes()
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
    pg, pc = lf_g.probes[0], lf_c.probes[0]
    np.testing.assert_allclose(pg.x, pc.x, rtol=0, atol=1e-15)
    scale = np.abs(pc.stress).max()
    assert np.abs(pg.stress - pc.stress).max() <= tol * scale


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (20, 1e-8)])
@pytest.mark.parametrize("moving", [False, True])
def test_trapdoor_parity(nsteps, tol, moving):
    lf_g, meta = _small(moving)
    lf_c, _ = _small(moving)
    _run(lf_g, "cuda", nsteps, meta["cfl"])
    c = _run(lf_c, "oracle", nsteps, meta["cfl"])
    _cmp(lf_g, lf_c, c, nsteps, tol)


@pytest.mark.gpu
def test_trapdoor_fp32c():
    lf_g, meta = _small(True)
    lf_c, _ = _small(True)
    _run(lf_g, "cuda", 20, meta["cfl"], prec=G.PRECISION_FP32_COMPENSATED)
    c = _run(lf_c, "oracle", 20, meta["cfl"])
    _cmp(lf_g, lf_c, c, 20, {"*": 1e-3, "strain": 1e-2, "strain_p": 1e-2})


@pytest.mark.gpu
@pytest.mark.parametrize("moving", [False, True])
def test_trapdoor_graph_steps_bit_identical(moving):
    out = []
    for graphs in (False, True):
        lf, meta = _small(moving)
        st = _run(lf, "cuda", 40, meta["cfl"], graphs=graphs).stats()
        out.append((lf, st))
    (le, _), (lg, st) = out
    assert st["graph_steps"] > 0
    for se, sg in zip(_systems(le), _systems(lg)):
        for name, _ in se.particle_fields():
            assert np.array_equal(getattr(se, name), getattr(sg, name)), f"{se.name}.{name}"
    for ve, vg in zip(le.virtual_systems, lg.virtual_systems):
        assert np.array_equal(ve.w_sum, vg.w_sum)
    assert np.array_equal(le.probes[0].stress, lg.probes[0].stress)


def test_trapdoor_script_size_on_the_oracle():
    """The script's sizes (264 x 100 soil, 10-layer bottom and trapdoor, wall
    ghosts, five probes) through two steps and a measurement on the oracle."""
    lf, meta = scenarios.trapdoor(geostatic=True)
    s = G.Session([lf], backend=make_backend("oracle"))
    s.push()
    s.step(2, meta["cfl"])
    s.measure_probes()
    s.pull()
    soil = lf.systems[0]
    assert np.all(np.isfinite(soil.x)) and np.all(np.isfinite(soil.stress))
    bottom, door = lf.virtual_systems
    assert (bottom.w_sum > 0).sum() > 0 and (door.w_sum > 0).sum() > 0
    probe = lf.probes[0]
    # geostatic σ_yy at the soil's base, 5 m of soil at 1600 kg/m³
    assert np.all(probe.stress[:, 1] < 0.0)
    assert np.all(np.abs(probe.stress[:, 1]) < 1600.0 * 9.81 * 5.0 * 1.1)


@pytest.mark.parametrize("be", BACKENDS)
def test_ghost_system_a_takes_no_velocity_adjustment(be):
    real, ghost, ge, src, virt, si, lf, h = _ghost_pair()
    it = G.SystemInteraction(G.CubicSplineKernel(h, ndims=2), G.InterpolateFieldFn("v"), ghost, virt,
                             velocity_adjust_pairwise_fn=G.XSPHPfn(0.5))
    lf2 = G.LeapFrogTimeIntegrator([real], [it], ghosts=(ge,), virtual_systems=(virt,))
    with pytest.raises(Exception):
        G.Session([lf2], backend=make_backend(be))
