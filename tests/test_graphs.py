"""Captured-step scheduling against exactly sized steps.

With graphs on, gc_step runs windows of captured steps sized from buffer
capacities and verifies each window; a window whose plan outgrew a capacity
is rolled back to its snapshot and re-run exactly.  Either way the result
must be bit-identical to stepping with one host read of the plan per step.
"""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
import parity
from gc_helpers import make_backend

pytestmark = pytest.mark.gpu

CASES = {
    "dambreak_2d": (scenarios.dambreak_2d, dict(nx=20, ny=40, dx=0.05, tank=(2.0, 2.5))),
    "dambreak_3d": (scenarios.dambreak_3d, dict(nx=8, ny=6, nz=12, dx=0.05, tank=(1.0, 0.5, 1.0))),
    "column": (scenarios.column_collapse, dict(nx=40, ny=20, dx=0.005)),
}


def _run(builder, kw, graphs, nsteps, sync_every=32, prec=G.PRECISION_FP64, tweak=None, calls=1, margin=0.0):
    lf, meta = builder(**kw)
    if tweak:
        tweak(lf)
    s = G.Session([lf], backend=make_backend("cuda"), precision=prec)
    s.backend.set_graphs(graphs, sync_every, margin)
    s.push()
    per = nsteps // calls
    for _ in range(calls):
        s.step(per, meta["cfl"])
    s.pull()
    return lf, s.stats()


def _same(lf_a, lf_b):
    for sa, sb in zip(lf_a.systems, lf_b.systems):
        for name, _ in sa.particle_fields():
            a, b = getattr(sa, name), getattr(sb, name)
            assert np.array_equal(a, b, equal_nan=True), f"{sa.name}.{name} differs"


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("prec", [G.PRECISION_FP64, G.PRECISION_FP32_COMPENSATED])
def test_graph_steps_bit_identical(case, prec):
    builder, kw = CASES[case]
    lf_e, st_e = _run(builder, kw, False, 70, prec=prec)
    lf_g, st_g = _run(builder, kw, True, 70, prec=prec, calls=2)
    _same(lf_g, lf_e)
    assert st_e["graph_steps"] == 0
    assert st_g["graph_steps"] >= 60
    assert st_g["steps_done"] == st_e["steps_done"] == 70


def _fling(lf):
    # one fluid particle, well clear of the others and of the walls, thrown
    # upward: every grid around it grows by many cells per step
    f = lf.systems[0]
    f.x[0] = (1.0, 10.0)
    f.v[0] = (0.0, 20000.0)


def test_capacity_overflow_rolls_back_bit_identical():
    builder, kw = CASES["dambreak_2d"]
    lf_e, _ = _run(builder, kw, False, 40, tweak=_fling)
    lf_g, st = _run(builder, kw, True, 40, sync_every=4, tweak=_fling, margin=1.0)
    _same(lf_g, lf_e)
    assert st["rollbacks"] > 0
    assert st["graph_steps"] > 0


@pytest.mark.parametrize("case", ["column", "dambreak_2d", "dambreak_3d"])
@pytest.mark.parametrize("prec", [G.PRECISION_FP64, G.PRECISION_FP32_COMPENSATED])
def test_sweep_configs_bit_identical(prec, case):
    """Every launch configuration the autotuner picks from gives the same
    bits: buffered and chunk-staged sweeps, for the stress functors of the
    column and the fluid functors of the dam breaks (walls included)."""
    builder, kw = CASES[case]
    ref = None
    for cfg in range(G.consts.GC_NUM_SWEEP_CONFIGS):
        lf, meta = builder(**kw)
        s = G.Session([lf], backend=make_backend("cuda"), precision=prec)
        s.backend.set_sweep_config(cfg)
        s.push()
        s.step(12, meta["cfl"])
        s.pull()
        if ref is None:
            ref = lf
        else:
            _same(lf, ref)


def test_autotune_chooses_every_sweep():
    builder, kw = CASES["column"]
    lf, st = _run(builder, kw, True, 40)
    # two stages of one system: both sweeps tuned, then graph replays
    assert sum(st["sweep_cfg_chosen"]) == 2
    assert st["graph_steps"] > 0


def _passing_block():
    """A fluid block sliding (no gravity) along a short static wall and past
    its end: the union box of the fluid-wall grid, hence its geometry, changes
    every few steps while the wall's particles never move."""
    dx, c = 0.02, 1.0
    h = 1.2 * dx
    n = 6
    fluid = G.FluidParticleSystem("fluid", n * n, 2, 1000.0 * dx * dx, c, state_updater=G.TaitEOSUpdater(1000.0))
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    fluid.x[:, 0] = (ii.ravel() + 0.5) * dx
    fluid.x[:, 1] = (jj.ravel() + 0.5) * dx
    fluid.v[:] = [1.0, 0.0]
    fluid.rho[:] = 1000.0
    xs = np.arange(-0.1, 0.2 + 1e-9, dx)
    wall = G.BasicParticleSystem("wall", 3 * len(xs), 2, 1000.0 * dx * dx, c)
    wall.x[:] = [(x, -(l + 0.5) * dx) for l in range(3) for x in xs]
    wall.rho[:] = 1000.0
    k = G.CubicSplineKernel(h, ndims=2)
    pfn = G.FluidPfn(0.1, 0.0, h)
    si = G.SystemInteraction(k, pfn, fluid, G.DynamicBoundarySystem(wall, (0.0, 1.0), (0.0, 0.0), 3.0))
    return G.LeapFrogTimeIntegrator([fluid, wall], [si]), 0.2


@pytest.mark.parametrize("graphs,profiling", [(False, False), (True, False), (True, True)])
def test_still_wall_grid_follows_geometry_changes(graphs, profiling):
    """The CSR over a wall that never moves is kept on the device while its
    grid's geometry is unchanged and recounted when it changes (in captured
    steps the batched count and scan return at once on a flag the step's
    plan sets): the device stays with the oracle while the block slides past
    the wall's end.
    With sweep timing on, the captured step also holds event nodes."""
    out, sessions = [], []
    for be in ("cuda", "oracle"):
        lf, cfl = _passing_block()
        s = G.Session([lf], backend=make_backend(be, track=parity.INPUTS if be == "oracle" else False))
        sessions.append(s)
        if be == "cuda":
            s.backend.set_graphs(graphs, 8)
            s.backend.set_profiling(profiling)
        s.push()
        s.step(40, cfl)
        s.pull()
        out.append(lf)
    st = sessions[0].stats()
    if graphs:
        assert st["graph_steps"] > 0  # the steps were captured, not run eagerly after a failed capture
    if profiling:
        assert st["sweep_launches"] > 0
    fc = out[1].systems[0]
    assert fc.x[:, 0].max() > 0.3  # the block left the wall's end behind
    # per-particle scale of tests/parity.py, the state on its integrated scale
    parity.compare_integrators(out[0], out[1], sessions[1], 1e-10, exact_ids=False, skip=parity.RATES)
