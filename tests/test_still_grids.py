"""Grids over walls that never move, built batched.

The still walls' counts and scans run as one launch each over a table of at
most 16 interactions; more walls take several table launches, and a wall
whose grid has more cells than the batched scan takes keeps its own count
and scan.  A fluid block slides over a floor made of 20 separate wall
systems (one dynamic-boundary interaction each), so the grids of the floor
pieces it passes change geometry while the others keep their CSR; with a
far-away wall the union box of that interaction's grid holds about ten
million cells.  The device follows the oracle in eager and captured steps.
"""
import numpy as np
import pytest

import grasph_b200 as G
import parity
from gc_helpers import make_backend

pytestmark = pytest.mark.gpu


def _segmented_floor(nseg=20, far_wall=False):
    dx, c = 0.02, 1.0
    h = 1.2 * dx
    n = 6
    mass = 1000.0 * dx * dx
    fluid = G.FluidParticleSystem("fluid", n * n, 2, mass, c, state_updater=G.TaitEOSUpdater(1000.0))
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    fluid.x[:, 0] = (ii.ravel() + 0.5) * dx
    fluid.x[:, 1] = (jj.ravel() + 0.5) * dx
    fluid.v[:] = [1.0, 0.0]
    fluid.rho[:] = 1000.0
    k = G.CubicSplineKernel(h, ndims=2)
    pfn = G.FluidPfn(0.1, 0.0, h)
    systems, inters = [fluid], [G.SystemInteraction(k, pfn, fluid)]
    # floor piece s: the column x = -0.1 + s dx, three layers deep
    for s in range(nseg):
        piece = G.BasicParticleSystem(f"floor{s}", 3, 2, mass, c)
        piece.x[:] = [(-0.1 + s * dx, -(l + 0.5) * dx) for l in range(3)]
        piece.rho[:] = 1000.0
        systems.append(piece)
        inters.append(G.SystemInteraction(k, pfn, fluid, G.DynamicBoundarySystem(piece, (0.0, 1.0), (0.0, 0.0), 3.0)))
    if far_wall:
        far = G.BasicParticleSystem("far", 4, 2, mass, c)
        far.x[:] = [(150.0 + q * dx, 150.0) for q in range(4)]
        far.rho[:] = 1000.0
        systems.append(far)
        inters.append(G.SystemInteraction(k, pfn, fluid, G.DynamicBoundarySystem(far, (0.0, -1.0), (0.0, 150.0), 3.0)))
    return G.LeapFrogTimeIntegrator(systems, inters), 0.2


@pytest.mark.parametrize("far_wall", [False, True])
@pytest.mark.parametrize("graphs", [False, True])
def test_many_still_walls_follow_the_oracle(graphs, far_wall):
    out, sessions = [], []
    for be in ("cuda", "oracle"):
        lf, cfl = _segmented_floor(far_wall=far_wall)
        s = G.Session([lf], backend=make_backend(be, track=parity.INPUTS if be == "oracle" else False))
        sessions.append(s)
        if be == "cuda":
            s.backend.set_graphs(graphs, 8)
        s.push()
        s.step(40, cfl)
        s.pull()
        out.append(lf)
    st = sessions[0].stats()
    if graphs:
        assert st["graph_steps"] > 0
    fc = out[1].systems[0]
    assert fc.x[:, 0].max() > 0.25  # the block moved over several floor pieces
    assert np.abs(fc.v[:, 1]).max() > 0  # the floor pushed back
    parity.compare_integrators(out[0], out[1], sessions[1], 1e-10, exact_ids=False, skip=parity.RATES)
