"""The sort's in-order fast path (src/Sorting.jl:176-186): when a moving
system's cell keys are already non-decreasing the reorder is the identity,
and the device skips the atomic placement and the per-cell fix-up.  Results
must not change: every case is compared bit for bit with the oracle, whose
sort takes the same early exit."""
import numpy as np
import pytest

import grasph_b200 as G
from gc_helpers import make_backend

pytestmark = pytest.mark.gpu


def _block(v0, seed):
    """A 2-D fluid block without gravity at the rest density: every pair
    term vanishes, so the block moves rigidly at `v0`.  Particles are listed
    in a shuffled order, so the first sort reorders."""
    nx, ny, dx = 24, 16, 0.01
    h = 1.3 * dx
    rng = np.random.default_rng(seed)
    fl = G.FluidParticleSystem("fluid", nx * ny, 2, 1000.0 * dx * dx, 20.0,
                               state_updater=G.TaitEOSUpdater(1000.0))
    x = np.array([[(i + 0.5) * dx, (j + 0.5) * dx] for j in range(ny) for i in range(nx)])
    fl.x[:] = x[rng.permutation(len(x))]
    fl.v[:] = v0
    fl.rho[:] = 1000.0
    k = G.CubicSplineKernel(h, ndims=2)
    lf = G.LeapFrogTimeIntegrator([fl], [G.SystemInteraction(k, G.FluidPfn(0.1, 0.0, h), fl)])
    return lf, fl


@pytest.mark.parametrize("v0,expect", [((0.0, 0.0), "all"), ((0.37, 0.11), "some")])
def test_in_order_sorts_skip_the_reorder_and_match_the_oracle(v0, expect):
    nsteps = 40
    runs = []
    for name in ("cuda", "oracle"):
        lf, fl = _block(v0, seed=5)
        s = G.Session([lf], backend=make_backend(name))
        s.push()
        s.step(nsteps, 0.3)
        s.pull()
        runs.append((fl, s))
    (fg, sg), (fc, _) = runs
    # the same order (ids), and the same rigid motion
    assert np.array_equal(fg.id, fc.id)
    for name, _ in fg.particle_fields():
        assert np.allclose(getattr(fg, name), getattr(fc, name), rtol=1e-15, atol=1e-15), name
    n_in_order = sg.stats()["sorts_in_order"]
    print(f"v0={v0}: {n_in_order} of {nsteps} step sorts in order")
    if expect == "all":
        # every step after the first finds the block in key order
        assert n_in_order >= nsteps - 1
    else:
        # the drifting block crosses cell faces on some steps only
        assert 0 < n_in_order < nsteps - 1
