"""The allocation-free sort entry point against the allocating one.

`gc_cell_sort_perm_noalloc` keeps its scratch in a static device array; its
permutation must equal `gc_sort_system`'s (which is 1-based and allocates
through its context) on the same points, call after call.
"""
import ctypes as ct

import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200.engine import load_library
from gc_helpers import make_backend

pytestmark = pytest.mark.gpu

MAX_N = 1 << 16


def _lib():
    lib = load_library()
    f = lib.gc_cell_sort_perm_noalloc
    f.restype = ct.c_int
    f.argtypes = [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_double, ct.c_void_p, ct.c_void_p]
    return f


def _noalloc_perm(x, cutoff):
    import torch
    n, nd = x.shape
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda")
    perm = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _lib()(xd.data_ptr(), n, nd, cutoff, perm.data_ptr(), stream)
    return st, perm[:n].cpu().numpy()


def _reference_perm(x, cutoff):
    n, nd = x.shape
    ps = G.BasicParticleSystem("p", n, nd, 1.0, 1.0)
    ps.x[:] = x
    k = G.CubicSplineKernel(cutoff / 2, ndims=nd)
    lf = G.LeapFrogTimeIntegrator([ps], [G.SystemInteraction(k, None, ps)])
    s = G.Session([lf], backend=make_backend("cuda"))
    s.push()
    return s.sort_particles(ps, cutoff) - 1


def _points(seed, n, nd, lo, hi, cutoff):
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo, hi, (n, nd))
    x[::5] = np.round(x[::5] / cutoff) * cutoff  # exactly on cell faces
    x[1::97] = x[0]                              # duplicates: ties keep source order
    return x


def test_noalloc_matches_sort_system_two_calls_in_a_row():
    cases = [
        (_points(3, 5000, 2, -1.3, 2.1, 0.02), 0.02),
        (_points(4, 40000, 3, -0.4, 0.9, 0.03), 0.03),
    ]
    for x, cutoff in cases:
        st, got = _noalloc_perm(x, cutoff)
        assert st == G.consts.GC_OK
        ref = _reference_perm(x, cutoff)
        assert np.array_equal(got, ref)


def test_noalloc_limits_and_recovery():
    # more particles than the static scratch holds: refused before any launch
    x = np.zeros((MAX_N + 1, 2))
    st, _ = _noalloc_perm(x, 1.0)
    assert st == G.consts.GC_ERR_CAPACITY
    # key lattice wider than the scratch's cell table
    x = _points(5, 1000, 2, 0.0, 1000.0, 1.0)
    st, _ = _noalloc_perm(x, 1.0)
    assert st == G.consts.GC_ERR_CAPACITY
    # non-finite coordinate
    x = _points(6, 1000, 2, 0.0, 1.0, 0.1)
    x[17, 1] = np.nan
    st, _ = _noalloc_perm(x, 0.1)
    assert st == G.consts.GC_ERR_NONFINITE
    # the next call starts from clean scratch
    x = _points(7, MAX_N, 2, 0.0, 3.0, 0.01)
    st, got = _noalloc_perm(x, 0.01)
    assert st == G.consts.GC_OK
    assert np.array_equal(got, _reference_perm(x, 0.01))
