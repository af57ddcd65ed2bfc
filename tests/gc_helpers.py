"""Helpers shared by the tests: backend construction and small builders."""
from __future__ import annotations

import os

import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import consts as C


def oracle_threads():
    """Host threads for oracle runs at the configs' sizes."""
    return max(1, min(32, os.cpu_count() or 1))


def make_backend(name, track=False, threads=1):
    """`track`: the oracle keeps magnitude shadows, the per-particle scale
    of tests/parity.py (True or 1: over the pair terms; 2: over the
    inputs)."""
    if name == "oracle":
        from pyoracle import OracleBackend
        return OracleBackend(threads=threads, track_magnitude=track)
    return G.CudaBackend()


def step_dt(lf, cfl):
    """The step's dt, CFL·h_min/c_max over the integrator's systems
    (src/TimeIntegration.jl:598)."""
    h = min(si.kernel.h for si in lf.interactions)
    c = max(ps.c for ps in lf.systems)
    return cfl * h / c


BACKENDS = ["oracle", pytest.param("cuda", marks=pytest.mark.gpu)]


def session(name, systems, interactions, ghosts=(), gamma=0.0):
    lf = G.LeapFrogTimeIntegrator(systems, interactions, ghosts=ghosts, gamma=gamma)
    s = G.Session([lf], backend=make_backend(name))
    s.push()
    return lf, s


def basic(n=8, nd=2, mass=1.0, c=1.0, **kw):
    return G.BasicParticleSystem("test", n, nd, mass, c, **kw)


def kernel(h=0.1, nd=2):
    return G.CubicSplineKernel(h, ndims=nd)


def lcg_vals(count, offset=0):
    """The reference tests' LCG (test/test_interaction_sweep.jl:134)."""
    out = []
    for i in range(1 + offset, count + 1 + offset):
        r = (i * 6364136223846793005 + 1442695040888963407) % (2 ** 32)
        out.append((r % 100) / 2000.0)
    return out


def keys(x, cutoff):
    return np.floor(x / cutoff).astype(np.int64)


def lex_sorted(k):
    for i in range(len(k) - 1):
        if tuple(k[i + 1]) < tuple(k[i]):
            return False
    return True


def rel_err(a, b, scale):
    """|a-b| / scale elementwise, with the scale floored at tiny."""
    scale = np.maximum(np.abs(scale), 1e-300)
    return np.abs(np.asarray(a) - np.asarray(b)) / scale
