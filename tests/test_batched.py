"""Batched stepping: many simulations of one model structure in one context.

Every instance's particles sort into their own cell range, warp groups never
span two instances, and every instance keeps its own dt, so an instance's
result in the mix is bit-identical to the same instance run alone, in both
precisions.  One instance of the mix is also checked against the oracle.
"""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
from gc_helpers import make_backend, oracle_threads
import parity

pytestmark = pytest.mark.gpu

STEPS = 15


def _columns(count=5):
    return scenarios.batched_columns(count=count, seed=7, nmin=200, nmax=2500, dx=0.002)


def _fields(lf):
    out = []
    for s in lf.systems:
        for name, _ in s.particle_fields():
            if name == "v_adjustment":
                continue
            out.append((f"{s.name}.{name}", np.array(getattr(s, name), copy=True)))
    return out


@pytest.mark.parametrize("prec", [G.PRECISION_FP64, G.PRECISION_FP32_COMPENSATED])
def test_instance_in_mix_equals_alone(prec):
    mix = _columns()
    sess = G.Session([lf for lf, _ in mix], backend=make_backend("cuda"), precision=prec)
    sess.push()
    sess.step(STEPS, mix[0][1]["cfl"])
    sess.pull()
    for k, (lf, meta) in enumerate(mix):
        alone, _ = _columns()[k]
        s1 = G.Session([alone], backend=make_backend("cuda"), precision=prec)
        s1.push()
        s1.step(STEPS, meta["cfl"])
        s1.pull()
        for (na, a), (nb, b) in zip(_fields(lf), _fields(alone)):
            assert na == nb
            assert np.array_equal(a, b, equal_nan=True), f"instance {k}: {na} differs alone vs in the mix"


def test_mix_instance_against_oracle():
    mix = _columns(count=3)
    sess = G.Session([lf for lf, _ in mix], backend=make_backend("cuda"))
    sess.push()
    sess.step(STEPS, mix[0][1]["cfl"])
    sess.pull()
    k = 1
    ref, meta = _columns(count=3)[k]
    c = G.Session([ref], backend=make_backend("oracle", track=parity.INPUTS))
    c.push()
    c.step(STEPS, meta["cfl"])
    c.pull()
    # per-particle scale of tests/parity.py, the state on its integrated scale
    parity.compare_integrators(mix[k][0], ref, c, 1e-8, exact_ids=False, skip=parity.RATES)


def test_fp32_compensated_mix_after_1000_steps():
    """Compensated mix against the FP64 oracle after 1000 steps, every
    instance on the per-particle scale: density within 1e-4 and stress
    within 1e-3 (the other state fields within 1e-3, the strains within
    1e-2: the FP32 records round v to FP32)."""
    mix32 = _columns(count=3)
    s32 = G.Session([lf for lf, _ in mix32], backend=make_backend("cuda"),
                    precision=G.PRECISION_FP32_COMPENSATED)
    s32.push()
    s32.step(1000, mix32[0][1]["cfl"])
    s32.pull()
    for k, (lf, meta) in enumerate(mix32):
        ref, _ = _columns(count=3)[k]
        c = G.Session([ref], backend=make_backend("oracle", track=parity.INPUTS, threads=oracle_threads()))
        c.push()
        c.step(1000, meta["cfl"])
        c.pull()
        rep = {}
        parity.compare_integrators(lf, ref, c, {"*": 1e-3, "rho": 1e-4, "stress": 1e-3, "strain": 1e-2,
                                                "strain_p": 1e-2}, exact_ids=False, skip=parity.RATES, report=rep)
        print(f"instance {k} FP32c after 1000 steps:", rep["soil"])
