"""Float32 particle systems: the element type of a system, kernel, functor
and integrator follows the reference's constructors, a functor of the wrong
float type is refused, and stepping keeps every array Float32.

Restates test/test_particles.jl:54-75, test/test_kernels.jl:31-43,
test/test_interaction_init.jl:132-170, test/test_elasto_plastic.jl:59-72
and test/test_time_integration.jl:144-166.  The device (and the oracle)
computes a Float32 system from its values widened to Float64 and rounds the
results back, so a Float32 system steps to exactly the Float32 rounding of
its Float64 twin built from the same Float32 values."""
import numpy as np
import pytest

import grasph_b200 as G
from gc_helpers import make_backend

f32 = np.float32


def test_system_dtype_propagation():
    ps = G.BasicParticleSystem("f32", 5, 2, 1.0, 2.0, dtype=np.float32)
    for name in ("x", "v", "dvdt", "rho", "drhodt", "v_adjustment"):
        assert getattr(ps, name).dtype == np.float32, name
    assert isinstance(ps.mass, np.float32) and isinstance(ps.c, np.float32)
    fl = G.FluidParticleSystem("f32", 5, 2, 1.0, 2.0, dtype=np.float32)
    assert fl.p.dtype == np.float32 and fl.rho.dtype == np.float32
    st = G.StressParticleSystem("s", 5, 2, 4, 1.0, 1.0, dtype=np.float32)
    assert st.stress.dtype == np.float32 and st.strain_rate.dtype == np.float32
    ep = G.ElastoPlasticParticleSystem("f32", 5, 2, 3, 1.0, 1.0, dtype=np.float32)
    for name in ("rho", "stress", "vorticity", "strain", "strain_p"):
        assert getattr(ep, name).dtype == np.float32, name
    assert ep.vorticity.shape == (5,) and isinstance(ep.mass, np.float32)
    ep3 = G.ElastoPlasticParticleSystem("f32_3d", 5, 3, 6, 1.0, 1.0, dtype=np.float32)
    assert ep3.vorticity.shape == (5, 3) and ep3.vorticity.dtype == np.float32
    d = G.BasicParticleSystem("f64", 5, 2, 1.0, 2.0)
    assert d.x.dtype == np.float64 and isinstance(d.mass, float)
    with pytest.raises(G.ArgumentError):
        G.BasicParticleSystem("f16", 5, 2, 1.0, 2.0, dtype=np.float16)


def test_kernel_dtype_propagation():
    k = G.CubicSplineKernel(f32(0.1), ndims=2)
    assert isinstance(k.h, np.float32) and isinstance(k.norm_coeff, np.float32)
    assert isinstance(k.interaction_length, np.float32)
    w = G.WenlandC2Kernel(f32(0.1), ndims=3)
    assert isinstance(w.norm_coeff, np.float32)
    k64 = G.CubicSplineKernel(0.1, ndims=2)
    assert isinstance(k64.h, float) and isinstance(k64.norm_coeff, float)
    assert isinstance(k64.interaction_length, float)
    # the Float64 values are unchanged: 10/(7π h²), 1/(π h³)
    assert k64.norm_coeff == 10.0 / ((7.0 * np.pi) * (0.1 * 0.1))
    assert G.CubicSplineKernel(1.0, ndims=3).norm_coeff == pytest.approx(1.0 / np.pi)


def test_pfn_float_type_and_mismatch():
    ps = G.FluidParticleSystem("test", 5, 2, 1.0, 1.0)
    k = G.CubicSplineKernel(0.1, ndims=2)
    assert G.float_type(G.FluidPfn(0.1, 0.0, 0.1)) is np.float64
    pfn = G.FluidPfn(f32(0.1), f32(0.0), f32(0.1))
    assert G.float_type(pfn) is np.float32
    assert isinstance(pfn.h, np.float32)
    # a mixed construction promotes to Float64, as Julia's promote does
    assert G.float_type(G.FluidPfn(f32(0.1), 0.0, f32(0.1))) is np.float64
    with pytest.raises(G.ArgumentError) as e:
        G.SystemInteraction(k, pfn, ps)
    msg = str(e.value)
    assert "FluidPfn" in msg and "Float32" in msg and "Float64" in msg
    # unparameterised functors pass; a mismatch in a tuple's second entry raises
    G.SystemInteraction(k, G.StrainRatePfn(), G.StressParticleSystem("s", 5, 2, 4, 1.0, 1.0))
    with pytest.raises(G.ArgumentError):
        G.SystemInteraction(k, (None, pfn), ps)
    ps32 = G.FluidParticleSystem("f32", 5, 2, 1.0, 1.0, dtype=np.float32)
    G.SystemInteraction(G.CubicSplineKernel(f32(0.1), ndims=2), pfn, ps32)


def test_state_updater_float_type():
    with pytest.raises(G.ArgumentError) as e:
        G.FluidParticleSystem("f", 5, 2, 1.0, 1.0, state_updater=G.TaitEOSUpdater(f32(1000.0)))
    assert "TaitEOSUpdater" in str(e.value)
    G.FluidParticleSystem("f", 5, 2, 1.0, 1.0, dtype=np.float32, state_updater=G.TaitEOSUpdater(f32(1000.0)))
    with pytest.raises(G.ArgumentError):
        G.FluidParticleSystem("f", 5, 2, 1.0, 1.0, dtype=np.float32, state_updater=G.LinearEOSUpdater(1000.0))
    u = G.ElastoPlasticStressUpdater(f32(1e6), f32(0.3), f32(0.5), f32(0.0), f32(0.0))
    assert G.float_type(u) is np.float32 and isinstance(u.E, np.float32)
    assert G.float_type(G.ElastoPlasticStressUpdater(f32(1e6), 0.3, 0.5, 0.0, 0.0)) is np.float64


def _tank(dtype, seed=7):
    """A 2-D fluid block over a dynamic-boundary floor, its parameters given
    as Float32 values (and widened for the Float64 twin)."""
    T = dtype
    dx = f32(0.05)
    h = f32(1.3) * dx
    nx, ny = 8, 10
    rng = np.random.default_rng(seed)
    fl = G.FluidParticleSystem("fluid", nx * ny, 2, T(f32(1000.0) * dx * dx), T(f32(30.0)), dtype=T,
                               source_v=np.array([0.0, -9.81], np.float32).astype(T),
                               state_updater=G.TaitEOSUpdater(T(f32(1000.0))))
    xs = np.array([[(i + 0.5) * dx, (j + 1.5) * dx] for j in range(ny) for i in range(nx)], np.float32)
    xs += (rng.uniform(-0.1, 0.1, xs.shape) * dx).astype(np.float32)
    fl.x[:] = xs
    fl.rho[:] = f32(1000.0) + rng.uniform(0.0, 2.0, fl.n).astype(np.float32)
    wall = G.FluidParticleSystem("floor", 3 * (nx + 6), 2, T(f32(1000.0) * dx * dx), T(f32(30.0)), dtype=T,
                                 state_updater=G.TaitEOSUpdater(T(f32(1000.0))))
    wall.x[:] = np.array([[(i - 3 + 0.5) * dx, -j * dx] for j in range(3) for i in range(nx + 6)], np.float32)
    wall.rho[:] = f32(1000.0)
    k = G.CubicSplineKernel(T(h), ndims=2)
    pfn = G.FluidPfn(T(f32(0.1)), T(f32(0.0)), T(h))
    inters = [G.SystemInteraction(k, pfn, fl),
              G.SystemInteraction(k, pfn, fl, G.DynamicBoundarySystem(wall, [0.0, 1.0], [0.0, 0.0], 1.5))]
    return G.LeapFrogTimeIntegrator([fl, wall], inters), fl, wall


def _run_pair(backend_name):
    lf32, fl32, w32 = _tank(np.float32)
    lf64, fl64, w64 = _tank(np.float64)
    assert isinstance(lf32.c, np.float32) and isinstance(lf32.h, np.float32)
    for lf in (lf32, lf64):
        s = G.Session([lf], backend=make_backend(backend_name))
        s.push()
        s.step(5, 0.3)
        s.pull()
    for a, b in ((fl32, fl64), (w32, w64)):
        for name, _ in a.particle_fields():
            x32, x64 = getattr(a, name), getattr(b, name)
            if name == "id":
                assert np.array_equal(x32, x64)
                continue
            assert x32.dtype == np.float32, f"{a.name}.{name}"
            assert np.array_equal(x32, x64.astype(np.float32)), f"{a.name}.{name}"
    assert fl32.v[:, 1].mean() < 0


def test_float32_system_steps_as_rounded_float64_twin_oracle():
    _run_pair("oracle")


@pytest.mark.gpu
def test_float32_system_steps_as_rounded_float64_twin_device():
    _run_pair("cuda")


@pytest.mark.gpu
def test_float32_integration_preserves_eltype():
    """test/test_time_integration.jl:144-166 through time_integrate."""
    ps = G.BasicParticleSystem("fluid", 4, 2, 1.0, 10.0, dtype=np.float32)
    vals = np.linspace(f32(0.2), f32(0.8), 8, dtype=np.float32)
    ps.x[:] = vals.reshape(4, 2)  # particle i takes (vals[2i], vals[2i+1])
    ps.v[:] = 0
    ps.rho[:] = f32(1000.0)
    k = G.CubicSplineKernel(f32(0.1), ndims=2)
    si = G.SystemInteraction(k, None, ps)
    lf = G.LeapFrogTimeIntegrator(ps, si)
    assert isinstance(lf.c, np.float32) and isinstance(lf.h, np.float32)
    G.time_integrate(lf, 3, 100, 100, 0.5, None)
    for name in ("x", "v", "dvdt", "rho", "drhodt"):
        assert getattr(ps, name).dtype == np.float32, name
