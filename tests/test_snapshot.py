"""Snapshots and restarts: write_h5 / read_h5! (src/Particles.jl:699-787),
_maybe_save! (src/TimeIntegration.jl:520-549) and _load_restart!
(src/Driver.jl:79-96), with the groups, attributes and datasets of the
reference's files in a NumPy container (no HDF5 library here).

A run that stops, saves and restarts in a fresh session from the file must
continue exactly as the uninterrupted run; read_h5!'s checks of n and ndims
are restated."""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
from grasph_b200.snapshot import read_snapshot, write_snapshot
from gc_helpers import BACKENDS, make_backend


def _fields(lf):
    out = {}
    for ps in list(lf.systems) + [v.source for v in getattr(lf, "virtual_systems", ())]:
        for name, _ in ps.particle_fields():
            out[(ps.name, name)] = np.array(getattr(ps, name), copy=True)
    return out


def _restart_case(build, be, tmp_path, n1=4, n2=5):
    lf, meta = build()
    s = G.Session([lf], backend=make_backend(be))
    s.push()
    s.step(n1, meta["cfl"])
    path = tmp_path / "snap.npz"
    s.save(path)
    s.step(n2, meta["cfl"])
    s.pull()
    straight = _fields(lf)
    lf2, _ = build()
    s2 = G.Session([lf2], backend=make_backend(be))
    step = s2.load(path)
    assert step == n1
    s2.step(n2, meta["cfl"])
    s2.pull()
    # a save after the restart records the global step (restart + steps since)
    path2 = tmp_path / "snap2.npz"
    s2.save(path2)
    with np.load(path2) as f:
        assert int(f["@step"]) == n1 + n2
    return straight, _fields(lf2)


@pytest.mark.parametrize("be", BACKENDS)
def test_restart_continues_the_run_dambreak(be, tmp_path):
    build = lambda: scenarios.dambreak_2d(nx=12, ny=24, dx=0.05, tank=(1.5, 2.0))
    a, b = _restart_case(build, be, tmp_path)
    for key in a:
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("be", BACKENDS)
def test_restart_continues_the_run_virtual_walls(be, tmp_path):
    build = lambda: scenarios.ep_column_virtual(dx=0.004, geostatic=True, bottom_v=(0.0, -0.05))
    a, b = _restart_case(build, be, tmp_path)
    for key in a:
        assert np.array_equal(a[key], b[key]), key


def test_snapshot_layout_and_checks(tmp_path):
    ps = G.FluidParticleSystem("fluid", 3, 2, 0.5, 10.0)
    ps.x[:] = [[0.0, 0.0], [1.0, 0.0], [2.0, 0.5]]
    ps.rho[:] = [1000.0, 1001.0, 1002.0]
    path = tmp_path / "s.npz"
    write_snapshot([ps], path, step=7)
    with np.load(path) as f:
        assert int(f["fluid/@n"]) == 3 and int(f["fluid/@ndims"]) == 2
        assert float(f["fluid/@mass"]) == 0.5 and float(f["fluid/@c"]) == 10.0
        np.testing.assert_array_equal(f["fluid/x"], ps.x)
        assert int(f["@step"]) == 7
    back = G.FluidParticleSystem("fluid", 3, 2, 0.5, 10.0)
    assert read_snapshot([back], path) == 7
    np.testing.assert_array_equal(back.rho, ps.rho)
    wrong_n = G.FluidParticleSystem("fluid", 4, 2, 0.5, 10.0)
    with pytest.raises(G.ArgumentError):
        read_snapshot([wrong_n], path)
    wrong_nd = G.FluidParticleSystem("fluid", 3, 3, 0.5, 10.0)
    with pytest.raises(G.ArgumentError):
        read_snapshot([wrong_nd], path)
    # _load_restart!: a system without a group is left untouched with a
    # warning; a file without a step restarts from step 0 with a warning
    other = G.FluidParticleSystem("other", 2, 2, 0.5, 10.0)
    other.rho[:] = 5.0
    with pytest.warns(UserWarning, match="no group for system 'other'"):
        assert read_snapshot([back, other], path) == 7
    assert np.all(other.rho == 5.0)
    nostep = tmp_path / "nostep.npz"
    write_snapshot([ps], nostep)
    with pytest.warns(UserWarning, match="assuming step 0"):
        assert read_snapshot([back], nostep) == 0


def test_restart_with_moving_probes_on_the_oracle(tmp_path):
    """Free probes moving with the trapdoor keep their positions across a
    restart; the measurement after it matches the uninterrupted run's."""
    def build():
        return scenarios.trapdoor(nx=48, ny=20, ntd_x=12, n_layers=4, moving=True, geostatic=True)
    lf, meta = build()
    s = G.Session([lf], backend=make_backend("oracle"))
    s.push()
    s.step(3, meta["cfl"])
    path = tmp_path / "td.npz"
    s.save(path)
    s.step(3, meta["cfl"])
    s.measure_probes()
    s.pull()
    lf2, _ = build()
    s2 = G.Session([lf2], backend=make_backend("oracle"))
    assert s2.load(path) == 3
    s2.step(3, meta["cfl"])
    s2.measure_probes()
    s2.pull()
    p1, p2 = lf.probes[0], lf2.probes[0]
    assert np.array_equal(p1.x, p2.x) and np.array_equal(p1.stress, p2.stress)
    a, b = _fields(lf), _fields(lf2)
    for key in a:
        assert np.array_equal(a[key], b[key]), key


# test/test_read_h5.jl restated (the container is NumPy's, the groups,
# attributes and checks the reference's)
from grasph_b200.snapshot import read_h5, system_from_h5, write_h5  # noqa: E402


def test_read_h5_basic_round_trip(tmp_path):
    ps1 = G.BasicParticleSystem("test1", 3, 2, 1.5, 2.0)
    ps1.x[:] = [[0.0, 1.0], [2.0, 3.0], [4.0, 5.0]]
    ps1.v[:] = [[0.1, 0.2], [0.3, 0.4], [0.5, 0.6]]
    ps1.rho[:] = [1.0, 2.0, 3.0]
    path = tmp_path / "out.npz"
    write_h5(ps1, path)
    ps2 = G.BasicParticleSystem("test2", 3, 2, 1.0, 1.0)
    read_h5(ps2, path)
    np.testing.assert_allclose(ps2.x, ps1.x)
    np.testing.assert_allclose(ps2.v, ps1.v)
    np.testing.assert_allclose(ps2.rho, ps1.rho)
    assert ps2.mass == 1.0 and ps2.c == 1.0  # metadata is not overwritten
    ps_new = system_from_h5(G.BasicParticleSystem, path, "test1")
    assert (ps_new.n, ps_new.ndims, ps_new.mass, ps_new.c) == (3, 2, 1.5, 2.0)
    np.testing.assert_allclose(ps_new.x, ps1.x)
    np.testing.assert_allclose(ps_new.v, ps1.v)
    np.testing.assert_allclose(ps_new.rho, ps1.rho)


def test_read_h5_fluid_path_constructor(tmp_path):
    ps1 = G.FluidParticleSystem("fluid1", 2, 2, 0.5, 10.0, source_v=[0.0, -9.81])
    ps1.x[:] = [[0.1, 0.2], [0.3, 0.4]]
    ps1.v[:] = [[0.5, 0.6], [0.7, 0.8]]
    ps1.rho[:] = 1000.0
    ps1.p[:] = [1.0, 2.0]
    path = tmp_path / "out.npz"
    write_h5(ps1, path)
    ps_new = system_from_h5(G.FluidParticleSystem, path, "fluid1", source_v=[0.0, -9.81])
    assert (ps_new.n, ps_new.mass, ps_new.c) == (2, 0.5, 10.0)
    for name in ("x", "v", "rho", "p"):
        np.testing.assert_allclose(getattr(ps_new, name), getattr(ps1, name))
    np.testing.assert_array_equal(ps_new.source_v, [0.0, -9.81])


def test_read_h5_stress_path_constructor(tmp_path):
    ps1 = G.StressParticleSystem("stress1", 2, 2, 3, 1.2, 5.0)
    ps1.x[:] = [[0.1, 0.2], [0.3, 0.4]]
    ps1.v[:] = [[0.5, 0.6], [0.7, 0.8]]
    ps1.rho[:] = 1800.0
    ps1.stress[:] = [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]
    ps1.strain_rate[:] = [[0.1, 0.2, 0.3], [0.4, 0.5, 0.6]]
    path = tmp_path / "out.npz"
    write_h5(ps1, path)
    ps_new = system_from_h5(G.StressParticleSystem, path, "stress1")
    assert ps_new.n == 2 and ps_new.stress.shape == (2, 3)
    assert (ps_new.mass, ps_new.c) == (1.2, 5.0)
    for name in ("x", "v", "rho", "stress", "strain_rate"):
        np.testing.assert_allclose(getattr(ps_new, name), getattr(ps1, name))


def test_read_h5_catches_mismatch_errors(tmp_path):
    ps1 = G.BasicParticleSystem("test1", 3, 2, 1.5, 2.0)
    path = tmp_path / "out.npz"
    write_h5(ps1, path)
    with pytest.raises(G.ArgumentError):
        read_h5(G.BasicParticleSystem("wrong_n", 4, 2, 1.0, 1.0), path)
    with pytest.raises(G.ArgumentError):
        read_h5(G.BasicParticleSystem("wrong_ndims", 3, 3, 1.0, 1.0), path)
