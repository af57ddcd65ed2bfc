"""Snapshots and restarts of device-resident state.

The reference writes one HDF5 group per particle system (`write_h5` /
`read_h5!`, src/Particles.jl:699-787): attributes `n`, `ndims`, `mass`, `c`,
the dataset `x` and the system's simulation fields; `_maybe_save!`
(src/TimeIntegration.jl:520-549) writes one such file per save step and
`_load_restart!` (src/Driver.jl:79-96) reads one back and continues from its
step.  No HDF5 library exists in this environment, so the same groups,
attributes and datasets are stored in a NumPy `.npz` container: key
`"<system>/<field>"` for a dataset and `"<system>/@<attr>"` for an attribute,
plus `"@step"` for the step the state belongs to.  Reading follows
`read_h5!`: the saved `n` and `ndims` must match the system
(`ArgumentError` otherwise) and only the arrays present in both are
updated.
"""
from __future__ import annotations

import warnings

import numpy as np

from .model import ArgumentError

__all__ = ["write_snapshot", "read_snapshot", "write_h5", "read_h5", "system_from_h5"]


def _systems_of(items):
    out = []
    for ps in items:
        if any(ps is q for q in out):
            continue
        out.append(ps)
    names = [ps.name for ps in out]
    if len(set(names)) != len(names):
        raise ArgumentError("systems in one snapshot need distinct names")
    return out


def _put_group(arrays, ps, prefix):
    """_write_to_group! (src/Particles.jl:720-734) under key prefix `prefix`."""
    arrays[f"{prefix}@n"] = np.int64(ps.n)
    arrays[f"{prefix}@ndims"] = np.int64(ps.ndims)
    arrays[f"{prefix}@mass"] = ps.dtype.type(ps.mass)
    arrays[f"{prefix}@c"] = ps.dtype.type(ps.c)
    for name, _ in ps.particle_fields():
        arrays[f"{prefix}{name}"] = np.asarray(getattr(ps, name))


def _get_group(f, ps, prefix):
    """_read_from_group! (src/Particles.jl:761-787): n and ndims checked,
    the arrays present in both read, mass and c left as they are."""
    _check_group(f, prefix, ps.n, ps.ndims)
    for name, _ in ps.particle_fields():
        key = f"{prefix}{name}"
        if key in f:
            getattr(ps, name)[...] = f[key]


def write_h5(ps, path):
    """write_h5(ps, path) (src/Particles.jl:711): one system at the file's
    root."""
    arrays = {}
    _put_group(arrays, ps, "")
    with open(path, "wb") as f:
        np.savez(f, **arrays)


def read_h5(ps, path):
    """read_h5!(ps, path) (src/Particles.jl:749): the file's root group into
    `ps` (its name need not match); returns `ps`."""
    with np.load(path) as f:
        _get_group(f, ps, "")
    return ps


def system_from_h5(cls, path, name, **kw):
    """The reference's path constructors (`FluidParticleSystem(path, name;
    kw...)` and the like): a new system of type `cls` sized and
    parameterised (n, ndims, mass, c, stress width) from the file's root
    group, its arrays read back."""
    with np.load(path) as f:
        n, nd = int(f["@n"]), int(f["@ndims"])
        mass, c = float(f["@mass"]), float(f["@c"])
        if getattr(cls, "has_stress", False):
            ps = cls(name, n, nd, int(f["stress"].shape[1]), mass, c, **kw)
        else:
            ps = cls(name, n, nd, mass, c, **kw)
        _get_group(f, ps, "")
    return ps


def write_snapshot(systems, path, step=None, probes=()):
    """Write every field of `systems` (and the positions and ids of
    `probes`) to `path`, one group per system as `_maybe_save!` lays it out."""
    arrays = {}
    for ps in _systems_of(systems):
        _put_group(arrays, ps, f"{ps.name}/")
    for pr in _systems_of(probes):
        g = pr.name
        arrays[f"{g}/@n"] = np.int64(pr.n)
        arrays[f"{g}/@ndims"] = np.int64(pr.ndims)
        arrays[f"{g}/x"] = np.asarray(pr.x)
        arrays[f"{g}/id"] = np.asarray(pr.id)
    if step is not None:
        arrays["@step"] = np.int64(step)
    with open(path, "wb") as f:
        np.savez(f, **arrays)


def _check_group(f, prefix, n, ndims):
    if f"{prefix}@n" not in f:
        raise ArgumentError(f"no saved group {prefix!r}")
    sn, snd = int(f[f"{prefix}@n"]), int(f[f"{prefix}@ndims"])
    if sn != n:
        raise ArgumentError(f"Saved particle count ({sn}) does not match system count ({n})")
    if snd != ndims:
        raise ArgumentError(f"Saved ndims ({snd}) does not match system ndims ({ndims})")


def read_snapshot(systems, path, probes=()):
    """Read `path` into `systems` (and `probes`) as `_load_restart!`
    (src/Driver.jl:79-96) does: a system or probe without a group in the
    file is left untouched with a warning, the others are read with
    `read_h5!`'s checks; returns the saved step, or 0 with a warning when
    the file holds none."""
    with np.load(path) as f:
        for ps in _systems_of(systems):
            if f"{ps.name}/@n" not in f:
                warnings.warn(f"Restart file {path} has no group for system {ps.name!r}; leaving it untouched")
                continue
            _get_group(f, ps, f"{ps.name}/")
        for pr in _systems_of(probes):
            g = pr.name
            if f"{g}/@n" not in f:
                warnings.warn(f"Restart file {path} has no group for probe {g!r}; leaving it untouched")
                continue
            _check_group(f, f"{g}/", pr.n, pr.ndims)
            pr.x[...] = f[f"{g}/x"]
            pr.id[...] = f[f"{g}/id"]
        if "@step" not in f:
            warnings.warn(f'Restart file {path} has no "step" attribute; assuming step 0')
            return 0
        return int(f["@step"])
