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

import numpy as np

from .model import ArgumentError

__all__ = ["write_snapshot", "read_snapshot"]


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


def write_snapshot(systems, path, step=None, probes=()):
    """Write every field of `systems` (and the positions and ids of
    `probes`) to `path`, one group per system as `write_h5` lays it out."""
    arrays = {}
    for ps in _systems_of(systems):
        g = ps.name
        arrays[f"{g}/@n"] = np.int64(ps.n)
        arrays[f"{g}/@ndims"] = np.int64(ps.ndims)
        arrays[f"{g}/@mass"] = np.float64(ps.mass)
        arrays[f"{g}/@c"] = np.float64(ps.c)
        for name, _ in ps.particle_fields():
            arrays[f"{g}/{name}"] = np.asarray(getattr(ps, name))
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


def _check_group(f, g, n, ndims):
    if f"{g}/@n" not in f:
        raise ArgumentError(f"no saved group for system {g!r}")
    sn, snd = int(f[f"{g}/@n"]), int(f[f"{g}/@ndims"])
    if sn != n:
        raise ArgumentError(f"Saved particle count ({sn}) does not match system count ({n})")
    if snd != ndims:
        raise ArgumentError(f"Saved ndims ({snd}) does not match system ndims ({ndims})")


def read_snapshot(systems, path, probes=()):
    """Read `path` into `systems` (and `probes`) as `read_h5!` does; returns
    the saved step, or None."""
    with np.load(path) as f:
        for ps in _systems_of(systems):
            g = ps.name
            _check_group(f, g, ps.n, ps.ndims)
            for name, _ in ps.particle_fields():
                key = f"{g}/{name}"
                if key in f:
                    getattr(ps, name)[...] = f[key]
        for pr in _systems_of(probes):
            g = pr.name
            _check_group(f, g, pr.n, pr.ndims)
            pr.x[...] = f[f"{g}/x"]
            pr.id[...] = f[f"{g}/id"]
        return int(f["@step"]) if "@step" in f else None
