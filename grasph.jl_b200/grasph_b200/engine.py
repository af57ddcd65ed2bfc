"""Drive libgrasph_cuda.so from the host mirror of Grasph.jl's API.

`compile_instance` walks a LeapFrogTimeIntegrator (systems, ghost entries,
interactions, updaters) and issues the C-ABI model-building calls — the same
sequence the Julia `ccall` binding (julia/GrasphCUDA.jl) issues.  `Device` owns one
context; `time_integrate` is the drop-in for
`time_integrate!(::LeapFrogTimeIntegrator, ...)` (src/TimeIntegration.jl:580).

There is no CPU fallback: if the shared library is missing or the context
cannot be created, every call raises.
"""
from __future__ import annotations

import ctypes as ct
import os
import time
from pathlib import Path

import numpy as np

from . import consts as C
from .model import (AbstractBoundarySystem, AbstractParticleSystem, ArgumentError,
                    GhostEntry, GhostParticleSystem, LeapFrogTimeIntegrator,
                    SystemInteraction, VirtualParticleSystem, ProbeParticleSystem, updater_chains, _pfn_kind,
                    _pfn_params)

PKG_DIR = Path(__file__).resolve().parents[1]
LIB_PATH = PKG_DIR / "libgrasph_cuda.so"

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)
_i64p = ct.POINTER(ct.c_int64)
_i32p = ct.POINTER(ct.c_int32)


class GcError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{C.STATUS_NAMES.get(status, status)}: {msg}")


class FieldIO(ct.Structure):
    _fields_ = [("inst", ct.c_int), ("handle", ct.c_int), ("field", ct.c_int), ("pad", ct.c_int32),
                ("host", ct.c_void_p), ("bytes", ct.c_size_t)]


class GcStats(ct.Structure):
    _fields_ = [("steps_done", ct.c_int64), ("pairs_last_step", ct.c_int64),
                ("grid_inconsistent", ct.c_int64), ("kernel_launches", ct.c_int64),
                ("sweep_launches", ct.c_int64), ("sweep_ms", ct.c_double),
                ("last_status", ct.c_int32), ("pad", ct.c_int32),
                ("graph_steps", ct.c_int64), ("rollbacks", ct.c_int64),
                ("sweep_cfg_chosen", ct.c_int32 * 4), ("sorts_in_order", ct.c_int64)]


_LIB = None


def load_library(path: os.PathLike | None = None):
    """Load libgrasph_cuda.so (built in-tree by __graft_entry__.build())."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is not built; run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ct.CDLL(str(p))
    sig = {
        "gc_ctx_create": (ct.c_int, [ct.c_int, ct.c_size_t, ct.POINTER(ct.c_void_p)]),
        "gc_ctx_destroy": (ct.c_int, [ct.c_void_p]),
        "gc_last_error": (ct.c_char_p, [ct.c_void_p]),
        "gc_status_string": (ct.c_char_p, [ct.c_int]),
        "gc_instance_add": (ct.c_int, [ct.c_void_p, _ip]),
        "gc_add_system": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int64, ct.c_int, ct.c_int,
                                     ct.c_double, ct.c_double, _dp, ct.c_double, _ip]),
        "gc_add_boundary": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, _dp, _dp, ct.c_double, _ip]),
        "gc_add_ghost": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, _ip, _ip, _ip, ct.c_int,
                                    _dp, _dp, ct.c_double, ct.c_int64, _ip]),
        "gc_add_interaction": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_double,
                                          ct.c_int, _ip, _dp, _ip]),
        "gc_set_updaters": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, _ip, _ip, _dp]),
        "gc_set_integrator": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double]),
        "gc_set_integrator_kind": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
        "gc_set_velocity_adjust": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_double]),
        "gc_add_virtual": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, _dp, _ip]),
        "gc_add_probe": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int64, ct.c_int, _dp, ct.c_int, ct.c_int, ct.c_int,
                                    _dp, _ip]),
        "gc_add_probe_interaction": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_double,
                                                ct.c_int, _dp, _ip]),
        "gc_measure_probes": (ct.c_int, [ct.c_void_p]),
        "gc_finalize": (ct.c_int, [ct.c_void_p]),
        "gc_upload_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
        "gc_download_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
        "gc_get_count": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _i64p]),
        "gc_set_precision": (ct.c_int, [ct.c_void_p, ct.c_int]),
        "gc_step": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double]),
        "gc_get_stats": (ct.c_int, [ct.c_void_p, ct.POINTER(GcStats)]),
        "gc_sort_system": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double, _i64p]),
        "gc_build_grid": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _i64p, ct.c_int64, _dp, _i64p, _i64p]),
        "gc_generate_ghosts": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
        "gc_update_ghost_kinematics": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
        "gc_update_ghost": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int]),
        "gc_sweep": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int]),
        "gc_update_state": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_double]),
        "gc_neighbor_counts": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _i32p, ct.c_int64]),
        "gc_stream": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_void_p)]),
        "gc_set_profiling": (ct.c_int, [ct.c_void_p, ct.c_int]),
        "gc_measure_fp64_peak": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_double)]),
        "gc_measure_fp32_peak": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_double)]),
        "gc_set_graphs": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double]),
        "gc_set_sweep_config": (ct.c_int, [ct.c_void_p, ct.c_int]),
        "gc_upload_fields": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p]),
        "gc_download_fields": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p]),
        "gc_stage_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
        "gc_serve_create": (ct.c_int, [ct.c_int, ct.c_size_t, ct.c_int, ct.c_int, ct.POINTER(ct.c_void_p)]),
        "gc_serve_destroy": (ct.c_int, [ct.c_void_p]),
        "gc_serve_last_error": (ct.c_char_p, [ct.c_void_p]),
        "gc_serve_submit": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_double, _i64p]),
        "gc_serve_pump": (ct.c_int, [ct.c_void_p, _ip]),
        "gc_serve_poll": (ct.c_int, [ct.c_void_p, ct.c_int64, _ip, _i64p, _dp, _dp, _dp]),
        "gc_serve_download": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
        "gc_serve_release": (ct.c_int, [ct.c_void_p, ct.c_int64]),
        "gc_serve_get_stats": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def _arr(a, dtype, ptr):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(ptr)


class CudaBackend:
    """C-ABI calls on one libgrasph_cuda.so context."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, lib=None):
        self.lib = lib or load_library()
        self.ctx = ct.c_void_p()
        self._chk(self.lib.gc_ctx_create(device, hbm_budget, ct.byref(self.ctx)), where="gc_ctx_create")

    # -- plumbing
    def _chk(self, st, where=""):
        if st != 0:
            msg = ""
            if self.ctx:
                msg = (self.lib.gc_last_error(self.ctx) or b"").decode()
            raise GcError(st, f"{where}: {msg}")

    def close(self):
        if self.ctx:
            self.lib.gc_ctx_destroy(self.ctx)
            self.ctx = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- model building
    def instance_add(self):
        out = ct.c_int()
        self._chk(self.lib.gc_instance_add(self.ctx, ct.byref(out)), "gc_instance_add")
        return out.value

    def add_system(self, inst, kind, n, nd, ns, mass, c, source_v, source_rho):
        sv, svp = _arr(source_v, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_system(self.ctx, inst, kind, n, nd, ns, mass, c, svp, source_rho,
                                         ct.byref(out)), "gc_add_system")
        return out.value

    def add_boundary(self, inst, sys, kind, normal, point, beta_or_lj):
        nrm, np_ = _arr(normal, np.float64, _dp)
        pt, pp = _arr(point, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_boundary(self.ctx, inst, sys, kind, np_, pp, beta_or_lj, ct.byref(out)),
                  "gc_add_boundary")
        return out.value

    def add_ghost(self, inst, src, copiers, normals, points, cutoff, capacity):
        nf = np.array([len(c) for c in copiers] or [0], dtype=np.int32)
        flds = np.array([f for c in copiers for f, _ in c] or [0], dtype=np.int32)
        mds = np.array([m for c in copiers for _, m in c] or [0], dtype=np.int32)
        nrm, nrmp = _arr(normals, np.float64, _dp)
        pts, ptsp = _arr(points, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_ghost(self.ctx, inst, src, len(copiers), nf.ctypes.data_as(_ip),
                                        flds.ctypes.data_as(_ip), mds.ctypes.data_as(_ip), nrm.shape[0],
                                        nrmp, ptsp, cutoff, capacity, ct.byref(out)), "gc_add_ghost")
        return out.value

    def add_interaction(self, inst, a, b, kernel_kind, h, pfn_kinds, pfn_params):
        k = np.asarray(pfn_kinds, dtype=np.int32)
        p, pp = _arr(pfn_params, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_interaction(self.ctx, inst, a, b, kernel_kind, h, len(k),
                                              k.ctypes.data_as(_ip), pp, ct.byref(out)), "gc_add_interaction")
        return out.value

    def set_velocity_adjust(self, inst, inter, kind, epsilon):
        self._chk(self.lib.gc_set_velocity_adjust(self.ctx, inst, inter, kind, epsilon), "gc_set_velocity_adjust")

    def add_virtual(self, inst, src, zero_mask, prescribed_v):
        pv, pvp = _arr(prescribed_v, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_virtual(self.ctx, inst, src, zero_mask, pvp, ct.byref(out)), "gc_add_virtual")
        return out.value

    def add_probe(self, inst, n, nd, positions, mirror, extras_mask, ns, prescribed_v):
        pos, posp = (None, None) if positions is None else _arr(positions, np.float64, _dp)
        pv, pvp = _arr(prescribed_v, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_probe(self.ctx, inst, n, nd, posp, mirror, extras_mask, ns, pvp, ct.byref(out)),
                  "gc_add_probe")
        return out.value

    def add_probe_interaction(self, inst, a, probe, kernel_kind, h, pfn_kind, pfn_params):
        p, pp = _arr(pfn_params, np.float64, _dp)
        out = ct.c_int()
        self._chk(self.lib.gc_add_probe_interaction(self.ctx, inst, a, probe, kernel_kind, h, pfn_kind, pp,
                                                    ct.byref(out)), "gc_add_probe_interaction")
        return out.value

    def measure_probes(self):
        self._chk(self.lib.gc_measure_probes(self.ctx), "gc_measure_probes")

    def set_updaters(self, inst, sys, chains):
        cl = np.array([len(c) for c in chains] or [0], dtype=np.int32)
        kinds = np.array([k for c in chains for k, _ in c] or [0], dtype=np.int32)
        prm = np.array([p for c in chains for _, p in c] or [np.zeros(C.GC_UPD_NPARAM)], dtype=np.float64)
        self._chk(self.lib.gc_set_updaters(self.ctx, inst, sys, len(chains), cl.ctypes.data_as(_ip),
                                           kinds.ctypes.data_as(_ip), prm.ctypes.data_as(_dp)),
                  "gc_set_updaters")

    def set_integrator(self, inst, gamma):
        self._chk(self.lib.gc_set_integrator(self.ctx, inst, gamma), "gc_set_integrator")

    def set_integrator_kind(self, inst, kind):
        self._chk(self.lib.gc_set_integrator_kind(self.ctx, inst, kind), "gc_set_integrator_kind")

    def finalize(self):
        self._chk(self.lib.gc_finalize(self.ctx), "gc_finalize")

    # -- state
    def stage(self, inst, handle, field, array):
        a = np.ascontiguousarray(array)
        self._chk(self.lib.gc_stage_field(self.ctx, inst, handle, field, a.ctypes.data, a.nbytes),
                  "gc_stage_field")

    def upload(self, inst, handle, field, array):
        a = np.ascontiguousarray(array)
        self._chk(self.lib.gc_upload_field(self.ctx, inst, handle, field, a.ctypes.data, a.nbytes),
                  "gc_upload_field")

    def upload_many(self, items):
        """items: (inst, handle, field, array) tuples; one device synchronisation."""
        keep = [np.ascontiguousarray(a) for *_, a in items]
        arr = (FieldIO * max(len(items), 1))()
        for q, ((inst, h, f, _), a) in enumerate(zip(items, keep)):
            arr[q] = FieldIO(inst, h, f, 0, a.ctypes.data, a.nbytes)
        self._chk(self.lib.gc_upload_fields(self.ctx, len(items), arr), "gc_upload_fields")

    def download_many(self, items):
        """items: (inst, handle, field, out_array) tuples, filled in place."""
        arr = (FieldIO * max(len(items), 1))()
        for q, (inst, h, f, a) in enumerate(items):
            assert a.flags["C_CONTIGUOUS"]
            arr[q] = FieldIO(inst, h, f, 0, a.ctypes.data, a.nbytes)
        self._chk(self.lib.gc_download_fields(self.ctx, len(items), arr), "gc_download_fields")

    def download_into(self, inst, handle, field, out):
        self._chk(self.lib.gc_download_field(self.ctx, inst, handle, field, out.ctypes.data, out.nbytes),
                  "gc_download_field")
        return out

    def count(self, inst, handle):
        n = ct.c_int64()
        self._chk(self.lib.gc_get_count(self.ctx, inst, handle, ct.byref(n)), "gc_get_count")
        return n.value

    def set_precision(self, mode):
        self._chk(self.lib.gc_set_precision(self.ctx, mode), "gc_set_precision")

    def set_profiling(self, on):
        """Time every sweep launch with CUDA events (gc_stats.sweep_ms)."""
        self._chk(self.lib.gc_set_profiling(self.ctx, 1 if on else 0), "gc_set_profiling")

    def set_graphs(self, on, sync_every=32, cap_margin=0.0):
        self._chk(self.lib.gc_set_graphs(self.ctx, 1 if on else 0, sync_every, cap_margin), "gc_set_graphs")

    def set_sweep_config(self, cfg):
        self._chk(self.lib.gc_set_sweep_config(self.ctx, cfg), "gc_set_sweep_config")

    def step(self, nsteps, cfl):
        self._chk(self.lib.gc_step(self.ctx, nsteps, cfl), "gc_step")

    def stats(self):
        s = GcStats()
        self._chk(self.lib.gc_get_stats(self.ctx, ct.byref(s)), "gc_get_stats")
        out = {f: getattr(s, f) for f, _ in GcStats._fields_ if f != "pad"}
        out["sweep_cfg_chosen"] = list(s.sweep_cfg_chosen)
        return out

    # -- phase hooks
    def sort(self, inst, handle, cutoff, n):
        perm = np.zeros(n, dtype=np.int64)
        self._chk(self.lib.gc_sort_system(self.ctx, inst, handle, cutoff, perm.ctypes.data_as(_i64p)),
                  "gc_sort_system")
        return perm

    def build_grid(self, inst, inter, nd):
        ming = np.zeros(nd)
        ng = np.zeros(nd, dtype=np.int64)
        ncells = ct.c_int64()
        self._chk(self.lib.gc_build_grid(self.ctx, inst, inter, None, 0, ming.ctypes.data_as(_dp),
                                         ng.ctypes.data_as(_i64p), ct.byref(ncells)), "gc_build_grid")
        cs = np.zeros(ncells.value + 1, dtype=np.int64)
        self._chk(self.lib.gc_build_grid(self.ctx, inst, inter, cs.ctypes.data_as(_i64p), cs.size, None,
                                         None, None), "gc_build_grid")
        return cs, ming, ng

    def generate_ghosts(self, inst, ghost):
        self._chk(self.lib.gc_generate_ghosts(self.ctx, inst, ghost), "gc_generate_ghosts")

    def update_ghost_kinematics(self, inst, ghost):
        self._chk(self.lib.gc_update_ghost_kinematics(self.ctx, inst, ghost), "gc_update_ghost_kinematics")

    def update_ghost(self, inst, ghost, stage):
        self._chk(self.lib.gc_update_ghost(self.ctx, inst, ghost, stage), "gc_update_ghost")

    def sweep(self, inst, inter, stage):
        self._chk(self.lib.gc_sweep(self.ctx, inst, inter, stage), "gc_sweep")

    def update_state(self, inst, sys, stage, dt):
        self._chk(self.lib.gc_update_state(self.ctx, inst, sys, stage, dt), "gc_update_state")

    def neighbor_counts(self, inst, inter, n):
        out = np.zeros(n, dtype=np.int32)
        self._chk(self.lib.gc_neighbor_counts(self.ctx, inst, inter, out.ctypes.data_as(_i32p), n),
                  "gc_neighbor_counts")
        return out


# ------------------------------------------------------------ compilation

class InstanceMap:
    """Object → handle map of one compiled instance."""

    def __init__(self, inst):
        self.inst = inst
        self.handles = {}
        self.inters = {}
        self.systems = []
        self.ghosts = []
        self.virtuals = []
        self.probes = []

    def h(self, obj):
        return self.handles[id(obj)]


def compile_instance(backend, inst, systems, interactions, ghosts=(), gamma=0.0,
                     kind=C.GC_INTEGRATOR_LEAPFROG, virtuals=(), probes=(), probe_interactions=()) -> InstanceMap:
    """Issue the model-building calls for one simulation (one instance)."""
    m = InstanceMap(inst)
    sys_ids = {id(ps) for ps in systems}
    for ps in systems:
        if not isinstance(ps, AbstractParticleSystem):
            raise ArgumentError("systems must be particle systems (wrap boundaries only as system_b)")
        m.handles[id(ps)] = backend.add_system(inst, ps.kind, ps.n, ps.ndims, ps.ns, ps.mass, ps.c,
                                               ps.source_v, ps.source_rho)
        m.systems.append(ps)
    for vps in virtuals:
        src = vps.source
        if id(src) in sys_ids:
            raise ArgumentError("a virtual system's source must not be one of the integrator's systems")
        if id(src) not in m.handles:
            # the source is a slot of its own: moved with the state, never integrated
            m.handles[id(src)] = backend.add_system(inst, src.kind, src.n, src.ndims, src.ns, src.mass, src.c,
                                                    src.source_v, src.source_rho)
            m.systems.append(src)
        m.handles[id(vps)] = backend.add_virtual(inst, m.h(src), vps.zero_mask, vps.prescribed_v)
        m.virtuals.append(vps)
        chains = updater_chains(vps)
        if chains:
            backend.set_updaters(inst, m.h(vps), chains)
    for ge in ghosts:
        g = ge.ghost
        if id(g.source) not in sys_ids:
            raise ArgumentError("a ghost's source system must be in the integrator's systems")
        copiers = []
        for u in g.updaters:
            copiers.append([] if u is None else
                           [({"p": C.GC_FIELD_P, "stress": C.GC_FIELD_STRESS, "rho": C.GC_FIELD_RHO}[f], md)
                            for f, md in u.entries])
        hnd = backend.add_ghost(inst, m.h(g.source), copiers, ge.normals, ge.points, ge.cutoff, ge.capacity)
        m.handles[id(g)] = hnd
        m.handles[id(ge)] = hnd
        m.ghosts.append(ge)
    for it in interactions:
        a = it.system_a
        if isinstance(a, GhostParticleSystem):
            # InterpolateFieldFn from the ghosts' current arrays (Trapdoor.jl's ghost_bottom)
            if id(a) not in m.handles:
                raise ArgumentError("a ghost used as system_a must belong to a GhostEntry in `ghosts`")
        elif id(a) not in sys_ids:
            raise ArgumentError("system_a must be in the integrator's systems")
        b = it.system_b
        if b is None:
            bh = -1
        elif isinstance(b, AbstractBoundarySystem):
            if id(b) not in m.handles:
                if id(b.inner) not in sys_ids:
                    raise ArgumentError("a boundary's inner system must be in the integrator's systems")
                if b.wrap_kind == C.GC_WRAP_DYNAMIC:
                    m.handles[id(b)] = backend.add_boundary(inst, m.h(b.inner), b.wrap_kind, b.boundary_normal,
                                                            b.boundary_point, b.boundary_beta)
                else:
                    nd = b.inner.ndims
                    m.handles[id(b)] = backend.add_boundary(inst, m.h(b.inner), b.wrap_kind, np.zeros(nd),
                                                            np.zeros(nd), b.lj_cutoff)
            bh = m.h(b)
        elif isinstance(b, GhostParticleSystem):
            if id(b) not in m.handles:
                raise ArgumentError("a ghost used as system_b must belong to a GhostEntry in `ghosts`")
            bh = m.h(b)
        elif isinstance(b, VirtualParticleSystem):
            if id(b) not in m.handles:
                raise ArgumentError("a virtual system used as system_b must be in `virtual_systems`")
            bh = m.h(b)
        else:
            if id(b) not in sys_ids:
                raise ArgumentError("system_b must be in the integrator's systems")
            bh = m.h(b)
        kinds = [_pfn_kind(p) for p in it.pfns]
        params = np.array([_pfn_params(p) for p in it.pfns], dtype=np.float64)
        m.inters[id(it)] = backend.add_interaction(inst, m.h(a), bh, it.kernel.kind, it.kernel.h, kinds, params)
        if getattr(it, "vadjust_pfn", None) is not None:
            backend.set_velocity_adjust(inst, m.inters[id(it)], it.vadjust_pfn.kind, it.vadjust_pfn.epsilon)
    for pr in probes:
        mh = -1
        if pr.mirror_target is not None:
            if id(pr.mirror_target) not in m.handles:
                raise ArgumentError("a probe's mirror target must be one of the systems")
            mh = m.h(pr.mirror_target)
        m.handles[id(pr)] = backend.add_probe(inst, pr.n, pr.ndims, pr.x, mh, pr.extras_mask, pr.ns,
                                              pr.prescribed_v)
        m.probes.append(pr)
        chains = updater_chains(pr)
        if chains:
            backend.set_updaters(inst, m.h(pr), chains)
    for it in probe_interactions:
        if id(it.system_a) not in sys_ids:
            raise ArgumentError("system_a must be in the integrator's systems")
        pf = it.pfns[0]
        if len(it.pfns) != 1 or pf is None:
            raise ArgumentError("a probe interaction takes one functor")
        m.inters[id(it)] = backend.add_probe_interaction(inst, m.h(it.system_a), m.h(it.system_b), it.kernel.kind,
                                                         it.kernel.h, _pfn_kind(pf), _pfn_params(pf))
    for ps in systems:
        chains = updater_chains(ps)
        if chains:
            backend.set_updaters(inst, m.h(ps), chains)
    backend.set_integrator(inst, gamma)
    if kind != C.GC_INTEGRATOR_LEAPFROG:
        backend.set_integrator_kind(inst, kind)
    return m


def _wide(a):
    """A Float32 field widened to the Float64 the library transfers."""
    return a.astype(np.float64) if a.dtype == np.float32 else a


def upload_instance(backend, m: InstanceMap, systems=None):
    items = [(m.inst, m.h(ps), fid, _wide(getattr(ps, name)))
             for ps in m.systems if systems is None or any(ps is q for q in systems)
             for name, fid in ps.particle_fields()]
    if hasattr(backend, "upload_many"):
        backend.upload_many(items)
    else:
        for inst, h, fid, a in items:
            backend.upload(inst, h, fid, a)


def download_instance(backend, m: InstanceMap, with_ghosts=True, systems=None):
    items, narrow = [], []
    for ps in m.systems:
        if systems is not None and not any(ps is q for q in systems):
            continue
        for name, fid in ps.particle_fields():
            a = getattr(ps, name)
            if a.dtype == np.float32:
                # downloaded in Float64, rounded to the system's Float32
                w = np.empty(a.shape)
                narrow.append((a, w))
                a = w
            items.append((m.inst, m.h(ps), fid, a))
    if hasattr(backend, "download_many"):
        backend.download_many(items)
    else:
        for inst, h, fid, a in items:
            backend.download_into(inst, h, fid, a)
    for a, w in narrow:
        a[...] = w
    if with_ghosts:
        for ge in m.ghosts:
            download_ghost(backend, m, ge)
        for vps in m.virtuals:
            backend.download_into(m.inst, m.h(vps), C.GC_FIELD_W_SUM, vps.w_sum)
        for pr in m.probes:
            download_probe(backend, m, pr)


def download_probe(backend, m: InstanceMap, pr):
    h = m.h(pr)
    backend.download_into(m.inst, h, C.GC_FIELD_X, pr.x)
    backend.download_into(m.inst, h, C.GC_FIELD_ID, pr.id)
    backend.download_into(m.inst, h, C.GC_FIELD_W_SUM, pr.w_sum)
    for k, arr in pr.extras.items():
        if k == pr.count_field:
            buf = np.zeros(pr.n)
            backend.download_into(m.inst, h, C.GC_FIELD_COUNT, buf)
            arr[:] = np.rint(buf).astype(np.int64)
        else:
            buf = np.zeros(arr.shape)
            backend.download_into(m.inst, h, ProbeParticleSystem._fields[k], buf)
            arr[:] = buf


def download_ghost(backend, m: InstanceMap, ge: GhostEntry):
    g = ge.ghost
    h = m.h(g)
    n = backend.count(m.inst, h)
    nd = g.ndims
    g.x = backend.download_into(m.inst, h, C.GC_FIELD_X, np.zeros((n, nd)))
    g.v = backend.download_into(m.inst, h, C.GC_FIELD_V, np.zeros((n, nd)))
    g.rho = backend.download_into(m.inst, h, C.GC_FIELD_RHO, np.zeros(n))
    g.idx_original = backend.download_into(m.inst, h, C.GC_FIELD_IDX_ORIGINAL, np.zeros(n, dtype=np.int64))
    g.idx_boundary = backend.download_into(m.inst, h, C.GC_FIELD_IDX_BOUNDARY, np.zeros(n, dtype=np.int64))
    g.normals = backend.download_into(m.inst, h, C.GC_FIELD_NORMALS, np.zeros((n, nd)))
    T = g.source.dtype
    if T != np.float64:
        g.x, g.v, g.rho, g.normals = (a.astype(T) for a in (g.x, g.v, g.rho, g.normals))
    for f in g.extras_fields:
        if f == "p":
            g.extras["p"] = backend.download_into(m.inst, h, C.GC_FIELD_P, np.zeros(n))
        elif f == "stress":
            g.extras["stress"] = backend.download_into(m.inst, h, C.GC_FIELD_STRESS,
                                                       np.zeros((n, g.source.ns)))


# --------------------------------------------------------------- sessions

class Session:
    """A device context holding one or more simulations (instances).

    ``Session([lf])`` is the single-rank drop-in; ``Session([lf1, lf2, ...])``
    packs independent simulations of one model structure into one context
    (batched stepping).  Per-phase methods mirror the reference's
    per-phase entry points for a single instance.
    """

    def __init__(self, integrators, *, device=0, precision=C.GC_PRECISION_FP64, hbm_budget=0,
                 backend=None):
        if isinstance(integrators, LeapFrogTimeIntegrator):
            integrators = [integrators]
        self.integrators = list(integrators)
        self.backend = backend or CudaBackend(device, hbm_budget)
        self.maps = []
        for lf in self.integrators:
            inst = self.backend.instance_add()
            self.maps.append(compile_instance(self.backend, inst, lf.systems, lf.interactions, lf.ghosts,
                                              lf.gamma, lf.kind, getattr(lf, "virtual_systems", ()),
                                              getattr(lf, "probes", ()), getattr(lf, "probe_interactions", ())))
        self.backend.finalize()
        self.backend.set_precision(precision)
        self.precision = precision
        # the global step of the loaded restart (_load_restart!'s return,
        # from which the reference's loop continues global_step)
        self.step_offset = 0

    # -- state transfer
    def push(self, systems=None):
        """Upload every field of every system (or of `systems` only)."""
        for m in self.maps:
            upload_instance(self.backend, m, systems)

    def pull(self, with_ghosts=True, systems=None):
        """Download every field of every system (or of `systems` only)."""
        for m in self.maps:
            download_instance(self.backend, m, with_ghosts, systems)

    def step(self, nsteps, cfl):
        self.backend.step(nsteps, cfl)

    def measure_probes(self, pull=True):
        """_measure_probes! (src/TimeIntegration.jl:454-502), then the probes'
        x, id, w_sum and extras downloaded in probe order."""
        self.backend.measure_probes()
        if pull:
            for m in self.maps:
                for pr in m.probes:
                    download_probe(self.backend, m, pr)

    def stats(self):
        return self.backend.stats()

    # -- snapshots and restarts (grasph_b200.snapshot: write_h5 / read_h5!'s layout)
    def save(self, path, inst=0):
        """_maybe_save! (src/TimeIntegration.jl:520-549) of one instance: its
        state downloaded and written to `path` with the step count."""
        from .snapshot import write_snapshot
        m = self._m(inst)
        download_instance(self.backend, m)
        write_snapshot(m.systems, path, step=self.step_offset + self.stats()["steps_done"],
                       probes=[pr for pr in m.probes if pr.mirror_target is None])

    def load(self, path, inst=0):
        """_load_restart! (src/Driver.jl:79-96) of one instance: `path` read
        into its systems (and free probes' positions) and uploaded; returns
        the saved step."""
        from .snapshot import read_snapshot
        m = self._m(inst)
        free = [pr for pr in m.probes if pr.mirror_target is None]
        step = read_snapshot(m.systems, path, probes=free)
        upload_instance(self.backend, m)
        for pr in free:
            self.backend.upload(m.inst, m.h(pr), C.GC_FIELD_X, pr.x)
        # later saves count from the restart's step
        self.step_offset = step - self.stats()["steps_done"]
        return step

    # -- per-phase hooks (instance 0 unless given)
    def _m(self, inst):
        return self.maps[inst]

    def sort_particles(self, ps, cutoff, inst=0):
        m = self._m(inst)
        n = ps.n if not isinstance(ps, GhostParticleSystem) else self.backend.count(m.inst, m.h(ps))
        return self.backend.sort(m.inst, m.h(ps), cutoff, n)

    def create_grid(self, si, inst=0):
        m = self._m(inst)
        return self.backend.build_grid(m.inst, m.inters[id(si)], si.ndims)

    def generate_ghosts(self, ge, inst=0):
        m = self._m(inst)
        self.backend.generate_ghosts(m.inst, m.h(ge))

    def update_ghost_kinematics(self, ge, inst=0):
        m = self._m(inst)
        self.backend.update_ghost_kinematics(m.inst, m.h(ge))

    def update_ghost(self, ge, stage, inst=0):
        m = self._m(inst)
        self.backend.update_ghost(m.inst, m.h(ge), stage)

    def sweep(self, si, stage=1, inst=0):
        m = self._m(inst)
        self.backend.sweep(m.inst, m.inters[id(si)], stage)

    def update_state(self, ps, stage=1, dt=0.0, inst=0):
        m = self._m(inst)
        self.backend.update_state(m.inst, m.h(ps), stage, dt)

    def neighbor_counts(self, si, inst=0):
        m = self._m(inst)
        return self.backend.neighbor_counts(m.inst, m.inters[id(si)], si.system_a.n)

    def pull_ghost(self, ge, inst=0):
        download_ghost(self.backend, self._m(inst), ge)

    def close(self):
        self.backend.close()


def _summary(ps):
    rows = []
    for name in ("v", "rho", "p", "stress"):
        if hasattr(ps, name):
            a = np.asarray(getattr(ps, name))
            rows.append(f"  {name:8s} min {a.min():.6g}  mean {a.mean():.6g}  max {a.max():.6g}")
    return "\n".join(rows)


def time_integrate(integrator: LeapFrogTimeIntegrator, num_timesteps: int, print_interval_step: int,
                   save_interval_step: int, CFL: float, output_prefix=None, *, step_offset: int = 0,
                   output_width=None, print_timer: bool = False, precision=C.GC_PRECISION_FP64,
                   verbose: bool = False):
    """Drop-in for ``time_integrate!`` (src/TimeIntegration.jl:580-697).

    Host arrays are uploaded at entry and written back at exit (and at each
    print/save boundary); all steps in between run on the device.  Snapshots
    go to ``{prefix}_{step}.npz`` (the reference writes HDF5).
    Returns a dict of wall-clock phase timings (the TimerOutputs stand-in).
    """
    t0 = time.perf_counter()
    sess = integrator._device
    if sess is None or sess.precision != precision:
        sess = Session([integrator], precision=precision)
        integrator._device = sess
    sess.push()
    t_up = time.perf_counter()
    width = output_width if output_width is not None else len(str(step_offset + num_timesteps))
    done = 0
    while done < num_timesteps:
        g = step_offset + done
        nxt = num_timesteps - done
        for interval in (print_interval_step, save_interval_step if output_prefix is not None else 0):
            if interval and interval > 0:
                nxt = min(nxt, interval - (g % interval))
        sess.step(nxt, CFL)
        done += nxt
        g = step_offset + done
        boundary_print = verbose and print_interval_step > 0 and g % print_interval_step == 0
        boundary_save = output_prefix is not None and save_interval_step > 0 and g % save_interval_step == 0
        if boundary_print or boundary_save:
            sess.pull()
            if boundary_print:
                print(f"\nStep {g}")
                for ps in integrator.systems:
                    print(ps.name)
                    print(_summary(ps))
            if boundary_save:
                path = f"{output_prefix}_{str(g).zfill(width)}.npz"
                d = os.path.dirname(path)
                if d:
                    os.makedirs(d, exist_ok=True)
                arrays = {}
                for ps in integrator.systems:
                    for name, _ in ps.particle_fields():
                        arrays[f"{ps.name}/{name}"] = getattr(ps, name)
                np.savez(path, step=g, **arrays)
    t_run = time.perf_counter()
    sess.pull()
    t_down = time.perf_counter()
    timer = {"upload_s": t_up - t0, "steps_s": t_run - t_up, "download_s": t_down - t_run,
             "steps": num_timesteps}
    if print_timer:
        print(timer)
    return timer


# ---------------------------------------------------------------- serving

class ServeStats(ct.Structure):
    _fields_ = [("queued", ct.c_int64), ("running", ct.c_int64), ("batches", ct.c_int64),
                ("rounds", ct.c_int64), ("repacks", ct.c_int64), ("particle_steps", ct.c_int64),
                ("device_bytes_reserved", ct.c_int64), ("repack_seconds", ct.c_double),
                ("repack_instances", ct.c_int64), ("retries", ct.c_int64)]


class Server:
    """Many simulations on one device (gc_serve_*): submit integrators at any
    time, pump rounds, fetch each result when its request is done.

    Simulations of one model structure share a packed context and step
    together; a result is bit-identical to the same simulation run alone in
    a Session of the same precision.
    """

    QUEUED, RUNNING, DONE, FAILED = C.GC_REQ_QUEUED, C.GC_REQ_RUNNING, C.GC_REQ_DONE, C.GC_REQ_FAILED

    def __init__(self, *, device=0, hbm_budget=150 * 10**9, round_steps=50,
                 precision=C.GC_PRECISION_FP32_COMPENSATED, lib=None):
        self.lib = lib or load_library()
        self.srv = ct.c_void_p()
        self.device = device
        self._chk(self.lib.gc_serve_create(device, int(hbm_budget), round_steps, precision, ct.byref(self.srv)),
                  "gc_serve_create")
        self.maps = {}

    def _chk(self, st, where=""):
        if st != 0:
            msg = (self.lib.gc_serve_last_error(self.srv) or b"").decode() if self.srv else ""
            raise GcError(st, f"{where}: {msg}")

    def close(self):
        if self.srv:
            self.lib.gc_serve_destroy(self.srv)
            self.srv = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, lf: LeapFrogTimeIntegrator, nsteps: int, cfl: float) -> int:
        """Queue one simulation; its current host state is copied now."""
        be = CudaBackend(self.device, 0, lib=self.lib)
        inst = be.instance_add()
        m = compile_instance(be, inst, lf.systems, lf.interactions, lf.ghosts, lf.gamma, lf.kind,
                             getattr(lf, "virtual_systems", ()), getattr(lf, "probes", ()),
                             getattr(lf, "probe_interactions", ()))
        for ps in m.systems:
            h = m.h(ps)
            for name, fid in ps.particle_fields():
                be.stage(inst, h, fid, _wide(getattr(ps, name)))
        req = ct.c_int64()
        st = self.lib.gc_serve_submit(self.srv, be.ctx, nsteps, cfl, ct.byref(req))
        if st != 0:
            be.close()
            self._chk(st, "gc_serve_submit")
        be.ctx = ct.c_void_p()  # owned by the server now
        self.maps[req.value] = (lf, m)
        return req.value

    def pump(self) -> int:
        n = ct.c_int()
        self._chk(self.lib.gc_serve_pump(self.srv, ct.byref(n)), "gc_serve_pump")
        return n.value

    def poll(self, req):
        st, done = ct.c_int(), ct.c_int64()
        ts, ta, td = ct.c_double(), ct.c_double(), ct.c_double()
        self._chk(self.lib.gc_serve_poll(self.srv, req, ct.byref(st), ct.byref(done), ct.byref(ts), ct.byref(ta),
                                         ct.byref(td)), "gc_serve_poll")
        return {"state": st.value, "steps_done": done.value, "t_submit": ts.value, "t_admit": ta.value,
                "t_done": td.value}

    def fetch(self, req):
        """Write a finished request's fields into its integrator's arrays."""
        lf, m = self.maps[req]
        for ps in m.systems:
            h = m.h(ps)
            for name, fid in ps.particle_fields():
                a = getattr(ps, name)
                w = np.empty(a.shape) if a.dtype == np.float32 else a
                self._chk(self.lib.gc_serve_download(self.srv, req, h, fid, w.ctypes.data, w.nbytes),
                          "gc_serve_download")
                if w is not a:
                    a[...] = w
        return lf

    def release(self, req):
        self._chk(self.lib.gc_serve_release(self.srv, req), "gc_serve_release")
        self.maps.pop(req, None)

    def stats(self):
        s = ServeStats()
        self._chk(self.lib.gc_serve_get_stats(self.srv, ct.byref(s)), "gc_serve_get_stats")
        return {f: getattr(s, f) for f, _ in ServeStats._fields_}
