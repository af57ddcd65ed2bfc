"""ctypes wrapper of liboracle.so — TEST INFRASTRUCTURE ONLY.

Exposes the CPU restatement of Grasph.jl's hot path with the same method
names as grasph_b200.engine.CudaBackend, so one model description can be
compiled into both and compared.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as ct
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)
_i64p = ct.POINTER(ct.c_int64)


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ct.CDLL(str(LIB))
        sig = {
            "oracle_create": (ct.c_int, [ct.POINTER(ct.c_void_p)]),
            "oracle_destroy": (ct.c_int, [ct.c_void_p]),
            "oracle_last_error": (ct.c_char_p, [ct.c_void_p]),
            "oracle_set_threads": (ct.c_int, [ct.c_void_p, ct.c_int]),
            "oracle_max_threads": (ct.c_int, []),
            "oracle_add_system": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int64, ct.c_int, ct.c_int, ct.c_double,
                                             ct.c_double, _dp, ct.c_double, _ip]),
            "oracle_add_boundary": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _dp, _dp, ct.c_double, _ip]),
            "oracle_add_ghost": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _ip, _ip, _ip, ct.c_int, _dp, _dp,
                                            ct.c_double, _ip]),
            "oracle_add_interaction": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_double,
                                                  ct.c_int, _ip, _dp, _ip]),
            "oracle_set_updaters": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _ip, _ip, _dp]),
            "oracle_set_integrator": (ct.c_int, [ct.c_void_p, ct.c_double]),
            "oracle_set_integrator_kind": (ct.c_int, [ct.c_void_p, ct.c_int]),
            "oracle_set_velocity_adjust": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double]),
            "oracle_add_virtual": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _dp, _ip]),
            "oracle_add_probe": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int, _dp, ct.c_int, ct.c_int, ct.c_int,
                                            _dp, _ip]),
            "oracle_add_probe_interaction": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_double,
                                                        ct.c_int, _dp, _ip]),
            "oracle_measure_probes": (ct.c_int, [ct.c_void_p]),
            "oracle_set_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
            "oracle_get_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
            "oracle_get_count": (ct.c_int, [ct.c_void_p, ct.c_int, _i64p]),
            "oracle_step": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double]),
            "oracle_sort_system": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double, _i64p]),
            "oracle_build_grid": (ct.c_int, [ct.c_void_p, ct.c_int, _i64p, ct.c_int64, _dp, _i64p, _i64p]),
            "oracle_grid_cell_start_a": (ct.c_int, [ct.c_void_p, ct.c_int, _i64p, ct.c_int64]),
            "oracle_generate_ghosts": (ct.c_int, [ct.c_void_p, ct.c_int]),
            "oracle_update_ghost_kinematics": (ct.c_int, [ct.c_void_p, ct.c_int]),
            "oracle_update_ghost": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
            "oracle_sweep": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
            "oracle_update_state": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double]),
            "oracle_kernel_norm": (ct.c_double, [ct.c_int, ct.c_int, ct.c_double]),
            "oracle_kernel_w": (ct.c_double, [ct.c_int, ct.c_int, ct.c_double, ct.c_double]),
            "oracle_kernel_dw_dq": (ct.c_double, [ct.c_int, ct.c_int, ct.c_double, ct.c_double]),
            "oracle_powi": (ct.c_double, [ct.c_double, ct.c_int64]),
            "oracle_steps": (ct.c_int64, [ct.c_void_p]),
            "oracle_set_track_magnitude": (ct.c_int, [ct.c_void_p, ct.c_int]),
            "oracle_get_magnitude": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_size_t]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"status {status}: {msg}")


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


class OracleBackend:
    """Same interface as CudaBackend; a single instance (inst must be 0)."""

    def __init__(self, threads: int = 1, track_magnitude=False):
        self.L = lib()
        self.ctx = ct.c_void_p()
        self.L.oracle_create(ct.byref(self.ctx))
        self.L.oracle_set_threads(self.ctx, threads)
        self._inst = 0
        # False/0: off; True/1: over the pair terms; 2: over the inputs
        self._track = int(track_magnitude)

    def _chk(self, st, where=""):
        if st != 0:
            raise OracleError(st, f"{where}: {self.L.oracle_last_error(self.ctx).decode()}")

    def close(self):
        if self.ctx:
            self.L.oracle_destroy(self.ctx)
            self.ctx = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n):
        self.L.oracle_set_threads(self.ctx, n)

    def instance_add(self):
        if self._inst:
            raise OracleError(1, "the oracle holds one simulation per backend")
        self._inst = 1
        return 0

    def add_system(self, inst, kind, n, nd, ns, mass, c, source_v, source_rho):
        sv = _a(source_v, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_system(self.ctx, kind, n, nd, ns, mass, c, sv.ctypes.data_as(_dp),
                                           source_rho, ct.byref(out)), "add_system")
        return out.value

    def add_boundary(self, inst, sys, kind, normal, point, beta_or_lj):
        nrm, pt = _a(normal, np.float64), _a(point, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_boundary(self.ctx, sys, kind, nrm.ctypes.data_as(_dp),
                                             pt.ctypes.data_as(_dp), beta_or_lj, ct.byref(out)), "add_boundary")
        return out.value

    def add_ghost(self, inst, src, copiers, normals, points, cutoff, capacity):
        nf = np.array([len(c) for c in copiers] or [0], dtype=np.int32)
        flds = np.array([f for c in copiers for f, _ in c] or [0], dtype=np.int32)
        mds = np.array([m for c in copiers for _, m in c] or [0], dtype=np.int32)
        nrm, pts = _a(normals, np.float64), _a(points, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_ghost(self.ctx, src, len(copiers), nf.ctypes.data_as(_ip),
                                          flds.ctypes.data_as(_ip), mds.ctypes.data_as(_ip), nrm.shape[0],
                                          nrm.ctypes.data_as(_dp), pts.ctypes.data_as(_dp), cutoff,
                                          ct.byref(out)), "add_ghost")
        return out.value

    def add_interaction(self, inst, a, b, kernel_kind, h, pfn_kinds, pfn_params):
        k = np.asarray(pfn_kinds, dtype=np.int32)
        p = _a(pfn_params, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_interaction(self.ctx, a, b, kernel_kind, h, len(k), k.ctypes.data_as(_ip),
                                                p.ctypes.data_as(_dp), ct.byref(out)), "add_interaction")
        return out.value

    def set_updaters(self, inst, sys, chains):
        cl = np.array([len(c) for c in chains] or [0], dtype=np.int32)
        kinds = np.array([k for c in chains for k, _ in c] or [0], dtype=np.int32)
        prm = np.array([p for c in chains for _, p in c] or [np.zeros(6)], dtype=np.float64)
        self._chk(self.L.oracle_set_updaters(self.ctx, sys, len(chains), cl.ctypes.data_as(_ip),
                                             kinds.ctypes.data_as(_ip), prm.ctypes.data_as(_dp)), "set_updaters")

    def set_integrator(self, inst, gamma):
        self._chk(self.L.oracle_set_integrator(self.ctx, gamma), "set_integrator")

    def add_virtual(self, inst, src, zero_mask, prescribed_v):
        pv = _a(prescribed_v, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_virtual(self.ctx, src, zero_mask, pv.ctypes.data_as(_dp), ct.byref(out)),
                  "add_virtual")
        return out.value

    def add_probe(self, inst, n, nd, positions, mirror, extras_mask, ns, prescribed_v):
        pos = None if positions is None else _a(positions, np.float64)
        pv = _a(prescribed_v, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_probe(self.ctx, n, nd, None if pos is None else pos.ctypes.data_as(_dp), mirror,
                                          extras_mask, ns, pv.ctypes.data_as(_dp), ct.byref(out)), "add_probe")
        return out.value

    def add_probe_interaction(self, inst, a, probe, kernel_kind, h, pfn_kind, pfn_params):
        p = _a(pfn_params, np.float64)
        out = ct.c_int()
        self._chk(self.L.oracle_add_probe_interaction(self.ctx, a, probe, kernel_kind, h, pfn_kind,
                                                      p.ctypes.data_as(_dp), ct.byref(out)), "add_probe_interaction")
        return out.value

    def measure_probes(self):
        self._chk(self.L.oracle_measure_probes(self.ctx), "measure_probes")

    def set_velocity_adjust(self, inst, inter, kind, epsilon):
        self._chk(self.L.oracle_set_velocity_adjust(self.ctx, inter, kind, epsilon), "set_velocity_adjust")

    def set_integrator_kind(self, inst, kind):
        self._chk(self.L.oracle_set_integrator_kind(self.ctx, kind), "set_integrator_kind")

    def finalize(self):
        if self._track:
            self.set_track_magnitude(self._track)

    def set_track_magnitude(self, mode):
        """Keep the magnitude shadows, the per-particle scale of the parity
        tests: mode 1 sums each pair term's magnitude (|initial| +
        Σ|terms|), mode 2 the magnitude each term takes with every
        difference of its inputs replaced by the sum of their magnitudes
        (inputs that carry relative errors); 0 turns them off."""
        self._track = int(mode)
        self._chk(self.L.oracle_set_track_magnitude(self.ctx, self._track), "set_track_magnitude")

    def magnitude(self, inst, handle, field, out):
        """The magnitude shadow of a rate field, in download_into's layout."""
        self._chk(self.L.oracle_get_magnitude(self.ctx, handle, field, out.ctypes.data, out.nbytes),
                  "get_magnitude")
        return out

    def set_precision(self, mode):
        pass

    def set_graphs(self, on, sync_every=32, cap_margin=0.0):
        pass

    def set_sweep_config(self, cfg):
        pass

    def upload(self, inst, handle, field, array):
        a = np.ascontiguousarray(array)
        self._chk(self.L.oracle_set_field(self.ctx, handle, field, a.ctypes.data, a.nbytes), "set_field")

    def download_into(self, inst, handle, field, out):
        self._chk(self.L.oracle_get_field(self.ctx, handle, field, out.ctypes.data, out.nbytes), "get_field")
        return out

    def count(self, inst, handle):
        n = ct.c_int64()
        self._chk(self.L.oracle_get_count(self.ctx, handle, ct.byref(n)), "get_count")
        return n.value

    def step(self, nsteps, cfl):
        self._chk(self.L.oracle_step(self.ctx, nsteps, cfl), "step")

    def stats(self):
        return {"steps_done": self.L.oracle_steps(self.ctx)}

    def sort(self, inst, handle, cutoff, n):
        perm = np.zeros(n, dtype=np.int64)
        self._chk(self.L.oracle_sort_system(self.ctx, handle, cutoff, perm.ctypes.data_as(_i64p)), "sort")
        return perm

    def build_grid(self, inst, inter, nd):
        ming = np.zeros(nd)
        ng = np.zeros(nd, dtype=np.int64)
        ncells = ct.c_int64()
        self._chk(self.L.oracle_build_grid(self.ctx, inter, None, 0, ming.ctypes.data_as(_dp),
                                           ng.ctypes.data_as(_i64p), ct.byref(ncells)), "build_grid")
        cs = np.zeros(ncells.value + 1, dtype=np.int64)
        self._chk(self.L.oracle_build_grid(self.ctx, inter, cs.ctypes.data_as(_i64p), cs.size, None, None,
                                           None), "build_grid")
        return cs, ming, ng

    def cell_start_a(self, inter, ncells):
        out = np.zeros(ncells + 1, dtype=np.int64)
        self._chk(self.L.oracle_grid_cell_start_a(self.ctx, inter, out.ctypes.data_as(_i64p), out.size),
                  "cell_start_a")
        return out

    def generate_ghosts(self, inst, ghost):
        self._chk(self.L.oracle_generate_ghosts(self.ctx, ghost), "generate_ghosts")

    def update_ghost_kinematics(self, inst, ghost):
        self._chk(self.L.oracle_update_ghost_kinematics(self.ctx, ghost), "update_ghost_kinematics")

    def update_ghost(self, inst, ghost, stage):
        self._chk(self.L.oracle_update_ghost(self.ctx, ghost, stage), "update_ghost")

    def sweep(self, inst, inter, stage):
        self._chk(self.L.oracle_sweep(self.ctx, inter, stage), "sweep")

    def update_state(self, inst, sys, stage, dt):
        self._chk(self.L.oracle_update_state(self.ctx, sys, stage, dt), "update_state")


def kernel_norm(kind, nd, H):
    return lib().oracle_kernel_norm(kind, nd, H)


def kernel_w(kind, nd, H, q):
    return lib().oracle_kernel_w(kind, nd, H, q)


def kernel_dw_dq(kind, nd, H, q):
    return lib().oracle_kernel_dw_dq(kind, nd, H, q)


def powi(x, n):
    return lib().oracle_powi(x, n)
