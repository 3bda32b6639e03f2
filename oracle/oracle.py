"""ctypes front-end of the CPU oracle (oracle/pgc_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  The product never imports it.
Parity status: unpinned against the reference binary (it cannot be built in
this environment); pinned against brute-force cycle enumeration instead.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_i64 = ctypes.c_longlong
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    """Compile the oracle library (make) and return its path."""
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [_dp, _i64, _ip, _i64, _dp, _i64, _ip, _i64, _dp, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_normals.argtypes = [ctypes.c_void_p, _dp, _i64, _dp, _i64]
        L.orc_set_mode.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p]
        L.orc_set_max_depth.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_robust_loss.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_generate.argtypes = [ctypes.c_void_p]
        L.orc_ensure_generated.argtypes = [ctypes.c_void_p]
        L.orc_recompute_energy.argtypes = [ctypes.c_void_p]
        L.orc_normals_2d.argtypes = [_dp, _i64, _ip, _i64, _dp]
        L.orc_normals_3d.argtypes = [_dp, _i64, _ip, _i64, _dp]
        L.orc_cost_shape.argtypes = [ctypes.c_void_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]
        L.orc_get_cost.argtypes = [ctypes.c_void_p, _dp]
        L.orc_set_cost.argtypes = [ctypes.c_void_p, _dp, _i64, _i64]
        L.orc_ps_shape.argtypes = [ctypes.c_void_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]
        L.orc_get_ps.argtypes = [ctypes.c_void_p, _ip]
        L.orc_get_src_trgt.argtypes = [ctypes.c_void_p, _ip, _ip]
        L.orc_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_float)]
        L.orc_matching_shape.argtypes = [ctypes.c_void_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]
        L.orc_get_matching.argtypes = [ctypes.c_void_p, _ip]
        L.orc_cycle_edges.restype = _i64
        L.orc_cycle_edges.argtypes = [ctypes.c_void_p, ctypes.POINTER(_i64), _i64]
        L.orc_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(_i64)]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_time_phases.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_double)]
        L.orc_time_sweeps.restype = ctypes.c_double
        L.orc_time_sweeps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def normals_2d(V, E):
    """utils::normals2d restated (helper/utils.cpp:93-157)."""
    V, E = _d(V), _i(E)
    out = np.empty_like(V)
    rc = lib().orc_normals_2d(V.ctypes.data_as(_dp), V.shape[0], E.ctypes.data_as(_ip), E.shape[0],
                              out.ctypes.data_as(_dp))
    if rc == -2:
        raise ValueError("V.rows() != E.rows()")
    if rc != 0:
        raise ValueError("points dont lie on xy, xz or yz plane")
    return out


def normals_3d(V, F):
    """utils::normals3d restated (helper/utils.cpp:86-90, libigl area weighting)."""
    V, F = _d(V), _i(F)
    out = np.empty_like(V)
    if lib().orc_normals_3d(V.ctypes.data_as(_dp), V.shape[0], F.ctypes.data_as(_ip), F.shape[0],
                            out.ctypes.data_as(_dp)) != 0:
        raise ValueError("F refers to a vertex outside V")
    return out


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class OracleGenerator:
    """Mirror of the reference's product_graph_generator, computed on the CPU."""

    def __init__(self, VX, EX, VY, EY, feat_diff, use_conjugate_graph, use_regularising_cost_term,
                 prune_intralayer=False):
        L = lib()
        self._keep = [_d(VX), _i(EX), _d(VY), _i(EY), _d(feat_diff)]
        VX, EX, VY, EY, FD = self._keep
        assert FD.shape == (VX.shape[0], VY.shape[0])
        self._h = L.orc_create(VX.ctypes.data_as(_dp), VX.shape[0], EX.ctypes.data_as(_ip), EX.shape[0],
                               VY.ctypes.data_as(_dp), VY.shape[0], EY.ctypes.data_as(_ip), EY.shape[0],
                               FD.ctypes.data_as(_dp), int(bool(use_conjugate_graph)),
                               int(bool(use_regularising_cost_term)), int(bool(prune_intralayer)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def set_normals(self, NX, NY):
        NX, NY = _d(NX), _d(NY)
        self._keep += [NX, NY]
        return lib().orc_set_normals(self._h, NX.ctypes.data_as(_dp), NX.shape[0], NY.ctypes.data_as(_dp),
                                     NY.shape[0])

    def set_cost_time_ratio_mode(self, cost: str, time: str):
        lib().orc_set_mode(self._h, cost.encode(), time.encode())

    def set_max_depth_cost_time_ratio(self, k: int):
        lib().orc_set_max_depth(self._h, int(k))

    def update_robust_loss_params(self, a, c, p):
        lib().orc_set_robust_loss(self._h, float(a), float(c), float(p))

    def generate(self):
        if lib().orc_generate(self._h) != 0:
            raise RuntimeError(lib().orc_last_error().decode())

    def recompute_energy(self):
        """The edge costs again on the product graph already built (a first call generates)."""
        if lib().orc_recompute_energy(self._h) != 0:
            raise RuntimeError(lib().orc_last_error().decode())

    def _ensure(self):
        if lib().orc_ensure_generated(self._h) != 0:
            raise RuntimeError(lib().orc_last_error().decode())

    def get_cost_vector(self):
        self._ensure()
        r, c = _i64(), _i64()
        lib().orc_cost_shape(self._h, ctypes.byref(r), ctypes.byref(c))
        out = np.empty((r.value, c.value), dtype=np.float64)
        lib().orc_get_cost(self._h, out.ctypes.data_as(_dp))
        return out

    def set_cost_vector(self, E):
        self._ensure()
        E = _d(E)
        if E.ndim == 1:
            E = E[:, None]
        if lib().orc_set_cost(self._h, E.ctypes.data_as(_dp), E.shape[0], E.shape[1]) != 0:
            raise ValueError("cost vector has the wrong number of rows")

    def product_space_rows(self) -> int:
        """Number of product edges, without copying the product space."""
        self._ensure()
        r, c = _i64(), _i64()
        lib().orc_ps_shape(self._h, ctypes.byref(r), ctypes.byref(c))
        return int(r.value)

    def get_product_space(self):
        self._ensure()
        r, c = _i64(), _i64()
        lib().orc_ps_shape(self._h, ctypes.byref(r), ctypes.byref(c))
        out = np.empty((r.value, c.value), dtype=np.int32)
        lib().orc_get_ps(self._h, out.ctypes.data_as(_ip))
        return out

    def get_src_trgt(self):
        self._ensure()
        r, c = _i64(), _i64()
        lib().orc_ps_shape(self._h, ctypes.byref(r), ctypes.byref(c))
        s = np.empty(r.value, dtype=np.int32)
        t = np.empty(r.value, dtype=np.int32)
        lib().orc_get_src_trgt(self._h, s.ctypes.data_as(_ip), t.ctypes.data_as(_ip))
        return s, t

    def _solve(self, which, k):
        p = ctypes.c_int()
        o = ctypes.c_float()
        if lib().orc_solve(self._h, which, int(k), ctypes.byref(p), ctypes.byref(o)) != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        r, c = _i64(), _i64()
        lib().orc_matching_shape(self._h, ctypes.byref(r), ctypes.byref(c))
        m = np.empty((r.value, c.value), dtype=np.int32)
        lib().orc_get_matching(self._h, m.ctypes.data_as(_ip))
        return bool(p.value), float(o.value), m

    def solve_with_cost_time_ratio(self, name="lawlercpu", k=-1):
        return self._solve(0, k)

    def solve_with_minimum_cost(self, name="dijkstracpu", k=-1):
        return self._solve(1, k)

    def last_cycle_edges(self):
        n = lib().orc_cycle_edges(self._h, None, 0)
        buf = (_i64 * max(1, n))()
        lib().orc_cycle_edges(self._h, buf, n)
        return np.array(buf[:n], dtype=np.int64)

    def last_stats(self):
        buf = (_i64 * 5)()
        lib().orc_stats(self._h, buf)
        return dict(zip(["bf_calls", "sweeps", "candidates_walked", "lawler_iters", "branches"], buf[:5]))

    def time_phases(self, k, lam, sweeps):
        """[energy, rescale, in-edge sets, seconds per sweep] of a CPU ratio solve."""
        buf = (ctypes.c_double * 4)()
        lib().orc_time_phases(self._h, int(k), float(lam), int(sweeps), buf)
        return dict(zip(["energy_s", "rescale_s", "in_graph_s", "sweep_s"], list(buf)))

    def time_sweeps(self, k, lam, sweeps):
        return lib().orc_time_sweeps(self._h, int(k), float(lam), int(sweeps))
