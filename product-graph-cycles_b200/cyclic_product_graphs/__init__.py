"""cyclic_product_graphs -- drop-in Python front-end of the sm_100a cycle search.

Mirrors the reference module of the same name (pythonbinding/bindings.cpp:22-48):
the class ``product_graph_generator`` with ``generate``, ``get_cost_vector``,
``update_robust_loss_params``, ``set_normals``, ``get_product_space``,
``solve_with_cost_time_ratio``, ``solve_with_minimum_cost``,
``set_max_depth_cost_time_ratio`` and ``set_cost_time_ratio_mode``, and the
helpers ``compute_normals_3d`` / ``compute_normals_2d``.  Solves return the
reference's tuple ``(passes_layers_just_once: bool, final_objective: float,
matching: int32 ndarray)``.

Everything runs through the C ABI of ``lib/libpgc.so`` (include/pgc.h); the
solvers execute on the GPU.  There is no CPU fallback: importing this module
without the built library raises ImportError.  The library is opened on the
first call that needs it, so importing the package (or its ``synthetic``
data module) changes nothing in the process: no library is mapped and no
environment variable is set.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

__all__ = ["product_graph_generator", "compute_normals_3d", "compute_normals_2d", "compute_local_thickness_3d",
           "compute_local_thickness_2d", "library_path", "PGCError", "solve_batch", "load_export", "from_export", "autotune", "release_cached_memory",
           "product_graph_sizes", "vertex_correspondences", "last_batch_profile", "kernel_launches",
           "set_feat_diffs_device", "backward_feat_diffs"]

_PKG = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(os.path.dirname(_PKG), "lib", "libpgc.so")

if not os.path.exists(library_path):
    raise ImportError(f"cyclic_product_graphs: {library_path} is missing; build it with "
                      "`python -c 'import __graft_entry__ as g; g.build()'` (or make -C product-graph-cycles_b200/csrc)")

_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lp = ctypes.POINTER(ctypes.c_int64)
_h = ctypes.c_void_p


def _declare(L):
    """Argument and result types of every C entry point the package calls."""
    L.pgc_create.argtypes = [_dp, _i64, _ip, _i64, _dp, _i64, _ip, _i64, _dp, ctypes.c_int, ctypes.c_int,
                             ctypes.c_int, ctypes.POINTER(_h)]
    L.pgc_destroy.argtypes = [_h]
    L.pgc_destroy.restype = None
    L.pgc_set_normals.argtypes = [_h, _dp, _i64, _i64, _dp, _i64, _i64]
    L.pgc_set_max_depth.argtypes = [_h, ctypes.c_int]
    L.pgc_set_cost_time_ratio_mode.argtypes = [_h, ctypes.c_char_p, ctypes.c_char_p]
    L.pgc_update_robust_loss_params.argtypes = [_h, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.pgc_generate.argtypes = [_h]
    L.pgc_cost_vector_shape.argtypes = [_h, _lp, _lp]
    L.pgc_get_cost_vector.argtypes = [_h, _dp]
    L.pgc_product_space_shape.argtypes = [_h, _lp, _lp]
    L.pgc_get_product_space.argtypes = [_h, _ip]
    L.pgc_solve_with_cost_time_ratio.argtypes = [_h, ctypes.c_char_p, ctypes.c_int]
    L.pgc_solve_with_minimum_cost.argtypes = [_h, ctypes.c_char_p, ctypes.c_int]
    L.pgc_result.argtypes = [_h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), _lp, _lp]
    L.pgc_result_matching.argtypes = [_h, _ip]
    L.pgc_result_cycle_edges.argtypes = [_h, _lp, _i64, _lp]
    L.pgc_result_stats.argtypes = [_h, _lp]
    L.pgc_compute_normals_2d.argtypes = [_dp, _i64, _ip, _i64, _dp]
    L.pgc_compute_normals_3d.argtypes = [_dp, _i64, _ip, _i64, _dp]
    L.pgc_graph_info.argtypes = [_h, _lp]
    L.pgc_result_profile.argtypes = [_h, _lp]
    L.pgc_result_profile_detail.argtypes = [_h, _lp]
    L.pgc_set_stream.argtypes = [_h, ctypes.c_void_p]
    L.pgc_set_team_cap.argtypes = [_h, ctypes.c_int]
    L.pgc_set_team_shape.argtypes = [_h, ctypes.c_int, ctypes.c_int]
    L.pgc_product_graph_sizes.argtypes = [_ip, _i64, _i64, _i64, ctypes.c_int, ctypes.c_int, _lp]
    L.pgc_backward_feat_diff.argtypes = [_h, ctypes.c_double, ctypes.c_void_p, ctypes.c_int]
    L.pgc_set_cost_vector.argtypes = [_h, _dp, _i64, _i64]
    L.pgc_set_feat_diff.argtypes = [_h, _dp, _i64, _i64]
    L.pgc_set_feat_diff_device.argtypes = [_h, ctypes.c_void_p, _i64, _i64]
    L.pgc_set_feat_diff_device_batch.argtypes = [ctypes.POINTER(_h), _i64, ctypes.POINTER(ctypes.c_void_p)]
    L.pgc_backward_feat_diff_batch.argtypes = [ctypes.POINTER(_h), _i64, _dp, ctypes.POINTER(ctypes.c_void_p),
                                               ctypes.c_int]
    L.pgc_solve_batch.argtypes = [ctypes.POINTER(_h), _i64, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.pgc_device_name.argtypes = [_h, ctypes.c_char_p, _i64]
    L.pgc_batch_profile.argtypes = [_dp]
    L.pgc_kernel_launches.argtypes = [_lp]
    L.pgc_last_error.restype = ctypes.c_char_p
    L.pgc_version.restype = ctypes.c_char_p


class _Library:
    """libpgc.so, opened with its entry points declared on first attribute access."""

    def __init__(self):
        self._cdll = None
        self._mutex = threading.Lock()

    def __getattr__(self, name):
        cdll = self._cdll
        if cdll is None:
            with self._mutex:
                if self._cdll is None:
                    L = ctypes.CDLL(library_path)
                    _declare(L)
                    self._cdll = L
                cdll = self._cdll
        return getattr(cdll, name)

    @property
    def loaded(self) -> bool:
        return self._cdll is not None


_lib = _Library()


class PGCError(RuntimeError):
    """A libpgc call failed; ``code`` is the PGC_ERR_* value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[pgc {code}] {message}")
        self.code = code


def _check(rc: int):
    if rc != 0:
        raise PGCError(rc, _lib.pgc_last_error().decode(errors="replace"))


def _f64(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if cols is not None and (a.ndim != 2 or a.shape[1] != cols):
        raise ValueError(f"expected an [n x {cols}] matrix, got shape {a.shape}")
    return a


def _i32(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    if cols is not None and (a.ndim != 2 or a.shape[1] != cols):
        raise ValueError(f"expected an [n x {cols}] matrix, got shape {a.shape}")
    return a


def version() -> str:
    return _lib.pgc_version().decode()


class product_graph_generator:
    """product_graph_generator(VX, EX, VY, EY, feat_diff, use_conjugate_graph,
    use_regularising_cost_term[, prune_intralayer])  (bindings.cpp:33-34)."""

    def __init__(self, VX, EX, VY, EY, feat_diff, use_conjugate_graph: bool, use_regularising_cost_term: bool,
                 prune_intralayer: bool = False):
        VX = _f64(VX, 3)
        EX = _i32(EX, 2)
        VY = _f64(VY, 3)
        EY = _i32(EY, 2)
        FD = _f64(feat_diff)
        if FD.shape != (VX.shape[0], VY.shape[0]):
            raise ValueError(f"feat_diff must be |VX| x |VY| = {(VX.shape[0], VY.shape[0])}, got {FD.shape}")
        h = _h()
        _check(_lib.pgc_create(VX.ctypes.data_as(_dp), VX.shape[0], EX.ctypes.data_as(_ip), EX.shape[0],
                               VY.ctypes.data_as(_dp), VY.shape[0], EY.ctypes.data_as(_ip), EY.shape[0],
                               FD.ctypes.data_as(_dp), int(bool(use_conjugate_graph)),
                               int(bool(use_regularising_cost_term)), int(bool(prune_intralayer)), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # at interpreter exit the module may already be torn down
            _lib.pgc_destroy(h)
            self._h = None

    # -- configuration -----------------------------------------------------
    def set_normals(self, NX, NY):
        """setNormals (product_graph_generators.cpp:118-130); shapes |VX| x 3 and |VY| x 3."""
        NX = _f64(NX)
        NY = _f64(NY)
        if NX.ndim != 2 or NY.ndim != 2:
            raise ValueError("normals must be 2-d matrices")
        _check(_lib.pgc_set_normals(self._h, NX.ctypes.data_as(_dp), NX.shape[0], NX.shape[1],
                                    NY.ctypes.data_as(_dp), NY.shape[0], NY.shape[1]))

    def set_max_depth_cost_time_ratio(self, max_depth: int):
        _check(_lib.pgc_set_max_depth(self._h, int(max_depth)))

    def set_cost_time_ratio_mode(self, cost_name: str, time_name: str):
        _check(_lib.pgc_set_cost_time_ratio_mode(self._h, str(cost_name).encode(), str(time_name).encode()))

    def update_robust_loss_params(self, alpha: float, c: float, pwr: float):
        _check(_lib.pgc_update_robust_loss_params(self._h, float(alpha), float(c), float(pwr)))

    # -- graph ---------------------------------------------------------------
    def generate(self):
        _check(_lib.pgc_generate(self._h))

    def get_cost_vector(self) -> np.ndarray:
        r, c = _i64(), _i64()
        _check(_lib.pgc_cost_vector_shape(self._h, ctypes.byref(r), ctypes.byref(c)))
        out = np.empty((r.value, c.value), dtype=np.float64)
        _check(_lib.pgc_get_cost_vector(self._h, out.ctypes.data_as(_dp)))
        return out

    def get_product_space(self) -> np.ndarray:
        r, c = _i64(), _i64()
        _check(_lib.pgc_product_space_shape(self._h, ctypes.byref(r), ctypes.byref(c)))
        out = np.empty((r.value, c.value), dtype=np.int32)
        _check(_lib.pgc_get_product_space(self._h, out.ctypes.data_as(_ip)))
        return out

    # -- solvers -------------------------------------------------------------
    def _result(self):
        p = ctypes.c_int()
        o = ctypes.c_float()
        r, c = _i64(), _i64()
        _check(_lib.pgc_result(self._h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(r), ctypes.byref(c)))
        m = np.empty((r.value, c.value), dtype=np.int32)
        _check(_lib.pgc_result_matching(self._h, m.ctypes.data_as(_ip)))
        return bool(p.value), float(o.value), m

    def solve_with_cost_time_ratio(self, solver_name: str, max_depth: int | None = None):
        """Minimum cost/time-ratio cycle (Lawler), bindings.cpp:41-42."""
        _check(_lib.pgc_solve_with_cost_time_ratio(self._h, str(solver_name).encode(),
                                                   -1 if max_depth is None else int(max_depth)))
        return self._result()

    def solve_with_minimum_cost(self, solver_name: str, max_depth: int | None = None):
        """Minimum-cost cycle, bindings.cpp:44-45."""
        _check(_lib.pgc_solve_with_minimum_cost(self._h, str(solver_name).encode(),
                                                -1 if max_depth is None else int(max_depth)))
        return self._result()

    # -- extras (no counterpart in the reference's binding) ------------------
    def last_cycle_edges(self) -> np.ndarray:
        """Edge ids (rows of get_product_space()) of the last returned cycle."""
        cnt = _i64()
        _check(_lib.pgc_result_cycle_edges(self._h, None, 0, ctypes.byref(cnt)))
        out = np.empty(cnt.value, dtype=np.int64)
        _check(_lib.pgc_result_cycle_edges(self._h, out.ctypes.data_as(_lp), cnt.value, ctypes.byref(cnt)))
        return out

    def last_profile(self) -> dict:
        """SM-cycle counters (one thread of CTA 0) and team shape of the last solve's Bellman-Ford launches."""
        buf = (ctypes.c_int64 * 8)()
        _check(_lib.pgc_result_profile(self._h, buf))
        detail = (ctypes.c_int64 * 4)()
        _check(_lib.pgc_result_profile_detail(self._h, detail))
        return dict(zip(["cycles_relax", "cycles_bookkeeping", "cycles_handoff", "cycles_sweep_tail", "steps",
                         "ctas", "threads", "wait_entries", "cycles_stage_wait", "cycles_tail_wrap",
                         "cycles_tail_candidates", "cycles_tail_lead"], list(buf) + list(detail)))

    def graph_info(self) -> dict:
        """Sizes of the generated product graph (generates it if needed)."""
        buf = (ctypes.c_int64 * 8)()
        _check(_lib.pgc_graph_info(self._h, buf))
        keys = ["nodes_per_layer", "layers", "edges_per_block", "inter_edges_per_layer", "intra_edges_per_layer",
                "inter_slots_per_layer", "intra_slots_per_layer", "cost_columns"]
        return dict(zip(keys, list(buf)))

    def set_cost_vector(self, E):
        """Set the edge costs [rows x 1|2] (edge-id order) in place of generate()."""
        E = np.ascontiguousarray(E, dtype=np.float64)
        if E.ndim == 1:
            E = E.reshape(-1, 1)
        _check(_lib.pgc_set_cost_vector(self._h, E.ctypes.data_as(_dp), E.shape[0], E.shape[1]))

    def set_feat_diff(self, feat_diff):
        """Replace feat_diff (|VX| x |VY|); the next solve regenerates the costs."""
        FD = np.ascontiguousarray(feat_diff, dtype=np.float64)
        if FD.ndim != 2:
            raise ValueError("feat_diff must be a 2-d matrix")
        _check(_lib.pgc_set_feat_diff(self._h, FD.ctypes.data_as(_dp), FD.shape[0], FD.shape[1]))

    def set_feat_diff_device(self, ptr: int, rows: int, cols: int):
        """Replace feat_diff from device memory: ``ptr`` addresses rows x cols
        row-major float64 on this handle's GPU, already written (synchronise
        its producer first).  Copied before the call returns."""
        _check(_lib.pgc_set_feat_diff_device(self._h, ctypes.c_void_p(int(ptr)), int(rows), int(cols)))

    def backward_feat_diff(self, grad_objective: float, grad_feat_diff_ptr: int, accumulate: bool = False):
        """grad_objective * d(last objective)/d(feat_diff) into a device buffer (|VX| x |VY| float64)."""
        _check(_lib.pgc_backward_feat_diff(self._h, float(grad_objective), ctypes.c_void_p(int(grad_feat_diff_ptr)),
                                           int(bool(accumulate))))

    def set_team_cap(self, max_ctas: int):
        """Most CTAs a Bellman-Ford launch of this graph may use (0: no limit)."""
        _check(_lib.pgc_set_team_cap(self._h, int(max_ctas)))

    def set_team_shape(self, ctas: int = 0, threads_per_cta: int = 0):
        """Bellman-Ford team of this graph: ctas CTAs of threads_per_cta
        threads (0: automatic).  Results do not depend on it (see autotune)."""
        _check(_lib.pgc_set_team_shape(self._h, int(ctas), int(threads_per_cta)))

    def set_stream(self, cuda_stream: int | None):
        """Issue all device work of this generator on `cuda_stream` (a cudaStream_t as int)."""
        _check(_lib.pgc_set_stream(self._h, ctypes.c_void_p(cuda_stream) if cuda_stream else None))

    def device_name(self) -> str:
        """Name of the GPU this generator's device work runs on (C: pgc_device_name)."""
        buf = ctypes.create_string_buffer(256)
        _check(_lib.pgc_device_name(self._h, buf, len(buf)))
        return buf.value.decode(errors="replace")

    def last_stats(self) -> dict:
        buf = (ctypes.c_int64 * 8)()
        _check(_lib.pgc_result_stats(self._h, buf))
        keys = ["bf_calls", "sweeps", "candidates", "lawler_iters", "branches", "fallback_walks", "device_us",
                "kernel_launches"]
        return dict(zip(keys, list(buf)))


def product_graph_sizes(EX, n_vertices_x: int, n_edges_y: int, conjugate: bool = False,
                        prune_intralayer_edges: bool = False) -> dict:
    """Sizes of the product graph of X and a closed curve with ``n_edges_y``
    edges, from the layer template built on the host (no GPU needed; no
    counterpart in the reference)."""
    EX = np.ascontiguousarray(EX, dtype=np.int32)
    if EX.ndim != 2 or EX.shape[1] != 2:
        raise ValueError("EX must be [n x 2]")
    out = (ctypes.c_int64 * 6)()
    _check(_lib.pgc_product_graph_sizes(EX.ctypes.data_as(_ip), EX.shape[0], int(n_vertices_x), int(n_edges_y),
                                        int(bool(conjugate)), int(bool(prune_intralayer_edges)), out))
    keys = ["nodes_per_layer", "edges_per_block", "inter_edges_per_block", "intra_edges_per_block", "slices",
            "ell_rows"]
    d = dict(zip(keys, list(out)))
    d["edges"] = d["edges_per_block"] * int(n_edges_y)
    return d


def release_cached_memory():
    """Returns the device memory and the pinned host memory that the
    library's allocators keep for reuse (no counterpart in the reference)."""
    _check(_lib.pgc_release_cached_memory())


def load_export(directory: str = ".") -> dict:
    """Reads back the CSV files that the "export" solver writes
    (product_graph_generators.cpp:272-282: VX, VY, EX, EY, FeatDiffMatrix and,
    for a conjugate graph, NX and NY; one row per line, values separated by
    ", ", doubles with 17 significant digits, so they round-trip exactly).

    Returns {"VX", "VY", "EX", "EY", "feat_diff"} and "NX", "NY" when those
    files exist.  No counterpart in the reference, which only writes them.
    """
    def read(name, dtype):
        return np.loadtxt(os.path.join(directory, name + ".csv"), delimiter=",", dtype=dtype, ndmin=2)

    out = {"VX": read("VX", np.float64), "VY": read("VY", np.float64), "EX": read("EX", np.int32),
           "EY": read("EY", np.int32), "feat_diff": read("FeatDiffMatrix", np.float64)}
    if os.path.exists(os.path.join(directory, "NX.csv")):
        out["NX"] = read("NX", np.float64)
        out["NY"] = read("NY", np.float64)
    return out


def from_export(directory: str = ".", conjugate: bool = False, regularising_cost_term: bool = False,
                prune_intralayer_edges: bool = False) -> "product_graph_generator":
    """A generator built from an "export" directory (load_export), with its
    normals set when the files hold them: replays an exported problem.  The
    flags are not part of the export and are given again."""
    d = load_export(directory)
    g = product_graph_generator(d["VX"], d["EX"], d["VY"], d["EY"], d["feat_diff"], conjugate,
                                regularising_cost_term, prune_intralayer_edges)
    if "NX" in d:
        g.set_normals(d["NX"], d["NY"])
    return g


def autotune(gen: "product_graph_generator", max_depth: int | None = None, candidates=None,
             cache_path: str | None = None, repeats: int = 2) -> dict:
    """Picks the Bellman-Ford team shape (CTAs, threads per CTA) for the shape
    bucket of ``gen`` and applies it (no counterpart in the reference).

    The bucket is (the GPU's name, nodes per layer rounded up to a power of
    two, layers rounded up to a power of two, max depth, whether layers have
    intralayer edges): a cache file written on one GPU type is not applied
    on another.  A bucket found in the JSON file ``cache_path`` is applied
    without timing.  Otherwise every candidate (ctas, threads_per_cta) --
    by default the automatic shape, the automatic CTA count with 320 and 480
    threads, and a half-size team -- is timed over ``repeats`` ratio solves
    (costs regenerated before each; the Bellman-Ford device time of the solve
    is compared), the fastest is applied, and the bucket's entry, with every
    candidate's time, is merged into the cache file as it is then.  The
    shape changes the speed only: every solve returns the same result.
    """
    import json

    info = gen.graph_info()
    k = int(max_depth) if max_depth is not None else None

    def p2(x):
        return 1 << max(0, int(x) - 1).bit_length()

    key = (f"{gen.device_name()}|n{p2(info['nodes_per_layer'])}-l{p2(info['layers'])}-k{k}"
           f"-intra{int(info['intra_edges_per_layer'] > 0)}")
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    if key in cache:
        e = cache[key]
        gen.set_team_shape(e["ctas"], e["threads_per_cta"])
        return dict(e, bucket=key, cached=True)

    def timed(shape):
        gen.set_team_shape(*shape)
        best = None
        for _ in range(max(1, repeats)):
            gen.generate()
            gen.solve_with_cost_time_ratio("lawlergpu", k)
            ms = gen.last_stats()["device_us"] / 1000.0
            best = ms if best is None else min(best, ms)
        return best, gen.last_profile()

    if candidates is None:
        _, prof = timed((0, 0))
        auto = int(prof["ctas"])
        candidates = [(0, 0), (auto, 320), (auto, 480), (max(1, auto // 2), 640)]
    results = []
    for shape in candidates:
        ms, prof = timed(tuple(shape))
        results.append({"ctas": int(shape[0]), "threads_per_cta": int(shape[1]), "bf_ms": ms,
                        "team": [int(prof["ctas"]), int(prof["threads"])]})
    best = min(results, key=lambda r: r["bf_ms"])
    entry = {"ctas": best["ctas"], "threads_per_cta": best["threads_per_cta"], "bf_ms": best["bf_ms"],
             "candidates": results}
    gen.set_team_shape(best["ctas"], best["threads_per_cta"])
    if cache_path:
        # buckets another tuner wrote meanwhile are kept; the file is
        # replaced in one rename, so a reader never sees half of it
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        cache[key] = entry
        tmp = f"{cache_path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, cache_path)
    return dict(entry, bucket=key, cached=False)


def solve_batch(generators, solver_name: str, max_depth: int | None = None, ctas_per_graph: int = 0,
                workers: int = 0, regenerate: bool = False):
    """Solve many generators concurrently (no counterpart in the reference).

    Each generator gets the result ``solve_with_cost_time_ratio`` (solver
    ``"lawlercpu"``/``"lawlergpu"``) or ``solve_with_minimum_cost`` (any other
    name) would give it; with ``regenerate`` each first recomputes its edge
    costs.  Returns the list of ``(passes_layers_just_once, final_objective,
    matching)`` triples.

    Ratio solvers: ``workers`` native threads (0: 64) generate and rescale the
    costs, then one persistent launch runs every graph's whole ratio solve on
    the device, teams of ``ctas_per_graph`` CTAs (0: ``PGC_BATCH_TEAM``, else
    8) taking the graphs largest first; a graph whose first-branch cycle wraps
    is finished on the host with branch and bound.  Other solvers run each
    graph on its own CUDA stream with a team of at most ``ctas_per_graph``
    CTAs (0: SMs / min(graphs, 32)); the device runs those streams side by
    side only as far as it has host work queues: CUDA's default is 8, and a
    process started with ``CUDA_DEVICE_MAX_CONNECTIONS=32`` (read when CUDA
    initialises) runs such a batch about 3x faster.  The package does not set
    it: that is the application's choice, since it changes how all of the
    process's streams share the device.
    """
    gens = list(generators)
    if len(set(id(g) for g in gens)) != len(gens):
        raise ValueError("solve_batch needs distinct generators")
    arr = (_h * len(gens))(*[g._h for g in gens])
    status = (ctypes.c_int * len(gens))()
    _check(_lib.pgc_solve_batch(arr, len(gens), str(solver_name).encode(), -1 if max_depth is None else int(max_depth),
                                int(ctas_per_graph), int(workers), int(bool(regenerate)), status))
    return [g._result() for g in gens]


def set_feat_diffs_device(generators, pointers):
    """``set_feat_diff_device`` for many distinct generators at once (no
    counterpart in the reference): pointers[i] addresses generator i's
    |VX| x |VY| float64 matrix on its GPU, already written.  The copies are
    enqueued together and waited for once per generator."""
    gens = list(generators)
    if len(set(id(g) for g in gens)) != len(gens):
        raise ValueError("set_feat_diffs_device needs distinct generators")
    arr = (_h * len(gens))(*[g._h for g in gens])
    ptrs = (ctypes.c_void_p * len(gens))(*[int(p) for p in pointers])
    _check(_lib.pgc_set_feat_diff_device_batch(arr, len(gens), ptrs))


def backward_feat_diffs(generators, grad_objectives, grad_pointers, accumulate: bool = False):
    """``backward_feat_diff`` for many distinct generators at once (no
    counterpart in the reference): the adjoint kernels are enqueued together,
    then every generator's stream is waited for once."""
    gens = list(generators)
    if len(set(id(g) for g in gens)) != len(gens):
        raise ValueError("backward_feat_diffs needs distinct generators")
    arr = (_h * len(gens))(*[g._h for g in gens])
    grads = (ctypes.c_double * len(gens))(*[float(x) for x in grad_objectives])
    ptrs = (ctypes.c_void_p * len(gens))(*[int(p) for p in grad_pointers])
    _check(_lib.pgc_backward_feat_diff_batch(arr, len(gens), grads, ptrs, int(bool(accumulate))))


def last_batch_profile() -> dict:
    """Where this thread's last solve_batch spent its time (no counterpart in
    the reference): host wall-clock ms of preparing the graphs, of the
    launch that solved them, and of taking the results over (or finishing
    handed-back graphs on the host); graph counts; the launch's shape."""
    buf = (ctypes.c_double * 8)()
    _check(_lib.pgc_batch_profile(buf))
    keys = ["prepare_ms", "launch_ms", "finish_ms", "handed_back", "solved_on_device", "ctas", "threads_per_cta",
            "smem_bytes"]
    return dict(zip(keys, list(buf)))


def kernel_launches() -> int:
    """Kernel launches the library has issued in this process so far (no
    counterpart in the reference): the difference across a region is the
    number of the library's kernels that ran in it."""
    out = ctypes.c_int64()
    _check(_lib.pgc_kernel_launches(ctypes.byref(out)))
    return int(out.value)


def vertex_correspondences(matching, conjugate: bool | None = None) -> np.ndarray:
    """Vertex correspondences of a returned matching: one [x, y] row per
    matching row, in the matching's cycle order (int32, L x 2).

    This is the step after the solve in the reference's usage example
    (README.md:79-85): column 0 of a matching row is the Y vertex it starts
    at, and the X vertex is column 2 of a plain row [y0, y1, x0, x1] or
    column 3 of a conjugate row [y0, y1, y2, x0, x1, x2].  `conjugate` None
    takes the graph kind from the column count (4 plain, 6 conjugate).
    """
    m = np.asarray(matching)
    if m.ndim != 2 or m.shape[1] not in (4, 6):
        raise ValueError(f"a matching has 4 (plain) or 6 (conjugate) columns, got shape {m.shape}")
    if conjugate is None:
        conjugate = m.shape[1] == 6
    if m.shape[1] != (6 if conjugate else 4):
        raise ValueError(f"a {'conjugate' if conjugate else 'plain'} matching has {6 if conjugate else 4} columns, "
                         f"got {m.shape[1]}")
    return np.column_stack((m[:, 3 if conjugate else 2], m[:, 0])).astype(np.int32, copy=False)


def compute_normals_2d(V, E) -> np.ndarray:
    """utils::normals2d (helper/utils.cpp:93-157)."""
    V = _f64(V, 3)
    E = _i32(E, 2)
    out = np.empty_like(V)
    _check(_lib.pgc_compute_normals_2d(V.ctypes.data_as(_dp), V.shape[0], E.ctypes.data_as(_ip), E.shape[0],
                                       out.ctypes.data_as(_dp)))
    return out


def compute_normals_3d(V, F) -> np.ndarray:
    """utils::normals3d (helper/utils.cpp:86-90): area-weighted vertex normals."""
    V = _f64(V, 3)
    F = _i32(F, 3)
    out = np.empty_like(V)
    _check(_lib.pgc_compute_normals_3d(V.ctypes.data_as(_dp), V.shape[0], F.ctypes.data_as(_ip), F.shape[0],
                                       out.ctypes.data_as(_dp)))
    return out


def compute_local_thickness_3d(*args, **kwargs):
    """Unimplemented in the reference as well (bindings.cpp:18-20, :28)."""
    print("TODO: IMPL")


def compute_local_thickness_2d(*args, **kwargs):
    """Unimplemented in the reference as well (bindings.cpp:18-20, :29)."""
    print("TODO: IMPL")
