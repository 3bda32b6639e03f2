"""pgc_get_cost_vector_noalloc, the cost export for callers that cannot let
the library allocate device memory (their GPU memory is held by their own
allocator, or they cannot afford cudaFree's device-wide synchronization). It
has no counterpart in the reference. Called through the C ABI, two calls in a
row must return the same matrix, bit for bit, as the allocating
pgc_get_cost_vector. That holds on plain and conjugate graphs, before and
after a ratio solve has rescaled the costs in place. Larger cost vectors than
the 2^21-value scratch, and graphs whose costs were never generated, are
refused."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PGC_ERR_ARG, PGC_ERR_STATE = -1, -2
MAX_VALUES = 1 << 21


def _abi(cpg):
    lib = ctypes.CDLL(cpg.library_path)
    for name in ("pgc_get_cost_vector", "pgc_get_cost_vector_noalloc"):
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.pgc_cost_vector_shape.restype = ctypes.c_int
    lib.pgc_cost_vector_shape.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int64)]
    lib.pgc_last_error.restype = ctypes.c_char_p
    return lib


def _shape(lib, g):
    r, c = ctypes.c_int64(), ctypes.c_int64()
    assert lib.pgc_cost_vector_shape(g._h, ctypes.byref(r), ctypes.byref(c)) == 0
    return r.value, c.value


def _export(lib, g, name):
    rows, cols = _shape(lib, g)
    out = np.full((rows, cols), np.nan)
    rc = getattr(lib, name)(g._h, out.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0, lib.pgc_last_error()
    return out


def _graph(cpg, conj, level=1, m=8, seed=0):
    from cyclic_product_graphs import synthetic

    p = synthetic.make_pair(icosphere_level=level, n_curve=m, feat_dim=8, seed=seed)
    g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, False)
    if conj:
        g.set_normals(p["NX"], p["NY"])
        g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    return g


def _check_two_in_a_row(lib, g):
    ref = _export(lib, g, "pgc_get_cost_vector")
    first = _export(lib, g, "pgc_get_cost_vector_noalloc")
    second = _export(lib, g, "pgc_get_cost_vector_noalloc")
    assert np.array_equal(first, ref)
    assert np.array_equal(second, ref)
    return ref


@pytest.mark.parametrize("conj", [False, True])
def test_noalloc_export_matches_existing_entry_point(cpg, conj):
    lib = _abi(cpg)
    g = _graph(cpg, conj)
    g.generate()
    before = _check_two_in_a_row(lib, g)
    assert np.isfinite(before).all()
    # a ratio solve rescales the costs in place; both exports see it
    g.solve_with_cost_time_ratio("lawlergpu", 2)
    after = _check_two_in_a_row(lib, g)
    assert not np.array_equal(before, after)


def test_noalloc_export_pruned_graph(cpg):
    """Pruned graphs have no intralayer edges: the export must still write
    every value of the smaller edge blocks, into a NaN-filled buffer."""
    lib = _abi(cpg)
    from cyclic_product_graphs import synthetic

    for conj in (False, True):
        p = synthetic.make_pair(icosphere_level=1, n_curve=8, feat_dim=8, seed=5)
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, True)
        if conj:
            g.set_normals(p["NX"], p["NY"])
            g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
        g.generate()
        ref = _check_two_in_a_row(lib, g)
        assert np.isfinite(ref).all()


@pytest.mark.parametrize("conj", [False, True])
def test_noalloc_export_of_imported_costs(cpg, conj):
    """Costs set with pgc_set_cost_vector instead of generated: the export
    returns exactly the imported matrix, every value finite."""
    lib = _abi(cpg)
    g = _graph(cpg, conj, seed=7)
    rows, cols = g.get_cost_vector().shape
    rng = np.random.default_rng(3)
    costs = rng.integers(1, 1000, size=(rows, cols)).astype(np.float64)
    g.set_cost_vector(costs)
    ref = _check_two_in_a_row(lib, g)
    assert np.array_equal(ref, costs)


def test_noalloc_export_alternates_between_graphs(cpg):
    lib = _abi(cpg)
    a, b = _graph(cpg, False, seed=1), _graph(cpg, True, seed=2)
    a.generate()
    b.generate()
    for g in (a, b, a):
        _check_two_in_a_row(lib, g)


def test_noalloc_export_needs_generated_costs(cpg):
    lib = _abi(cpg)
    g = _graph(cpg, False)
    out = np.zeros(16)
    assert lib.pgc_get_cost_vector_noalloc(g._h, out.ctypes.data_as(ctypes.c_void_p)) == PGC_ERR_STATE
    assert b"generate" in lib.pgc_last_error()


def test_noalloc_export_rejects_more_than_its_scratch(cpg):
    lib = _abi(cpg)
    g = _graph(cpg, False, level=4, m=100)
    g.generate()
    rows, cols = _shape(lib, g)
    assert rows * cols > MAX_VALUES
    out = np.zeros(16)
    assert lib.pgc_get_cost_vector_noalloc(g._h, out.ctypes.data_as(ctypes.c_void_p)) == PGC_ERR_ARG
    assert b"at most 2097152" in lib.pgc_last_error()
    # the graph is still usable through the allocating export afterwards
    full = _export(lib, g, "pgc_get_cost_vector")
    assert full.shape == (rows, cols) and np.isfinite(full).all()
