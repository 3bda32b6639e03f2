"""C ABI of libpgc.so without a GPU: the library loads, exports every entry
point that include/pgc.h declares, and its host-only helpers and argument
checks behave like the reference.  (The normals helpers run on the device:
tests/test_gpu_normals.py; their restatement in the oracle is checked on the
CPU in tests/test_oracle_normals.py.)"""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pgc.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pgc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(cpg):
    lib = ctypes.CDLL(cpg.library_path)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_library_is_sm100a_build(cpg):
    assert "sm_100a" in cpg.version()


def test_create_rejects_bad_shapes(cpg):
    VX = np.zeros((4, 3))
    EX = np.array([[0, 1], [1, 0]], dtype=np.int32)
    VY = np.zeros((3, 3))
    EY = np.array([[0, 1], [1, 2], [2, 0]], dtype=np.int32)
    with pytest.raises(ValueError, match="feat_diff"):
        cpg.product_graph_generator(VX, EX, VY, EY, np.zeros((3, 3)), False, False)
    with pytest.raises(ValueError):
        cpg.product_graph_generator(VX[:, :2], EX, VY, EY, np.zeros((4, 3)), False, False)


def test_null_arguments_return_arg_error(cpg):
    lib = ctypes.CDLL(cpg.library_path)
    lib.pgc_create.restype = ctypes.c_int
    out = ctypes.c_void_p()
    rc = lib.pgc_create(None, 0, None, 0, None, 0, None, 0, None, 0, 0, 0, ctypes.byref(out))
    assert rc == -1
    lib.pgc_last_error.restype = ctypes.c_char_p
    assert b"null" in lib.pgc_last_error()


def test_local_thickness_stubs_match_reference(cpg, capsys):
    cpg.compute_local_thickness_3d()
    cpg.compute_local_thickness_2d()
    assert capsys.readouterr().out == "TODO: IMPL\nTODO: IMPL\n"


# (name, argument types after the handle); every value passed is zero / null
_HANDLE_CALLS = [
    ("pgc_set_normals", [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                         ctypes.c_int64]),
    ("pgc_set_max_depth", [ctypes.c_int]),
    ("pgc_set_cost_time_ratio_mode", [ctypes.c_char_p, ctypes.c_char_p]),
    ("pgc_update_robust_loss_params", [ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    ("pgc_set_stream", [ctypes.c_void_p]),
    ("pgc_generate", []),
    ("pgc_cost_vector_shape", [ctypes.c_void_p, ctypes.c_void_p]),
    ("pgc_get_cost_vector", [ctypes.c_void_p]),
    ("pgc_get_cost_vector_noalloc", [ctypes.c_void_p]),
    ("pgc_product_space_shape", [ctypes.c_void_p, ctypes.c_void_p]),
    ("pgc_get_product_space", [ctypes.c_void_p]),
    ("pgc_solve_with_cost_time_ratio", [ctypes.c_char_p, ctypes.c_int]),
    ("pgc_solve_with_minimum_cost", [ctypes.c_char_p, ctypes.c_int]),
    ("pgc_backward_feat_diff", [ctypes.c_double, ctypes.c_void_p, ctypes.c_int]),
    ("pgc_set_cost_vector", [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]),
    ("pgc_set_feat_diff", [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]),
    ("pgc_set_team_cap", [ctypes.c_int]),
    ("pgc_set_team_shape", [ctypes.c_int, ctypes.c_int]),
    ("pgc_result", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pgc_result_matching", [ctypes.c_void_p]),
    ("pgc_result_cycle_edges", [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    ("pgc_result_stats", [ctypes.c_void_p]),
    ("pgc_result_profile", [ctypes.c_void_p]),
    ("pgc_result_profile_detail", [ctypes.c_void_p]),
    ("pgc_graph_info", [ctypes.c_void_p]),
    ("pgc_device_name", [ctypes.c_char_p, ctypes.c_int64]),
]


@pytest.mark.parametrize("name,argtypes", _HANDLE_CALLS, ids=[c[0] for c in _HANDLE_CALLS])
def test_null_handle_is_an_argument_error(cpg, name, argtypes):
    """Every entry point that takes a handle answers a null one with
    PGC_ERR_ARG instead of dereferencing it (no GPU is touched first)."""
    lib = ctypes.CDLL(cpg.library_path)
    fn = getattr(lib, name)
    fn.argtypes = [ctypes.c_void_p] + argtypes
    fn.restype = ctypes.c_int
    assert fn(None, *[t(0) if t is not ctypes.c_char_p else None for t in argtypes]) == -1
    lib.pgc_last_error.restype = ctypes.c_char_p
    assert b"null" in lib.pgc_last_error()


def test_null_arrays_are_argument_errors(cpg):
    lib = ctypes.CDLL(cpg.library_path)
    lib.pgc_last_error.restype = ctypes.c_char_p
    for name in ("pgc_compute_normals_2d", "pgc_compute_normals_3d"):
        fn = getattr(lib, name)
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        assert fn(None, 3, None, 3, None) == -1
        assert b"null" in lib.pgc_last_error()
    lib.pgc_solve_batch.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    assert lib.pgc_solve_batch(None, 2, b"lawlergpu", 2, 0, 0, 0, None) == -1
    lib.pgc_product_graph_sizes.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    assert lib.pgc_product_graph_sizes(None, 4, 4, 3, 0, 0, None) == -1
    lib.pgc_destroy.argtypes = [ctypes.c_void_p]
    lib.pgc_destroy(None)  # a no-op
