"""The MATLAB entry point (product-graph-cycles_b200/mex/product_graph_generator_mex.cpp)
built against a small fake of MATLAB's mex API (tests/mex_fake) and driven
from Python: argument forms of 8, 12 and 14 inputs, 1-based indices, the
reference's solver-id dispatch and messages, and results equal to the Python
API's on the same pair."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def mex(tmp_path_factory, cpg):
    out = tmp_path_factory.mktemp("mex") / "libmexshim.so"
    lib = os.path.dirname(cpg.library_path)
    subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(ROOT, "tests", "mex_fake"),
                    "-I", os.path.join(ROOT, "include"), "-o", str(out),
                    os.path.join(ROOT, "product-graph-cycles_b200", "mex", "product_graph_generator_mex.cpp"),
                    os.path.join(ROOT, "tests", "mex_fake", "mex_fake.cpp"), "-L", lib, "-lpgc",
                    f"-Wl,-rpath,{lib}"], check=True)
    m = ctypes.CDLL(str(out))
    m.fake_mx_new.restype = ctypes.c_void_p
    m.fake_mx_new.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p]
    m.fake_mx_free.argtypes = [ctypes.c_void_p]
    m.mxGetM.restype = m.mxGetN.restype = ctypes.c_size_t
    m.mxGetM.argtypes = m.mxGetN.argtypes = [ctypes.c_void_p]
    m.mxGetPr.restype = ctypes.POINTER(ctypes.c_double)
    m.mxGetPr.argtypes = [ctypes.c_void_p]
    m.fake_mex_output.restype = m.fake_mex_error.restype = ctypes.c_char_p
    m.fake_mex_call.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    return m


def _call(mex, args, nlhs=3):
    prhs = (ctypes.c_void_p * len(args))()
    for i, a in enumerate(args):
        a = np.atleast_2d(np.asarray(a, dtype=np.float64))
        col = np.asfortranarray(a)
        prhs[i] = mex.fake_mx_new(a.shape[0], a.shape[1], col.ctypes.data)
    plhs = (ctypes.c_void_p * 3)()
    rc = mex.fake_mex_call(nlhs, plhs, len(args), prhs)
    outs = []
    if rc == 0:
        for j in range(nlhs):
            m, n = mex.mxGetM(plhs[j]), mex.mxGetN(plhs[j])
            data = np.ctypeslib.as_array(mex.mxGetPr(plhs[j]), shape=(m * n,)) if m * n else np.zeros(0)
            outs.append(np.array(data).reshape((m, n), order="F"))
            mex.fake_mx_free(plhs[j])
    for i in range(len(args)):
        mex.fake_mx_free(prhs[i])
    return rc, outs, mex.fake_mex_output().decode(), mex.fake_mex_error().decode()


def _pair(level=1, m=8, seed=0):
    from cyclic_product_graphs import synthetic

    return synthetic.make_pair(icosphere_level=level, n_curve=m, feat_dim=8, seed=seed)


def _base_args(p, conj, solver_id):
    return [p["VX"], p["EX"] + 1, p["VY"], p["EY"] + 1, p["feat_diff"], float(conj), 0.0, float(solver_id)]


def test_usage_error_for_a_wrong_argument_count(mex):
    rc, _, _, err = _call(mex, [np.zeros((1, 1))] * 7)
    assert rc == 1 and err.startswith("Usage: [passes_layers_once")


@pytest.mark.gpu
def test_ratio_solve_with_twelve_inputs_matches_the_python_api(mex, cpg):
    p = _pair(seed=1)
    rc, (passes, obj, matching), out, err = _call(mex, _base_args(p, False, 6) + [0.0, 2.0, 0.0, -1.0])
    assert rc == 0, err
    # -1 maps to "nomode" and still prints the reference's error line
    assert "pruneIntralayerEdges 0" in out and "[CPG-MEX] error: id not supported" in out
    g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False, False)
    g.set_cost_time_ratio_mode("vanilla", "nomode")
    want = g.solve_with_cost_time_ratio("lawlergpu", 2)
    assert passes[0, 0] == float(want[0]) and obj[0, 0] == float(np.float32(want[1]))
    assert np.array_equal(matching, want[2].astype(np.float64) + 1)


@pytest.mark.gpu
def test_min_cost_conjugate_with_fourteen_inputs_matches_the_python_api(mex, cpg):
    p = _pair(seed=2)
    args = _base_args(p, True, 8) + [0.0, 3.0, 0.0, 2.0, p["NX"], p["NY"]]
    rc, (passes, obj, matching), _, err = _call(mex, args)
    assert rc == 0, err
    g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], True, False, False)
    g.set_normals(p["NX"], p["NY"])
    g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    want = g.solve_with_minimum_cost("dijkstragpu", 3)
    assert passes[0, 0] == float(want[0]) and obj[0, 0] == float(np.float32(want[1]))
    assert matching.shape == want[2].shape and np.array_equal(matching, want[2] + 1.0)


@pytest.mark.gpu
def test_eight_inputs_use_the_generator_defaults(mex, cpg):
    p = _pair(seed=3)
    rc, (passes, obj, matching), out, err = _call(mex, _base_args(p, False, 5))
    assert rc == 0, err
    assert "pruneIntralayerEdges" not in out
    g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False, False)
    want = g.solve_with_cost_time_ratio("lawlercpu")
    assert obj[0, 0] == float(np.float32(want[1])) and np.array_equal(matching, want[2] + 1.0)


@pytest.mark.gpu
def test_other_solver_ids_are_not_supported(mex):
    p = _pair(seed=4)
    rc, (passes, obj, matching), out, err = _call(mex, _base_args(p, False, -1))
    assert rc == 0, err
    assert "solver not supported" in out
    assert passes[0, 0] == 0 and obj[0, 0] == 0 and matching.size == 0
