"""compute_normals_2d / compute_normals_3d run on the device and must equal,
bit for bit, the oracle's restatement of the reference's host helpers
(utils::normals2d / normals3d, helper/utils.cpp:86-157; libigl's area-weighted
per_vertex_normals): same operations, same order.  Covered: meshes from 12
to 20,000 vertices (perturbed), faces with a repeated vertex (zero area),
curves in each coordinate plane, curves flipped inward, two- and three-point
curves, and the argument errors."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _perturbed(V, F, seed):
    rng = np.random.default_rng(seed)
    return V * (1.0 + 0.1 * rng.standard_normal((len(V), 1))), F


@pytest.mark.parametrize("level", [0, 1, 3, 5])
def test_normals_3d_icospheres(cpg, oracle, level):
    V, F = _perturbed(*synthetic.icosphere(level), seed=level)
    assert np.array_equal(cpg.compute_normals_3d(V, F), oracle.normals_3d(V, F))


@pytest.mark.parametrize("n", [5000, 20000])
def test_normals_3d_benchmark_meshes(cpg, oracle, n):
    V, F = _perturbed(*synthetic.fibonacci_sphere(n), seed=n)
    assert np.array_equal(cpg.compute_normals_3d(V, F), oracle.normals_3d(V, F))


def test_normals_3d_degenerate_faces_and_isolated_vertices(cpg, oracle):
    V, F = _perturbed(*synthetic.icosphere(2), seed=3)
    F = np.vstack([F, [[0, 0, 1], [2, 3, 3]]]).astype(np.int32)  # zero-area faces, listed twice at a corner
    V = np.vstack([V, [[5.0, 5.0, 5.0]]])                       # a vertex in no face: normal 0
    got = cpg.compute_normals_3d(V, F)
    assert np.array_equal(got, oracle.normals_3d(V, F))
    assert np.array_equal(got[-1], np.zeros(3))


def test_normals_3d_rejects_out_of_range_faces(cpg):
    V, F = synthetic.icosphere(1)
    F = F.copy()
    F[3, 1] = len(V)
    with pytest.raises(cpg.PGCError, match="outside"):
        cpg.compute_normals_3d(V, F)


def _curve(m, plane, center=(3.0, 1.0), clockwise=False):
    t = np.linspace(0, 2 * np.pi, m, endpoint=False)
    if clockwise:
        t = -t
    a = center[0] + 2 * np.cos(t) + 0.3 * np.cos(5 * t)
    b = center[1] + np.sin(t)
    V = np.zeros((m, 3))
    cols = {"xy": (0, 1), "xz": (0, 2), "yz": (1, 2)}[plane]
    V[:, cols[0]], V[:, cols[1]] = a, b
    E = np.stack([np.arange(m), (np.arange(m) + 1) % m], axis=1).astype(np.int32)
    return V, E


@pytest.mark.parametrize("plane", ["xy", "xz", "yz"])
@pytest.mark.parametrize("clockwise", [False, True])
@pytest.mark.parametrize("m", [3, 60, 500, 2049])
def test_normals_2d_curves(cpg, oracle, plane, clockwise, m):
    V, E = _curve(m, plane, clockwise=clockwise)
    assert np.array_equal(cpg.compute_normals_2d(V, E), oracle.normals_2d(V, E))


def test_normals_2d_benchmark_curve(cpg, oracle):
    p = synthetic.make_pair(n_vertices=5000, n_curve=200, feat_dim=4, seed=1)
    V = p["VY"] + np.array([10.0, 10.0, 0.0])
    assert np.array_equal(cpg.compute_normals_2d(V, p["EY"]), oracle.normals_2d(V, p["EY"]))


def test_normals_2d_two_points_and_repeated_points(cpg, oracle):
    V, E = _curve(2, "xy")
    assert np.array_equal(cpg.compute_normals_2d(V, E), oracle.normals_2d(V, E))  # cancelling normals stay 0
    V, E = _curve(12, "xy")
    V[5] = V[4]  # a zero-length edge
    assert np.array_equal(cpg.compute_normals_2d(V, E), oracle.normals_2d(V, E))


def test_normals_2d_errors(cpg):
    V = np.random.default_rng(0).normal(size=(5, 3)) + 1.0
    E = np.stack([np.arange(5), (np.arange(5) + 1) % 5], axis=1)
    with pytest.raises(cpg.PGCError, match="plane"):
        cpg.compute_normals_2d(V, E)
    V, E = _curve(6, "xy")
    E = E.copy()
    E[2, 1] = 6
    with pytest.raises(cpg.PGCError, match="outside"):
        cpg.compute_normals_2d(V, E)
    with pytest.raises(cpg.PGCError, match="rows"):
        cpg.compute_normals_2d(V, E[:5])
