"""The oracle's restatement of the reference's normals helpers
(utils::normals2d / normals3d, helper/utils.cpp:86-157), on the CPU, against
independent numpy restatements: the checker the device normals are compared
with (tests/test_gpu_normals.py)."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic


def test_normals_2d_matches_reference_rule(oracle):
    m = 37
    t = np.linspace(0, 2 * np.pi, m, endpoint=False)
    # off the origin: the reference picks the plane by the first coordinate
    # column whose SUM is ~0 (utils.cpp:102-108), so a centred curve would be
    # taken to lie in the yz-plane
    V = np.stack([3 + 2 * np.cos(t), 1 + np.sin(t), np.zeros(m)], axis=1)
    E = np.stack([np.arange(m), (np.arange(m) + 1) % m], axis=1).astype(np.int32)
    got = oracle.normals_2d(V, E)
    np.testing.assert_allclose(got, synthetic.normals_2d(V, E), atol=1e-12)
    assert got[0, 0] > 0.99  # outward: the normal at the rightmost point points to +x


def test_normals_2d_rejects_non_planar(oracle):
    V = np.random.default_rng(0).normal(size=(5, 3)) + 1.0
    E = np.stack([np.arange(5), (np.arange(5) + 1) % 5], axis=1)
    with pytest.raises(ValueError, match="plane"):
        oracle.normals_2d(V, E)


def test_normals_3d_area_weighted(oracle):
    V, F = synthetic.icosphere(2)
    got = oracle.normals_3d(V, F)
    np.testing.assert_allclose(got, synthetic.vertex_normals(V, F), atol=1e-12)
    np.testing.assert_allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-12)
    # on the unit sphere the normals are the positions
    np.testing.assert_allclose(got, V / np.linalg.norm(V, axis=1, keepdims=True), atol=0.05)


def test_normals_3d_rejects_out_of_range_faces(oracle):
    V, F = synthetic.icosphere(1)
    F = F.copy()
    F[3, 1] = len(V)
    with pytest.raises(ValueError, match="outside"):
        oracle.normals_3d(V, F)
