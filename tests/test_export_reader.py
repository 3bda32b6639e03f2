"""load_export reads the files of the "export" solver without a GPU: one row
per line, values separated by ", ", doubles with 17 significant digits
(product_graph_generators.cpp:272-282 writes VX, VY, EX, EY, FeatDiffMatrix
and, for a conjugate graph, NX and NY), so the arrays come back exactly."""
import numpy as np


def _write(path, m, fmt):
    m = np.atleast_2d(m)
    with open(path, "w") as f:
        f.write("\n".join(", ".join(fmt % x for x in row) for row in m))


def test_load_export_round_trips_exactly(cpg, tmp_path):
    rng = np.random.default_rng(5)
    arrays = {"VX": rng.normal(size=(7, 3)), "VY": rng.normal(size=(5, 3)) * 1e-7,
              "EX": rng.integers(0, 7, size=(9, 2)).astype(np.int32), "EY": np.array([[0, 1], [1, 2], [2, 0]], np.int32),
              "FeatDiffMatrix": rng.random((7, 5)) * 1e3, "NX": rng.normal(size=(7, 3)), "NY": rng.normal(size=(5, 3))}
    for name, m in arrays.items():
        _write(tmp_path / f"{name}.csv", m, "%d" if m.dtype.kind == "i" else "%.17g")
    d = cpg.load_export(str(tmp_path))
    for key, name in (("VX", "VX"), ("VY", "VY"), ("EX", "EX"), ("EY", "EY"), ("feat_diff", "FeatDiffMatrix"),
                      ("NX", "NX"), ("NY", "NY")):
        assert d[key].shape == arrays[name].shape, key
        assert np.array_equal(d[key], arrays[name]), key
    assert d["EX"].dtype == np.int32 and d["feat_diff"].dtype == np.float64


def test_load_export_without_normals(cpg, tmp_path):
    for name, m in {"VX": np.eye(3), "VY": np.eye(3), "EX": np.array([[0, 1], [1, 2], [2, 0]]),
                    "EY": np.array([[0, 1], [1, 0]]), "FeatDiffMatrix": np.ones((3, 3))}.items():
        _write(tmp_path / f"{name}.csv", m, "%d" if np.asarray(m).dtype.kind == "i" else "%.17g")
    d = cpg.load_export(str(tmp_path))
    assert "NX" not in d and "NY" not in d
    assert d["EY"].shape == (2, 2)
