"""Pins the CPU oracle against exact known answers (tests/golden/toy_cases.json,
tests/golden/mesh_cases.json, tests/golden/pruned_cases.json,
tests/golden/conj_cases.json).

The fixtures come from tests/golden/make_golden.py, which builds the toy
product graphs, their costs and the rescale from their definitions and finds
the optima by exact enumeration -- independently of the oracle.
"""
import hashlib
import json
import math
import os
from fractions import Fraction

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "toy_cases.json")) as f:
    CASES = json.load(f)["cases"]
with open(os.path.join(HERE, "golden", "conj_cases.json")) as f:
    CONJ_CASES = json.load(f)["cases"]
with open(os.path.join(HERE, "golden", "pruned_cases.json")) as f:
    PRUNED_CASES = json.load(f)["cases"]
with open(os.path.join(HERE, "golden", "mesh_cases.json")) as f:
    MESH_CASES = json.load(f)["cases"]


def _arrays(c):
    return (np.array(c["VX"]), np.array(c["EX"], dtype=np.int32), np.array(c["VY"]), np.array(c["EY"], dtype=np.int32),
            np.array(c["feat_diff"]))


def check_case(gen_factory, c):
    """Ratio solve, then min-cost on the rescaled costs, then min-cost on raw costs."""
    VX, EX, VY, EY, fd = _arrays(c)
    g = gen_factory(VX, EX, VY, EY, fd)
    g.set_cost_time_ratio_mode("vanilla", "nomode")
    passes, obj, m = g.solve_with_cost_time_ratio("lawlercpu", c["K"])
    want = Fraction(c["ratio"][0], c["ratio"][1])
    assert passes
    assert obj == np.float32(float(want)), (obj, float(want))
    edges = sorted(g.last_cycle_edges().tolist())
    assert edges in c["ratio_cycles"], "returned ratio cycle is not one of the optimal cycles"
    assert m.shape == (len(edges), 4)

    passes, obj, m = g.solve_with_minimum_cost("dijkstracpu", c["K"])
    assert passes
    assert obj == np.float32(c["min_cost_after_ratio"])
    assert sorted(g.last_cycle_edges().tolist()) in c["min_cost_after_ratio_cycles"]

    g2 = gen_factory(VX, EX, VY, EY, fd)
    passes, obj, m = g2.solve_with_minimum_cost("dijkstracpu", c["K"])
    want = Fraction(c["min_cost_raw"][0], c["min_cost_raw"][1])
    assert obj == np.float32(float(want))
    assert sorted(g2.last_cycle_edges().tolist()) in c["min_cost_raw_cycles"]


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_known_answers(oracle, c):
    check_case(lambda *a: oracle.OracleGenerator(*a, False, False), c)


def test_fixture_product_space_matches_oracle(oracle):
    """The fixture generator's product graph equals the oracle's restatement."""
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    c = CASES[0]
    VX, EX, VY, EY, fd = _arrays(c)
    ps, src, trgt = make_golden.plain_product(EX, EY, VX.shape[0])
    o = oracle.OracleGenerator(VX, EX, VY, EY, fd, False, False)
    assert np.array_equal(o.get_product_space(), ps)
    s2, t2 = o.get_src_trgt()
    assert np.array_equal(s2, np.array(src)) and np.array_equal(t2, np.array(trgt))


def check_bounded_plain_case(make, c):
    """Plain graph (pruned or on an icosphere): product space digest; the
    ratio against its own cycle and, from below, against the optimum (the
    reference's Lawler can stop above it); the exact minimum cost on the
    rescaled and on the raw costs."""
    VX, EX, VY, EY, fd = _arrays(c)
    prune = c.get("prune", False)
    g = make(VX, EX, VY, EY, fd, False, False, prune)
    ps = g.get_product_space()
    assert _digest(ps) == c["rows_digest"]
    g.set_cost_time_ratio_mode("vanilla", "nomode")
    passes, obj, m = g.solve_with_cost_time_ratio("lawlercpu", c["K"])
    assert passes
    e = g.last_cycle_edges()
    assert m.shape == (len(e), 4) and np.array_equal(m, ps[e])
    scaled = g.get_cost_vector()[:, 0]
    assert obj == pytest.approx(scaled[e].sum() / (50000.0 * len(e)), rel=1e-6)
    assert obj >= np.float32(float(Fraction(*c["ratio"]))) * (1 - 1e-6)

    passes, obj, m = g.solve_with_minimum_cost("dijkstracpu", c["K"])
    assert passes
    assert obj == np.float32(c["min_cost_after_ratio"])
    assert sorted(g.last_cycle_edges().tolist()) in c["min_cost_after_ratio_cycles"]

    g2 = make(VX, EX, VY, EY, fd, False, False, prune)
    passes, obj, m = g2.solve_with_minimum_cost("dijkstracpu", c["K"])
    assert passes
    assert obj == np.float32(float(Fraction(*c["min_cost_raw"])))
    assert sorted(g2.last_cycle_edges().tolist()) in c["min_cost_raw_cycles"]


BOUNDED_PLAIN_CASES = MESH_CASES + PRUNED_CASES


@pytest.mark.parametrize("c", BOUNDED_PLAIN_CASES, ids=[c["name"] for c in BOUNDED_PLAIN_CASES])
def test_oracle_matches_bounded_plain_known_answers(oracle, c):
    check_bounded_plain_case(oracle.OracleGenerator, c)
    VX, EX, VY, EY, fd = _arrays(c)
    s_, t_ = oracle.OracleGenerator(VX, EX, VY, EY, fd, False, False, c.get("prune", False)).get_src_trgt()
    assert _digest(s_, t_) == c["src_trgt_digest"]


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(np.asarray(a, dtype="<i4")).tobytes())
    return h.hexdigest()


def conj_generator(make, c):
    """A conjugate generator on the case's graph with its cost/time matrix set
    (feature differences and normals are placeholders: no energy is used)."""
    VX, EX, VY = np.array(c["VX"]), np.array(c["EX"], dtype=np.int32), np.array(c["VY"])
    EY = np.array(c["EY"], dtype=np.int32)
    g = make(VX, EX, VY, EY, np.ones((len(VX), len(VY))), True, False, c["prune"])
    g.set_normals(VX / np.linalg.norm(VX, axis=1, keepdims=True), np.tile([0.0, 0.0, 1.0], (len(VY), 1)))
    g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    g.set_cost_vector(np.array(c["cost_time_e4"]) / 1e4)
    return g


def check_conj_case(make, c):
    """Product space digest, then the bounds the reference's solvers keep on a
    conjugate graph.  Neither solver is exact there: Lawler stops when the
    cycle of the best Bellman-Ford candidate is not negative
    (cost_time_ratio_solver.cpp:443-489), and the minimum-cost branch and
    bound returns the first branch popped with a valid bound even after a
    cheaper cycle was found past the first candidate of another branch
    (dijkstra_solver.cpp:455-461, :361-371).  So each objective is checked
    against its own cycle and against the exact optimum from below; with
    K = 1 a 2D-degenerate upper-bound start gives a 0/0 ratio and no cycle."""
    g = conj_generator(make, c)
    ps = g.get_product_space()
    assert ps.shape == (c["product_rows"], 6)
    assert _digest(ps) == c["rows_digest"]
    raw = np.array(c["cost_time_e4"]) / 1e4

    passes, obj, m = g.solve_with_cost_time_ratio("lawlercpu", c["K"])
    assert passes
    start, kind = c["ratio_upper_bound_start"]
    scaled = g.get_cost_vector()  # rescaled in place by the ratio solve
    if c["K"] == 1 and kind == "degenerate2d":
        assert np.isnan(obj) and m.shape[0] == 0
    else:
        e = g.last_cycle_edges()
        assert m.shape == (len(e), 6) and np.array_equal(m, ps[e])
        assert obj == pytest.approx(scaled[e, 0].sum() / scaled[e, 1].sum(), rel=1e-6)
        assert obj >= np.float32(float(Fraction(*c["ratio_optimum"]))) * (1 - 1e-6)

    passes, obj, m = g.solve_with_minimum_cost("dijkstracpu", c["K"])
    e = g.last_cycle_edges()
    assert passes and m.shape == (len(e), 6) and np.array_equal(m, ps[e])
    assert obj == pytest.approx(scaled[e, 0].sum(), rel=1e-6)
    assert obj >= np.float32(c["min_cost_after_ratio"])

    g2 = conj_generator(make, c)
    passes, obj, m = g2.solve_with_minimum_cost("dijkstracpu", c["K"])
    e = g2.last_cycle_edges()
    assert passes and m.shape == (len(e), 6) and np.array_equal(m, ps[e])
    assert obj == pytest.approx(raw[e, 0].sum(), rel=1e-6)
    assert obj >= np.float32(float(Fraction(*c["min_cost_raw"]))) * (1 - 1e-6)


@pytest.mark.parametrize("c", CONJ_CASES, ids=[c["name"] for c in CONJ_CASES])
def test_oracle_matches_conjugate_known_answers(oracle, c):
    check_conj_case(oracle.OracleGenerator, c)
    s, t = conj_generator(oracle.OracleGenerator, c).get_src_trgt()
    assert _digest(s, t) == c["src_trgt_digest"]


@pytest.mark.parametrize("ny", [2, 3, 5])
@pytest.mark.parametrize("kind", ["plain", "plain_pruned", "conj", "conj_pruned"])
@pytest.mark.parametrize("mesh", ["tetrahedron", "octahedron"])
def test_fixture_generators_match_oracle_product_spaces(oracle, mesh, kind, ny):
    """The fixture script's product spaces (restated from product_space.cpp
    and conj_product_space.cpp) equal the oracle's, rows and SRC/TRGT, also
    for layer counts the fixtures do not hold (two layers included)."""
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    VX, und = make_golden.MESHES[mesh]
    EX = make_golden.directed(und)
    t = np.linspace(0, 2 * np.pi, ny, endpoint=False)
    VY = np.stack([np.cos(t), np.sin(t), np.zeros(ny)], axis=1)
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    conj, prune = kind.startswith("conj"), kind.endswith("pruned")
    if conj:
        ps, src, trgt = make_golden.conj_product(EX, EY, prune)
    else:
        ps, src, trgt = make_golden.plain_product(EX, EY, len(VX), prune)
    o = oracle.OracleGenerator(VX, EX, VY, EY, np.ones((len(VX), ny)), conj, False, prune)
    if conj:
        o.set_normals(VX / np.linalg.norm(VX, axis=1, keepdims=True), np.tile([0.0, 0.0, 1.0], (ny, 1)))
    assert np.array_equal(o.get_product_space(), ps)
    s_, t_ = o.get_src_trgt()
    assert np.array_equal(s_, np.array(src)) and np.array_equal(t_, np.array(trgt))


def _plain_energy(VX, VY, fd, ps, reg, cost, time):
    """deformationEnergy.cpp:11-78 restated in numpy, in its operation order:
    L = sqrt of the squared coordinate differences summed per axis, the Y
    one before the X one (1 without the regulariser unless the mode needs
    it); one column 0.5 * (fd0 + fd1) * L, or for ("feature",
    "lengthnormalisation") the two columns fd0 + fd1 and L."""
    y0, y1, x0, x1 = ps[:, 0], ps[:, 1], ps[:, 2], ps[:, 3]
    two = cost == "feature" and time == "lengthnormalisation"
    if reg or two:
        L = np.zeros(len(ps))
        for j in range(3):
            dy = VY[y0, j] - VY[y1, j]
            dx = VX[x0, j] - VX[x1, j]
            L = L + dy * dy
            L = L + dx * dx
        L = np.sqrt(L)
    else:
        L = np.ones(len(ps))
    f = fd[x0, y0] + fd[x1, y1]
    return np.stack([f, L], axis=1) if two else ((0.5 * f) * L)[:, None]


@pytest.mark.parametrize("prune", [False, True])
@pytest.mark.parametrize("reg", [False, True])
@pytest.mark.parametrize("cost,time", [("vanilla", "nomode"), ("feature", "lengthnormalisation"),
                                       ("vanilla", "lengthnormalisation"), ("feature", "")])
def test_oracle_plain_energy_matches_the_restatement(oracle, cost, time, reg, prune):
    """The oracle's plain-graph costs equal deformationEnergy.cpp restated
    here, bit for bit, on a perturbed octahedron."""
    rng = np.random.default_rng(7)
    V, und = MESHES_FOR_ENERGY
    VX = V * (1 + 0.2 * rng.random((len(V), 1)))
    EX = np.array(sorted([(a, b) for a, b in und] + [(b, a) for a, b in und]), dtype=np.int32)
    ny = 5
    t = np.linspace(0, 2 * np.pi, ny, endpoint=False)
    VY = np.stack([np.cos(t), np.sin(t), 0.3 * rng.random(ny)], axis=1)
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    fd = rng.uniform(0.1, 2.0, size=(len(VX), ny))
    o = oracle.OracleGenerator(VX, EX, VY, EY, fd, False, reg, prune)
    o.set_cost_time_ratio_mode(cost, time)
    got = o.get_cost_vector()
    want = _plain_energy(VX, VY, fd, o.get_product_space(), reg, cost, time)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


MESHES_FOR_ENERGY = (np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=np.float64),
                     [(0, 2), (0, 3), (0, 4), (0, 5), (1, 2), (1, 3), (1, 4), (1, 5), (2, 4), (2, 5), (3, 4), (3, 5)])


def _mode(name):
    """stringToMode (higherOrderDeformationEnergy.cpp:396-412), with its
    missing `== 0`: "penalisedegenerate" maps to vanilla and every unknown
    name to penalise-degenerate."""
    known = {"nomode": "nomode", "vanilla": "vanilla", "feature": "feature", "lengthnormalisation": "length",
             "plainso3": "so3plain", "robustso3": "so3robust"}
    if name in known:
        return known[name]
    return "vanilla" if name == "penalisedegenerate" else "penalise"


def _robust(x, alpha=0.7, c=0.6, pwr=4.0):
    """robustSO3Dif (higherOrderDeformationEnergy.cpp:55-63), same operations."""
    a2 = abs(alpha - 2)
    return a2 / alpha * (math.pow(math.pow(x / c, pwr) / a2 + 1, 0.5 * alpha) - 1)


def _conj_energy_without_so3(VX, VY, fd, ps, cost, time):
    """higherOrderDeformationEnergy.cpp:209-339 without the regulariser (the
    SO(3) distance is 0, and so is its robust loss).  The column-1 writes of
    the one-column modes fall outside the matrix in the reference; they are
    left out."""
    cm, tm = _mode(cost), _mode(time)
    y0, y1, y2, x0, x1, x2 = (ps[:, i] for i in range(6))
    f = fd[x2, y2]
    L = np.zeros(len(ps))
    for j in range(3):
        dy = VY[y0, j] - VY[y1, j]
        dx = VX[x0, j] - VX[x1, j]
        L = L + dy * dy
        L = L + dx * dx
    L = np.sqrt(L)
    so3 = _robust(0.0)
    deg = np.where((y2 == y1) | (x2 == x1), 0.1, 1.0)
    two_pi = 2 * math.pi
    maxso3 = float(np.float32(_robust(two_pi)))
    maxfd = float(np.float32(fd.max()))
    table = {
        ("vanilla", "vanilla"): [so3 + f],
        ("vanilla", "length"): [so3 + f, L],
        ("length", "vanilla"): [L],
        ("vanilla", "penalise"): [so3 + f, deg],
        ("penalise", "vanilla"): [deg],
        ("feature", "so3plain"): [f, np.maximum(0.0, two_pi - 0.0) + 0 * f],
        ("feature", "so3robust"): [f, np.maximum(0.0, maxso3 - so3) + 0 * f],
        ("so3robust", "feature"): [so3 + 0 * f, np.maximum(0.0, maxfd - f)],
        ("so3plain", "feature"): [0.0 * f, np.maximum(0.0, maxfd - f)],
    }
    return np.stack(table[(cm, tm)], axis=1)


@pytest.mark.parametrize("prune", [False, True])
@pytest.mark.parametrize("cost,time", [("vanilla", "vanilla"), ("vanilla", "lengthnormalisation"),
                                       ("lengthnormalisation", "vanilla"), ("vanilla", ""),
                                       ("", "vanilla"), ("penalisedegenerate", "vanilla"),
                                       ("feature", "plainso3"), ("feature", "robustso3"),
                                       ("robustso3", "feature"), ("plainso3", "feature")])
def test_oracle_conjugate_energy_matches_the_restatement(oracle, cost, time, prune):
    """The oracle's conjugate-graph costs without the regulariser equal
    higherOrderDeformationEnergy.cpp restated here, bit for bit, on a
    perturbed octahedron."""
    rng = np.random.default_rng(11)
    V, und = MESHES_FOR_ENERGY
    VX = V * (1 + 0.2 * rng.random((len(V), 1)))
    EX = np.array(sorted([(a, b) for a, b in und] + [(b, a) for a, b in und]), dtype=np.int32)
    ny = 5
    t = np.linspace(0, 2 * np.pi, ny, endpoint=False)
    VY = np.stack([np.cos(t), np.sin(t), 0.3 * rng.random(ny)], axis=1)
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    fd = rng.uniform(0.1, 2.0, size=(len(VX), ny))
    o = oracle.OracleGenerator(VX, EX, VY, EY, fd, True, False, prune)
    o.set_normals(VX / np.linalg.norm(VX, axis=1, keepdims=True), np.tile([0.0, 0.0, 1.0], (ny, 1)))
    o.set_cost_time_ratio_mode(cost, time)
    got = o.get_cost_vector()
    want = _conj_energy_without_so3(VX, VY, fd, o.get_product_space(), cost, time)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def _rotation_quaternion(R):
    """Unit quaternion (w, x, y, z) of a rotation matrix, from whichever of
    the trace and the diagonal entries is largest (sign is irrelevant here)."""
    t = np.trace(R)
    if t > max(R[0, 0], R[1, 1], R[2, 2]):
        w = math.sqrt(1 + t) / 2
        return np.array([w, (R[2, 1] - R[1, 2]) / (4 * w), (R[0, 2] - R[2, 0]) / (4 * w), (R[1, 0] - R[0, 1]) / (4 * w)])
    i = int(np.argmax(np.diag(R)))
    j, k = (i + 1) % 3, (i + 2) % 3
    s = math.sqrt(1 + R[i, i] - R[j, j] - R[k, k]) * 2
    q = np.empty(4)
    q[0] = (R[k, j] - R[j, k]) / s
    q[1 + i] = s / 4
    q[1 + j] = (R[j, i] + R[i, j]) / s
    q[1 + k] = (R[k, i] + R[i, k]) / s
    return q


def _node_quaternions(VX, EX, NX, VY, EY, NY, prune):
    """precomputeAllQuaternionds with the MATLAB convention
    (higherOrderDeformationEnergy.cpp:95-134) and precomputeRotation
    (:16-53): one rotation per product node, aligning the curve frame [n, e,
    e x n] of its Y edge (the previous one for a 2D-degenerate node) with the
    mesh frame of its X edge (normal: mean of the endpoint normals), taken
    as U diag(1, 1, det(U V^T)) V^T from the SVD of X^T Y (numpy's LAPACK
    SVD here)."""
    nEX, nEY = len(EX), len(EY)
    eX = VX[EX[:, 1]] - VX[EX[:, 0]]
    eY = VY[EY[:, 1]] - VY[EY[:, 0]]
    unit = lambda v: v / np.linalg.norm(v)
    out = []
    for i in range(nEY):
        for j in range(3 * nEX):
            jj = j % nEX
            iy = (i + nEY - 1) % nEY if (nEX <= j < 2 * nEX and not prune) else i
            e2, n2 = eY[iy], NY[EY[iy, 0]]
            e3, n3 = eX[jj], (NX[EX[jj, 0]] + NX[EX[jj, 1]]) / 2
            X = np.stack([unit(n2), unit(e2), unit(np.cross(e2, n2))])
            Y = np.stack([unit(n3), unit(e3), unit(np.cross(e3, n3))])
            U, _, Vt = np.linalg.svd(X.T @ Y)
            d = np.linalg.det(U @ Vt)
            out.append(_rotation_quaternion(U @ np.diag([1.0, 1.0, d]) @ Vt))
    return np.array(out)


@pytest.mark.parametrize("prune", [False, True])
@pytest.mark.parametrize("cost,time", [("vanilla", "vanilla"), ("vanilla", "lengthnormalisation"),
                                       ("vanilla", ""), ("feature", "plainso3"), ("feature", "robustso3"),
                                       ("robustso3", "feature"), ("plainso3", "feature")])
def test_oracle_so3_energy_matches_the_restatement(oracle, cost, time, prune):
    """The oracle's conjugate-graph costs with the regulariser (the SO(3)
    distance 2 acos|q0 . q1| between the rotations of an edge's two nodes)
    against the restatement above, within 1e-9: the oracle takes its SVD by
    one-sided Jacobi rotations, numpy by LAPACK."""
    rng = np.random.default_rng(13)
    V, und = MESHES_FOR_ENERGY
    VX = V * (1 + 0.2 * rng.random((len(V), 1)))
    EX = np.array(sorted([(a, b) for a, b in und] + [(b, a) for a, b in und]), dtype=np.int32)
    NX = VX / np.linalg.norm(VX, axis=1, keepdims=True)
    ny = 5
    t = np.linspace(0, 2 * np.pi, ny, endpoint=False)
    VY = np.stack([np.cos(t), np.sin(t), 0.3 * rng.random(ny)], axis=1)
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    NY = np.tile([0.0, 0.0, 1.0], (ny, 1))
    fd = rng.uniform(0.1, 2.0, size=(len(VX), ny))
    o = oracle.OracleGenerator(VX, EX, VY, EY, fd, True, True, prune)
    o.set_normals(NX, NY)
    o.set_cost_time_ratio_mode(cost, time)
    got = o.get_cost_vector()
    ps = o.get_product_space()
    src, trgt = o.get_src_trgt()
    q = _node_quaternions(VX, EX, NX, VY, EY, NY, prune)
    dot = np.minimum(np.abs(np.sum(q[src] * q[trgt], axis=1)), 1.0)
    dist = 2 * np.arccos(dot)
    robust = np.array([_robust(x) for x in dist])
    f = fd[ps[:, 5], ps[:, 2]]
    L = np.zeros(len(ps))
    for j in range(3):
        dy = VY[ps[:, 0], j] - VY[ps[:, 1], j]
        dx = VX[ps[:, 3], j] - VX[ps[:, 4], j]
        L = L + dy * dy + dx * dx
    L = np.sqrt(L)
    deg = np.where((ps[:, 2] == ps[:, 1]) | (ps[:, 5] == ps[:, 4]), 0.1, 1.0)
    maxso3 = float(np.float32(_robust(2 * math.pi)))
    maxfd = float(np.float32(fd.max()))
    want = {
        ("vanilla", "vanilla"): [robust + f],
        ("vanilla", "lengthnormalisation"): [robust + f, L],
        ("vanilla", ""): [robust + f, deg],
        ("feature", "plainso3"): [f, np.maximum(0.0, 2 * math.pi - dist)],
        ("feature", "robustso3"): [f, np.maximum(0.0, maxso3 - robust)],
        ("robustso3", "feature"): [robust, np.maximum(0.0, maxfd - f)],
        ("plainso3", "feature"): [dist, np.maximum(0.0, maxfd - f)],
    }[(cost, time)]
    want = np.stack(want, axis=1)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-9)
    assert dist.max() > 0.1  # the frames do differ


@pytest.mark.parametrize("ny", [4, 5])
@pytest.mark.parametrize("column", ["halves", "tiny", "outliers", "random"])
def test_oracle_rescale_matches_the_restatement(oracle, column, ny):
    """The ratio solve's in-place rescale (cost_time_ratio_solver.cpp:709-721,
    utils.hpp:196-209) against tests/golden/make_golden.py's restatement, bit
    for bit, per column: halves that round away from zero (numpy's rounding
    would take them to even), a median below 0.001, outliers clipped at 1e7,
    and column lengths of both parities."""
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    if ny == 5:  # a square pyramid: 5 vertices, 8 edges, 37 rows per layer, an odd count
        V = np.array([[1, 1, 0], [-1, 1, 0], [-1, -1, 0], [1, -1, 0], [0, 0, 1]], dtype=np.float64)
        und = [(0, 1), (1, 2), (2, 3), (0, 3), (0, 4), (1, 4), (2, 4), (3, 4)]
    else:
        V, und = MESHES_FOR_ENERGY
    EX = np.array(sorted([(a, b) for a, b in und] + [(b, a) for a, b in und]), dtype=np.int32)
    t = np.linspace(0, 2 * np.pi, ny, endpoint=False)
    VY = np.stack([np.cos(t), np.sin(t), np.zeros(ny)], axis=1)
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    o = oracle.OracleGenerator(V, EX, VY, EY, np.ones((len(V), ny)), False, False)
    rows = o.product_space_rows()
    assert rows % 2 == (ny % 2)
    rng = np.random.default_rng(ny)
    if column == "halves":  # median 5e4 makes the scale factor exactly 1
        c = np.full(rows, 5e4)
        c[: rows // 3] = rng.integers(1, 1000, rows // 3) + 0.5
    elif column == "tiny":
        c = rng.uniform(1e-6, 1e-5, rows)
    elif column == "outliers":
        c = rng.uniform(1.0, 2.0, rows)
        c[::7] *= 1e4
    else:
        c = rng.uniform(0.1, 2.0, rows)
    E = np.stack([c, rng.uniform(0.5, 1.5, rows)], axis=1)
    o.set_cost_vector(E)
    o.solve_with_cost_time_ratio("lawlercpu", 2)
    got = o.get_cost_vector()
    want = np.stack([make_golden.rescale(E[:, 0]), make_golden.rescale(E[:, 1])], axis=1)
    assert np.array_equal(got, want)
    if column == "halves":
        assert not np.array_equal(want[:, 0], np.minimum(np.round(E[:, 0]), 1e7))
    if column == "outliers":
        assert (want[:, 0] == 1e7).any()
    if column == "tiny":
        assert float(np.median(c)) < 0.001
