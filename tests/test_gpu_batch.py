"""Batched solves (solve_batch / pgc_solve_batch): many graphs of uneven size
solved concurrently with one-CTA teams must return exactly what the oracle
returns for each of them, for the ratio and the minimum-cost solver, and a
failing member must be reported without affecting the others.

Ratio solves run in one launch whose CTAs each solve whole graphs on the
device; a graph whose cycle needs branch and bound, or outgrows the device's
cycle record, is handed back to the host.  Both routes, and the route with
one stream and launch sequence per graph (PGC_BATCH_STREAMS=1), must agree."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _same(got, want):
    assert got[0] == want[0]
    assert got[1] == want[1], (got[1], want[1])
    assert np.array_equal(got[2], want[2])


def _specs():
    # (n_vertices, n_curve, K, conjugate, seed); the seeds keep the oracle's
    # branch-and-bound short (some pairs need thousands of branches)
    return [(150, 10, 2, False, 10), (300, 14, 3, False, 11), (90, 8, 1, False, 12), (200, 12, 2, True, 14),
            (120, 6, 3, True, 14), (400, 16, 2, False, 15), (250, 9, 2, False, 16), (180, 10, 3, True, 13)]


def _build(cpg, oracle, spec):
    nv, m, K, conj, seed = spec
    p = synthetic.make_pair(n_vertices=nv, n_curve=m, feat_dim=16, seed=seed)
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, False)
    g, o = cpg.product_graph_generator(*args), oracle.OracleGenerator(*args)
    if conj:
        for x in (g, o):
            x.set_normals(p["NX"], p["NY"])
            x.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    g.set_max_depth_cost_time_ratio(K)
    o.set_max_depth_cost_time_ratio(K)
    return g, o


@pytest.mark.parametrize("solver,ref", [("lawlergpu", "lawlercpu"), ("dijkstragpu", "dijkstracpu")])
def test_batch_matches_oracle(cpg, oracle, solver, ref):
    pairs = [_build(cpg, oracle, s) for s in _specs()]
    gens = [g for g, _ in pairs]
    got = cpg.solve_batch(gens, solver, None, ctas_per_graph=1, workers=4, regenerate=True)
    for (g, o), res in zip(pairs, got):
        want = o.solve_with_cost_time_ratio(ref) if solver.startswith("lawler") else o.solve_with_minimum_cost(ref)
        _same(res, want)
        assert g.last_profile()["ctas"] == 1


def test_batch_equals_single_solves_with_full_teams(cpg, oracle):
    pairs = [_build(cpg, oracle, s) for s in _specs()[:4]]
    batched = cpg.solve_batch([g for g, _ in pairs], "lawlergpu", None, ctas_per_graph=2)
    for (g, _), res in zip(pairs, batched):
        g.generate()
        _same(res, g.solve_with_cost_time_ratio("lawlergpu"))


def test_batch_reports_a_failing_member(cpg, oracle):
    good = [_build(cpg, oracle, s)[0] for s in _specs()[:3]]
    p = synthetic.make_pair(n_vertices=100, n_curve=8, feat_dim=8, seed=3)
    bad = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], True, False)  # no normals
    with pytest.raises(cpg.PGCError, match="graph 1 of the batch failed"):
        cpg.solve_batch([good[0], bad, good[1], good[2]], "lawlergpu", None)
    # the others were solved all the same
    _, o = _build(cpg, oracle, _specs()[2])
    _same(good[2]._result(), o.solve_with_cost_time_ratio("lawlercpu"))


def test_batch_rejects_repeated_generators(cpg, oracle):
    g, _ = _build(cpg, oracle, _specs()[0])
    with pytest.raises(ValueError):
        cpg.solve_batch([g, g], "lawlergpu", 2)


def test_batch_device_solves_equal_the_stream_route(cpg, oracle, monkeypatch):
    pairs = [_build(cpg, oracle, s) for s in _specs()]
    gens = [g for g, _ in pairs]
    device = cpg.solve_batch(gens, "lawlergpu", None, regenerate=True)
    monkeypatch.setenv("PGC_BATCH_STREAMS", "1")
    streams = cpg.solve_batch(gens, "lawlergpu", None, regenerate=True)
    for a, b in zip(device, streams):
        _same(a, b)


def test_batch_hands_long_cycles_back_to_the_host(cpg, oracle, monkeypatch):
    """With a cycle record of 8 edges every graph is handed back to the host,
    which finishes it from the rescaled costs: the answers do not change."""
    monkeypatch.setenv("PGC_BATCH_CYCLE_CAP", "8")
    pairs = [_build(cpg, oracle, s) for s in _specs()[:5]]
    got = cpg.solve_batch([g for g, _ in pairs], "lawlergpu", None, regenerate=True)
    for (g, o), res in zip(pairs, got):
        _same(res, o.solve_with_cost_time_ratio("lawlercpu"))


def test_batch_adjoint_after_device_solves(cpg, oracle):
    """The adjoint of a batched ratio solve equals the adjoint after a single
    solve of the same graph (the device solve records the cycle and its time
    sum the same way)."""
    import torch

    pairs = [_build(cpg, oracle, s) for s in _specs()[:3]]
    gens = [g for g, _ in pairs]
    cpg.solve_batch(gens, "lawlergpu", None, regenerate=True)
    grads = []
    for g, spec in zip(gens, _specs()[:3]):
        p = synthetic.make_pair(n_vertices=spec[0], n_curve=spec[1], feat_dim=16, seed=spec[4])
        buf = torch.zeros(p["feat_diff"].shape, dtype=torch.float64, device="cuda")
        g.backward_feat_diff(1.0, buf.data_ptr())
        grads.append(buf.cpu().numpy())
    for g, gb in zip(gens, grads):
        g.generate()
        g.solve_with_cost_time_ratio("lawlergpu")
        buf = torch.zeros(gb.shape, dtype=torch.float64, device="cuda")
        g.backward_feat_diff(1.0, buf.data_ptr())
        assert np.array_equal(buf.cpu().numpy(), gb)


def test_launch_counter_and_batch_profile(cpg, oracle):
    """kernel_launches() counts the library's launches (the bench's
    gpu_launches); last_batch_profile() describes the last batched call."""
    pairs = [synthetic.make_pair(n_vertices=200 + 40 * i, n_curve=8, feat_dim=8, seed=60 + i) for i in range(3)]
    gens = []
    for p in pairs:
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False)
        g.set_cost_time_ratio_mode("vanilla", "nomode")
        gens.append(g)
    n0 = cpg.kernel_launches()
    cpg.solve_batch(gens, "lawlergpu", 2, regenerate=True)
    n1 = cpg.kernel_launches()
    # per graph at least the energy kernel and the median chain, plus the batched launch
    assert n1 - n0 >= 3 * 2 + 1
    prof = cpg.last_batch_profile()
    assert prof["solved_on_device"] + prof["handed_back"] == 3
    assert prof["ctas"] >= 1 and prof["threads_per_cta"] == 256
    assert prof["launch_ms"] > 0 and prof["prepare_ms"] > 0
    # a single solve launches too, and the counter only grows
    gens[0].solve_with_cost_time_ratio("lawlergpu", 2)
    assert cpg.kernel_launches() > n1
