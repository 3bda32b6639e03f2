"""Differentiation of the cycle objectives (no counterpart in the reference).

* The adjoint kernel's d lambda*/d feat_diff equals the gradient assembled in
  numpy from the ORACLE's cycle: its edges, the reference's rescale factor
  (1e5 / (2 max(median, 0.001))) and T = sum of the cycle's rescaled times.
* The minimum-cost adjoint agrees with central finite differences
  (h = 1e-3) at points where the cycle does not change within +-h.
* The ratio adjoint agrees with central finite differences of
  lambda = s_c C(fd) / (s_t T(fd)) over the solved cycle, the rescale factors
  s held fixed (rounding passed straight through), where the cycle does not
  change within +-h: plain graphs (also at the differentiation
  configuration's size, 2,000 x 100, K = 2) and the conjugate mode whose time
  column reads feat_diff, max(0, maxFd - fd).
* torch carries the gradient on to learnable features; the batched forward
  gives the single-pair results and gradients.
* Blackbox interpolation reproduces its definition -(y(w) - y(w + tau g)) / tau,
  with both solves recomputed independently by the oracle.
* Conjugate graph: the adjoint scatters into fd[x2, y2] of every cycle edge
  (ratio: the rescale factor over T; minimum cost: 1); a ratio whose time
  column reads feat_diff ("feature": max(0, maxFd - fd)) adds lambda* s_t / T
  at fd[x2, y2] of every cycle edge with a positive time and subtracts it at
  the matrix maximum's entry (a subgradient).
"""
import numpy as np
import pytest
import torch

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _pair(nv=150, m=10, seed=0, dim=16):
    return synthetic.make_pair(n_vertices=nv, n_curve=m, feat_dim=dim, seed=seed)


def _gens(cpg, oracle, p, reg=False, cost="vanilla", time="nomode"):
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, reg, False)
    g, o = cpg.product_graph_generator(*args), oracle.OracleGenerator(*args)
    g.set_cost_time_ratio_mode(cost, time)
    o.set_cost_time_ratio_mode(cost, time)
    return g, o


def _line_integral(p, y0, y1, x0, x1):
    dy = p["VY"][y0] - p["VY"][y1]
    dx = p["VX"][x0] - p["VX"][x1]
    return float(np.sqrt(np.sum(dy * dy) + np.sum(dx * dx)))


def _device_grad(g, shape, grad=1.0):
    out = torch.empty(shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    g.backward_feat_diff(grad, out.data_ptr())
    return out.cpu().numpy()


@pytest.mark.parametrize("reg,cost,time", [(False, "vanilla", "nomode"), (True, "vanilla", "nomode"),
                                           (False, "feature", "lengthnormalisation")])
def test_ratio_adjoint_matches_gradient_from_oracle_cycle(cpg, oracle, reg, cost, time):
    p = _pair(seed=3)
    g, o = _gens(cpg, oracle, p, reg, cost, time)
    raw = o.get_cost_vector()
    K = 2
    rg = g.solve_with_cost_time_ratio("lawlergpu", K)
    ro = o.solve_with_cost_time_ratio("lawlercpu", K)
    assert rg[1] == ro[1] and np.array_equal(rg[2], ro[2])
    edges = o.last_cycle_edges()
    assert np.array_equal(np.sort(g.last_cycle_edges()), np.sort(edges))
    s0 = 1e5 / (2 * max(np.median(raw[:, 0]), 0.001))
    scaled = o.get_cost_vector()
    T = scaled[edges, 1].sum() if raw.shape[1] > 1 else 5e4 * len(edges)
    ps = o.get_product_space()
    want = np.zeros(p["feat_diff"].shape)
    length_mode = cost == "feature" and time == "lengthnormalisation"
    for e in edges:
        y0, y1, x0, x1 = ps[e]
        li = _line_integral(p, y0, y1, x0, x1) if (reg or length_mode) else 1.0
        d = s0 / T * (1.0 if length_mode else 0.5 * li)
        want[x0, y0] += d
        want[x1, y1] += d
    got = _device_grad(g, want.shape)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-18)
    # the gradient of grad * objective scales linearly
    np.testing.assert_allclose(_device_grad(g, want.shape, -2.5), -2.5 * want, rtol=1e-12, atol=1e-18)


def test_min_cost_adjoint_matches_central_differences(cpg, oracle):
    p = _pair(nv=120, m=8, seed=5)
    g, _ = _gens(cpg, oracle, p)
    fd0 = p["feat_diff"].copy()
    K, h = 2, 1e-3

    def solve(fd):
        g.set_feat_diff(fd)
        res = g.solve_with_minimum_cost("dijkstragpu", K)
        return res[1], np.sort(g.last_cycle_edges())

    obj0, edges0 = solve(fd0)
    grad = _device_grad(g, fd0.shape)
    rng = np.random.default_rng(0)
    checked = 0
    for _ in range(6):
        direction = rng.standard_normal(fd0.shape)
        plus, e_plus = solve(fd0 + h * direction)
        minus, e_minus = solve(fd0 - h * direction)
        if not (np.array_equal(e_plus, edges0) and np.array_equal(e_minus, edges0)):
            continue  # the cycle changes within +-h: not a differentiable point along this direction
        fdiff = (plus - minus) / (2 * h)
        analytic = float((grad * direction).sum())
        assert abs(fdiff - analytic) <= 2e-3 * max(1.0, abs(analytic)), (fdiff, analytic)
        checked += 1
    assert checked >= 3


def test_autograd_reaches_learnable_features(cpg, oracle):
    from cyclic_product_graphs.autograd import RatioCycleObjective

    p = _pair(seed=7)
    g, _ = _gens(cpg, oracle, p)
    fX = torch.tensor(p["fX"], dtype=torch.float64, device="cuda", requires_grad=True)
    fY = torch.tensor(p["fY"], dtype=torch.float64, device="cuda")
    fd = torch.cdist(fX, fY)
    lam = RatioCycleObjective.apply(fd, g, 2)
    lam.backward()
    assert fX.grad is not None and torch.isfinite(fX.grad).all() and fX.grad.abs().sum() > 0
    # the chain rule from the adjoint's d lambda / d feat_diff
    G = torch.tensor(_device_grad(g, tuple(fd.shape)), device="cuda")
    fX2 = fX.detach().clone().requires_grad_(True)
    (want,) = torch.autograd.grad(torch.cdist(fX2, fY), fX2, G)
    torch.testing.assert_close(fX.grad, want, rtol=1e-10, atol=1e-12)


def test_batched_objectives_equal_single_solves(cpg, oracle):
    from cyclic_product_graphs.autograd import RatioCycleObjective, ratio_cycle_objectives

    pairs = [_pair(nv=100 + 30 * i, m=8 + 2 * i, seed=20 + i) for i in range(4)]
    gens = [_gens(cpg, oracle, p)[0] for p in pairs]
    fds = [torch.tensor(p["feat_diff"], device="cuda", requires_grad=True) for p in pairs]
    lams = ratio_cycle_objectives(gens, fds, 2)
    lams.sum().backward()
    for p, fd, lam in zip(pairs, fds, lams):
        g1 = _gens(cpg, oracle, p)[0]
        fd1 = torch.tensor(p["feat_diff"], device="cuda", requires_grad=True)
        l1 = RatioCycleObjective.apply(fd1, g1, 2)
        l1.backward()
        assert float(l1) == float(lam)
        torch.testing.assert_close(fd.grad, fd1.grad, rtol=0, atol=0)


def test_blackbox_interpolation_reproduces_its_definition(cpg, oracle):
    from cyclic_product_graphs.autograd import BlackboxMinCostCycle

    p = _pair(nv=100, m=8, seed=9)
    g, o = _gens(cpg, oracle, p)
    w0 = o.get_cost_vector()[:, 0].copy()
    K, tau = 2, 10.0
    w = torch.tensor(w0, device="cuda", requires_grad=True)
    y = BlackboxMinCostCycle.apply(w, g, tau, K)
    gy = torch.randn(y.shape, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    y.backward(gy)

    def oracle_y(costs):
        o.set_cost_vector(costs.reshape(-1, 1))
        o.solve_with_minimum_cost("dijkstracpu", K)
        ind = np.zeros(len(costs))
        np.add.at(ind, o.last_cycle_edges(), 1.0)
        return ind

    y_w = oracle_y(w0)
    assert np.array_equal(y.detach().cpu().numpy(), y_w)
    y_w2 = oracle_y(w0 + tau * gy.cpu().numpy())
    np.testing.assert_array_equal(w.grad.cpu().numpy(), -(y_w - y_w2) / tau)


def _conj_gens(cpg, oracle, p, reg, cost, time):
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], True, reg, False)
    g, o = cpg.product_graph_generator(*args), oracle.OracleGenerator(*args)
    for x in (g, o):
        x.set_normals(p["NX"], p["NY"])
        x.set_cost_time_ratio_mode(cost, time)
    # the SO(3) energies agree to 1e-9, not bitwise: both sides use the device's
    o.set_cost_vector(g.get_cost_vector())
    return g, o


@pytest.mark.parametrize("reg,cost,time", [(False, "vanilla", "lengthnormalisation"), (False, "vanilla", "vanilla"),
                                           (True, "feature", "plainso3")])
def test_conjugate_ratio_adjoint_matches_gradient_from_oracle_cycle(cpg, oracle, reg, cost, time):
    p = synthetic.make_pair(icosphere_level=1, n_curve=8, feat_dim=8, seed=13)
    g, o = _conj_gens(cpg, oracle, p, reg, cost, time)
    raw = o.get_cost_vector()
    K = 2
    rg = g.solve_with_cost_time_ratio("lawlergpu", K)
    ro = o.solve_with_cost_time_ratio("lawlercpu", K)
    assert rg[1] == ro[1] and np.array_equal(rg[2], ro[2])
    edges = o.last_cycle_edges()
    assert np.array_equal(np.sort(g.last_cycle_edges()), np.sort(edges))
    s0 = 1e5 / (2 * max(np.median(raw[:, 0]), 0.001))
    scaled = o.get_cost_vector()
    T = scaled[edges, 1].sum() if raw.shape[1] > 1 else 5e4 * len(edges)
    ps = o.get_product_space()
    want = np.zeros(p["feat_diff"].shape)
    for e in edges:  # cost = (robust loss +) fd[x2, y2]
        y2, x2 = ps[e][2], ps[e][5]
        want[x2, y2] += s0 / T
    got = _device_grad(g, want.shape)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-18)


def test_conjugate_min_cost_adjoint_and_unsupported_time_mode(cpg, oracle):
    p = synthetic.make_pair(icosphere_level=1, n_curve=8, feat_dim=8, seed=13)
    g, o = _conj_gens(cpg, oracle, p, False, "vanilla", "lengthnormalisation")
    rg = g.solve_with_minimum_cost("dijkstragpu", 2)
    ro = o.solve_with_minimum_cost("dijkstracpu", 2)
    assert rg[1] == ro[1] and np.array_equal(rg[2], ro[2])
    ps = o.get_product_space()
    want = np.zeros(p["feat_diff"].shape)
    for e in o.last_cycle_edges():
        want[ps[e][5], ps[e][2]] += 1.0
    np.testing.assert_allclose(_device_grad(g, want.shape, 3.0), 3.0 * want, rtol=1e-12, atol=1e-18)


@pytest.mark.parametrize("cost,time", [("robustso3", "feature"), ("plainso3", "feature")])
def test_conjugate_feature_time_adjoint_matches_gradient_from_oracle_cycle(cpg, oracle, cost, time):
    p = synthetic.make_pair(icosphere_level=1, n_curve=8, feat_dim=8, seed=13)
    g, o = _conj_gens(cpg, oracle, p, True, cost, time)
    raw = o.get_cost_vector()
    K = 2
    try:
        ro = o.solve_with_cost_time_ratio("lawlercpu", K)
    except RuntimeError:
        pytest.skip("the reference stops with no nodes in branch on this pair")
    rg = g.solve_with_cost_time_ratio("lawlergpu", K)
    assert rg[1] == ro[1] and np.array_equal(rg[2], ro[2])
    edges = o.last_cycle_edges()
    scaled = o.get_cost_vector()
    C, T = scaled[edges, 0].sum(), scaled[edges, 1].sum()  # integers: exact in any order
    lam = C / T
    s_t = 1e5 / (2 * max(np.median(raw[:, 1]), 0.001))
    fd = p["feat_diff"]
    max_fd = float(np.float32(fd.max()))
    argmax = np.unravel_index(int(np.argmax(fd)), fd.shape)
    ps = o.get_product_space()
    want = np.zeros(fd.shape)
    for e in edges:  # the cost column (SO(3) terms) does not read feat_diff
        y2, x2 = ps[e][2], ps[e][5]
        if max_fd - fd[x2, y2] > 0:
            want[x2, y2] += lam * s_t / T
            want[argmax] -= lam * s_t / T
    got = _device_grad(g, want.shape)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-16)


def _ratio_fd_check(cpg, g, make, fd0, K, h, directions, seed, tol):
    """Central differences of lambda = s_c C / (s_t T) over the solved cycle
    with the solve's rescale factors held fixed, along random directions
    where the cycle (and the matrix maximum's entry) stays the same within
    +-h, against the adjoint.  Returns how many directions were checked."""
    raw = g.get_cost_vector()
    g.solve_with_cost_time_ratio("lawlergpu", K)
    scaled = g.get_cost_vector()
    s = scaled.sum(axis=0) / raw.sum(axis=0)  # the factors (rounding averages out over every edge)
    edges = g.last_cycle_edges()
    edges_sorted = np.sort(edges)
    grad = _device_grad(g, fd0.shape)
    probe = make()

    def lam_fixed(fd):
        probe.set_feat_diff(fd)
        c = probe.get_cost_vector()
        C = s[0] * c[edges, 0].sum()
        T = s[1] * c[edges, 1].sum() if c.shape[1] > 1 else 5e4 * len(edges)
        return C / T

    def same_cycle(fd):
        probe.set_feat_diff(fd)
        try:
            probe.solve_with_cost_time_ratio("lawlergpu", K)
        except cpg.PGCError:  # the reference's "no nodes in branch" end: no cycle to compare
            return False
        return np.array_equal(np.sort(probe.last_cycle_edges()), edges_sorted)

    rng = np.random.default_rng(seed)
    checked = 0
    for _ in range(directions):
        d = rng.standard_normal(fd0.shape)
        plus, minus = fd0 + h * d, fd0 - h * d
        if np.argmax(plus) != np.argmax(fd0) or np.argmax(minus) != np.argmax(fd0):
            continue
        if not (same_cycle(plus) and same_cycle(minus)):
            continue
        fdiff = (lam_fixed(plus) - lam_fixed(minus)) / (2 * h)
        analytic = float((grad * d).sum())
        assert abs(fdiff - analytic) <= tol * abs(analytic) + 1e-9, (fdiff, analytic)
        checked += 1
    return checked


@pytest.mark.parametrize("nv,m,K,seed", [(150, 10, 2, 3), (2000, 100, 2, 100000)])
def test_ratio_adjoint_matches_central_differences(cpg, oracle, nv, m, K, seed):
    p = synthetic.make_pair(n_vertices=nv, n_curve=m, feat_dim=64 if nv >= 2000 else 16, seed=seed)

    def make():
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False, False)
        g.set_cost_time_ratio_mode("vanilla", "nomode")
        return g

    assert _ratio_fd_check(cpg, make(), make, p["feat_diff"].copy(), K, 1e-3, 6, seed, 1e-3) >= 3


@pytest.mark.parametrize("cost,seed", [("robustso3", 24), ("plainso3", 14)])
def test_conjugate_feature_time_adjoint_matches_central_differences(cpg, oracle, cost, seed):
    """The ("*", "feature") time column divides by maxFd, the matrix maximum:
    the adjoint's subgradient puts that term on the maximum's entry.  The
    maximum is raised by 0.5 so that +-h moves keep it on the same entry; the
    pairs are ones where the oracle keeps the solved cycle along at least
    three of the ten directions (elsewhere the branch and bound changes the
    cycle or ends with "no nodes in branch")."""
    p = synthetic.make_pair(icosphere_level=1, n_curve=8, feat_dim=8, seed=seed)
    fd0 = p["feat_diff"].copy()
    fd0.flat[np.argmax(fd0)] += 0.5

    def make():
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], fd0, True, True, False)
        g.set_normals(p["NX"], p["NY"])
        g.set_cost_time_ratio_mode(cost, "feature")
        return g

    # h = 2e-3: maxFd (about 1.5) passes through float, whose spacing there is ~1.2e-7
    assert _ratio_fd_check(cpg, make(), make, fd0.copy(), 2, 2e-3, 10, 4, 2e-3) >= 3


@pytest.mark.parametrize("conj", [False, True])
def test_device_feat_diff_equals_host_feat_diff(cpg, oracle, conj):
    """set_feat_diff_device (a device-to-device copy, the host copy read back
    only when a host reader needs it) gives the costs, solve and adjoint that
    set_feat_diff gives; the conjugate case's time column reads feat_diff
    through its maximum, computed from that host copy."""
    p = synthetic.make_pair(icosphere_level=1, n_curve=8, feat_dim=8, seed=14)
    fd = p["feat_diff"] * 1.25 + 0.01
    gens = []
    for _ in range(2):
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, conj, False)
        if conj:
            g.set_normals(p["NX"], p["NY"])
            g.set_cost_time_ratio_mode("plainso3", "feature")
        gens.append(g)
    host, dev = gens
    host.set_feat_diff(fd)
    t = torch.tensor(fd, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    dev.set_feat_diff_device(t.data_ptr(), *fd.shape)
    del t
    assert np.array_equal(host.get_cost_vector(), dev.get_cost_vector())
    rh = host.solve_with_cost_time_ratio("lawlergpu", 2)
    rd = dev.solve_with_cost_time_ratio("lawlergpu", 2)
    assert rh[0] == rd[0] and rh[1] == rd[1] and np.array_equal(rh[2], rd[2])
    np.testing.assert_array_equal(_device_grad(host, fd.shape), _device_grad(dev, fd.shape))
