"""Exact optima of toy cyclic product graphs, independent of both solvers.

A feasible cycle starts at a node u of layer 0 (depth 0), moves through the
layers in order -- inside a layer it may take up to K-1 intralayer edges, an
interlayer edge goes to depth 0 of the next layer -- and returns to u through
an interlayer edge of the last layer (one lap).  This is the set of cycles
the reference's branch and bound searches.

* minimum cost: per start node, a shortest path over the layered DAG;
* minimum cost/time ratio: per start node, Dinkelbach iterations with exact
  rational arithmetic (the rescaled costs and times are integers).

Both return the optimum and the edge lists of all optimal cycles of the
smallest start node that attains it (for tie-aware comparisons).
"""
from __future__ import annotations

from fractions import Fraction


def _edge_lists(src, trgt, n, nY):
    """Out-edges per global node, split by kind: intra[node] and inter[node]."""
    intra, inter = {}, {}
    for e, (s, t) in enumerate(zip(src, trgt)):
        ls, lt = s // n, t // n
        if ls == lt:
            intra.setdefault(s, []).append(e)
        elif lt == (ls + 1) % nY:
            inter.setdefault(s, []).append(e)
    return intra, inter


def _best_paths(u, weight, src, trgt, n, nY, K, intra, inter):
    """Min weight over one-lap closed walks from node u of layer 0, with all
    minimising edge lists.  weight(e) returns an exact number."""
    # states: (layer, depth, local node) -> (best value, list of edge paths)
    cur = {(0, 0, u): (0, [[]])}
    for layer in range(nY):
        # intralayer moves, depth by depth
        frontier = {key: val for key, val in cur.items() if key[0] == layer}
        allstates = dict(frontier)
        for k in range(K - 1):
            nxt = {}
            for (l, d, v), (val, paths) in frontier.items():
                if d != k:
                    continue
                g = l * n + v
                for e in intra.get(g, []):
                    w = val + weight(e)
                    key = (l, d + 1, trgt[e] % n)
                    if key not in nxt or w < nxt[key][0]:
                        nxt[key] = (w, [p + [e] for p in paths])
                    elif w == nxt[key][0]:
                        nxt[key][1].extend(p + [e] for p in paths)
            for key, val in nxt.items():
                if key not in allstates or val[0] < allstates[key][0]:
                    allstates[key] = val
                elif val[0] == allstates[key][0]:
                    allstates[key] = (val[0], allstates[key][1] + val[1])
            frontier = nxt
        # interlayer moves to depth 0 of the next layer
        nxt = {}
        for (l, d, v), (val, paths) in allstates.items():
            g = l * n + v
            for e in inter.get(g, []):
                t = trgt[e] % n
                if layer == nY - 1 and t != u:
                    continue
                w = val + weight(e)
                key = (layer + 1, 0, t)
                if key not in nxt or w < nxt[key][0]:
                    nxt[key] = (w, [p + [e] for p in paths])
                elif w == nxt[key][0]:
                    nxt[key][1].extend(p + [e] for p in paths)
        cur = nxt
    return cur.get((nY, 0, u), (None, []))


def min_cost_cycle(src, trgt, cost, n, nY, K):
    intra, inter = _edge_lists(src, trgt, n, nY)
    best, where = None, None
    for u in range(n):
        val, paths = _best_paths(u, lambda e: Fraction(cost[e]), src, trgt, n, nY, K, intra, inter)
        if val is not None and (best is None or val < best):
            best, where = val, (u, paths)
    return best, where


def min_ratio_cycle(src, trgt, cost, time, n, nY, K):
    """Exact minimum of sum(cost)/sum(time) over one-lap cycles."""
    intra, inter = _edge_lists(src, trgt, n, nY)
    best, where = None, None
    for u in range(n):
        # Dinkelbach from the ratio of any feasible cycle
        val, paths = _best_paths(u, lambda e: Fraction(cost[e]), src, trgt, n, nY, K, intra, inter)
        if val is None:
            continue
        path = paths[0]
        lam = Fraction(sum(Fraction(cost[e]) for e in path), sum(Fraction(time[e]) for e in path))
        for _ in range(200):
            val, paths = _best_paths(u, lambda e: Fraction(cost[e]) - lam * Fraction(time[e]), src, trgt, n, nY, K,
                                     intra, inter)
            if val >= 0:
                break
            path = paths[0]
            lam = Fraction(sum(Fraction(cost[e]) for e in path), sum(Fraction(time[e]) for e in path))
        opt = [p for p in _best_paths(u, lambda e: Fraction(cost[e]) - lam * Fraction(time[e]), src, trgt, n, nY, K,
                                      intra, inter)[1]]
        if best is None or lam < best:
            best, where = lam, (u, opt)
    return best, where
