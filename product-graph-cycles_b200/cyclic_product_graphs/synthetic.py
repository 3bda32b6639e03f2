"""Seeded synthetic shape pairs for the cycle-search path.

A shape pair is a closed triangle mesh X (3D) and an ordered closed curve Y
(2D, embedded in the xy-plane with z = 0) together with the |VX| x |VY|
feature-difference matrix.  The generator follows the recipe used for the
benchmark workloads:

* X: a sphere mesh (a subdivided icosahedron, or the convex hull of a
  Fibonacci point set when an arbitrary vertex count is wanted), pushed out
  radially by smooth noise, r = 1 + amp * noise, where the noise is Gaussian
  and smoothed by uniform Laplacian averaging over the mesh.  EX holds both
  orientations of every undirected mesh edge.  Vertex normals are
  area-weighted face normals.
* Y: the orthographic projection of X onto the xy-plane; its silhouette is
  taken as the convex hull of the projected vertices, resampled at m points
  uniformly by arc length, counter-clockwise, with z = 0.  EY[i] = (i, i+1).
  Curve normals follow the reference's compute_normals_2d rule.
* Features: f_X is mesh-smoothed Gaussian noise of dimension d; f_Y[j] is
  f_X at the mesh vertex whose projection is nearest to curve point j, plus
  N(0, sigma^2) noise; feat_diff[x, y] = ||f_X[x] - f_Y[y]||_2 computed in
  float32 and returned as float64.

No dataset is read: every array is drawn from numpy's default_rng(seed).
"""
from __future__ import annotations

import numpy as np


def icosphere(subdivisions: int):
    """Vertices and faces of a unit icosphere after `subdivisions` 1:4 splits."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in V]
    for _ in range(subdivisions):
        mid = {}
        newF = []

        def midpoint(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in mid:
                m = V[a] + V[b]
                V.append(m / np.linalg.norm(m))
                mid[key] = len(V) - 1
            return mid[key]

        for a, b, c in F:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            newF += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = newF
    return np.array(V), np.array(F, dtype=np.int64)


def fibonacci_sphere(n: int):
    """Triangulated unit sphere with exactly n vertices (convex hull of a Fibonacci lattice)."""
    from scipy.spatial import ConvexHull

    i = np.arange(n, dtype=np.float64) + 0.5
    phi = np.arccos(1.0 - 2.0 * i / n)
    theta = np.pi * (1.0 + 5.0 ** 0.5) * i
    V = np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], axis=1)
    hull = ConvexHull(V)
    F = hull.simplices.astype(np.int64)
    # orient faces outward
    c = V[F].mean(axis=1)
    nrm = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = (nrm * c).sum(axis=1) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return V, F


def undirected_edges(F: np.ndarray) -> np.ndarray:
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0)
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0)


def directed_edges(F: np.ndarray) -> np.ndarray:
    """Both orientations of every undirected edge, as int32 [2|E| x 2]."""
    u = undirected_edges(F)
    both = np.concatenate([u, u[:, ::-1]], axis=0)
    order = np.lexsort((both[:, 1], both[:, 0]))
    return np.ascontiguousarray(both[order].astype(np.int32))


def smooth_over_mesh(values: np.ndarray, F: np.ndarray, iterations: int) -> np.ndarray:
    n = values.shape[0]
    u = undirected_edges(F)
    deg = np.bincount(u.ravel(), minlength=n).astype(np.float64)
    x = values.astype(np.float64).copy()
    for _ in range(iterations):
        acc = np.zeros_like(x)
        np.add.at(acc, u[:, 0], x[u[:, 1]])
        np.add.at(acc, u[:, 1], x[u[:, 0]])
        x = 0.5 * x + 0.5 * acc / deg.reshape((-1,) + (1,) * (x.ndim - 1))
    return x


def vertex_normals(V: np.ndarray, F: np.ndarray) -> np.ndarray:
    fn = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])  # length = 2 * area
    N = np.zeros_like(V)
    for k in range(3):
        np.add.at(N, F[:, k], fn)
    return _unit_rows(N, "mesh vertex")


def _unit_rows(N: np.ndarray, what: str) -> np.ndarray:
    """Rows of N scaled to unit length; a zero (or non-finite) row has no
    direction, so it is refused instead of turning into NaN."""
    length = np.linalg.norm(N, axis=1, keepdims=True)
    bad = ~(np.isfinite(length[:, 0]) & (length[:, 0] > 1e-300))
    if bad.any():
        raise ValueError(f"degenerate input: the {what} normal of row {int(np.flatnonzero(bad)[0])} has no direction")
    return N / length


def normals_2d(V: np.ndarray, E: np.ndarray) -> np.ndarray:
    """Outward in-plane normals of an ordered closed curve (utils.cpp:93-157 rule).

    Edge normals are the edge vectors rotated about z, flipped if they point
    inward; a vertex normal is the length-weighted sum of the normals of the
    edge ending at it and the edge starting at it.
    """
    V = np.asarray(V, dtype=np.float64)
    if V.shape[0] != E.shape[0]:
        raise ValueError("V.rows() != E.rows()")
    zero = -1
    for i in range(3):
        if abs(V[:, i].sum()) < 1e-4:
            zero = i
            break
    if zero == -1:
        raise ValueError("points do not lie on the xy, xz or yz plane")
    if zero != 2:
        V = V[:, [0, 2, 1]] if zero == 1 else V[:, [1, 2, 0]]
    ev = V[E[:, 0]] - V[E[:, 1]]
    el = np.linalg.norm(ev, axis=1)
    R = np.array([[0.0, 1.0, 0.0], [-1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    en = ev @ R.T
    en = en / np.linalg.norm(en, axis=1, keepdims=True)
    maxx, minx = np.float32(V[:, 0].max()), np.float32(V[:, 0].min())
    maxy, miny = np.float32(V[:, 1].max()), np.float32(V[:, 1].min())
    mult = np.float32(0.1 * min(abs(maxx - minx), abs(maxy - miny)))
    if np.float32((V + float(mult) * en)[:, 0].max()) < maxx:
        en = -en
    m = V.shape[0]
    vn = np.zeros((m, 3))
    for i in range(1, m + 1):
        j = i % m
        vn[j] = el[i - 1] * en[i - 1] + el[j] * en[j]
    return _unit_rows(vn, "curve vertex")


def silhouette_curve(VX: np.ndarray, m: int):
    """m points uniformly (by arc length) on the convex silhouette of VX projected to xy, CCW, z=0."""
    from scipy.spatial import ConvexHull

    P = VX[:, :2]
    hull = ConvexHull(P)
    poly = P[hull.vertices]  # CCW for 2D hulls
    closed = np.vstack([poly, poly[:1]])
    seg = np.linalg.norm(np.diff(closed, axis=0), axis=1)
    cum = np.concatenate([[0.0], np.cumsum(seg)])
    s = np.linspace(0.0, cum[-1], m, endpoint=False)
    idx = np.searchsorted(cum, s, side="right") - 1
    idx = np.clip(idx, 0, len(seg) - 1)
    t = (s - cum[idx]) / np.where(seg[idx] > 0, seg[idx], 1.0)
    pts = closed[idx] + t[:, None] * (closed[idx + 1] - closed[idx])
    VY = np.zeros((m, 3))
    VY[:, :2] = pts
    EY = np.stack([np.arange(m), (np.arange(m) + 1) % m], axis=1).astype(np.int32)
    return VY, EY


def make_pair(n_vertices: int = 642, n_curve: int = 60, feat_dim: int = 32, seed: int = 0, amp: float = 0.1,
              feat_noise: float = 0.05, icosphere_level: int | None = None, smooth_iters: int = 4,
              with_normals: bool | None = None):
    """Return a dict with VX, EX, VY, EY, feat_diff (and NX, NY) for one synthetic pair.

    `with_normals` None gives normals when the curve has at least three
    points: a two-point curve runs back along itself, so its vertex normals
    cancel and have no direction (asking for them then raises ValueError)."""
    if with_normals is None:
        with_normals = n_curve >= 3
    rng = np.random.default_rng(seed)
    if icosphere_level is not None:
        V, F = icosphere(icosphere_level)
    else:
        V, F = fibonacci_sphere(n_vertices)
    noise = smooth_over_mesh(rng.standard_normal(V.shape[0]), F, smooth_iters)
    noise = noise / (np.abs(noise).max() + 1e-12)
    VX = V * (1.0 + amp * noise)[:, None]
    EX = directed_edges(F)
    VY, EY = silhouette_curve(VX, n_curve)
    fX = smooth_over_mesh(rng.standard_normal((VX.shape[0], feat_dim)), F, smooth_iters).astype(np.float32)
    d2 = ((VX[None, :, :2] - VY[:, None, :2]) ** 2).sum(axis=2)
    nearest = d2.argmin(axis=1)
    fY = (fX[nearest] + rng.normal(0.0, feat_noise, size=(n_curve, feat_dim))).astype(np.float32)
    fd = np.empty((VX.shape[0], n_curve), dtype=np.float64)
    step = max(1, (1 << 24) // max(1, VX.shape[0] * feat_dim))
    for j0 in range(0, n_curve, step):
        diff = fX[:, None, :] - fY[None, j0:j0 + step, :]
        fd[:, j0:j0 + step] = np.sqrt((diff * diff).sum(axis=2, dtype=np.float32))
    out = dict(VX=np.ascontiguousarray(VX), EX=EX, VY=np.ascontiguousarray(VY), EY=EY,
               feat_diff=np.ascontiguousarray(fd), F=F, fX=fX, fY=fY, nearest=nearest)
    if with_normals:
        out["NX"] = vertex_normals(VX, F)
        # normals_2d picks the plane by the first coordinate column whose sum is
        # ~0; a curve around the origin would be misread, so detect the plane
        # on a translated copy (edge vectors, hence normals, are unchanged)
        out["NY"] = normals_2d(VY + np.array([10.0, 10.0, 0.0]), EY)
    return out
