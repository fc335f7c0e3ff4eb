"""CPU restatement of the reference's stencil helper (test infrastructure only).

Follows ``native/cat_surface_stencil_builder.c`` of the reference project:

* the input sphere is centred on its vertex mean and unit-normalised unless
  ``normalize`` is false (``:374-382``);
* the resampling sphere's unit directions are placed at
  ``centre + r * u`` with ``centre`` the per-axis sum of the minimum and the
  maximum coordinate and ``r = 0.975 * mean |p|`` (``:383-388``, the
  tetrahedral sphere of ``:389-390``);
* surface barycentrics: the triangle picked for each placed point by the
  closest-polygon rule and the weights of the picked point (``:107-134``);
  the resampled sphere is the input sphere interpolated with them (``:424``);
* sheet barycentrics of the cell centres on the unit-normalised resampled
  sphere (``:138-170, 239-295``).

The closest-polygon rule is the reference's restatement for its rotation
search (``src/cat_surface_gpu/surface_rotation.py:316-425``), in float64:
plane projection accepted within a 1e-3 parametric tolerance, otherwise the
nearer edge at the triangle's nearest vertex; smallest candidate distance,
lowest triangle index on ties; weights by ``_barycentric`` (``:335-352``).
Candidates are every triangle with a vertex within
``d_nearest_vertex + longest_edge + slack`` of the query, which contains the
winner.  Pinned to the helper's own output by ``tests/test_stencil_helper.py``.
"""

from __future__ import annotations

import math

import numpy as np
from scipy.spatial import cKDTree

TOL = 1.0e-3


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack((a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]), axis=-1)


def _segment(p, first, second):
    direction = second - first
    offset = p - first
    den = _dot(direction, direction)
    with np.errstate(divide="ignore", invalid="ignore"):
        alpha = np.where(den != 0.0, _dot(offset, direction) / den, 0.0)
    alpha = np.minimum(np.maximum(alpha, 0.0), 1.0)
    q = first + alpha[..., None] * direction
    d = p - q
    return _dot(d, d), q


def candidate(p, a, b, c):
    """Candidate distance and point of query p on triangles abc (broadcast over leading axes)."""

    ea, eb = b - a, c - a
    n = _cross(ea, eb)
    nsq = _dot(n, n)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.where(nsq != 0.0, _dot(a - p, n) / nsq, 0.0)
        proj = p + t[..., None] * n
        po = proj - a
        xx, xy, xv, yy, yv = _dot(ea, ea), _dot(ea, eb), _dot(ea, po), _dot(eb, eb), _dot(eb, po)
        den = xx * yy - xy * xy
        xpos = np.where(den != 0.0, (xv * yy - yv * xy) / den, 0.0)
        ypos = np.where(den != 0.0, (yv * xx - xv * xy) / den, 0.0)
    s = xpos + ypos
    top = 1.0 + TOL
    inside = (den != 0.0) & (xpos >= -TOL) & (xpos <= top) & (ypos >= -TOL) & (ypos <= top) & (s >= -TOL) & (s <= top)
    verts = np.stack(np.broadcast_arrays(a, b, c), axis=-2)
    vd = np.stack([_dot(p - verts[..., k, :], p - verts[..., k, :]) for k in range(3)], axis=-1)
    cv = np.argmin(vd, axis=-1)  # the first minimum

    def take(k):
        return np.take_along_axis(verts, k[..., None, None].repeat(3, -1), axis=-2)[..., 0, :]

    cur, prev, nxt = take(cv), take((cv + 2) % 3), take((cv + 1) % 3)
    d1, q1 = _segment(p, prev, cur)
    d2, q2 = _segment(p, cur, nxt)
    first = d1 < d2
    out_d = np.where(first, d1, d2)
    out_q = np.where(first[..., None], q1, q2)
    return np.where(inside, t * t * nsq, out_d), np.where(inside[..., None], proj, out_q)


def weights(p, a, b, c):
    """Barycentric weights of p in abc (the reference's three-cross-product form)."""

    t = (a, b, c)
    out = []
    for k in range(3):
        first, second, third = t[(k + 1) % 3], t[(k + 2) % 3], t[k]
        po, hz, up = p - first, second - first, third - first
        vert = _cross(_cross(hz, up), hz)
        out.append(_dot(po, vert) / _dot(up, vert))
    return np.stack(out, axis=-1)


def locate(points: np.ndarray, faces: np.ndarray, queries: np.ndarray):
    """Picked triangle and weights for each query on the mesh (points, faces)."""

    points = np.asarray(points, dtype=np.float64)
    faces = np.asarray(faces, dtype=np.int64)
    queries = np.asarray(queries, dtype=np.float64)
    edges = points[faces] - points[np.roll(faces, -1, axis=1)]
    longest = float(np.sqrt(_dot(edges, edges)).max())
    reach = longest + 6.0e-3 * longest
    corner_faces = np.argsort(faces.ravel(), kind="stable") // 3  # faces grouped by vertex
    ends = np.cumsum(np.bincount(faces.ravel(), minlength=points.shape[0]))
    incident = np.split(corner_faces, ends[:-1])
    tree = cKDTree(points)
    nearest, _ = tree.query(queries)
    face_out = np.empty(queries.shape[0], dtype=np.int64)
    w_out = np.empty((queries.shape[0], 3))
    for start in range(0, queries.shape[0], 4096):
        q = queries[start:start + 4096]
        balls = tree.query_ball_point(q, nearest[start:start + 4096] + reach)
        cands = [np.unique(np.concatenate([incident[v] for v in ball])) for ball in balls]
        width = max(len(c) for c in cands)
        cand = np.full((q.shape[0], width), -1, dtype=np.int64)
        for i, c in enumerate(cands):
            cand[i, :len(c)] = c  # ascending: the first minimum is the lowest index
        tri = points[faces[np.maximum(cand, 0)]]
        d, pt = candidate(q[:, None, :], tri[..., 0, :], tri[..., 1, :], tri[..., 2, :])
        d = np.where(cand >= 0, d, np.inf)
        best = np.argmin(d, axis=1)
        rows = np.arange(q.shape[0])
        f = cand[rows, best]
        t = points[faces[f]]
        face_out[start:start + 4096] = f
        w_out[start:start + 4096] = weights(pt[rows, best], t[:, 0], t[:, 1], t[:, 2])
    return face_out, w_out


def tetrahedral_sphere(levels: int = 6):
    """The helper's resampling sphere (its tetrahedral sphere of 20 * 4^levels triangles).

    An icosahedron with vertices (+-a, +-b, 0), (0, +-a, +-b), (+-b, 0, +-a),
    a = phi / sqrt(1 + phi^2), b = 1 / sqrt(1 + phi^2), in the helper's vertex
    and face order, split 1-to-4 per level: each face (p, q, r) in order gives
    (p, pq, rp), (pq, q, qr), (rp, pq, qr), (rp, qr, r), an edge midpoint is
    numbered when its edge is first met (edges pq, qr, rp) and is the
    normalised sum of its ends.  One edge at a time, with a dictionary.
    """

    phi = (1.0 + math.sqrt(5.0)) / 2.0
    a, b = phi / math.sqrt(1.0 + phi * phi), 1.0 / math.sqrt(1.0 + phi * phi)
    signs = [(1, 1), (1, -1), (-1, 1), (-1, -1)]
    points = [(sa * a, sb * b, 0.0) for sa, sb in signs] + [(0.0, sa * a, sb * b) for sa, sb in signs] + \
        [(sa * b, 0.0, sb * a) for sa, sb in ((1, 1), (-1, 1), (1, -1), (-1, -1))]
    faces = [(2, 11, 3), (2, 5, 11), (11, 5, 10), (5, 0, 10), (0, 5, 4), (4, 5, 2), (4, 2, 9), (9, 2, 3),
             (9, 3, 6), (9, 6, 8), (4, 9, 8), (4, 8, 0), (0, 8, 1), (1, 8, 6), (1, 6, 7), (7, 6, 3),
             (11, 7, 3), (11, 10, 7), (10, 1, 7), (10, 0, 1)]
    points = [np.array(pt) for pt in points]
    for _ in range(levels):
        middle = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in middle:
                m = points[i] + points[j]
                middle[key] = len(points)
                points.append(m / math.sqrt(float(m @ m)))
            return middle[key]

        split = []
        for p_, q_, r_ in faces:
            pq, qr, rp = mid(p_, q_), mid(q_, r_), mid(r_, p_)
            split += [(p_, pq, rp), (pq, q_, qr), (rp, pq, qr), (rp, qr, r_)]
        faces = split
    return np.array(points), np.array(faces, dtype=np.int32)


def _unit(p):
    """p / |p| as the reciprocal times p, row by row."""

    return (1.0 / np.sqrt(_dot(p, p)))[:, None] * p


def _sequential_sum(values: np.ndarray) -> np.ndarray:
    """Left-to-right sum over the first axis (numpy's own sum is pairwise)."""

    return np.cumsum(values, axis=0)[-1]


def sheet_directions(nx: int, ny: int) -> np.ndarray:
    """Unit points of the sheet cell centres, (u, v) = ((x + 0.5) / nx, (y + 0.5) / ny).

    Uses the C library's sin and cos (Python's ``math``), not numpy's own.
    """

    out = np.empty((nx * ny, 3))
    for cell in range(nx * ny):
        u = ((cell % nx) + 0.5) / nx
        v = ((cell // nx) + 0.5) / ny
        out[cell] = (math.sin(v * math.pi) * math.cos(2.0 * math.pi * u),
                     math.sin(v * math.pi) * math.sin(2.0 * math.pi * u), math.cos(v * math.pi))
    return out


def surface_stencil(sphere, sphere_faces, resampling_points, normalize: bool = True, rows=None):
    """(sphere points, surface indices, surface weights, normalised input points) of the helper.

    With ``rows`` only those resampling points are located (the placement
    still uses every input point).
    """

    p = np.asarray(sphere, dtype=np.float32).astype(np.float64)
    faces = np.asarray(sphere_faces, dtype=np.int64)
    if normalize:
        p = _unit(p - (1.0 / p.shape[0]) * _sequential_sum(p))
    radius = 0.975 * _sequential_sum(np.sqrt(_dot(p, p))) / p.shape[0]
    centre = p.min(axis=0) + p.max(axis=0)
    u = _unit(np.asarray(resampling_points, dtype=np.float64))
    if rows is not None:
        u = u[np.asarray(rows)]
    face, w = locate(p, faces, centre + radius * u)
    tri = faces[face]
    resampled = (w[:, 0:1] * p[tri[:, 0]] + w[:, 1:2] * p[tri[:, 1]]) + w[:, 2:3] * p[tri[:, 2]]
    return resampled, tri.astype(np.int32), w, p


def sheet_stencil(sphere_points, faces, nx: int, ny: int, cells=None):
    """Sheet indices [ny, nx, 3] and weights of the cell centres on the unit-normalised sphere points.

    With ``cells`` (flat cell ids) only those cells, as [len(cells), 3] arrays.
    """

    p = _unit(np.asarray(sphere_points, dtype=np.float64))
    faces = np.asarray(faces, dtype=np.int64)
    directions = sheet_directions(nx, ny)
    if cells is not None:
        face, w = locate(p, faces, directions[np.asarray(cells)])
        return faces[face].astype(np.int32), w
    face, w = locate(p, faces, directions)
    return faces[face].astype(np.int32).reshape(ny, nx, 3), w.reshape(ny, nx, 3)
