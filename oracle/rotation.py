"""ORACLE (test infrastructure): NumPy restatement of the reference's rotation search.

Follows ``src/cat_surface_gpu/surface_rotation.py``:

* ``seed_angles``            -- official_seed_grid_angles (14-23)
* ``build_grid``             -- RotationGridIndex.from_geometry (58-120)
* ``rotation_matrices``      -- _rotation_matrices (223-292), float32
* ``locate``                 -- _locate_chunk (354-453) + _query_grid (455-477)
* ``cost_batch``             -- cost_batch_prepared (512-546)
* ``nelder_mead``            -- refine_nelder_mead_prepared (594-699)

Geometry is float32 with one rounding per operation in a fixed order:
3-term dot products are ``(a0 b0 + a1 b1) + a2 b2``; rotated coordinates
are ``(p0 m[3j] + p1 m[3j+1]) + p2 m[3j+2]`` (the reference multiplies by
the transpose of the row-major reshape of its column-major matrix).
"""

from __future__ import annotations

import numpy as np

F = np.float32


def seed_angles() -> np.ndarray:
    seed0 = (-0.6, -0.3, 0.0, 0.3, 0.6)
    seed12 = (-0.3, 0.0, 0.3)
    values = [(0.0, 0.0, 0.0)] + [(a, b, c) for a in seed0 for b in seed12 for c in seed12]
    return np.asarray(values, dtype=np.float64)


def build_grid(points, faces, grid_size=128, margin=1):
    """CSR (offsets [G^3 + 1], faces) of the triangles whose padded bbox covers each cell."""

    pts = np.asarray(points, dtype=np.float64)
    tri = pts[np.asarray(faces, dtype=np.int64)]
    cell = 2.0 / float(grid_size)
    lower = np.floor((tri.min(axis=1) + 1.0) / cell).astype(np.int64)
    upper = np.floor((tri.max(axis=1) + 1.0) / cell).astype(np.int64)
    lower = np.clip(lower - margin, 0, grid_size - 1)
    upper = np.clip(upper + margin, 0, grid_size - 1)
    cells: dict[int, list[int]] = {}
    for face, (lo, hi) in enumerate(zip(lower, upper)):
        for z in range(lo[2], hi[2] + 1):
            for y in range(lo[1], hi[1] + 1):
                base = grid_size * (y + grid_size * z)
                for x in range(lo[0], hi[0] + 1):
                    cells.setdefault(base + x, []).append(face)
    offsets = np.zeros(grid_size ** 3 + 1, dtype=np.int64)
    flat: list[int] = []
    for c in range(grid_size ** 3):
        flat.extend(cells.get(c, ()))
        offsets[c + 1] = len(flat)
    return offsets.astype(np.int32), np.asarray(flat, dtype=np.int32)


def rotation_matrices(angles) -> np.ndarray:
    """Column-major flat 3x3 matrices Rz (Ry Rx), float32, as the reference builds them."""

    a = np.asarray(angles, dtype=np.float64).reshape(-1, 3).astype(F)
    al, be, ga = a[:, 0], a[:, 1], a[:, 2]
    z, o = np.zeros_like(al), np.ones_like(al)
    rx = np.stack((o, z, z, z, np.cos(al), np.sin(al), z, -np.sin(al), np.cos(al)), axis=1)
    ry = np.stack((np.cos(be), z, np.sin(be), z, o, z, -np.sin(be), z, np.cos(be)), axis=1)
    rz = np.stack((np.cos(ga), np.sin(ga), z, -np.sin(ga), np.cos(ga), z, z, z, o), axis=1)
    first = np.empty_like(rx)
    out = np.empty_like(rx)
    for r in range(3):
        for c in range(3):
            first[:, r + 3 * c] = (ry[:, r] * rx[:, 3 * c] + ry[:, r + 3] * rx[:, 1 + 3 * c]) + ry[:, r + 6] * rx[:, 2 + 3 * c]
    for r in range(3):
        for c in range(3):
            out[:, r + 3 * c] = (rz[:, r] * first[:, 3 * c] + rz[:, r + 3] * first[:, 1 + 3 * c]) + rz[:, r + 6] * first[:, 2 + 3 * c]
    return out


def rotate(points, m) -> np.ndarray:
    p = np.asarray(points, dtype=F)
    return np.stack([(p[:, 0] * m[3 * j] + p[:, 1] * m[3 * j + 1]) + p[:, 2] * m[3 * j + 2] for j in range(3)], axis=1)


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack(
        (
            a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
            a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
            a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0],
        ),
        axis=-1,
    )


def _segment(q, first, second):
    direction = second - first
    offset = q - first
    den = _dot(direction, direction)
    with np.errstate(divide="ignore", invalid="ignore"):
        alpha = np.where(den != 0, _dot(offset, direction) / den, F(0))
    alpha = np.clip(alpha, F(0), F(1)).astype(F)
    closest = first + alpha[..., None] * direction
    d = q - closest
    return _dot(d, d), closest


def locate(q, triangles, candidates):
    """Closest candidate triangle per query point -> (face, barycentric weights [3]).

    q [M, 3] float32; candidates [M, W] int (-1 padded); triangles [F, 3, 3] float32.
    """

    valid = candidates >= 0
    if not valid.any(axis=1).all():
        raise RuntimeError("Rotation is not covered by target sphere candidate index")
    tri = triangles[np.maximum(candidates, 0)]  # [M, W, 3, 3]
    p0, p1, p2 = tri[..., 0, :], tri[..., 1, :], tri[..., 2, :]
    qq = q[:, None, :]
    ea, eb = p1 - p0, p2 - p0
    normal = _cross(ea, eb)
    nsq = _dot(normal, normal)
    with np.errstate(divide="ignore", invalid="ignore"):
        plane_t = np.where(nsq != 0, _dot(p0 - qq, normal) / nsq, F(0)).astype(F)
        projected = qq + plane_t[..., None] * normal
        po = projected - p0
        xx, xy, xv, yy, yv = _dot(ea, ea), _dot(ea, eb), _dot(ea, po), _dot(eb, eb), _dot(eb, po)
        den = xx * yy - xy * xy
        xpos = np.where(den != 0, (xv * yy - yv * xy) / den, F(0)).astype(F)
        ypos = np.where(den != 0, (yv * xx - xv * xy) / den, F(0)).astype(F)
    tol = F(1.0e-3)
    one = F(1.0) + tol
    s = xpos + ypos
    inside = (den != 0) & (xpos >= -tol) & (xpos <= one) & (ypos >= -tol) & (ypos <= one) & (s >= -tol) & (s <= one)
    plane_d = plane_t * plane_t * nsq
    verts = np.stack((p0, p1, p2), axis=-2)
    vd = np.stack([_dot(qq - verts[..., k, :], qq - verts[..., k, :]) for k in range(3)], axis=-1)
    cv = np.argmin(vd, axis=-1)
    take = lambda k: np.take_along_axis(verts, k[..., None, None].repeat(3, -1), axis=-2)[..., 0, :]
    closest = take(cv)
    prev = take((cv - 1) % 3)
    nxt = take((cv + 1) % 3)
    d1, pt1 = _segment(qq, prev, closest)
    d2, pt2 = _segment(qq, closest, nxt)
    first = d1 < d2
    out_d = np.where(first, d1, d2)
    out_p = np.where(first[..., None], pt1, pt2)
    cand_d = np.where(inside, plane_d, out_d)
    cand_p = np.where(inside[..., None], projected, out_p)
    cand_d = np.where(valid, cand_d, F(np.inf))
    best = np.argmin(cand_d, axis=-1)
    rows = np.arange(q.shape[0])
    face = candidates[rows, best]
    point = cand_p[rows, best]
    t = tri[rows, best]
    weights = []
    for a, b, c in ((1, 2, 0), (2, 0, 1), (0, 1, 2)):
        fo = point - t[:, a]
        hz = t[:, b] - t[:, a]
        up = t[:, c] - t[:, a]
        n = _cross(hz, up)
        vert = _cross(n, hz)
        weights.append(_dot(fo, vert) / _dot(up, vert))
    return face, np.stack(weights, axis=-1).astype(F)


def candidates_for(points, offsets, flat, grid_size):
    cell = np.floor((points.astype(F) + F(1.0)) * F(grid_size / 2.0)).astype(np.int64)
    cell = np.clip(cell, 0, grid_size - 1)
    cid = cell[:, 0] + grid_size * (cell[:, 1] + grid_size * cell[:, 2])
    starts, stops = offsets[cid], offsets[cid + 1]
    width = int((stops - starts).max())
    pos = starts[:, None] + np.arange(width)[None, :]
    valid = pos < stops[:, None]
    return np.where(valid, flat[np.minimum(pos, flat.size - 1)], -1)


def cost_batch(target_points, target_faces, target_values, source_points, source_values, angles, grid=None,
               grid_size=128, margin=1):
    """SSD cost per candidate rotation (surface_rotation.py:512-546), float64."""

    tp = np.asarray(target_points, dtype=np.float64)
    tf = np.asarray(target_faces, dtype=np.int64)
    if grid is None:
        grid = build_grid(tp, tf, grid_size, margin)
    offsets, flat = grid
    triangles = tp[tf].astype(F)
    mats = rotation_matrices(angles)
    tv = np.asarray(target_values, dtype=np.float64)
    sv = np.asarray(source_values, dtype=np.float64)
    costs = np.zeros(mats.shape[0])
    for c, m in enumerate(mats):
        q = rotate(source_points, m)
        face, w = locate(q, triangles, candidates_for(q, offsets, flat, grid_size))
        v = tf[face]
        w64 = w.astype(np.float64)
        sampled = (tv[v[:, 0]] * w64[:, 0] + tv[v[:, 1]] * w64[:, 1]) + tv[v[:, 2]] * w64[:, 2]
        d = sv - sampled
        costs[c] = float(np.sum(d * d))
    return costs


def nelder_mead(cost, seed, max_iter=500, tol=1e-4, step=0.1):
    """CAT-ordered Nelder-Mead (surface_rotation.py:594-699); cost(angles [k,3]) -> [k]."""

    seed = np.asarray(seed, dtype=np.float64).reshape(3)
    simplex = np.stack([seed, seed + (step, 0, 0), seed + (0, step, 0), seed + (0, 0, step)])
    f = np.asarray(cost(simplex), dtype=np.float64)
    it = 0
    for it in range(max_iter):
        hi, lo, sh = 0, 0, 1
        for i in range(4):
            if f[i] > f[hi]:
                sh, hi = hi, i
            elif f[i] > f[sh] and i != hi:
                sh = i
            if f[i] < f[lo]:
                lo = i
        centroid = np.zeros(3)
        for i in range(4):
            if i != hi:
                centroid += simplex[i]
        centroid /= 3.0
        refl = centroid + (centroid - simplex[hi])
        fr = cost(refl[None])[0]
        if fr < f[lo]:
            exp = centroid + 2.0 * (refl - centroid)
            fe = cost(exp[None])[0]
            if fe < fr:
                simplex[hi], f[hi] = exp, fe
            else:
                simplex[hi], f[hi] = refl, fr
        elif fr < f[sh]:
            simplex[hi], f[hi] = refl, fr
        else:
            con = centroid + 0.5 * (simplex[hi] - centroid)
            fc = cost(con[None])[0]
            if fc < f[hi]:
                simplex[hi], f[hi] = con, fc
            else:
                for i in range(4):
                    if i != lo:
                        simplex[i] = simplex[lo] + 0.5 * (simplex[i] - simplex[lo])
                        f[i] = cost(simplex[i][None])[0]
        if np.max(np.abs(f - f[lo])) < tol:
            break
    return simplex[lo].copy(), float(f[lo]), it + 1
