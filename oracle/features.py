"""ORACLE (test infrastructure): NumPy restatement of the stencil feature operators.

Follows ``src/cat_surface_gpu/surface_stencil.py``:

* ``resample_vertices``       (282-306)   ``map_values_to_sheet`` (308-317)
* ``heat_parameters``         (359-369)   ``edge_mean_distance``  (347-356)
* ``smooth_geometry``         (372-388)   ``smooth_values``       (390-412)
* ``smooth_values_many``      (414-476)   ``vertex_normals``      (478-505)
* ``curvature_type5``         (507-519)   ``curvature_type5_to_sheet_many`` (521-550)
* ``curvature_type2``         (552-622)   ``curvature_to_sheet``  (624-644)

Neighbour sums run over the unique sorted 1-ring in ascending id order (the
reference's padded neighbour table, ``_build_neighbour_table`` 36-66);
per-vertex normal accumulation runs corner 0 over all faces, then corner 1,
then corner 2, each in face order (the reference's three ``index_add_``).
"""

from __future__ import annotations

import math

import numpy as np


def neighbour_table(faces, n):
    f = np.asarray(faces, dtype=np.int64)
    directed = np.concatenate((f[:, [0, 1]], f[:, [1, 0]], f[:, [1, 2]], f[:, [2, 1]], f[:, [2, 0]], f[:, [0, 2]]))
    directed = np.unique(directed, axis=0)
    counts = np.bincount(directed[:, 0], minlength=n)
    width = int(counts.max())
    table = np.zeros((n, width), dtype=np.int64)
    mask = np.zeros((n, width), dtype=bool)
    offsets = np.concatenate(([0], np.cumsum(counts)))
    for v in range(n):
        row = directed[offsets[v] : offsets[v + 1], 1]
        table[v, : row.size] = row
        mask[v, : row.size] = True
    return table, mask


def _sum_slots(values, mask):
    """Sequential sum over the padded slot axis (axis 1), masked slots add exact zeros."""

    total = np.zeros(values.shape[:1] + values.shape[2:], dtype=values.dtype)
    for k in range(values.shape[1]):
        m = mask[:, k].reshape((-1,) + (1,) * (values.ndim - 2))
        total = total + values[:, k] * m
    return total


def _norm3(v):
    return np.sqrt((v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2])


def edge_mean_distance(vertices, faces):
    g = np.asarray(vertices).astype(np.float64)
    fp = g[np.asarray(faces, dtype=np.int64)]
    return float(np.mean(_norm3(fp[:, [1, 2, 0]] - fp)))


def heat_parameters(vertices, faces, fwhm):
    em = edge_mean_distance(vertices, faces)
    raw = float(fwhm) * float(fwhm) * 0.541011 / (em * em)
    iterations = max(1, int(math.ceil(raw)))
    sigma = float(fwhm) * 0.7355345 / float(iterations ** 0.5)
    return iterations, sigma


def resample_vertices(vertices, indices, weights):
    v = np.asarray(vertices)
    if v.dtype == np.float32:
        result = np.zeros((indices.shape[0], 3), dtype=np.float32)
        for corner in range(3):
            result = result + (v[indices[:, corner]].astype(np.float64) * weights[:, corner, None]).astype(np.float32)
        return result
    s = v[indices] * weights[..., None]
    return (s[:, 0] + s[:, 1]) + s[:, 2]


def map_values_to_sheet(values, sheet_indices, sheet_weights):
    v = np.asarray(values, dtype=np.float64).reshape(-1)
    s = v[sheet_indices] * sheet_weights
    return (s[..., 0] + s[..., 1]) + s[..., 2]


def smooth_geometry(vertices, faces, fwhm, table=None):
    if table is None:
        table = neighbour_table(faces, vertices.shape[0])
    nb, mask = table
    iterations, _ = heat_parameters(vertices, faces, fwhm)
    maskf = mask.astype(np.float64)
    value = np.asarray(vertices, dtype=np.float32)
    count = maskf[:, 0].copy()
    for k in range(1, maskf.shape[1]):
        count = count + maskf[:, k]
    den = 1.0 + count / 3.0
    for _ in range(iterations):
        nv = value[nb].astype(np.float64)
        num = value.astype(np.float64) + _sum_slots(nv, mask) / 3.0
        value = (num / den[:, None]).astype(np.float32)
    return value


def _weights(vertices, nb, mask, sigma, via_norm):
    g = np.asarray(vertices).astype(np.float64)
    diff = g[nb] - g[:, None, :]
    if via_norm:
        d = _norm3(diff)
        dsq = d * d
    else:
        dsq = (diff[..., 0] ** 2 + diff[..., 1] ** 2) + diff[..., 2] ** 2
    return np.exp(-dsq / (2.0 * sigma * sigma)) * mask.astype(np.float64)


def _smooth(values, weights, nb, mask, iterations):
    value = np.asarray(values, dtype=np.float64).copy()
    wsum = _sum_slots(weights, mask)
    for _ in range(iterations):
        num = value + _sum_slots(weights * value[nb], mask)
        value = num / (1.0 + wsum)
    return value


def smooth_values(values, vertices, faces, fwhm, table=None):
    """Single-FWHM smoothing (distances through a vector norm, then squared)."""

    if table is None:
        table = neighbour_table(faces, vertices.shape[0])
    nb, mask = table
    iterations, sigma = heat_parameters(vertices, faces, fwhm)
    return _smooth(values, _weights(vertices, nb, mask, sigma, True), nb, mask, iterations)


def smooth_values_many(values, vertices, faces, fwhms, table=None):
    """Several FWHMs (squared distances summed directly)."""

    if table is None:
        table = neighbour_table(faces, vertices.shape[0])
    nb, mask = table
    out = []
    for fwhm in fwhms:
        iterations, sigma = heat_parameters(np.asarray(vertices, dtype=np.float64), faces, fwhm)
        out.append(_smooth(values, _weights(vertices, nb, mask, sigma, False), nb, mask, iterations))
    return tuple(out)


def vertex_normals(vertices, faces):
    g = np.asarray(vertices, dtype=np.float32)
    f = np.asarray(faces, dtype=np.int64)
    fp = g[f]
    ea = fp[:, 1] - fp[:, 0]
    eb = fp[:, 2] - fp[:, 0]
    fn = np.stack(
        (ea[:, 1] * eb[:, 2] - ea[:, 2] * eb[:, 1], ea[:, 2] * eb[:, 0] - ea[:, 0] * eb[:, 2],
         ea[:, 0] * eb[:, 1] - ea[:, 1] * eb[:, 0]), axis=1)
    eps = np.float32(np.finfo(np.float32).eps)
    fn = fn / np.maximum(_norm3(fn), eps)[:, None]
    acc = np.zeros_like(g)
    for corner in range(3):
        prev = fp[:, (corner - 1) % 3] - fp[:, corner]
        foll = fp[:, (corner + 1) % 3] - fp[:, corner]
        den = np.maximum(_norm3(prev) * _norm3(foll), eps)
        dot = (prev[:, 0] * foll[:, 0] + prev[:, 1] * foll[:, 1]) + prev[:, 2] * foll[:, 2]
        angle = np.arccos(np.clip(dot / den, np.float32(-1.0), np.float32(1.0))).astype(np.float32)
        np.add.at(acc, f[:, corner], fn * angle[:, None])
    return acc / np.maximum(_norm3(acc), eps)[:, None]


def _minmax(values):
    mn, mx = values.min(), values.max()
    return (values - mn) / (mx - mn)


def curvature_type5(vertices, faces, fwhm, table=None):
    if table is None:
        table = neighbour_table(faces, vertices.shape[0])
    g = np.asarray(vertices, dtype=np.float32)
    smoothed = smooth_geometry(g, faces, 50.0, table)
    normals = vertex_normals(smoothed, faces)
    d = smoothed - g
    values = ((d[:, 0] * normals[:, 0] + d[:, 1] * normals[:, 1]) + d[:, 2] * normals[:, 2]).astype(np.float64)
    return _minmax(smooth_values(values, g, faces, fwhm, table))


def curvature_type5_to_sheet_many(vertices, faces, fwhms, sheet_indices, sheet_weights, table=None):
    if table is None:
        table = neighbour_table(faces, vertices.shape[0])
    g = np.asarray(vertices, dtype=np.float32)
    smoothed = smooth_geometry(g, faces, 50.0, table)
    normals = vertex_normals(smoothed, faces)
    d = smoothed - g
    base = ((d[:, 0] * normals[:, 0] + d[:, 1] * normals[:, 1]) + d[:, 2] * normals[:, 2]).astype(np.float64)
    maps = []
    for values in smooth_values_many(base, g, faces, fwhms, table):
        mapped = map_values_to_sheet(_minmax(values), sheet_indices, sheet_weights)
        maps.append(_minmax(mapped))
    return tuple(maps)


def curvature_type2(vertices, faces, fwhm, table=None):
    if table is None:
        table = neighbour_table(faces, vertices.shape[0])
    nb, mask = table
    g = np.asarray(vertices, dtype=np.float32)
    m = mask.astype(np.float64)
    counts = _sum_slots(m[:, :, None], mask)[:, 0] if False else m.sum(axis=1)
    normals = vertex_normals(g, faces).astype(np.float64)
    pts = g.astype(np.float64)
    dc = pts[nb] - pts[:, None, :]
    dn = normals[nb] - normals[:, None, :]
    dot = lambda a, b: (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]
    b0 = dc[:, 0, :]
    b0 = b0 - dot(b0, normals)[:, None] * normals
    b0 = b0 / np.maximum(_norm3(b0), np.finfo(np.float64).eps)[:, None]
    nb_ = -b0
    b1 = np.stack((nb_[:, 1] * normals[:, 2] - nb_[:, 2] * normals[:, 1],
                   nb_[:, 2] * normals[:, 0] - nb_[:, 0] * normals[:, 2],
                   nb_[:, 0] * normals[:, 1] - nb_[:, 1] * normals[:, 0]), axis=1)
    pc = dc - dot(dc, normals[:, None, :])[..., None] * normals[:, None, :]
    pn = dn - dot(dn, normals[:, None, :])[..., None] * normals[:, None, :]
    dcx, dcy = dot(pc, b0[:, None, :]), dot(pc, b1[:, None, :])
    dnx, dny = dot(pn, b0[:, None, :]), dot(pn, b1[:, None, :])
    s1 = (dcx * dnx * m).sum(1)
    s2 = ((dcx * dny + dcy * dnx) * m).sum(1)
    s3 = (dcy * dny * m).sum(1)
    wx = (dcx * dcx * m).sum(1)
    wy = (dcy * dcy * m).sum(1)
    wxy = (dcx * dcy * m).sum(1)
    wx2, wy2, wxy2 = wx * wx, wy * wy, wxy * wxy
    den = (wx + wy) * (-wxy2 + wx * wy)
    safe = np.where(den != 0.0, den, 1.0)
    a = (s3 * wxy2 - s2 * wxy * wy + s1 * (-wxy2 + wx * wy + wy2)) / safe
    b = (-s3 * wx * wxy + s2 * wx * wy - s1 * wxy * wy) / safe
    c = (-s2 * wx * wxy + s1 * wxy2 + s3 * (wx2 - wxy2 + wx * wy)) / safe
    tr = a + c
    det = a * c - b * b
    root = np.sqrt(np.maximum(tr * tr - 4.0 * det, 0.0))
    k1, k2 = (tr + root) / 2.0, (tr - root) / 2.0
    values = np.where(counts > 2.0, np.sqrt((k1 * k1 + k2 * k2) / 2.0), 0.0)
    return _minmax(smooth_values(values, g, faces, fwhm, table))


def curvature_to_sheet(vertices, faces, fwhm, curvtype, sheet_indices, sheet_weights, table=None):
    if curvtype == 5:
        values = curvature_type5(vertices, faces, fwhm, table)
    elif curvtype == 2:
        values = curvature_type2(vertices, faces, fwhm, table)
    else:
        raise NotImplementedError("curvtype must be 2 or 5")
    return _minmax(map_values_to_sheet(values, sheet_indices, sheet_weights))
