"""ORACLE (test infrastructure): ctypes front end of ``depth_oracle.c``.

Restates the depth-potential rotation feature of
``src/cat_surface_gpu/rotation_feature.py`` (stable normals 37-74, mixed
Voronoi areas 77-128, system entries 131-171, CG 189-250, coloured SOR
253-317, ``compute_rotation_feature`` 320-401) and the greedy colouring of
``src/cat_surface_gpu/surface_stencil.py:69-91``.  Pinned against the
reference's own torch CPU outputs in ``tests/golden/depth_golden.npz``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import features as ofeat
from .build import build

EPS = float(np.finfo(np.float64).eps)
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(str(build()))
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib.od_depth_setup.restype = I
        lib.od_depth_setup.argtypes = [P, I, P, I, P, P, D, P, P, P, P, P, P, P, P]
        lib.od_depth_sor.restype = I
        lib.od_depth_sor.argtypes = [I, P, P, P, P, P, D, P, P, I, I, D, P, P]
        lib.od_depth_pcg.restype = I
        lib.od_depth_pcg.argtypes = [I, P, P, P, P, P, D, I, D, P, P, P]
        lib.od_blocked_sum.restype = D
        lib.od_blocked_sum.argtypes = [P, ctypes.c_int64]
        _LIB = lib
    return _LIB


def blocked_sum(terms) -> float:
    t = np.ascontiguousarray(terms, dtype=np.float64)
    return float(_lib().od_blocked_sum(t.ctypes.data, t.size))


def incidences(faces, n):
    """Per-vertex incidences ``face << 2 | corner`` sorted by (corner, face): index_add_'s order."""

    f = np.asarray(faces, dtype=np.int64)
    vertex = f.T.reshape(-1)
    corner = np.repeat(np.arange(3), f.shape[0])
    face = np.tile(np.arange(f.shape[0]), 3)
    order = np.lexsort((face, corner, vertex))
    inc = ((face[order] << 2) | corner[order]).astype(np.int32)
    off = np.concatenate(([0], np.cumsum(np.bincount(vertex, minlength=n)))).astype(np.int32)
    return off, inc


def colour_groups(faces, n):
    """Greedy first-fit colouring in vertex order; each colour's vertices ascending."""

    nb, mask = ofeat.neighbour_table(faces, n)
    colours = np.full(n, -1, dtype=np.int64)
    for v in range(n):
        used = {int(colours[w]) for w in nb[v, mask[v]] if colours[w] >= 0}
        c = 0
        while c in used:
            c += 1
        colours[v] = c
    return tuple(np.flatnonzero(colours == c) for c in range(int(colours.max()) + 1))


class System:
    """Normals, areas, the rows of the system, its diagonal and the right-hand side."""

    def __init__(self, points, faces, alpha=1.0 / 1000.0):
        pts = np.ascontiguousarray(points, dtype=np.float32)
        tri = np.ascontiguousarray(faces, dtype=np.int32)
        n = pts.shape[0]
        inc_off, inc = incidences(tri, n)
        nnz = 3 * int(inc_off[-1]) + n
        self.n = n
        self.normals = np.zeros((n, 3))
        self.areas = np.zeros(n)
        self.row_off = np.zeros(n + 1, dtype=np.int32)
        self.col = np.zeros(nnz, dtype=np.int32)
        self.val = np.zeros(nnz)
        self.diag = np.zeros(n)
        self.rhs = np.zeros(n)
        norm = ctypes.c_double()
        rc = _lib().od_depth_setup(pts.ctypes.data, n, tri.ctypes.data, tri.shape[0], inc_off.ctypes.data,
                                   inc.ctypes.data, float(alpha), self.normals.ctypes.data, self.areas.ctypes.data,
                                   self.row_off.ctypes.data, self.col.ctypes.data, self.val.ctypes.data,
                                   self.diag.ctypes.data, self.rhs.ctypes.data, ctypes.byref(norm))
        if rc != 0:
            raise ValueError(f"od_depth_setup failed ({rc})")
        self.rhs_norm = norm.value

    def sor(self, groups, max_iter, relaxation=1.90):
        off = np.concatenate(([0], np.cumsum([len(g) for g in groups]))).astype(np.int32)
        members = np.concatenate(groups).astype(np.int32)
        x = np.zeros(self.n)
        res = ctypes.c_double()
        _lib().od_depth_sor(self.n, self.row_off.ctypes.data, self.col.ctypes.data, self.val.ctypes.data,
                            self.diag.ctypes.data, self.rhs.ctypes.data, self.rhs_norm, off.ctypes.data,
                            members.ctypes.data, len(groups), int(max_iter), float(relaxation), x.ctypes.data,
                            ctypes.byref(res))
        return x, int(max_iter), res.value

    def pcg(self, max_iter, tolerance):
        x = np.zeros(self.n)
        its, res = ctypes.c_int(), ctypes.c_double()
        _lib().od_depth_pcg(self.n, self.row_off.ctypes.data, self.col.ctypes.data, self.val.ctypes.data,
                            self.diag.ctypes.data, self.rhs.ctypes.data, self.rhs_norm, int(max_iter),
                            float(tolerance), x.ctypes.data, ctypes.byref(its), ctypes.byref(res))
        return x, its.value, res.value


def rotation_feature(smoothed, faces, *, solver="colored-sor", alpha=1.0 / 1000.0, max_iter=1000,
                     tolerance=1.0e-9, groups=None):
    """Normalised feature from the smoothed coarse surface: (values, iterations, residual) (reference 320-401)."""

    system = System(smoothed, faces, alpha)
    if solver == "colored-sor":
        groups = colour_groups(faces, system.n) if groups is None else groups
        values, iterations, residual = system.sor(groups, max_iter)
    else:
        values, iterations, residual = system.pcg(max_iter, tolerance)
    values = ofeat.smooth_values(values, smoothed, faces, 50.0)
    lo, hi = values.min(), values.max()
    return (values - lo) / max(hi - lo, EPS), iterations, residual
