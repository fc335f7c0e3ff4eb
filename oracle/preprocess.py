"""ORACLE (test infrastructure): ctypes front end of ``preprocess_oracle.c``.

Sequential CPU restatement of CAT_Surf2Sphere's stages 1-5 as the reference
describes them (``src/cat_surface_gpu/surf2sphere.py:283-397, 474-862``), in
the upstream binary's vertex-index Gauss-Seidel order.  Pinned to the
upstream binary's stage-5 outputs committed in ``tests/golden``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .build import build

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(str(build()))
        lib.oracle_surf2sphere_preprocess.restype = ctypes.c_int
        lib.oracle_surf2sphere_preprocess.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _LIB = lib
    return _LIB


def neighbour_csr(faces, n_points: int) -> tuple[np.ndarray, np.ndarray]:
    """Unique ascending 1-ring of every vertex as CSR (surface_stencil.py:36-66)."""

    f = np.asarray(faces, dtype=np.int64)
    pairs = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]], f[:, [1, 0]], f[:, [2, 1]], f[:, [0, 2]]])
    pairs = np.unique(pairs, axis=0)  # sorted by (vertex, neighbour)
    off = np.zeros(n_points + 1, dtype=np.int32)
    np.add.at(off, pairs[:, 0] + 1, 1)
    return np.cumsum(off).astype(np.int32), pairs[:, 1].astype(np.int32)


def preprocess(vertices, faces, stop_at: int = 5) -> np.ndarray:
    """Stages 1..stop_at on a copy of ``vertices`` (float32); no ellipsoid-to-sphere step."""

    points = np.array(vertices, dtype=np.float32, order="C", copy=True)
    tri = np.ascontiguousarray(faces, dtype=np.int32)
    off, nb = neighbour_csr(tri, points.shape[0])
    rc = _lib().oracle_surf2sphere_preprocess(points.ctypes.data, points.shape[0], tri.ctypes.data, tri.shape[0],
                                              off.ctypes.data, nb.ctypes.data, int(stop_at))
    if rc != 0:
        raise ValueError(f"oracle_surf2sphere_preprocess failed ({rc})")
    return points
