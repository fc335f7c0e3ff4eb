"""ORACLE (test infrastructure): ctypes front end of ``areal_oracle.c``.

Sequential CPU restatement of the reference's ordered area-smoothing sweeps
(``src/cat_surface_gpu/surf2sphere.py:35-280, 1039-1092``) and of its
host-side helpers ``surface_area`` (``surf2sphere.py:461-471``) and
``convert_ellipsoid_to_sphere_with_surface_area`` (``surf2sphere.py:919-937``).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from .build import build

_MODES = {"cat": 0, "fp32": 1, "fp64": 2}
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(str(build()))
        lib.oracle_areal_sweeps.restype = ctypes.c_int
        lib.oracle_areal_sweeps.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
        ]
        lib.oracle_dependency_levels.restype = ctypes.c_int
        lib.oracle_dependency_levels.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        _LIB = lib
    return _LIB


def areal_sweeps(vertices, faces, *, iterations: int, project_every: int, radius: float, arithmetic: str = "cat") -> np.ndarray:
    """Run sweeps 1 .. iterations-1 sequentially; returns a new array."""

    mode = _MODES[arithmetic]
    dtype = np.float64 if mode == 2 else np.float32
    points = np.array(vertices, dtype=dtype, order="C", copy=True)
    tri = np.ascontiguousarray(faces, dtype=np.int32)
    rc = _lib().oracle_areal_sweeps(
        points.ctypes.data, points.shape[0], tri.ctypes.data, tri.shape[0],
        int(iterations), int(project_every), float(radius), mode,
    )
    if rc != 0:
        raise ValueError(f"oracle_areal_sweeps failed ({rc})")
    return points


def dependency_levels(n_points: int, faces) -> np.ndarray:
    """level(v) = 1 + max level of lower-index neighbours (surface_stencil.py:94-109)."""

    tri = np.ascontiguousarray(faces, dtype=np.int32)
    levels = np.zeros(int(n_points), dtype=np.int32)
    count = _lib().oracle_dependency_levels(int(n_points), tri.ctypes.data, tri.shape[0], levels.ctypes.data)
    if count < 0:
        raise ValueError("bad faces")
    return levels


def surface_area(vertices, faces) -> float:
    """Total triangle area in float64 (surf2sphere.py:461-471)."""

    v = np.asarray(vertices).astype(np.float64)
    tri = v[np.asarray(faces).astype(np.int64)]
    cross = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    return float(0.5 * np.linalg.norm(cross, axis=1).sum(dtype=np.float64))


def ellipsoid_to_sphere(vertices, desired_surface_area: float) -> np.ndarray:
    """Scale to the sphere of the given area (surf2sphere.py:919-937)."""

    g = np.ascontiguousarray(vertices, dtype=np.float32)
    radius = math.sqrt(desired_surface_area / (4.0 * math.pi))
    axes = (np.abs(g.min(axis=0)) + np.abs(g.max(axis=0))) * 0.5
    axes = np.maximum(axes, 1.0e-20)
    values = g.astype(np.float64)
    scaled = values / axes[None, :]
    norm = np.sqrt((scaled * scaled).sum(axis=1))
    out = np.zeros_like(values)
    nz = norm != 0.0
    out[nz] = radius * values[nz] / norm[nz, None]
    out[nz] /= axes[None, :]
    return np.ascontiguousarray(out, dtype=np.float32)


def error_stats(reference, candidate) -> dict:
    """max / mean / p99 of |reference - candidate| over all coordinates."""

    d = np.abs(np.asarray(reference, dtype=np.float64) - np.asarray(candidate, dtype=np.float64))
    return {"max": float(d.max()), "mean": float(d.mean()), "p99": float(np.quantile(d, 0.99))}
