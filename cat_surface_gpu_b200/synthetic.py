"""Seeded synthetic cortical-like meshes for parity tests and benchmarks.

There are no public anatomical inputs for these paths (the reference's own
anatomical fixtures are private), so every test and benchmark input is built
here from a seed:

* ``folded_icosphere`` -- an icosahedron subdivided ``k`` times
  (``k = 5``: 10,242 vertices, 20,480 triangles), radially displaced by
  ``r = 1 + sum_{l=4..16} sum_m c_lm Y_lm`` with ``c_lm ~ N(0, 0.08^2 / l)``,
  scaled to 60 mm.
* ``folded_hull`` -- the convex hull of ``n`` seeded, jittered Fibonacci points
  on the unit sphere (``n = 61,442``: 122,880 triangles), folded radially by
  ``r = exp(sum_{l=8..40} sum_m c_lm Y_lm)`` with ``c_lm ~ N(0, 0.15^2 / l)``,
  scaled to 70 mm.  The exponential keeps every radius positive; the plain
  ``1 + sum`` form with these coefficients crosses zero and produces a surface
  through the origin.
* ``unit_icosphere`` -- the unit icosphere used for resampling spheres
  (subdivision 6: 40,962 vertices, 81,920 triangles).

``Y_lm`` are real orthonormal spherical harmonics.
"""

from __future__ import annotations

import numpy as np


def _icosahedron() -> tuple[np.ndarray, np.ndarray]:
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = np.array(
        [
            [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
            [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
            [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
        ],
        dtype=np.float64,
    )
    faces = np.array(
        [
            [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
            [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
            [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
            [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
        ],
        dtype=np.int64,
    )
    return verts / np.linalg.norm(verts, axis=1, keepdims=True), faces


def unit_icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere by repeated 1-to-4 midpoint subdivision (vectorised)."""

    verts, faces = _icosahedron()
    for _ in range(int(subdivisions)):
        edges = np.concatenate((faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]), axis=0)
        edges.sort(axis=1)
        unique, inverse = np.unique(edges, axis=0, return_inverse=True)
        inverse = inverse.reshape(-1)
        mid = verts[unique[:, 0]] + verts[unique[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = verts.shape[0]
        nf = faces.shape[0]
        m01 = base + inverse[:nf]
        m12 = base + inverse[nf : 2 * nf]
        m20 = base + inverse[2 * nf :]
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.concatenate(
            (
                np.stack((a, m01, m20), axis=1),
                np.stack((b, m12, m01), axis=1),
                np.stack((c, m20, m12), axis=1),
                np.stack((m01, m12, m20), axis=1),
            ),
            axis=0,
        )
        verts = np.concatenate((verts, mid), axis=0)
    return verts, faces.astype(np.int32)


def _normalised_legendre(x: np.ndarray, lmax: int) -> list[list[np.ndarray]]:
    """Orthonormal associated Legendre functions ``Pbar[m][l]`` for 0 <= m <= l <= lmax.

    Standard three-term recurrence in ``l`` for fixed ``m``, seeded by the
    sectoral terms; normalised so that ``Pbar_l^m(cos t) e^{i m p}`` is
    orthonormal on the unit sphere.
    """

    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    table: list[list[np.ndarray]] = []
    sectoral = np.full_like(x, np.sqrt(1.0 / (4.0 * np.pi)))
    for m in range(lmax + 1):
        if m > 0:
            sectoral = -np.sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * sectoral
        column: list[np.ndarray] = [np.zeros_like(x)] * m + [sectoral]
        if m + 1 <= lmax:
            column.append(np.sqrt(2.0 * m + 3.0) * x * sectoral)
        for degree in range(m + 2, lmax + 1):
            a = np.sqrt((4.0 * degree * degree - 1.0) / (degree * degree - m * m))
            b = np.sqrt(((degree - 1.0) ** 2 - m * m) / (4.0 * (degree - 1.0) ** 2 - 1.0))
            column.append(a * (x * column[degree - 1] - b * column[degree - 2]))
        table.append(column)
    return table


def real_sph_harm_sum(points: np.ndarray, degrees: range, sigma: float, rng: np.random.Generator) -> np.ndarray:
    """``sum_l sum_m c_lm Y_lm(p)`` with ``c_lm ~ N(0, sigma^2 / l)``.

    Coefficients are drawn degree by degree, ``2l + 1`` per degree in the
    order ``m = -l .. l``.
    """

    p = np.asarray(points, dtype=np.float64)
    x = np.clip(p[:, 2] / np.linalg.norm(p, axis=1), -1.0, 1.0)
    phi = np.arctan2(p[:, 1], p[:, 0])
    lmax = max(degrees)
    legendre = _normalised_legendre(x, lmax)
    cos_m = [np.cos(m * phi) for m in range(lmax + 1)]
    sin_m = [np.sin(m * phi) for m in range(lmax + 1)]
    total = np.zeros(p.shape[0], dtype=np.float64)
    root2 = np.sqrt(2.0)
    for degree in degrees:
        coeffs = rng.normal(0.0, sigma / np.sqrt(degree), size=2 * degree + 1)
        for index, order in enumerate(range(-degree, degree + 1)):
            m = abs(order)
            if order < 0:
                basis = root2 * legendre[m][degree] * sin_m[m]
            elif order == 0:
                basis = legendre[0][degree]
            else:
                basis = root2 * legendre[m][degree] * cos_m[m]
            total += coeffs[index] * basis
    return total


def folded_icosphere(subdivisions: int = 5, seed: int = 0, radius_mm: float = 60.0) -> tuple[np.ndarray, np.ndarray]:
    """Folded icosphere (10,242 vertices at the default subdivision 5)."""

    rng = np.random.default_rng(seed)
    verts, faces = unit_icosphere(subdivisions)
    r = 1.0 + real_sph_harm_sum(verts, range(4, 17), 0.08, rng)
    return (verts * (r * radius_mm)[:, None]).astype(np.float32), faces


def fibonacci_points(n: int, rng: np.random.Generator, jitter: float = 0.3) -> np.ndarray:
    """Jittered Fibonacci points on the unit sphere, ordered by descending z."""

    index = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * index + 1.0) / n
    golden = np.pi * (3.0 - np.sqrt(5.0))
    azimuth = golden * index
    spacing = np.sqrt(4.0 * np.pi / n)
    polar = np.arccos(z) + jitter * spacing * rng.uniform(-0.5, 0.5, n)
    polar = np.clip(polar, 1e-6, np.pi - 1e-6)
    azimuth = azimuth + jitter * spacing * rng.uniform(-0.5, 0.5, n) / np.maximum(np.sin(polar), 1e-3)
    return np.stack(
        (np.sin(polar) * np.cos(azimuth), np.sin(polar) * np.sin(azimuth), np.cos(polar)),
        axis=1,
    )


def hull_faces(points: np.ndarray) -> np.ndarray:
    """Outward-oriented triangles of the convex hull of points on a sphere."""

    from scipy.spatial import ConvexHull

    hull = ConvexHull(points)
    faces = hull.simplices.astype(np.int64)
    tri = points[faces]
    normal = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    flip = (normal * tri.mean(axis=1)).sum(axis=1) < 0.0
    faces[flip] = faces[flip][:, [0, 2, 1]]
    if np.unique(faces).size != points.shape[0]:
        raise RuntimeError("convex hull dropped vertices; use a smaller jitter")
    return faces.astype(np.int32)


def folded_hull(n_vertices: int = 61442, seed: int = 0, radius_mm: float = 70.0) -> tuple[np.ndarray, np.ndarray]:
    """Folded convex-hull mesh (61,442 vertices / 122,880 triangles by default)."""

    rng = np.random.default_rng(seed)
    points = fibonacci_points(int(n_vertices), rng)
    faces = hull_faces(points)
    r = np.exp(real_sph_harm_sum(points, range(8, 41), 0.15, rng))
    return (points * (r * radius_mm)[:, None]).astype(np.float32), faces


def folded_hull_and_sphere(n_vertices: int, seed: int, radius_mm: float = 70.0):
    """:func:`folded_hull` and its spherical parametrisation (the unfolded points at 100 mm).

    The fold is radial, so the hull's own unit points map the folded surface
    to the sphere: (vertices float32 [n, 3], faces int32 [m, 3], sphere
    float32 [n, 3]).
    """

    rng = np.random.default_rng(seed)
    points = fibonacci_points(int(n_vertices), rng)
    faces = hull_faces(points)
    r = np.exp(real_sph_harm_sum(points, range(8, 41), 0.15, rng))
    return ((points * (r * radius_mm)[:, None]).astype(np.float32), faces,
            (100.0 * points).astype(np.float32))


def registration_subjects(count: int = 16, seed: int = 5005) -> list[tuple[int, int]]:
    """(vertex count, seed) of the subjects of the batched registration workload.

    Vertex counts are drawn uniformly from 40,962..163,842 (sorted); each
    subject is ``folded_hull_and_sphere(n, seed)``.
    """

    rng = np.random.default_rng(seed)
    sizes = sorted(int(v) for v in rng.integers(40962, 163843, size=int(count)))
    return [(n, 700 + i) for i, n in enumerate(sizes)]


def smooth_sheet(ny: int, nx: int, seed: int, n_modes: int = 12) -> np.ndarray:
    """A smooth, periodic-in-x feature sheet in [0, 1] (synthetic DARTEL input)."""

    rng = np.random.default_rng(seed)
    y = (np.arange(ny) + 0.5) / ny
    x = (np.arange(nx) + 0.5) / nx
    yy, xx = np.meshgrid(y, x, indexing="ij")
    total = np.zeros((ny, nx), dtype=np.float64)
    for _ in range(n_modes):
        kx = rng.integers(1, 6)
        ky = rng.integers(1, 6)
        total += rng.normal() * np.cos(2 * np.pi * kx * xx + rng.uniform(0, 2 * np.pi)) * np.sin(np.pi * ky * yy + rng.uniform(0, np.pi))
    total -= total.min()
    total /= max(total.max(), 1e-12)
    return total
