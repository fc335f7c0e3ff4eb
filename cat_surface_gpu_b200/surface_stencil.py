"""Spherical resampling stencils (drop-in for the reference's surface_stencil).

``SurfaceStencil`` reads the ``.stencil`` v1/v2 files written by the
upstream helper (format of ``src/cat_surface_gpu/surface_stencil.py:16-17,
128-191``): an 8 x int32 header (magic 0x46534354, version, points,
triangles, sheet cells, nx, ny, source points), float64 sphere points, int32
faces, int32 + float64 surface barycentrics, int32 + float64 sheet
barycentrics and (v2) float32 unit-sphere points of the source mesh.
``SurfaceStencilDevice`` holds the device copies and runs the feature
operators on native kernels (``csrc/features.cu``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path
import struct

import numpy as np
import torch

from .device import resolve_device

_HEADER = struct.Struct("<8i")
_MAGIC = 0x46534354


@dataclass(frozen=True)
class SurfaceStencil:
    """CPU indices, barycentric weights, topology, and unit-sphere points."""

    sphere_points: np.ndarray
    faces: np.ndarray
    surface_indices: np.ndarray
    surface_weights: np.ndarray
    sheet_indices: np.ndarray
    sheet_weights: np.ndarray
    nx: int
    ny: int
    source_points: int
    unit_sphere_points: np.ndarray | None = None
    # page-locked block holding the arrays above (a GPU-built stencil): uploads copy from views of
    # it, so torch's pinned-memory cache keeps the block until those copies have run
    pinned: torch.Tensor | None = field(default=None, repr=False, compare=False)

    @classmethod
    def from_file(cls, path) -> "SurfaceStencil":
        """Read a versioned stencil (reference 128-191); ValueError on a bad file."""

        with Path(path).open("rb") as stream:
            header = stream.read(_HEADER.size)
            if len(header) != _HEADER.size:
                raise ValueError("Stencil file")
            magic, version, n_points, n_tri, n_sheet, nx, ny, source_points = _HEADER.unpack(header)
            if magic != _MAGIC or version not in (1, 2):
                raise ValueError("Stencil file magic or")
            if min(n_points, n_tri, n_sheet, nx, ny, source_points) < 0 or n_sheet != nx * ny:
                raise ValueError(f"Stencil file header: points {n_points}, triangles {n_tri}, sheet {n_sheet} "
                                 f"({nx} x {ny}), source points {source_points}")
            sphere_points = np.fromfile(stream, dtype="<f8", count=3 * n_points)
            faces = np.fromfile(stream, dtype="<i4", count=3 * n_tri)
            surface_indices = np.fromfile(stream, dtype="<i4", count=3 * n_points)
            surface_weights = np.fromfile(stream, dtype="<f8", count=3 * n_points)
            sheet_indices = np.fromfile(stream, dtype="<i4", count=3 * n_sheet)
            sheet_weights = np.fromfile(stream, dtype="<f8", count=3 * n_sheet)
            unit = np.fromfile(stream, dtype="<f4", count=3 * source_points) if version == 2 else None
        sizes = (sphere_points.size, faces.size, surface_indices.size, surface_weights.size, sheet_indices.size,
                 sheet_weights.size)
        expected = (3 * n_points, 3 * n_tri, 3 * n_points, 3 * n_points, 3 * n_sheet, 3 * n_sheet)
        if sizes != expected:
            raise ValueError("Stencil file length")
        if unit is not None and unit.size != 3 * source_points:
            raise ValueError("Stencil unit sphere length")
        stencil = cls(
            sphere_points=sphere_points.reshape(n_points, 3),
            faces=faces.reshape(n_tri, 3),
            surface_indices=surface_indices.reshape(n_points, 3),
            surface_weights=surface_weights.reshape(n_points, 3),
            sheet_indices=sheet_indices.reshape(ny, nx, 3),
            sheet_weights=sheet_weights.reshape(ny, nx, 3),
            nx=nx,
            ny=ny,
            source_points=source_points,
            unit_sphere_points=None if unit is None else unit.reshape(source_points, 3),
        )
        stencil.validate()
        return stencil

    def validate(self) -> None:
        """``ValueError`` unless every index is in range and every value finite.

        The device kernels gather with these indices, so a corrupt file must
        be refused on the host: faces and sheet barycentrics index the sphere
        points, surface barycentrics the source mesh's vertices.
        """

        n = int(self.sphere_points.shape[0])
        checks = (("faces", self.faces, n), ("surface_indices", self.surface_indices, int(self.source_points)),
                  ("sheet_indices", self.sheet_indices, n))
        for name, indices, bound in checks:
            if indices.size and (int(indices.min()) < 0 or int(indices.max()) >= bound):
                raise ValueError(f"Stencil {name} outside [0, {bound})")
        for name, values in (("sphere points", self.sphere_points), ("surface weights", self.surface_weights),
                             ("sheet weights", self.sheet_weights), ("unit sphere points", self.unit_sphere_points)):
            if values is not None and not np.isfinite(values).all():
                raise ValueError(f"Stencil {name} are not finite")

    def to_file(self, path) -> None:
        """Write the v2 (v1 without unit points) layout read by ``from_file``."""

        version = 1 if self.unit_sphere_points is None else 2
        with Path(path).open("wb") as stream:
            stream.write(_HEADER.pack(_MAGIC, version, self.sphere_points.shape[0], self.faces.shape[0],
                                      self.nx * self.ny, self.nx, self.ny, self.source_points))
            for array, dtype in ((self.sphere_points, "<f8"), (self.faces, "<i4"), (self.surface_indices, "<i4"),
                                 (self.surface_weights, "<f8"), (self.sheet_indices, "<i4"),
                                 (self.sheet_weights, "<f8")):
                np.ascontiguousarray(array, dtype=dtype).tofile(stream)
            if self.unit_sphere_points is not None:
                np.ascontiguousarray(self.unit_sphere_points, dtype="<f4").tofile(stream)

    def to(self, device, *, geometry_dtype: torch.dtype = torch.float32,
           weight_dtype: torch.dtype = torch.float64) -> "SurfaceStencilDevice":
        """Upload the stencil and its topology tables to one CUDA device (reference 193-272)."""

        from . import features

        target = resolve_device(device)
        return features.upload_stencil(self, target, geometry_dtype, weight_dtype)


@dataclass
class SurfaceStencilDevice:
    """Device-resident stencil, neighbour CSR and per-device feature workspace."""

    sphere_points: torch.Tensor
    faces: torch.Tensor
    surface_indices: torch.Tensor
    surface_weights: torch.Tensor
    sheet_indices: torch.Tensor
    sheet_weights: torch.Tensor
    nx: int
    ny: int
    source_points: int
    unit_sphere_points: torch.Tensor | None = None
    neighbour_offsets: torch.Tensor | None = None
    neighbour_indices: torch.Tensor | None = None
    max_degree: int = 0
    _cache: dict = field(default_factory=dict, repr=False)

    def resample_vertices(self, vertices):
        from . import features

        return features.resample_vertices(self, vertices)

    def map_values_to_sheet(self, values):
        from . import features

        return features.map_values_to_sheet(self, values)

    def smooth_geometry(self, vertices, fwhm: float):
        from . import features

        return features.smooth_geometry(self, vertices, fwhm)

    def smooth_values(self, values, vertices, fwhm: float):
        from . import features

        return features.smooth_values(self, values, vertices, float(fwhm))

    def smooth_values_many(self, values, vertices, fwhms):
        from . import features

        return features.smooth_values_many(self, values, vertices, tuple(float(f) for f in fwhms))

    def vertex_normals(self, vertices):
        from . import features

        return features.vertex_normals(self, vertices)

    def curvature_type5(self, vertices, fwhm: float):
        from . import features

        return features.curvature_type5(self, vertices, fwhm)

    def curvature_type5_to_sheet_many(self, vertices, fwhms):
        from . import features

        return features.curvature_type5_to_sheet_many(self, vertices, tuple(float(f) for f in fwhms))

    def curvature_type2(self, vertices, fwhm: float):
        from . import features

        return features.curvature_type2(self, vertices, fwhm)

    def curvature_to_sheet(self, vertices, fwhm: float, *, curvtype: int = 5):
        from . import features

        return features.curvature_to_sheet(self, vertices, fwhm, curvtype)

    def color_groups(self) -> tuple[torch.Tensor, ...]:
        """Greedy first-fit colouring of the stencil mesh (reference 69-91, 333-347), one index tensor per colour."""

        from .rotation_feature import _stencil_topology

        return tuple(torch.as_tensor(g, device=self.faces.device) for g in _stencil_topology(self).groups)


_RESAMPLING_SPHERES: dict[int, tuple[np.ndarray, np.ndarray]] = {}

# The base icosahedron of the resampling sphere, in the vertex and face order
# of the upstream tetrahedral sphere the stencil helper builds
# (create_tetrahedral_sphere, called at native/cat_surface_stencil_builder.c:
# 406-421): vertices (+-a, +-b, 0), (0, +-a, +-b), (+-b, 0, +-a) with
# a = phi / sqrt(1 + phi^2), b = 1 / sqrt(1 + phi^2) (phi the golden ratio).
# The order of vertices and faces is the helper's, read off the face list of
# its stencil files; the subdivision below then reproduces that face list
# exactly, so stencils index the same resampling points as the helper's.
_ICOSA_A = 0.85065080835203993  # phi / sqrt(1 + phi^2)
_ICOSA_B = 0.52573111211913359  # 1 / sqrt(1 + phi^2)
_ICOSA_SIGNS = ((1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1),
                (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1))
_ICOSA_FACES = ((2, 11, 3), (2, 5, 11), (11, 5, 10), (5, 0, 10), (0, 5, 4), (4, 5, 2), (4, 2, 9), (9, 2, 3),
                (9, 3, 6), (9, 6, 8), (4, 9, 8), (4, 8, 0), (0, 8, 1), (1, 8, 6), (1, 6, 7), (7, 6, 3),
                (11, 7, 3), (11, 10, 7), (10, 1, 7), (10, 0, 1))


def tetrahedral_sphere(subdivisions: int = 6) -> tuple[np.ndarray, np.ndarray]:
    """Unit sphere of 20 * 4^subdivisions triangles in the upstream tetrahedral-sphere order.

    Each level splits every triangle (a, b, c), in face order, into
    (a, ab, ca), (ab, b, bc), (ca, ab, bc), (ca, bc, c); a new edge midpoint
    takes the next vertex number the first time its edge is met (edges
    visited ab, bc, ca) and is the normalised sum of its end points.  Six
    levels give the helper's 40,962 points and 81,920 faces.
    """

    if subdivisions < 0:
        raise ValueError("subdivisions must be non-negative")
    a, b = _ICOSA_A, _ICOSA_B
    points = np.array([(sx * a, sy * b, 0.0) if i < 4 else (0.0, sy * a, sz * b) if i < 8 else (sx * b, 0.0, sz * a)
                       for i, (sx, sy, sz) in enumerate(_ICOSA_SIGNS)], dtype=np.float64)
    faces = np.array(_ICOSA_FACES, dtype=np.int64)
    for _ in range(int(subdivisions)):
        nf = faces.shape[0]
        ends = np.stack((faces, np.roll(faces, -1, axis=1)), axis=2).reshape(3 * nf, 2)  # ab, bc, ca per face
        keys = np.sort(ends, axis=1)
        unique, first, inverse = np.unique(keys, axis=0, return_index=True, return_inverse=True)
        rank = np.empty(unique.shape[0], dtype=np.int64)
        rank[np.argsort(first, kind="stable")] = np.arange(unique.shape[0])
        mids = points.shape[0] + rank[inverse.reshape(-1)].reshape(nf, 3)
        summed = points[unique[:, 0]] + points[unique[:, 1]]
        new_points = np.empty_like(summed)
        new_points[rank] = summed / np.sqrt((summed * summed).sum(axis=1, keepdims=True))
        ab, bc, ca = mids[:, 0], mids[:, 1], mids[:, 2]
        fa, fb, fc = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.stack((np.stack((fa, ab, ca), 1), np.stack((ab, fb, bc), 1), np.stack((ca, ab, bc), 1),
                          np.stack((ca, bc, fc), 1)), axis=1).reshape(4 * nf, 3)
        points = np.concatenate((points, new_points), axis=0)
    return points, faces.astype(np.int32)


def resampling_sphere(subdivisions: int = 6) -> tuple[np.ndarray, np.ndarray]:
    """The stencil helper's resampling sphere: :func:`tetrahedral_sphere` (6: 40,962 points / 81,920 triangles)."""

    if subdivisions not in _RESAMPLING_SPHERES:
        points, faces = tetrahedral_sphere(subdivisions)
        points = np.array(points, dtype=np.float64, order="C")
        faces = np.array(faces, dtype=np.int32, order="C")
        # shared by every stencil of this resolution (lookups key on the array itself): read-only
        points.flags.writeable = False
        faces.flags.writeable = False
        _RESAMPLING_SPHERES[subdivisions] = (points, faces)
    return _RESAMPLING_SPHERES[subdivisions]


def build_surface_stencil(sphere_vertices, sphere_faces, *, nx: int = 512, ny: int = 256, normalize: bool = True,
                          subdivisions: int = 6, threads: int = 0, device=None) -> SurfaceStencil:
    """Build a resampling stencil for a sphere mesh.

    The reference's stencil helper (``native/cat_surface_stencil_builder.c``;
    ``--surface`` mode: the surface shares the sphere's topology, so surface
    indices are sphere vertex ids), restated in float64: the helper's
    tetrahedral resampling sphere placed at the per-axis (min + max) centre
    with 0.975 x the mean radius, its closest-polygon rule, the resampled
    sphere and the sheet of the cell centres.  It equals the helper's files
    up to the helper's own float32 rounding (``tests/test_stencil_helper.py``)
    and writes any sheet size, not only the helper's 512 x 256.
    ``normalize=False`` matches the helper's ``--no-normalize`` (for spheres
    that are already unit and centred).  With a CUDA ``device`` the queries
    run on that GPU (``csg_stencil_build_device``); otherwise the threaded
    host builder (``csg_stencil_build``).  Both give bit-identical stencils.
    """

    from . import _native

    sphere = np.ascontiguousarray(sphere_vertices, dtype=np.float32)
    faces = np.ascontiguousarray(sphere_faces, dtype=np.int32)
    if sphere.ndim != 2 or sphere.shape[1] != 3 or faces.ndim != 2 or faces.shape[1] != 3:
        raise ValueError("sphere_vertices and sphere_faces must have shape [n, 3] and [m, 3]")
    rpts, rfaces = resampling_sphere(subdivisions)
    n = rpts.shape[0]
    target = None if device is None else torch.device(device)
    on_gpu = target is not None and target.type == "cuda"

    shapes = (((n, 3), np.float64), ((n, 3), np.int32), ((n, 3), np.float64), ((ny, nx, 3), np.int32),
              ((ny, nx, 3), np.float64), (tuple(sphere.shape), np.float32))
    if on_gpu:
        # a GPU build reads its results back into one page-locked block (the build writes every
        # element), which the upload to the device (SurfaceStencil.to) then copies asynchronously
        sizes = [(int(np.prod(shape)) * np.dtype(dt).itemsize + 7) // 8 * 8 for shape, dt in shapes]
        pinned = torch.empty(sum(sizes), dtype=torch.uint8, pin_memory=True)
        block = pinned.numpy()
        arrays, offset = [], 0
        for (shape, dt), size in zip(shapes, sizes):
            arrays.append(block[offset: offset + int(np.prod(shape)) * np.dtype(dt).itemsize].view(dt).reshape(shape))
            offset += size
    else:
        pinned = None
        arrays = [np.zeros(shape, dtype=dt) for shape, dt in shapes]
    sphere_points, surface_indices, surface_weights, sheet_indices, sheet_weights, unit = arrays
    lib = _native.library()
    outputs = (sphere_points.ctypes.data, surface_indices.ctypes.data, surface_weights.ctypes.data,
               sheet_indices.ctypes.data, sheet_weights.ctypes.data, unit.ctypes.data)
    inputs = (sphere.ctypes.data, sphere.shape[0], faces.ctypes.data, faces.shape[0], rpts.ctypes.data, n,
              rfaces.ctypes.data, rfaces.shape[0], int(nx), int(ny), int(bool(normalize)))
    if on_gpu:
        need = int(lib.csg_stencil_scratch_bytes(sphere.shape[0], faces.shape[0], n, rfaces.shape[0], int(nx),
                                                 int(ny)))
        if need == 0:
            raise ValueError("stencil build: bad sizes")
        with torch.cuda.device(target):
            scratch = torch.empty(need, dtype=torch.uint8, device=target)
            _native.check(lib.csg_stencil_build_device(*inputs, *outputs, scratch.data_ptr(), need,
                                                       _native.stream_handle(like=scratch)),
                          "csg_stencil_build_device")
    else:
        _native.check(lib.csg_stencil_build(*inputs, int(threads), *outputs), "csg_stencil_build")
    return SurfaceStencil(sphere_points=sphere_points, faces=rfaces, surface_indices=surface_indices,
                          surface_weights=surface_weights, sheet_indices=sheet_indices, sheet_weights=sheet_weights,
                          nx=int(nx), ny=int(ny), source_points=int(sphere.shape[0]), unit_sphere_points=unit,
                          pinned=pinned)
