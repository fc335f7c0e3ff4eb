"""SurfWarp initial-rotation search on a B200 (drop-in for the reference's surface_rotation).

Public names and behaviour follow ``src/cat_surface_gpu/surface_rotation.py``:
the 46 official seeds, the CSR grid index over target-sphere triangles,
candidate costs, first-equal-minimum seed choice and CAT-ordered
Nelder-Mead.  The grid is built by the native host builder; every cost is
evaluated by ``csg_rotation_cost_batch`` (one persistent launch for any
number of candidates and surfaces).  Rotation matrices are float32, built on
the host exactly as the reference builds them.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .device import resolve_device


def official_seed_grid_angles() -> np.ndarray:
    """46 upstream seeds: identity, then alpha x beta x gamma (reference 14-23)."""

    seed0 = (-0.6, -0.3, 0.0, 0.3, 0.6)
    seed12 = (-0.3, 0.0, 0.3)
    values = [(0.0, 0.0, 0.0)]
    values.extend((a, b, c) for a in seed0 for b in seed12 for c in seed12)
    return np.asarray(values, dtype=np.float64)


def euler_grid_angles(step_deg: float, center=None, half_width_deg: float | None = None) -> np.ndarray:
    """Euler-angle candidates [C, 3] (radians) on a regular grid, x slowest, z fastest.

    Without ``center``: all of SO(3) -- x and z over [-180, 180), y over
    [-90, 90] -- every ``step_deg`` degrees.  With ``center`` (radians) and
    ``half_width_deg``: ``center + k * step`` for every k with
    |k * step| <= half_width on each axis.  The search takes the first
    minimum in this order.
    """

    step = float(step_deg)
    if step <= 0:
        raise ValueError("step_deg must be positive")
    if center is None:
        ax = np.arange(-180.0, 180.0 - 1e-9, step)
        ay = np.arange(-90.0, 90.0 + 1e-9, step)
        axes = [np.deg2rad(ax), np.deg2rad(ay), np.deg2rad(ax)]
    else:
        if half_width_deg is None or half_width_deg < 0:
            raise ValueError("a centred grid needs a non-negative half_width_deg")
        k = np.arange(-np.floor(half_width_deg / step + 1e-9), np.floor(half_width_deg / step + 1e-9) + 1)
        c = np.asarray(center, dtype=np.float64).reshape(3)
        axes = [c[i] + np.deg2rad(k * step) for i in range(3)]
    grid = np.meshgrid(*axes, indexing="ij")
    return np.stack([g.ravel() for g in grid], axis=1)


def zscore(values) -> np.ndarray:
    """(v - mean) / std per feature row (population std), rounded to float32 and widened back."""

    v = np.asarray(values, dtype=np.float64)
    mean = v.mean(axis=-1, keepdims=True)
    std = v.std(axis=-1, keepdims=True)
    return ((v - mean) / np.where(std > 0, std, 1.0)).astype(np.float32).astype(np.float64)


_ROW0 = np.array([r for c in range(3) for r in range(3)])
_ROW1 = _ROW0 + 3
_ROW2 = _ROW0 + 6
_COL0 = np.array([3 * c for c in range(3) for _ in range(3)])
_COL1 = _COL0 + 1
_COL2 = _COL0 + 2


def rotation_matrices_flat(angles) -> np.ndarray:
    """Column-major flat float32 matrices Rz (Ry Rx) per angle row (reference 223-292)."""

    a = np.asarray(angles, dtype=np.float64).reshape(-1, 3).astype(np.float32)
    al, be, ga = a[:, 0], a[:, 1], a[:, 2]
    z, o = np.zeros_like(al), np.ones_like(al)
    ca, sa, cb, sb, cg, sg = np.cos(al), np.sin(al), np.cos(be), np.sin(be), np.cos(ga), np.sin(ga)
    rx = np.stack((o, z, z, z, ca, sa, z, -sa, ca), axis=1)
    ry = np.stack((cb, z, sb, z, o, z, -sb, z, cb), axis=1)
    rz = np.stack((cg, sg, z, -sg, cg, z, z, z, o), axis=1)
    # entry r + 3 c of left @ right (column-major): (l[r] R[3c] + l[r+3] R[3c+1]) + l[r+6] R[3c+2],
    # all nine entries at once -- the same float32 multiplies and adds per entry
    first = (ry[:, _ROW0] * rx[:, _COL0] + ry[:, _ROW1] * rx[:, _COL1]) + ry[:, _ROW2] * rx[:, _COL2]
    out = (rz[:, _ROW0] * first[:, _COL0] + rz[:, _ROW1] * first[:, _COL1]) + rz[:, _ROW2] * first[:, _COL2]
    return np.ascontiguousarray(out)


@dataclass(frozen=True)
class RotationGridIndex:
    """Reusable CPU spatial index over target-sphere triangles (reference 26-179)."""

    points: np.ndarray
    faces: np.ndarray
    candidate_table: np.ndarray | None
    grid_size: int
    margin: int
    candidate_offsets: np.ndarray | None = None
    candidate_faces: np.ndarray | None = None

    @classmethod
    def from_stencil(cls, stencil, *, grid_size: int = 128, margin: int = 1,
                     include_dense_candidate_table: bool = True) -> "RotationGridIndex":
        return cls.from_geometry(stencil.sphere_points, stencil.faces, grid_size=grid_size, margin=margin,
                                 include_dense_candidate_table=include_dense_candidate_table)

    @classmethod
    def from_geometry(cls, points, faces, *, grid_size: int = 128, margin: int = 1,
                      include_dense_candidate_table: bool = True) -> "RotationGridIndex":
        points = np.ascontiguousarray(points, dtype=np.float64)
        faces = np.ascontiguousarray(faces, dtype=np.int32)
        if points.ndim != 2 or points.shape[1] != 3:
            raise ValueError("points must have shape [n, 3]")
        if faces.ndim != 2 or faces.shape[1] != 3:
            raise ValueError("faces must have shape [m, 3]")
        if grid_size < 4 or margin < 0:
            raise ValueError("grid_size must be at least 4 and margin must be non-negative")
        lib = _native.library()
        offsets = np.zeros(grid_size ** 3 + 1, dtype=np.int32)
        count = ctypes.c_longlong(0)
        _native.check(
            lib.csg_rotation_grid_build(points.ctypes.data, points.shape[0], faces.ctypes.data, faces.shape[0],
                                        grid_size, margin, offsets.ctypes.data, None, 0, ctypes.addressof(count)),
            "csg_rotation_grid_build",
        )
        flat = np.zeros(max(1, count.value), dtype=np.int32)
        _native.check(
            lib.csg_rotation_grid_build(points.ctypes.data, points.shape[0], faces.ctypes.data, faces.shape[0],
                                        grid_size, margin, offsets.ctypes.data, flat.ctypes.data, flat.size,
                                        ctypes.addressof(count)),
            "csg_rotation_grid_build",
        )
        flat = flat[: count.value]
        if count.value == 0:
            raise ValueError("At least one triangle does not cover any spatial grid cell")
        table = None
        if include_dense_candidate_table:
            widths = np.diff(offsets)
            table = np.full((grid_size ** 3, int(widths.max())), -1, dtype=np.int32)
            rows = np.repeat(np.arange(grid_size ** 3), widths)
            cols = np.arange(flat.size) - np.repeat(offsets[:-1], widths)
            table[rows, cols] = flat
        return cls(points=points, faces=faces, candidate_table=table, grid_size=int(grid_size), margin=int(margin),
                   candidate_offsets=offsets, candidate_faces=flat)

    @property
    def max_candidates(self) -> int:
        if self.candidate_offsets is not None:
            return int(np.diff(self.candidate_offsets).max())
        return 0 if self.candidate_table is None else int(self.candidate_table.shape[1])

    def to(self, device, *, geometry_dtype: torch.dtype = torch.float32, candidate_table_dtype: torch.dtype = torch.int32,
           compressed_candidate_table: bool = True) -> "RotationGridIndexDevice":
        """Upload the index (CSR always; candidate_table_dtype is accepted for compatibility)."""

        target = resolve_device(device)
        if geometry_dtype != torch.float32:
            raise ValueError("the native rotation cost evaluates geometry in float32")
        if self.candidate_offsets is None or self.candidate_faces is None:
            raise ValueError("RotationGridIndex is missing candidate index")
        triangles = self.points[self.faces.astype(np.int64)].astype(np.float32)
        return RotationGridIndexDevice(
            target_points=torch.from_numpy(np.array(self.points, dtype=np.float32)).to(target),
            target_faces=torch.from_numpy(np.array(self.faces, dtype=np.int32)).to(target),
            target_triangles=torch.as_tensor(triangles, device=target).contiguous(),
            candidate_table=torch.empty(0, dtype=candidate_table_dtype, device=target),
            grid_size=self.grid_size,
            candidate_offsets=torch.as_tensor(self.candidate_offsets, device=target).contiguous(),
            candidate_faces=torch.as_tensor(self.candidate_faces, device=target).contiguous(),
        )


@dataclass(frozen=True)
class RotationCostInputs:
    """Validated device tensors reused by every rotation candidate."""

    source_points: torch.Tensor
    source_values: torch.Tensor
    target_values: torch.Tensor
    n_features: int = 1


@dataclass(frozen=True)
class RotationSearchResult:
    """Seed costs, refined angles, matrix, cost, and iteration count."""

    seed_angle: torch.Tensor
    seed_cost: torch.Tensor
    seed_costs: torch.Tensor
    angle: torch.Tensor
    cost: torch.Tensor
    rotation_matrix: torch.Tensor
    iterations: int


class _Costing:
    """Device buffers for repeated cost evaluations of one (index, inputs) pair."""

    def __init__(self, index: "RotationGridIndexDevice", inputs: RotationCostInputs, capacity: int, tile: int = 256):
        self.index, self.inputs, self.tile = index, inputs, tile
        self.capacity = max(1, int(capacity))
        dev = index.device
        self.matrices = torch.empty((self.capacity, 9), dtype=torch.float32, device=dev)
        self.costs = torch.empty(self.capacity, dtype=torch.float64, device=dev)
        n_src = (ctypes.c_int * 1)(int(inputs.source_points.shape[0]))
        n_cand = (ctypes.c_int * 1)(self.capacity)
        need = _native.library().csg_rotation_scratch_bytes(1, ctypes.addressof(n_src), ctypes.addressof(n_cand), tile)
        self.scratch = torch.empty(int(need), dtype=torch.uint8, device=dev)
        self.pinned = torch.empty(self.capacity, dtype=torch.float64, pin_memory=True)
        self.staging = torch.empty((self.capacity, 9), dtype=torch.float32, pin_memory=True)
        self.staging_host = self.staging.numpy()
        # the kernel's coverage status word, read back with the costs in one synchronisation
        offset = int(_native.library().csg_rotation_status_offset(1))
        self.status_device = self.scratch[offset:offset + 4].view(torch.int32)
        self.status_host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        # host-driven evaluations (csg_rotation_cost_host): one page-locked block for the
        # status and the costs, and the surface description built once
        self.readback = torch.zeros(8 + 8 * _native.CSG_ROTATION_HOST_MAX_CANDIDATES, dtype=torch.uint8,
                                    pin_memory=True)
        self.readback_host = self.readback.numpy()
        self.surface = _native.RotationSurface(
            inputs.source_points.data_ptr(), inputs.source_values.data_ptr(), index.target_triangles.data_ptr(),
            index.target_faces.data_ptr(), inputs.target_values.data_ptr(), index.candidate_offsets.data_ptr(),
            index.candidate_faces.data_ptr(), self.matrices.data_ptr(), int(inputs.source_points.shape[0]),
            int(index.grid_size), 1, int(inputs.n_features), int(index.target_points.shape[0]),
            index.target_records.data_ptr(),
        )

    def evaluate(self, angles: np.ndarray, *, host: bool = False):
        """Costs of these candidates: a device tensor, or (``host``) a NumPy copy read back in the
        same synchronisation as the coverage status."""

        mats = rotation_matrices_flat(angles)
        count = mats.shape[0]
        if count > self.capacity:
            raise ValueError("more candidates than this costing context holds")
        if host and count <= _native.CSG_ROTATION_HOST_MAX_CANDIDATES:
            # one native call: upload from the staging rows, the cost launches, one readback, synchronise
            np.copyto(self.staging_host[:count], mats)
            self.surface.n_candidates = count
            lib = _native.library()
            _native.check(
                lib.csg_rotation_cost_host(ctypes.addressof(self.surface), self.staging.data_ptr(),
                                           self.matrices.data_ptr(), self.readback.data_ptr(), self.tile,
                                           self.scratch.data_ptr(), self.scratch.numel(),
                                           _native.stream_handle(like=self.costs)),
                "csg_rotation_cost_host",
            )
            if int(self.readback_host[:4].view(np.int32)[0]) != 0:
                raise RuntimeError("Rotation is not covered by target sphere candidate index")
            return self.readback_host[8:8 + 8 * count].view(np.float64).copy()
        # page-locked staging: an asynchronous upload (the previous call's status read has
        # synchronised, so the staging rows are free)
        np.copyto(self.staging_host[:count], mats)
        self.matrices[:count].copy_(self.staging[:count], non_blocking=True)
        surface = _native.RotationSurface(
            self.inputs.source_points.data_ptr(), self.inputs.source_values.data_ptr(),
            self.index.target_triangles.data_ptr(), self.index.target_faces.data_ptr(),
            self.inputs.target_values.data_ptr(), self.index.candidate_offsets.data_ptr(),
            self.index.candidate_faces.data_ptr(), self.matrices.data_ptr(),
            int(self.inputs.source_points.shape[0]), int(self.index.grid_size), int(count),
            int(self.inputs.n_features), int(self.index.target_points.shape[0]),
            self.index.target_records.data_ptr(),
        )
        lib = _native.library()
        stream = _native.stream_handle(like=self.costs)
        _native.check(
            lib.csg_rotation_cost_batch(1, ctypes.addressof(surface), self.costs.data_ptr(), self.tile, 0,
                                        self.scratch.data_ptr(), self.scratch.numel(), stream),
            "csg_rotation_cost_batch",
        )
        if host:
            self.pinned[:count].copy_(self.costs[:count], non_blocking=True)
        self.status_host.copy_(self.status_device, non_blocking=True)
        torch.cuda.current_stream(self.costs.device).synchronize()
        if int(self.status_host[0]) != 0:
            raise RuntimeError("Rotation is not covered by target sphere candidate index")
        if host:
            return self.pinned[:count].numpy().copy()
        return self.costs[:count]


@dataclass
class RotationGridIndexDevice:
    """Evaluate CAT rotation candidates against a device-resident spatial index."""

    target_points: torch.Tensor
    target_faces: torch.Tensor
    target_triangles: torch.Tensor
    candidate_table: torch.Tensor
    grid_size: int
    candidate_offsets: torch.Tensor | None = None
    candidate_faces: torch.Tensor | None = None

    @property
    def device(self) -> torch.device:
        return self.target_points.device

    @property
    def target_records(self) -> torch.Tensor:
        """[n_tri, 20] float32 per-triangle terms of the closest-polygon test and a bounding sphere (built once, on the device)."""

        records = self.__dict__.get("_records")
        if records is None:
            tri = self.target_triangles.reshape(-1, 9).contiguous()
            records = torch.empty((tri.shape[0], 20), dtype=torch.float32, device=self.device)
            _native.check(_native.library().csg_rotation_triangle_records(
                tri.data_ptr(), int(tri.shape[0]), records.data_ptr(), _native.stream_handle(like=records)),
                "csg_rotation_triangle_records")
            self.__dict__["_records"] = records
        return records

    @classmethod
    def build(cls, points, faces, *, device, grid_size: int = 128, margin: int = 1) -> "RotationGridIndexDevice":
        """Build the candidate grid directly on a CUDA device (``csg_rotation_grid_build_device``).

        Same CSR (cells, face order) as ``RotationGridIndex.from_geometry(...).to(device)``.
        """

        target = resolve_device(device)
        pts = np.ascontiguousarray(points, dtype=np.float64)
        tri = np.ascontiguousarray(faces, dtype=np.int32)
        if pts.ndim != 2 or pts.shape[1] != 3 or tri.ndim != 2 or tri.shape[1] != 3:
            raise ValueError("points and faces must have shape [n, 3] and [m, 3]")
        if grid_size < 4 or margin < 0:
            raise ValueError("grid_size must be at least 4 and margin must be non-negative")
        if tri.min(initial=0) < 0 or tri.max(initial=0) >= pts.shape[0]:
            raise ValueError("faces reference a missing point")
        from .features import _device_faces

        lib = _native.library()
        # torch.from_numpy refuses to wrap a read-only array without a warning; the upload
        # only reads it, but a caller's read-only view (np.load mmap, a frozen golden) gets a copy
        d_pts = torch.from_numpy(pts if pts.flags.writeable else pts.copy()).to(target)
        d_faces = _device_faces(tri, target)
        offsets = torch.empty(grid_size ** 3 + 1, dtype=torch.int32, device=target)
        scratch = torch.empty(int(lib.csg_rotation_grid_scratch_bytes(grid_size)), dtype=torch.uint8, device=target)
        count = ctypes.c_longlong(0)
        stream = _native.stream_handle(like=scratch)
        args = (d_pts.data_ptr(), pts.shape[0], d_faces.data_ptr(), tri.shape[0], grid_size, margin,
                offsets.data_ptr())
        _native.check(lib.csg_rotation_grid_build_device(*args, None, 0, ctypes.addressof(count), scratch.data_ptr(),
                                                         scratch.numel(), stream), "csg_rotation_grid_build_device")
        if count.value == 0:
            raise ValueError("At least one triangle does not cover any spatial grid cell")
        flat = torch.empty(count.value, dtype=torch.int32, device=target)
        _native.check(lib.csg_rotation_grid_build_device(*args, flat.data_ptr(), count.value, ctypes.addressof(count),
                                                         scratch.data_ptr(), scratch.numel(), stream),
                      "csg_rotation_grid_build_device")
        # corner gather and float64 -> float32 rounding on the device (the same values as on the host)
        triangles = d_pts[d_faces.long()].to(torch.float32).contiguous()
        return cls(target_points=d_pts.to(torch.float32).contiguous(), target_faces=d_faces,
                   target_triangles=triangles,
                   candidate_table=torch.empty(0, dtype=torch.int32, device=target), grid_size=int(grid_size),
                   candidate_offsets=offsets, candidate_faces=flat)

    def _rotation_matrices(self, angles) -> torch.Tensor:
        a = torch.as_tensor(angles, dtype=torch.float64).detach().cpu().numpy()
        if a.ndim == 1:
            a = a.reshape(1, 3)
        if a.ndim != 2 or a.shape[1] != 3:
            raise ValueError("angles must have shape [candidates, 3]")
        return torch.as_tensor(rotation_matrices_flat(a), device=self.device).reshape(-1, 3, 3)

    def rotation_matrix(self, angles) -> torch.Tensor:
        matrices = self._rotation_matrices(angles)
        if matrices.shape[0] != 1:
            raise ValueError("rotation_matrix accepts exactly one angle vector")
        return matrices[0]

    def rotate_points(self, source_points, angles) -> torch.Tensor:
        """[C, n, 3]: p'_j = (p0 m[3j] + p1 m[3j+1]) + p2 m[3j+2] (reference 294-313)."""

        source = torch.as_tensor(source_points, dtype=torch.float32, device=self.device).contiguous()
        if source.ndim != 2 or source.shape[1] != 3:
            raise ValueError("source_points must have shape [n, 3]")
        m = self._rotation_matrices(angles).reshape(-1, 9)
        p = source.unsqueeze(0)
        cols = [(p[..., 0] * m[:, 3 * j, None] + p[..., 1] * m[:, 3 * j + 1, None]) + p[..., 2] * m[:, 3 * j + 2, None]
                for j in range(3)]
        return torch.stack(cols, dim=-1)

    def prepare_cost_inputs(self, source_points, source_values, target_values) -> RotationCostInputs:
        """Upload points and features once.  Values are [n] (one feature, the
        reference's form) or [F, n] (F features; the cost sums all F SSDs)."""

        source = torch.as_tensor(source_points, dtype=torch.float32, device=self.device).contiguous()
        sv = torch.as_tensor(source_values, dtype=torch.float64, device=self.device)
        tv = torch.as_tensor(target_values, dtype=torch.float64, device=self.device)
        if source.ndim != 2 or source.shape[1] != 3:
            raise ValueError("source_points must have shape [n, 3]")
        features = int(sv.shape[0]) if sv.ndim == 2 else 1
        if sv.ndim > 2 or tv.ndim > 2 or (tv.shape[0] if tv.ndim == 2 else 1) != features:
            raise ValueError("source_values and target_values must both be [n] or both [F, n] with the same F")
        sv = sv.reshape(-1).contiguous()
        tv = tv.reshape(-1).contiguous()
        if sv.numel() != features * source.shape[0]:
            raise ValueError("source_values length does not match source_points")
        if tv.numel() != features * self.target_points.shape[0]:
            raise ValueError("target_values length does not match the target sphere")
        return RotationCostInputs(source_points=source, source_values=sv, target_values=tv, n_features=features)

    def _costing(self, inputs: RotationCostInputs, capacity: int) -> _Costing:
        cache = self.__dict__.setdefault("_costing_cache", {})
        key = (id(inputs), capacity)
        if key not in cache:
            cache.clear()
            cache[key] = _Costing(self, inputs, capacity)
        return cache[key]

    def cost_batch_prepared(self, inputs: RotationCostInputs, angles, *, point_chunk: int = 1024) -> torch.Tensor:
        """float64 SSD per candidate rotation [C] (reference 512-546)."""

        if point_chunk < 1:
            raise ValueError("point_chunk must be positive")
        if inputs.source_points.device != self.device:
            raise ValueError("RotationCostInputs and the index must be on the same device")
        a = torch.as_tensor(angles, dtype=torch.float64).detach().cpu().numpy()
        if a.ndim == 1:
            a = a.reshape(1, 3)
        if a.ndim != 2 or a.shape[1] != 3:
            raise ValueError("angles must have shape [candidates, 3]")
        costing = self._costing(inputs, max(64, a.shape[0]))
        return costing.evaluate(a).clone()

    def cost_batch(self, source_points, source_values, target_values, angles, *, point_chunk: int = 1024):
        inputs = self.prepare_cost_inputs(source_points, source_values, target_values)
        return self.cost_batch_prepared(inputs, angles, point_chunk=point_chunk)

    def coarse_seed_search_prepared(self, inputs: RotationCostInputs, *, point_chunk: int = 1024):
        angles = torch.as_tensor(official_seed_grid_angles(), dtype=torch.float64, device=self.device)
        costs = self.cost_batch_prepared(inputs, angles, point_chunk=point_chunk)
        best = torch.argmin(costs)
        return angles[best], costs[best], costs

    def coarse_seed_search(self, source_points, source_values, target_values, *, point_chunk: int = 1024):
        inputs = self.prepare_cost_inputs(source_points, source_values, target_values)
        return self.coarse_seed_search_prepared(inputs, point_chunk=point_chunk)

    def refine_nelder_mead_prepared(self, inputs: RotationCostInputs, initial_angles, *, point_chunk: int = 1024,
                                    max_iter: int = 500, tol: float = 1.0e-4, simplex_step: float = 0.1):
        """CAT-ordered Nelder-Mead with device-evaluated costs (reference 594-699)."""

        if max_iter < 1 or tol < 0.0 or simplex_step <= 0.0:
            raise ValueError("max_iter, tol, and simplex_step must be positive")
        seed = torch.as_tensor(initial_angles, dtype=torch.float64).detach().cpu().numpy().reshape(-1)
        if seed.size != 3:
            raise ValueError("initial_angles must contain exactly three angles")
        costing = self._costing(inputs, 64)

        def cost(points: np.ndarray) -> np.ndarray:
            return costing.evaluate(points, host=True)

        simplex = np.stack((seed, seed + (simplex_step, 0.0, 0.0), seed + (0.0, simplex_step, 0.0),
                            seed + (0.0, 0.0, simplex_step)))
        f = cost(simplex).astype(np.float64)
        iteration = 0
        for iteration in range(max_iter):
            highest, lowest, second = 0, 0, 1
            for index in range(4):
                if f[index] > f[highest]:
                    second, highest = highest, index
                elif f[index] > f[second] and index != highest:
                    second = index
                if f[index] < f[lowest]:
                    lowest = index
            centroid = np.zeros(3)
            for index in range(4):
                if index != highest:
                    centroid += simplex[index]
            centroid /= 3.0
            reflected = centroid + (centroid - simplex[highest])
            expanded = centroid + 2.0 * (reflected - centroid)
            contracted = centroid + 0.5 * (simplex[highest] - centroid)
            # The three trial points depend only on the simplex, and each cost is
            # computed on its own (fixed summation order), so one launch evaluates
            # all three; the branch below uses exactly the costs the reference's
            # one-at-a-time evaluation would, and the same decisions follow.
            fr, fe, fc = cost(np.stack((reflected, expanded, contracted)))
            if fr < f[lowest]:
                if fe < fr:
                    simplex[highest], f[highest] = expanded, fe
                else:
                    simplex[highest], f[highest] = reflected, fr
            elif fr < f[second]:
                simplex[highest], f[highest] = reflected, fr
            else:
                if fc < f[highest]:
                    simplex[highest], f[highest] = contracted, fc
                else:
                    shrunk = [simplex[lowest] + 0.5 * (simplex[index] - simplex[lowest]) for index in range(4)]
                    targets = [index for index in range(4) if index != lowest]
                    values = cost(np.stack([shrunk[index] for index in targets]))
                    for index, value in zip(targets, values):
                        simplex[index], f[index] = shrunk[index], value
            if np.max(np.abs(f - f[lowest])) < tol:
                break
        dev = self.device
        return (torch.as_tensor(simplex[lowest].copy(), device=dev), torch.as_tensor(float(f[lowest]), dtype=torch.float64, device=dev),
                iteration + 1)

    def refine_nelder_mead(self, source_points, source_values, target_values, initial_angles, *,
                           point_chunk: int = 1024, max_iter: int = 500, tol: float = 1.0e-4,
                           simplex_step: float = 0.1):
        inputs = self.prepare_cost_inputs(source_points, source_values, target_values)
        return self.refine_nelder_mead_prepared(inputs, initial_angles, point_chunk=point_chunk, max_iter=max_iter,
                                                tol=tol, simplex_step=simplex_step)

    def euler_grid_search_prepared(self, inputs: RotationCostInputs, *, coarse_step_deg: float = 10.0,
                                   fine_step_deg: float = 2.0, fine_half_width_deg: float = 10.0):
        """Two-level Euler-grid search: all of SO(3) every ``coarse_step_deg``, then
        every ``fine_step_deg`` within +-``fine_half_width_deg`` of the coarse best.

        The rotation search of the 10-degree-then-2-degree configuration
        (an alternative to the reference's 46 seeds + Nelder-Mead); each
        level is one batched cost launch; first minimum in grid order.
        """

        coarse = torch.as_tensor(euler_grid_angles(coarse_step_deg), dtype=torch.float64)
        coarse_costs = self.cost_batch_prepared(inputs, coarse)
        best = int(torch.argmin(coarse_costs))
        fine = torch.as_tensor(euler_grid_angles(fine_step_deg, coarse[best].numpy(), fine_half_width_deg),
                               dtype=torch.float64)
        fine_costs = self.cost_batch_prepared(inputs, fine)
        pick = int(torch.argmin(fine_costs))
        angle = fine[pick].to(self.device)
        return RotationSearchResult(seed_angle=coarse[best].to(self.device), seed_cost=coarse_costs[best].clone(),
                                    seed_costs=coarse_costs, angle=angle, cost=fine_costs[pick].clone(),
                                    rotation_matrix=self.rotation_matrix(angle), iterations=0)

    def search_rotation(self, source_points, source_values, target_values, *, point_chunk: int = 1024,
                        refine: bool = True, max_iter: int = 500, tol: float = 1.0e-4, simplex_step: float = 0.1):
        inputs = self.prepare_cost_inputs(source_points, source_values, target_values)
        return self.search_rotation_prepared(inputs, point_chunk=point_chunk, refine=refine, max_iter=max_iter,
                                             tol=tol, simplex_step=simplex_step)

    def search_rotation_prepared(self, inputs: RotationCostInputs, *, point_chunk: int = 1024, refine: bool = True,
                                 max_iter: int = 500, tol: float = 1.0e-4, simplex_step: float = 0.1):
        """46 seeds, then optional refinement (reference 749-785)."""

        seed_angle, seed_cost, seed_costs = self.coarse_seed_search_prepared(inputs, point_chunk=point_chunk)
        if refine:
            angle, cost, iterations = self.refine_nelder_mead_prepared(inputs, seed_angle, point_chunk=point_chunk,
                                                                       max_iter=max_iter, tol=tol,
                                                                       simplex_step=simplex_step)
        else:
            angle, cost, iterations = seed_angle.clone(), seed_cost.clone(), 0
        return RotationSearchResult(seed_angle=seed_angle.clone(), seed_cost=seed_cost.clone(), seed_costs=seed_costs,
                                    angle=angle, cost=cost, rotation_matrix=self.rotation_matrix(angle),
                                    iterations=iterations)


def quaternion_matrices(quaternions) -> np.ndarray:
    """[C, 9] float32 rotation matrices (row-major R, q_rotated = R p) of unit quaternions (w, x, y, z)."""

    q = np.asarray(quaternions, dtype=np.float64).reshape(-1, 4)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    r = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                  2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                  2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], axis=1)
    return np.ascontiguousarray(r, dtype=np.float32)


def uniform_quaternions(count: int, seed: int) -> np.ndarray:
    """Seeded uniform random unit quaternions (Shoemake's subgroup algorithm), [count, 4] as (w, x, y, z)."""

    rng = np.random.default_rng(seed)
    u1, u2, u3 = rng.random((3, int(count)))
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    return np.stack([b * np.cos(2 * np.pi * u3), a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                     b * np.sin(2 * np.pi * u3)], axis=1)


def batched_costs(indices, inputs, angle_sets=None, *, matrix_sets=None, tile: int = 256,
                  n_ctas: int = 0) -> list[torch.Tensor]:
    """Costs of many candidate sets on many surfaces in ONE persistent launch.

    ``indices[i]`` (a RotationGridIndexDevice), ``inputs[i]`` (its
    RotationCostInputs) and ``angle_sets[i]`` ([C_i, 3] Euler angles) or
    ``matrix_sets[i]`` ([C_i, 9] float32 matrices, e.g. from
    :func:`quaternion_matrices`) describe surface i; surfaces may differ in
    size, feature count and candidate count.  Returns one float64 cost tensor
    per surface, identical to
    ``indices[i].cost_batch_prepared(inputs[i], angle_sets[i])``.
    ``tile`` (128/256/512 source points per work item) is the launch shape
    chosen by :mod:`cat_surface_gpu_b200.autotune`.
    """

    n = len(indices)
    sets = angle_sets if matrix_sets is None else matrix_sets
    if (angle_sets is None) == (matrix_sets is None):
        raise ValueError("give exactly one of angle_sets and matrix_sets")
    if n == 0 or len(inputs) != n or len(sets) != n:
        raise ValueError("indices, inputs and candidate sets must be non-empty and of equal length")
    dev = indices[0].device
    if matrix_sets is None:
        mats = [torch.as_tensor(rotation_matrices_flat(np.asarray(a)), device=dev) for a in angle_sets]
    else:
        mats = [torch.as_tensor(np.asarray(m, dtype=np.float32).reshape(-1, 9), device=dev).contiguous()
                for m in matrix_sets]
    counts = [int(m.shape[0]) for m in mats]
    costs = torch.empty(sum(counts), dtype=torch.float64, device=dev)
    surfaces = (_native.RotationSurface * n)()
    for i, (index, inp, m) in enumerate(zip(indices, inputs, mats)):
        surfaces[i] = _native.RotationSurface(
            inp.source_points.data_ptr(), inp.source_values.data_ptr(), index.target_triangles.data_ptr(),
            index.target_faces.data_ptr(), inp.target_values.data_ptr(), index.candidate_offsets.data_ptr(),
            index.candidate_faces.data_ptr(), m.data_ptr(), int(inp.source_points.shape[0]), int(index.grid_size),
            counts[i], int(inp.n_features), int(index.target_points.shape[0]), index.target_records.data_ptr(),
        )
    n_src = (ctypes.c_int * n)(*[int(inp.source_points.shape[0]) for inp in inputs])
    n_cand = (ctypes.c_int * n)(*counts)
    lib = _native.library()
    need = lib.csg_rotation_scratch_bytes(n, ctypes.addressof(n_src), ctypes.addressof(n_cand), tile)
    scratch = torch.empty(int(need), dtype=torch.uint8, device=dev)
    stream = _native.stream_handle(like=scratch)
    _native.check(lib.csg_rotation_cost_batch(n, ctypes.addressof(surfaces), costs.data_ptr(), tile, n_ctas,
                                              scratch.data_ptr(), scratch.numel(), stream), "csg_rotation_cost_batch")
    status = ctypes.c_int(0)
    _native.check(lib.csg_rotation_status(scratch.data_ptr(), n, stream, ctypes.addressof(status)), "csg_rotation_status")
    if status.value != 0:
        raise RuntimeError("Rotation is not covered by target sphere candidate index")
    return list(torch.split(costs, counts))
