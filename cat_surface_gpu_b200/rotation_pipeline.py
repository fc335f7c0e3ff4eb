"""Initial-rotation pipeline over prepared inputs (drop-in for the reference's rotation_pipeline).

Follows ``src/cat_surface_gpu/rotation_pipeline.py``: the binary readers for
rotation points / values and ``RotationPipeline`` (build + upload the grid
index once, then seed search and Nelder-Mead on the device).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

from .device import resolve_device
from .surface_rotation import RotationCostInputs, RotationGridIndex, RotationGridIndexDevice, RotationSearchResult
from .surface_stencil import SurfaceStencil


def read_rotation_values(path) -> tuple[np.ndarray, np.ndarray]:
    """``[i32 ns, i32 nt, f64 source[ns], f64 target[nt]]`` (reference 23-40)."""

    path = Path(path)
    with path.open("rb") as stream:
        header = np.fromfile(stream, dtype="<i4", count=2)
        if header.size != 2:
            raise ValueError(f"Rotation feature file : {path}")
        source = np.fromfile(stream, dtype="<f8", count=int(header[0]))
        target = np.fromfile(stream, dtype="<f8", count=int(header[1]))
        trailing = stream.read(1)
    if source.size != int(header[0]) or target.size != int(header[1]):
        raise ValueError(f"Rotation feature file length : {path}")
    if trailing:
        raise ValueError(f"Rotation feature file : {path}")
    return np.ascontiguousarray(source), np.ascontiguousarray(target)


def read_rotation_points(path) -> np.ndarray:
    """``[i32 n, f32|f64 points[n][3]]`` (reference 43-67)."""

    path = Path(path)
    with path.open("rb") as stream:
        header = np.fromfile(stream, dtype="<i4", count=1)
        if header.size != 1:
            raise ValueError(f"Rotation file : {path}")
        n_points = int(header[0])
        if n_points < 0:
            raise ValueError(f"Rotation file : {path}")
        payload = stream.read()
    n_values = 3 * n_points
    if len(payload) == 4 * n_values:
        points = np.frombuffer(payload, dtype="<f4", count=n_values)
    elif len(payload) == 8 * n_values:
        points = np.frombuffer(payload, dtype="<f8", count=n_values)
    else:
        raise ValueError(f"Rotation file length : {path}, {len(payload)} ,{4 * n_values} or {8 * n_values}")
    return np.ascontiguousarray(points.reshape(n_points, 3))


class RotationPipeline:
    """A reusable target index plus CAT-compatible rotation search (reference 70-164).

    ``from_stencil`` builds the candidate grid on the GPU; ``index_cpu`` (the
    host copy the reference also keeps) is then built on first access.
    """

    def __init__(self, index_cpu: RotationGridIndex | None, index: RotationGridIndexDevice, geometry=None):
        self._index_cpu, self.index, self._geometry = index_cpu, index, geometry

    @property
    def index_cpu(self) -> RotationGridIndex:
        if self._index_cpu is None:
            points, faces, grid_size, margin = self._geometry
            self._index_cpu = RotationGridIndex.from_geometry(points, faces, grid_size=grid_size, margin=margin,
                                                              include_dense_candidate_table=False)
        return self._index_cpu

    @classmethod
    def from_stencil(cls, target_stencil: SurfaceStencil, *, device="auto", grid_size: int = 128, margin: int = 1,
                     candidate_table_dtype: torch.dtype = torch.int32, geometry_dtype: torch.dtype = torch.float32,
                     compressed_candidate_table: bool = True) -> "RotationPipeline":
        target = resolve_device(device)
        if geometry_dtype != torch.float32:
            raise ValueError("the native rotation cost evaluates geometry in float32")
        index = RotationGridIndexDevice.build(target_stencil.sphere_points, target_stencil.faces, device=target,
                                              grid_size=grid_size, margin=margin)
        return cls(None, index, (target_stencil.sphere_points, target_stencil.faces, grid_size, margin))

    @classmethod
    def from_index_cpu(cls, index_cpu: RotationGridIndex, *, device="auto",
                       candidate_table_dtype: torch.dtype = torch.int32,
                       geometry_dtype: torch.dtype = torch.float32) -> "RotationPipeline":
        index = index_cpu.to(resolve_device(device), geometry_dtype=geometry_dtype,
                             candidate_table_dtype=candidate_table_dtype)
        return cls(index_cpu=index_cpu, index=index)

    @property
    def device(self) -> torch.device:
        return self.index.device

    def prepare_inputs(self, source_points, source_values, target_values) -> RotationCostInputs:
        return self.index.prepare_cost_inputs(source_points, source_values, target_values)

    def search(self, source_points, source_values, target_values, *, point_chunk: int = 1024, refine: bool = True,
               max_iter: int = 500, tol: float = 1.0e-4, simplex_step: float = 0.1) -> RotationSearchResult:
        inputs = self.prepare_inputs(source_points, source_values, target_values)
        return self.index.search_rotation_prepared(inputs, point_chunk=point_chunk, refine=refine, max_iter=max_iter,
                                                   tol=tol, simplex_step=simplex_step)

    def search_euler_grid(self, source_points, source_values, target_values, *, coarse_step_deg: float = 10.0,
                          fine_step_deg: float = 2.0, fine_half_width_deg: float = 10.0) -> RotationSearchResult:
        """The 10-degree then 2-degree Euler-grid search (values [n] or [F, n])."""

        inputs = self.prepare_inputs(source_points, source_values, target_values)
        return self.index.euler_grid_search_prepared(inputs, coarse_step_deg=coarse_step_deg,
                                                     fine_step_deg=fine_step_deg,
                                                     fine_half_width_deg=fine_half_width_deg)


def run_rotation_pipeline(target_stencil, source_points, source_values, target_values, *, device="auto",
                          grid_size: int = 128, margin: int = 1, candidate_table_dtype=torch.int32,
                          geometry_dtype=torch.float32, point_chunk: int = 1024, refine: bool = True,
                          max_iter: int = 500, tol: float = 1.0e-4, simplex_step: float = 0.1) -> RotationSearchResult:
    pipeline = RotationPipeline.from_stencil(target_stencil, device=device, grid_size=grid_size, margin=margin,
                                             candidate_table_dtype=candidate_table_dtype, geometry_dtype=geometry_dtype)
    return pipeline.search(source_points, source_values, target_values, point_chunk=point_chunk, refine=refine,
                           max_iter=max_iter, tol=tol, simplex_step=simplex_step)


def run_rotation_pipeline_from_files(source_points_path, target_stencil_path, rotation_values_path, **kwargs):
    source_points = read_rotation_points(source_points_path)
    source_values, target_values = read_rotation_values(rotation_values_path)
    target_stencil = SurfaceStencil.from_file(target_stencil_path)
    return run_rotation_pipeline(target_stencil, source_points, source_values, target_values, **kwargs)
