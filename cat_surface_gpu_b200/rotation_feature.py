"""Depth-potential rotation features on the GPU (reference ``src/cat_surface_gpu/rotation_feature.py``).

Same API as the reference module: :class:`RotationFeatureResult`,
:func:`compute_rotation_feature` and :func:`compute_rotation_features`
(reference 320-458).  The solve (stable normals, mixed Voronoi areas, the
cotangent system, coloured SOR or Jacobi-preconditioned CG, reference
37-317) is ``csg_depth_potential``; the smoothing of the potential (FWHM 50)
and the min-max normalisation are the stencil feature kernels.  Surfaces
that share one triangulation are solved in one batched launch.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from . import _native

_TOPOLOGIES: dict[tuple, "DepthTopology"] = {}


@dataclass(frozen=True)
class RotationFeatureResult:
    """Normalised rotation feature and solver diagnostics (reference 15-21)."""

    values: torch.Tensor
    iterations: int
    relative_residual: float


def colour_groups(faces: np.ndarray, n_points: int) -> tuple[np.ndarray, ...]:
    """Greedy first-fit colouring in vertex order (reference ``surface_stencil.py:69-91``)."""

    tri = np.ascontiguousarray(faces, dtype=np.int32)
    n = int(n_points)
    lib = _native.library()
    off = np.zeros(n + 1, dtype=np.int32)
    nbr = np.zeros(max(1, 6 * tri.shape[0]), dtype=np.int32)
    count = _native.check(lib.csg_mesh_neighbours(n, _native.ptr(tri), tri.shape[0], _native.ptr(off),
                                                  _native.ptr(nbr), nbr.size), "csg_mesh_neighbours")
    nbr = np.ascontiguousarray(nbr[: max(1, count)])
    colour_off = np.zeros(n + 1, dtype=np.int32)
    members = np.zeros(n, dtype=np.int32)
    k = _native.check(lib.csg_colour_groups(n, _native.ptr(off), _native.ptr(nbr), _native.ptr(colour_off),
                                            _native.ptr(members)), "csg_colour_groups")
    return tuple(members[colour_off[c]: colour_off[c + 1]].astype(np.int64) for c in range(k))


@dataclass
class DepthTopology:
    """Device tables of one triangulation: incidences, colours and the SOR sweep schedule."""

    n: int
    nf: int
    faces: torch.Tensor
    inc_off: torch.Tensor
    inc: torch.Tensor
    max_incidences: int
    groups: tuple[np.ndarray, ...]
    order: torch.Tensor
    level_begin: torch.Tensor
    level_end: torch.Tensor
    n_levels: int
    level_stride: int

    @classmethod
    def build(cls, faces: np.ndarray, n_points: int, device: torch.device) -> "DepthTopology":
        from .features import _topology
        from .surf2sphere import SweepPlan

        tri = np.ascontiguousarray(faces, dtype=np.int32)
        n = int(n_points)
        key = (device.type, device.index, n, tri.shape, tri.tobytes())
        cached = _TOPOLOGIES.get(key)
        if cached is not None:
            return cached
        _, _, inc_off, inc, _ = _topology(tri, n, device)
        groups = colour_groups(tri, n)
        # One coloured SOR sweep is one Gauss-Seidel pass in colour-major order:
        # the wavefront schedule of the relabelled mesh, mapped back to vertex ids.
        perm = np.concatenate(groups).astype(np.int32)
        relabel = np.empty(n, dtype=np.int32)
        relabel[perm] = np.arange(n, dtype=np.int32)
        plan = SweepPlan.build(relabel[tri], n)
        order = perm[plan.order]
        topo = cls(
            n=n, nf=int(tri.shape[0]), faces=torch.from_numpy(np.array(tri)).to(device), inc_off=inc_off, inc=inc,
            max_incidences=int(np.bincount(tri.reshape(-1), minlength=n).max()), groups=groups,
            order=torch.from_numpy(np.ascontiguousarray(order)).to(device),
            level_begin=torch.from_numpy(plan.level_begin).to(device),
            level_end=torch.from_numpy(plan.level_end).to(device),
            n_levels=int(plan.n_levels), level_stride=int(plan.level_stride))
        _TOPOLOGIES[key] = topo
        return topo


def depth_potential(geometries: torch.Tensor, topology: DepthTopology, *, solver: str = "colored-sor",
                    alpha: float = 1.0 / 1000.0, max_iter: int = 1000, tolerance: float = 1.0e-9,
                    relaxation: float = 1.90, with_geometry: bool = False, launch: dict | None = None,
                    timeout_s: float = 2.0):
    """Raw depth potential of ``geometries`` [B, n, 3] (float32, one triangulation).

    Returns ``(values [B, n] float64, iterations [B], residuals [B])`` and,
    with ``with_geometry``, also ``(normals [B, n, 3], areas [B, n])``.
    """

    if solver not in {"colored-sor", "pcg"}:
        raise ValueError("rotation feature solver must be 'colored-sor' or 'pcg'")
    g = torch.as_tensor(geometries).to(torch.float32).contiguous()
    if g.ndim == 2:
        g = g.unsqueeze(0)
    if g.ndim != 3 or tuple(g.shape[1:]) != (topology.n, 3):
        raise ValueError(f"geometries must have shape [batch, {topology.n}, 3], got {tuple(g.shape)}")
    if g.device.type != "cuda":
        raise ValueError("depth_potential runs on a CUDA device")
    batch = int(g.shape[0])
    lib = _native.library()
    device = g.device
    values = torch.empty((batch, topology.n), dtype=torch.float64, device=device)
    iterations = torch.zeros(batch, dtype=torch.int32, device=device)
    residual = torch.zeros(batch, dtype=torch.float64, device=device)
    normals = torch.empty((batch, topology.n, 3), dtype=torch.float64, device=device) if with_geometry else None
    areas = torch.empty((batch, topology.n), dtype=torch.float64, device=device) if with_geometry else None
    scratch = torch.empty(int(lib.csg_depth_scratch_bytes(topology.n, topology.nf, batch)), dtype=torch.uint8,
                          device=device)
    # measured on the 40,962-point stencil sphere, two sides, 1,000 sweeps: 4 lanes x 512 threads 18.4 ms,
    # 8 lanes 19.0 ms, 16 lanes 32.0 ms
    cfg = {"n_ctas": 0, "threads_per_cta": 512, "lanes_per_row": 4}
    if launch:
        cfg.update(launch)
    code = _native.CSG_DEPTH_SOR if solver == "colored-sor" else _native.CSG_DEPTH_PCG
    _native.check(lib.csg_depth_potential(
        _native.ptr(g), batch, topology.n, _native.ptr(topology.faces), topology.nf, _native.ptr(topology.inc_off),
        _native.ptr(topology.inc), topology.max_incidences, float(alpha), code, int(max_iter), float(tolerance),
        float(relaxation), _native.ptr(topology.order), _native.ptr(topology.level_begin),
        _native.ptr(topology.level_end), topology.n_levels, topology.level_stride, _native.ptr(values),
        _native.ptr(iterations), _native.ptr(residual), _native.ptr(normals) if normals is not None else None,
        _native.ptr(areas) if areas is not None else None, _native.ptr(scratch), scratch.numel(),
        int(cfg["n_ctas"]), int(cfg["threads_per_cta"]), int(cfg["lanes_per_row"]), float(timeout_s),
        _native.stream_handle(like=scratch)), "csg_depth_potential")
    status = int(scratch[:8].cpu().view(torch.int32)[1])
    if status != 0:
        raise RuntimeError(f"depth potential kernel failed (status {status})")
    its = [int(v) for v in iterations.cpu().tolist()]
    res = [float(v) for v in residual.cpu().tolist()]
    if with_geometry:
        return values, its, res, normals, areas
    return values, its, res


_TOPOLOGY_BY_FACES: dict[tuple, tuple] = {}


def _stencil_topology(stencil) -> DepthTopology:
    cached = stencil._cache.get("depth_topology")
    if cached is None:
        # stencils of one resampling sphere share one device face tensor: look it up by identity
        # before copying the faces back to hash them
        ident = (id(stencil.faces), int(stencil.sphere_points.shape[0]))
        hit = _TOPOLOGY_BY_FACES.get(ident)
        if hit is not None and hit[0] is stencil.faces:
            cached = hit[1]
        else:
            faces = stencil.faces.detach().cpu().numpy()
            cached = DepthTopology.build(faces, int(stencil.sphere_points.shape[0]), stencil.faces.device)
            _TOPOLOGY_BY_FACES[ident] = (stencil.faces, cached)
        stencil._cache["depth_topology"] = cached
    return cached


def _smoothed_surface(stencil, surface_vertices, heat_fwhm, smoothed_surface):
    if smoothed_surface is None:
        return stencil.smooth_geometry(stencil.resample_vertices(surface_vertices), heat_fwhm)
    smoothed = torch.as_tensor(smoothed_surface, dtype=torch.float32, device=stencil.faces.device).contiguous()
    expected = (int(stencil.sphere_points.shape[0]), 3)
    if tuple(smoothed.shape) != expected:
        raise ValueError(f"Upstream coarse-feature geometry must have shape [points, 3]{expected}, "
                         f"{tuple(smoothed.shape)}")
    return smoothed


def _finish(stencil, values, smoothed, iterations, residual, edge_mean: float | None = None) -> RotationFeatureResult:
    from .features import _minmax, _smooth_series

    # stencil.smooth_values(values, smoothed, 50.0); edge_mean (of `smoothed`) saves its synchronisation
    smoothed_values = _smooth_series(stencil, values, smoothed, (50.0,), True, edge_mean)[0]
    return RotationFeatureResult(values=_minmax(stencil, smoothed_values).contiguous(), iterations=int(iterations),
                                 relative_residual=float(residual))


def _given_depth(stencil, depth_values) -> torch.Tensor:
    values = torch.as_tensor(depth_values, dtype=torch.float64, device=stencil.faces.device).reshape(-1).contiguous()
    if values.numel() != stencil.sphere_points.shape[0]:
        raise ValueError("Upstream depth-potential length must match the coarse sphere")
    return values


def compute_rotation_feature(stencil, surface_vertices, *, heat_fwhm: float, smoothed_surface=None,
                             depth_values=None, depth_alpha: float = 1.0 / 1000.0, max_iter: int = 1000,
                             tolerance: float = 1.0e-9, solver: str = "colored-sor") -> RotationFeatureResult:
    """One CAT-compatible smoothed depth-potential feature (reference 320-401)."""

    if solver not in {"colored-sor", "pcg"}:
        raise ValueError("rotation feature solver must be 'colored-sor' or 'pcg'")
    smoothed = _smoothed_surface(stencil, surface_vertices, heat_fwhm, smoothed_surface)
    if depth_values is not None:
        return _finish(stencil, _given_depth(stencil, depth_values), smoothed, 0, 0.0)
    values, its, res = depth_potential(smoothed, _stencil_topology(stencil), solver=solver, alpha=depth_alpha,
                                       max_iter=max_iter, tolerance=tolerance)
    return _finish(stencil, values[0], smoothed, its[0], res[0])


def compute_rotation_features(stencils: Sequence, surfaces: Sequence, *, heat_fwhms: Sequence[float] = (15.0, 10.0),
                              smoothed_surfaces: Sequence | None = None, depth_values: Sequence | None = None,
                              depth_alpha: float = 1.0 / 1000.0, max_iter: int = 1000, tolerance: float = 1.0e-9,
                              solver: str = "colored-sor",
                              parallel_sides: bool = True) -> tuple[RotationFeatureResult, ...]:
    """Source and target features (reference 404-458); sides of one triangulation share one solve launch.

    ``parallel_sides`` is accepted for compatibility: batching replaces the
    reference's one CUDA stream per side.
    """

    if len(stencils) != len(surfaces) or len(stencils) != len(heat_fwhms):
        raise ValueError("stencils, surfaces, and heat_fwhms must have equal lengths")
    if smoothed_surfaces is not None and len(smoothed_surfaces) != len(stencils):
        raise ValueError("smoothed_surfaces length must match stencils")
    if depth_values is not None and len(depth_values) != len(stencils):
        raise ValueError("depth_values length must match stencils")
    if solver not in {"colored-sor", "pcg"}:
        raise ValueError("rotation feature solver must be 'colored-sor' or 'pcg'")
    from .features import edge_means, smooth_geometry

    given = [None if smoothed_surfaces is None else smoothed_surfaces[i] for i in range(len(stencils))]
    smoothed = [None if g is None else _smoothed_surface(st, None, 0.0, g) for st, g in zip(stencils, given)]
    todo = [i for i, g in enumerate(given) if g is None]
    if todo:
        # stencil.smooth_geometry(stencil.resample_vertices(surface), fwhm) per side, with the
        # sides' mean edge lengths read back together
        mapped = {i: stencils[i].resample_vertices(surfaces[i]).to(torch.float32).contiguous() for i in todo}
        means = edge_means([(stencils[i], mapped[i]) for i in todo])
        for i, mean in zip(todo, means):
            smoothed[i] = smooth_geometry(stencils[i], mapped[i], float(heat_fwhms[i]), mean)
    finish_means = edge_means([(st, sm) for st, sm in zip(stencils, smoothed)])
    if depth_values is not None:
        return tuple(_finish(st, _given_depth(st, dv), sm, 0, 0.0, mean)
                     for st, dv, sm, mean in zip(stencils, depth_values, smoothed, finish_means))
    # group the sides by triangulation; each group is one batched solve
    topologies = [_stencil_topology(st) for st in stencils]
    results: list[RotationFeatureResult | None] = [None] * len(stencils)
    pending = list(range(len(stencils)))
    while pending:
        topo = topologies[pending[0]]
        group = [i for i in pending if topologies[i] is topo]
        pending = [i for i in pending if topologies[i] is not topo]
        values, its, res = depth_potential(torch.stack([smoothed[i] for i in group]), topo, solver=solver,
                                           alpha=depth_alpha, max_iter=max_iter, tolerance=tolerance)
        for k, i in enumerate(group):
            results[i] = _finish(stencils[i], values[k], smoothed[i], its[k], res[k], finish_means[i])
    return tuple(r for r in results if r is not None)
