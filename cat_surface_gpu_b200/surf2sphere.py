"""CAT_Surf2Sphere with the ordered area-smoothing sweeps on a B200.

Public names and signatures follow the reference module
``src/cat_surface_gpu/surf2sphere.py``:

* ``Surf2SphereTopology.from_mesh`` (reference 401-448) -- built by the native
  host builders (C++, O(faces)) instead of Python loops.
* ``run_areal_smoothing_cuda`` (reference 940-1104) -- all sweeps in ONE
  persistent cooperative CUDA launch (``csg_areal_sweeps``) instead of one
  Triton launch per dependency level per sweep.
* ``convert_ellipsoid_to_sphere_with_surface_area`` (reference 919-937) and
  ``surface_area`` (reference 461-471) -- host NumPy, same arithmetic.
* ``run_cat_surf2sphere_gpu`` (reference 1107-1295) -- stages 1-5, the
  sweeps and the ellipsoid-to-sphere steps, all on the GPU.
"""

from __future__ import annotations

from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
import math
from pathlib import Path
import time

import numpy as np
import torch

from . import _native
from .device import DeviceUnavailable, resolve_device
from .gifti import GiftiMesh, check_vertices, read_gifti_mesh, write_vertices_like


@dataclass(frozen=True)
class SweepPlan:
    """Host arrays of the wavefront schedule (see include/catsurf_b200.h)."""

    slot_off: np.ndarray
    slot_tri: np.ndarray
    order: np.ndarray
    level_begin: np.ndarray
    level_end: np.ndarray
    n_levels: int
    level_stride: int
    max_degree: int

    @classmethod
    def build(cls, faces: np.ndarray, n_points: int) -> "SweepPlan":
        tri = np.ascontiguousarray(faces, dtype=np.int32)
        if tri.ndim != 2 or tri.shape[1] != 3:
            raise ValueError(f"faces must have shape [m, 3], got {tri.shape}")
        n = int(n_points)
        slot_off = np.zeros(n + 1, dtype=np.int32)
        slot_tri = np.zeros((max(1, 3 * tri.shape[0]), 4), dtype=np.int32)
        order = np.zeros(n, dtype=np.int32)
        level_begin = np.zeros(n, dtype=np.int32)
        level_end = np.zeros(n, dtype=np.int32)
        info = _native.PlanInfo()
        lib = _native.library()
        _native.check(
            lib.csg_areal_plan_build(
                n, _native.ptr(tri), tri.shape[0], _native.ptr(slot_off), _native.ptr(slot_tri),
                _native.ptr(order), _native.ptr(level_begin), _native.ptr(level_end), ctypes_ref(info),
            ),
            "csg_areal_plan_build",
        )
        return cls(
            slot_off=slot_off,
            slot_tri=slot_tri,
            order=order,
            level_begin=level_begin,
            level_end=level_end,
            n_levels=int(info.n_levels),
            level_stride=int(info.level_stride),
            max_degree=int(info.max_degree),
        )

    def to_device(self, device: torch.device) -> dict[str, torch.Tensor]:
        return {
            name: torch.from_numpy(getattr(self, name)).to(device, non_blocking=False)
            for name in ("slot_off", "slot_tri", "order", "level_begin", "level_end")
        }


def ctypes_ref(struct) -> int:
    import ctypes

    return ctypes.addressof(struct)


def _padded(off: np.ndarray, values: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray]:
    counts = np.diff(off)
    width = max(1, int(counts.max()) if counts.size else 1)
    table = np.zeros((n, width), dtype=np.int64)
    mask = np.arange(width)[None, :] < counts[:, None]
    table[mask] = values[: int(off[-1])]
    return table, mask


def _groups(labels: np.ndarray, count: int) -> tuple[np.ndarray, ...]:
    order = np.argsort(labels, kind="stable")
    bounds = np.searchsorted(labels[order], np.arange(count + 1))
    return tuple(order[bounds[i] : bounds[i + 1]].astype(np.int64) for i in range(count))


@dataclass(frozen=True)
class Surf2SphereTopology:
    """Triangle incidence, 1-ring neighbours, colour and dependency-level groups.

    Same fields as the reference (``surf2sphere.py:401-448``); built by the
    native host builders.  ``plan`` holds the wavefront schedule of the sweeps.
    """

    incident_faces: np.ndarray
    incident_mask: np.ndarray
    neighbours: np.ndarray
    neighbour_mask: np.ndarray
    color_groups: tuple[np.ndarray, ...]
    ordered_groups: tuple[np.ndarray, ...]
    plan: SweepPlan | None = field(default=None, compare=False, repr=False)

    @classmethod
    def from_mesh(cls, mesh: GiftiMesh) -> "Surf2SphereTopology":
        faces = np.ascontiguousarray(mesh.faces, dtype=np.int32)
        n = int(mesh.vertices.shape[0])
        if faces.ndim != 2 or faces.shape[1] != 3:
            raise ValueError(f"faces must have shape [m, 3], got {faces.shape}")
        lib = _native.library()
        inc_off = np.zeros(n + 1, dtype=np.int32)
        inc = np.zeros(max(1, 3 * faces.shape[0]), dtype=np.int32)
        _native.check(
            lib.csg_mesh_incidence(n, _native.ptr(faces), faces.shape[0], _native.ptr(inc_off), _native.ptr(inc)),
            "csg_mesh_incidence",
        )
        nbr_off = np.zeros(n + 1, dtype=np.int32)
        nbr = np.zeros(max(1, 6 * faces.shape[0]), dtype=np.int32)
        _native.check(
            lib.csg_mesh_neighbours(
                n, _native.ptr(faces), faces.shape[0], _native.ptr(nbr_off), _native.ptr(nbr), nbr.size
            ),
            "csg_mesh_neighbours",
        )
        colours = np.zeros(n, dtype=np.int32)
        n_colours = _native.check(
            lib.csg_greedy_colours(n, _native.ptr(nbr_off), _native.ptr(nbr), _native.ptr(colours)),
            "csg_greedy_colours",
        )
        levels = np.zeros(n, dtype=np.int32)
        n_levels = _native.check(
            lib.csg_dependency_levels(n, _native.ptr(nbr_off), _native.ptr(nbr), _native.ptr(levels)),
            "csg_dependency_levels",
        )
        incident_faces, incident_mask = _padded(inc_off, inc, n)
        neighbours, neighbour_mask = _padded(nbr_off, nbr, n)
        return cls(
            incident_faces=incident_faces,
            incident_mask=incident_mask,
            neighbours=neighbours,
            neighbour_mask=neighbour_mask,
            color_groups=_groups(colours, n_colours),
            ordered_groups=_groups(levels, n_levels),
            plan=SweepPlan.build(faces, n),
        )


    @classmethod
    def plan_only(cls, mesh: GiftiMesh) -> "Surf2SphereTopology":
        """Only ``plan`` (the sweep schedule): the GPU path reads nothing else, so the
        reference-compatible tables are left empty instead of being built."""

        faces = np.ascontiguousarray(mesh.faces, dtype=np.int32)
        if faces.ndim != 2 or faces.shape[1] != 3:
            raise ValueError(f"faces must have shape [m, 3], got {faces.shape}")
        empty = np.zeros((0, 0), dtype=np.int64)
        return cls(incident_faces=empty, incident_mask=empty.astype(bool), neighbours=empty,
                   neighbour_mask=empty.astype(bool), color_groups=(), ordered_groups=(),
                   plan=SweepPlan.build(faces, int(mesh.vertices.shape[0])))


@dataclass(frozen=True)
class CatSurf2SphereGpuResult:
    """Store the generated sphere path and synchronized stage timings."""

    vertices: np.ndarray
    faces: np.ndarray
    timings: dict[str, float]
    output_path: Path


def surface_area(mesh: GiftiMesh) -> float:
    """Total surface area in float64 (reference ``surf2sphere.py:461-471``)."""

    vertices = mesh.vertices.astype(np.float64, copy=False)
    triangles = vertices[mesh.faces.astype(np.int64, copy=False)]
    cross = np.cross(triangles[:, 1] - triangles[:, 0], triangles[:, 2] - triangles[:, 0])
    return float(0.5 * np.linalg.norm(cross, axis=1).sum(dtype=np.float64))


def convert_ellipsoid_to_sphere_with_surface_area(vertices: np.ndarray, desired_surface_area: float) -> np.ndarray:
    """Scale to the sphere of area ``desired_surface_area`` (reference 919-937)."""

    geometry = np.ascontiguousarray(vertices, dtype=np.float32)
    radius = math.sqrt(desired_surface_area / (4.0 * math.pi))
    bounds = np.stack((geometry.min(axis=0), geometry.max(axis=0)), axis=1)
    axes = (np.abs(bounds[:, 0]) + np.abs(bounds[:, 1])) * 0.5
    axes = np.maximum(axes, 1.0e-20)
    values = geometry.astype(np.float64)
    scaled = values / axes[None, :]
    norm = np.sqrt((scaled * scaled).sum(axis=1))
    result = np.zeros_like(values)
    nonzero = norm != 0.0
    result[nonzero] = radius * values[nonzero] / norm[nonzero, None]
    result[nonzero] /= axes[None, :]
    return np.ascontiguousarray(result, dtype=np.float32)


def _resolve_dtype(dtype: str | torch.dtype) -> torch.dtype:
    if isinstance(dtype, torch.dtype):
        result = dtype
    else:
        mapping = {"float32": torch.float32, "fp32": torch.float32, "float64": torch.float64, "fp64": torch.float64}
        try:
            result = mapping[str(dtype).lower().replace("torch.", "")]
        except KeyError as exc:
            raise ValueError(f"Unsupported CAT_Surf2Sphere dtype: {dtype}") from exc
    if result not in (torch.float32, torch.float64):
        raise ValueError(f"CAT_Surf2Sphere supports only FP32 and FP64, got {result}")
    return result


def sweep_launch_default(device, arithmetic: str = "cat") -> dict:
    """Launch shape of the sweep kernel: 2 CTAs x 384 threads per SM, 8 lanes per vertex (float32 modes).

    Measured on the 61,442-vertex hull (4,999 sweeps, dataflow form): 76.1 ms,
    against 97.5 ms at 1 x 512 and 78.6 ms at 3 x 256; every shape gives
    identical results (``launch="auto"`` times the candidates instead).  The
    plain float32 mode (more registers per thread) and the float64 mode
    (barrier form) keep 1 x 512.
    """

    from .autotune import sm_count

    if arithmetic != "cat":
        return {"n_ctas": sm_count(device), "threads_per_cta": 512, "lanes_per_vertex": 8}
    return {"n_ctas": 2 * sm_count(device), "threads_per_cta": 384, "lanes_per_vertex": 8}


def ellipsoid_to_sphere_device(points: torch.Tensor, desired_surface_area: float) -> torch.Tensor:
    """:func:`convert_ellipsoid_to_sphere_with_surface_area` in place on a device float32 [n, 3] tensor.

    ``csg_ellipsoid_to_sphere``: the same float32 bounds and float64
    arithmetic, so the result equals the host function bit for bit.
    """

    if points.dtype != torch.float32 or points.ndim != 2 or points.shape[1] != 3 or not points.is_contiguous():
        raise ValueError("points must be a contiguous float32 [n, 3] device tensor")
    radius = math.sqrt(desired_surface_area / (4.0 * math.pi))
    scratch = torch.empty(16, dtype=torch.uint8, device=points.device)
    _native.check(_native.library().csg_ellipsoid_to_sphere(
        _native.ptr(points), int(points.shape[0]), float(radius), _native.ptr(scratch), scratch.numel(),
        _native.stream_handle(like=points)), "csg_ellipsoid_to_sphere")
    return points


def projection_radius_device(points: torch.Tensor) -> float:
    """sqrt(max |p|^2) in float64, |p|^2 = (x x + y y) + z z (the host form of the sweeps' radius)."""

    x = points.to(torch.float64)
    squared = (x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1]) + x[:, 2] * x[:, 2]
    return float(torch.sqrt(squared.max()).item())


def areal_sweeps_device(
    points: torch.Tensor,
    plan_device: dict[str, torch.Tensor],
    plan: SweepPlan,
    *,
    iterations: int,
    project_every: int,
    radius: float,
    arithmetic: str,
    launch: dict | str | None = None,
    timeout_s: float = 2.0,
    scratch: torch.Tensor | None = None,
    stream: torch.cuda.Stream | None = None,
) -> torch.Tensor:
    """Run the sweeps in place on a device tensor (no host synchronisation).

    Returns the scratch tensor; its first 256 bytes hold the kernel's status
    word (read it with :func:`read_status` once the stream is synchronised).
    """

    mode = _native.ARITH[arithmetic]
    n = int(points.shape[0])
    lib = _native.library()
    need = int(lib.csg_areal_scratch_bytes(n, mode))
    if scratch is None or scratch.numel() < need:
        scratch = torch.empty(need, dtype=torch.uint8, device=points.device)
    if launch == "auto":
        cfg = tuned_areal_launch(points, plan_device, plan, arithmetic=arithmetic, radius=radius)
    elif launch:
        # keys the caller leaves out come from the 1 CTA x 512 threads per SM base shape
        cfg = sweep_launch_default(points.device, "fp64")
        cfg.update(launch)
    else:
        cfg = sweep_launch_default(points.device, arithmetic)
    _native.check(
        lib.csg_areal_sweeps(
            _native.ptr(points), n, _native.ptr(plan_device["slot_off"]), _native.ptr(plan_device["slot_tri"]),
            _native.ptr(plan_device["order"]), _native.ptr(plan_device["level_begin"]),
            _native.ptr(plan_device["level_end"]), plan.n_levels, plan.level_stride, plan.max_degree, int(iterations),
            int(project_every), float(radius), mode, _native.ptr(scratch), scratch.numel(),
            int(cfg["n_ctas"]), int(cfg["threads_per_cta"]), int(cfg["lanes_per_vertex"]), float(timeout_s),
            _native.stream_handle(stream, like=points),
        ),
        "csg_areal_sweeps",
    )
    return scratch


def tuned_areal_launch(points: torch.Tensor, plan_device: dict[str, torch.Tensor], plan: SweepPlan, *,
                       arithmetic: str, radius: float, sweeps: int = 200, force: bool = False) -> dict:
    """Fastest launch shape of the sweep kernel for this mesh (autotuned once per mesh size and device).

    Times :func:`cat_surface_gpu_b200.autotune.areal_candidates` on ``sweeps``
    sweeps of a copy of ``points``; every shape gives bit-identical results
    (the update order is fixed by the plan, not by the launch).
    """

    from . import autotune

    key = (int(points.shape[0]), plan.n_levels, plan.level_stride, plan.max_degree, arithmetic, points.dtype)
    if not force:
        hit = autotune.cached("areal_sweeps", key, points.device)
        if hit is not None:
            return hit
    work = torch.empty_like(points)
    scratch = [None]

    def run(shape):
        work.copy_(points)
        scratch[0] = areal_sweeps_device(work, plan_device, plan, iterations=sweeps + 1, project_every=1000,
                                         radius=radius, arithmetic=arithmetic, launch=shape, scratch=scratch[0])

    best = autotune.tune("areal_sweeps", key, autotune.areal_candidates(points.device), run, device=points.device,
                         force=force)
    status, where = read_status(scratch[0])
    if status != 0:
        raise RuntimeError(f"areal sweep kernel failed while tuning (status {status} at {where})")
    return best


def read_status(scratch: torch.Tensor) -> tuple[int, int]:
    """(status, where) of a finished persistent launch (synchronises the stream)."""

    words = scratch[:12].cpu().view(torch.int32).tolist()
    return int(words[1]), int(words[2])


def run_areal_smoothing_cuda(
    vertices: np.ndarray,
    faces: np.ndarray,
    topology: Surf2SphereTopology,
    *,
    iterations: int,
    project_every: int,
    radius: float,
    device: str | torch.device = "cuda",
    dtype: str | torch.dtype = torch.float32,
    kernel: str = "triton",
    schedule: str = "ordered",
    arithmetic: str = "cat",
    schedule_block_size: int | None = None,
    launch: dict | str | None = None,
) -> tuple[np.ndarray, dict[str, float]]:
    """Run every CAT area-smoothing sweep on CUDA in dependency order.

    Same contract as the reference (``surf2sphere.py:940-1104``): sweeps
    ``1 .. iterations-1``, projection to ``radius`` after sweep ``s`` when
    ``s % project_every == 0``; returns ``(float32 [N, 3], timings)``.
    ``kernel`` accepts the reference's names ("triton", "torch") and both run
    the native sm_100a kernel.  Only the exact ``"ordered"`` schedule exists.
    ``dtype=float64`` runs float64 storage and arithmetic and, unlike the
    reference's float64 Triton path, applies the sphere projection.
    ``launch`` is a launch shape dict, ``"auto"`` (autotuned once per mesh
    size and device) or None (the default shape).
    """

    geometry_dtype = _resolve_dtype(dtype)
    if kernel not in ("torch", "triton", "cuda"):
        raise ValueError(f"Unsupported CAT_Surf2Sphere kernel: {kernel}")
    if schedule not in ("ordered", "color"):
        raise ValueError(f"Unsupported CAT_Surf2Sphere schedule: {schedule}")
    if schedule != "ordered":
        raise NotImplementedError("only the exact ordered schedule is implemented (it is also the fastest)")
    if arithmetic not in ("cat", "fp32"):
        raise ValueError(f"Unsupported CAT_Surf2Sphere arithmetic: {arithmetic}")
    if iterations < 1:
        raise ValueError("Must be at least 1")
    if project_every < 0:
        raise ValueError("sphere projection period must be non-negative")
    points_host = np.asarray(vertices)
    if points_host.ndim != 2 or points_host.shape[1] != 3:
        raise ValueError(f"vertices must have shape [n, 3], got {points_host.shape}")
    check_vertices(points_host, "areal smoothing input")
    try:
        target = resolve_device(device)
    except DeviceUnavailable as exc:
        raise RuntimeError(f"CAT_Surf2Sphere CUDA backend: {exc}") from exc
    if geometry_dtype == torch.float64:
        mode = "fp64"
    else:
        mode = "cat" if arithmetic == "cat" else "fp32"
    plan = topology.plan
    if plan is None or plan.slot_off.shape[0] != points_host.shape[0] + 1:
        plan = SweepPlan.build(faces, points_host.shape[0])

    with torch.no_grad(), torch.cuda.device(target):
        points = torch.as_tensor(np.ascontiguousarray(points_host), dtype=geometry_dtype).to(target).contiguous()
        plan_device = plan.to_device(target)
        torch.cuda.synchronize(target)
        start = time.perf_counter()
        scratch = areal_sweeps_device(
            points, plan_device, plan, iterations=iterations, project_every=project_every, radius=radius,
            arithmetic=mode, launch=launch,
        )
        torch.cuda.synchronize(target)
        elapsed = time.perf_counter() - start
        status, where = read_status(scratch)
        if status != 0:
            raise RuntimeError(f"areal sweep kernel reported status {status} at barrier {where}")
        result = points.cpu().numpy()
    return np.ascontiguousarray(result, dtype=np.float32), {
        "areal_smoothing_seconds": elapsed,
        "color_groups": float(plan.n_levels),
        "ordered_schedule": 1.0,
        "cat_mixed_arithmetic": float(mode == "cat"),
        "iterations_requested": float(iterations),
        "iterations_executed": float(max(0, iterations - 1)),
        "wavefront_stride": float(plan.level_stride),
    }


def preprocess_launch_default(device) -> dict:
    """Launch shape of the stages 1-5 pass kernel: 2 CTAs x 384 threads per SM, 8 lanes per vertex.

    Measured on the 61,442-vertex hull (stages 1-5, dataflow form): 49.2 ms,
    against 52.0 ms at 1 x 512 and 49.5 ms at 3 x 256; every shape gives
    identical results.
    """

    from .autotune import sm_count

    return {"n_ctas": 2 * sm_count(device), "threads_per_cta": 384, "lanes_per_vertex": 8}


def preprocess_device(
    points: torch.Tensor,
    faces_device: torch.Tensor,
    topology_device: tuple,
    plan_device: dict[str, torch.Tensor],
    plan: SweepPlan,
    *,
    stop_at: int = 5,
    launch: dict | None = None,
    timeout_s: float = 2.0,
    scratch: torch.Tensor | None = None,
) -> torch.Tensor:
    """Stages 1..stop_at in place on a float32 device tensor (no host synchronisation, no ellipsoid step).

    ``topology_device`` is ``(nb_off, nb, inc_off, inc[, max_degree])`` on
    the device (the 1-ring CSR, the corner-sorted incidences and the largest
    1-ring, which lets the kernel keep the rings in shared memory).  Returns
    the scratch tensor whose first 256 bytes hold the status word
    (:func:`read_status`).
    """

    n, nf = int(points.shape[0]), int(faces_device.shape[0])
    lib = _native.library()
    need = int(lib.csg_preprocess_scratch_bytes(n, nf))
    if scratch is None or scratch.numel() < need:
        scratch = torch.empty(need, dtype=torch.uint8, device=points.device)
    if launch:
        # keys the caller leaves out come from the 1 CTA x 512 threads per SM base shape
        cfg = {"n_ctas": 0, "threads_per_cta": 512, "lanes_per_vertex": 8}
        cfg.update(launch)
    else:
        cfg = preprocess_launch_default(points.device)
    nb_off, nb, inc_off, inc = topology_device[:4]
    max_degree = int(topology_device[4]) if len(topology_device) > 4 else 0
    _native.check(lib.csg_surf2sphere_preprocess(
        _native.ptr(points), n, _native.ptr(faces_device), nf, _native.ptr(nb_off), _native.ptr(nb),
        _native.ptr(inc_off), _native.ptr(inc), _native.ptr(plan_device["order"]),
        _native.ptr(plan_device["level_begin"]), _native.ptr(plan_device["level_end"]), plan.n_levels,
        plan.level_stride, max_degree, int(stop_at), _native.ptr(scratch), scratch.numel(), int(cfg["n_ctas"]),
        int(cfg["threads_per_cta"]), int(cfg["lanes_per_vertex"]), float(timeout_s),
        _native.stream_handle(like=points)), "csg_surf2sphere_preprocess")
    return scratch


def run_surf2sphere_preprocess_cuda(
    vertices: np.ndarray,
    faces: np.ndarray,
    topology: Surf2SphereTopology,
    *,
    stop_at: int = 5,
    desired_surface_area: float,
    device: str | torch.device = "cuda",
    dtype: str | torch.dtype = torch.float32,
    schedule_block_size: int | None = 131072,
    launch: dict | None = None,
    timeout_s: float = 2.0,
) -> tuple[np.ndarray, dict[str, float]]:
    """CAT_Surf2Sphere stages 1..stop_at on the GPU (reference ``surf2sphere.py:716-862``).

    Same contract as the reference: returns ``(float32 [N, 3], timings)``,
    and for ``stop_at >= 5`` the ellipsoid-to-sphere conversion to
    ``desired_surface_area`` is applied.  The distance-smoothing passes run
    in the upstream binary's vertex order (``csg_surf2sphere_preprocess``);
    ``schedule_block_size`` (the reference's colour-group blocking) has no
    meaning for that order and is accepted for compatibility.  Positions are
    float32 with float64 arithmetic; ``dtype=float64`` is not offered.
    """

    if _resolve_dtype(dtype) != torch.float32:
        raise ValueError("the GPU preprocess keeps float32 positions (float64 arithmetic)")
    if stop_at < 1 or stop_at > 5:
        raise ValueError("CUDA preprocessing stop_at must be between 1 and 5")
    check_vertices(vertices, "CAT_Surf2Sphere input")
    try:
        target = resolve_device(device)
    except DeviceUnavailable as exc:
        raise RuntimeError(f"CAT_Surf2Sphere CUDA backend: {exc}") from exc
    points_host = np.ascontiguousarray(np.asarray(vertices, dtype=np.float32))
    tri = np.ascontiguousarray(faces, dtype=np.int32)
    if points_host.ndim != 2 or points_host.shape[1] != 3 or tri.ndim != 2 or tri.shape[1] != 3:
        raise ValueError("vertices and faces must have shape [n, 3] and [m, 3]")
    n, nf = points_host.shape[0], tri.shape[0]
    plan = topology.plan
    if plan is None or plan.slot_off.shape[0] != n + 1:
        plan = SweepPlan.build(tri, n)
    from .features import _topology

    if launch:
        cfg = {"n_ctas": 0, "threads_per_cta": 512, "lanes_per_vertex": 8}
        cfg.update(launch)
    else:
        cfg = preprocess_launch_default(target)
    lib = _native.library()
    timings: dict[str, float] = {}
    with torch.no_grad(), torch.cuda.device(target):
        start = time.perf_counter()
        points = torch.from_numpy(points_host).to(target)
        face_dev = torch.from_numpy(tri).to(target)
        rings = _topology(tri, n, target)
        plan_device = plan.to_device(target)
        scratch = torch.empty(int(lib.csg_preprocess_scratch_bytes(n, nf)), dtype=torch.uint8, device=target)
        torch.cuda.synchronize(target)
        timings["preprocess_upload_seconds"] = time.perf_counter() - start
        start = time.perf_counter()
        preprocess_device(points, face_dev, rings, plan_device, plan, stop_at=stop_at,
                          launch=cfg, timeout_s=timeout_s, scratch=scratch)
        status, where = read_status(scratch)
        if status != 0:
            raise RuntimeError(f"CAT_Surf2Sphere preprocess kernel failed (status {status} at barrier {where})")
        timings["preprocess_kernel_seconds"] = time.perf_counter() - start
        if stop_at >= 5:
            start = time.perf_counter()
            ellipsoid_to_sphere_device(points, desired_surface_area)
            result = points.cpu().numpy()
            timings["ellipsoid_to_sphere_seconds"] = time.perf_counter() - start
        else:
            result = points.cpu().numpy()
    timings["preprocess_total_seconds"] = sum(timings.values())
    return np.ascontiguousarray(result, dtype=np.float32), timings


def _surf2sphere_on_device(mesh: GiftiMesh, topology: "Surf2SphereTopology | Future", area: float, stop_at: int,
                           device, arithmetic: str, timings: dict) -> np.ndarray:
    """Stages 1-5, the ellipsoid step, the sweeps and the final ellipsoid step without leaving the GPU.

    Same results as running :func:`run_surf2sphere_preprocess_cuda` and
    :func:`run_areal_smoothing_cuda` with the host conversions between them:
    the device conversion and projection radius use the host arithmetic.
    ``topology`` may be a future of one (the plan still being built on
    another thread); it is resolved once the upload and ring tables are done.
    """

    from .features import _topology

    if arithmetic not in ("cat", "fp32"):
        raise ValueError(f"Unsupported CAT_Surf2Sphere arithmetic: {arithmetic}")
    try:
        target = resolve_device(device)
    except DeviceUnavailable as exc:
        raise RuntimeError(f"CAT_Surf2Sphere CUDA backend: {exc}") from exc
    tri = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    n = int(mesh.vertices.shape[0])
    with torch.no_grad(), torch.cuda.device(target):
        start = time.perf_counter()
        points = torch.from_numpy(np.ascontiguousarray(mesh.vertices, dtype=np.float32)).to(target)
        rings = _topology(tri, n, target)
        if isinstance(topology, Future):  # the plan was being built while the lines above ran
            topology = topology.result()
        plan = topology.plan
        if plan is None or plan.slot_off.shape[0] != n + 1:
            plan = SweepPlan.build(tri, n)
        plan_device = plan.to_device(target)
        faces_device = torch.from_numpy(tri).to(target)
        timings["preprocess_upload_seconds"] = time.perf_counter() - start
        start = time.perf_counter()
        scratch = preprocess_device(points, faces_device, rings, plan_device, plan, stop_at=5)
        ellipsoid_to_sphere_device(points, area)
        radius = projection_radius_device(points)  # synchronises
        status, where = read_status(scratch)
        if status != 0:
            raise RuntimeError(f"CAT_Surf2Sphere preprocess kernel failed (status {status} at barrier {where})")
        timings["preprocess_kernel_seconds"] = time.perf_counter() - start
        start = time.perf_counter()
        iterations = 1000 * (stop_at - 5)
        scratch = areal_sweeps_device(points, plan_device, plan, iterations=iterations, project_every=1000,
                                      radius=radius, arithmetic=arithmetic)
        ellipsoid_to_sphere_device(points, area)
        result = points.cpu().numpy()
        status, where = read_status(scratch)
        if status != 0:
            raise RuntimeError(f"areal sweep kernel reported status {status} at barrier {where}")
        timings["areal_smoothing_seconds"] = time.perf_counter() - start
    timings.update({"color_groups": float(plan.n_levels), "ordered_schedule": 1.0,
                    "cat_mixed_arithmetic": float(arithmetic == "cat"), "iterations_requested": float(iterations),
                    "iterations_executed": float(max(0, iterations - 1)), "wavefront_stride": float(plan.level_stride)})
    return np.ascontiguousarray(result, dtype=np.float32)


def run_cat_surf2sphere_gpu(
    input_surface: str | Path,
    output_surface: str | Path,
    *,
    reference_cli: str | Path | None = None,
    stop_at: int = 10,
    device: str | torch.device = "cuda",
    dtype: str | torch.dtype = torch.float32,
    kernel: str = "triton",
    preprocess_kernel: str = "triton",
    preprocess_block_size: int | None = 131072,
    areal_schedule: str = "ordered",
    areal_arithmetic: str = "cat",
    areal_block_size: int | None = None,
) -> CatSurf2SphereGpuResult:
    """CAT_Surf2Sphere with every stage on the GPU (reference 1107-1295).

    Stages 1-5, the ellipsoid step, the area-smoothing sweeps and the final
    ellipsoid step run on the native kernels; no process is spawned.  The
    reference's ``preprocess_kernel="cpu"`` ran stages 1-5 on the upstream
    CPU binary ``reference_cli``; this package has no CPU path, so ``"cpu"``
    raises ``ValueError``.  ``"triton"`` (the reference's name for its GPU
    preprocess, the default here) selects the native stages.
    ``reference_cli`` is accepted for signature compatibility and not used.
    """

    if stop_at < 1:
        raise ValueError("stop_at must be at least 1")
    if preprocess_kernel == "cpu":
        raise ValueError("preprocess_kernel='cpu' ran CAT_Surf2Sphere stages 1-5 on the upstream CPU binary; this "
                         "package runs every stage on the GPU: use preprocess_kernel='triton'")
    if preprocess_kernel != "triton":
        raise ValueError(f"Unsupported CAT_Surf2Sphere preprocess kernel: {preprocess_kernel}")
    input_path = Path(input_surface)
    output_path = Path(output_surface)
    timings: dict[str, float] = {}
    total_start = time.perf_counter()
    # every stage on the GPU (reference 1135-1213 with the native preprocess)
    input_mesh = read_gifti_mesh(input_path).check(str(input_path))
    on_device = _resolve_dtype(dtype) == torch.float32 and stop_at > 5
    if on_device:
        # the host plan build (native code, the GIL released) runs beside the surface area,
        # the upload and the ring tables; topology_build_seconds is its own duration
        def timed_plan():
            begin = time.perf_counter()
            built = Surf2SphereTopology.plan_only(input_mesh)
            timings["topology_build_seconds"] = time.perf_counter() - begin
            return built

        with ThreadPoolExecutor(max_workers=1) as pool:
            future = pool.submit(timed_plan)
            area = surface_area(input_mesh)
            pre = _surf2sphere_on_device(input_mesh, future, area, stop_at, device, areal_arithmetic, timings)
        write_start = time.perf_counter()
        write_vertices_like(input_path, output_path, pre)
        timings["output_write_seconds"] = time.perf_counter() - write_start
        timings["total_seconds"] = time.perf_counter() - total_start
        # the file holds exactly these arrays (float32 vertices, the input's faces)
        return CatSurf2SphereGpuResult(np.ascontiguousarray(pre, dtype=np.float32), input_mesh.faces, timings,
                                       output_path)
    topology_start = time.perf_counter()
    topology = Surf2SphereTopology.from_mesh(input_mesh)
    timings["topology_build_seconds"] = time.perf_counter() - topology_start
    area = surface_area(input_mesh)
    pre, pre_timings = run_surf2sphere_preprocess_cuda(
        input_mesh.vertices, input_mesh.faces, topology, stop_at=min(stop_at, 5), desired_surface_area=area,
        device=device, dtype=dtype, schedule_block_size=preprocess_block_size)
    timings.update(pre_timings)
    if stop_at > 5:
        radius = float(np.sqrt(np.max(np.sum(pre.astype(np.float64) ** 2, axis=1))))
        smoothed, smooth_timings = run_areal_smoothing_cuda(
            pre, input_mesh.faces, topology, iterations=1000 * (stop_at - 5), project_every=1000, radius=radius,
            device=device, dtype=dtype, kernel=kernel, schedule=areal_schedule, arithmetic=areal_arithmetic,
            schedule_block_size=areal_block_size)
        timings.update(smooth_timings)
        conversion_start = time.perf_counter()
        pre = convert_ellipsoid_to_sphere_with_surface_area(smoothed, area)
        timings["ellipsoid_to_sphere_seconds"] = time.perf_counter() - conversion_start
    write_start = time.perf_counter()
    write_vertices_like(input_path, output_path, pre)
    timings["output_write_seconds"] = time.perf_counter() - write_start
    result_mesh = read_gifti_mesh(output_path)
    timings["total_seconds"] = time.perf_counter() - total_start
    return CatSurf2SphereGpuResult(result_mesh.vertices, result_mesh.faces, timings, output_path)
