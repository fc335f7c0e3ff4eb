"""End-to-end CAT_SurfWarp-compatible registration on a B200 (drop-in for the reference's gpu_pipeline).

``run_cat_surface_gpu_pipeline`` follows the reference's flow
(``src/cat_surface_gpu/gpu_pipeline.py:468-1326``): stencils for both
spheres, rotation features, 46-seed + Nelder-Mead rotation search, the
rotated source stencil, ``runs`` DARTEL solves with the final warp applied
between runs, the ``-avg`` pole-rotated solve and its blend, GIFTI output.

Every stencil is built by this package's GPU stencil builder
(``stencil_builder="native"``).  Rotation features come from
``rotation_values_path``; from the depth potential on the GPU (``"cuda"``, the
reference's default that ``"auto"`` resolves to -- ``rotation_feature.py``);
or from ``"native-curvature"`` (an option of this package): the type-5
curvature of the resampled surfaces heat-smoothed with the rotation FWHMs
(15 source, 10 target) and min-max normalised.

No process is spawned.  The reference's options that ran its helper
binaries -- a stencil-builder path, the ``official-cpu``,
``cuda-official-depth`` and ``cuda-official-geometry`` feature backends and
the ``rotation_*_probe`` executables -- are parsed and rejected with
``ValueError`` before any file is read.
"""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
import math
from pathlib import Path
import time
from typing import Sequence

import numpy as np
import torch

from . import _native
from .device import resolve_device
from .gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh
from .rotation_pipeline import RotationPipeline, read_rotation_values
from .surface_stencil import SurfaceStencil, build_surface_stencil
from .surface_warp import (apply_flow_to_stenciled_sphere, average_xz_surfaces, solve_dartel_from_surfaces,
                           solve_dartel_from_surfaces_many)


@dataclass(frozen=True)
class CatSurfaceGpuResult:
    """Final mesh data, rotation diagnostics, timings, and output path."""

    vertices: np.ndarray
    faces: np.ndarray
    rotation_angle: np.ndarray
    rotation_cost: float
    timings: dict[str, float]
    output_path: Path


def _resolve_dartel_dtype(value) -> torch.dtype:
    if isinstance(value, torch.dtype):
        resolved = value
    else:
        mapping = {"float32": torch.float32, "fp32": torch.float32, "float64": torch.float64, "fp64": torch.float64}
        try:
            resolved = mapping[str(value).lower().replace("torch.", "")]
        except KeyError as error:
            raise ValueError("dartel_dtype must be float32/fp32 or float64/fp64") from error
    if resolved not in {torch.float32, torch.float64}:
        raise ValueError("dartel_dtype must be torch.float32 or torch.float64")
    return resolved


def normalise_sphere(vertices: np.ndarray) -> np.ndarray:
    """Centre on the vertex mean and project to unit length (reference 274-305).

    The centre is the sequential float64 sum of the float32 coordinates, as in
    the reference's per-vertex loop.
    """

    value = np.ascontiguousarray(np.asarray(vertices, dtype=np.float32))
    if value.ndim != 2 or value.shape[1] != 3:
        raise ValueError(f"Sphere vertices must have shape [n, 3], got {value.shape}")
    out = np.empty_like(value)
    rc = _native.library().csg_normalise_sphere(value.shape[0], _native.ptr(value), _native.ptr(out))
    if rc != 0:
        raise ValueError("Sphere contains a vertex that cannot be normalized")
    return out


def rotation_matrix_from_angles(angles) -> torch.Tensor:
    """float64 Rz (Ry Rx) as a 3x3 CPU tensor (reference 308-369).

    Built with torch's float64 sin/cos and the same column-major product
    order as the reference, so the matrix is bit-identical to it.
    """

    value = torch.as_tensor(np.asarray(angles, dtype=np.float64)).reshape(-1)
    if value.numel() != 3:
        raise ValueError("Rotation must contain exactly three angles")
    # torch's float64 sin/cos of each angle (as the reference takes them); the products are
    # plain float64 multiplies and adds, one rounding each, so Python floats give the same bits
    ca = [float(torch.cos(angle)) for angle in value.unbind()]
    sa = [float(torch.sin(angle)) for angle in value.unbind()]
    one, zero = 1.0, 0.0
    rx = (one, zero, zero, zero, ca[0], sa[0], zero, -sa[0], ca[0])
    ry = (ca[1], zero, sa[1], zero, one, zero, -sa[1], zero, ca[1])
    rz = (ca[2], sa[2], zero, -sa[2], ca[2], zero, zero, zero, one)

    def product(left, right):
        out = [0.0] * 9
        for r in range(3):
            for c in range(3):
                out[r + 3 * c] = ((zero + left[r] * right[3 * c]) + left[r + 3] * right[1 + 3 * c]) \
                    + left[r + 6] * right[2 + 3 * c]
        return out

    return torch.tensor(product(rz, product(ry, rx)), dtype=torch.float64).reshape(3, 3)


def rotate_vertices(vertices: np.ndarray, angles) -> np.ndarray:
    """float32(vertices @ M^T) in float64 on the CPU, M = rotation_matrix_from_angles (reference 372-378)."""

    sphere = torch.as_tensor(np.asarray(vertices), dtype=torch.float64)
    rotated = sphere @ rotation_matrix_from_angles(angles).transpose(0, 1)
    return np.ascontiguousarray(rotated.numpy(), dtype=np.float32)


class _Stencils:
    """Builds stencils with the native builder on the pipeline's device.

    Both sides' builds launch on the current stream.  Giving each builder thread a
    stream of its own was measured and left out: the pool's streams each keep their
    own cached device blocks, so builds on a stream the allocator had not seen paid
    for fresh allocations (73 and 80 ms stencil stages in one run, against 6 and 8).
    """

    def __init__(self, threads: int, nx: int, ny: int, device=None):
        self.threads, self.nx, self.ny, self.device = threads, nx, ny, device

    def build(self, sphere: GiftiMesh, *, normalize: bool) -> SurfaceStencil:
        return build_surface_stencil(sphere.vertices, sphere.faces, nx=self.nx, ny=self.ny, normalize=normalize,
                                     threads=self.threads, device=self.device)


def native_rotation_features(source_stencil, target_stencil, source_surface, target_surface, device,
                             heat_fwhms=(15.0, 10.0)) -> tuple[np.ndarray, np.ndarray]:
    """Type-5 curvature of the resampled surfaces at the rotation FWHMs, min-max normalised."""

    out = []
    for stencil, surface, fwhm in ((source_stencil, source_surface, heat_fwhms[0]),
                                   (target_stencil, target_surface, heat_fwhms[1])):
        st = stencil.to(device, geometry_dtype=torch.float32)
        mapped = st.resample_vertices(torch.as_tensor(surface, dtype=torch.float32, device=device))
        out.append(st.curvature_type5(mapped, float(fwhm)).cpu().numpy())
    return out[0], out[1]


def depth_rotation_features(source_stencil, target_stencil, source_surface, target_surface, device, *,
                            solver: str = "colored-sor", smoothed_surfaces=None, depth_values=None,
                            timings: dict | None = None):
    """Depth-potential features of both sides (the reference's "cuda" backend, reference 836-893).

    One batched solve for both sides on the stencils' shared triangulation;
    returns the normalised device values (source, target).
    """

    from .rotation_feature import compute_rotation_features

    stencils = [st.to(device, geometry_dtype=torch.float32) for st in (source_stencil, target_stencil)]
    surfaces = [torch.as_tensor(np.asarray(v), dtype=torch.float32, device=device).contiguous()
                for v in (source_surface, target_surface)]
    results = compute_rotation_features(stencils, surfaces, heat_fwhms=(15.0, 10.0),
                                        smoothed_surfaces=smoothed_surfaces, depth_values=depth_values, solver=solver)
    if timings is not None:
        for side, result in zip(("source", "target"), results):
            timings[f"rotation_feature_{side}_iterations"] = float(result.iterations)
            timings[f"rotation_feature_{side}_residual"] = float(result.relative_residual)
    return results[0].values, results[1].values


_BACKENDS = {"auto", "native-curvature", "cuda"}
# the reference's feature backends that run its helper binaries (reference 550-560, 836-893)
_HELPER_BACKENDS = {"official-cpu", "cuda-official-depth", "cuda-official-geometry"}
_SOLVERS = {"colored-sor", "pcg"}
_SEARCHES = {"nelder-mead", "euler-grid"}


def _validate_options(*, steps=2, runs=1, stencil_threads=8, curvtypes=(5, 5, 2), fwhm=(5.0, 5.0 / 3.0, 5.0 / 9.0),
                      rotation_max_iter=500, rotation_tol=1.0e-4, rotation_simplex_step=0.1,
                      rotation_feature_backend="auto", rotation_feature_solver="colored-sor", has_values=False,
                      dartel_dtype=torch.float64, device="cuda", stencil_builder="native", rotated_stencil_builder=None,
                      rotation_values_probe=None, rotation_geometry_probe=None, rotation_depth_probe=None,
                      rotation_search="nelder-mead", **_unused) -> None:
    """Argument checks of the reference pipeline (reference 514-560), before any file is read.

    Options that would run one of the reference's helper binaries raise
    ``ValueError``: this package computes stencils and rotation features on
    the GPU and spawns no process.
    """

    if steps < 1 or steps > 3:
        raise ValueError("steps must be between 1 and 3")
    if runs < 1:
        raise ValueError("runs must be positive")
    if stencil_threads < 1 or stencil_threads > 256:
        raise ValueError("stencil_threads must be between 1 and 256")
    if len(curvtypes) < steps or len(fwhm) < steps:
        raise ValueError("curvtypes and fwhm must contain at least 'steps' entries")
    if rotation_max_iter < 1 or rotation_tol < 0.0 or rotation_simplex_step <= 0.0:
        raise ValueError("rotation_max_iter, rotation_tol, and rotation_simplex_step must be positive")
    if rotation_feature_backend in _HELPER_BACKENDS:
        raise ValueError(f"rotation_feature_backend={rotation_feature_backend!r} runs the reference's helper "
                         "binaries; this package computes the rotation features on the GPU ('auto' or 'cuda', or "
                         "'native-curvature')")
    if rotation_feature_backend not in _BACKENDS:
        raise ValueError(f"rotation_feature_backend must be one of {sorted(_BACKENDS)}")
    for name, builder in (("stencil_builder", stencil_builder), ("rotated_stencil_builder", rotated_stencil_builder)):
        if builder not in (None, "native"):
            raise ValueError(f"{name}={builder!r}: the reference's stencil helper binary is not run; stencils are "
                             "built on the GPU (stencil_builder='native')")
    for name, probe in (("rotation_values_probe", rotation_values_probe),
                        ("rotation_geometry_probe", rotation_geometry_probe),
                        ("rotation_depth_probe", rotation_depth_probe)):
        if probe is not None:
            raise ValueError(f"{name}: the reference's feature helper binaries are not run; rotation features are "
                             "computed on the GPU")
    if rotation_feature_solver not in _SOLVERS:
        raise ValueError("rotation_feature_solver must be 'colored-sor' or 'pcg'")
    if rotation_search not in _SEARCHES:
        raise ValueError(f"rotation_search must be one of {sorted(_SEARCHES)}")
    if rotation_search == "euler-grid" and has_values:
        raise ValueError("rotation_search='euler-grid' computes its own two features; rotation values are not used")
    _resolve_dartel_dtype(dartel_dtype)
    if device == "cpu" or str(device) == "cpu":
        raise ValueError("The explicit GPU pipeline requires a CUDA device")


def run_cat_surface_gpu_pipeline(
    source_surface_path, source_sphere_path, target_surface_path, target_sphere_path, output_path, *,
    source_stencil_path=None, target_stencil_path=None, rotation_values_path=None, **options,
) -> CatSurfaceGpuResult:
    """Rotation, DARTEL runs, -avg blend and GIFTI output (reference 468-1326).

    Reads the four GIFTI meshes, runs :func:`register_meshes` and writes the
    registered sphere with the source sphere's topology and array intents.
    ``options`` are :func:`register_meshes`'s keyword arguments.
    """

    _validate_options(has_values=rotation_values_path is not None, **options)
    total_start = time.perf_counter()
    with ThreadPoolExecutor(max_workers=4) as pool:  # the four decodes overlap where zlib releases the GIL
        meshes = list(pool.map(read_gifti_mesh, (source_surface_path, source_sphere_path, target_surface_path,
                                                 target_sphere_path)))
    read_seconds = time.perf_counter() - total_start
    stencils = {}
    if source_stencil_path is not None:
        stencils["source_stencil"] = SurfaceStencil.from_file(source_stencil_path)
    if target_stencil_path is not None:
        stencils["target_stencil"] = SurfaceStencil.from_file(target_stencil_path)
    rotation_values = read_rotation_values(rotation_values_path) if rotation_values_path is not None else None
    vertices, angle, cost, timings = register_meshes(
        *meshes, paths=(source_surface_path, source_sphere_path, target_surface_path, target_sphere_path),
        rotation_values=rotation_values, **stencils, **options)
    timings["input_read_seconds"] = read_seconds
    output = Path(output_path)
    write_start = time.perf_counter()
    final_mesh = GiftiMesh(vertices, meshes[1].faces)
    write_gifti_mesh(output, final_mesh, reference_path=source_sphere_path)
    timings["output_write_seconds"] = time.perf_counter() - write_start
    timings["total_seconds"] = time.perf_counter() - total_start
    return CatSurfaceGpuResult(vertices=final_mesh.vertices, faces=final_mesh.faces, rotation_angle=angle,
                               rotation_cost=cost, timings=timings, output_path=output)


def register_meshes(
    source_surface: GiftiMesh, source_sphere: GiftiMesh, target_surface: GiftiMesh, target_sphere: GiftiMesh, *,
    paths=None, source_stencil: SurfaceStencil | None = None, target_stencil: SurfaceStencil | None = None,
    rotation_values=None, rotation_values_probe=None, rotation_geometry_probe=None, rotation_depth_probe=None,
    stencil_builder="native", rotated_stencil_builder=None, stencil_threads: int = 8, device="cuda",
    kernel: str = "triton", dartel_dtype=torch.float64, squaring_kernel: str | None = None, steps: int = 2,
    runs: int = 1, avg: bool = False, curvtypes: Sequence[int] = (5, 5, 2),
    fwhm: Sequence[float] = (5.0, 5.0 / 3.0, 5.0 / 9.0), loop: int = 6, cycles: int = 3, nit: int = 3, its: int = 3,
    code: int = 1, point_chunk: int = 4096, rotation_grid_size: int = 128, rotation_margin: int = 1,
    rotation_refine: bool = True, rotation_max_iter: int = 500, rotation_tol: float = 1.0e-4,
    rotation_simplex_step: float = 0.1, rotation_feature_backend: str = "auto",
    rotation_feature_solver: str = "colored-sor", parallel_sides: bool = True, optimized_dartel: bool = True,
    cuda_graph: bool = True, sheet_size: tuple[int, int] = (512, 256), rotation_search: str = "nelder-mead",
) -> tuple[np.ndarray, np.ndarray, float, dict[str, float]]:
    """In-memory SurfWarp registration: returns (sphere vertices f32, angle, rotation cost, timings).

    Same flow and options as :func:`run_cat_surface_gpu_pipeline`.  ``paths``
    (the four input files) is accepted for signature compatibility and not
    used.  ``sheet_size`` is the DARTEL sheet (nx, ny) of the stencils built
    here.  Every launch runs with ``device`` as the current CUDA device.
    ``rotation_search`` is the reference's 46 seeds + Nelder-Mead
    (``"nelder-mead"``, default) or ``"euler-grid"``: all of SO(3) on a 10
    degree Euler grid, then a 2 degree grid round the best, on two features
    per side -- the type-5 curvature (FWHM 15 / 10) and the depth potential,
    each z-scored and rounded to float32.
    """

    _validate_options(steps=steps, runs=runs, stencil_threads=stencil_threads, curvtypes=curvtypes, fwhm=fwhm,
                      rotation_max_iter=rotation_max_iter, rotation_tol=rotation_tol,
                      rotation_simplex_step=rotation_simplex_step, rotation_feature_backend=rotation_feature_backend,
                      rotation_feature_solver=rotation_feature_solver, has_values=rotation_values is not None,
                      dartel_dtype=dartel_dtype, device=device, stencil_builder=stencil_builder,
                      rotation_search=rotation_search,
                      rotated_stencil_builder=rotated_stencil_builder, rotation_values_probe=rotation_values_probe,
                      rotation_geometry_probe=rotation_geometry_probe, rotation_depth_probe=rotation_depth_probe)
    if rotation_feature_backend == "auto":
        # the reference's resolution without a values probe (reference 550-553)
        rotation_feature_backend = "cuda"
    # the kernels trust the meshes: refuse bad ones before any launch
    for label, surface, sphere in (("source", source_surface, source_sphere), ("target", target_surface, target_sphere)):
        surface.check(f"{label} surface")
        sphere.check(f"{label} sphere")
        if surface.vertices.shape[0] != sphere.vertices.shape[0]:
            raise ValueError(f"{label} surface has {surface.vertices.shape[0]} vertices but its sphere has "
                             f"{sphere.vertices.shape[0]}")
    for label, stencil in (("source", source_stencil), ("target", target_stencil)):
        if stencil is not None:
            stencil.validate()
    if rotation_values is not None:
        for label, values in zip(("source", "target"), rotation_values):
            if not np.isfinite(np.asarray(values, dtype=np.float64)).all():
                raise ValueError(f"{label} rotation values are not finite")
    solve_dtype = _resolve_dartel_dtype(dartel_dtype)
    target_device = resolve_device(device)
    graph_requested = bool(cuda_graph and (runs + int(avg) >= 3))
    timings: dict[str, float] = {}
    total_start = time.perf_counter()
    nx, ny = (int(v) for v in sheet_size)

    # the native entry points launch on the current device: make it the pipeline's
    with torch.cuda.device(target_device):
        builder = _Stencils(stencil_threads, nx, ny, target_device)
        rotated_builder = builder
        start = time.perf_counter()
        with ThreadPoolExecutor(max_workers=2) as pool:
            src_future = None if source_stencil is not None else pool.submit(builder.build, source_sphere,
                                                                             normalize=True)
            tgt_future = None if target_stencil is not None else pool.submit(builder.build, target_sphere,
                                                                             normalize=True)
            source_stencil = source_stencil if src_future is None else src_future.result()
            target_stencil = target_stencil if tgt_future is None else tgt_future.result()
        timings["initial_stencil_seconds"] = time.perf_counter() - start

        start = time.perf_counter()
        if rotation_search == "euler-grid":
            from .surface_rotation import zscore

            curvature = native_rotation_features(source_stencil, target_stencil, source_surface.vertices,
                                                 target_surface.vertices, target_device)
            depth = depth_rotation_features(source_stencil, target_stencil, source_surface.vertices,
                                            target_surface.vertices, target_device, solver=rotation_feature_solver,
                                            timings=timings)
            source_values = zscore(np.stack([np.asarray(curvature[0]), depth[0].cpu().numpy()]))
            target_values = zscore(np.stack([np.asarray(curvature[1]), depth[1].cpu().numpy()]))
        elif rotation_values is not None:
            source_values, target_values = rotation_values
        elif rotation_feature_backend == "native-curvature":
            source_values, target_values = native_rotation_features(
                source_stencil, target_stencil, source_surface.vertices, target_surface.vertices, target_device)
        else:
            source_values, target_values = depth_rotation_features(
                source_stencil, target_stencil, source_surface.vertices, target_surface.vertices, target_device,
                solver=rotation_feature_solver, timings=timings)
        torch.cuda.synchronize(target_device)
        timings["rotation_feature_seconds"] = time.perf_counter() - start

        start = time.perf_counter()
        rotation_pipeline = RotationPipeline.from_stencil(target_stencil, device=target_device,
                                                          grid_size=rotation_grid_size, margin=rotation_margin)
        torch.cuda.synchronize(target_device)
        timings["rotation_index_upload_seconds"] = time.perf_counter() - start
        start = time.perf_counter()
        if rotation_search == "euler-grid":
            rotation = rotation_pipeline.search_euler_grid(source_stencil.sphere_points, source_values, target_values)
        else:
            rotation = rotation_pipeline.search(source_stencil.sphere_points, source_values, target_values,
                                                point_chunk=point_chunk, refine=rotation_refine,
                                                max_iter=rotation_max_iter, tol=rotation_tol,
                                                simplex_step=rotation_simplex_step)
        torch.cuda.synchronize(target_device)
        timings["rotation_search_seconds"] = time.perf_counter() - start

        angle = rotation.angle.detach().cpu().numpy()
        current_sphere = rotate_vertices(normalise_sphere(source_sphere.vertices), angle)
        pole = np.asarray((0.0, np.pi / 2.0, 0.0))
        avg_target_surface = rotate_vertices(target_surface.vertices, pole)
        avg_target_sphere = rotate_vertices(normalise_sphere(target_sphere.vertices), pole)
        start = time.perf_counter()
        with ThreadPoolExecutor(max_workers=2) as pool:
            cur_future = pool.submit(rotated_builder.build, GiftiMesh(current_sphere, source_sphere.faces),
                                     normalize=False)
            avg_future = pool.submit(rotated_builder.build, GiftiMesh(avg_target_sphere, target_sphere.faces),
                                     normalize=False) if avg else None
            current_stencil = cur_future.result()
            avg_target_stencil = avg_future.result() if avg_future is not None else None
        timings["rotated_stencil_seconds"] = time.perf_counter() - start

        target_dev = target_stencil.to(target_device)
        current_dev = current_stencil.to(target_device)

        def on_device(array):
            return torch.as_tensor(np.ascontiguousarray(array), dtype=torch.float32, device=target_device)

        source_surface_dev = on_device(source_surface.vertices)
        target_surface_dev = on_device(target_surface.vertices)

        def solve_one(src_vertices, tgt_vertices, src_stencil, tgt_stencil, solve_fwhm, solve_loop):
            return solve_dartel_from_surfaces(src_vertices, tgt_vertices, src_stencil, tgt_stencil, fwhm=solve_fwhm,
                                              curvtypes=tuple(curvtypes), n_steps=steps, loop=solve_loop,
                                              cycles=cycles, nit=nit, its=its, code=code, kernel=kernel,
                                              device=target_device, dtype=solve_dtype, squaring_kernel=squaring_kernel,
                                              parallel_sides=parallel_sides, optimized=optimized_dartel,
                                              cuda_graph=graph_requested)

        dartel_start = time.perf_counter()
        last_flow = avg_flow = None
        final_prewarp = None
        avg_source_dev = None
        avg_source_sphere = None
        avg_fwhm = tuple(float(fwhm[0]) / (3.0 ** (steps * (runs + 1) + i)) for i in range(steps))
        for run_index in range(runs):
            run_start = time.perf_counter()
            base = float(fwhm[0])
            run_fwhm = tuple(base / (3.0 ** (steps * (run_index + 1) + i)) for i in range(steps))
            if avg and run_index == runs - 1:
                # the -avg solve starts from the same sphere as the last run and does not depend on its
                # result (reference 1140-1177, 1229-1268): both registrations go through one batched
                # solve, whose flows equal the two separate solves
                final_prewarp = current_sphere.copy()
                avg_source_surface = rotate_vertices(source_surface.vertices, pole)
                avg_source_sphere = rotate_vertices(final_prewarp, pole)
                avg_source_stencil = rotated_builder.build(GiftiMesh(avg_source_sphere, source_sphere.faces),
                                                           normalize=False)
                avg_source_dev = avg_source_stencil.to(target_device)
                last_flow, avg_flow = solve_dartel_from_surfaces_many(
                    [(source_surface_dev, target_surface_dev, current_dev, target_dev, run_fwhm),
                     (on_device(avg_source_surface), on_device(avg_target_surface), avg_source_dev,
                      avg_target_stencil.to(target_device), avg_fwhm)],
                    curvtypes=tuple(curvtypes), loop=loop, n_steps=steps, cycles=cycles, nit=nit, its=its, code=code,
                    device=target_device, dtype=solve_dtype, parallel_sides=parallel_sides, cuda_graph=graph_requested)
            else:
                last_flow = solve_one(source_surface_dev, target_surface_dev, current_dev, target_dev, run_fwhm,
                                      loop).flow
                current_sphere = apply_flow_to_stenciled_sphere(
                    on_device(current_sphere), last_flow, current_dev, inverse=True, device=target_device,
                    dtype=solve_dtype).cpu().numpy().astype(np.float32)
            torch.cuda.synchronize(target_device)
            timings[f"dartel_run_{run_index}_seconds"] = time.perf_counter() - run_start
            if run_index + 1 < runs:
                current_stencil = rotated_builder.build(GiftiMesh(current_sphere, source_sphere.faces),
                                                        normalize=False)
                current_dev = current_stencil.to(target_device)
        if avg:
            avg_start = time.perf_counter()
            main_warped = apply_flow_to_stenciled_sphere(on_device(final_prewarp), last_flow, current_dev,
                                                         inverse=True, device=target_device, dtype=solve_dtype)
            avg_warped = apply_flow_to_stenciled_sphere(on_device(avg_source_sphere), avg_flow, avg_source_dev,
                                                        inverse=True, device=target_device, dtype=solve_dtype)
            reverse = rotation_matrix_from_angles(-pole).to(device=target_device)
            unrotated = avg_warped.to(torch.float64) @ reverse.transpose(0, 1)
            combined = average_xz_surfaces(unrotated, main_warped, device=target_device)
            current_sphere = combined.cpu().numpy().astype(np.float32)
            timings["avg_dartel_seconds"] = time.perf_counter() - avg_start
        timings["dartel_total_seconds"] = time.perf_counter() - dartel_start
    timings["register_seconds"] = time.perf_counter() - total_start
    return (np.ascontiguousarray(current_sphere, dtype=np.float32), np.ascontiguousarray(angle, dtype=np.float64),
            float(rotation.cost.detach().cpu()), timings)
