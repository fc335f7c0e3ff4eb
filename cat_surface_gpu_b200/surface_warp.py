"""DARTEL solves and the final warp on a B200 (drop-in for the reference's surface_warp).

Follows ``src/cat_surface_gpu/surface_warp.py``.  ``solve_dartel_maps`` runs
every step map of a solve as one batch through ``csg_dartel_solve`` (the maps
are independent: each starts from zero velocity, and the flow is the
exponential of the last map's velocity), optionally captured once in a CUDA
graph keyed like the reference's graph cache.  ``solve_dartel_batch``
exposes the same solve for many registrations at once.
"""

from __future__ import annotations

from dataclasses import dataclass
import time
from typing import Sequence

import torch

from . import _native, features
from .dartel_grid import _addr, _dtype_code, _scratch, _tensor, expdef, resolve_device


@dataclass(frozen=True)
class DartelSolveResult:
    """Store a solved flow, warped feature maps, and DARTEL diagnostics."""

    flow: torch.Tensor
    source_maps: torch.Tensor
    target_maps: torch.Tensor
    metrics: torch.Tensor


def default_dartel_parameters(loop: int = 6, *, mu: float = 0.125, lambda_: float = 0.0, lmreg: float = 1e-3,
                              muchange: int = 4, murate: float = 1.25):
    """Upstream regulariser schedule per loop (reference 76-107)."""

    if loop <= 0:
        raise ValueError(f"loop must be positive, got {loop}")
    if muchange <= 0 or murate <= 0:
        raise ValueError("muchange and murate must be positive")
    values = []
    current_mu = float(mu)
    current_lambda = float(lambda_)
    for index in range(loop):
        values.append((1.0, 1.0, current_mu, current_lambda, current_lambda / 2.0))
        if (index + 1) % muchange == 0:
            current_mu /= murate
        current_lambda /= 5.0
    return tuple(values)


class _Solver:
    """Owns the device buffers of one (batch, ny, nx, dtype, schedule) solve."""

    def __init__(self, batch, ny, nx, dtype, device, loop, lmreg, cycles, nit, its, code, assume):
        self.batch, self.ny, self.nx, self.dtype, self.device = batch, ny, nx, dtype, device
        self.loop, self.lmreg, self.cycles, self.nit, self.its, self.code = loop, lmreg, cycles, nit, its, code
        self.assume = assume
        params = default_dartel_parameters(loop)
        self._params = _native.doubles([value for row in params for value in row])
        self.source = torch.zeros((batch, ny, nx), dtype=dtype, device=device)
        self.target = torch.zeros_like(self.source)
        self.velocity = torch.zeros((batch, 2, ny, nx), dtype=dtype, device=device)
        self.metrics = torch.zeros((batch, loop * its, 3), dtype=dtype, device=device)
        self.scratch = _scratch(dtype, device, batch, nx, ny)
        self.expdef_scratch = _scratch(dtype, device, 1, nx, ny)
        self.flow = torch.empty((2, ny, nx), dtype=dtype, device=device)
        self.flows = torch.empty((batch, 2, ny, nx), dtype=dtype, device=device)
        self.last_velocity = None

    def launch(self, stream_handle: int, flows: str = "last", steps_per_registration: int = 1) -> None:
        """Enqueue the whole solve on a stream (no host synchronisation when `assume`).

        flows: "last" -- exponential of the last map's velocity (one registration);
        "all" -- of every map's velocity; "registrations" -- of the last map
        of each run of ``steps_per_registration`` maps (many registrations).
        Torch's current stream must be the stream of ``stream_handle``.
        """

        lib = _native.library()
        self.velocity.zero_()
        _native.check(
            lib.csg_dartel_solve(
                _dtype_code(self.dtype), self.batch, self.nx, self.ny, self.source.data_ptr(), self.target.data_ptr(),
                self.velocity.data_ptr(), self.metrics.data_ptr(), self.loop, _addr(self._params), self.its,
                float(self.lmreg), self.cycles, self.nit, self.code, int(self.assume), self.scratch.data_ptr(),
                self.scratch.numel(), stream_handle,
            ),
            "csg_dartel_solve",
        )
        if flows == "last":
            _native.check(
                lib.csg_dartel_expdef(
                    _dtype_code(self.dtype), 1, self.nx, self.ny, self.velocity[self.batch - 1].data_ptr(), 10,
                    self.flow.data_ptr(), None, self.expdef_scratch.data_ptr(), self.expdef_scratch.numel(),
                    stream_handle,
                ),
                "csg_dartel_expdef",
            )
        elif flows == "registrations":
            steps = int(steps_per_registration)
            count = self.batch // steps
            if self.last_velocity is None:
                self.last_velocity = torch.empty((count, 2, self.ny, self.nx), dtype=self.dtype, device=self.device)
            self.last_velocity.copy_(self.velocity.view(count, steps, 2, self.ny, self.nx)[:, steps - 1])
            _native.check(
                lib.csg_dartel_expdef(
                    _dtype_code(self.dtype), count, self.nx, self.ny, self.last_velocity.data_ptr(), 10,
                    self.flows.data_ptr(), None, self.scratch.data_ptr(), self.scratch.numel(), stream_handle,
                ),
                "csg_dartel_expdef",
            )
        else:
            _native.check(
                lib.csg_dartel_expdef(
                    _dtype_code(self.dtype), self.batch, self.nx, self.ny, self.velocity.data_ptr(), 10,
                    self.flows.data_ptr(), None, self.scratch.data_ptr(), self.scratch.numel(), stream_handle,
                ),
                "csg_dartel_expdef",
            )


@dataclass
class _GraphEntry:
    graph: torch.cuda.CUDAGraph
    solver: _Solver
    capture_seconds: float
    kernels: int = 0  # native kernels inside the graph

    def replay(self) -> None:
        self.graph.replay()
        _native.note_graph_replay(self.kernels)


_GRAPH_CACHE: dict[tuple, _GraphEntry] = {}


def _graph_key(source, target, *, loop, lmreg, cycles, nit, its, code, kernel, squaring_kernel, optimized):
    return (
        source.device.type, source.device.index, source.dtype, tuple(source.shape), tuple(target.shape), int(loop),
        float(lmreg), int(cycles), int(nit), int(its), int(code), str(kernel),
        "auto" if squaring_kernel is None else str(squaring_kernel), bool(optimized),
    )


def _capture(source, target, *, loop, lmreg, cycles, nit, its, code, device, flows: str = "last",
             steps_per_registration: int = 1) -> _GraphEntry:
    batch = int(source.shape[0]) if flows != "registrations" else int(source.shape[0] * source.shape[1])
    ny, nx = (int(v) for v in source.shape[-2:])
    solver = _Solver(batch, ny, nx, source.dtype, device, loop, lmreg, cycles, nit, its, code, True)
    solver.source.copy_(source.reshape(batch, ny, nx))
    solver.target.copy_(target.reshape(batch, ny, nx))
    torch.cuda.synchronize(device)
    started = time.perf_counter()
    side = torch.cuda.Stream(device=device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        solver.launch(_native.stream_handle(side), flows, steps_per_registration)  # warm up outside capture
    torch.cuda.synchronize(device)
    graph = torch.cuda.CUDAGraph()
    before = _native.library().csg_kernel_launches()
    with torch.cuda.graph(graph, stream=side):
        solver.launch(_native.stream_handle(side), flows, steps_per_registration)
    kernels = int(_native.library().csg_kernel_launches() - before)
    torch.cuda.synchronize(device)
    return _GraphEntry(graph=graph, solver=solver, capture_seconds=time.perf_counter() - started, kernels=kernels)


def prepare_dartel_cuda_graph(source_maps, target_maps, *, loop: int = 6, lmreg: float = 1e-3, cycles: int = 3,
                              nit: int = 3, its: int = 3, code: int = 1, kernel: str = "auto",
                              squaring_kernel: str | None = None, device="auto", dtype=torch.float64,
                              optimized: bool = True) -> float:
    """Capture (once) the whole-solve CUDA graph for these shapes (reference 169-224)."""

    dev = resolve_device(device)
    source = _tensor(source_maps, dev, dtype)
    target = _tensor(target_maps, dev, dtype)
    if tuple(source.shape) != tuple(target.shape):
        raise ValueError("source_maps and target_maps must have the same shape")
    key = _graph_key(source, target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its, code=code,
                     kernel=kernel, squaring_kernel=squaring_kernel, optimized=optimized)
    if key in _GRAPH_CACHE:
        return 0.0
    entry = _capture(source, target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its, code=code, device=dev)
    _GRAPH_CACHE[key] = entry
    return entry.capture_seconds


def clear_dartel_cuda_graph_cache() -> None:
    """Drop every captured DARTEL graph (reference 227-230)."""

    _GRAPH_CACHE.clear()


def solve_dartel_maps(source_maps, target_maps, *, loop: int = 6, lmreg: float = 1e-3, cycles: int = 3, nit: int = 3,
                      its: int = 3, code: int = 1, kernel: str = "auto", squaring_kernel: str | None = None,
                      device="auto", dtype=torch.float64, optimized: bool = True,
                      assume_initial_nonzero: bool = False, cuda_graph: bool = False) -> DartelSolveResult:
    """Solve DARTEL feature maps with the upstream loop semantics (reference 239-367).

    ``metrics`` is ``[steps, loop * its, 3]``; ``flow`` is
    ``expdef(velocity of the last step map, k=10)``.
    """

    if cycles < 0 or nit < 0 or its < 0:
        raise ValueError("cycles, nit, and its must be non-negative")
    if squaring_kernel not in {None, "auto", "torch", "triton"}:
        raise ValueError("squaring_kernel must be None, 'auto', 'torch', or 'triton'")
    dev = resolve_device(device)
    source = _tensor(source_maps, dev, dtype)
    target = _tensor(target_maps, dev, dtype)
    if source.ndim != 3 or target.ndim != 3:
        raise ValueError("source_maps and target_maps must have shape [steps, ny, nx]")
    if tuple(source.shape) != tuple(target.shape):
        raise ValueError("Source_maps target_maps shape must")
    if source.shape[0] < 1:
        raise ValueError("At least one DARTEL step is required")
    if loop <= 0:
        raise ValueError(f"loop must be positive, got {loop}")
    if cuda_graph:
        key = _graph_key(source, target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its, code=code,
                         kernel=kernel, squaring_kernel=squaring_kernel, optimized=optimized)
        entry = _GRAPH_CACHE.get(key)
        if entry is None:
            entry = _capture(source, target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its, code=code,
                             device=dev)
            _GRAPH_CACHE[key] = entry
        entry.solver.source.copy_(source)
        entry.solver.target.copy_(target)
        entry.replay()
        s = entry.solver
        return DartelSolveResult(s.flow.clone(), s.source.clone(), s.target.clone(), s.metrics.clone())
    steps, ny, nx = (int(v) for v in source.shape)
    solver = _Solver(steps, ny, nx, dtype, dev, loop, lmreg, cycles, nit, its, code, assume_initial_nonzero)
    solver.source.copy_(source)
    solver.target.copy_(target)
    solver.launch(_native.stream_handle(like=solver.source))
    return DartelSolveResult(solver.flow, source, target, solver.metrics)


def solve_dartel_batch(source_maps, target_maps, *, loop: int = 6, lmreg: float = 1e-3, cycles: int = 3,
                       nit: int = 3, its: int = 3, code: int = 1, device="auto", dtype=torch.float64):
    """Solve many independent (source, target) sheet pairs in one batched launch sequence.

    ``source_maps`` / ``target_maps`` are ``[batch, ny, nx]``; returns
    ``(flows [batch, 2, ny, nx], velocities, metrics [batch, loop * its, 3])``
    where each flow is ``expdef(velocity, 10)`` of that pair.  Results equal
    one ``solve_dartel_maps`` call per pair (with a single step map).
    """

    dev = resolve_device(device)
    source = _tensor(source_maps, dev, dtype)
    target = _tensor(target_maps, dev, dtype)
    if source.ndim != 3 or tuple(source.shape) != tuple(target.shape):
        raise ValueError("source_maps and target_maps must have the same shape [batch, ny, nx]")
    batch, ny, nx = (int(v) for v in source.shape)
    solver = _Solver(batch, ny, nx, dtype, dev, loop, lmreg, cycles, nit, its, code, True)
    solver.source.copy_(source)
    solver.target.copy_(target)
    solver.launch(_native.stream_handle(like=solver.source), flows="all")
    return solver.flows, solver.velocity, solver.metrics


def solve_dartel_registrations(source_maps, target_maps, *, loop: int = 6, lmreg: float = 1e-3, cycles: int = 3,
                               nit: int = 3, its: int = 3, code: int = 1, device="auto", dtype=torch.float64,
                               assume_initial_nonzero: bool = False, cuda_graph: bool = False):
    """Many SurfWarp registrations' DARTEL solves as ONE batched solve.

    ``source_maps`` / ``target_maps`` are ``[registrations, steps, ny, nx]``
    (the step maps of each registration, as ``solve_dartel_maps`` takes them
    one registration at a time).  All registrations x steps maps go through
    one ``csg_dartel_solve`` launch sequence, then the exponential of each
    registration's last-map velocity.  Returns ``(flows [R, 2, ny, nx],
    metrics [R, steps, loop * its, 3])``; each flow equals
    ``solve_dartel_maps(source_maps[r], target_maps[r], assume_initial_nonzero=...,
    cuda_graph=...).flow``.  With ``cuda_graph`` the whole batched solve is
    captured once per shape and replayed; like the reference's graph path it
    then assumes a nonzero initial update in every multigrid solve.
    """

    dev = resolve_device(device)
    source = _tensor(source_maps, dev, dtype)
    target = _tensor(target_maps, dev, dtype)
    if source.ndim != 4 or tuple(source.shape) != tuple(target.shape):
        raise ValueError("source_maps and target_maps must have the same shape [registrations, steps, ny, nx]")
    if loop <= 0 or cycles < 0 or nit < 0 or its < 0:
        raise ValueError("loop must be positive; cycles, nit and its non-negative")
    regs, steps, ny, nx = (int(v) for v in source.shape)
    if cuda_graph:
        key = ("registrations",) + _graph_key(source, target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit,
                                              its=its, code=code, kernel="native", squaring_kernel=None,
                                              optimized=True)
        entry = _GRAPH_CACHE.get(key)
        if entry is None:
            entry = _capture(source, target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its, code=code,
                             device=dev, flows="registrations", steps_per_registration=steps)
            _GRAPH_CACHE[key] = entry
        entry.solver.source.copy_(source.reshape(regs * steps, ny, nx))
        entry.solver.target.copy_(target.reshape(regs * steps, ny, nx))
        entry.replay()
        solver = entry.solver
        return solver.flows[:regs].clone(), solver.metrics.view(regs, steps, -1, 3).clone()
    solver = _Solver(regs * steps, ny, nx, dtype, dev, loop, lmreg, cycles, nit, its, code,
                     bool(assume_initial_nonzero))
    solver.source.copy_(source.reshape(regs * steps, ny, nx))
    solver.target.copy_(target.reshape(regs * steps, ny, nx))
    solver.launch(_native.stream_handle(like=solver.source), "registrations", steps)
    return solver.flows[:regs], solver.metrics.view(regs, steps, -1, 3)


def _surface_sheets(source_vertices, target_vertices, source_stencil, target_stencil, fwhm, curvtypes, n_steps, dev,
                    dtype, parallel_sides):
    """Curvature sheets [n_steps, ny, nx] of both surfaces (reference 370-470)."""

    if n_steps < 1 or n_steps > len(fwhm) or n_steps > len(curvtypes):
        raise ValueError("n_steps must not exceed the lengths of fwhm and curvtypes")
    src_st = source_stencil.to(dev, geometry_dtype=torch.float32) if hasattr(source_stencil, "from_file") else source_stencil
    tgt_st = target_stencil.to(dev, geometry_dtype=torch.float32) if hasattr(target_stencil, "from_file") else target_stencil
    source = torch.as_tensor(source_vertices, device=dev).to(torch.float32).contiguous()
    target = torch.as_tensor(target_vertices, device=dev).to(torch.float32).contiguous()
    types = tuple(int(item) for item in curvtypes[:n_steps])
    if any(item not in (2, 5) for item in types):
        raise NotImplementedError("The device surface backend supports only upstream curvtype 2 and 5")

    many = n_steps > 1 and all(item == 5 for item in types)

    def build_maps(stencil, mapped, edge_mean):
        if many:
            return features.curvature_type5_to_sheet_many(stencil, mapped, tuple(float(item) for item in fwhm[:n_steps]),
                                                          edge_mean)
        return tuple(stencil.curvature_to_sheet(mapped, float(fwhm[i]), curvtype=types[i]) for i in range(n_steps))

    mapped = [src_st.resample_vertices(source), tgt_st.resample_vertices(target)]
    # the heat kernels' iteration counts come from each side's mean edge length: both read back at once
    means = features.edge_means([(src_st, mapped[0]), (tgt_st, mapped[1])]) if many else [None, None]
    # ``parallel_sides`` (the reference's two-stream option) is accepted; both sides run on the
    # current stream, which measured faster for these few-microsecond launches on a 61k hull
    # (0.67 vs 0.80 ms median, 0.77 vs 2.5 ms p99 for both sides' sheets) with identical sheets
    source_maps = build_maps(src_st, mapped[0], means[0])
    target_maps = build_maps(tgt_st, mapped[1], means[1])
    return (torch.stack(source_maps, dim=0).to(dtype=dtype).contiguous(),
            torch.stack(target_maps, dim=0).to(dtype=dtype).contiguous())


def solve_dartel_from_surfaces(source_vertices, target_vertices, source_stencil, target_stencil, *,
                               fwhm: Sequence[float] = (5.0, 5.0 / 3.0, 5.0 / 9.0), curvtypes: Sequence[int] = (5, 5, 2),
                               loop: int = 6, n_steps: int = 2, lmreg: float = 1e-3, cycles: int = 3, nit: int = 3,
                               its: int = 3, code: int = 1, kernel: str = "auto", squaring_kernel: str | None = None,
                               device="auto", dtype=torch.float64, parallel_sides: bool = True, optimized: bool = True,
                               assume_initial_nonzero: bool = False, cuda_graph: bool = False) -> DartelSolveResult:
    """Curvature sheets of both surfaces, then their DARTEL solve (reference 370-488)."""

    if squaring_kernel not in {None, "auto", "torch", "triton"}:
        raise ValueError("squaring_kernel must be None, 'auto', 'torch', or 'triton'")
    dev = resolve_device(device)
    stacked_source, stacked_target = _surface_sheets(source_vertices, target_vertices, source_stencil, target_stencil,
                                                     fwhm, curvtypes, n_steps, dev, dtype, parallel_sides)
    return solve_dartel_maps(stacked_source, stacked_target, loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its,
                             code=code, kernel=kernel, squaring_kernel=squaring_kernel, device=dev, dtype=dtype,
                             optimized=optimized, assume_initial_nonzero=assume_initial_nonzero, cuda_graph=cuda_graph)


def solve_dartel_from_surfaces_many(problems, *, curvtypes: Sequence[int] = (5, 5, 2), loop: int = 6,
                                    n_steps: int = 2, lmreg: float = 1e-3, cycles: int = 3, nit: int = 3, its: int = 3,
                                    code: int = 1, device="auto", dtype=torch.float64, parallel_sides: bool = True,
                                    assume_initial_nonzero: bool = False, cuda_graph: bool = False) -> list:
    """Several independent surface registrations as ONE batched DARTEL solve.

    ``problems`` holds ``(source_vertices, target_vertices, source_stencil,
    target_stencil, fwhm)`` per registration (sheets of one size).  Returns
    the flows ``[2, ny, nx]`` in order; each equals
    ``solve_dartel_from_surfaces(...).flow`` of that registration with the
    same ``assume_initial_nonzero`` / ``cuda_graph``.
    """

    dev = resolve_device(device)
    sheets = [_surface_sheets(sv, tv, ss, ts, f, curvtypes, n_steps, dev, dtype, parallel_sides)
              for sv, tv, ss, ts, f in problems]
    if len({tuple(src.shape) for src, _ in sheets}) != 1:
        raise ValueError("batched registrations need sheets of one size")
    flows, _ = solve_dartel_registrations(torch.stack([src for src, _ in sheets]), torch.stack([tgt for _, tgt in sheets]),
                                          loop=loop, lmreg=lmreg, cycles=cycles, nit=nit, its=its, code=code,
                                          device=dev, dtype=dtype, assume_initial_nonzero=assume_initial_nonzero,
                                          cuda_graph=cuda_graph)
    return [flows[r] for r in range(len(problems))]


def apply_flow_to_sphere(sphere_vertices, flow, *, unit_sphere_vertices=None, inverse: bool = True, device="auto",
                         dtype=torch.float64) -> torch.Tensor:
    """Warp sphere points by a solved flow (reference 500-584)."""

    dev = resolve_device(device)
    sphere = torch.as_tensor(sphere_vertices, device=dev)
    deformation = _tensor(flow, dev, dtype)
    if sphere.ndim != 2 or sphere.shape[1] != 3:
        raise ValueError("sphere_vertices must have shape [points, 3]")
    if deformation.ndim != 3 or deformation.shape[0] != 2:
        raise ValueError("flow must have shape [2, ny, nx]")
    if unit_sphere_vertices is None:
        points = sphere.to(torch.float32)
        points = points / torch.linalg.vector_norm(points, dim=-1, keepdim=True).clamp_min(torch.finfo(torch.float32).eps)
    else:
        points = torch.as_tensor(unit_sphere_vertices, device=dev, dtype=torch.float32)
        if points.shape != sphere.shape:
            raise ValueError("unit_sphere_vertices must match sphere_vertices shape")
    points = points.contiguous()
    out = torch.empty((points.shape[0], 3), dtype=dtype, device=dev)
    lib = _native.library()
    _native.check(
        lib.csg_apply_flow_to_sphere(_dtype_code(dtype), int(points.shape[0]), points.data_ptr(),
                                     int(deformation.shape[2]), int(deformation.shape[1]), deformation.data_ptr(),
                                     int(bool(inverse)), out.data_ptr(),
                                     _native.stream_handle(like=out)),
        "csg_apply_flow_to_sphere",
    )
    return out


def apply_flow_to_stenciled_sphere(sphere_vertices, flow, stencil, *, inverse: bool = True, device="auto",
                                   dtype=torch.float64) -> torch.Tensor:
    """apply_flow_to_sphere with the stencil's unit-sphere points (reference 587-617)."""

    dev = resolve_device(device)
    device_stencil = stencil.to(dev, geometry_dtype=torch.float32) if hasattr(stencil, "from_file") else stencil
    if device_stencil.unit_sphere_points is None:
        raise ValueError("stencil does not contain unit-sphere points required by apply_warp")
    return apply_flow_to_sphere(sphere_vertices, flow, unit_sphere_vertices=device_stencil.unit_sphere_points,
                                inverse=inverse, device=dev, dtype=dtype)


def average_xz_surfaces(x_surface, z_surface, *, device="auto") -> torch.Tensor:
    """-avg blend of the x- and z-pole solutions (reference gpu_pipeline.py:248-271)."""

    dev = resolve_device(device)
    xv = torch.as_tensor(x_surface, dtype=torch.float64, device=dev).contiguous()
    zv = torch.as_tensor(z_surface, dtype=torch.float64, device=dev).contiguous()
    if xv.shape != zv.shape or xv.ndim != 2 or xv.shape[1] != 3:
        raise ValueError("Both sphere arrays must have shape [points, 3]")
    out = torch.empty(xv.shape, dtype=torch.float32, device=dev)
    _native.check(
        _native.library().csg_average_xz(int(xv.shape[0]), xv.data_ptr(), zv.data_ptr(), out.data_ptr(),
                                         _native.stream_handle(like=out)),
        "csg_average_xz",
    )
    return out
