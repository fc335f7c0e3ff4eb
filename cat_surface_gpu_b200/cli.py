"""Command-line entry points with the reference's names and options.

``cat-surf2sphere-gpu`` -> :func:`surf2sphere_main`,
``cat-surfwarp-gpu`` -> :func:`surfwarp_main`,
``cat-surface-rotation-gpu`` -> :func:`rotation_main`
(reference ``src/cat_surface_gpu/cli.py:35-332``).  Each prints a timings
JSON like the reference.  ``python -m cat_surface_gpu_b200.cli <command> ...``
runs the same functions.
"""

from __future__ import annotations

import argparse
import hashlib
import json
from pathlib import Path
import sys
import time

import numpy as np
import torch


def _synchronize(device: torch.device) -> None:
    if device.type == "cuda":
        torch.cuda.synchronize(device)


def surf2sphere_main(argv: list[str] | None = None) -> int:
    """Stages 1-5, the area-smoothing sweeps and the ellipsoid steps on the GPU (reference 35-94).

    The reference's options are all parsed.  ``--preprocess-kernel cpu`` (the
    reference ran stages 1-5 on its CPU binary) is rejected with a usage
    error; ``--reference-cli`` is accepted and not used.
    """

    from .surf2sphere import run_cat_surf2sphere_gpu

    parser = argparse.ArgumentParser(description="Run strict CAT_Surf2Sphere area smoothing on CUDA.")
    parser.add_argument("--reference-cli", type=Path,
                        help="accepted for compatibility; not used (no CPU stage is run)")
    parser.add_argument("--input-surface", type=Path, required=True)
    parser.add_argument("--output-surface", type=Path, required=True)
    parser.add_argument("--stop-at", type=int, default=10)
    parser.add_argument("--device", default="cuda")
    parser.add_argument("--dtype", choices=("float32", "float64"), default="float32")
    parser.add_argument("--kernel", choices=("torch", "triton"), default="triton")
    parser.add_argument("--preprocess-kernel", choices=("cpu", "triton"), default="triton",
                        help="triton (default): stages 1-5 on the GPU; cpu is not supported")
    parser.add_argument("--preprocess-block-size", type=int, default=131072)
    parser.add_argument("--areal-block-size", type=int)
    parser.add_argument("--areal-schedule", choices=("ordered", "color"), default="ordered")
    parser.add_argument("--areal-arithmetic", choices=("cat", "fp32"), default="cat")
    args = parser.parse_args(argv)
    if args.preprocess_kernel == "cpu":
        parser.error("--preprocess-kernel cpu ran stages 1-5 on the upstream CPU binary; this package runs them on "
                     "the GPU (--preprocess-kernel triton, the default)")
    result = run_cat_surf2sphere_gpu(
        args.input_surface, args.output_surface, stop_at=args.stop_at,
        device=args.device, dtype=args.dtype, kernel=args.kernel, preprocess_kernel=args.preprocess_kernel,
        preprocess_block_size=args.preprocess_block_size, areal_schedule=args.areal_schedule,
        areal_arithmetic=args.areal_arithmetic, areal_block_size=args.areal_block_size,
    )
    print(json.dumps({
        "backend": f"surf2sphere_pre_{args.preprocess_kernel}_{args.areal_schedule}_wavefront_sm100a",
        "device": args.device, "dtype": args.dtype, "areal_arithmetic": args.areal_arithmetic,
        "stop_at": args.stop_at, "output_surface": str(result.output_path),
        "timings": result.timings,
    }, ensure_ascii=False, indent=2))
    return 0


def surfwarp_main(argv: list[str] | None = None) -> int:
    """CAT_SurfWarp-compatible registration (reference 97-252)."""

    from .gpu_pipeline import run_cat_surface_gpu_pipeline

    parser = argparse.ArgumentParser(description="Run CAT_SurfWarp-compatible registration with native DARTEL.")
    parser.add_argument("--source-surface", type=Path, required=True)
    parser.add_argument("--source-sphere", type=Path, required=True)
    parser.add_argument("--target-surface", type=Path, required=True)
    parser.add_argument("--target-sphere", type=Path, required=True)
    parser.add_argument("--output", type=Path, required=True)
    parser.add_argument("--source-stencil", type=Path)
    parser.add_argument("--target-stencil", type=Path)
    parser.add_argument("--rotation-values", type=Path)
    parser.add_argument("--rotation-values-probe", type=Path)
    parser.add_argument("--rotation-geometry-probe", type=Path)
    parser.add_argument("--rotation-depth-probe", type=Path)
    parser.add_argument("--rotation-feature-backend", default="auto",
                        choices=("auto", "native-curvature", "cuda", "cuda-official-geometry", "cuda-official-depth",
                                 "official-cpu"))
    parser.add_argument("--rotation-feature-solver", choices=("colored-sor", "pcg"), default="colored-sor")
    parser.add_argument("--stencil-builder", default="native",
                        help="'native' (default, the GPU builder); a path to the reference's helper is rejected")
    parser.add_argument("--rotated-stencil-builder")
    parser.add_argument("--stencil-threads", type=int, default=8)
    parser.add_argument("--sheet-size", type=int, nargs=2, default=(512, 256), metavar=("NX", "NY"))
    parser.add_argument("--device", default="cuda")
    parser.add_argument("--kernel", default="triton")
    parser.add_argument("--dartel-dtype", choices=("float64", "float32"), default="float64")
    parser.add_argument("--squaring-kernel", choices=("auto", "torch", "triton"), default="triton")
    parser.add_argument("--steps", type=int, default=2)
    parser.add_argument("--runs", type=int, default=2)
    parser.add_argument("--avg", action=argparse.BooleanOptionalAction, default=True)
    parser.add_argument("--loop", type=int, default=6)
    parser.add_argument("--cycles", type=int, default=3)
    parser.add_argument("--nit", type=int, default=3)
    parser.add_argument("--its", type=int, default=3)
    parser.add_argument("--code", type=int, default=1)
    parser.add_argument("--parallel-sides", action=argparse.BooleanOptionalAction, default=True)
    parser.add_argument("--optimized-dartel", action=argparse.BooleanOptionalAction, default=True)
    parser.add_argument("--cuda-graph", action=argparse.BooleanOptionalAction, default=True)
    parser.add_argument("--point-chunk", type=int, default=4096)
    parser.add_argument("--rotation-grid-size", type=int, default=128)
    parser.add_argument("--rotation-margin", type=int, default=1)
    parser.add_argument("--no-rotation-refine", action="store_true")
    parser.add_argument("--rotation-max-iter", type=int, default=500)
    parser.add_argument("--rotation-tol", type=float, default=1.0e-4)
    parser.add_argument("--rotation-simplex-step", type=float, default=0.1)
    parser.add_argument("--rotation-search", choices=("nelder-mead", "euler-grid"), default="nelder-mead",
                        help="nelder-mead: the reference's 46 seeds + Nelder-Mead; euler-grid: 10 then 2 degree "
                             "Euler grids on z-scored curvature and depth")
    args = parser.parse_args(argv)
    result = run_cat_surface_gpu_pipeline(
        args.source_surface, args.source_sphere, args.target_surface, args.target_sphere, args.output,
        source_stencil_path=args.source_stencil, target_stencil_path=args.target_stencil,
        rotation_values_path=args.rotation_values, rotation_values_probe=args.rotation_values_probe,
        rotation_geometry_probe=args.rotation_geometry_probe, rotation_depth_probe=args.rotation_depth_probe,
        rotation_feature_backend=args.rotation_feature_backend, rotation_feature_solver=args.rotation_feature_solver,
        stencil_builder=args.stencil_builder, rotated_stencil_builder=args.rotated_stencil_builder,
        stencil_threads=args.stencil_threads, device=args.device, kernel=args.kernel, dartel_dtype=args.dartel_dtype,
        squaring_kernel=args.squaring_kernel, steps=args.steps, runs=args.runs, avg=args.avg, loop=args.loop,
        cycles=args.cycles, nit=args.nit, its=args.its, code=args.code, point_chunk=args.point_chunk,
        rotation_grid_size=args.rotation_grid_size, rotation_margin=args.rotation_margin,
        rotation_refine=not args.no_rotation_refine, rotation_max_iter=args.rotation_max_iter,
        rotation_tol=args.rotation_tol, rotation_simplex_step=args.rotation_simplex_step,
        parallel_sides=args.parallel_sides, optimized_dartel=args.optimized_dartel, cuda_graph=args.cuda_graph,
        sheet_size=tuple(args.sheet_size), rotation_search=args.rotation_search,
    )
    device = torch.device(args.device)
    print(json.dumps({
        "backend": "native_sm100a_cat_surface_pipeline", "device": str(device),
        "device_name": torch.cuda.get_device_name(device) if device.type == "cuda" else "CPU",
        "torch": torch.__version__, "steps": args.steps, "runs": args.runs, "avg": args.avg,
        "source_shape": list(result.vertices.shape), "faces_shape": list(result.faces.shape),
        "rotation_angle": result.rotation_angle.tolist(), "rotation_cost": result.rotation_cost,
        "timings": result.timings, "output": str(result.output_path),
    }, ensure_ascii=False, indent=2))
    return 0


def rotation_main(argv: list[str] | None = None) -> int:
    """CAT-compatible initial-rotation search on prepared inputs (reference 255-332)."""

    from .device import resolve_device
    from .rotation_pipeline import RotationPipeline, read_rotation_points, read_rotation_values
    from .surface_stencil import SurfaceStencil

    parser = argparse.ArgumentParser(description="Run CAT initial-rotation search.")
    parser.add_argument("--source-points", type=Path, required=True)
    parser.add_argument("--target-stencil", type=Path, required=True)
    parser.add_argument("--rotation-values", type=Path, required=True)
    parser.add_argument("--device", default="auto")
    parser.add_argument("--grid-size", type=int, default=128)
    parser.add_argument("--margin", type=int, default=1)
    parser.add_argument("--point-chunk", type=int, default=4096)
    parser.add_argument("--candidate-table-dtype", choices=("int32", "int64"), default="int32")
    parser.add_argument("--no-refine", action="store_true")
    parser.add_argument("--max-iter", type=int, default=500)
    parser.add_argument("--tol", type=float, default=1.0e-4)
    parser.add_argument("--simplex-step", type=float, default=0.1)
    args = parser.parse_args(argv)
    device = resolve_device(args.device)
    source_points = read_rotation_points(args.source_points)
    source_values, target_values = read_rotation_values(args.rotation_values)
    target_stencil = SurfaceStencil.from_file(args.target_stencil)
    started = time.perf_counter()
    pipeline = RotationPipeline.from_stencil(target_stencil, device=device, grid_size=args.grid_size,
                                             margin=args.margin)
    _synchronize(device)
    build_upload = time.perf_counter() - started
    started = time.perf_counter()
    result = pipeline.search(source_points, source_values, target_values, point_chunk=args.point_chunk,
                             refine=not args.no_refine, max_iter=args.max_iter, tol=args.tol,
                             simplex_step=args.simplex_step)
    _synchronize(device)
    seed_costs = result.seed_costs.detach().cpu().numpy()
    print(json.dumps({
        "feature_backend": "c_probe_rotation_values", "cost_backend": "native_sm100a", "device": str(device),
        "device_name": torch.cuda.get_device_name(device), "source_points": int(source_points.shape[0]),
        "target_points": int(target_stencil.sphere_points.shape[0]), "build_upload_seconds": build_upload,
        "search_seconds": time.perf_counter() - started,
        "seed_cost_sha256": hashlib.sha256(np.ascontiguousarray(seed_costs).tobytes()).hexdigest(),
        "angle": result.angle.detach().cpu().tolist(), "cost": float(result.cost.detach().cpu()),
        "rotation_matrix": result.rotation_matrix.detach().cpu().tolist(), "iterations": result.iterations,
    }, ensure_ascii=False, indent=2))
    return 0


COMMANDS = {"surf2sphere": surf2sphere_main, "surfwarp": surfwarp_main, "rotation": rotation_main}


def main(argv: list[str] | None = None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] not in COMMANDS:
        print(f"usage: python -m cat_surface_gpu_b200.cli {{{','.join(COMMANDS)}}} ...", file=sys.stderr)
        return 2
    return COMMANDS[argv[0]](argv[1:])


if __name__ == "__main__":
    raise SystemExit(main())
