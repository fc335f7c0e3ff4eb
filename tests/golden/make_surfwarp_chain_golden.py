"""Generate an end-to-end SurfWarp golden by running the reference package on CPU.

Development container only (imports ``cat_surface_gpu`` from the reference
checkout).  Follows ``src/cat_surface_gpu/gpu_pipeline.py:468-1326`` step by
step with the reference's own operators on the CPU: stencils written by the
reference's own helper (``bin/linux-x86_64/cat_surface_stencil_builder``,
executed; read back through the reference's reader -- the helper's sheet is
fixed at 512 x 256, so for other sheet sizes the sheet part is the oracle's
restatement of the helper's sheet, ``oracle/stencil.py``, pinned to the helper
by ``tests/test_stencil_helper.py``),
rotation features (the reference's default "cuda" backend:
``compute_rotation_features`` -- the depth potential by coloured SOR of the
smoothed coarse surfaces at FWHM 15 / 10 -- run on the CPU), the 46-seed +
Nelder-Mead rotation search, ``runs`` DARTEL solves with the inverse warp between runs, the
pole-rotated ``-avg`` solve and the blend.

Inputs: two folded icospheres (10,242 vertices, subdivision 5) with shared
folding plus a per-subject perturbation; the source sphere is the unit
icosphere under a known rotation, scaled to radius 100.  Writes
``surfwarp_chain_golden.npz`` (inputs, parameters, rotation features, the
type-5 curvature features of this package's "native-curvature" option,
rotation angle/cost, the rotated sphere, the sphere after run 0, the final
sphere; and both feature kinds recomputed by the reference on this package's
own stencils of the two spheres, ``builder_*``).

``--workload hemisphere`` instead runs the 61,442-vertex hemisphere chain of
the benchmark: source = the ``surf2sphere_c2`` surface with the upstream
binary's sphere, target = the ``surf2sphere_c3`` surface and sphere, two runs
of two steps on a 256 x 128 sheet with ``-avg``; it writes
``surfwarp_chain_hemisphere_golden.npz`` (parameters, rotation angle/cost, the
number of rotation candidates the search evaluated, the final sphere and the
CPU wall time of the chain), plus the same chain run on this package's host
stencil builder instead of the helper (``builder_rotation_angle``,
``builder_final_sphere``).

Usage: ``python tests/golden/make_surfwarp_chain_golden.py [--workload small|hemisphere]``
"""

from __future__ import annotations

import argparse
import dataclasses
import os
from pathlib import Path
import subprocess
import sys
import tempfile
import time

import numpy as np

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))
from _reference import reference_binary, use_reference_package  # noqa: E402

use_reference_package()
HELPER = reference_binary("cat_surface_stencil_builder")

import torch  # noqa: E402

from cat_surface_gpu.gpu_pipeline import (  # noqa: E402
    _average_xz_surfaces, _normalise_sphere, _rotate_vertices, _rotation_matrix_from_angles)
from cat_surface_gpu.rotation_feature import compute_rotation_features  # noqa: E402
from cat_surface_gpu.rotation_pipeline import RotationPipeline  # noqa: E402
from cat_surface_gpu.surface_stencil import SurfaceStencil as ReferenceStencil  # noqa: E402
from cat_surface_gpu.surface_warp import apply_flow_to_stenciled_sphere, solve_dartel_from_surfaces  # noqa: E402

from cat_surface_gpu_b200 import synthetic  # noqa: E402
from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh  # noqa: E402
from cat_surface_gpu_b200.surface_stencil import SurfaceStencil  # noqa: E402
from oracle import stencil as oracle_stencil  # noqa: E402

PARAMS = dict(nx=128, ny=64, steps=2, runs=2, avg=True, loop=6, rotation_grid_size=128)
CPU = torch.device("cpu")


def chain_inputs(seed: int = 5):
    """Source/target surfaces and spheres on one 10,242-vertex icosphere topology."""

    rng = np.random.default_rng(seed)
    points, faces = synthetic.unit_icosphere(5)
    shared = synthetic.real_sph_harm_sum(points, range(3, 15), 0.08, rng)
    target_r = 1.0 + shared + synthetic.real_sph_harm_sum(points, range(3, 10), 0.02, rng)
    source_r = 1.0 + shared + synthetic.real_sph_harm_sum(points, range(3, 10), 0.02, rng)
    angle = np.array([0.12, -0.08, 0.18])
    c, s = np.cos(angle), np.sin(angle)
    rx = np.array([[1, 0, 0], [0, c[0], -s[0]], [0, s[0], c[0]]])
    ry = np.array([[c[1], 0, s[1]], [0, 1, 0], [-s[1], 0, c[1]]])
    rz = np.array([[c[2], -s[2], 0], [s[2], c[2], 0], [0, 0, 1]])
    rotated = points @ (rz @ ry @ rx).T
    jitter = rng.normal(scale=2e-3, size=points.shape)
    return dict(
        faces=faces.astype(np.int32),
        source_surface=(points * (60.0 * source_r)[:, None]).astype(np.float32),
        target_surface=(points * (60.0 * target_r)[:, None]).astype(np.float32),
        source_sphere=(100.0 * (rotated + jitter)).astype(np.float32),
        target_sphere=(100.0 * (points + rng.normal(scale=2e-3, size=points.shape))).astype(np.float32),
    )


def reference_chain(data, nx, ny, steps, runs, avg, loop, rotation_grid_size, target_faces=None, stencils="helper"):
    source_faces = data["faces"]
    target_faces = source_faces if target_faces is None else target_faces
    temp = Path(tempfile.mkdtemp(prefix="chain_golden_"))
    count = [0]

    def stencil(sphere, normalize, faces=None):
        """The helper's stencil of this sphere (the reference pipeline's call, gpu_pipeline.py:144-166)."""

        count[0] += 1
        mesh_path, path = temp / f"s{count[0]}.gii", temp / f"s{count[0]}.stencil"
        faces = source_faces if faces is None else faces
        if stencils == "builder":  # this package's host builder, read back through the reference's reader
            from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

            build_surface_stencil(np.asarray(sphere, dtype=np.float32), np.asarray(faces, dtype=np.int32), nx=nx,
                                  ny=ny, normalize=normalize, threads=8).to_file(path)
            return ReferenceStencil.from_file(path)
        write_gifti_mesh(mesh_path, GiftiMesh(np.asarray(sphere, dtype=np.float32), faces))
        command = [str(HELPER), str(mesh_path), str(path), "--threads", "8"]
        if not normalize:
            command.insert(3, "--no-normalize")
        subprocess.run(command, check=True, capture_output=True)
        if (nx, ny) != (512, 256):
            written = SurfaceStencil.from_file(path)
            sheet_indices, sheet_weights = oracle_stencil.sheet_stencil(written.sphere_points, written.faces, nx, ny)
            dataclasses.replace(written, sheet_indices=sheet_indices, sheet_weights=sheet_weights, nx=nx,
                                ny=ny).to_file(path)
        return ReferenceStencil.from_file(path)

    def on_cpu(st):
        return st.to(CPU, geometry_dtype=torch.float32)

    source_stencil = stencil(data["source_sphere"], True)
    target_stencil = stencil(data["target_sphere"], True, target_faces)
    curvature = []
    for st, surface, fwhm in ((source_stencil, data["source_surface"], 15.0),
                              (target_stencil, data["target_surface"], 10.0)):
        dev = on_cpu(st)
        mapped = dev.resample_vertices(torch.as_tensor(surface))
        curvature.append(dev.curvature_type5(mapped, fwhm).numpy())
    features = compute_rotation_features(
        (on_cpu(source_stencil), on_cpu(target_stencil)),
        (torch.as_tensor(data["source_surface"]), torch.as_tensor(data["target_surface"])), heat_fwhms=(15.0, 10.0),
        solver="colored-sor")
    values = [f.values.numpy() for f in features]
    pipeline = RotationPipeline.from_stencil(target_stencil, device=CPU, grid_size=rotation_grid_size, margin=1)
    evaluated = [0]
    plain_cost = pipeline.index.cost_batch_prepared

    def counting_cost(inputs, angles, **kwargs):
        evaluated[0] += int(torch.as_tensor(angles).reshape(-1, 3).shape[0])
        return plain_cost(inputs, angles, **kwargs)

    pipeline.index.cost_batch_prepared = counting_cost
    rotation = pipeline.search(source_stencil.sphere_points, values[0], values[1], point_chunk=4096)
    angle = rotation.angle.detach().cpu().numpy()
    current_sphere = _rotate_vertices(_normalise_sphere(data["source_sphere"]), angle)
    rotated_initial = current_sphere.copy()
    pole = np.asarray((0.0, np.pi / 2.0, 0.0), dtype=np.float64)
    avg_target_surface = _rotate_vertices(data["target_surface"], pole)
    avg_target_sphere = _rotate_vertices(_normalise_sphere(data["target_sphere"]), pole)
    current_dev = on_cpu(stencil(current_sphere, False))
    target_dev = on_cpu(target_stencil)
    source_surface = torch.as_tensor(data["source_surface"])
    target_surface = torch.as_tensor(data["target_surface"])

    def solve(src, tgt, src_st, tgt_st, fwhm):
        return solve_dartel_from_surfaces(src, tgt, src_st, tgt_st, fwhm=fwhm, curvtypes=(5, 5, 2), n_steps=steps,
                                          loop=loop, kernel="torch", device=CPU, dtype=torch.float64,
                                          parallel_sides=False)

    after_run0 = None
    final_prewarp = avg_source_sphere = avg_source_surface = avg_source_dev = None
    last = None
    for run_index in range(runs):
        run_fwhm = tuple(5.0 / (3.0 ** (steps * (run_index + 1) + i)) for i in range(steps))
        if avg and run_index == runs - 1:
            final_prewarp = current_sphere.copy()
            avg_source_surface = _rotate_vertices(data["source_surface"], pole)
            avg_source_sphere = _rotate_vertices(final_prewarp, pole)
            avg_source_dev = on_cpu(stencil(avg_source_sphere, False))
        last = solve(source_surface, target_surface, current_dev, target_dev, run_fwhm)
        if not (avg and run_index == runs - 1):
            current_sphere = apply_flow_to_stenciled_sphere(torch.as_tensor(current_sphere), last.flow, current_dev,
                                                            inverse=True, device=CPU,
                                                            dtype=torch.float64).numpy().astype(np.float32)
        if run_index == 0:
            after_run0 = current_sphere.copy()
        if run_index + 1 < runs:
            current_dev = on_cpu(stencil(current_sphere, False))
    if avg:
        avg_fwhm = tuple(5.0 / (3.0 ** (steps * (runs + 1) + i)) for i in range(steps))
        avg_result = solve(torch.as_tensor(avg_source_surface), torch.as_tensor(avg_target_surface), avg_source_dev,
                           on_cpu(stencil(avg_target_sphere, False, target_faces)), avg_fwhm)
        main_warped = apply_flow_to_stenciled_sphere(torch.as_tensor(final_prewarp), last.flow, current_dev,
                                                     inverse=True, device=CPU, dtype=torch.float64)
        avg_warped = apply_flow_to_stenciled_sphere(torch.as_tensor(avg_source_sphere), avg_result.flow,
                                                    avg_source_dev, inverse=True, device=CPU, dtype=torch.float64)
        reverse = _rotation_matrix_from_angles(-pole)
        unrotated = avg_warped.to(torch.float64) @ reverse.transpose(0, 1)
        current_sphere = _average_xz_surfaces(unrotated, main_warped, device=CPU).numpy().astype(np.float32)
    return dict(rotation_angle=angle.astype(np.float64), rotation_cost=float(rotation.cost),
                rotation_candidates_evaluated=np.int64(evaluated[0]),
                source_values=values[0], target_values=values[1], curv_source_values=curvature[0],
                curv_target_values=curvature[1],
                rotated_initial=rotated_initial, after_run0=after_run0, final_sphere=current_sphere)


def builder_features(data, nx, ny):
    """The reference's rotation and curvature features on this package's own stencils of the two spheres.

    Pins the feature operators on identical inputs (the chain itself uses the
    helper's stencils, which this package's builder matches to the helper's
    float32 rounding only).
    """

    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    temp = Path(tempfile.mkdtemp(prefix="chain_builder_"))
    stencils = []
    for side in ("source", "target"):
        build_surface_stencil(data[f"{side}_sphere"], data["faces"], nx=nx, ny=ny, normalize=True).to_file(
            temp / f"{side}.stencil")
        stencils.append(ReferenceStencil.from_file(temp / f"{side}.stencil").to(CPU, geometry_dtype=torch.float32))
    surfaces = (torch.as_tensor(data["source_surface"]), torch.as_tensor(data["target_surface"]))
    features = compute_rotation_features(tuple(stencils), surfaces, heat_fwhms=(15.0, 10.0), solver="colored-sor")
    curvature = [st.curvature_type5(st.resample_vertices(surface), fwhm).numpy()
                 for st, surface, fwhm in zip(stencils, surfaces, (15.0, 10.0))]
    return dict(builder_source_values=features[0].values.numpy(), builder_target_values=features[1].values.numpy(),
                builder_curv_source_values=curvature[0], builder_curv_target_values=curvature[1])


HEMISPHERE_PARAMS = dict(nx=256, ny=128, steps=2, runs=2, avg=True, loop=6, rotation_grid_size=128)


def hemisphere_inputs():
    """The benchmark's hemisphere pair: c2 (source) and c3 (target) with the upstream binary's spheres."""

    return np.load(HERE / "surf2sphere_c2.npz"), np.load(HERE / "surf2sphere_c3.npz")


def reference_hemisphere_chain():
    source, target = hemisphere_inputs()
    data = dict(faces=source["faces"].astype(np.int32), source_surface=source["surface"],
                source_sphere=source["final"], target_surface=target["surface"], target_sphere=target["final"])
    return data, target["faces"].astype(np.int32)


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--workload", choices=("small", "hemisphere"), default="small")
    args = parser.parse_args()
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    if args.workload == "small":
        data = chain_inputs()
        started = time.perf_counter()
        result = reference_chain(data, **PARAMS)
        seconds = time.perf_counter() - started
        result.update(builder_features(data, PARAMS["nx"], PARAMS["ny"]))
        np.savez_compressed(HERE / "surfwarp_chain_golden.npz", **data, **result,
                            **{f"param_{k}": np.asarray(v) for k, v in PARAMS.items()})
    else:
        data, target_faces = reference_hemisphere_chain()
        started = time.perf_counter()
        result = reference_chain(data, target_faces=target_faces, **HEMISPHERE_PARAMS)
        seconds = time.perf_counter() - started
        keep = ("rotation_angle", "rotation_cost", "rotation_candidates_evaluated", "final_sphere")
        # the same chain on this package's stencils: separates the chain's arithmetic from its
        # sensitivity to the helper's float32 stencil rounding
        builder = reference_chain(data, target_faces=target_faces, stencils="builder", **HEMISPHERE_PARAMS)
        np.savez_compressed(HERE / "surfwarp_chain_hemisphere_golden.npz", **{k: result[k] for k in keep},
                            **{f"builder_{k}": builder[k] for k in ("rotation_angle", "final_sphere")},
                            cpu_seconds=np.float64(seconds), cpu_threads=np.int64(torch.get_num_threads()),
                            **{f"param_{k}": np.asarray(v) for k, v in HEMISPHERE_PARAMS.items()})
    print(f"reference chain on CPU ({args.workload}): {seconds:.1f} s, angle {result['rotation_angle']}, "
          f"cost {result['rotation_cost']:.6f}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
