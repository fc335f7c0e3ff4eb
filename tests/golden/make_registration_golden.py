"""Generate the batched-registration golden by running the reference package on CPU.

Development checkout only.  The batched registration workload registers
subjects ``synthetic.registration_subjects()`` (folded hulls of 40,962 to
163,842 vertices with their spherical parametrisation) to the
61,442-vertex hull ``surf2sphere_c3`` with its upstream sphere: the
subject's sphere normalised (the reference's ``_normalise_sphere``), the
stencils of both spheres, one DARTEL run of two steps on a 256 x 128 sheet
in float64 (FWHM 5/9 and 5/27, curvature types 5 and 5), and the inverse
warp of the subject's sphere.  This script runs that registration with the
reference's own CPU functions -- stencils from the reference's helper
(executed; the 256 x 128 sheet from the oracle's restatement of the
helper's sheet), ``solve_dartel_from_surfaces`` and
``apply_flow_to_stenciled_sphere`` -- for the two smallest subjects and
stores their warped spheres.  Writes ``registration_golden.npz``.

Usage: ``python tests/golden/make_registration_golden.py``
"""

from __future__ import annotations

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

from cat_surface_gpu.gpu_pipeline import _normalise_sphere  # noqa: E402
from cat_surface_gpu.surface_stencil import SurfaceStencil as ReferenceStencil  # noqa: E402
from cat_surface_gpu.surface_warp import apply_flow_to_stenciled_sphere, solve_dartel_from_surfaces  # noqa: E402

from cat_surface_gpu_b200 import synthetic  # noqa: E402
from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh  # noqa: E402
from cat_surface_gpu_b200.surface_stencil import SurfaceStencil  # noqa: E402
from oracle import stencil as oracle_stencil  # noqa: E402

NX, NY, STEPS, LOOP = 256, 128, 2, 6
FWHM = tuple(5.0 / (3.0 ** (STEPS + i)) for i in range(STEPS))
CPU = torch.device("cpu")


def helper_stencil(sphere, faces, normalize, temp: Path, name: str):
    mesh, path = temp / f"{name}.gii", temp / f"{name}.stencil"
    write_gifti_mesh(mesh, GiftiMesh(np.asarray(sphere, dtype=np.float32), faces))
    command = [str(HELPER), str(mesh), str(path), "--threads", "8"]
    if not normalize:
        command.insert(3, "--no-normalize")
    subprocess.run(command, check=True, capture_output=True)
    written = SurfaceStencil.from_file(path)
    sheet_indices, sheet_weights = oracle_stencil.sheet_stencil(written.sphere_points, written.faces, NX, NY)
    dataclasses.replace(written, sheet_indices=sheet_indices, sheet_weights=sheet_weights, nx=NX, ny=NY).to_file(path)
    return ReferenceStencil.from_file(path).to(CPU, geometry_dtype=torch.float32)


def main() -> int:
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    target = np.load(HERE / "surf2sphere_c3.npz")
    subjects = synthetic.registration_subjects()[:2]
    out = {"subjects": np.array(subjects, dtype=np.int64)}
    with tempfile.TemporaryDirectory(prefix="registration_golden_") as name:
        temp = Path(name)
        target_stencil = helper_stencil(target["final"], target["faces"].astype(np.int32), True, temp, "target")
        for k, (n, seed) in enumerate(subjects):
            started = time.perf_counter()
            vertices, faces, sphere = synthetic.folded_hull_and_sphere(n, seed)
            current = _normalise_sphere(sphere)
            stencil = helper_stencil(current, faces, False, temp, f"subject{k}")
            result = solve_dartel_from_surfaces(torch.as_tensor(vertices), torch.as_tensor(target["surface"]),
                                                stencil, target_stencil, fwhm=FWHM, curvtypes=(5, 5, 2),
                                                n_steps=STEPS, loop=LOOP, kernel="torch", device=CPU,
                                                dtype=torch.float64, parallel_sides=False)
            warped = apply_flow_to_stenciled_sphere(torch.as_tensor(current), result.flow, stencil, inverse=True,
                                                    device=CPU, dtype=torch.float64)
            out[f"warped_{k}"] = warped.numpy().astype(np.float32)
            out[f"cpu_seconds_{k}"] = np.float64(time.perf_counter() - started)
            print(f"subject {k}: {n} vertices, {out[f'cpu_seconds_{k}']:.1f} s")
    out["cpu_threads"] = np.int64(torch.get_num_threads())
    np.savez_compressed(HERE / "registration_golden.npz", **out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
