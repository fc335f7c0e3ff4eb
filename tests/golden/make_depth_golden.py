"""Generate depth-potential rotation-feature golden vectors by running the reference package on CPU.

Development container only (imports ``cat_surface_gpu`` from the reference
checkout).  Uses the seeded synthetic stencil of ``make_features_golden.py``
(2,562-point icosphere stencil, folded source surface) and evaluates the
reference's ``rotation_feature.py`` on the torch CPU path: stable normals,
mixed Voronoi areas, the system entries, the coloured SOR solve (20 and 1,000
sweeps), the Jacobi-preconditioned CG solve, and the full
``compute_rotation_feature`` for both solvers (heat FWHM 15 and 10).
Writes ``depth_golden.npz``.
"""

from __future__ import annotations

import importlib.util
import os
from pathlib import Path
import sys

import numpy as np

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))
from _reference import use_reference_package  # noqa: E402

use_reference_package()

import torch  # noqa: E402

from cat_surface_gpu import rotation_feature as rf  # noqa: E402


def _features_module():
    spec = importlib.util.spec_from_file_location("make_features_golden", HERE / "make_features_golden.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def main() -> int:
    torch.set_num_threads(1)
    rng = np.random.default_rng(17)
    stencil, surface = _features_module().make_stencil(rng)
    dev = stencil.to("cpu", geometry_dtype=torch.float32)
    surf32 = torch.as_tensor(surface.astype(np.float32))
    smoothed = dev.smooth_geometry(dev.resample_vertices(surf32), 15.0)
    faces = dev.faces
    normals = rf._stable_normals(smoothed, faces)
    areas = rf._mixed_voronoi_areas(smoothed, faces)
    rows, cols, values = rf._system_entries(smoothed, faces, areas, 1.0 / 1000.0)
    groups = dev.color_groups()
    labels = np.full(stencil.sphere_points.shape[0], -1, dtype=np.int32)
    for colour, members in enumerate(groups):
        labels[members.numpy()] = colour
    out = {
        "surface": surface.astype(np.float32), "smoothed": smoothed.numpy(), "normals": normals.numpy(),
        "areas": areas.numpy(), "rows": rows.numpy().astype(np.int32), "cols": cols.numpy().astype(np.int32),
        "values": values.numpy(),
        "colours": labels,
    }
    for sweeps in (20, 1000):
        sol, its, res = rf._solve_depth_potential_colored_sor(smoothed, faces, areas, normals, groups,
                                                              alpha=1.0 / 1000.0, max_iter=sweeps)
        out[f"sor{sweeps}"], out[f"sor{sweeps}_residual"] = sol.numpy(), res
    sol, its, res = rf._solve_depth_potential_cg(smoothed, faces, areas, normals, alpha=1.0 / 1000.0,
                                                 max_iter=1000, tolerance=1.0e-9)
    out["pcg"], out["pcg_iterations"], out["pcg_residual"] = sol.numpy(), its, res
    for solver, fwhm, key in (("colored-sor", 15.0, "feature_sor"), ("pcg", 10.0, "feature_pcg")):
        result = rf.compute_rotation_feature(dev, surf32, heat_fwhm=fwhm, solver=solver)
        out[key] = result.values.numpy()
        out[key + "_iterations"] = result.iterations
        out[key + "_residual"] = result.relative_residual
    np.savez_compressed(HERE / "depth_golden.npz", **out)
    print({k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items()})
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
