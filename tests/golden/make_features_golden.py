"""Generate stencil-feature golden vectors by running the reference package on CPU.

Development container only (imports ``cat_surface_gpu`` from the reference
checkout).  A seeded synthetic stencil is assembled directly (stencil sphere =
unit icosphere with 4 subdivisions; the "surface" is a folded mesh of the same
topology resampled through per-point barycentric weights; a 64 x 32 sheet
with barycentric weights on random stencil triangles), and the reference's
``SurfaceStencilDevice`` feature operators are evaluated on it.  Writes
``features_golden.npz``.
"""

from __future__ import annotations

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

from cat_surface_gpu.surface_stencil import SurfaceStencil  # noqa: E402
from cat_surface_gpu_b200 import synthetic  # noqa: E402


def make_stencil(rng):
    sphere, faces = synthetic.unit_icosphere(4)
    surface, _ = synthetic.folded_icosphere(4, seed=5, radius_mm=60.0)
    n = sphere.shape[0]
    first_face = np.full(n, -1)
    for f, tri in enumerate(faces):
        for v in tri:
            if first_face[v] < 0:
                first_face[v] = f
    surface_indices = faces[first_face].astype(np.int32)
    w = rng.uniform(0.05, 1.0, size=(n, 3))
    corner = (faces[first_face] == np.arange(n)[:, None])
    w = np.where(corner, w + 4.0, w)
    w /= w.sum(axis=1, keepdims=True)
    nx, ny = 64, 32
    sheet_faces = rng.integers(0, faces.shape[0], size=(ny, nx))
    sw = rng.uniform(0.0, 1.0, size=(ny, nx, 3))
    sw /= sw.sum(axis=2, keepdims=True)
    stencil = SurfaceStencil(
        sphere_points=sphere, faces=faces.astype(np.int32), surface_indices=surface_indices, surface_weights=w,
        sheet_indices=faces[sheet_faces].astype(np.int32), sheet_weights=sw, nx=nx, ny=ny,
        source_points=surface.shape[0], unit_sphere_points=(sphere / np.linalg.norm(sphere, axis=1, keepdims=True)).astype(np.float32),
    )
    return stencil, surface


def main() -> int:
    rng = np.random.default_rng(17)
    stencil, surface = make_stencil(rng)
    dev = stencil.to("cpu", geometry_dtype=torch.float32)
    surf32 = torch.as_tensor(surface.astype(np.float32))
    mapped = dev.resample_vertices(surf32)
    mapped64 = dev.resample_vertices(torch.as_tensor(surface.astype(np.float64)))
    values = torch.as_tensor(rng.normal(size=stencil.sphere_points.shape[0]))
    out = {
        "sphere_points": stencil.sphere_points, "faces": stencil.faces, "surface_indices": stencil.surface_indices,
        "surface_weights": stencil.surface_weights, "sheet_indices": stencil.sheet_indices,
        "sheet_weights": stencil.sheet_weights, "unit_sphere_points": stencil.unit_sphere_points,
        "surface": surface.astype(np.float32), "values": values.numpy(),
        "resampled32": mapped.numpy(), "resampled64": mapped64.numpy(),
        "sheet": dev.map_values_to_sheet(values).numpy(),
        "smooth_geometry": dev.smooth_geometry(mapped, 50.0).numpy(),
        "normals": dev.vertex_normals(mapped).numpy(),
        "smooth_values": dev.smooth_values(values, mapped, 5.0).numpy(),
        "type5": dev.curvature_type5(mapped, 5.0).numpy(),
        "type2": dev.curvature_type2(mapped, 5.0 / 9.0).numpy(),
        "sheet_type2": dev.curvature_to_sheet(mapped, 5.0 / 9.0, curvtype=2).numpy(),
    }
    many = dev.curvature_type5_to_sheet_many(mapped, (5.0, 5.0 / 3.0))
    out["sheet5_many_0"], out["sheet5_many_1"] = many[0].numpy(), many[1].numpy()
    smv = dev.smooth_values_many(values, mapped, (5.0, 5.0 / 3.0))
    out["smooth_many_0"], out["smooth_many_1"] = smv[0].numpy(), smv[1].numpy()
    np.savez_compressed(HERE / "features_golden.npz", **out)
    print(len(out), "arrays")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
