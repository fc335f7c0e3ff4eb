"""Generate rotation-search golden vectors by running the reference package on CPU.

Development container only (imports ``cat_surface_gpu`` from the reference
checkout).  Writes ``rotation_golden.npz``: a seeded target sphere (unit
icosphere, 4 subdivisions) with a smooth feature, a perturbed and rotated
source point set with its feature, the reference's candidate costs for the 46
official seeds plus random angles, and the reference's full search result
(seed search + Nelder-Mead).

Usage: ``python tests/golden/make_rotation_golden.py``
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

from cat_surface_gpu.surface_rotation import RotationGridIndex, official_seed_grid_angles  # noqa: E402
from cat_surface_gpu_b200 import synthetic  # noqa: E402


def feature(points):
    x, y, z = points[:, 0], points[:, 1], points[:, 2]
    return np.sin(3 * x) * np.cos(2 * y) + 0.5 * z * z + 0.3 * np.sin(5 * z + x)


def main() -> int:
    rng = np.random.default_rng(11)
    tp, tf = synthetic.unit_icosphere(4)
    sp, _ = synthetic.unit_icosphere(4)
    sp = sp + rng.normal(scale=0.01, size=sp.shape)
    sp /= np.linalg.norm(sp, axis=1, keepdims=True)
    true = np.array([0.15, -0.1, 0.2])
    # source = target rotated by the inverse of `true` (so the search should recover ~true)
    c, s = np.cos(true), np.sin(true)
    rx = np.array([[1, 0, 0], [0, c[0], -s[0]], [0, s[0], c[0]]])
    ry = np.array([[c[1], 0, s[1]], [0, 1, 0], [-s[1], 0, c[1]]])
    rz = np.array([[c[2], -s[2], 0], [s[2], c[2], 0], [0, 0, 1]])
    rot = rz @ ry @ rx
    sp = sp @ rot  # rows: rot^T p
    source_points = sp.astype(np.float32)
    source_values = feature(sp @ rot.T)
    target_values = feature(tp)
    index = RotationGridIndex.from_geometry(tp, tf, grid_size=32, margin=1, include_dense_candidate_table=False)
    device_index = index.to("cpu")
    angles = np.concatenate((official_seed_grid_angles(), rng.uniform(-0.7, 0.7, size=(10, 3))))
    costs = device_index.cost_batch(torch.as_tensor(source_points), torch.as_tensor(source_values),
                                    torch.as_tensor(target_values), torch.as_tensor(angles), point_chunk=1024).numpy()
    result = device_index.search_rotation(torch.as_tensor(source_points), torch.as_tensor(source_values),
                                          torch.as_tensor(target_values), point_chunk=1024)
    np.savez_compressed(
        HERE / "rotation_golden.npz",
        target_points=tp, target_faces=tf, target_values=target_values,
        source_points=source_points, source_values=source_values, angles=angles, costs=costs,
        grid_offsets=index.candidate_offsets, grid_faces=index.candidate_faces, grid_size=np.int64(32),
        seed_angle=result.seed_angle.numpy(), seed_costs=result.seed_costs.numpy(), angle=result.angle.numpy(),
        cost=result.cost.numpy(), matrix=result.rotation_matrix.numpy(), iterations=np.int64(result.iterations),
        rotated=device_index.rotate_points(torch.as_tensor(source_points), torch.as_tensor(angles[:5])).numpy(),
    )
    print("angle", result.angle.numpy(), "cost", float(result.cost), "iterations", result.iterations)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
