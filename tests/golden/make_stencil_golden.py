"""Generate stencil golden vectors by running the reference's stencil helper.

Development checkout only: executes the bundled
``bin/linux-x86_64/cat_surface_stencil_builder`` (run as a program; nothing
else of it is used) on three spheres and keeps seeded subsets of what it
writes, so the tests pin this package's stencil builder to the helper
without the reference at test time:

* ``c1``: the upstream Surf2Sphere sphere of the 10,242-vertex golden mesh
  (``surf2sphere_c1.npz``), default options (centred and unit-normalised);
* ``c3``: the 61,442-vertex hull sphere (``surf2sphere_c3.npz``), default;
* ``c1r``: the ``c1`` sphere centred, unit-normalised and rotated by
  (0.3, -0.2, 0.5) rad, with ``--no-normalize`` (the rotated-stencil call of
  the SurfWarp pipeline).

For each: the SHA-256 of the helper's face array (the resampling sphere's
topology), 8,192 seeded rows of the surface barycentrics and resampled
sphere points, 8,192 seeded sheet cells, 4,096 unit-sphere points, and the
header sizes.  The ``c1`` / ``c3`` spheres are read back from their
Surf2Sphere goldens; the rotated ``c1r`` sphere is stored.  Writes
``stencil_helper_golden.npz``.

Usage: ``python tests/golden/make_stencil_golden.py`` (``CAT_SURFACE_REFERENCE``
names the reference checkout).
"""

from __future__ import annotations

import hashlib
import os
from pathlib import Path
import subprocess
import sys
import tempfile

import numpy as np

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))
from _reference import reference_binary  # noqa: E402

from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh  # noqa: E402
from cat_surface_gpu_b200.surface_stencil import SurfaceStencil  # noqa: E402

HELPER = reference_binary("cat_surface_stencil_builder")
ROWS, CELLS, UNIT = 8192, 8192, 4096


def rotated_unit(vertices: np.ndarray, angles) -> np.ndarray:
    p = vertices.astype(np.float64)
    p = p - p.mean(axis=0)
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    c, s = np.cos(angles), np.sin(angles)
    rx = np.array([[1, 0, 0], [0, c[0], -s[0]], [0, s[0], c[0]]])
    ry = np.array([[c[1], 0, s[1]], [0, 1, 0], [-s[1], 0, c[1]]])
    rz = np.array([[c[2], -s[2], 0], [s[2], c[2], 0], [0, 0, 1]])
    return (p @ (rz @ ry @ rx).T).astype(np.float32)


def run_helper(sphere: np.ndarray, faces: np.ndarray, normalize: bool, temp: Path) -> SurfaceStencil:
    write_gifti_mesh(temp / "sphere.gii", GiftiMesh(sphere, faces))
    command = [str(HELPER), str(temp / "sphere.gii"), str(temp / "out.stencil"), "--threads", "8"]
    if not normalize:
        command.insert(3, "--no-normalize")
    subprocess.run(command, check=True, capture_output=True)
    return SurfaceStencil.from_file(temp / "out.stencil")


def main() -> None:
    cases = {}
    for name in ("c1", "c3"):
        data = np.load(HERE / f"surf2sphere_{name}.npz")
        cases[name] = (data["final"].astype(np.float32), data["faces"].astype(np.int32), True)
    c1 = np.load(HERE / "surf2sphere_c1.npz")
    cases["c1r"] = (rotated_unit(c1["final"], (0.3, -0.2, 0.5)), c1["faces"].astype(np.int32), False)
    out = {}
    rng = np.random.default_rng(2024)
    with tempfile.TemporaryDirectory(prefix="stencil_golden_") as name_dir:
        temp = Path(name_dir)
        for name, (sphere, faces, normalize) in cases.items():
            st = run_helper(sphere, faces, normalize, temp)
            n_points = st.sphere_points.shape[0]
            rows = np.sort(rng.choice(n_points, size=ROWS, replace=False))
            cells = np.sort(rng.choice(st.nx * st.ny, size=CELLS, replace=False))
            unit = np.sort(rng.choice(st.source_points, size=min(UNIT, st.source_points), replace=False))
            if name == "c1r":  # c1 and c3 are read from their Surf2Sphere goldens
                out[f"{name}_sphere"] = sphere
            out[f"{name}_normalize"] = np.array(normalize)
            out[f"{name}_sizes"] = np.array([n_points, st.faces.shape[0], st.nx, st.ny, st.source_points])
            out[f"{name}_faces_sha256"] = np.array(hashlib.sha256(
                np.ascontiguousarray(st.faces, dtype="<i4").tobytes()).hexdigest())
            out[f"{name}_rows"] = rows.astype(np.int32)
            out[f"{name}_surface_indices"] = st.surface_indices[rows]
            out[f"{name}_surface_weights"] = st.surface_weights[rows]
            out[f"{name}_sphere_points"] = st.sphere_points[rows]
            out[f"{name}_cells"] = cells.astype(np.int32)
            out[f"{name}_sheet_indices"] = st.sheet_indices.reshape(-1, 3)[cells]
            out[f"{name}_sheet_weights"] = st.sheet_weights.reshape(-1, 3)[cells]
            out[f"{name}_unit_rows"] = unit.astype(np.int32)
            out[f"{name}_unit_points"] = st.unit_sphere_points[unit]
            print(name, n_points, st.faces.shape[0], st.nx, st.ny, st.source_points)
    np.savez_compressed(HERE / "stencil_helper_golden.npz", **out)


if __name__ == "__main__":
    main()
