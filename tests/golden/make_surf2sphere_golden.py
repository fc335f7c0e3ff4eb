"""Generate the Surf2Sphere golden fixtures from the upstream CPU binary.

Runs in the development container only (it needs the reference checkout's
bundled ``bin/linux-x86_64/CAT_Surf2Sphere``); the resulting ``.npz`` files
are committed so GPU tests never need the reference at run time.

For each seeded synthetic mesh (``cat_surface_gpu_b200.synthetic``):

* ``faces``       -- triangle array (int32; uint16 on disk when it fits)
* ``surface``     -- the input surface (float32)
* ``prefix``      -- the binary's stage 1-5 output (``CAT_Surf2Sphere in out 5 0``):
                     the input of the ordered sweeps
* ``final``       -- the binary's full output (``CAT_Surf2Sphere in out 10 0``)
* ``source_area`` -- float64 surface area of the input mesh
* ``cpu_seconds`` -- wall time of the stop_at=10 run (single-threaded binary)

Usage: ``python tests/golden/make_surf2sphere_golden.py [--only c1]``
"""

from __future__ import annotations

import argparse
from pathlib import Path
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from cat_surface_gpu_b200 import synthetic  # noqa: E402
from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh  # noqa: E402
from cat_surface_gpu_b200.surf2sphere import surface_area  # noqa: E402

sys.path.insert(0, str(HERE))
from _reference import reference_binary  # noqa: E402

BINARY = reference_binary("CAT_Surf2Sphere")

CASES = {
    # folded icosphere, subdivision 5: 10,242 vertices / 20,480 faces, 60 mm
    "c1": lambda: synthetic.folded_icosphere(5, seed=1, radius_mm=60.0),
    # folded Fibonacci convex hull: 61,442 vertices / 122,880 faces, 70 mm
    "c2": lambda: synthetic.folded_hull(61442, seed=2, radius_mm=70.0),
    # a second, differently seeded folded hull: the SurfWarp target of the chain workload
    "c3": lambda: synthetic.folded_hull(61442, seed=3, radius_mm=70.0),
}


def run_binary(source: Path, output: Path, stop_at: int) -> float:
    start = time.perf_counter()
    subprocess.run([str(BINARY), str(source), str(output), str(stop_at), "0"], check=True, capture_output=True)
    return time.perf_counter() - start


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--only", choices=sorted(CASES))
    args = parser.parse_args()
    for name, make in CASES.items():
        if args.only and name != args.only:
            continue
        vertices, faces = make()
        with tempfile.TemporaryDirectory() as tmp:
            tmp = Path(tmp)
            write_gifti_mesh(tmp / "in.gii", GiftiMesh(vertices, faces))
            run_binary(tmp / "in.gii", tmp / "s5.gii", 5)
            seconds = run_binary(tmp / "in.gii", tmp / "s10.gii", 10)
            prefix = read_gifti_mesh(tmp / "s5.gii")
            final = read_gifti_mesh(tmp / "s10.gii")
        if not (np.array_equal(prefix.faces, faces) and np.array_equal(final.faces, faces)):
            raise RuntimeError("the binary changed the triangle array")
        face_dtype = np.uint16 if vertices.shape[0] <= 65535 else np.int32
        np.savez_compressed(
            HERE / f"surf2sphere_{name}.npz",
            faces=faces.astype(face_dtype),
            surface=vertices.astype(np.float32),
            prefix=prefix.vertices.astype(np.float32),
            final=final.vertices.astype(np.float32),
            source_area=np.float64(surface_area(GiftiMesh(vertices, faces))),
            cpu_seconds=np.float64(seconds),
        )
        print(name, vertices.shape, f"binary stop_at=10: {seconds:.2f} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
