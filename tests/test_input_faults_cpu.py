"""Host-side fault injection: corrupt inputs are refused with ``ValueError`` before any launch.

The GPU kernels gather with the indices they are given and do arithmetic on
the coordinates they are given, so every public entry point checks its
inputs on the host first.  Each case here plants one fault in an otherwise
valid input -- a truncated or bad-magic ``.stencil`` (the reader's checks
follow ``src/cat_surface_gpu/surface_stencil.py:133-175``), stencil indices
outside their range, a GIFTI file that does not parse or decode, NaN
vertices, faces outside the mesh, a surface and sphere of different vertex
counts -- and checks the error.  No GPU is needed: the faults are caught
before device resolution.
"""

from __future__ import annotations

import base64
from pathlib import Path
import struct
import zlib

import numpy as np
import pytest

from cat_surface_gpu_b200 import synthetic
from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh
from cat_surface_gpu_b200.surface_stencil import SurfaceStencil


@pytest.fixture(scope="module")
def stencil():
    points, faces = synthetic.unit_icosphere(2)
    n = points.shape[0]
    rng = np.random.default_rng(3)
    nx, ny = 8, 4
    weights = rng.uniform(0.1, 1.0, size=(n, 3))
    sheet_w = rng.uniform(0.1, 1.0, size=(ny, nx, 3))
    return SurfaceStencil(
        sphere_points=points.astype(np.float64), faces=faces.astype(np.int32),
        surface_indices=rng.integers(0, 100, size=(n, 3), dtype=np.int32),
        surface_weights=weights / weights.sum(1, keepdims=True),
        sheet_indices=rng.integers(0, n, size=(ny, nx, 3), dtype=np.int32),
        sheet_weights=sheet_w / sheet_w.sum(2, keepdims=True), nx=nx, ny=ny, source_points=100,
        unit_sphere_points=rng.normal(size=(100, 3)).astype(np.float32))


def test_valid_stencil_round_trips(tmp_path, stencil):
    stencil.to_file(tmp_path / "ok.stencil")
    back = SurfaceStencil.from_file(tmp_path / "ok.stencil")
    assert np.array_equal(back.surface_indices, stencil.surface_indices)
    assert np.array_equal(back.sheet_weights, stencil.sheet_weights)


@pytest.mark.parametrize("cut", [0, 7, 32, 100, -1, -13])
def test_truncated_stencil_is_refused(tmp_path, stencil, cut):
    stencil.to_file(tmp_path / "ok.stencil")
    raw = (tmp_path / "ok.stencil").read_bytes()
    (tmp_path / "cut.stencil").write_bytes(raw[:cut] if cut >= 0 else raw[:len(raw) + cut])
    with pytest.raises(ValueError, match="Stencil"):
        SurfaceStencil.from_file(tmp_path / "cut.stencil")


@pytest.mark.parametrize("field, value", [(0, 0x12345678), (1, 3), (2, -5), (4, 33), (5, -8)])
def test_bad_stencil_header_is_refused(tmp_path, stencil, field, value):
    stencil.to_file(tmp_path / "ok.stencil")
    raw = bytearray((tmp_path / "ok.stencil").read_bytes())
    struct.pack_into("<i", raw, 4 * field, value)
    (tmp_path / "bad.stencil").write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="Stencil"):
        SurfaceStencil.from_file(tmp_path / "bad.stencil")


@pytest.mark.parametrize("what", ["faces", "surface_indices", "sheet_indices", "surface_weights", "sphere_points"])
def test_stencil_contents_out_of_range_are_refused(tmp_path, stencil, what):
    arrays = {name: getattr(stencil, name).copy() for name in
              ("sphere_points", "faces", "surface_indices", "surface_weights", "sheet_indices", "sheet_weights")}
    if what == "faces":
        arrays["faces"][5, 1] = stencil.sphere_points.shape[0]
    elif what == "surface_indices":
        arrays["surface_indices"][0, 2] = stencil.source_points
    elif what == "sheet_indices":
        arrays["sheet_indices"][1, 1, 0] = -1
    elif what == "surface_weights":
        arrays["surface_weights"][3, 0] = np.nan
    else:
        arrays["sphere_points"][7, 2] = np.inf
    bad = SurfaceStencil(**arrays, nx=stencil.nx, ny=stencil.ny, source_points=stencil.source_points,
                         unit_sphere_points=stencil.unit_sphere_points)
    bad.to_file(tmp_path / "bad.stencil")
    with pytest.raises(ValueError, match="Stencil"):
        SurfaceStencil.from_file(tmp_path / "bad.stencil")
    with pytest.raises(ValueError, match="Stencil"):
        bad.validate()


def _gifti(tmp_path: Path, name: str = "mesh.gii") -> Path:
    vertices, faces = synthetic.folded_icosphere(2, seed=5)
    write_gifti_mesh(tmp_path / name, GiftiMesh(vertices, faces))
    return tmp_path / name


def _payloads(text: str) -> list[tuple[int, int]]:
    spans, at = [], 0
    while True:
        start = text.find("<Data>", at)
        if start < 0:
            return spans
        end = text.find("</Data>", start)
        spans.append((start + len("<Data>"), end))
        at = end


def test_gifti_that_does_not_parse_is_refused(tmp_path):
    path = _gifti(tmp_path)
    text = path.read_text()
    (tmp_path / "cut.gii").write_text(text[: len(text) // 2])
    with pytest.raises(ValueError, match="GIFTI"):
        read_gifti_mesh(tmp_path / "cut.gii")
    (tmp_path / "other.gii").write_text(text.replace("<GIFTI", "<NOTGIFTI").replace("</GIFTI>", "</NOTGIFTI>"))
    with pytest.raises(ValueError, match="GIFTI"):
        read_gifti_mesh(tmp_path / "other.gii")


@pytest.mark.parametrize("fault", ["base64", "zlib", "short"])
def test_gifti_payload_that_does_not_decode_is_refused(tmp_path, fault):
    path = _gifti(tmp_path)
    text = path.read_text()
    start, end = _payloads(text)[0]
    payload = "".join(text[start:end].split())
    if fault == "base64":
        bad = payload[:-5] + "!!!!!"
    elif fault == "zlib":
        raw = bytearray(base64.b64decode(payload))
        raw[len(raw) // 2:len(raw) // 2 + 8] = b"\xff" * 8
        bad = base64.b64encode(bytes(raw)).decode()
    else:
        raw = zlib.decompress(base64.b64decode(payload))
        bad = base64.b64encode(zlib.compress(raw[:-12])).decode()
    (tmp_path / "bad.gii").write_text(text[:start] + bad + text[end:])
    with pytest.raises(ValueError, match="GIFTI"):
        read_gifti_mesh(tmp_path / "bad.gii")


def test_surf2sphere_refuses_nan_vertices_and_faces_outside(tmp_path):
    from cat_surface_gpu_b200.surf2sphere import (Surf2SphereTopology, run_areal_smoothing_cuda,
                                                  run_cat_surf2sphere_gpu, run_surf2sphere_preprocess_cuda)

    vertices, faces = synthetic.folded_icosphere(2, seed=5)
    nan = vertices.copy()
    nan[17, 1] = np.nan
    write_gifti_mesh(tmp_path / "nan.gii", GiftiMesh(nan, faces))
    with pytest.raises(ValueError, match="finite"):
        run_cat_surf2sphere_gpu(tmp_path / "nan.gii", tmp_path / "out.gii")
    outside = faces.copy()
    outside[3, 0] = vertices.shape[0]
    write_gifti_mesh(tmp_path / "outside.gii", GiftiMesh(vertices, outside))
    with pytest.raises(ValueError, match="outside"):
        run_cat_surf2sphere_gpu(tmp_path / "outside.gii", tmp_path / "out.gii")
    assert not (tmp_path / "out.gii").exists()
    topology = Surf2SphereTopology.from_mesh(GiftiMesh(vertices, faces))
    with pytest.raises(ValueError, match="finite"):
        run_areal_smoothing_cuda(nan, faces, topology, iterations=3, project_every=0, radius=1.0)
    with pytest.raises(ValueError, match="finite"):
        run_surf2sphere_preprocess_cuda(nan, faces, topology, stop_at=1, desired_surface_area=1.0)


def _four_meshes(tmp_path: Path) -> list[Path]:
    """Source surface, source sphere, target surface, target sphere (valid, 162 vertices each)."""

    paths = []
    for seed, name in ((5, "ss"), (6, "sp"), (7, "ts"), (8, "tp")):
        vertices, faces = synthetic.folded_icosphere(2, seed=seed)
        write_gifti_mesh(tmp_path / f"{name}.gii", GiftiMesh(vertices, faces))
        paths.append(tmp_path / f"{name}.gii")
    return paths


def test_surfwarp_refuses_bad_meshes_before_any_launch(tmp_path):
    from cat_surface_gpu_b200.gpu_pipeline import register_meshes, run_cat_surface_gpu_pipeline

    paths = _four_meshes(tmp_path)
    meshes = [read_gifti_mesh(p) for p in paths]
    # a sphere with fewer vertices than its surface
    small_v, small_f = synthetic.folded_icosphere(1, seed=9)
    with pytest.raises(ValueError, match="vertices"):
        register_meshes(meshes[0], GiftiMesh(small_v, small_f), meshes[2], meshes[3])
    write_gifti_mesh(tmp_path / "small.gii", GiftiMesh(small_v, small_f))
    with pytest.raises(ValueError, match="vertices"):
        run_cat_surface_gpu_pipeline(paths[0], paths[1], paths[2], tmp_path / "small.gii", tmp_path / "out.gii")
    # NaN coordinates on the target surface
    nan = meshes[2].vertices.copy()
    nan[0, 0] = np.nan
    with pytest.raises(ValueError, match="finite"):
        register_meshes(meshes[0], meshes[1], GiftiMesh(nan, meshes[2].faces), meshes[3])
    # a face outside the source sphere
    bad_faces = meshes[1].faces.copy()
    bad_faces[0, 2] = -1
    with pytest.raises(ValueError, match="outside"):
        register_meshes(meshes[0], GiftiMesh(meshes[1].vertices, bad_faces), meshes[2], meshes[3])
    # non-finite rotation values
    n = meshes[0].vertices.shape[0]
    with pytest.raises(ValueError, match="rotation values"):
        register_meshes(*meshes, rotation_values=(np.full(n, np.nan), np.zeros(n)))
    assert not (tmp_path / "out.gii").exists()
