"""The product path spawns no process.

The reference ran stages 1-5 of CAT_Surf2Sphere on its upstream CPU binary
(``surf2sphere.py:1201-1246``) and could build stencils and rotation features
with helper binaries (``gpu_pipeline.py:144-166, 206-229``).  This package
runs all of it on the GPU: no module but the build recipe imports
``subprocess``, the default CLI and API calls never start a process, and the
options that named a helper binary are rejected with ``ValueError`` before any
file is read or any kernel is launched.
"""

from __future__ import annotations

import ast
import os
from pathlib import Path
import subprocess

import numpy as np
import pytest

from conftest import ROOT

PACKAGE = ROOT / "cat_surface_gpu_b200"
SPAWNING = {"subprocess", "multiprocessing", "pty"}
OS_SPAWN = {"system", "popen", "fork", "forkpty", "posix_spawn", "posix_spawnp", "spawnv", "spawnve", "spawnl",
            "execv", "execve", "execvp", "execl"}


def _spawning_uses(path: Path) -> list[str]:
    tree = ast.parse(path.read_text(), filename=str(path))
    found = []
    for node in ast.walk(tree):
        if isinstance(node, ast.Import):
            found += [alias.name for alias in node.names if alias.name.split(".")[0] in SPAWNING]
        elif isinstance(node, ast.ImportFrom) and node.module and node.module.split(".")[0] in SPAWNING:
            found.append(node.module)
        elif isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id == "os" \
                and node.attr in OS_SPAWN:
            found.append(f"os.{node.attr}")
    return found


def test_only_the_build_recipe_spawns_processes():
    offenders = {}
    for path in sorted(PACKAGE.glob("*.py")):
        if path.name == "build.py":  # nvcc, at build time only
            continue
        uses = _spawning_uses(path)
        if uses:
            offenders[path.name] = uses
    assert offenders == {}


@pytest.fixture
def no_spawn(monkeypatch):
    """Fail any attempt to start a process inside the test."""

    calls = []

    def refuse(*args, **kwargs):
        calls.append(args)
        raise AssertionError(f"the product path tried to start a process: {args[:1]}")

    monkeypatch.setattr(subprocess, "Popen", refuse)
    monkeypatch.setattr(subprocess, "run", refuse)
    for name in ("fork", "posix_spawn", "posix_spawnp", "system"):
        if hasattr(os, name):
            monkeypatch.setattr(os, name, refuse)
    return calls


def _write_mesh(path: Path, seed: int, subdivisions: int = 3) -> None:
    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh

    vertices, faces = synthetic.folded_icosphere(subdivisions, seed=seed)
    write_gifti_mesh(path, GiftiMesh(vertices, faces))


def test_surf2sphere_rejects_the_cpu_preprocess(tmp_path, no_spawn):
    from cat_surface_gpu_b200.cli import surf2sphere_main
    from cat_surface_gpu_b200.surf2sphere import run_cat_surf2sphere_gpu

    with pytest.raises(ValueError, match="GPU"):
        run_cat_surf2sphere_gpu(tmp_path / "missing.gii", tmp_path / "out.gii", preprocess_kernel="cpu")
    with pytest.raises(ValueError):
        run_cat_surf2sphere_gpu(tmp_path / "missing.gii", tmp_path / "out.gii", preprocess_kernel="nope")
    with pytest.raises(SystemExit) as exit_info:
        surf2sphere_main(["--input-surface", str(tmp_path / "missing.gii"), "--output-surface",
                          str(tmp_path / "out.gii"), "--preprocess-kernel", "cpu"])
    assert exit_info.value.code == 2
    assert no_spawn == []


@pytest.mark.parametrize("options", [
    {"rotation_feature_backend": "official-cpu"},
    {"rotation_feature_backend": "cuda-official-depth"},
    {"rotation_feature_backend": "cuda-official-geometry"},
    {"stencil_builder": "/usr/bin/cat_surface_stencil_builder"},
    {"rotated_stencil_builder": "/usr/bin/cat_surface_stencil_builder"},
    {"rotation_values_probe": "/usr/bin/cat_surface_rotation_values"},
    {"rotation_geometry_probe": "/usr/bin/cat_surface_rotation_geometry"},
    {"rotation_depth_probe": "/usr/bin/cat_surface_rotation_depth"},
])
def test_surfwarp_rejects_helper_binaries_before_reading(tmp_path, no_spawn, options):
    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline

    missing = [tmp_path / f"{name}.gii" for name in ("ss", "sp", "ts", "tp")]
    with pytest.raises(ValueError, match="GPU"):
        run_cat_surface_gpu_pipeline(*missing, tmp_path / "out.gii", **options)
    assert no_spawn == []


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="the GPU variant below runs the full call")
def test_default_cli_calls_reach_the_device_without_spawning(tmp_path, no_spawn):
    """Without a GPU the default calls stop at device resolution, having started nothing."""

    from cat_surface_gpu_b200.cli import surf2sphere_main, surfwarp_main

    _write_mesh(tmp_path / "in.gii", 3)
    with pytest.raises(RuntimeError):
        surf2sphere_main(["--input-surface", str(tmp_path / "in.gii"), "--output-surface", str(tmp_path / "o.gii")])
    with pytest.raises(RuntimeError):
        surfwarp_main(["--source-surface", str(tmp_path / "in.gii"), "--source-sphere", str(tmp_path / "in.gii"),
                       "--target-surface", str(tmp_path / "in.gii"), "--target-sphere", str(tmp_path / "in.gii"),
                       "--output", str(tmp_path / "w.gii")])
    assert no_spawn == []
    assert not (tmp_path / "o.gii").exists()


@pytest.mark.gpu
def test_default_cli_calls_run_on_the_gpu_without_spawning(native_library, tmp_path, no_spawn, capsys):
    """cat-surf2sphere-gpu and cat-surfwarp-gpu with their default options, with process creation refused."""

    from cat_surface_gpu_b200.cli import surf2sphere_main, surfwarp_main
    from cat_surface_gpu_b200.gifti import read_gifti_mesh

    # 10,242-vertex folded icospheres: CAT_Surf2Sphere's stages 1-4 shrink much coarser meshes to a point
    for seed, name in ((3, "a"), (4, "b")):
        _write_mesh(tmp_path / f"{name}.gii", seed, subdivisions=5)
        assert surf2sphere_main(["--input-surface", str(tmp_path / f"{name}.gii"), "--output-surface",
                                 str(tmp_path / f"{name}.sphere.gii"), "--device", "cuda:0"]) == 0
        sphere = read_gifti_mesh(tmp_path / f"{name}.sphere.gii").vertices.astype(np.float64)
        assert np.all(np.isfinite(sphere))
    assert surfwarp_main(["--source-surface", str(tmp_path / "a.gii"), "--source-sphere",
                          str(tmp_path / "a.sphere.gii"), "--target-surface", str(tmp_path / "b.gii"),
                          "--target-sphere", str(tmp_path / "b.sphere.gii"), "--output", str(tmp_path / "w.gii"),
                          "--sheet-size", "128", "64", "--device", "cuda:0"]) == 0
    warped = read_gifti_mesh(tmp_path / "w.gii").vertices.astype(np.float64)
    assert np.allclose(np.linalg.norm(warped, axis=1), 1.0, atol=1e-5)
    assert no_spawn == []
    capsys.readouterr()
