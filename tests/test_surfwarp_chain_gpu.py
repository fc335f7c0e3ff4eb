"""End-to-end SurfWarp parity on the GPU against the reference chain golden.

The golden (``tests/golden/make_surfwarp_chain_golden.py``) ran the reference
package's operators on the CPU in the order of its ``run_cat_surface_gpu_pipeline``:
stencils from the reference's own stencil helper (its 128 x 64 sheet from the
oracle's restatement of the helper's sheet), the default ("cuda") rotation
features -- the depth potential by coloured SOR, ``compute_rotation_features``
-- the rotation search, two DARTEL runs of two steps, the ``-avg`` solve and
blend.  This runs ``run_cat_surface_gpu_pipeline`` (its own GPU-built
stencils) on the same GIFTI inputs and bounds the final unit-sphere vertex
error at 1e-3 (max), the accuracy the Surf2Sphere+SurfWarp chain is quoted
at.  The feature operators are pinned on identical stencils: the golden
also holds the reference's features on this package's stencils.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chain():
    return dict(np.load(GOLDEN / "surfwarp_chain_golden.npz"))


def _write_inputs(chain, directory):
    from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh

    paths = {}
    for name in ("source_surface", "source_sphere", "target_surface", "target_sphere"):
        paths[name] = directory / f"{name}.gii"
        write_gifti_mesh(paths[name], GiftiMesh(chain[name], chain["faces"]))
    return paths


def test_rotation_features_match_reference(native_library, chain):
    """Depth-potential features (both sides in one batched solve) and the type-5 curvature option."""

    from cat_surface_gpu_b200.gpu_pipeline import depth_rotation_features, native_rotation_features
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    nx, ny = int(chain["param_nx"]), int(chain["param_ny"])
    stencils = [build_surface_stencil(chain[f"{side}_sphere"], chain["faces"], nx=nx, ny=ny, normalize=True)
                for side in ("source", "target")]
    timings = {}
    values = depth_rotation_features(stencils[0], stencils[1], chain["source_surface"], chain["target_surface"],
                                     torch.device("cuda:0"), timings=timings)
    assert timings["rotation_feature_source_iterations"] == 1000.0
    for got, want in zip(values, (chain["builder_source_values"], chain["builder_target_values"])):
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=0, atol=1e-12)
    values = native_rotation_features(stencils[0], stencils[1], chain["source_surface"], chain["target_surface"],
                                      torch.device("cuda:0"))
    for got, want in zip(values, (chain["builder_curv_source_values"], chain["builder_curv_target_values"])):
        scale = float(np.abs(want).max())
        assert np.abs(got.astype(np.float64) - want).max() <= 1e-5 * scale


def test_surfwarp_chain_matches_reference(native_library, chain, tmp_path):
    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline

    paths = _write_inputs(chain, tmp_path)
    result = run_cat_surface_gpu_pipeline(
        paths["source_surface"], paths["source_sphere"], paths["target_surface"], paths["target_sphere"],
        tmp_path / "out.gii", device="cuda:0", steps=int(chain["param_steps"]), runs=int(chain["param_runs"]),
        avg=bool(chain["param_avg"]), loop=int(chain["param_loop"]),
        rotation_grid_size=int(chain["param_rotation_grid_size"]),
        sheet_size=(int(chain["param_nx"]), int(chain["param_ny"])), stencil_threads=8,
    )
    error = np.linalg.norm(result.vertices.astype(np.float64) - chain["final_sphere"], axis=1)
    print(f"chain vertex error: max {error.max():.3e} mean {error.mean():.3e} p99 {np.quantile(error, 0.99):.3e}; "
          f"angle {np.abs(result.rotation_angle - chain['rotation_angle']).max():.3e}")
    # the golden's stencils are the helper's (float32 points), the pipeline's its own float64 build: the
    # Nelder-Mead optimum moves within the search's tolerance, the final sphere stays within the contract
    assert np.abs(result.rotation_angle - chain["rotation_angle"]).max() <= 1e-3
    assert error.max() <= 1e-3
    assert (tmp_path / "out.gii").exists()


@pytest.mark.parametrize("normalize,size", [(True, (64, 32)), (False, (256, 128))])
def test_device_stencil_builder_equals_host_builder(native_library, chain, normalize, size):
    """The GPU stencil builder reproduces the host builder bit for bit."""

    from cat_surface_gpu_b200.gpu_pipeline import normalise_sphere
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    nx, ny = size
    sphere = chain["target_sphere"] if normalize else normalise_sphere(chain["source_sphere"])
    host = build_surface_stencil(sphere, chain["faces"], nx=nx, ny=ny, normalize=normalize, threads=4)
    dev = build_surface_stencil(sphere, chain["faces"], nx=nx, ny=ny, normalize=normalize, device="cuda:0")
    for name in ("sphere_points", "surface_indices", "surface_weights", "sheet_indices", "sheet_weights",
                 "unit_sphere_points"):
        np.testing.assert_array_equal(getattr(dev, name), getattr(host, name), err_msg=name)


def test_device_stencil_builder_on_hemisphere_mesh(native_library):
    """61,442-vertex hull sphere (the benchmark's target): device == host."""

    from conftest import GOLDEN
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    c3 = np.load(GOLDEN / "surf2sphere_c3.npz")
    faces = c3["faces"].astype(np.int32)
    host = build_surface_stencil(c3["final"], faces, nx=256, ny=128, threads=8)
    dev = build_surface_stencil(c3["final"], faces, nx=256, ny=128, device="cuda:0")
    for name in ("sphere_points", "surface_indices", "surface_weights", "sheet_indices", "sheet_weights",
                 "unit_sphere_points"):
        np.testing.assert_array_equal(getattr(dev, name), getattr(host, name), err_msg=name)


def test_hemisphere_chain_matches_reference_on_the_same_stencils(native_library):
    """The benchmark's hemisphere (61,442-vertex hulls c2 -> c3, 256 x 128, steps 2, runs 2, -avg).

    The golden holds the reference's CPU chain twice: on its helper's float32
    stencils and on this package's host stencils.  The two reference results
    differ by up to ~9e-3 (the stencils' rounding moves the rotation pick by
    ~4e-5 rad and the registration carries that), so the GPU chain is held to
    1e-3 against the reference run on the same stencils, and to the helper
    chain's own spread against the other.
    """

    from cat_surface_gpu_b200.gifti import GiftiMesh
    from cat_surface_gpu_b200.gpu_pipeline import register_meshes

    source, target = (np.load(GOLDEN / f"surf2sphere_{name}.npz") for name in ("c2", "c3"))
    gold = np.load(GOLDEN / "surfwarp_chain_hemisphere_golden.npz")
    faces, target_faces = source["faces"].astype(np.int32), target["faces"].astype(np.int32)
    final, angle, _, _ = register_meshes(
        GiftiMesh(source["surface"], faces), GiftiMesh(source["final"], faces),
        GiftiMesh(target["surface"], target_faces), GiftiMesh(target["final"], target_faces), device="cuda:0",
        steps=2, runs=2, avg=True, loop=6, sheet_size=(256, 128), rotation_feature_backend="cuda",
        rotation_feature_solver="colored-sor")
    final = np.asarray(final, dtype=np.float64)
    same = np.linalg.norm(final - gold["builder_final_sphere"], axis=1)
    helper = np.linalg.norm(final - gold["final_sphere"], axis=1)
    spread = np.linalg.norm(gold["builder_final_sphere"] - gold["final_sphere"], axis=1)
    print(f"hemisphere chain error: same stencils max {same.max():.3g}, helper stencils max {helper.max():.3g} "
          f"(reference spread {spread.max():.3g})")
    assert np.abs(angle - gold["builder_rotation_angle"]).max() <= 1e-5
    assert same.max() <= 1e-3
    assert helper.max() <= 1.5 * spread.max()
    torch.cuda.synchronize()
