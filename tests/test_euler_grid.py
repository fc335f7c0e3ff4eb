"""The 10-degree-then-2-degree Euler-grid rotation search (the rotation mode of the
SurfWarp configuration on z-scored curvature and depth features).

CPU: the candidate grids and the z-scoring.  GPU: grid costs against the
oracle's restatement of the reference's cost (``surface_rotation.py:512-546``,
pinned to the reference by ``test_rotation.py``) on a sample of candidates, the
two-level choice, and the option through the SurfWarp pipeline.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN


def test_coarse_grid_covers_so3_in_10_degree_steps():
    from cat_surface_gpu_b200.surface_rotation import euler_grid_angles

    a = np.rad2deg(euler_grid_angles(10.0))
    assert a.shape == (36 * 19 * 36, 3)
    assert np.allclose(np.unique(a[:, 0]), np.arange(-180, 180, 10))
    assert np.allclose(np.unique(a[:, 1]), np.arange(-90, 91, 10))
    assert np.allclose(np.unique(a[:, 2]), np.arange(-180, 180, 10))
    # x slowest, z fastest
    assert np.allclose(a[1] - a[0], [0, 0, 10]) and np.allclose(a[36] - a[0], [0, 10, 0])


def test_fine_grid_is_centred_on_the_coarse_pick():
    from cat_surface_gpu_b200.surface_rotation import euler_grid_angles

    centre = np.deg2rad([30.0, -40.0, 170.0])
    f = euler_grid_angles(2.0, centre, 10.0)
    assert f.shape == (11 ** 3, 3)
    d = np.rad2deg(f - centre)
    assert np.allclose(d.min(axis=0), -10) and np.allclose(d.max(axis=0), 10)
    assert np.allclose(np.rad2deg(f[11 ** 3 // 2]), [30.0, -40.0, 170.0])
    with pytest.raises(ValueError):
        euler_grid_angles(0.0)
    with pytest.raises(ValueError):
        euler_grid_angles(2.0, centre)


def test_zscore_is_float32_rounded_and_per_feature():
    from cat_surface_gpu_b200.surface_rotation import zscore

    rng = np.random.default_rng(1)
    v = np.stack([rng.normal(3.0, 2.0, 500), rng.uniform(-1, 7, 500)])
    z = zscore(v)
    assert z.dtype == np.float64 and np.array_equal(z, z.astype(np.float32).astype(np.float64))
    assert np.allclose(z.mean(axis=1), 0.0, atol=1e-6) and np.allclose(z.std(axis=1), 1.0, atol=1e-6)
    assert np.array_equal(zscore(np.full(4, 2.0)), np.zeros(4))


def test_pipeline_rejects_values_with_the_grid_search(tmp_path):
    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline

    paths = [tmp_path / f"{i}.gii" for i in range(5)]
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, rotation_search="grid")
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, rotation_values_path=paths[0], rotation_search="euler-grid")


@pytest.fixture(scope="module")
def chain():
    return dict(np.load(GOLDEN / "surfwarp_chain_golden.npz"))


@pytest.mark.gpu
def test_grid_costs_match_the_oracle_and_pick_the_first_minimum(native_library, chain):
    from cat_surface_gpu_b200.surface_rotation import RotationGridIndexDevice, euler_grid_angles, zscore
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil
    from oracle import rotation as orot

    stencils = [build_surface_stencil(chain[f"{side}_sphere"], chain["faces"], nx=64, ny=32, normalize=True)
                for side in ("source", "target")]
    sv = zscore(np.stack([chain["builder_curv_source_values"], chain["builder_source_values"]]))
    tv = zscore(np.stack([chain["builder_curv_target_values"], chain["builder_target_values"]]))
    target = stencils[1]
    index = RotationGridIndexDevice.build(target.sphere_points, target.faces, device="cuda:0")
    inputs = index.prepare_cost_inputs(stencils[0].sphere_points.astype(np.float32), sv, tv)
    result = index.euler_grid_search_prepared(inputs)
    coarse = euler_grid_angles(10.0)
    costs = result.seed_costs.cpu().numpy()
    assert costs.shape == (coarse.shape[0],)
    assert np.allclose(result.seed_angle.cpu().numpy(), coarse[int(np.argmin(costs))])
    assert float(result.cost) <= float(result.seed_cost)  # the fine grid holds the coarse pick
    # a seeded sample of the coarse candidates, costed by the oracle feature by feature
    pick = np.random.default_rng(5).choice(coarse.shape[0], size=4, replace=False)
    grid = orot.build_grid(target.sphere_points, target.faces)
    want = sum(orot.cost_batch(target.sphere_points, target.faces, tv[f], stencils[0].sphere_points.astype(np.float32),
                               sv[f], coarse[pick], grid=grid) for f in range(2))
    np.testing.assert_allclose(costs[pick], want, rtol=1e-10, atol=0)


@pytest.mark.gpu
def test_pipeline_runs_the_grid_search(native_library, chain, tmp_path):
    from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh
    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline

    paths = []
    for name in ("source_surface", "source_sphere", "target_surface", "target_sphere"):
        paths.append(tmp_path / f"{name}.gii")
        write_gifti_mesh(paths[-1], GiftiMesh(chain[name], chain["faces"]))
    result = run_cat_surface_gpu_pipeline(*paths, tmp_path / "out.gii", device="cuda:0", steps=1, runs=1, avg=False,
                                          sheet_size=(64, 32), rotation_search="euler-grid")
    assert np.all(np.isfinite(result.vertices)) and result.rotation_angle.shape == (3,)
    # within a coarse cell of the reference search's angle on these two meshes
    assert np.abs(result.rotation_angle - chain["rotation_angle"]).max() <= np.deg2rad(10.0)
    torch.cuda.synchronize()
