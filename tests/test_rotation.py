"""Rotation search: oracle pinned to the reference's outputs; native kernel parity.

``tests/golden/rotation_golden.npz`` holds the reference's own results
(torch CPU path) on a seeded sphere: grid CSR, candidate costs for the 46
seeds plus random angles, and the full seed + Nelder-Mead search.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import rotation as orot

R = np.load(GOLDEN / "rotation_golden.npz")
GRID = int(R["grid_size"])


def _oracle_cost(angles):
    return orot.cost_batch(R["target_points"], R["target_faces"], R["target_values"], R["source_points"],
                           R["source_values"], angles, grid=(R["grid_offsets"], R["grid_faces"]), grid_size=GRID)


def test_oracle_matches_reference_costs_and_search():
    off, flat = orot.build_grid(R["target_points"], R["target_faces"], GRID, 1)
    np.testing.assert_array_equal(off, R["grid_offsets"])
    np.testing.assert_array_equal(flat, R["grid_faces"])
    costs = _oracle_cost(R["angles"])
    np.testing.assert_allclose(costs, R["costs"], rtol=1e-6)
    best = int(np.argmin(costs[:46]))
    np.testing.assert_array_equal(orot.seed_angles()[best], R["seed_angle"])
    angle, cost, iterations = orot.nelder_mead(_oracle_cost, orot.seed_angles()[best])
    np.testing.assert_allclose(angle, R["angle"], atol=1e-9)
    np.testing.assert_allclose(cost, float(R["cost"]), rtol=1e-5)
    assert iterations == int(R["iterations"])


def test_seed_grid_order_like_reference():
    """Reference test_surface_rotation.py:138-146."""

    from cat_surface_gpu_b200.surface_rotation import official_seed_grid_angles

    angles = official_seed_grid_angles()
    assert angles.shape == (46, 3)
    np.testing.assert_array_equal(angles[0], (0.0, 0.0, 0.0))
    np.testing.assert_array_equal(angles[1], (-0.6, -0.3, -0.3))
    np.testing.assert_array_equal(angles[23], (0.0, 0.0, 0.0))
    np.testing.assert_array_equal(angles[-1], (0.6, 0.3, 0.3))


def test_native_grid_builder_matches_reference(native_library):
    from cat_surface_gpu_b200.surface_rotation import RotationGridIndex

    index = RotationGridIndex.from_geometry(R["target_points"], R["target_faces"], grid_size=GRID, margin=1,
                                            include_dense_candidate_table=True)
    np.testing.assert_array_equal(index.candidate_offsets, R["grid_offsets"])
    np.testing.assert_array_equal(index.candidate_faces, R["grid_faces"])
    assert index.max_candidates == int(np.diff(R["grid_offsets"]).max())
    row = int(np.argmax(np.diff(R["grid_offsets"])))
    width = int(np.diff(R["grid_offsets"])[row])
    np.testing.assert_array_equal(index.candidate_table[row, :width],
                                  R["grid_faces"][R["grid_offsets"][row]: R["grid_offsets"][row] + width])


@pytest.fixture(scope="module")
def device_index(native_library):
    from cat_surface_gpu_b200.surface_rotation import RotationGridIndex

    return RotationGridIndex.from_geometry(R["target_points"], R["target_faces"], grid_size=GRID, margin=1,
                                           include_dense_candidate_table=False).to("cuda")



def _matrices_per_entry(angles):
    """Rz (Ry Rx) column-major float32, one numpy operation per matrix entry (the reference's form)."""

    a = np.asarray(angles, dtype=np.float64).reshape(-1, 3).astype(np.float32)
    al, be, ga = a[:, 0], a[:, 1], a[:, 2]
    z, o = np.zeros_like(al), np.ones_like(al)
    rx = np.stack((o, z, z, z, np.cos(al), np.sin(al), z, -np.sin(al), np.cos(al)), axis=1)
    ry = np.stack((np.cos(be), z, np.sin(be), z, o, z, -np.sin(be), z, np.cos(be)), axis=1)
    rz = np.stack((np.cos(ga), np.sin(ga), z, -np.sin(ga), np.cos(ga), z, z, z, o), axis=1)
    first, out = np.empty_like(rx), np.empty_like(rx)
    for r in range(3):
        for c in range(3):
            first[:, r + 3 * c] = (ry[:, r] * rx[:, 3 * c] + ry[:, r + 3] * rx[:, 1 + 3 * c]) + ry[:, r + 6] * rx[:, 2 + 3 * c]
    for r in range(3):
        for c in range(3):
            out[:, r + 3 * c] = (rz[:, r] * first[:, 3 * c] + rz[:, r + 3] * first[:, 1 + 3 * c]) + rz[:, r + 6] * first[:, 2 + 3 * c]
    return out


def test_rotation_matrices_bit_identical_to_per_entry_form():
    from cat_surface_gpu_b200.surface_rotation import official_seed_grid_angles, rotation_matrices_flat

    rng = np.random.default_rng(7)
    batches = [official_seed_grid_angles(), np.zeros((1, 3)), np.array([[0.0, np.pi / 2.0, -0.0]])]
    batches += [rng.uniform(-7.0, 7.0, (n, 3)) for n in (1, 2, 3, 4, 5, 17, 64, 1000)]
    for angles in batches:
        got, want = rotation_matrices_flat(angles), _matrices_per_entry(angles)
        assert got.dtype == np.float32 and got.shape == want.shape
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))

@pytest.mark.gpu
def test_costs_match_oracle_and_reference(device_index):
    got = device_index.cost_batch(R["source_points"], R["source_values"], R["target_values"], R["angles"]).cpu().numpy()
    np.testing.assert_allclose(got, _oracle_cost(R["angles"]), rtol=1e-12)
    np.testing.assert_allclose(got, R["costs"], rtol=1e-6)


@pytest.mark.gpu
def test_rotate_points_identity_and_convention(device_index):
    pts = torch.as_tensor(R["source_points"])
    rotated = device_index.rotate_points(pts, torch.zeros((1, 3), dtype=torch.float64))
    np.testing.assert_array_equal(rotated[0].cpu().numpy(), R["source_points"])
    got = device_index.rotate_points(pts, R["angles"][:5]).cpu().numpy()
    np.testing.assert_allclose(got, R["rotated"], rtol=0, atol=3e-7)


@pytest.mark.gpu
def test_search_matches_reference(device_index):
    result = device_index.search_rotation(R["source_points"], R["source_values"], R["target_values"])
    np.testing.assert_array_equal(result.seed_angle.cpu().numpy(), R["seed_angle"])
    np.testing.assert_allclose(result.seed_costs.cpu().numpy(), R["seed_costs"], rtol=1e-6)
    np.testing.assert_allclose(result.angle.cpu().numpy(), R["angle"], atol=1e-6)
    np.testing.assert_allclose(float(result.cost), float(R["cost"]), rtol=1e-5)
    assert result.iterations == int(R["iterations"])
    np.testing.assert_allclose(result.rotation_matrix.cpu().numpy(), R["matrix"], atol=1e-6)


@pytest.mark.gpu
def test_batched_surfaces_equal_single_surface_costs(native_library):
    """Uneven surfaces and candidate counts in one persistent launch == per-surface launches."""

    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.surface_rotation import RotationGridIndex, batched_costs

    rng = np.random.default_rng(3)
    indices, inputs, angle_sets = [], [], []
    for n_sub, count in ((3, 7), (4, 130), (2, 33)):
        tp, tf = synthetic.unit_icosphere(n_sub)
        sp = tp + rng.normal(scale=0.02, size=tp.shape)
        sp /= np.linalg.norm(sp, axis=1, keepdims=True)
        index = RotationGridIndex.from_geometry(tp, tf, grid_size=24, margin=1,
                                                include_dense_candidate_table=False).to("cuda")
        indices.append(index)
        inputs.append(index.prepare_cost_inputs(sp.astype(np.float32), np.sin(3 * sp[:, 0]), np.sin(3 * tp[:, 0])))
        angle_sets.append(rng.uniform(-0.5, 0.5, size=(count, 3)))
    together = batched_costs(indices, inputs, angle_sets)
    for index, inp, angles, got in zip(indices, inputs, angle_sets, together):
        alone = index.cost_batch_prepared(inp, angles)
        np.testing.assert_array_equal(got.cpu().numpy(), alone.cpu().numpy())


@pytest.mark.gpu
def test_two_features_and_quaternion_candidates(native_library):
    """F = 2 features sum both SSDs; quaternion matrices rotate like Euler matrices of the same rotation."""

    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.surface_rotation import (RotationGridIndex, batched_costs, quaternion_matrices,
                                                       rotation_matrices_flat, uniform_quaternions)

    rng = np.random.default_rng(9)
    tp, tf = synthetic.unit_icosphere(4)
    sp = tp + rng.normal(scale=0.02, size=tp.shape)
    sp = (sp / np.linalg.norm(sp, axis=1, keepdims=True)).astype(np.float32)
    index = RotationGridIndex.from_geometry(tp, tf, grid_size=32, margin=1,
                                            include_dense_candidate_table=False).to("cuda")
    f_src = np.stack([np.sin(3 * sp[:, 0]), np.cos(2 * sp[:, 1] + sp[:, 2])])
    f_tgt = np.stack([np.sin(3 * tp[:, 0]), np.cos(2 * tp[:, 1] + tp[:, 2])])
    both = index.prepare_cost_inputs(sp, f_src, f_tgt)
    one = [index.prepare_cost_inputs(sp, f_src[k], f_tgt[k]) for k in range(2)]
    quats = uniform_quaternions(64, seed=4)
    mats = quaternion_matrices(quats)
    got = batched_costs([index], [both], matrix_sets=[mats])[0].cpu().numpy()
    parts = [batched_costs([index], [inp], matrix_sets=[mats])[0].cpu().numpy() for inp in one]
    np.testing.assert_allclose(got, parts[0] + parts[1], rtol=1e-12)
    # matrices given directly reproduce the Euler-angle path bit for bit
    angles = rng.uniform(-0.6, 0.6, size=(16, 3))
    np.testing.assert_array_equal(batched_costs([index], [one[0]], matrix_sets=[rotation_matrices_flat(angles)])[0]
                                  .cpu().numpy(), index.cost_batch_prepared(one[0], angles).cpu().numpy())
    # a quaternion and its negative are the same rotation; rows of R are orthonormal
    np.testing.assert_allclose(quaternion_matrices(-quats), mats, atol=1e-7)
    r = mats.reshape(-1, 3, 3).astype(np.float64)
    np.testing.assert_allclose(r @ r.transpose(0, 2, 1), np.broadcast_to(np.eye(3), r.shape), atol=1e-6)


@pytest.mark.gpu
def test_device_grid_build_equals_host_build(native_library):
    """The GPU candidate grid has the host builder's cells and per-cell face order."""

    from cat_surface_gpu_b200.surface_rotation import RotationGridIndex, RotationGridIndexDevice
    from cat_surface_gpu_b200.surface_stencil import resampling_sphere

    rng = np.random.default_rng(5)
    points, faces = resampling_sphere(6)
    points = points + rng.normal(scale=1e-3, size=points.shape)
    for grid_size, margin in ((128, 1), (37, 0), (16, 3)):
        host = RotationGridIndex.from_geometry(points, faces, grid_size=grid_size, margin=margin,
                                               include_dense_candidate_table=False)
        dev = RotationGridIndexDevice.build(points, faces, device="cuda", grid_size=grid_size, margin=margin)
        np.testing.assert_array_equal(dev.candidate_offsets.cpu().numpy(), host.candidate_offsets)
        np.testing.assert_array_equal(dev.candidate_faces.cpu().numpy(), host.candidate_faces)


@pytest.mark.gpu
def test_tetrahedron_known_answers(native_library):
    """Reference test_surface_rotation.py:37-62 and 149-202: identity cost 0, first-minimum rules."""

    from cat_surface_gpu_b200.surface_rotation import RotationGridIndex

    points = np.asarray(((1.0, 0.0, 0.0), (-1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)), dtype=np.float32)
    faces = np.asarray(((0, 2, 3), (2, 1, 3), (1, 0, 3), (0, 1, 2)), dtype=np.int32)
    index = RotationGridIndex.from_geometry(points, faces, grid_size=16, margin=16).to("cuda")
    values = np.array([1.0, 2.0, 3.0, 4.0])
    costs = index.cost_batch(points, values, values, np.zeros((1, 3)))
    assert float(costs[0]) == 0.0
    zeros = np.zeros(4)
    best_angle, best_cost, seed_costs = index.coarse_seed_search(points, zeros, zeros)
    assert seed_costs.shape == (46,)
    np.testing.assert_array_equal(best_angle.cpu().numpy(), np.zeros(3))
    assert float(best_cost) == 0.0
    angle, cost, iterations = index.refine_nelder_mead(points, zeros, zeros, np.zeros(3))
    np.testing.assert_array_equal(angle.cpu().numpy(), np.zeros(3))
    assert float(cost) == 0.0 and iterations == 1


@pytest.mark.gpu
def test_triangle_records_give_the_same_costs(native_library):
    """Costs with precomputed triangle records equal costs formed per query, bit for bit."""

    import ctypes

    import torch

    from cat_surface_gpu_b200 import _native
    from cat_surface_gpu_b200.surface_rotation import RotationGridIndexDevice, rotation_matrices_flat
    from cat_surface_gpu_b200.surface_stencil import resampling_sphere

    rng = np.random.default_rng(12)
    tp, tf = resampling_sphere(5)
    index = RotationGridIndexDevice.build(tp, tf, device="cuda:0", grid_size=64, margin=1)
    src = rng.normal(size=(20000, 3))
    src = (src / np.linalg.norm(src, axis=1, keepdims=True)).astype(np.float32)
    inputs = index.prepare_cost_inputs(src, np.sin(4 * src[:, 0]).astype(np.float64), np.sin(4 * tp[:, 0]))
    mats = torch.as_tensor(rotation_matrices_flat(rng.uniform(-1, 1, size=(24, 3))), device="cuda:0")
    lib = _native.library()
    out = []
    for records in (None, index.target_records.data_ptr()):
        surface = _native.RotationSurface(
            inputs.source_points.data_ptr(), inputs.source_values.data_ptr(), index.target_triangles.data_ptr(),
            index.target_faces.data_ptr(), inputs.target_values.data_ptr(), index.candidate_offsets.data_ptr(),
            index.candidate_faces.data_ptr(), mats.data_ptr(), src.shape[0], index.grid_size, 24, 1,
            int(index.target_points.shape[0]), records)
        n_src, n_cand = (ctypes.c_int * 1)(src.shape[0]), (ctypes.c_int * 1)(24)
        need = lib.csg_rotation_scratch_bytes(1, ctypes.addressof(n_src), ctypes.addressof(n_cand), 256)
        scratch = torch.empty(int(need), dtype=torch.uint8, device="cuda:0")
        costs = torch.empty(24, dtype=torch.float64, device="cuda:0")
        _native.check(lib.csg_rotation_cost_batch(1, ctypes.addressof(surface), costs.data_ptr(), 256, 0,
                                                  scratch.data_ptr(), scratch.numel(),
                                                  _native.stream_handle(like=costs)), "csg_rotation_cost_batch")
        out.append(costs.cpu().numpy())
    assert np.array_equal(out[0], out[1])
    records = index.target_records.cpu().numpy()
    tri = index.target_triangles.reshape(-1, 9).cpu().numpy()
    assert np.array_equal(records[:, :9], tri)


@pytest.mark.gpu
def test_host_driven_evaluations_equal_the_batched_costs(device_index):
    """csg_rotation_cost_host (the Nelder-Mead evaluations: matrices from page-locked host memory,
    status and costs back in one copy) gives the batched device path's costs bit for bit, for 1 to
    31 candidates, and the batched path takes over above that."""

    inputs = device_index.prepare_cost_inputs(R["source_points"], R["source_values"], R["target_values"])
    costing = device_index._costing(inputs, 64)
    rng = np.random.default_rng(21)
    for count in (1, 3, 4, 31, 32, 40):
        angles = rng.uniform(-0.8, 0.8, size=(count, 3))
        host = costing.evaluate(angles, host=True)
        device = costing.evaluate(angles).cpu().numpy()
        assert host.shape == (count,)
        np.testing.assert_array_equal(host, device)
        np.testing.assert_allclose(host, _oracle_cost(angles), rtol=1e-12)
