"""Surf2Sphere stages 1-5.

CPU: the oracle's restatement (vertex-order Gauss-Seidel, float64 arithmetic
on float32 positions) against the upstream binary's stage-5 output committed
in the Surf2Sphere goldens (after the ellipsoid-to-sphere step), and the
whole conversion (stages 1-5 + 4,999 sweeps) against the binary's final
sphere on the 10,242-vertex mesh.  GPU: ``csg_surf2sphere_preprocess``
against the oracle bit for bit (stop_at 1..5), and ``run_cat_surf2sphere_gpu``
with every stage on the GPU against the binary's final sphere.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import areal as oa
from oracle import preprocess as op


def _golden(name):
    g = np.load(GOLDEN / f"surf2sphere_{name}.npz")
    return {k: g[k] for k in g.files}


@pytest.mark.parametrize("name,bound", [("c1", 5e-5), ("c2", 2e-4)])
def test_oracle_stage5_matches_binary(name, bound):
    g = _golden(name)
    faces = g["faces"].astype(np.int32)
    sphere = oa.ellipsoid_to_sphere(op.preprocess(g["surface"], faces, 5), float(g["source_area"]))
    stats = oa.error_stats(g["prefix"], sphere)
    assert stats["max"] <= bound, stats


def test_oracle_full_conversion_matches_binary():
    g = _golden("c1")
    faces = g["faces"].astype(np.int32)
    area = float(g["source_area"])
    prefix = oa.ellipsoid_to_sphere(op.preprocess(g["surface"], faces, 5), area)
    radius = float(np.sqrt(np.max(np.sum(prefix.astype(np.float64) ** 2, axis=1))))
    final = oa.ellipsoid_to_sphere(oa.areal_sweeps(prefix, faces, iterations=5000, project_every=1000,
                                                   radius=radius), area)
    assert oa.error_stats(g["final"], final)["max"] <= 1e-4


def test_neighbour_csr_is_sorted_unique_ring():
    faces = np.array([[0, 1, 2], [0, 2, 3], [0, 3, 1], [1, 3, 2]], dtype=np.int32)
    off, nb = op.neighbour_csr(faces, 4)
    assert off.tolist() == [0, 3, 6, 9, 12]
    assert nb.tolist() == [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2]


@pytest.mark.gpu
@pytest.mark.parametrize("stop_at", [1, 2, 3, 4, 5])
def test_gpu_preprocess_bit_exact_to_oracle(native_library, stop_at):
    from cat_surface_gpu_b200 import surf2sphere
    from cat_surface_gpu_b200.gifti import GiftiMesh

    g = _golden("c1")
    faces = g["faces"].astype(np.int32)
    topology = surf2sphere.Surf2SphereTopology.from_mesh(GiftiMesh(g["surface"], faces))
    got, _ = surf2sphere.run_surf2sphere_preprocess_cuda(g["surface"], faces, topology, stop_at=stop_at,
                                                         desired_surface_area=float(g["source_area"]),
                                                         device="cuda:0")
    want = op.preprocess(g["surface"], faces, stop_at)
    if stop_at == 5:
        want = oa.ellipsoid_to_sphere(want, float(g["source_area"]))
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_gpu_preprocess_launch_shapes_agree(native_library):
    from cat_surface_gpu_b200 import surf2sphere
    from cat_surface_gpu_b200.gifti import GiftiMesh

    g = _golden("c1")
    faces = g["faces"].astype(np.int32)
    topology = surf2sphere.Surf2SphereTopology.from_mesh(GiftiMesh(g["surface"], faces))
    outs = [surf2sphere.run_surf2sphere_preprocess_cuda(g["surface"], faces, topology, stop_at=4,
                                                        desired_surface_area=1.0, device="cuda:0",
                                                        launch=shape)[0]
            for shape in ({"n_ctas": 148, "threads_per_cta": 512, "lanes_per_vertex": 8},
                          {"n_ctas": 64, "threads_per_cta": 256, "lanes_per_vertex": 4},
                          {"n_ctas": 100, "threads_per_cta": 128, "lanes_per_vertex": 16})]
    for other in outs[1:]:
        np.testing.assert_array_equal(other, outs[0])


@pytest.mark.gpu
def test_gpu_preprocess_shared_memory_rings_match_global_rings(native_library):
    """Rings kept in shared memory (max_degree given) == rings read from global memory (max_degree 0);
    a max_degree below the largest ring is reported as CSG_ERR_ARG in the status word."""

    import torch

    from cat_surface_gpu_b200 import surf2sphere
    from cat_surface_gpu_b200.features import _topology
    from cat_surface_gpu_b200.gifti import GiftiMesh

    g = _golden("c1")
    faces = g["faces"].astype(np.int32)
    n = g["surface"].shape[0]
    topology = surf2sphere.Surf2SphereTopology.from_mesh(GiftiMesh(g["surface"], faces))
    plan = topology.plan
    plan_device = plan.to_device("cuda:0")
    rings = _topology(faces, n, torch.device("cuda:0"))
    faces_device = torch.from_numpy(faces).to("cuda:0")
    outs = []
    for max_degree in (rings[4], 0, rings[4] - 1):
        pts = torch.from_numpy(g["surface"]).to("cuda:0")
        scratch = surf2sphere.preprocess_device(pts, faces_device, rings[:4] + (max_degree,), plan_device, plan,
                                                stop_at=5)
        outs.append((pts.cpu().numpy(), surf2sphere.read_status(scratch)[0]))
    assert outs[0][1] == 0 and outs[1][1] == 0
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    assert outs[2][1] == -1  # CSG_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1", "c2"])
def test_all_stages_on_gpu_match_binary(native_library, tmp_path, name):
    """Stages 1-5, 4,999 sweeps and the ellipsoid step on the GPU vs the upstream binary's stop_at=10 sphere."""

    from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh
    from cat_surface_gpu_b200.surf2sphere import run_cat_surf2sphere_gpu

    g = _golden(name)
    faces = g["faces"].astype(np.int32)
    write_gifti_mesh(tmp_path / "in.gii", GiftiMesh(g["surface"], faces))
    result = run_cat_surf2sphere_gpu(tmp_path / "in.gii", tmp_path / "out.gii", stop_at=10,
                                     preprocess_kernel="triton", device="cuda:0")
    np.testing.assert_array_equal(result.faces, faces)
    stats = oa.error_stats(g["final"], result.vertices)
    print(name, stats)
    assert stats["max"] <= 1e-3
