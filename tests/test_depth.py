"""Depth-potential rotation feature: oracle pinned to the reference; native kernel parity.

``tests/golden/depth_golden.npz`` holds the reference's own outputs
(``rotation_feature.py`` on the torch CPU path) on the seeded synthetic
stencil of ``features_golden.npz``: normals, areas, the system entries, the
colouring, coloured SOR after 20 and 1,000 sweeps, CG, and the normalised
features of both solvers.  The C oracle reproduces every per-vertex quantity,
every system row and both SOR solutions bit for bit; CG goes through whole-
vector dot products whose order differs from torch's and agrees to 1e-10.
The CUDA kernels equal the oracle bit for bit (SOR, CG, normals, areas).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import depth as od
from oracle import features as of

G = np.load(GOLDEN / "depth_golden.npz")
F = np.load(GOLDEN / "features_golden.npz")
FACES = F["faces"]
N = F["sphere_points"].shape[0]


def _groups_from_labels(labels):
    return tuple(np.flatnonzero(labels == c) for c in range(int(labels.max()) + 1))


def test_oracle_matches_reference_depth_golden():
    sm = G["smoothed"]
    tab = of.neighbour_table(FACES, N)
    np.testing.assert_array_equal(
        of.smooth_geometry(of.resample_vertices(G["surface"], F["surface_indices"], F["surface_weights"]), FACES, 15.0,
                           tab), sm)
    system = od.System(sm, FACES)
    np.testing.assert_array_equal(system.normals, G["normals"])
    np.testing.assert_array_equal(system.areas, G["areas"])
    # per row, the reference's COO entries in their order
    order = np.argsort(G["rows"], kind="stable")
    np.testing.assert_array_equal(system.col, G["cols"][order])
    np.testing.assert_array_equal(system.val, G["values"][order])
    groups = od.colour_groups(FACES, N)
    np.testing.assert_array_equal(np.concatenate(groups), np.concatenate(_groups_from_labels(G["colours"])))
    for sweeps in (20, 1000):
        x, its, res = system.sor(groups, sweeps)
        np.testing.assert_array_equal(x, G[f"sor{sweeps}"])
        assert its == sweeps
        assert res == pytest.approx(float(G[f"sor{sweeps}_residual"]), rel=1e-9, abs=1e-15)
    x, its, res = system.pcg(1000, 1.0e-9)
    assert its == int(G["pcg_iterations"])
    np.testing.assert_allclose(x, G["pcg"], rtol=0, atol=1e-10 * np.abs(G["pcg"]).max())
    assert res == pytest.approx(float(G["pcg_residual"]), rel=1e-2)
    feat, its, _ = od.rotation_feature(sm, FACES, groups=groups)
    assert its == 1000
    np.testing.assert_allclose(feat, G["feature_sor"], rtol=0, atol=1e-13)
    sm10 = of.smooth_geometry(of.resample_vertices(G["surface"], F["surface_indices"], F["surface_weights"]), FACES,
                              10.0, tab)
    feat, its, _ = od.rotation_feature(sm10, FACES, solver="pcg")
    assert its == int(G["feature_pcg_iterations"])
    np.testing.assert_allclose(feat, G["feature_pcg"], rtol=0, atol=1e-8)


def test_native_colouring_matches_reference(native_library):
    from cat_surface_gpu_b200.rotation_feature import colour_groups

    got = colour_groups(FACES, N)
    want = _groups_from_labels(G["colours"])
    assert len(got) == len(want)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    # a second, irregular mesh against the oracle's loop
    from cat_surface_gpu_b200 import synthetic

    pts, tri = synthetic.folded_icosphere(3, seed=2, radius_mm=50.0)
    tri = tri[np.random.default_rng(1).permutation(tri.shape[0])]
    for a, b in zip(colour_groups(tri, pts.shape[0]), od.colour_groups(tri, pts.shape[0])):
        np.testing.assert_array_equal(a, b)


def test_colour_major_schedule_is_a_valid_sor_order(native_library):
    """Vertex v of sweep s runs at step s D + f(v): every edge from a lower to a higher colour keeps
    1 <= f(w) - f(v) <= D - 1, so each vertex reads its neighbours' values of the colour sweep order."""

    from cat_surface_gpu_b200.rotation_feature import DepthTopology

    topo = DepthTopology.build(FACES, N, torch.device("cpu"))
    colour = np.empty(N, dtype=np.int64)
    for c, members in enumerate(topo.groups):
        colour[members] = c
    level = np.empty(N, dtype=np.int64)
    order = topo.order.numpy()
    for lv in range(topo.n_levels):
        level[order[int(topo.level_begin[lv]): int(topo.level_end[lv])]] = lv
    e = np.concatenate([FACES[:, [0, 1]], FACES[:, [1, 2]], FACES[:, [2, 0]]]).astype(np.int64)
    lo = np.where(colour[e[:, 0]] < colour[e[:, 1]], e[:, 0], e[:, 1])
    hi = np.where(colour[e[:, 0]] < colour[e[:, 1]], e[:, 1], e[:, 0])
    assert np.all(colour[lo] != colour[hi])
    gap = level[hi] - level[lo]
    assert gap.min() >= 1 and gap.max() <= topo.level_stride - 1
    assert topo.level_stride <= len(topo.groups)
    print("colours", len(topo.groups), "stride", topo.level_stride, "levels", topo.n_levels)


def _stencil_device():
    from cat_surface_gpu_b200.surface_stencil import SurfaceStencil

    st = SurfaceStencil(F["sphere_points"], FACES, F["surface_indices"], F["surface_weights"], F["sheet_indices"],
                        F["sheet_weights"], 64, 32, F["surface"].shape[0], F["unit_sphere_points"])
    return st.to("cuda:0", geometry_dtype=torch.float32)


@pytest.mark.gpu
def test_gpu_sor_and_geometry_equal_oracle(native_library):
    from cat_surface_gpu_b200.rotation_feature import DepthTopology, depth_potential

    topo = DepthTopology.build(FACES, N, torch.device("cuda:0"))
    sm = torch.as_tensor(G["smoothed"], device="cuda:0")
    system = od.System(G["smoothed"], FACES)
    groups = od.colour_groups(FACES, N)
    for sweeps in (0, 1, 20, 1000):
        values, its, res, normals, areas = depth_potential(sm, topo, max_iter=sweeps, with_geometry=True)
        x, _, want_res = system.sor(groups, sweeps)
        np.testing.assert_array_equal(values[0].cpu().numpy(), x)
        assert its == [sweeps] and res[0] == want_res
        np.testing.assert_array_equal(normals[0].cpu().numpy(), system.normals)
        np.testing.assert_array_equal(areas[0].cpu().numpy(), system.areas)
    np.testing.assert_array_equal(values[0].cpu().numpy(), G["sor1000"])


@pytest.mark.gpu
def test_gpu_pcg_equals_oracle(native_library):
    from cat_surface_gpu_b200.rotation_feature import DepthTopology, depth_potential

    topo = DepthTopology.build(FACES, N, torch.device("cuda:0"))
    system = od.System(G["smoothed"], FACES)
    for tol in (1.0e-9, 1.0e-3, 10.0):
        values, its, res = depth_potential(torch.as_tensor(G["smoothed"], device="cuda:0"), topo, solver="pcg",
                                           tolerance=tol)
        x, want_its, want_res = system.pcg(1000, tol)
        np.testing.assert_array_equal(values[0].cpu().numpy(), x)
        assert its == [want_its] and res == [want_res]
    assert its == [0]  # tolerance 10: the zero start is accepted


@pytest.mark.gpu
def test_gpu_batched_sides_equal_single_solves(native_library):
    """Three folded surfaces of one triangulation in one launch == three launches; launch shapes agree."""

    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.rotation_feature import DepthTopology, depth_potential
    from cat_surface_gpu_b200.surface_stencil import resampling_sphere

    sphere, tri = resampling_sphere(5)
    n = sphere.shape[0]
    geoms = []
    for seed in (3, 4, 5):
        r = 50.0 * (1.0 + 0.08 * synthetic.real_sph_harm_sum(sphere, range(4, 16), 0.2, np.random.default_rng(seed)))
        geoms.append((sphere * r[:, None]).astype(np.float32))
    topo = DepthTopology.build(tri, n, torch.device("cuda:0"))
    stack = torch.as_tensor(np.stack(geoms), device="cuda:0")
    for solver, sweeps in (("colored-sor", 200), ("pcg", 1000)):
        together, its, res = depth_potential(stack, topo, solver=solver, max_iter=sweeps)
        for k in range(3):
            alone, its1, res1 = depth_potential(stack[k], topo, solver=solver, max_iter=sweeps,
                                                launch={"n_ctas": 64, "threads_per_cta": 256, "lanes_per_row": 4})
            np.testing.assert_array_equal(together[k].cpu().numpy(), alone[0].cpu().numpy())
            assert its[k] == its1[0] and res[k] == res1[0]
    # against the oracle at this size (SOR, 200 sweeps, first surface)
    system = od.System(geoms[0], tri)
    x, _, _ = system.sor(od.colour_groups(tri, n), 200)
    sor, _, _ = depth_potential(stack[0], topo, max_iter=200, launch={"lanes_per_row": 16})
    np.testing.assert_array_equal(sor[0].cpu().numpy(), x)


@pytest.mark.gpu
def test_gpu_rotation_feature_matches_reference(native_library):
    from cat_surface_gpu_b200.rotation_feature import compute_rotation_feature, compute_rotation_features

    st = _stencil_device()
    surf = torch.as_tensor(G["surface"], device="cuda:0")
    one = compute_rotation_feature(st, surf, heat_fwhm=15.0)
    assert one.iterations == 1000
    np.testing.assert_allclose(one.values.cpu().numpy(), G["feature_sor"], rtol=0, atol=1e-13)
    pcg = compute_rotation_feature(st, surf, heat_fwhm=10.0, solver="pcg")
    assert pcg.iterations == int(G["feature_pcg_iterations"])
    np.testing.assert_allclose(pcg.values.cpu().numpy(), G["feature_pcg"], rtol=0, atol=1e-8)
    both = compute_rotation_features((st, st), (surf, surf), heat_fwhms=(15.0, 10.0), solver="pcg")
    np.testing.assert_array_equal(both[1].values.cpu().numpy(), pcg.values.cpu().numpy())
    given = compute_rotation_feature(st, surf, heat_fwhm=15.0, depth_values=G["sor1000"])
    assert given.iterations == 0
    np.testing.assert_allclose(given.values.cpu().numpy(), G["feature_sor"], rtol=0, atol=1e-13)
    with pytest.raises(ValueError):
        compute_rotation_feature(st, surf, heat_fwhm=15.0, solver="jacobi")
    with pytest.raises(ValueError):
        compute_rotation_feature(st, surf, heat_fwhm=15.0, depth_values=np.zeros(5))
