"""CPU tests of the SurfWarp pipeline's host logic: sphere normalisation and
rotation (bit-exact against the reference chain golden), the native stencil
builder (properties and file round trip), and the command-line front end."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def chain():
    return dict(np.load(GOLDEN / "surfwarp_chain_golden.npz"))


def test_normalise_and_rotate_match_reference_chain(chain):
    from cat_surface_gpu_b200.gpu_pipeline import normalise_sphere, rotate_vertices

    rotated = rotate_vertices(normalise_sphere(chain["source_sphere"]), chain["rotation_angle"])
    assert rotated.dtype == np.float32
    assert np.array_equal(rotated, chain["rotated_initial"])


def test_rotation_matrix_is_orthonormal_and_inverts():
    from cat_surface_gpu_b200.gpu_pipeline import rotation_matrix_from_angles

    pole = np.array([0.0, np.pi / 2.0, 0.0])
    m = rotation_matrix_from_angles(pole).numpy()
    assert np.allclose(m @ m.T, np.eye(3), atol=1e-15)
    # the -avg pole rotation takes the x axis onto the -z axis
    assert np.allclose(np.array([1.0, 0.0, 0.0]) @ m.T, [0.0, 0.0, -1.0], atol=1e-15)
    assert np.allclose(rotation_matrix_from_angles(-pole).numpy() @ m, np.eye(3), atol=1e-15)


def _matrix_by_torch_ops(angles):
    """Rz (Ry Rx) from 0-dim float64 torch operations, one per multiply and add (the reference's form)."""

    import torch

    value = torch.as_tensor(np.asarray(angles, dtype=np.float64)).reshape(-1)
    ca = [torch.cos(a) for a in value.unbind()]
    sa = [torch.sin(a) for a in value.unbind()]
    one, zero = torch.ones((), dtype=torch.float64), torch.zeros((), dtype=torch.float64)
    rx = (one, zero, zero, zero, ca[0], sa[0], zero, -sa[0], ca[0])
    ry = (ca[1], zero, sa[1], zero, one, zero, -sa[1], zero, ca[1])
    rz = (ca[2], sa[2], zero, -sa[2], ca[2], zero, zero, zero, one)

    def product(left, right):
        out = [None] * 9
        for r in range(3):
            for c in range(3):
                out[r + 3 * c] = ((zero + left[r] * right[3 * c]) + left[r + 3] * right[1 + 3 * c]) \
                    + left[r + 6] * right[2 + 3 * c]
        return out

    return torch.stack(product(rz, product(ry, rx))).reshape(3, 3).numpy()


def test_rotation_matrix_bit_identical_to_torch_operations():
    """The matrix is built from float64 Python products; every bit equals the 0-dim torch form."""

    from cat_surface_gpu_b200.gpu_pipeline import rotation_matrix_from_angles

    rng = np.random.default_rng(11)
    cases = [rng.uniform(-4.0, 4.0, 3) for _ in range(400)]
    cases += [np.zeros(3), np.array([0.0, np.pi / 2.0, 0.0]), np.array([-0.0, 0.0, -0.0]),
              np.array([np.pi, -np.pi, 1e-300]), np.array([1e-8, -1e-12, 3e-5])]
    for angles in cases:
        got = rotation_matrix_from_angles(angles).numpy()
        assert got.dtype == np.float64
        np.testing.assert_array_equal(got.view(np.uint64), _matrix_by_torch_ops(angles).view(np.uint64))


def test_shared_resampling_faces_hit_the_identity_cache(native_library):
    """Stencils share one read-only face array; the identity lookup returns the bytes-keyed tables."""

    import torch

    from cat_surface_gpu_b200 import features
    from cat_surface_gpu_b200.surface_stencil import resampling_sphere

    points, faces = resampling_sphere(3)
    assert not faces.flags.writeable and not points.flags.writeable
    with pytest.raises(ValueError):
        faces[0, 0] = 1
    cpu = torch.device("cpu")
    first = features._topology(faces, points.shape[0], cpu)
    assert features._topology(faces, points.shape[0], cpu) is first
    fresh = features._topology(np.array(faces), points.shape[0], cpu)  # a writable copy: the bytes key
    for a, b in zip(first[:4], fresh[:4]):
        assert torch.equal(a, b)
    assert first[4] == fresh[4]


def test_normalise_rejects_degenerate_sphere():
    from cat_surface_gpu_b200.gpu_pipeline import normalise_sphere

    points = np.array([[1.0, 0.0, 0.0], [-1.0, 0.0, 0.0], [0.0, 0.0, 0.0]], dtype=np.float32)
    with pytest.raises(ValueError):
        normalise_sphere(points)
    with pytest.raises(ValueError):
        normalise_sphere(np.zeros((4, 2), dtype=np.float32))


@pytest.fixture(scope="module")
def stencil(native_library, chain):
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    return build_surface_stencil(chain["target_sphere"], chain["faces"], nx=64, ny=32, normalize=True, threads=4)


def test_stencil_builder_properties(stencil, chain):
    n_source = chain["target_sphere"].shape[0]
    assert stencil.sphere_points.shape == (40962, 3) and stencil.faces.shape == (81920, 3)
    assert stencil.sheet_indices.shape == (32, 64, 3)
    # surface barycentrics index the source mesh; sheet barycentrics index the resampling sphere
    for idx, w, bound in ((stencil.surface_indices, stencil.surface_weights, n_source),
                          (stencil.sheet_indices, stencil.sheet_weights, 40962)):
        assert idx.min() >= 0 and idx.max() < bound
        # the closest-polygon rule accepts plane projections up to 1e-3 outside a triangle
        assert w.min() >= -1.1e-3
        assert np.allclose(w.sum(axis=-1), 1.0, atol=1e-9)
    unit = stencil.unit_sphere_points.astype(np.float64)
    assert np.allclose(np.linalg.norm(unit, axis=1), 1.0, atol=1e-6)
    # sphere points are closest points on the flat triangles of the unit input sphere
    norms = np.linalg.norm(stencil.sphere_points, axis=1)
    assert norms.max() <= 1.0 + 1e-12 and norms.min() > 0.999
    # surface barycentrics sit on a triangle next to the resampling direction: the interpolated
    # unit sphere deviates from it by less than one input edge
    edges = unit[chain["faces"][:, 0]] - unit[chain["faces"][:, 1]]
    edge_angle = float(np.mean(np.linalg.norm(edges, axis=1)))
    recon = np.einsum("pk,pkc->pc", stencil.surface_weights, unit[stencil.surface_indices])
    direction = stencil.sphere_points / norms[:, None]
    cosine = np.einsum("pc,pc->p", recon / np.linalg.norm(recon, axis=1, keepdims=True), direction)
    assert cosine.min() > np.cos(edge_angle)


def test_stencil_builder_is_deterministic_across_threads(stencil, chain):
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    other = build_surface_stencil(chain["target_sphere"], chain["faces"], nx=64, ny=32, normalize=True, threads=1)
    for name in ("sphere_points", "surface_indices", "surface_weights", "sheet_indices", "sheet_weights",
                 "unit_sphere_points"):
        assert np.array_equal(getattr(stencil, name), getattr(other, name)), name


def test_stencil_file_round_trip(stencil, tmp_path):
    from cat_surface_gpu_b200.surface_stencil import SurfaceStencil

    path = tmp_path / "s.stencil"
    stencil.to_file(path)
    back = SurfaceStencil.from_file(path)
    assert (back.nx, back.ny, back.source_points) == (stencil.nx, stencil.ny, stencil.source_points)
    for name in ("sphere_points", "faces", "surface_indices", "surface_weights", "sheet_indices", "sheet_weights",
                 "unit_sphere_points"):
        assert np.array_equal(getattr(back, name), getattr(stencil, name)), name
    path.write_bytes(path.read_bytes()[:100])
    with pytest.raises(ValueError):
        SurfaceStencil.from_file(path)


def test_stencil_builder_rejects_bad_topology(native_library):
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

    points = np.eye(3, dtype=np.float32)
    with pytest.raises(ValueError):
        build_surface_stencil(points, np.array([[0, 1, 7]], dtype=np.int32), nx=8, ny=4)


def test_cli_dispatch_and_pipeline_argument_checks(tmp_path):
    from cat_surface_gpu_b200 import cli
    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline

    assert cli.main([]) == 2
    with pytest.raises(SystemExit):
        cli.surfwarp_main(["--help"])
    paths = [tmp_path / f"{i}.gii" for i in range(5)]
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, steps=4)
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, runs=0)
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, rotation_feature_backend="nope")
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, device="cpu")
    # reference 536-548: the solver name, and no provided values with the hybrid backends
    with pytest.raises(ValueError):
        run_cat_surface_gpu_pipeline(*paths, rotation_feature_solver="jacobi")
    for backend in ("cuda-official-geometry", "cuda-official-depth"):
        with pytest.raises(ValueError):
            run_cat_surface_gpu_pipeline(*paths[:5], rotation_values_path=paths[0], rotation_feature_backend=backend)


def test_stable_order_equals_numpy_stable_argsort():
    """The incidence tables' vertex order: 16-bit keys (a radix sort) where they fit, int32 beyond."""

    from cat_surface_gpu_b200.features import _stable_order

    rng = np.random.default_rng(4)
    for n in (3, 1000, 1 << 16, (1 << 16) + 1, 200_000):
        keys = rng.integers(0, n, 50_000).astype(np.int32)
        np.testing.assert_array_equal(_stable_order(keys, n), np.argsort(keys, kind="stable"))


@pytest.mark.parametrize("thread_count", [0, -1, 257])
def test_stencil_thread_count_rejects_invalid_values(thread_count, tmp_path):
    """Reference test_gpu_pipeline.py:11-22: the check runs before any file is read."""

    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline

    paths = [tmp_path / name for name in ("s.white.gii", "s.sphere.gii", "t.white.gii", "t.sphere.gii", "o.gii")]
    with pytest.raises(ValueError, match="stencil_threads"):
        run_cat_surface_gpu_pipeline(*paths, stencil_threads=thread_count)


def test_synthetic_meshes_are_deterministic(tmp_path):
    """The seeded synthetic meshes written as GIFTI twice give the same arrays."""

    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh

    for seed in (1, 2):
        first = synthetic.folded_icosphere(2, seed=seed)
        second = synthetic.folded_icosphere(2, seed=seed)
        write_gifti_mesh(tmp_path / f"a{seed}.gii", GiftiMesh(*first))
        write_gifti_mesh(tmp_path / f"b{seed}.gii", GiftiMesh(*second))
        a, b = read_gifti_mesh(tmp_path / f"a{seed}.gii"), read_gifti_mesh(tmp_path / f"b{seed}.gii")
        np.testing.assert_array_equal(a.vertices, b.vertices)
        np.testing.assert_array_equal(a.faces, b.faces)
        assert a.faces.shape[1] == 3 and a.vertices.shape[1] == 3
