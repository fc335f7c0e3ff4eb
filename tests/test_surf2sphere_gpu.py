"""GPU parity tests of the Surf2Sphere sweeps (through the C ABI).

The native kernel must be bit-identical to the oracle's sequential
restatement (``oracle/areal_oracle.c``) for every arithmetic mode and launch
shape, and the full Surf2Sphere output must stay within 1e-3 (max, mean,
p99 of per-coordinate error) of the upstream binary's own output stored in
``tests/golden``.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_surf2sphere_golden
from oracle import areal as oracle

pytestmark = pytest.mark.gpu

TOLERANCE = 1e-3  # max / mean / p99 vertex error against the CPU reference


def _prefix_radius(prefix):
    return float(np.sqrt(np.max(np.sum(prefix.astype(np.float64) ** 2, axis=1))))


@pytest.fixture(scope="module")
def s2s(native_library):
    from cat_surface_gpu_b200 import surf2sphere

    assert torch.cuda.is_available()
    return surf2sphere


def _topology(s2s, vertices, faces):
    from cat_surface_gpu_b200.gifti import GiftiMesh

    return s2s.Surf2SphereTopology.from_mesh(GiftiMesh(np.asarray(vertices, dtype=np.float32), faces))


@pytest.fixture(scope="module")
def golden_c1():
    return load_surf2sphere_golden("c1")


@pytest.fixture(scope="module")
def golden_c2():
    return load_surf2sphere_golden("c2")


@pytest.mark.parametrize("arithmetic", ["cat", "fp32", "fp64"])
def test_sweeps_bit_exact_vs_oracle_c1(s2s, golden_c1, arithmetic):
    g = golden_c1
    radius = _prefix_radius(g["prefix"])
    topo = _topology(s2s, g["prefix"], g["faces"])
    dtype = torch.float64 if arithmetic == "fp64" else torch.float32
    out, timings = s2s.run_areal_smoothing_cuda(
        g["prefix"] if arithmetic != "fp64" else g["prefix"].astype(np.float64), g["faces"], topo,
        iterations=5000, project_every=1000, radius=radius, dtype=dtype,
        arithmetic="fp32" if arithmetic == "fp32" else "cat",
    )
    expected = oracle.areal_sweeps(
        g["prefix"] if arithmetic != "fp64" else g["prefix"].astype(np.float64), g["faces"],
        iterations=5000, project_every=1000, radius=radius, arithmetic=arithmetic,
    ).astype(np.float32)
    np.testing.assert_array_equal(out, expected)
    assert timings["iterations_executed"] == 4999.0


def test_surf2sphere_end_to_end_vs_binary_c1(s2s, golden_c1, tmp_path):
    from cat_surface_gpu_b200.gifti import GiftiMesh, read_gifti_mesh, write_gifti_mesh, write_vertices_like

    g = golden_c1
    topo = _topology(s2s, g["prefix"], g["faces"])
    out, _ = s2s.run_areal_smoothing_cuda(
        g["prefix"], g["faces"], topo, iterations=5000, project_every=1000, radius=_prefix_radius(g["prefix"])
    )
    final = s2s.convert_ellipsoid_to_sphere_with_surface_area(out, g["source_area"])
    stats = oracle.error_stats(g["final"], final)
    assert stats["max"] <= TOLERANCE and stats["mean"] <= TOLERANCE and stats["p99"] <= TOLERANCE, stats
    # triangles are carried over byte-for-byte
    write_gifti_mesh(tmp_path / "prefix.gii", GiftiMesh(g["prefix"], g["faces"]))
    write_vertices_like(tmp_path / "prefix.gii", tmp_path / "out.gii", final)
    np.testing.assert_array_equal(read_gifti_mesh(tmp_path / "out.gii").faces, g["faces"])


def test_surf2sphere_c2_bit_exact_and_within_contract(s2s, golden_c2):
    """61,442-vertex mesh: GPU == oracle bit-for-bit; GPU vs binary <= 1e-3."""

    g = golden_c2
    radius = _prefix_radius(g["prefix"])
    topo = _topology(s2s, g["prefix"], g["faces"])
    out, timings = s2s.run_areal_smoothing_cuda(
        g["prefix"], g["faces"], topo, iterations=5000, project_every=1000, radius=radius
    )
    expected = oracle.areal_sweeps(g["prefix"], g["faces"], iterations=5000, project_every=1000, radius=radius)
    np.testing.assert_array_equal(out, expected)
    final = s2s.convert_ellipsoid_to_sphere_with_surface_area(out, g["source_area"])
    stats = oracle.error_stats(g["final"], final)
    assert stats["max"] <= TOLERANCE and stats["mean"] <= TOLERANCE and stats["p99"] <= TOLERANCE, stats
    # FP64 run of the same kernel: stated error of the float32 output
    out64, _ = s2s.run_areal_smoothing_cuda(
        g["prefix"].astype(np.float64), g["faces"], topo, iterations=5000, project_every=1000, radius=radius,
        dtype=torch.float64,
    )
    final64 = s2s.convert_ellipsoid_to_sphere_with_surface_area(out64, g["source_area"])
    stats64 = oracle.error_stats(final64, final)
    print("c2 vs binary", stats, "c2 vs fp64 run", stats64, "seconds", timings["areal_smoothing_seconds"])
    assert stats64["max"] <= TOLERANCE


@pytest.mark.parametrize(
    "launch",
    [
        {"lanes_per_vertex": 4},
        {"lanes_per_vertex": 16},
        {"threads_per_cta": 128},
        {"threads_per_cta": 512, "n_ctas": 37},
        {"n_ctas": 16, "lanes_per_vertex": 8},
    ],
)
def test_launch_shapes_do_not_change_results(s2s, golden_c1, launch):
    g = golden_c1
    radius = _prefix_radius(g["prefix"])
    topo = _topology(s2s, g["prefix"], g["faces"])
    ref, _ = s2s.run_areal_smoothing_cuda(g["prefix"], g["faces"], topo, iterations=1300, project_every=1000, radius=radius)
    out, _ = s2s.run_areal_smoothing_cuda(
        g["prefix"], g["faces"], topo, iterations=1300, project_every=1000, radius=radius, launch=launch
    )
    np.testing.assert_array_equal(out, ref)


def test_edge_cases(s2s):
    # iterations == 1: no sweep at all
    v = np.asarray(((1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1), (5, 5, 5)), dtype=np.float32)
    f = np.asarray(((0, 1, 2), (0, 3, 1), (0, 2, 3), (1, 3, 2)), dtype=np.int32)  # vertex 4 is isolated
    topo = _topology(s2s, v, f)
    out, _ = s2s.run_areal_smoothing_cuda(v, f, topo, iterations=1, project_every=0, radius=1.0)
    np.testing.assert_array_equal(out, v)
    for iterations, project in ((2, 0), (9, 2), (10, 3), (7, 1)):
        out, _ = s2s.run_areal_smoothing_cuda(v, f, topo, iterations=iterations, project_every=project, radius=1.5)
        expected = oracle.areal_sweeps(v, f, iterations=iterations, project_every=project, radius=1.5)
        np.testing.assert_array_equal(out, expected)
    # a single triangle (every vertex has one incident face)
    v1 = np.asarray(((0, 0, 0), (2, 0, 0), (0, 1, 0)), dtype=np.float32)
    f1 = np.asarray(((0, 1, 2),), dtype=np.int32)
    topo1 = _topology(s2s, v1, f1)
    out, _ = s2s.run_areal_smoothing_cuda(v1, f1, topo1, iterations=4, project_every=0, radius=1.0)
    np.testing.assert_array_equal(out, oracle.areal_sweeps(v1, f1, iterations=4, project_every=0, radius=1.0))


def test_argument_errors(s2s, golden_c1):
    g = golden_c1
    topo = _topology(s2s, g["prefix"], g["faces"])
    with pytest.raises(ValueError):
        s2s.run_areal_smoothing_cuda(g["prefix"], g["faces"], topo, iterations=0, project_every=1, radius=1.0)
    with pytest.raises(ValueError):
        s2s.run_areal_smoothing_cuda(g["prefix"], g["faces"], topo, iterations=3, project_every=-1, radius=1.0)
    with pytest.raises(ValueError):
        s2s.run_areal_smoothing_cuda(g["prefix"], g["faces"], topo, iterations=3, project_every=1, radius=1.0, launch={"lanes_per_vertex": 3})
    with pytest.raises(RuntimeError):
        s2s.run_areal_smoothing_cuda(g["prefix"], g["faces"], topo, iterations=3, project_every=1, radius=1.0, device="cpu")


def test_bounded_wait_reports_timeout_and_context_survives(s2s, native_library):
    from cat_surface_gpu_b200 import _native

    scratch = torch.zeros(256, dtype=torch.uint8, device="cuda")
    _native.check(
        native_library.csg_selftest_barrier_timeout(_native.ptr(scratch), 256, 0.05, _native.stream_handle()),
        "selftest",
    )
    torch.cuda.synchronize()
    status, where = s2s.read_status(scratch)
    assert status == _native.CSG_ERR_TIMEOUT and where == 1
    # the context is still usable
    v = np.asarray(((1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1)), dtype=np.float32)
    f = np.asarray(((0, 1, 2), (0, 3, 1), (0, 2, 3), (1, 3, 2)), dtype=np.int32)
    out, _ = s2s.run_areal_smoothing_cuda(v, f, _topology(s2s, v, f), iterations=5, project_every=2, radius=1.0)
    np.testing.assert_array_equal(out, oracle.areal_sweeps(v, f, iterations=5, project_every=2, radius=1.0))


@pytest.mark.gpu
def test_division_by_three_is_correctly_rounded(native_library):
    """The kernels' two-multiply x / 3 equals the IEEE division on 16M doubles across binades and edge cases."""

    from cat_surface_gpu_b200 import _native

    rng = np.random.default_rng(3)
    mant = rng.random(1 << 24) + 1.0
    expo = rng.integers(-1000, 1000, size=mant.size)
    x = np.ldexp(mant, expo) * rng.choice([-1.0, 1.0], size=mant.size)
    x[:8] = [0.0, -0.0, 1.0, 3.0, 6.0, 2.0 ** -1000, 1.7e308, np.nextafter(3.0, 0.0)]
    xd = torch.as_tensor(x, device="cuda")
    a, b = torch.empty_like(xd), torch.empty_like(xd)
    _native.check(native_library.csg_selftest_div3(xd.data_ptr(), xd.numel(), a.data_ptr(), b.data_ptr(),
                                                   _native.stream_handle()), "csg_selftest_div3")
    assert torch.equal(a.view(torch.int64), b.view(torch.int64))
    np.testing.assert_array_equal(a.cpu().numpy(), x / 3.0)


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_device_ellipsoid_step_and_radius_equal_host(s2s, name):
    """csg_ellipsoid_to_sphere and the device projection radius equal the host NumPy arithmetic bit for bit."""

    g = load_surf2sphere_golden(name)
    area = float(g["source_area"])
    for points in (g["prefix"], g["final"]):
        want = s2s.convert_ellipsoid_to_sphere_with_surface_area(points, area)
        dev = torch.from_numpy(np.ascontiguousarray(points, dtype=np.float32)).to("cuda:0")
        got = s2s.ellipsoid_to_sphere_device(dev, area).cpu().numpy()
        np.testing.assert_array_equal(got, want)
        assert s2s.projection_radius_device(dev) == float(np.sqrt(np.max(np.sum(want.astype(np.float64) ** 2, axis=1))))
    zeros = torch.zeros((5, 3), dtype=torch.float32, device="cuda:0")
    np.testing.assert_array_equal(s2s.ellipsoid_to_sphere_device(zeros, 1.0).cpu().numpy(),
                                  s2s.convert_ellipsoid_to_sphere_with_surface_area(np.zeros((5, 3), np.float32), 1.0))
