"""Stencil feature operators: oracle pinned to the reference; native kernel parity.

``tests/golden/features_golden.npz`` holds the reference's own outputs (torch
CPU path) on a seeded synthetic stencil.  Pure arithmetic steps (resampling,
sheet map, geometry heat smoothing) match bit-for-bit; steps through float32
normals (acos) and float64 exp match to the stated tolerances.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import features as of

F = np.load(GOLDEN / "features_golden.npz")


def _table():
    return of.neighbour_table(F["faces"], F["sphere_points"].shape[0])


def test_oracle_matches_reference_outputs():
    faces, m, tab = F["faces"], F["resampled32"], _table()
    np.testing.assert_array_equal(of.resample_vertices(F["surface"], F["surface_indices"], F["surface_weights"]), F["resampled32"])
    np.testing.assert_array_equal(of.map_values_to_sheet(F["values"], F["sheet_indices"], F["sheet_weights"]), F["sheet"])
    np.testing.assert_array_equal(of.smooth_geometry(m, faces, 50.0, tab), F["smooth_geometry"])
    np.testing.assert_allclose(of.vertex_normals(m, faces), F["normals"], atol=5e-7)
    np.testing.assert_allclose(of.smooth_values(F["values"], m, faces, 5.0, tab), F["smooth_values"], atol=1e-14)
    many = of.smooth_values_many(F["values"], m, faces, (5.0, 5.0 / 3.0), tab)
    np.testing.assert_allclose(many[0], F["smooth_many_0"], atol=1e-14)
    np.testing.assert_allclose(many[1], F["smooth_many_1"], atol=1e-14)
    np.testing.assert_allclose(of.curvature_type5(m, faces, 5.0, tab), F["type5"], atol=1e-6)
    np.testing.assert_allclose(of.curvature_type2(m, faces, 5.0 / 9.0, tab), F["type2"], atol=1e-6)
    sheets = of.curvature_type5_to_sheet_many(m, faces, (5.0, 5.0 / 3.0), F["sheet_indices"], F["sheet_weights"], tab)
    np.testing.assert_allclose(sheets[0], F["sheet5_many_0"], atol=1e-6)
    np.testing.assert_allclose(sheets[1], F["sheet5_many_1"], atol=1e-6)


def test_stencil_file_round_trip(tmp_path):
    from cat_surface_gpu_b200.surface_stencil import SurfaceStencil

    st = SurfaceStencil(F["sphere_points"], F["faces"], F["surface_indices"], F["surface_weights"], F["sheet_indices"],
                        F["sheet_weights"], 64, 32, F["surface"].shape[0], F["unit_sphere_points"])
    st.to_file(tmp_path / "a.stencil")
    back = SurfaceStencil.from_file(tmp_path / "a.stencil")
    for name in ("sphere_points", "faces", "surface_indices", "surface_weights", "sheet_indices", "sheet_weights",
                 "unit_sphere_points"):
        np.testing.assert_array_equal(getattr(back, name), getattr(st, name))
    raw = (tmp_path / "a.stencil").read_bytes()
    (tmp_path / "b.stencil").write_bytes(raw[:-8])
    with pytest.raises(ValueError):
        SurfaceStencil.from_file(tmp_path / "b.stencil")
    (tmp_path / "c.stencil").write_bytes(b"\0" * 32 + raw[32:])
    with pytest.raises(ValueError):
        SurfaceStencil.from_file(tmp_path / "c.stencil")


@pytest.fixture(scope="module")
def device_stencil(native_library):
    from cat_surface_gpu_b200.surface_stencil import SurfaceStencil

    st = SurfaceStencil(F["sphere_points"], F["faces"], F["surface_indices"], F["surface_weights"], F["sheet_indices"],
                        F["sheet_weights"], 64, 32, F["surface"].shape[0], F["unit_sphere_points"])
    return st.to("cuda")


def host(t):
    return t.detach().cpu().numpy()


@pytest.mark.gpu
def test_native_features_match_reference(device_stencil):
    st = device_stencil
    surface = torch.as_tensor(F["surface"]).cuda()
    mapped = st.resample_vertices(surface)
    np.testing.assert_array_equal(host(mapped), F["resampled32"])
    np.testing.assert_array_equal(host(st.resample_vertices(surface.double())), F["resampled64"])
    np.testing.assert_array_equal(host(st.map_values_to_sheet(torch.as_tensor(F["values"]).cuda())), F["sheet"])
    np.testing.assert_array_equal(host(st.smooth_geometry(mapped, 50.0)), F["smooth_geometry"])
    np.testing.assert_allclose(host(st.vertex_normals(mapped)), F["normals"], atol=5e-7)
    values = torch.as_tensor(F["values"]).cuda()
    np.testing.assert_allclose(host(st.smooth_values(values, mapped, 5.0)), F["smooth_values"], atol=1e-13)
    many = st.smooth_values_many(values, mapped, (5.0, 5.0 / 3.0))
    np.testing.assert_allclose(host(many[0]), F["smooth_many_0"], atol=1e-13)
    np.testing.assert_allclose(host(many[1]), F["smooth_many_1"], atol=1e-13)
    np.testing.assert_allclose(host(st.curvature_type5(mapped, 5.0)), F["type5"], atol=1e-6)
    np.testing.assert_allclose(host(st.curvature_type2(mapped, 5.0 / 9.0)), F["type2"], atol=1e-6)
    np.testing.assert_allclose(host(st.curvature_to_sheet(mapped, 5.0 / 9.0, curvtype=2)), F["sheet_type2"], atol=1e-6)
    sheets = st.curvature_type5_to_sheet_many(mapped, (5.0, 5.0 / 3.0))
    np.testing.assert_allclose(host(sheets[0]), F["sheet5_many_0"], atol=1e-6)
    np.testing.assert_allclose(host(sheets[1]), F["sheet5_many_1"], atol=1e-6)


@pytest.mark.gpu
def test_native_features_match_oracle_closely(device_stencil):
    """Against the oracle (same operation order): smoothing chains stay within a few ulp."""

    st = device_stencil
    m = F["resampled32"]
    tab = _table()
    got = host(st.smooth_values_many(torch.as_tensor(F["values"]).cuda(), torch.as_tensor(m).cuda(), (5.0,))[0])
    want = of.smooth_values_many(F["values"], m, F["faces"], (5.0,), tab)[0]
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-14)


@pytest.mark.gpu
def test_smoothing_with_even_and_odd_iteration_counts(device_stencil):
    """Jacobi smoothing never updates in place: both iteration parities match the oracle and repeat exactly."""

    from cat_surface_gpu_b200 import features

    st = device_stencil
    m = F["resampled32"]
    tab = _table()
    mapped = torch.as_tensor(m).cuda()
    values = torch.as_tensor(F["values"]).cuda()
    parities = set()
    for fwhm in (5.0, 10.0, 20.0, 30.0, 40.0):  # 1, 2, 7, 15 and 26 iterations
        iterations, _ = features.heat_parameters(st, mapped, fwhm)
        parities.add(iterations % 2)
        first = host(st.smooth_values(values, mapped, fwhm))
        np.testing.assert_array_equal(host(st.smooth_values(values, mapped, fwhm)), first)
        want = of.smooth_values(F["values"], m, F["faces"], fwhm, tab)
        np.testing.assert_allclose(first, want, rtol=0, atol=1e-13)
    assert parities == {0, 1}


@pytest.mark.gpu
def test_edge_means_read_back_together_equal_single_reads(device_stencil):
    """The batched edge-mean read-back equals one read per surface, and a float32 surface and
    its float64 copy give the same mean (the sums widen float32 coordinates first)."""

    from cat_surface_gpu_b200 import features

    st = device_stencil
    m32 = torch.as_tensor(F["resampled32"], device="cuda:0")
    other = (m32 * 1.01).contiguous()
    singles = [features._edge_mean(st, m32), features._edge_mean(st, other)]
    together = features.edge_means([(st, m32), (st, other), (st, m32.to(torch.float64))])
    assert together[:2] == singles
    assert together[2] == singles[0]
    # the sheets built with the shared mean equal the ones that compute it themselves
    fw = (5.0, 5.0 / 3.0)
    for a, b in zip(features.curvature_type5_to_sheet_many(st, m32, fw),
                    features.curvature_type5_to_sheet_many(st, m32, fw, together[0])):
        assert torch.equal(a, b)
