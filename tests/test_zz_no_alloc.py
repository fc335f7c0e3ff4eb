"""The allocation-free Surf2Sphere sweep entry point (``csg_areal_sweeps_noalloc``).

Some callers of this library cannot call cudaMalloc -- code running inside a
CUDA stream capture, hosts whose device memory belongs to their own pool
allocator, bindings without a device allocator.  For them the sweep kernel's
working memory lives in a fixed device array inside the library.  These tests
call that entry point through the C ABI and check that its output is exactly
the output of the regular entry point (``csg_areal_sweeps``, which takes a
caller-provided scratch buffer) on two calls in a row -- the second call on a
different mesh, so leftovers of the first call in the shared array must not
matter -- and that meshes larger than the array are rejected before any work.

This file is collected last on purpose: it exercises state that persists for
the whole process (the library's device array).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import load_surf2sphere_golden

pytestmark = pytest.mark.gpu


def _plan(faces, n):
    from cat_surface_gpu_b200.surf2sphere import SweepPlan

    return SweepPlan.build(faces, n)


def _noalloc(lib, points, plan_device, plan, iterations, project_every, radius, arithmetic=0):
    from cat_surface_gpu_b200 import _native

    status = ctypes.c_int(12345)
    rc = lib.csg_areal_sweeps_noalloc(
        points.data_ptr(), points.shape[0], plan_device["slot_off"].data_ptr(), plan_device["slot_tri"].data_ptr(),
        plan_device["order"].data_ptr(), plan_device["level_begin"].data_ptr(), plan_device["level_end"].data_ptr(),
        plan.n_levels, plan.level_stride, plan.max_degree, iterations, project_every, radius, arithmetic, 0, 0, 0,
        2.0, ctypes.addressof(status), _native.stream_handle(),
    )
    return rc, status.value


def _regular(points, plan_device, plan, iterations, project_every, radius, arithmetic="cat"):
    from cat_surface_gpu_b200 import surf2sphere

    scratch = surf2sphere.areal_sweeps_device(points, plan_device, plan, iterations=iterations,
                                              project_every=project_every, radius=radius, arithmetic=arithmetic)
    torch.cuda.synchronize()
    assert surf2sphere.read_status(scratch) == (0, 0)


def test_noalloc_matches_regular_entry_point_on_two_calls(native_library):
    from cat_surface_gpu_b200 import synthetic

    g = load_surf2sphere_golden("c1")
    small_v, small_f = synthetic.folded_icosphere(3, seed=21)
    cases = [
        (g["prefix"], g["faces"], 1300, 1000),  # 10,242 vertices, crosses one projection
        (small_v, small_f, 41, 10),  # a different, smaller mesh on the second call
    ]
    for vertices, faces, iterations, project_every in cases:
        plan = _plan(faces, vertices.shape[0])
        plan_device = plan.to_device(torch.device("cuda"))
        radius = float(np.sqrt(np.max(np.sum(vertices.astype(np.float64) ** 2, axis=1))))
        expected = torch.from_numpy(np.ascontiguousarray(vertices, dtype=np.float32)).cuda()
        _regular(expected, plan_device, plan, iterations, project_every, radius)
        got = torch.from_numpy(np.ascontiguousarray(vertices, dtype=np.float32)).cuda()
        rc, status = _noalloc(native_library, got, plan_device, plan, iterations, project_every, radius)
        assert rc == 0 and status == 0
        np.testing.assert_array_equal(got.cpu().numpy(), expected.cpu().numpy())


def test_noalloc_float64_matches_regular_entry_point(native_library):
    """The float64 mode (a double4 working copy in the same array), twice in a row, bit for bit."""

    from cat_surface_gpu_b200 import _native

    g = load_surf2sphere_golden("c1")
    plan = _plan(g["faces"], g["prefix"].shape[0])
    plan_device = plan.to_device(torch.device("cuda"))
    vertices = g["prefix"].astype(np.float64)
    radius = float(np.sqrt(np.max(np.sum(vertices ** 2, axis=1))))
    expected = torch.from_numpy(np.ascontiguousarray(vertices)).cuda()
    _regular(expected, plan_device, plan, 1100, 1000, radius, arithmetic="fp64")
    for _ in range(2):
        got = torch.from_numpy(np.ascontiguousarray(vertices)).cuda()
        rc, status = _noalloc(native_library, got, plan_device, plan, 1100, 1000, radius, _native.ARITH["fp64"])
        assert rc == 0 and status == 0
        np.testing.assert_array_equal(got.cpu().numpy(), expected.cpu().numpy())


def test_noalloc_rejects_meshes_larger_than_its_array(native_library):
    from cat_surface_gpu_b200 import _native

    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    status = ctypes.c_int(0)
    rc = native_library.csg_areal_sweeps_noalloc(
        dummy.data_ptr(), 262145, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
        dummy.data_ptr(), 1, 1, 1, 2, 0, 1.0, 0, 0, 0, 0, 2.0, ctypes.addressof(status), _native.stream_handle(),
    )
    assert rc == _native.CSG_ERR_ARG
    assert "262,144" in _native.last_error() or "262144" in _native.last_error()
    rc = native_library.csg_areal_sweeps_noalloc(
        dummy.data_ptr(), 131073, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
        dummy.data_ptr(), 1, 1, 1, 2, 0, 1.0, 2, 0, 0, 0, 2.0, ctypes.addressof(status), _native.stream_handle(),
    )
    assert rc == _native.CSG_ERR_ARG
