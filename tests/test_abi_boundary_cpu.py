"""The C ABI's error behaviour, checked without a GPU.

Every entry point that returns a status validates its arguments before it
touches the device: null buffers and bad sizes come back as CSG_ERR_ARG with a
message from csg_last_error(), never as a CUDA error (which is what a call
reaching the device on a machine without a GPU would return).  Host builders
report face indices outside the mesh as CSG_ERR_TOPOLOGY; size queries return 0
for sizes they cannot serve.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

INTS = (ctypes.c_int, ctypes.c_int32, ctypes.c_longlong, ctypes.c_size_t, ctypes.c_int64, ctypes.c_uint64)
# status-returning functions whose integer result is a count, not a status
COUNTS = {"csg_abi_version", "csg_dartel_data_checkpoints"}


def _status_entries(_native):
    return sorted(name for name, (restype, argtypes) in _native.SIGNATURES.items()
                  if restype is ctypes.c_int and argtypes and name not in COUNTS)


@pytest.fixture(scope="module")
def native():
    from cat_surface_gpu_b200 import _native

    _native.library()
    return _native


def test_every_entry_point_rejects_null_buffers_before_the_device(native):
    lib = native.library()
    names = _status_entries(native)
    assert len(names) >= 45
    for name in names:
        _, argtypes = native.SIGNATURES[name]
        args = [1.0 if t in (ctypes.c_double, ctypes.c_float) else (8 if t in INTS else None) for t in argtypes]
        rc = getattr(lib, name)(*args)
        assert rc == native.CSG_ERR_ARG, (name, rc, native.last_error())
        assert native.last_error(), name


def test_empty_inputs_are_no_ops(native):
    lib = native.library()
    assert lib.csg_average_xz(0, None, None, None, None) == 0
    assert lib.csg_feature_resample(native.CSG_DTYPE_F32, 0, None, None, None, None, None) == 0
    assert lib.csg_feature_sheet_map(0, None, None, None, None, None) == 0
    assert lib.csg_average_xz(-1, None, None, None, None) == native.CSG_ERR_ARG


def test_size_queries_return_zero_for_sizes_they_cannot_serve(native):
    lib = native.library()
    assert lib.csg_areal_scratch_bytes(-1, 0) == 0
    assert lib.csg_areal_scratch_bytes(100, 9) == 0  # no such arithmetic
    assert lib.csg_areal_scratch_bytes(100, 0) > 0
    assert lib.csg_preprocess_scratch_bytes(-1, 10) == 0
    assert lib.csg_depth_scratch_bytes(100, 196, 0) == 0  # an empty batch
    assert lib.csg_depth_scratch_bytes(100, 196, 1) > 0
    assert lib.csg_dartel_scratch_bytes(5, 1, 8, 8) == 0  # no such dtype
    assert lib.csg_dartel_scratch_bytes(native.CSG_DTYPE_F32, 1, 8, 8) > 0


def test_host_builders_report_faces_outside_the_mesh(native):
    lib = native.library()
    faces = np.array([[0, 1, 2], [0, 2, 9]], dtype=np.int32)
    off, inc, nbr = np.zeros(4, np.int32), np.zeros(6, np.int32), np.zeros(12, np.int32)
    assert lib.csg_mesh_incidence(3, faces.ctypes.data, 2, off.ctypes.data, inc.ctypes.data) == native.CSG_ERR_TOPOLOGY
    assert "outside" in native.last_error()
    assert lib.csg_mesh_neighbours(3, faces.ctypes.data, 2, off.ctypes.data, nbr.ctypes.data, 12) \
        == native.CSG_ERR_TOPOLOGY
    negative = np.array([[0, 1, -1]], dtype=np.int32)
    assert lib.csg_mesh_incidence(3, negative.ctypes.data, 1, off.ctypes.data, inc.ctypes.data) \
        == native.CSG_ERR_TOPOLOGY
    points, count = np.zeros((3, 3)), ctypes.c_longlong(0)
    offsets = np.zeros(4 ** 3 + 1, np.int32)
    assert lib.csg_rotation_grid_build(points.ctypes.data, 3, faces.ctypes.data, 2, 4, 1, offsets.ctypes.data, None, 0,
                                       ctypes.addressof(count)) == native.CSG_ERR_TOPOLOGY
    sphere, out = np.zeros((3, 3), np.float32), np.zeros((3, 3), np.float32)
    assert lib.csg_normalise_sphere(3, sphere.ctypes.data, out.ctypes.data) == native.CSG_ERR_ARG
    assert "normalised" in native.last_error()
