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
import re

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


def _prototypes() -> dict[str, list[str]]:
    """Parameter names of every entry point declared in include/catsurf_b200.h."""

    from conftest import ROOT

    header = (ROOT / "include" / "catsurf_b200.h").read_text()
    out = {}
    for m in re.finditer(r"CSG_API\s+[\w\s\*]+?\b(csg_\w+)\s*\(([^;]*?)\)\s*;", header, re.S):
        params = [q.strip() for q in m.group(2).split(",") if q.strip() and q.strip() != "void"]
        out[m.group(1)] = [re.findall(r"(\w+)\s*$", q)[0] for q in params]
    return out


# Pointers the header documents as optional (NULL selects a documented behaviour).
OPTIONAL = {
    "csg_areal_sweeps_noalloc": {"status_out"},
    "csg_dartel_data_backward": {"grad_scale"},
    "csg_dartel_expdef": {"jac_out"},
    "csg_dartel_objfun": {"weights"},
    "csg_dartel_smalldef": {"map_out", "jac_out"},
    "csg_dartel_squaring": {"map_out", "jac_out", "scratch_map_out"},
    "csg_depth_potential": {"normals", "areas"},
    "csg_read_status": {"where"},
    "csg_gifti_decode": {"chunk_lengths", "adler32_out"},
    "csg_rotation_grid_build": {"cell_faces"},
    "csg_rotation_grid_build_device": {"cell_faces"},
    # host builders read the neighbour array only where an offset range is non-empty
    "csg_dependency_levels": {"nbr"},
    "csg_greedy_colours": {"nbr"},
    "csg_mesh_neighbours": {"nbr"},
}
# Entry points whose other arguments, zero-filled, already fail a data check
# (zero sphere points, an empty surface record): one-at-a-time says nothing there.
DATA_CHECKED = {"csg_feature_smooth_values", "csg_normalise_sphere", "csg_rotation_cost_batch", "csg_stencil_build",
                "csg_stencil_build_device", "csg_rotation_cost_host"}
# Small valid values for integer parameters (by name); others are 8.
INT_VALUES = {"dtype": 0, "arithmetic": 0, "stop_at": 1, "tile": 256, "solver": 0, "series": 1, "k": 1, "n_levels": 1,
              "level_stride": 1, "iterations": 2, "project_every": 0, "code": 0, "rtype": 1, "checkpoint_every": 1,
              "n_candidates": 1, "n_surfaces": 1, "capacity": 1 << 16, "grid_size": 4, "margin": 1,
              "threads_per_cta": 0, "lanes_per_vertex": 0, "lanes_per_row": 0, "n_ctas": 0, "max_iter": 1,
              "gzip": 0}


@pytest.mark.skipif(__import__("torch").cuda.is_available(),
                    reason="passes host buffers where device pointers go; only safe where no GPU can be reached")
def test_each_pointer_is_checked_on_its_own(native):
    """Null one pointer argument at a time, every other argument valid-looking.

    With all pointers set (zero-filled host buffers, sizes that fit) an entry
    point gets past its argument checks: to a host result, or to the first
    CUDA call, which fails on a machine without a GPU.  Nulling any one
    required pointer must turn that into CSG_ERR_ARG; the stream and the
    pointers the header documents as optional are exempt.
    """

    lib = native.library()
    protos = _prototypes()
    buffers = [np.zeros(1 << 22, dtype=np.uint8) for _ in range(32)]
    bases = [(b.ctypes.data + 255) // 256 * 256 for b in buffers]
    checked = 0
    for name in _status_entries(native):
        _, argtypes = native.SIGNATURES[name]
        params = protos[name]
        assert len(params) == len(argtypes), name

        def call(null=None):
            for b in buffers:
                b[:] = 0
            args = []
            for i, t in enumerate(argtypes):
                if t is ctypes.c_void_p:
                    args.append(None if i == null else bases[i])
                elif t in (ctypes.c_double, ctypes.c_float):
                    args.append(1.0)
                elif t is ctypes.c_size_t:
                    args.append(1 << 20)
                else:
                    args.append(INT_VALUES.get(params[i], 8))
            return getattr(lib, name)(*args)

        baseline = call()
        if name in DATA_CHECKED:
            assert baseline == native.CSG_ERR_ARG, (name, baseline, native.last_error())
            continue
        assert baseline != native.CSG_ERR_ARG, (name, native.last_error())
        for i, t in enumerate(argtypes):
            if t is not ctypes.c_void_p or params[i] == "stream" or params[i] in OPTIONAL.get(name, ()):
                continue
            rc = call(i)
            assert rc == native.CSG_ERR_ARG, (name, params[i], rc, native.last_error())
            checked += 1
    assert checked >= 150


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


def test_operands_on_another_device_are_rejected(monkeypatch):
    """The native entry points launch on the current device: operands elsewhere raise ValueError first."""

    import types

    import torch

    from cat_surface_gpu_b200 import _native

    monkeypatch.setattr(torch.cuda, "current_device", lambda: 0)
    here = types.SimpleNamespace(device=torch.device("cuda", 0))
    there = types.SimpleNamespace(device=torch.device("cuda", 1))
    _native.require_current_device(here, torch.device("cuda", 0), torch.device("cuda"))
    with pytest.raises(ValueError, match="cuda:1"):
        _native.require_current_device(here, there)
    with pytest.raises(ValueError, match="CUDA tensors"):
        _native.require_current_device(types.SimpleNamespace(device=torch.device("cpu")))
    with pytest.raises(ValueError, match="cuda:1"):
        _native.stream_handle(like=there)
    with pytest.raises(ValueError, match="cuda:1"):
        _native.stream_handle(types.SimpleNamespace(device=torch.device("cuda", 1), cuda_stream=0))
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 1)
    assert _native.stream_handle(types.SimpleNamespace(device=torch.device("cuda", 1), cuda_stream=1234),
                                 like=[there]) == 1234
