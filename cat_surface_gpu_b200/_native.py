"""ctypes binding of ``libcatsurf_b200.so`` (the C ABI in include/catsurf_b200.h).

The product path has no CPU fallback: if the library is missing or a CUDA
device is absent, calls raise ``RuntimeError`` / ``DeviceUnavailable``.
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_int, c_size_t, c_void_p
from pathlib import Path
import threading

LIBRARY_PATH = Path(__file__).resolve().parent / "libcatsurf_b200.so"

CSG_OK = 0
CSG_ERR_ARG = -1
CSG_ERR_CUDA = -2
CSG_ERR_TIMEOUT = -3
CSG_ERR_LAUNCH = -4
CSG_ERR_TOPOLOGY = -5
CSG_ERR_UNSUPPORTED = -6
CSG_ERR_COVERAGE = -7
CSG_ERR_FORMAT = -8
CSG_ROTATION_HOST_MAX_CANDIDATES = 31

ARITH = {"cat": 0, "fp32": 1, "fp64": 2}
CSG_DTYPE_F32 = 0
CSG_DTYPE_F64 = 1
CSG_DEPTH_SOR = 0
CSG_DEPTH_PCG = 1

_P = c_void_p
_I = c_int

# name -> (restype, argtypes).  Kept in the order of include/catsurf_b200.h.
SIGNATURES: dict[str, tuple[object, list[object]]] = {
    "csg_last_error": (ctypes.c_char_p, []),
    "csg_abi_version": (_I, []),
    "csg_kernel_launches": (ctypes.c_longlong, []),
    "csg_selftest_div3": (_I, [_P, ctypes.c_longlong, _P, _P, _P]),
    "csg_preprocess_scratch_bytes": (c_size_t, [_I, _I]),
    "csg_surf2sphere_preprocess": (_I, [_P, _I, _P, _I, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P, c_size_t, _I,
                                        _I, _I, ctypes.c_double, _P]),
    "csg_ellipsoid_to_sphere": (_I, [_P, _I, c_double, _P, c_size_t, _P]),
    "csg_depth_scratch_bytes": (c_size_t, [_I, _I, _I]),
    "csg_depth_potential": (_I, [_P, _I, _I, _P, _I, _P, _P, _I, c_double, _I, _I, c_double, c_double, _P, _P, _P, _I,
                                 _I, _P, _P, _P, _P, _P, _P, c_size_t, _I, _I, _I, c_double, _P]),
    "csg_mesh_incidence": (_I, [_I, _P, _I, _P, _P]),
    "csg_mesh_neighbours": (_I, [_I, _P, _I, _P, _P, _I]),
    "csg_colour_groups": (_I, [_I, _P, _P, _P, _P]),
    "csg_normalise_sphere": (_I, [_I, _P, _P]),
    "csg_dependency_levels": (_I, [_I, _P, _P, _P]),
    "csg_greedy_colours": (_I, [_I, _P, _P, _P]),
    "csg_areal_plan_build": (_I, [_I, _P, _I, _P, _P, _P, _P, _P, _P]),
    "csg_areal_scratch_bytes": (c_size_t, [_I, _I]),
    "csg_areal_sweeps": (
        _I,
        [_P, _I, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, c_double, _I, _P, c_size_t, _I, _I, _I, c_double, _P],
    ),
    "csg_areal_sweeps_noalloc": (
        _I,
        [_P, _I, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, c_double, _I, _I, _I, _I, c_double, _P, _P],
    ),
    "csg_selftest_barrier_timeout": (_I, [_P, c_size_t, c_double, _P]),
    "csg_dartel_scratch_bytes": (c_size_t, [_I, _I, _I, _I]),
    "csg_dartel_solve": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _I, _P, _I, c_double, _I, _I, _I, _I, _P, c_size_t, _P]),
    "csg_dartel_step": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _I, _P, c_double, _I, _I, _I, _I, _P, c_size_t, _P]),
    "csg_dartel_smalldef": (_I, [_I, _I, _I, _I, _P, c_double, _P, _P, _P]),
    "csg_dartel_compose": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "csg_dartel_jac_div": (_I, [_I, _I, _I, _I, _P, _P, c_double, _P, _P]),
    "csg_dartel_objfun": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, c_size_t, _P]),
    "csg_dartel_squaring": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P, _P, c_size_t, _P]),
    "csg_dartel_regularization": (_I, [_I, _I, _I, _I, _P, _P, _I, _P, _P]),
    "csg_dartel_membrane_apply": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "csg_dartel_relax": (_I, [_I, _I, _I, _I, _P, _P, _P, _I, _P, _P]),
    "csg_dartel_resize": (_I, [_I, _I, _I, _I, _P, _I, _I, _P, _I, _P]),
    "csg_dartel_fmg": (_I, [_I, _I, _I, _I, _P, _P, _P, _I, _I, _P, _I, _I, _P, c_size_t, _P]),
    "csg_dartel_expdef": (_I, [_I, _I, _I, _I, _P, _I, _P, _P, _P, c_size_t, _P]),
    "csg_dartel_sample": (_I, [_I, _I, _I, _P, _I, _P, _P, _P, _P]),
    "csg_dartel_data_scratch_bytes": (c_size_t, [_I, _I, _I, _I, _I, _I]),
    "csg_dartel_data_checkpoints": (_I, [_I, _I]),
    "csg_dartel_data_forward": (_I, [_I, _I, _I, _I, _P, _P, _P, _I, _I, _P, _P, _P, c_size_t, _P]),
    "csg_dartel_data_backward": (_I, [_I, _I, _I, _I, _P, _P, _I, _I, _P, _P, _P, _P, c_size_t, _P]),
    "csg_apply_flow_to_sphere": (_I, [_I, _I, _P, _I, _I, _P, _I, _P, _P]),
    "csg_average_xz": (_I, [_I, _P, _P, _P, _P]),
    "csg_rotation_grid_build": (_I, [_P, _I, _P, _I, _I, _I, _P, _P, ctypes.c_longlong, _P]),
    "csg_rotation_scratch_bytes": (c_size_t, [_I, _P, _P, _I]),
    "csg_rotation_grid_scratch_bytes": (c_size_t, [_I]),
    "csg_rotation_grid_build_device": (_I, [_P, _I, _P, _I, _I, _I, _P, _P, ctypes.c_longlong, _P, _P, c_size_t, _P]),
    "csg_rotation_cost_batch": (_I, [_I, _P, _P, _I, _I, _P, c_size_t, _P]),
    "csg_rotation_triangle_records": (_I, [_P, _I, _P, _P]),
    "csg_rotation_status_offset": (c_size_t, [_I]),
    "csg_rotation_cost_host": (_I, [_P, _P, _P, _P, _I, _P, c_size_t, _P]),
    "csg_rotation_status": (_I, [_P, _I, _P, _P]),
    "csg_feature_resample": (_I, [_I, _I, _P, _P, _P, _P, _P]),
    "csg_feature_sheet_map": (_I, [_I, _P, _P, _P, _P, _P]),
    "csg_feature_scratch_bytes": (c_size_t, [_I, _I, _I, _I]),
    "csg_feature_edge_sum": (_I, [_I, _I, _P, _P, _P, _P, c_size_t, _P]),
    "csg_feature_smooth_geometry": (_I, [_I, _P, _P, _P, _I, _P, _P, c_size_t, _P]),
    "csg_feature_smooth_values": (_I, [_I, _P, _P, _I, _I, _P, _P, _I, _P, _P, _I, _P, _P, c_size_t, _P]),
    "csg_feature_vertex_normals": (_I, [_I, _P, _P, _P, _P, _P, _P]),
    "csg_feature_normal_displacement": (_I, [_I, _P, _P, _P, _P, _P]),
    "csg_feature_curvature2": (_I, [_I, _P, _P, _P, _P, _P, _P]),
    "csg_feature_minmax": (_I, [_I, _I, _P, _P, _P, c_size_t, _P]),
    "csg_stencil_build": (_I, [_P, _I, _P, _I, _P, _I, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "csg_stencil_scratch_bytes": (c_size_t, [_I, _I, _I, _I, _I, _I]),
    "csg_stencil_build_device": (_I, [_P, _I, _P, _I, _P, _I, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P,
                                      c_size_t, _P]),
    "csg_gifti_decode": (_I, [_P, c_size_t, _I, _P, _I, ctypes.c_longlong, _P, c_size_t, _P]),
    "csg_read_status": (_I, [_P, _P, _P, _P]),
}


class RotationSurface(ctypes.Structure):
    _fields_ = [
        ("src_points", c_void_p),
        ("src_values", c_void_p),
        ("triangles", c_void_p),
        ("faces", c_void_p),
        ("tgt_values", c_void_p),
        ("grid_offsets", c_void_p),
        ("grid_faces", c_void_p),
        ("matrices", c_void_p),
        ("n_src", ctypes.c_int32),
        ("grid_size", ctypes.c_int32),
        ("n_candidates", ctypes.c_int32),
        ("n_features", ctypes.c_int32),
        ("n_tgt_points", ctypes.c_int32),
        ("records", c_void_p),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int32),
        ("n_faces", ctypes.c_int32),
        ("n_levels", ctypes.c_int32),
        ("level_stride", ctypes.c_int32),
        ("max_degree", ctypes.c_int32),
        ("n_slots", ctypes.c_int32),
    ]


_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def library() -> ctypes.CDLL:
    """Load the native library once; raise if it has not been built."""

    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIBRARY_PATH.exists():
                raise RuntimeError(
                    f"{LIBRARY_PATH.name} is not built; run `python -m cat_surface_gpu_b200.build` "
                    "(there is no CPU fallback)"
                )
            lib = ctypes.CDLL(str(LIBRARY_PATH))
            for name, (restype, argtypes) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _lib = lib
    return _lib


def last_error() -> str:
    message = library().csg_last_error()
    return message.decode("utf-8", "replace") if message else ""


def check(status: int, what: str) -> int:
    """Raise on a negative status: ValueError for argument errors, RuntimeError otherwise."""

    if status >= 0:
        return status
    message = f"{what}: {last_error()} (status {status})"
    if status in (CSG_ERR_ARG, CSG_ERR_TOPOLOGY):
        raise ValueError(message)
    raise RuntimeError(message)


def ptr(tensor) -> int:
    """Raw address of a torch tensor or numpy array (None -> 0)."""

    if tensor is None:
        return 0
    if hasattr(tensor, "data_ptr"):
        return int(tensor.data_ptr())
    return int(tensor.ctypes.data)


def require_current_device(*operands) -> None:
    """Raise ``ValueError`` unless every operand (tensor or device) is on the current CUDA device.

    The native entry points launch on the CUDA runtime's current device, so a
    device pointer from another GPU would be read through the wrong context.
    """

    import torch

    current = torch.cuda.current_device()
    for operand in operands:
        device = operand if isinstance(operand, torch.device) else getattr(operand, "device", None)
        if device is None:
            continue
        if device.type != "cuda":
            raise ValueError(f"native operands must be CUDA tensors, got one on {device}")
        if device.index is not None and device.index != current:
            raise ValueError(f"operand on cuda:{device.index} but the current device is cuda:{current}; "
                             f"call under torch.cuda.device(cuda:{device.index})")


def stream_handle(stream=None, *, like=None) -> int:
    """cudaStream_t of the given (or the current device's current) torch CUDA stream.

    ``like`` (a tensor, device or sequence of them) must be on the current
    device; the stream must belong to it too.
    """

    import torch

    if like is not None:
        require_current_device(*(like if isinstance(like, (tuple, list)) else (like,)))
    if stream is None:
        stream = torch.cuda.current_stream()
    else:
        require_current_device(stream.device)
    return int(stream.cuda_stream)


def doubles(values) -> "ctypes.Array":
    """A C array of doubles (kept alive by the caller for the call's duration)."""

    values = [float(v) for v in values]
    return (ctypes.c_double * len(values))(*values)


_GRAPH_REPLAYED_KERNELS = 0


def note_graph_replay(kernels: int) -> None:
    """Account the native kernels of one CUDA-graph replay (counted at capture)."""

    global _GRAPH_REPLAYED_KERNELS
    _GRAPH_REPLAYED_KERNELS += int(kernels)


def kernel_launches() -> int:
    """Native kernels launched in this process: direct launches plus kernels replayed from captured graphs."""

    return int(library().csg_kernel_launches()) + _GRAPH_REPLAYED_KERNELS
