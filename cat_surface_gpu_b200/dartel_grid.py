"""CAT-Surface 2-D DARTEL operators on a B200 (drop-in for the reference's dartel_grid).

Public names, signatures, shapes and error behaviour follow the reference
module ``src/cat_surface_gpu/dartel_grid.py``; every operator runs a native
sm_100a kernel through the C ABI (``include/catsurf_b200.h``).  There is no
CPU or torch fallback: tensors are moved to the requested CUDA device and a
missing device raises ``DeviceUnavailable``.  The ``kernel`` / ``optimized``
keywords of the reference are accepted for compatibility and do not change
the computation (every path is the single native implementation).

Fields are ``[channels, ny, nx]`` float32 or float64 tensors; maps are
CAT's one-based coordinates; Jacobians are ``(j00, j10, j01, j11)``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import torch

from . import _native
from .device import DeviceUnavailable, resolve_device

__all__ = [
    "DeviceUnavailable",
    "GridSpec",
    "apply_membrane_system",
    "composition",
    "composition_jacobian",
    "dartel_step",
    "expdef",
    "fmg2_membrane",
    "from_c_layout",
    "initialise_objfun",
    "jac_div_smalldef",
    "jacobian_of_displacement",
    "make_identity_map",
    "regularization_operator",
    "relax_membrane",
    "resize_field",
    "resolve_device",
    "sample_field",
    "smalldef_jac",
    "squaring_update",
    "to_c_layout",
]


@dataclass(frozen=True)
class GridSpec:
    """Describe the x and y dimensions of a DARTEL grid."""

    nx: int
    ny: int

    def __post_init__(self) -> None:
        if self.nx < 1 or self.ny < 1:
            raise ValueError(f"Grid dimensions must be positive, got {(self.nx, self.ny)}")

    @property
    def points(self) -> int:
        return self.nx * self.ny

    @classmethod
    def from_shape(cls, shape: Sequence[int]) -> "GridSpec":
        if len(shape) != 3 or shape[0] != 2:
            raise ValueError(f"Grid shape must be [2, ny, nx], got {tuple(shape)}")
        return cls(nx=int(shape[2]), ny=int(shape[1]))


def _dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return _native.CSG_DTYPE_F64
    if dtype == torch.float32:
        return _native.CSG_DTYPE_F32
    raise ValueError(f"DARTEL supports float32 and float64, got {dtype}")


def _tensor(value, device: torch.device, dtype: torch.dtype) -> torch.Tensor:
    return torch.as_tensor(value, dtype=dtype, device=device).contiguous()


def _grid(value, spec: GridSpec, device, dtype, name: str, channels: int = 2) -> torch.Tensor:
    tensor = _tensor(value, device, dtype)
    expected = (channels, spec.ny, spec.nx)
    if tuple(tensor.shape) != expected:
        raise ValueError(f"{name} shape must be {expected}, got {tuple(tensor.shape)}")
    return tensor


def _stream(operand: torch.Tensor) -> int:
    """The current stream, after checking that ``operand`` lives on the current device."""

    return _native.stream_handle(like=operand)


def _call(name: str, *args) -> None:
    lib = _native.library()
    _native.check(getattr(lib, name)(*args), name)


def _scratch(dtype: torch.dtype, device, batch: int, nx: int, ny: int) -> torch.Tensor:
    need = int(_native.library().csg_dartel_scratch_bytes(_dtype_code(dtype), batch, nx, ny))
    return torch.empty(max(need, 256), dtype=torch.uint8, device=device)


def _params(params: Sequence[float]):
    if len(params) != 5:
        raise ValueError(f"regularization parameters must contain 5 values, got {len(params)}")
    return _native.doubles(params)


def _addr(array) -> int:
    return ctypes.addressof(array)


def from_c_layout(value, nx: int, ny: int, components: int = 2, *, device="auto", dtype=torch.float64) -> torch.Tensor:
    """Reshape a flat C-layout buffer to ``[components, ny, nx]`` (reference 148-166)."""

    spec = GridSpec(nx=nx, ny=ny)
    tensor = torch.as_tensor(value, dtype=dtype, device=resolve_device(device))
    if tensor.numel() != components * spec.points:
        raise ValueError(f"CAT C layout requires {components * spec.points} elements, got {tensor.numel()}")
    return tensor.reshape(components, spec.ny, spec.nx).contiguous()


def to_c_layout(value: torch.Tensor) -> torch.Tensor:
    """Flatten ``[components, ny, nx]`` to CAT's C layout (reference 169-171)."""

    if value.ndim != 3:
        raise ValueError(f"Input must be a three-dimensional tensor, got {tuple(value.shape)}")
    return value.contiguous().reshape(-1)


def make_identity_map(spec: GridSpec, *, device="auto", dtype=torch.float64) -> torch.Tensor:
    """CAT's one-based identity coordinate map ``[2, ny, nx]`` (reference 174-187)."""

    target = resolve_device(device)
    x = torch.arange(1, spec.nx + 1, device=target, dtype=dtype).view(1, 1, spec.nx).expand(1, spec.ny, spec.nx)
    y = torch.arange(1, spec.ny + 1, device=target, dtype=dtype).view(1, spec.ny, 1).expand(1, spec.ny, spec.nx)
    return torch.cat((x, y), dim=0).contiguous()


def composition(a, b, *, device="auto", dtype=torch.float64, optimized: bool = True) -> torch.Tensor:
    """Compose two coordinate maps with CAT's mixed boundary conditions (reference 510-531)."""

    target = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(a).shape))
    at = _grid(a, spec, target, dtype, "A")
    bt = _grid(b, spec, target, dtype, "B")
    out = torch.empty_like(at)
    _call("csg_dartel_compose", _dtype_code(dtype), 1, spec.nx, spec.ny, at.data_ptr(), None, bt.data_ptr(), None,
          out.data_ptr(), None, _stream(out))
    return out


def composition_jacobian(a, ja, b, jb, *, device="auto", dtype=torch.float64, optimized: bool = True):
    """(b o a, J_b(a) J_a) (reference 534-587)."""

    target = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(a).shape))
    at = _grid(a, spec, target, dtype, "A")
    bt = _grid(b, spec, target, dtype, "B")
    jat = _grid(ja, spec, target, dtype, "JA", 4)
    jbt = _grid(jb, spec, target, dtype, "JB", 4)
    out = torch.empty_like(at)
    jout = torch.empty_like(jat)
    _call("csg_dartel_compose", _dtype_code(dtype), 1, spec.nx, spec.ny, at.data_ptr(), jat.data_ptr(), bt.data_ptr(),
          jbt.data_ptr(), out.data_ptr(), jout.data_ptr(), _stream(jout))
    return out, jout


def jacobian_of_displacement(displacement, scale: float = 1.0, *, device="auto", dtype=torch.float64) -> torch.Tensor:
    """I + central differences of v * scale / 2 (reference 624-652)."""

    target = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(displacement).shape))
    v = _grid(displacement, spec, target, dtype, "displacement")
    jac = torch.empty((4, spec.ny, spec.nx), dtype=dtype, device=target)
    _call("csg_dartel_smalldef", _dtype_code(dtype), 1, spec.nx, spec.ny, v.data_ptr(), float(scale), None,
          jac.data_ptr(), _stream(jac))
    return jac


def smalldef_jac(displacement, scale: float, *, device="auto", dtype=torch.float64):
    """(id + v * scale, Jacobian) (reference 655-675)."""

    target = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(displacement).shape))
    v = _grid(displacement, spec, target, dtype, "displacement")
    out = torch.empty_like(v)
    jac = torch.empty((4, spec.ny, spec.nx), dtype=dtype, device=target)
    _call("csg_dartel_smalldef", _dtype_code(dtype), 1, spec.nx, spec.ny, v.data_ptr(), float(scale), out.data_ptr(),
          jac.data_ptr(), _stream(jac))
    return out, jac


def jac_div_smalldef(jacobian, displacement, scale: float, *, device="auto", dtype=torch.float64) -> torch.Tensor:
    """J (I + s grad v)^-1 (reference 678-720)."""

    target = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(displacement).shape))
    v = _grid(displacement, spec, target, dtype, "displacement")
    jac = _grid(jacobian, spec, target, dtype, "jacobian", 4)
    out = torch.empty_like(jac)
    _call("csg_dartel_jac_div", _dtype_code(dtype), 1, spec.nx, spec.ny, jac.data_ptr(), v.data_ptr(), float(scale),
          out.data_ptr(), _stream(out))
    return out


def initialise_objfun(source, target, transformation, jacobian, distortion=None, *, device="auto",
                      dtype=torch.float64):
    """Gauss-Newton gradient and Hessian of the SSD term (reference 723-775).

    Returns ``(objective, right_hand [2, ny, nx], hessian [3, ny, nx])``.
    """

    dev = resolve_device(device)
    src = _tensor(source, dev, dtype)
    tgt = _tensor(target, dev, dtype)
    if src.ndim != 2 or tgt.ndim != 2:
        raise ValueError("initialise_objfun source and target must be 2D scalar fields")
    if tuple(src.shape) != tuple(tgt.shape):
        raise ValueError("initialise_objfun source and target must have the same shape")
    spec = GridSpec(nx=int(src.shape[1]), ny=int(src.shape[0]))
    tmap = _grid(transformation, spec, dev, dtype, "transformation")
    jac = _grid(jacobian, spec, dev, dtype, "jacobian", 4)
    weights = None
    if distortion is not None:
        weights = _tensor(distortion, dev, dtype)
        if tuple(weights.shape) != (spec.ny, spec.nx):
            raise ValueError(f"Distortion shape must be {(spec.ny, spec.nx)}")
    rhs = torch.empty((2, spec.ny, spec.nx), dtype=dtype, device=dev)
    hess = torch.empty((3, spec.ny, spec.nx), dtype=dtype, device=dev)
    objective = torch.empty((1,), dtype=dtype, device=dev)
    scratch = _scratch(dtype, dev, 1, spec.nx, spec.ny)
    _call("csg_dartel_objfun", _dtype_code(dtype), 1, spec.nx, spec.ny, src.data_ptr(), tgt.data_ptr(),
          tmap.data_ptr(), jac.data_ptr(), None if weights is None else weights.data_ptr(), rhs.data_ptr(),
          hess.data_ptr(), objective.data_ptr(), scratch.data_ptr(), scratch.numel(), _stream(scratch))
    return objective[0], rhs, hess


def squaring_update(right_hand, hessian, transformation, jacobian, k: int, *, save_transformation: bool = False,
                    return_scratch: bool = False, device="auto", dtype=torch.float64, optimized: bool = True,
                    kernel: str = "auto"):
    """Push the gradient / Hessian through k squaring steps (reference 778-914)."""

    if k < 0:
        raise ValueError(f"squaring step count k must be non-negative, got {k}")
    if kernel not in {"auto", "torch", "triton"}:
        raise ValueError(f"kernel must be 'auto', 'torch', or 'triton', got {kernel!r}")
    dev = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(transformation).shape))
    rhs = _grid(right_hand, spec, dev, dtype, "right_hand")
    hess = _tensor(hessian, dev, dtype)
    if tuple(hess.shape) != (3, spec.ny, spec.nx):
        raise ValueError(f"Hessian shape must be {(3, spec.ny, spec.nx)}")
    tmap = _grid(transformation, spec, dev, dtype, "transformation")
    jac = _grid(jacobian, spec, dev, dtype, "jacobian", 4)
    b_out, a_out = torch.empty_like(rhs), torch.empty_like(hess)
    m_out, j_out, s_out = torch.empty_like(tmap), torch.empty_like(jac), torch.empty_like(tmap)
    scratch = _scratch(dtype, dev, 1, spec.nx, spec.ny)
    _call("csg_dartel_squaring", _dtype_code(dtype), 1, spec.nx, spec.ny, rhs.data_ptr(), hess.data_ptr(),
          tmap.data_ptr(), jac.data_ptr(), int(k), int(bool(save_transformation)), b_out.data_ptr(), a_out.data_ptr(),
          m_out.data_ptr(), j_out.data_ptr(), s_out.data_ptr(), scratch.data_ptr(), scratch.numel(), _stream(scratch))
    result = (b_out, a_out, m_out, j_out)
    return result + (s_out,) if return_scratch else result


def regularization_operator(field, params: Sequence[float], rtype: int = 1, *, device="auto", dtype=torch.float64):
    """Membrane (1), linear-elastic (0) or bending (2) operator (reference 917-1015)."""

    if len(params) != 5:
        raise ValueError(f"regularization parameters must contain 5 values, got {len(params)}")
    if rtype not in {0, 1, 2}:
        raise ValueError(f"regularization type must be 0, 1, or 2, got {rtype}")
    dev = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(field).shape))
    v = _grid(field, spec, dev, dtype, "field")
    out = torch.empty_like(v)
    p = _params(params)
    _call("csg_dartel_regularization", _dtype_code(dtype), 1, spec.nx, spec.ny, v.data_ptr(), _addr(p), int(rtype),
          out.data_ptr(), _stream(out))
    return out


def apply_membrane_system(hessian, field, params: Sequence[float], *, kernel: str = "auto", device="auto",
                          dtype=torch.float64):
    """(H + L_membrane) u (reference 1018-1070)."""

    if kernel not in {"auto", "torch", "triton"}:
        raise ValueError(f"kernel must be 'auto', 'torch', or 'triton', got {kernel!r}")
    dev = resolve_device(device)
    field_t = torch.as_tensor(field)
    spec = GridSpec(nx=int(field_t.shape[-1]), ny=int(field_t.shape[-2]))
    hess = _tensor(hessian, dev, dtype)
    if tuple(hess.shape) != (3, spec.ny, spec.nx):
        raise ValueError(f"Hessian shape must be {(3, spec.ny, spec.nx)}")
    v = _grid(field, spec, dev, dtype, "field")
    out = torch.empty_like(v)
    p = _params(params)
    _call("csg_dartel_membrane_apply", _dtype_code(dtype), 1, spec.nx, spec.ny, hess.data_ptr(), v.data_ptr(),
          _addr(p), out.data_ptr(), _stream(out))
    return out


def relax_membrane(hessian, right_hand, params: Sequence[float], nit: int, initial=None, *, kernel: str = "auto",
                   device="auto", dtype=torch.float64):
    """nit red-black sweeps with a 2x2 point solve (reference 1073-1208).

    As on the reference's CUDA path, an odd x size (other than 1) raises
    ``ValueError``.
    """

    if nit < 0:
        raise ValueError(f"relaxation count must be non-negative, got {nit}")
    if kernel not in {"auto", "torch", "triton"}:
        raise ValueError(f"kernel must be 'auto', 'torch', or 'triton', got {kernel!r}")
    dev = resolve_device(device)
    b = _tensor(right_hand, dev, dtype)
    if b.ndim != 3 or b.shape[0] != 2:
        raise ValueError("right_hand must have shape [2, ny, nx]")
    spec = GridSpec(nx=int(b.shape[2]), ny=int(b.shape[1]))
    hess = _tensor(hessian, dev, dtype)
    if tuple(hess.shape) != (3, spec.ny, spec.nx):
        raise ValueError(f"Hessian shape must be {(3, spec.ny, spec.nx)}")
    if len(params) != 5:
        raise ValueError(f"regularization parameters must contain 5 values, got {len(params)}")
    if spec.nx % 2 == 1 and spec.nx != 1:
        raise ValueError("CUDA red-black relaxation requires an even x dimension")
    u = torch.zeros_like(b) if initial is None else _grid(initial, spec, dev, dtype, "initial").clone()
    p = _params(params)
    _call("csg_dartel_relax", _dtype_code(dtype), 1, spec.nx, spec.ny, hess.data_ptr(), b.data_ptr(), _addr(p),
          int(nit), u.data_ptr(), _stream(u))
    return u


def resize_field(field, target: GridSpec, *, kernel: str = "auto", device="auto", dtype=torch.float64):
    """Separable quadratic B-spline resize of ``[channels, ny, nx]`` (reference 239-305)."""

    if kernel not in {"auto", "torch", "triton"}:
        raise ValueError(f"kernel must be 'auto', 'torch', or 'triton', got {kernel!r}")
    dev = resolve_device(device)
    value = _tensor(field, dev, dtype)
    if value.ndim == 2:
        value = value.unsqueeze(0)
    if value.ndim != 3:
        raise ValueError(f"resize_field expects [channel, y, x], got {tuple(value.shape)}")
    out = torch.empty((value.shape[0], target.ny, target.nx), dtype=dtype, device=dev)
    _call("csg_dartel_resize", _dtype_code(dtype), int(value.shape[0]), int(value.shape[2]), int(value.shape[1]),
          value.data_ptr(), target.nx, target.ny, out.data_ptr(), 0, _stream(out))
    return out


def fmg2_membrane(hessian, right_hand, params: Sequence[float], cycles: int = 3, nit: int = 3, initial=None, *,
                  kernel: str = "auto", device="auto", dtype=torch.float64, assume_initial_nonzero: bool = False):
    """Full multigrid for (H + L_membrane) u = b (reference 1211-1417)."""

    if cycles < 0 or nit < 0:
        raise ValueError(f"FMG cycles and nit must be non-negative, got {(cycles, nit)}")
    dev = resolve_device(device)
    b = _tensor(right_hand, dev, dtype)
    if b.ndim != 3 or b.shape[0] != 2:
        raise ValueError("right_hand must have shape [2, ny, nx]")
    spec = GridSpec(nx=int(b.shape[2]), ny=int(b.shape[1]))
    hess = _tensor(hessian, dev, dtype)
    if tuple(hess.shape) != (3, spec.ny, spec.nx):
        raise ValueError(f"Hessian shape must be {(3, spec.ny, spec.nx)}")
    if len(params) != 5:
        raise ValueError(f"regularization parameters must contain 5 values, got {len(params)}")
    u = torch.zeros_like(b) if initial is None else _grid(initial, spec, dev, dtype, "initial").clone()
    p = _params(params)
    scratch = _scratch(dtype, dev, 1, spec.nx, spec.ny)
    _call("csg_dartel_fmg", _dtype_code(dtype), 1, spec.nx, spec.ny, hess.data_ptr(), b.data_ptr(), _addr(p),
          int(cycles), int(nit), u.data_ptr(), int(initial is not None), int(bool(assume_initial_nonzero)),
          scratch.data_ptr(), scratch.numel(), _stream(scratch))
    return u


def dartel_step(source, target, velocity, *, k: int, rtype: int = 1, params=(1.0, 1.0, 0.125, 0.0, 0.0),
                lmreg: float = 1e-3, cycles: int = 3, nit: int = 3, code: int = 1, distortion=None,
                kernel: str = "auto", squaring_kernel: str | None = None, device="auto", dtype=torch.float64,
                optimized: bool = True, assume_initial_nonzero: bool = False):
    """One membrane-regularised DARTEL step (reference 1420-1616).

    Returns ``(updated_velocity [2, ny, nx], metrics [3])``.
    """

    if k < 0:
        raise ValueError(f"DARTEL step count k must be non-negative, got {k}")
    if cycles < 0 or nit < 0:
        raise ValueError(f"DARTEL cycles and nit must be non-negative, got {(cycles, nit)}")
    if squaring_kernel not in {None, "auto", "torch", "triton"}:
        raise ValueError("squaring_kernel must be None, 'auto', 'torch', or 'triton'")
    if code not in {0, 1}:
        raise NotImplementedError("DARTEL supports only code 0 and 1")
    if rtype != 1:
        raise NotImplementedError("dartel_step supports only rtype 1")
    if len(params) != 5:
        raise ValueError(f"DARTEL regularization parameters must contain 5 values, got {len(params)}")
    if distortion is not None:
        raise NotImplementedError("distortion weights are not supported by the native dartel_step")
    dev = resolve_device(device)
    src = _tensor(source, dev, dtype)
    tgt = _tensor(target, dev, dtype)
    if src.ndim != 2 or tgt.ndim != 2:
        raise ValueError("DARTEL source and target must be 2D scalar fields")
    if tuple(src.shape) != tuple(tgt.shape):
        raise ValueError("DARTEL source and target must have the same shape")
    spec = GridSpec(nx=int(src.shape[1]), ny=int(src.shape[0]))
    v = _grid(velocity, spec, dev, dtype, "velocity").clone()
    metrics = torch.empty(3, dtype=dtype, device=dev)
    p = _params(params)
    scratch = _scratch(dtype, dev, 1, spec.nx, spec.ny)
    _call("csg_dartel_step", _dtype_code(dtype), 1, spec.nx, spec.ny, src.data_ptr(), tgt.data_ptr(), v.data_ptr(),
          metrics.data_ptr(), int(k), _addr(p), float(lmreg), int(cycles), int(nit), int(code),
          int(bool(assume_initial_nonzero)), scratch.data_ptr(), scratch.numel(), _stream(scratch))
    return v, metrics


def expdef(displacement, k: int, *, return_jacobian: bool = False, device="auto", dtype=torch.float64,
           optimized: bool = True):
    """Exponentiate a velocity field by CAT scaling and squaring (reference 1619-1666)."""

    if k < 0:
        raise ValueError(f"exponentiation step count k must be non-negative, got {k}")
    dev = resolve_device(device)
    spec = GridSpec.from_shape(tuple(torch.as_tensor(displacement).shape))
    v = _grid(displacement, spec, dev, dtype, "displacement")
    out = torch.empty_like(v)
    jac = torch.empty((4, spec.ny, spec.nx), dtype=dtype, device=dev) if return_jacobian else None
    scratch = _scratch(dtype, dev, 1, spec.nx, spec.ny)
    _call("csg_dartel_expdef", _dtype_code(dtype), 1, spec.nx, spec.ny, v.data_ptr(), int(k), out.data_ptr(),
          None if jac is None else jac.data_ptr(), scratch.data_ptr(), scratch.numel(), _stream(scratch))
    return (out, jac) if return_jacobian else out


def sample_field(field, x, y, *, device="auto", dtype=torch.float64) -> torch.Tensor:
    """Bilinear samples of a 2-D field at zero-based (x, y) (reference 590-621)."""

    dev = resolve_device(device)
    f = _tensor(field, dev, dtype)
    if f.ndim != 2:
        raise ValueError(f"sample_field accepts a 2D scalar field, got {tuple(f.shape)}")
    xt = _tensor(x, dev, dtype)
    yt = _tensor(y, dev, dtype)
    if xt.shape != yt.shape:
        raise ValueError("sample_field x and y coordinates must have the same shape")
    out = torch.empty_like(xt)
    _call("csg_dartel_sample", _dtype_code(dtype), int(f.shape[1]), int(f.shape[0]), f.data_ptr(), xt.numel(),
          xt.data_ptr(), yt.data_ptr(), out.data_ptr(), _stream(out))
    return out
