"""Hand-written adjoint of the DARTEL data term behind ``torch.autograd``.

``dartel_data_term(velocity, source, target, k)`` returns, per registration
``b``, ``E_b = 1/2 sum_x (S_b(exp(v_b)(x)) - T_b(x))^2`` where ``exp`` is
DARTEL's scaling and squaring (``phi_0 = id + v / 2^k``, ``k`` self
compositions, the maps of ``expdef``; reference
``src/cat_surface_gpu/dartel_grid.py:1619-1666``) and ``S(phi)`` is the
bilinear sample of the sheet with the grid's boundary rule.  Its backward is
``csg_dartel_data_backward``: the exact reverse-mode derivative of those
bilinear stencils (position part plus an atomic scatter of the value part
for every composition), batched over registrations.

Memory: the forward keeps only every ``checkpoint_every``-th map (default
ceil(sqrt(k))); the backward recomputes the squarings between checkpoints,
so a batch of B registrations holds ``ceil(k / c)`` maps each instead of
``k + 1``.

The reference has no such function: its DARTEL step forms a Gauss-Newton
gradient of the same term by pulling the residual gradient back through
the squaring recursion (``initialise_objfun`` + ``squaring_update``,
dartel_grid.py:723-914).  That gradient equals this one at ``k = 0`` and
approximates it for ``k > 0``; the tests pin both statements.
"""

from __future__ import annotations

import math

import torch

from . import _native
from .dartel_grid import _dtype_code


def default_checkpoint_every(k: int) -> int:
    return max(1, math.ceil(math.sqrt(max(k, 1))))


def _batched(velocity, source, target):
    v = velocity if velocity.ndim == 4 else velocity.unsqueeze(0)
    s = source if source.ndim == 3 else source.unsqueeze(0)
    t = target if target.ndim == 3 else target.unsqueeze(0)
    if v.ndim != 4 or v.shape[1] != 2 or s.shape != t.shape or tuple(s.shape) != (v.shape[0],) + tuple(v.shape[2:]):
        raise ValueError("velocity must be [B, 2, ny, nx] (or [2, ny, nx]) and source/target [B, ny, nx] (or [ny, nx])")
    if v.dtype not in (torch.float32, torch.float64) or s.dtype != v.dtype or t.dtype != v.dtype:
        raise ValueError("velocity, source and target must share one dtype (float32 or float64)")
    if v.device.type != "cuda" or s.device != v.device or t.device != v.device:
        raise ValueError("velocity, source and target must live on one CUDA device")
    return v.contiguous(), s.contiguous(), t.contiguous()


def _scratch(dtype, device, batch, nx, ny, k, every):
    need = int(_native.library().csg_dartel_data_scratch_bytes(_dtype_code(dtype), batch, nx, ny, k, every))
    if need == 0:
        raise ValueError("bad data-term arguments (k must be 0..30, checkpoint_every >= 1)")
    return torch.empty(need, dtype=torch.uint8, device=device)


class DartelDataTerm(torch.autograd.Function):
    """E_b(v) of a batch; gradient through the hand-written checkpointed adjoint."""

    @staticmethod
    def forward(ctx, velocity, source, target, k: int, checkpoint_every: int):
        v, s, t = _batched(velocity, source, target)
        batch, _, ny, nx = (int(x) for x in v.shape)
        lib = _native.library()
        count = int(lib.csg_dartel_data_checkpoints(int(k), int(checkpoint_every)))
        if count < 1:
            raise ValueError("k must be 0..30 and checkpoint_every >= 1")
        with torch.cuda.device(v.device):  # the native launch uses the current device
            checkpoints = torch.empty((count, batch, 2, ny, nx), dtype=v.dtype, device=v.device)
            objective = torch.empty(batch, dtype=v.dtype, device=v.device)
            scratch = _scratch(v.dtype, v.device, batch, nx, ny, int(k), int(checkpoint_every))
            _native.check(lib.csg_dartel_data_forward(
                _dtype_code(v.dtype), batch, nx, ny, v.data_ptr(), s.data_ptr(), t.data_ptr(), int(k),
                int(checkpoint_every), checkpoints.data_ptr(), objective.data_ptr(), scratch.data_ptr(),
                scratch.numel(), _native.stream_handle(like=v)), "csg_dartel_data_forward")
        ctx.save_for_backward(checkpoints, s, t)
        ctx.k, ctx.every, ctx.squeeze = int(k), int(checkpoint_every), velocity.ndim == 3
        return objective if velocity.ndim == 4 else objective[0]

    @staticmethod
    def backward(ctx, grad_objective):
        checkpoints, s, t = ctx.saved_tensors
        batch, ny, nx = (int(x) for x in s.shape)
        with torch.cuda.device(s.device):  # the native launch uses the current device
            scale = grad_objective.reshape(-1).to(device=s.device, dtype=s.dtype).contiguous()
            grad = torch.empty((batch, 2, ny, nx), dtype=s.dtype, device=s.device)
            scratch = _scratch(s.dtype, s.device, batch, nx, ny, ctx.k, ctx.every)
            _native.check(_native.library().csg_dartel_data_backward(
                _dtype_code(s.dtype), batch, nx, ny, s.data_ptr(), t.data_ptr(), ctx.k, ctx.every,
                checkpoints.data_ptr(), scale.data_ptr(), grad.data_ptr(), scratch.data_ptr(), scratch.numel(),
                _native.stream_handle(like=s)), "csg_dartel_data_backward")
        return (grad[0] if ctx.squeeze else grad), None, None, None, None


def dartel_data_term(velocity: torch.Tensor, source: torch.Tensor, target: torch.Tensor, k: int = 7,
                     checkpoint_every: int | None = None) -> torch.Tensor:
    """Per-registration data term E_b (differentiable in ``velocity``); see the module docstring."""

    every = default_checkpoint_every(k) if checkpoint_every is None else int(checkpoint_every)
    return DartelDataTerm.apply(velocity, source, target, int(k), every)
