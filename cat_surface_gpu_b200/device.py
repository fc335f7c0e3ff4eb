"""Device resolution shared by every operator (no CPU fallback).

Mirrors ``resolve_device`` / ``DeviceUnavailable`` of the reference
(``src/cat_surface_gpu/dartel_grid.py:35-87``), except that this package only
executes on CUDA: asking for ``cpu`` raises instead of running a CPU path.
"""

from __future__ import annotations

import torch


class DeviceUnavailable(RuntimeError):
    """Report that an explicitly requested Torch device is unavailable."""


def resolve_device(device: str | torch.device = "auto") -> torch.device:
    """Resolve an explicit CUDA device; CPU or a missing GPU raises."""

    if isinstance(device, str) and device == "auto":
        device = "cuda"
    resolved = torch.device(device)
    if resolved.type != "cuda":
        raise DeviceUnavailable(
            f"cat_surface_gpu_b200 runs only on CUDA devices (sm_100a); got {resolved}. "
            "There is no CPU fallback."
        )
    if not torch.cuda.is_available():
        raise DeviceUnavailable("CUDA was requested but no CUDA device is available")
    if resolved.index is not None and resolved.index >= torch.cuda.device_count():
        raise DeviceUnavailable(f"CUDA device {resolved.index} does not exist ({torch.cuda.device_count()} present)")
    if resolved.index is None:
        resolved = torch.device("cuda", torch.cuda.current_device())
    return resolved
