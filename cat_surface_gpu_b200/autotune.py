"""Launch-shape autotuner for the native kernels.

A tuning problem is a kernel name, a shape key (the sizes that decide the
best launch: vertex/face counts, surface sizes, candidate counts) and a list
of candidate launch shapes.  :func:`tune` times every candidate on the real
inputs with CUDA events on the launching stream (after a warm-up call, best
of ``repeats``), keeps the fastest, and remembers it per (device name,
kernel, key) in memory and, when ``CAT_SURFACE_B200_AUTOTUNE_CACHE`` names a
JSON file, on disk.  Every candidate must compute the same result: the
tuner only picks among launch shapes of one deterministic kernel.

Candidate sets used by the package:

* :func:`areal_candidates` -- persistent sweep kernel: threads per CTA x
  lanes per vertex x resident CTAs (multiples of the SM count);
* :func:`rotation_candidates` -- batched rotation cost: source points per
  work item (128/256/512) x CTAs (SM count x 1, 2, 4, 8 per SM).
"""

from __future__ import annotations

import json
import os
from pathlib import Path
import threading
from typing import Callable, Sequence

import torch

_LOCK = threading.Lock()
_MEMORY: dict[str, dict] = {}
_ENV = "CAT_SURFACE_B200_AUTOTUNE_CACHE"


def _cache_path() -> Path | None:
    value = os.environ.get(_ENV)
    return Path(value) if value else None


def _load_disk() -> dict:
    path = _cache_path()
    if path is None or not path.exists():
        return {}
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store_disk(entry_key: str, value: dict) -> None:
    path = _cache_path()
    if path is None:
        return
    data = _load_disk()
    data[entry_key] = value
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(path.suffix + ".tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    tmp.replace(path)


def _entry_key(kernel: str, key: Sequence, device: torch.device) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return f"{name}|{kernel}|{','.join(str(k) for k in key)}"


def cached(kernel: str, key: Sequence, device=None) -> dict | None:
    """The remembered best shape for (kernel, key) on this device, or None."""

    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    entry = _entry_key(kernel, key, device)
    with _LOCK:
        if entry in _MEMORY:
            return dict(_MEMORY[entry]["shape"])
        disk = _load_disk().get(entry)
        if disk is not None:
            _MEMORY[entry] = disk
            return dict(disk["shape"])
    return None


def time_call(run: Callable[[], None], *, repeats: int = 3, warmup: int = 1) -> float:
    """Best-of-``repeats`` milliseconds of ``run()`` on the current stream (CUDA events)."""

    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        run()
    best = float("inf")
    for _ in range(repeats):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        run()
        stop.record(stream)
        stop.synchronize()
        best = min(best, start.elapsed_time(stop))
    return best


def tune(kernel: str, key: Sequence, candidates: Sequence[dict], run: Callable[[dict], None], *,
         repeats: int = 3, warmup: int = 1, device=None, force: bool = False) -> dict:
    """Pick the fastest launch shape of ``candidates`` for (kernel, key); ``run(shape)`` launches once."""

    if not candidates:
        raise ValueError("autotune needs at least one candidate")
    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    if not force:
        hit = cached(kernel, key, device)
        if hit is not None:
            return hit
    timings, rejected = [], []
    for shape in candidates:
        try:
            ms = time_call(lambda: run(shape), repeats=repeats, warmup=warmup)
        except (ValueError, RuntimeError) as error:  # a shape the kernel refuses (e.g. shared memory)
            rejected.append({"shape": dict(shape), "error": str(error)[:200]})
            continue
        timings.append((ms, dict(shape)))
    if not timings:
        raise RuntimeError(f"autotune: every candidate of {kernel} failed: {rejected[:2]}")
    best_ms, best = min(timings, key=lambda item: item[0])
    record = {"shape": best, "ms": best_ms, "tried": [{"shape": s, "ms": t} for t, s in timings],
              "rejected": rejected}
    entry = _entry_key(kernel, key, device)
    with _LOCK:
        _MEMORY[entry] = record
        _store_disk(entry, record)
    return dict(best)


def report(kernel: str, key: Sequence, device=None) -> dict | None:
    """The full tuning record (best shape, its time, every candidate's time) if one exists."""

    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    entry = _entry_key(kernel, key, device)
    with _LOCK:
        return _MEMORY.get(entry) or _load_disk().get(entry)


def sm_count(device=None) -> int:
    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    return int(torch.cuda.get_device_properties(device).multi_processor_count)


def areal_candidates(device=None) -> list[dict]:
    """Launch shapes of the persistent sweep kernel: (n_ctas, threads_per_cta, lanes_per_vertex)."""

    sms = sm_count(device)
    shapes = []
    for threads in (256, 384, 512):
        for lanes in (4, 8, 16):
            for per_sm in (1, 2, 3, 4):
                if threads * per_sm > 1024:
                    continue
                shapes.append({"n_ctas": sms * per_sm, "threads_per_cta": threads, "lanes_per_vertex": lanes})
    return shapes


def rotation_candidates(device=None) -> list[dict]:
    """Launch shapes of the batched rotation cost kernel: (tile, n_ctas)."""

    sms = sm_count(device)
    return [{"tile": tile, "n_ctas": sms * per_sm} for tile in (128, 256, 512) for per_sm in (1, 2, 4, 8)
            if tile * per_sm <= 2048]
