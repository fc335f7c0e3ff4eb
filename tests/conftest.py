"""Test configuration: registers the ``gpu`` marker and puts the repo root on sys.path."""

from __future__ import annotations

from pathlib import Path
import sys

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def native_library():
    from cat_surface_gpu_b200 import build

    build.build()
    from cat_surface_gpu_b200 import _native

    return _native.library()


def load_surf2sphere_golden(name: str) -> dict:
    import numpy as np

    data = np.load(GOLDEN / f"surf2sphere_{name}.npz")
    return {
        "faces": data["faces"].astype(np.int32),
        "prefix": data["prefix"],
        "final": data["final"],
        "source_area": float(data["source_area"]),
        "cpu_seconds": float(data["cpu_seconds"]),
    }
