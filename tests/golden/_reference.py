"""Where the golden-vector generators find the reference checkout.

The generators run in a development checkout that has the reference project
beside it; nothing under ``tests/`` reads the reference at test time.  The
checkout's root comes from the ``CAT_SURFACE_REFERENCE`` environment variable
(default ``/root/reference``).  ``use_reference_package()`` puts its ``src``
directory on ``sys.path`` so ``import cat_surface_gpu`` loads the reference.
"""

from __future__ import annotations

import os
from pathlib import Path
import sys

REFERENCE_ROOT = Path(os.environ.get("CAT_SURFACE_REFERENCE", "/root/reference"))


def use_reference_package() -> Path:
    src = REFERENCE_ROOT / "src"
    if not (src / "cat_surface_gpu").is_dir():
        raise SystemExit(f"reference package not found under {src}; set CAT_SURFACE_REFERENCE")
    if str(src) not in sys.path:
        sys.path.insert(0, str(src))
    return src


def reference_binary(name: str) -> Path:
    path = REFERENCE_ROOT / "bin" / "linux-x86_64" / name
    if not path.is_file():
        raise SystemExit(f"reference binary {name} not found under {path.parent}; set CAT_SURFACE_REFERENCE")
    return path
