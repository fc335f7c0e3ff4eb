"""Build recipe for the oracle's C restatements (test infrastructure only).

``python -m oracle.build`` compiles every ``oracle/*.c`` into
``oracle/_build/liboracle.so`` with ``-O2 -ffp-contract=off`` so that each
floating-point operation is rounded exactly once, as written.
"""

from __future__ import annotations

from pathlib import Path
import subprocess
import sys

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    sources = sorted(HERE.glob("*.c"))
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", str(OUT), *map(str, sources), "-lm"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
