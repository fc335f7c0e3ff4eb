"""Build recipe for the native library ``libcatsurf_b200.so`` (sm_100a).

``python -m cat_surface_gpu_b200.build`` compiles every ``csrc/*.cu`` and
``csrc/*.cpp`` with nvcc into one shared library next to this file.  The
library exports only the ``extern "C"`` entry points of
``include/catsurf_b200.h``; CUDA runtime is linked statically.
"""

from __future__ import annotations

import os
from pathlib import Path
import subprocess
import sys

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIBRARY = HERE / "libcatsurf_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources() -> list[Path]:
    return sorted((HERE / "csrc").glob("*.cu")) + sorted((HERE / "csrc").glob("*.cpp"))


def _inputs() -> list[Path]:
    return _sources() + sorted((HERE / "csrc").glob("*.h")) + sorted((HERE / "csrc").glob("*.cuh")) + sorted(
        (ROOT / "include").glob("*.h")
    )


def needs_build() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(path.stat().st_mtime > built for path in _inputs())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIBRARY
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    common = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", *ARCH]
    if verbose:
        common += ["-Xptxas", "-v"]
    objects = []
    procs = []
    for source in _sources():
        obj = objdir / (source.name + ".o")
        cmd = [nvcc, *common, "-I", str(ROOT / "include"), "-c", str(source), "-o", str(obj)]
        if source.suffix == ".cpp":
            cmd = [nvcc, "-x", "cu", *cmd[1:]]
        procs.append((source, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objects.append(str(obj))
    failed = []
    for source, proc in procs:
        out, _ = proc.communicate()
        if verbose and out:
            print(out)
        if proc.returncode != 0:
            failed.append(f"{source.name}:\n{out}")
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    tmp = LIBRARY.with_suffix(".so.tmp")
    subprocess.run([nvcc, *ARCH, "-shared", "-o", str(tmp), *objects, "-lz"], check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
