"""Build the sm_100a shared library ``libfdtd_b200.so`` in-tree with nvcc.

The library holds every CUDA kernel of the package and the C ABI declared in
``include/fdtd_b200.h``.  It is built next to this file so that it travels with
the source tree; nothing is JIT-compiled at import time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC = PACKAGE_DIR / "csrc"
LIB_PATH = PACKAGE_DIR / "libfdtd_b200.so"
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(cuda_home) / "bin" / "nvcc"
    if candidate.exists():
        return str(candidate)
    found = shutil.which("nvcc")
    if found is None:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    return found


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_rebuild() -> bool:
    if not LIB_PATH.exists():
        return True
    mtime = LIB_PATH.stat().st_mtime
    deps = list(CSRC.glob("*")) + [PACKAGE_DIR.parent / "include" / "fdtd_b200.h", Path(__file__)]
    return any(p.stat().st_mtime > mtime for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile every ``csrc/*.cu`` to an object (in parallel, one nvcc per
    source) and link them into ``libfdtd_b200.so``."""
    if not force and not needs_rebuild():
        return LIB_PATH
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    flags = [*GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *(extra_flags or [])]
    with tempfile.TemporaryDirectory(prefix="fdtd_b200_build_") as tmp:
        objs = []
        cmds = []
        for src in sources():
            obj = Path(tmp) / (src.stem + ".o")
            objs.append(obj)
            cmds.append([_nvcc(), *flags, "-c", str(src), "-o", str(obj)])

        def run(cmd: list[str]) -> None:
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True, cwd=str(PACKAGE_DIR))

        workers = max(1, min(len(cmds), os.cpu_count() or 1))
        with ThreadPoolExecutor(max_workers=workers) as pool:
            for fut in [pool.submit(run, c) for c in cmds]:
                fut.result()
        link = [_nvcc(), *GENCODE, "-shared", "-o", str(LIB_PATH) + ".tmp", *[str(o) for o in objs]]
        run(link)
    os.replace(str(LIB_PATH) + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
