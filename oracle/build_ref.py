"""Compile the reference's own CUDA FDTD ops into oracle/_ref (GPU checker).

Test infrastructure only: the library built here is what the GPU parity tests
compare the fused engine and the per-op kernels against ("the reference's own
CUDA FDTD kernels on identical inputs").  It is built from the reference's
sources where they lie (witwin/maxwell/fdtd/cuda/extension.cpp and kernels/*.cu,
the list in witwin/maxwell/fdtd/cuda/build.py:181-197), with the defines that
file passes (build.py:300-310), for sm_100.  Nothing is copied; the outputs
(objects, ninja files, the .so) go to oracle/_ref/, which git ignores.

Usage: python oracle/build_ref.py [reference checkout]

The checkout is the argument, else the WITWIN_MAXWELL_REFERENCE environment
variable, else the build container's read-only copy (REFERENCE_DEFAULT).
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# where the build container mounts the reference checkout (read-only); this
# recipe and the golden-vector scripts are the only files that name it
REFERENCE_DEFAULT = "/root/reference"


def reference_checkout(arg: str | None = None) -> Path | None:
    """The reference checkout to read, or None when none is present."""
    path = Path(arg or os.environ.get("WITWIN_MAXWELL_REFERENCE") or REFERENCE_DEFAULT)
    return path if (path / "witwin" / "maxwell").is_dir() else None
OUT = HERE / "_ref"
LIB_NAME = "witwin_maxwell_fdtd_cuda"
SOURCES = ("extension.cpp", "kernels/common.cu", "kernels/magnetic.cu", "kernels/electric.cu", "kernels/boundary.cu",
           "kernels/projection.cu", "kernels/aniso.cu", "kernels/dispersive.cu", "kernels/sources.cu",
           "kernels/spectral.cu", "kernels/observers.cu", "kernels/wire.cu", "kernels/adjoint.cu")


def library_path() -> Path:
    return OUT / f"{LIB_NAME}.so"


def build(reference: Path) -> Path:
    from torch.utils.cpp_extension import load

    root = reference / "witwin" / "maxwell" / "fdtd" / "cuda"
    missing = [s for s in SOURCES if not (root / s).exists()]
    if missing:
        raise FileNotFoundError(f"reference sources missing under {root}: {missing}")
    OUT.mkdir(parents=True, exist_ok=True)
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    define = "-DTORCH_TARGET_VERSION=0x020a000000000000"
    path = load(
        name=LIB_NAME,
        sources=[str(root / s) for s in SOURCES],
        build_directory=str(OUT),
        extra_include_paths=[str(root), str(root / "kernels")],
        extra_cflags=["-O3", define],
        extra_cuda_cflags=["-O3", define, "-DUSE_CUDA", "-gencode=arch=compute_100,code=sm_100"],
        is_python_module=False,
        verbose=False,
    )
    return Path(path)


if __name__ == "__main__":
    ref = reference_checkout(sys.argv[1] if len(sys.argv) > 1 else None)
    if ref is None:
        sys.exit("no reference checkout: pass its path or set WITWIN_MAXWELL_REFERENCE")
    print(build(ref))
