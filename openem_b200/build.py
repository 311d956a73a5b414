"""Build ``liboem_b200.so`` in-tree with nvcc for sm_100a.

    python -m openem_b200.build            # rebuild if a source is newer than the library
    python -m openem_b200.build --force

The library is a plain C-ABI shared object (``include/oem_b200.h``) with the CUDA runtime linked
statically, so it loads in any process on a machine with the NVIDIA driver.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liboem_b200.so"
SOURCES = ["oem_api.cu", "oem_kernels.cu", "oem_yee_stream.cu", "oem_yee_tma.cu",
           "oem_noalloc.cu", "oem_yee_ws.cu", "oem_ade.cu", "oem_complex.cu", "oem_adjoint.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[pathlib.Path]:
    return [CSRC / s for s in SOURCES]


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "oem_b200.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> pathlib.Path:
    """Compile the library if it is missing or older than its sources; return its path."""
    if not force and not stale():
        return LIB
    tmp = LIB.with_suffix(f".so.{os.getpid()}.tmp")
    cmd = [nvcc_path(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-O3", "--shared", "-o", str(tmp), *map(str, sources())]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, cwd=str(ROOT), capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr, flush=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    extra = ["-Xptxas", "-v"] if "--ptxas" in args else None
    p = build(force="--force" in args or extra is not None, verbose=True, extra=extra)
    print(p)
