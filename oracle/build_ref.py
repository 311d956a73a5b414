"""Recipe: compile OpenEM's own CUDA kernels, unchanged, into ``oracle/_ref/`` -- TEST
INFRASTRUCTURE ONLY.

OpenEM's kernels (``openem/kernels/*.cu``) are plain ``extern "C" __global__`` CUDA C that OpenEM
compiles at run time with NVRTC through cupy (options ``-std=c++17 --use_fast_math``,
``openem/device.py:25``). cupy is absent here, so this recipe compiles the same files with nvcc and
the same options into sm_100a cubins, read straight from a checkout of OpenEM (``OPENEM_SRC``,
default the checkout this build was made against). Nothing is copied: the sources stay where they
lie, and only the cubins land in ``oracle/_ref/`` (git-ignored; they travel with the tree to a GPU
machine). ``oracle/ref_kernels.py`` loads them with the CUDA driver API to run OpenEM's arithmetic
beside the FP64 oracle and the engine in the tests; the engine never loads them.

    OPENEM_SRC=<openem checkout> python -m oracle.build_ref
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
OUT = HERE / "_ref"
#: the kernel files whose arithmetic the tests compare against: the Yee updates with CPML
#: (yee.cu), the ADE passes (dispersion.cu), the point-dipole injection and step counter
#: (source_dft.cu)
KERNEL_FILES = ("yee.cu", "dispersion.cu", "source_dft.cu")
OPTIONS = ("-std=c++17", "--use_fast_math", "-O3")
ARCH = ("-gencode", "arch=compute_100a,code=sm_100a")


def source_dir() -> pathlib.Path | None:
    src = os.environ.get("OPENEM_SRC") or "/root/reference"
    d = pathlib.Path(src) / "openem" / "kernels"
    return d if d.is_dir() else None


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cubin_path(name: str) -> pathlib.Path:
    return OUT / (pathlib.Path(name).stem + ".cubin")


def build(verbose: bool = False) -> bool:
    """Compile every kernel file whose cubin is missing or older than its source. Returns False
    (and builds nothing) when no OpenEM checkout is present."""
    src = source_dir()
    if src is None:
        return False
    OUT.mkdir(exist_ok=True)
    for name in KERNEL_FILES:
        s, o = src / name, cubin_path(name)
        if o.exists() and o.stat().st_mtime >= s.stat().st_mtime:
            continue
        cmd = [nvcc(), "-cubin", *ARCH, *OPTIONS, "-o", str(o), str(s)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{r.stdout}\n{r.stderr}")
    return True


def available() -> bool:
    return all(cubin_path(n).exists() for n in KERNEL_FILES)


if __name__ == "__main__":
    ok = build(verbose=True)
    print("built" if ok else "no OpenEM checkout found (set OPENEM_SRC)", file=sys.stderr)
