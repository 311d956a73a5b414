"""Generate ``ref_kernels_disp.npz``: fields after 100 steps of OpenEM's own CUDA kernels.

Runs on a machine with a GPU after ``python -m oracle.build_ref`` has compiled
``openem/kernels/{yee,dispersion,source_dft}.cu`` (unchanged) into ``oracle/_ref/``. The scene is
``scenes.small_dispersive(n=24, n_sph=2, n_pml=6, num_steps=100, nfreq=2)``: 24^3 cells, CPML 6
on all faces, Drude+Lorentz spheres, the z dipole; the start is six seeded standard-normal float32
fields (``numpy.random.default_rng(21)``, Ex..Hz in order). The file holds the six final float32
fields, which ``tests/test_oracle_golden.py`` compares with the FP64 oracle on the CPU.

    python tests/golden/gen_ref_kernel_fields.py [output directory, default tests/golden]
"""

from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from openem_b200 import scenes  # noqa: E402
from oracle.ref_kernels import ReferenceKernels  # noqa: E402

STEPS, SEED = 100, 21


def start_fields(shape):
    rng = np.random.default_rng(SEED)
    return [rng.standard_normal(shape).astype(np.float32) for _ in range(6)]


def main() -> None:
    sc = scenes.small_dispersive(n=24, n_sph=2, n_pml=6, num_steps=STEPS, nfreq=2)
    rk = ReferenceKernels(sc, STEPS)
    rk.load_fields(start_fields(sc.shape))
    out = rk.run(STEPS)
    dst = pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    np.savez_compressed(dst / "ref_kernels_disp.npz", steps=np.int32(STEPS),
                        seed=np.int32(SEED), **out)
    print("ref_kernels_disp.npz", (dst / "ref_kernels_disp.npz").stat().st_size)


if __name__ == "__main__":
    main()
