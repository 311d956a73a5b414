"""The FP64 oracle and the engine against OpenEM's own CUDA kernels.

``oracle/ref_kernels.py`` runs ``openem/kernels/yee.cu`` (update_h, update_e),
``dispersion.cu`` (dispersion_pre / dispersion_post) and ``source_dft.cu`` (inject_dipole,
step_advance), compiled unchanged from OpenEM's sources by ``oracle/build_ref.py``, in OpenEM's
launch order and table layout. On a 24^3 Drude+Lorentz scene (CPML 6 on all faces, the z dipole)
started from seeded random fields, after 100 steps:

* the oracle (float64) is within 1e-5 of each field family's norm of OpenEM's float32 kernels,
  and every cell within 1e-4 of the local scale: the oracle restates their arithmetic;
* the engine's default kernels for this size are within the same bounds: the engine computes
  what OpenEM computes.

Skipped when the cubins were not built (no OpenEM checkout where the tree was built).
"""

import numpy as np
import pytest

from oracle import build_ref, ref64
from openem_b200 import scenes, solver
from test_gpu_scale_parity import check_fields, random_start

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not build_ref.available(),
                                 reason="OpenEM's kernels were not compiled (oracle/build_ref.py)")]

STEPS = 100


@pytest.fixture(scope="module")
def runs():
    from oracle.ref_kernels import ReferenceKernels
    sc = scenes.small_dispersive(n=24, n_sph=2, n_pml=6, num_steps=STEPS, nfreq=2)
    start = random_start(sc.shape, 21)
    rk = ReferenceKernels(sc, STEPS)
    rk.load_fields(start)
    ref = rk.run(STEPS)
    o = ref64.Oracle(sc, STEPS)
    o.load_fields(start)
    orc = o.run(STEPS).fields
    plan = solver.Plan(sc, STEPS)
    try:
        for c, f in enumerate(start):
            plan.write_field(c, f)
        plan.run(STEPS)
        plan.status()
        eng = {nm: plan.read_field(c) for c, nm in enumerate(solver.COMPONENTS)}
    finally:
        plan.close()
    return ref, orc, eng


def test_oracle_matches_openem_kernels(runs):
    ref, orc, _ = runs
    check_fields(orc, ref)


def test_engine_matches_openem_kernels(runs):
    ref, _, eng = runs
    check_fields(eng, ref)


def test_the_run_is_not_trivial(runs):
    """The poles and the dipole act: dropping the dispersion moves the result far outside the
    tolerance."""
    ref, _, _ = runs
    from dataclasses import replace
    from oracle.ref_kernels import ReferenceKernels
    sc = scenes.small_dispersive(n=24, n_sph=2, n_pml=6, num_steps=STEPS, nfreq=2)
    plain = replace(sc, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    rk = ReferenceKernels(plain, STEPS)
    rk.load_fields(random_start(sc.shape, 21))
    other = rk.run(STEPS)
    d = np.linalg.norm(other["Ez"] - ref["Ez"]) / np.linalg.norm(ref["Ez"])
    assert d > 1e-3
