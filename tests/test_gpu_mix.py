"""Slanted-interface mixed dispersion on the GPU (openem/kernels/dispersion_mix.cu): a Lorentz
sphere whose surface cells take the mixed form against the FP64 oracle on every kernel
variant, and OpenEM's two limits and discriminating-power criterion
(tests/test_dispersion.py: test_mix_beta_zero_equals_e_form,
test_mix_middle_beta_lies_between_and_is_stable) on bulk media."""

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver

import test_oracle_golden as tg

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def sphere_ref():
    sc = scenes.mixed_sphere(num_steps=300)
    r = ref64.run(sc)
    return sc, r, ref64.fp32_floor(sc, clean=r)


@pytest.mark.parametrize("kind", [None, "ws", "fused"])
def test_mixed_sphere_matches_oracle(sphere_ref, monkeypatch, kind):
    """E-form interior, mixed-form surface (beta the squared normal projection, fill from the
    signed distance). Each component's error, measured against the norm of its family (Hx is
    near-null beside an x dipole, a few percent of the H family), stays within
    max(2e-5, 3 x that component's float32 floor on the same scale); the probe phasors within
    1e-4 of the largest."""
    sc, r, floor = sphere_ref
    if kind:
        monkeypatch.setenv("OEM_B200_KERNELS", kind)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        fn = np.sqrt(sum(np.linalg.norm(np.asarray(r.fields[c], float)) ** 2 for c in fam))
        for c in fam:
            rc = np.asarray(r.fields[c], float)
            err = np.linalg.norm(np.asarray(g.fields[c], float) - rc) / fn
            fl = floor[c] * np.linalg.norm(rc) / fn
            assert err < max(2e-5, 3.0 * fl), (c, err, fl)
    pg, pr = g.field_phasors["probe"], r.field_phasors["probe"]
    assert np.abs(pg - pr).max() < 1e-4 * np.abs(pr).max()


def test_mix_launches_two_passes():
    """One table adds exactly its two passes (first and second) to every step."""
    from dataclasses import replace
    sc = scenes.mixed_sphere(num_steps=20)
    counts = []
    for s in (sc, replace(sc, dispersion_mix=None)):
        plan = solver.Plan(s)
        counts.append(plan.launches_per_step())
        plan.close()
    assert counts[0] - counts[1] == 2


def _run_e(sc):
    r = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    return tg._e_fields(r)


def test_mix_limits_on_gpu():
    """beta = 0 equals the E form of the same poles and beta = 1 (the pure harmonic branch)
    equals it too (the trapezoidal maps of eps and 1/eps are one bilinear map), within the
    reference's 1e-4 bound; in float32 they round differently."""
    e5 = _run_e(tg._mix_bulk("e", fill=0.5))
    m0 = _run_e(tg._mix_bulk("mix", beta=0.0, fill=0.5))
    assert rel_l2(m0, e5) < 1e-4
    e1 = _run_e(tg._mix_bulk("e"))
    d1 = _run_e(tg._mix_bulk("mix", beta=1.0))
    assert rel_l2(d1, e1) < 1e-4


def test_mix_middle_beta_on_gpu():
    out = {b: _run_e(tg._mix_bulk("mix", beta=b, fill=0.5)) for b in (0.0, 0.35, 0.7, 1.0)}
    span = np.abs(out[1.0] - out[0.0]).max()
    assert span / np.abs(out[0.0]).max() > 0.05
    for b in (0.35, 0.7):
        assert np.isfinite(out[b]).all()
        assert np.abs(out[b] - out[0.0]).max() < 1.05 * span
        assert np.abs(out[b] - out[1.0]).max() < 1.05 * span
        ref = tg._e_fields(ref64.run(tg._mix_bulk("mix", beta=b, fill=0.5)))
        assert rel_l2(out[b], ref) < 1e-4
