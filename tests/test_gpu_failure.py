"""Failure detection on the device, made to happen without faulting or hanging the GPU.

* A bounded wait that runs out: with ``Plan(wait_expiry_polls=...)`` every consumer warp of the
  warp-specialised E update also waits on a shared-memory barrier that no thread arrives at
  (a flag nothing sets). The wait gives up after its short bound and records the expiry; every
  warp leaves its pipeline (the producers first wait for their own copies) and the host reads
  ``OEM_ERR_TIMEOUT`` from the plan's status. A fresh plan on the same device then runs
  normally and matches the one-thread-per-cell kernels.
* Non-finite input: a NaN in one permittivity cell is named at set-up and again at the
  readout (OpenEM's ``_warn_nonfinite``, ``openem/solver.py:347-370``, warns and goes on).
"""

import time
from dataclasses import replace

import numpy as np
import pytest

from openem_b200 import scenes, solver

pytestmark = pytest.mark.gpu


def family_err(fa, fb, names):
    den = np.sqrt(sum(float(np.linalg.norm(fb[n].ravel())) ** 2 for n in names))
    return max(float(np.linalg.norm((fa[n] - fb[n]).ravel())) for n in names) / max(den, 1e-300)


def test_wait_expiry_reports_timeout_and_device_stays_usable(monkeypatch):
    monkeypatch.setenv("OEM_B200_KERNELS", "ws")
    sc = scenes.small_dispersive(n=40, n_sph=4, num_steps=30, n_pml=8, nfreq=2)
    plan = solver.Plan(sc, 30, wait_expiry_polls=64)
    try:
        t0 = time.perf_counter()
        plan.run(3)
        with pytest.raises(RuntimeError, match="exceeded its bound"):
            plan.status()
        assert time.perf_counter() - t0 < 30.0  # every block gave up quickly
        plan.status()  # the error word was cleared by the read
    finally:
        plan.close()
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    monkeypatch.setenv("OEM_B200_KERNELS", "basic")
    b = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    assert family_err(a.fields, b.fields, ("Ex", "Ey", "Ez")) < 1e-6
    assert family_err(a.fields, b.fields, ("Hx", "Hy", "Hz")) < 1e-6
    assert np.abs(a.fields["Ez"]).max() > 0


def test_nonfinite_permittivity_is_reported(capsys):
    sc = scenes.small_dispersive(n=24, n_sph=2, num_steps=40, n_pml=6, nfreq=2)
    eps = np.array(sc.eps_ex)
    eps[12, 12, 12] = np.nan
    r = solver.run(replace(sc, eps_ex=eps), use_shutoff=False, verbose=False)
    out = capsys.readouterr().out
    assert "eps or sigma holds non-finite values" in out
    assert "holds non-finite values; the field has most likely diverged" in out
    assert not all(np.isfinite(v).all() for v in r.field_phasors.values())
