"""Early termination on the device against the oracle running the same policy.

``solver.run(..., use_shutoff=True)`` checks every 400 steps: the float64 field sums on the
device (``oem_plan_energy``), the monitors' partial DFT batch folded in before the flux is read
(``oem_plan_flush``), the policy, and the rule that a stop waits for the sources to end. The
oracle runs the identical policy on its own float64 sums and phasors at the same cadence
(``ref64.run_shutoff``). Both must stop at the same step for the same reason, with per-check
sums within 1e-5 relative and final phasors within 1e-4 relative L2: a fold that counted a
partial batch twice, or a check at the wrong step, changes the flux series and the phasors.
"""

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, shutoff, solver

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def run_both(sc, make_policy):
    g = solver.run(sc, use_shutoff=True, policy=make_policy(), verbose=False)
    pol = make_policy()
    r, n, trig, trace = ref64.run_shutoff(sc, pol)
    return g, (r, n, trig, trace, pol)


def check_same_stop(g, ref):
    r, n, trig, trace, pol = ref
    assert g.steps_run == n and g.shutoff_triggered == trig
    assert g.stop_reason.split("(")[0] == pol.reason.split("(")[0]
    assert [s for s, _ in g.energy_trace] == [s for s, _, _ in trace]
    e_dev = np.array([e for _, e in g.energy_trace])
    e_ref = np.array([e for _, _, e in trace])
    np.testing.assert_allclose(e_dev, e_ref, rtol=1e-5, atol=1e-5 * e_ref.max())
    for name, data in r.phasors.items():
        assert rel_l2(g.phasors[name].data, data) < 1e-4, name
    for name, data in r.field_phasors.items():
        assert rel_l2(g.field_phasors[name], data) < 1e-4, name


def test_slab_default_policy_stops_like_oracle():
    """OpenEM's default policy on the plane-wave slab: the decay tests fire at step 1200 of
    10,491, after the source has ended (step ~600)."""
    sc = scenes.slab_plane_wave(nxy=1)
    g, ref = run_both(sc, lambda: shutoff.default_policy(sc.shutoff))
    assert g.shutoff_triggered and g.steps_run < sc.num_time_steps
    check_same_stop(g, ref)


def test_slab_flux_convergence_stops_like_oracle():
    """Only the flux test can fire (the decay thresholds are out of reach): the fluxes of the
    T and R planes, read after every partial-batch fold, settle and stop the run."""
    sc = scenes.slab_plane_wave(nxy=1)
    make = lambda: shutoff.Policy(shutoff.Criteria(field_threshold=None, energy_threshold=1e-30,
                                                   flux_tol=1e-3))
    g, ref = run_both(sc, make)
    assert g.stop_reason.startswith("phasor_converged")
    check_same_stop(g, ref)


def test_dispersive_loose_policy_stops_like_oracle():
    """A 32^3 Drude+Lorentz scene with field monitors and decay thresholds of 2e-2: more than
    800 steps (several checks) before the resonant spheres ring down far enough."""
    sc = scenes.small_dispersive(n=32, n_sph=4, num_steps=4000, n_pml=8, nfreq=3)
    make = lambda: shutoff.Policy(shutoff.Criteria(field_threshold=2e-2, energy_threshold=2e-2,
                                                   flux_tol=None))
    g, ref = run_both(sc, make)
    assert g.shutoff_triggered and 800 <= g.steps_run < 4000
    check_same_stop(g, ref)
