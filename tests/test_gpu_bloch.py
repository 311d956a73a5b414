"""Complex-field (Bloch) path and mode sources on the GPU against the FP64 oracle.

Tolerances: fields within 1e-5 of their field family's norm (E or H), flux and field phasors
within 1e-4 relative L2, time samples within 1e-5 of the family norm. At zero Bloch phase the
complex path must reproduce two real runs, driven by the real and the imaginary part of the
injection, bit for bit.
"""

from dataclasses import replace

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver
from openem_b200.model import PointDipole

pytestmark = pytest.mark.gpu

E3 = ("Ex", "Ey", "Ez")
H3 = ("Hx", "Hy", "Hz")


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def family_err(fa, fb, names):
    den = np.sqrt(sum(float(np.linalg.norm(np.asarray(fb[n]).ravel())) ** 2 for n in names))
    return max(float(np.linalg.norm((np.asarray(fa[n]) - np.asarray(fb[n])).ravel()))
               for n in names) / max(den, 1e-300)


def small_bloch(num_steps=300, k=(0.05, 0.0, 0.0)):
    sc = scenes.bloch_metasurface(nx=16, ny=8, nz=64, n_pml=8, npix=4, layer_cells=8, nfreq=5,
                                  num_steps=num_steps, bloch_k=k, field_monitor=True)
    return scenes.with_time_monitor(sc, box=(4, 4, 4), interval=6)


@pytest.fixture(scope="module")
def bloch_runs():
    sc = small_bloch()
    return {"sc": sc, "ref": ref64.run(sc),
            "gpu": solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)}


def test_bloch_mode_fields_match_oracle(bloch_runs):
    r, g = bloch_runs["ref"], bloch_runs["gpu"]
    assert np.iscomplexobj(g.fields["Ey"])
    assert family_err(g.fields, r.fields, E3) < 1e-5
    assert family_err(g.fields, r.fields, H3) < 1e-5


def test_bloch_phasors_match_oracle(bloch_runs):
    r, g = bloch_runs["ref"], bloch_runs["gpu"]
    assert rel_l2(g.phasors["T"].data, r.phasors["T"]) < 1e-4
    for name, data in r.field_phasors.items():
        assert rel_l2(g.field_phasors[name], data) < 1e-4, name


def test_bloch_time_samples_match_oracle(bloch_runs):
    r, g = bloch_runs["ref"], bloch_runs["gpu"]
    for name, data in r.time_samples.items():
        assert g.time_slots[name] == r.time_slots[name]
        assert np.iscomplexobj(g.time_samples[name])
        assert rel_l2(g.time_samples[name], data) < 1e-5, name


@pytest.mark.parametrize("k", [(0.12, 0.0, 0.0), (0.05, 0.03, 0.0)])
@pytest.mark.parametrize("kind", [None, "ws"])
def test_bloch_dipole_matches_oracle(monkeypatch, kind, k):
    """A z dipole in the Bloch cell (no mode source): complex analytic amplitude injection, on
    the complex one-thread-per-cell kernels and on the split update (the warp-specialised real
    kernels on each part plus the seam terms), with a Bloch phase on x and on x and y."""
    if kind:
        monkeypatch.setenv("OEM_B200_KERNELS", kind)
    sc = small_bloch(num_steps=250, k=k)
    idx, coef = scenes.dipole_stencil(sc.grid, 2, (0.5 * 16 * 0.01e-6, 0.5 * 8 * 0.01e-6, 0.0))
    from openem_b200.model import GaussianPulse, sample_waveform
    wf = sample_waveform(GaussianPulse(freq0=3e14, fwidth=0.9e14), sc.dt, 250)
    sc = replace(sc, mode_sources=[], dipoles=[PointDipole(component=2, indices=idx, coef=coef,
                                                           waveform=wf)])
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    assert family_err(g.fields, r.fields, E3) < 1e-5
    assert family_err(g.fields, r.fields, H3) < 1e-5


def test_gaussian_beam_real_path_matches_oracle():
    """Mode source (y-polarised Gaussian beam) on the real path: fields and flux phasors. The
    waist keeps the profile ~1e-7 at the PEC-backed wall cells of the source plane, where this
    engine injects nothing (cb = 0 there) and OpenEM injects and zeroes at the next update."""
    sc = scenes.beam_slab(nx=32, ny=32, nz=40, n_pml=8, design=(8, 8), waist=0.1e-6,
                          slab_cells=4, num_steps=300)
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    assert family_err(g.fields, r.fields, E3) < 1e-5
    assert family_err(g.fields, r.fields, H3) < 1e-5
    assert rel_l2(g.phasors["T"].data, r.phasors["T"]) < 1e-4


@pytest.mark.parametrize("kind", [None, "ws"])
def test_complex_at_zero_phase_is_two_real_runs(monkeypatch, kind):
    """force_complex at k = 0: the real part is the real run driven by amp, the imaginary part
    the real run driven by -i amp (Im(p a) = Re(p a (-i))), bit for bit, on both complex
    update paths."""
    if kind:
        monkeypatch.setenv("OEM_B200_KERNELS", kind)
    sc = scenes.beam_slab(nx=24, ny=24, nz=36, n_pml=6, design=(6, 6), waist=0.15e-6,
                          slab_cells=4, num_steps=160)
    c = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False, force_complex=True)
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    m = sc.mode_sources[0]
    sc_i = replace(sc, mode_sources=[replace(m, amp_e=m.amp_e * -1j, amp_h=m.amp_h * -1j)])
    b = solver.run(sc_i, use_shutoff=False, return_fields=True, verbose=False)
    for nm in E3 + H3:
        np.testing.assert_array_equal(np.real(c.fields[nm]), a.fields[nm])
        np.testing.assert_array_equal(np.imag(c.fields[nm]), b.fields[nm])
    np.testing.assert_allclose(c.phasors["T"].data,
                               a.phasors["T"].data + 1j * b.phasors["T"].data,
                               rtol=1e-6, atol=1e-12 * np.abs(c.phasors["T"].data).max())


def test_split_complex_update_matches_oracle(bloch_runs, monkeypatch):
    """The mode-source Bloch cell on the split complex update: fields, flux and field phasors
    and time samples against the FP64 oracle with the bounds of the complex kernels."""
    monkeypatch.setenv("OEM_B200_KERNELS", "ws")
    r = bloch_runs["ref"]
    g = solver.run(bloch_runs["sc"], use_shutoff=False, return_fields=True, verbose=False)
    assert family_err(g.fields, r.fields, E3) < 1e-5
    assert family_err(g.fields, r.fields, H3) < 1e-5
    assert rel_l2(g.phasors["T"].data, r.phasors["T"]) < 1e-4
    for name, data in r.time_samples.items():
        assert rel_l2(g.time_samples[name], data) < 1e-5, name


def test_split_complex_update_launches():
    """The split update runs the real kernels twice per family plus one seam face per side."""
    sc = small_bloch(num_steps=20, k=(0.12, 0.0, 0.0))
    counts = {}
    for kind in ("basic", "ws"):
        import os
        os.environ["OEM_B200_KERNELS"] = kind
        try:
            plan = solver.Plan(sc, 20, cplx=True)
            counts[kind] = plan.launches_per_step()
            plan.close()
        finally:
            del os.environ["OEM_B200_KERNELS"]
    assert counts["ws"] - counts["basic"] == 4
