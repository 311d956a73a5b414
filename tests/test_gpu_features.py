"""Boundary and medium features on the GPU against the FP64 oracle: absorber slabs (real and
complex paths) and time-modulated permittivity (lossless, lossy, dispersive; zero-amplitude
identity; first-order sidebands). Tolerance: fields within 1e-5 of their field family's norm
(dispersive scenes: max(2e-5, 3x the measured float32 floor))."""

from dataclasses import replace

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver
from openem_b200 import model as M
from openem_b200.model import Axis, Grid

pytestmark = pytest.mark.gpu


def family_err(fa, fb, names):
    den = np.sqrt(sum(float(np.linalg.norm(np.asarray(fb[n]).ravel())) ** 2 for n in names))
    return max(float(np.linalg.norm((np.asarray(fa[n]) - np.asarray(fb[n])).ravel()))
               for n in names) / max(den, 1e-300)


def absorber_scene(n=28, layers=6, steps=220):
    """Dipole in vacuum; CPML on x and y, PEC-backed z walls lined with graded absorbers."""
    sc = scenes.small_dispersive(n=n, n_sph=1, n_pml=4, num_steps=steps)
    ax = sc.grid.axes
    grid = Grid(ax[0], ax[1], Axis(ax[2].edges, "PEC", "PEC"))
    return replace(sc, grid=grid, pml={k: v for k, v in sc.pml.items() if k[0] != 2},
                   dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None,
                   absorbers=scenes.absorber_slabs(grid, 2, layers, strength=0.2))


def test_absorber_matches_oracle():
    sc = absorber_scene()
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        assert family_err(g.fields, r.fields, fam) < 1e-5
    # the absorber is active: without it the fields differ by far more than the tolerance
    g0 = solver.run(replace(sc, absorbers=[]), use_shutoff=False, return_fields=True,
                    verbose=False)
    assert family_err(g0.fields, g.fields, ("Ex", "Ey", "Ez")) > 1e-3


def test_absorber_on_complex_path_matches_oracle():
    sc = absorber_scene(steps=160)
    r = ref64.BlochOracle(sc).run()
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False,
                   force_complex=True)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        assert family_err(g.fields, r.fields, fam) < 1e-5


# ---- time-modulated permittivity (openem/kernels/modulation.cu) --------------------------------

C0 = 2.99792458e8


def modulated_scene(steps=1500, **kw):
    """2 x 2 periodic cell, eps_s = 2.5 slab with delta = 0.3 at fm = 0.1 f0 and a phase that
    varies across the cell, so the four columns differ."""
    args = dict(nxy=2, num_steps=steps, eps_s=2.5, delta=0.3, fm_rel=0.1,
                phase=lambda x, y, z: 4e7 * x + 2e7 * y)
    args.update(kw)
    return scenes.modulated_slab(**args)


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel())
                 / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def test_modulation_matches_oracle():
    sc = modulated_scene()
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        assert family_err(g.fields, r.fields, fam) < 1e-5
    assert rel_l2(g.phasors["T"].data, r.phasors["T"]) < 1e-4
    # the modulation is active: the static slab differs by far more than the tolerance
    g0 = solver.run(replace(sc, modulation=None), use_shutoff=False, return_fields=True,
                    verbose=False)
    assert family_err(g0.fields, g.fields, ("Ex", "Ey", "Ez")) > 1e-3


def test_modulation_with_loss_matches_oracle():
    sc = modulated_scene(steps=1200)
    sig = [np.where(np.asarray(e) > 1.5, 2e3, 0.0) for e in (sc.eps_ex, sc.eps_ey, sc.eps_ez)]
    sc = replace(sc, sigma_ex=sig[0], sigma_ey=sig[1], sigma_ez=sig[2])
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        assert family_err(g.fields, r.fields, fam) < 1e-5


def test_modulation_with_dispersion_matches_oracle():
    """Modulation riding on eps_inf of Drude + Lorentz spheres: the D-form denominators carry the
    Drude DC coupling G; the pole pass is unchanged."""
    sd = scenes.small_dispersive(n=24, n_sph=2, n_pml=4, num_steps=200)
    d = sd.dispersion
    comp = np.asarray(d.comp)[::3]
    cell = np.asarray(d.cell)[::3]
    mo = M.TimeModulation(4e13, comp, cell, np.full(comp.size, 0.2),
                          np.linspace(0.0, 3.0, comp.size))
    sc = replace(sd, modulation=mo)
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    floor = ref64.fp32_floor(sc, clean=r)
    for nm in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert rel_l2(g.fields[nm], r.fields[nm]) < max(2e-5, 3.0 * floor[nm]), (nm, floor[nm])


def test_zero_amplitude_modulation_matches_static():
    """The reference's criterion (tests/test_timemod.py:230-252): amp = 0 differs from the static
    scene only by the float32 rounding of the rewritten coefficients, |dE| <= 1e-5 max|E|."""
    sc = modulated_scene(steps=1500, delta=0.0)
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    b = solver.run(replace(sc, modulation=None), use_shutoff=False, return_fields=True,
                   verbose=False)
    for nm in ("Ex", "Hy"):
        scale = float(np.max(np.abs(b.fields[nm])))
        assert scale > 0
        assert float(np.max(np.abs(a.fields[nm] - b.fields[nm]))) <= 1e-5 * scale, nm
    from openem_b200 import flux
    np.testing.assert_allclose(flux.plane_flux(a.phasors["T"].data, sc.grid),
                               flux.plane_flux(b.phasors["T"].data, sc.grid), rtol=1e-4)


def test_modulation_first_order_sidebands():
    """Transmitted sidebands of an index-matched weakly modulated slab against the first-order
    closed form (tests/test_timemod.py:255-300, 5% there) and against the FP64 oracle."""
    from openem_b200 import flux
    sc = scenes.modulated_slab(num_steps=12000)
    g = solver.run(sc, use_shutoff=False, verbose=False)
    fl = flux.plane_flux(g.phasors["T"].data, sc.grid, axis=2)
    r = ref64.run(sc)
    fr = flux.plane_flux(r.phasors["T"], sc.grid, axis=2)
    f = sc.flux_monitors[0].freqs
    mo = sc.modulation
    nz = sc.shape[2]
    kk = np.unique(mo.cell[mo.comp == 0] % nz)
    z = sc.grid.axes[2].edges[kk]
    dz = sc.grid.axes[2].dl_dual[kk]
    k0 = 2 * np.pi * f[1] / C0
    for i in (0, 2):
        kpm = 2 * np.pi * f[i] / C0
        S = abs(np.sum(dz * np.exp(1j * (k0 - kpm) * z)))
        pred = (kpm * 0.01 / 4.0 * S) ** 2
        assert fl[i] / fl[1] == pytest.approx(pred, rel=0.05)
        assert fl[i] / fl[1] == pytest.approx(fr[i] / fr[1], rel=1e-3)


def test_modulation_device_tables_match_host(monkeypatch):
    """The material records of the modulated cells isolated on the device give the same bits as
    the host build."""
    sc = modulated_scene(steps=300)
    monkeypatch.setenv("OEM_B200_TABLES", "host")
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    monkeypatch.setenv("OEM_B200_TABLES", "device")
    b = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for nm in a.fields:
        np.testing.assert_array_equal(a.fields[nm], b.fields[nm])


# ---- fully anisotropic media (openem/kernels/tensor.cu) ----------------------------------------

def test_tensor_rotation_superposition_on_gpu():
    """OpenEM's rotation identity (tests/test_tensor.py:247-288) on the transmitted-plane
    phasors: the tensor run equals cos^2 / sin^2 / sin cos combinations of two scalar runs within
    2e-5 of the largest phasor, the reference's own bound."""
    import test_oracle_golden as tg
    th = 0.37
    sc_t, sc_a, sc_b = tg._tensor_slab(th)
    run = lambda s: solver.run(s, use_shutoff=False, verbose=False)
    rt, ra, rb = run(sc_t), run(sc_a), run(sc_b)
    c, s = np.cos(th), np.sin(th)
    for name in ("T", "R"):
        pt, pa, pb = (r.phasors[name].data for r in (rt, ra, rb))
        want_x = c * c * pa[0] + s * s * pb[0]
        want_y = s * c * (pa[0] - pb[0])
        scale = np.abs(pa[0]).max()
        assert np.abs(pt[0] - want_x).max() < 2e-5 * scale, name
        assert np.abs(pt[1] - want_y).max() < 2e-5 * scale, name
        assert np.abs(want_y).max() > 1e-2 * scale  # the coupling is exercised


def tensor_block_scene(diag=False):
    sd = scenes.small_dispersive(n=30, n_sph=1, n_pml=6, num_steps=200)
    sc = replace(sd, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    rng = np.random.default_rng(4)
    A = rng.normal(size=(3, 3))
    eps = 3.0 * np.eye(3) + 0.4 * (A + A.T)
    sig = np.zeros((3, 3)) if diag else np.array([[0, 150.0, 0], [-150.0, 0, 0], [0, 0, 20.0]])
    if diag:
        eps = np.diag(np.diag(eps))
    ten = scenes.tensor_region(sc, (11, 9, 12), (19, 20, 17), eps, sig)
    return sc, ten, eps


def test_tensor_block_matches_oracle():
    """A symmetric eps tensor with a gyrotropic (antisymmetric) sigma on a block beside a dipole:
    every off-diagonal coupling and the 4-neighbour averages against the FP64 oracle."""
    sc, ten, _ = tensor_block_scene()
    sc = replace(sc, tensor=ten)
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    floor = ref64.fp32_floor(sc, clean=r)
    for nm in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert rel_l2(g.fields[nm], r.fields[nm]) < max(2e-5, 3.0 * floor[nm]), (nm, floor[nm])


def test_diagonal_tensor_equals_scalar_path():
    """OpenEM's degeneracy criterion (tests/test_tensor.py:93-116): a diagonal tensor block
    equals the scalar update with the same eps to float32 rounding. The two runs round
    differently where the point dipole sits inside the block (its current enters the pass-through
    value and is scaled by the M2 row), so each component is held to the float32 floor of the
    scene rather than to zero."""
    sc, ten, eps = tensor_block_scene(diag=True)
    e = [np.array(x) for x in (sc.eps_ex, sc.eps_ey, sc.eps_ez)]
    for c in range(3):
        e[c][11:19, 9:20, 12:17] = eps[c, c]
    scal = replace(sc, eps_ex=e[0], eps_ey=e[1], eps_ez=e[2])
    tens = replace(scal, tensor=ten)
    a = solver.run(tens, use_shutoff=False, return_fields=True, verbose=False)
    b = solver.run(scal, use_shutoff=False, return_fields=True, verbose=False)
    floor = ref64.fp32_floor(scal)
    for nm in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert rel_l2(a.fields[nm], b.fields[nm]) < max(2e-6, 3.0 * floor[nm]), (nm, floor[nm])
