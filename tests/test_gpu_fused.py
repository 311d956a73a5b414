"""The fused H + E step (two field banks) against the two-kernel warp-specialised step: bit for
bit on fields, DFT phasors, time samples and flux-time series, over grids with ragged sizes
(ny not a multiple of 4, nz not of 128, nx not of the x chunk), mixed boundaries (CPML, PEC,
PMC, symmetry, periodic x), Drude + Lorentz media with loss, modulation, and x chunks short
enough that every chunk starts with its neighbour-plane pass. Also against the FP64 oracle."""

from dataclasses import replace

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver
from openem_b200.model import (Axis, FieldMonitor, FluxMonitor, FluxTimeMonitor, GaussianPulse,
                               Grid, PointDipole, Scene, TimeModulation, sample_waveform)

pytestmark = pytest.mark.gpu

DL = 0.02e-6


def axis(n, lo, hi, n_pml):
    a = n_pml if lo == "PML" else 0
    b = n_pml if hi == "PML" else 0
    k = np.arange(-a, n - a + 1, dtype=np.float64)
    del b
    return Axis(k * DL, lo, hi)


def mixed_scene(shape=(37, 23, 150), bounds=(("PML", "PML"), ("PEC", "PML"), ("PML", "PMC")),
                n_pml=6, steps=140, seed=3, disp=True):
    axes = [axis(n, lo, hi, n_pml) for n, (lo, hi) in zip(shape, bounds)]
    grid = Grid(*axes)
    dt = scenes.courant_dt([a.dl for a in axes])
    pml = {}
    from openem_b200.model import PMLParams, pml_build
    for a, ax in enumerate(axes):
        for side, bnd in (("lo", ax.boundary_lo), ("hi", ax.boundary_hi)):
            if bnd == "PML":
                pml[(a, side)] = pml_build(PMLParams(num_layers=n_pml),
                                           float(ax.dl[0] if side == "lo" else ax.dl[-1]),
                                           side, dt)
    rng = np.random.default_rng(seed)
    eps = [np.ones(shape) for _ in range(3)]
    for c in range(3):
        sl = tuple(slice(s // 3, 2 * s // 3) for s in shape)
        eps[c][sl] = 1.0 + 3.0 * rng.random(tuple(x.stop - x.start for x in sl))
    sig = [np.where(e > 3.5, 500.0, 0.0) for e in eps]
    pulse = GaussianPulse(freq0=2e14, fwidth=1e14)
    wf = sample_waveform(pulse, dt, steps)
    c = tuple(s // 2 for s in shape)
    dips = [PointDipole(component=2, indices=np.array([c]), coef=np.array([1.0 / DL ** 3]),
                        waveform=wf),
            PointDipole(component=0, indices=np.array([(c[0] - 3, c[1] + 2, c[2] + 5)]),
                        coef=np.array([0.7 / DL ** 3]), waveform=wf)]
    freqs = np.linspace(1.5e14, 2.5e14, 5)
    fmon = FieldMonitor(name="box", freqs=freqs, origin=(3, 2, 40), box=(20, 15, 60))
    flux = FluxMonitor(name="fz", axis=2, plane_index=100, normal_dir=1, freqs=freqs,
                       source_spectrum=np.ones(5, complex))
    ft = FluxTimeMonitor(name="ftz", axis=2, plane_index=90, normal_dir=1, step_begin=5,
                         step_end=steps, interval=2, num_slots=(steps - 5 + 1) // 2,
                         t_bounds=((axes[0].edges[8], axes[0].edges[30]),
                                   (axes[1].edges[3], axes[1].edges[18])), frac=0.25)
    sc = Scene(grid=grid, dt=dt, num_time_steps=steps, shutoff=1e-5, eps_ex=eps[0],
               eps_ey=eps[1], eps_ez=eps[2], pml=pml, sigma_ex=sig[0], sigma_ey=sig[1],
               sigma_ez=sig[2], dipoles=dips, field_monitors=[fmon], flux_monitors=[flux],
               flux_time_monitors=[ft])
    sc = scenes.with_time_monitor(sc, box=(5, 4, 7), interval=3)
    if disp:
        # Drude + Lorentz poles (the DC pole folded into sigma) on the dielectric block
        dt_ = sc.dt
        poles, sigma = scenes.split_dc(scenes.drude_poles(1.4e16, 1e14)
                                       + scenes.lorentz_poles(1.5, 4e14, 5e13), dt_)
        am1, b = scenes.trap_coeffs(poles, dt_)
        masks = [e > 3.0 for e in eps]
        disp_ = scenes.build_dispersion(masks, am1, b, shape)
        sig2 = [np.where(masks[c], sigma, sig[c]) for c in range(3)]
        sc = replace(sc, dispersion=disp_, sigma_ex=sig2[0], sigma_ey=sig2[1], sigma_ez=sig2[2])
    return sc


def run_both(sc, monkeypatch, steps=None, xchunk=None):
    out = {}
    for kind in ("fused", "ws"):
        monkeypatch.setenv("OEM_B200_KERNELS", kind)
        if xchunk:
            monkeypatch.setenv("OEM_B200_XCHUNK", str(xchunk))
        stats = {}
        out[kind] = solver.run(sc, num_steps=steps, use_shutoff=False, return_fields=True,
                               verbose=False, stats=stats)
        out[kind + "_launches"] = stats["launches_per_step"]
    # the fused pair replaces the two update kernels (and a separate pole pass stays)
    assert out["fused_launches"] == out["ws_launches"] - 1
    return out


def assert_same(a, b):
    for nm in a.fields:
        np.testing.assert_array_equal(a.fields[nm], b.fields[nm], err_msg=nm)
    for nm in a.phasors:
        np.testing.assert_array_equal(a.phasors[nm].data, b.phasors[nm].data, err_msg=nm)
    for nm in a.field_phasors:
        np.testing.assert_array_equal(a.field_phasors[nm], b.field_phasors[nm], err_msg=nm)
    for nm in a.time_samples:
        np.testing.assert_array_equal(a.time_samples[nm], b.time_samples[nm], err_msg=nm)
    for nm in a.flux_time:
        np.testing.assert_array_equal(a.flux_time[nm], b.flux_time[nm], err_msg=nm)


@pytest.mark.parametrize("bounds,xchunk", [
    ((("PML", "PML"), ("PEC", "PML"), ("PML", "PMC")), None),
    ((("PML", "PML"), ("PEC", "PML"), ("PML", "PMC")), 5),
    ((("Periodic", "Periodic"), ("PMC", "PEC"), ("SymmetryPEC", "PML")), 7),
    ((("SymmetryPMC", "PML"), ("PML", "SymmetryPEC"), ("PEC", "PEC")), 3),
])
def test_fused_equals_two_kernel_path(monkeypatch, bounds, xchunk):
    sc = mixed_scene(bounds=bounds)
    r = run_both(sc, monkeypatch, xchunk=xchunk)
    assert_same(r["fused"], r["ws"])
    assert np.abs(r["fused"].fields["Ez"]).max() > 0


def test_fused_with_modulation_equals_two_kernel_path(monkeypatch):
    sc = mixed_scene(disp=False)
    nx, ny, nz = sc.shape
    cells = np.arange(0, nx * ny * nz, 97)
    mo = TimeModulation(3e13, np.repeat([0, 1, 2], cells.size)[:cells.size],
                        cells, np.full(cells.size, 0.2), np.linspace(0, 2, cells.size))
    r = run_both(replace(sc, modulation=mo), monkeypatch)
    assert_same(r["fused"], r["ws"])


def test_fused_large_grid_equals_two_kernel_path(monkeypatch):
    """A 200^3 dispersive-spheres grid: several 128-cell z tiles, device-built tables."""
    sc = scenes.dispersive_spheres(n=200, n_sph=6, num_steps=30)
    r = run_both(sc, monkeypatch)
    assert_same(r["fused"], r["ws"])


def test_fused_matches_oracle(monkeypatch):
    monkeypatch.setenv("OEM_B200_KERNELS", "fused")
    sc = mixed_scene(disp=False, steps=120)
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        den = np.sqrt(sum(np.linalg.norm(r.fields[n]) ** 2 for n in fam))
        err = max(np.linalg.norm(g.fields[n] - r.fields[n]) for n in fam) / den
        assert err < 1e-5, fam
