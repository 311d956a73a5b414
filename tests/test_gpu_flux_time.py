"""Flux time monitors on the GPU against the FP64 oracle: the per-sample instantaneous flux
series of on-grid, off-grid (two planes), interval / start-step and fully spanned periodic planes,
plus a dipole in a CPML box with planes on all three normal axes. Tolerance: each sample within
1e-4 of the series' peak magnitude. A scene without the monitor keeps bitwise identical
frequency-domain phasors."""

from dataclasses import replace

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver
from openem_b200.model import FluxTimeMonitor

pytestmark = pytest.mark.gpu


def series_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("kw", [dict(), dict(plane_z=0.3125e-6, interval=2, start_step=100),
                                dict(full_span=True)], ids=["on_grid", "frac_interval", "wrap"])
def test_flux_time_matches_oracle(kw):
    sc = scenes.flux_time_plane(nfreq=3, **kw)
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, verbose=False)
    assert series_err(g.flux_time["ft"], r.flux_time["ft"]) < 1e-4


def test_flux_time_all_normal_axes_in_a_cpml_box():
    """A z dipole in vacuum with CPML on every face; flux planes normal to x, y and z with bounds
    off the grid points and planes between Yee boundaries."""
    sd = scenes.small_dispersive(n=28, n_sph=1, n_pml=4, num_steps=260)
    sc = replace(sd, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    grid = sc.grid
    mons = []
    for ax, (name, nd) in enumerate((("fx", 1), ("fy", -1), ("fz", 1))):
        e = np.asarray(grid.axes[ax].edges)
        km = 18
        t = [a for a in range(3) if a != ax]
        tb = tuple((float(grid.axes[a].edges[6]) + 0.3e-9,
                    float(grid.axes[a].edges[21]) - 0.7e-9) for a in t)
        mons.append(FluxTimeMonitor(name=name, axis=ax, plane_index=km, normal_dir=nd,
                                    step_begin=10, step_end=250, interval=3, num_slots=80,
                                    t_bounds=tb, frac=0.35 if ax != 1 else 0.0))
        assert e.size > km + 2
    sc = replace(sc, flux_time_monitors=mons, field_time_monitors=[])
    r = ref64.run(sc)
    g = solver.run(sc, use_shutoff=False, verbose=False)
    for m in mons:
        assert np.abs(r.flux_time[m.name]).max() > 0
        assert series_err(g.flux_time[m.name], r.flux_time[m.name]) < 1e-4, m.name


def test_flux_time_leaves_phasors_bitwise_unchanged():
    sc = scenes.flux_time_plane(nfreq=5, num_steps=600)
    a = solver.run(sc, use_shutoff=False, verbose=False)
    b = solver.run(replace(sc, flux_time_monitors=[]), use_shutoff=False, verbose=False)
    assert np.array_equal(a.phasors["fx"].data, b.phasors["fx"].data)
    assert a.flux_time["ft"].size == 600 and not b.flux_time
