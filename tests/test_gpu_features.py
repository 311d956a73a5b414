"""Boundary and medium features on the GPU against the FP64 oracle: absorber slabs (real and
complex paths). Tolerance: fields within 1e-5 of their field family's norm."""

from dataclasses import replace

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver
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
