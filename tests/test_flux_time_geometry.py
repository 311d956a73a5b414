"""Geometry of the instantaneous colocated flux (openem/flux.py:307-578), checked with the
known-answer properties OpenEM's own tests use (tests/test_fluxtime.py): linear colocation is
exact on affine fields, a fully spanned periodic plane wraps and covers one whole period, the
flux follows a one-cell translation of a periodic field, and the face elements are the clipped
trapezoid widths."""

import numpy as np
import pytest

from openem_b200 import flux_time as FT
from openem_b200.model import Axis, FluxTimeMonitor, Grid

UM = 1e-6


def mon(axis, km, t_bounds, frac=0.0, normal_dir=1, name="ft"):
    return FluxTimeMonitor(name=name, axis=axis, plane_index=km, normal_dir=normal_dir,
                           step_begin=0, step_end=1, interval=1, num_slots=1,
                           t_bounds=t_bounds, frac=frac)


def yee(grid, comp):
    kind, d = comp[0], "xyz".index(comp[1])
    out = []
    for i, ax in enumerate(grid.axes):
        on_center = (i == d) if kind == "E" else (i != d)
        out.append(ax.centers if on_center else np.asarray(ax.edges[:-1], np.float64))
    return out


def test_colocation_exact_on_affine_fields():
    rng = np.random.default_rng(1)
    edges = [np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, n))]) for n in (12, 14, 16)]
    grid = Grid(*(Axis(edges=e, boundary_lo="PML", boundary_hi="PML") for e in edges))
    a, b = rng.standard_normal(), rng.standard_normal(3)
    for ax in range(3):
        t1, t2 = FT.transverse_axes(ax)
        e = grid.axes[ax].edges
        x0 = 0.6 * e[4] + 0.4 * e[5]
        km = int(np.searchsorted(e, x0, side="right")) - 1
        et = [grid.axes[t].edges for t in (t1, t2)]
        m = mon(ax, km, ((et[0][2] + 0.13, et[0][-3] - 0.2), (et[1][3] - 0.1, et[1][-2] - 0.3)),
                frac=(x0 - e[km]) / (e[km + 1] - e[km]))
        g = FT.geometry(grid, m)
        for p, pe in enumerate(g["planes"]):
            xs = [None, None, None]
            xs[ax] = np.array([grid.axes[ax].edges[pe["ke"]]])
            xs[t1] = np.asarray(grid.axes[t1].edges)[g["t"][0]["edges"]]
            xs[t2] = np.asarray(grid.axes[t2].edges)[g["t"][1]["edges"]]
            want = a + b[ax] * xs[ax][0] + b[t1] * xs[t1][:, None] + b[t2] * xs[t2][None, :]
            for lbl, comp in (("Eu", "E" + "xyz"[t1]), ("Ev", "E" + "xyz"[t2]),
                              ("Hu", "H" + "xyz"[t1]), ("Hv", "H" + "xyz"[t2])):
                X, Y, Z = np.meshgrid(*yee(grid, comp), indexing="ij")
                F = a + b[0] * X + b[1] * Y + b[2] * Z
                np.testing.assert_allclose(FT.colocate(F, g, lbl, p), want, rtol=1e-12,
                                           atol=1e-12)


def periodic_grid():
    edges = [np.linspace(0.0, 0.4 * UM, 17), np.linspace(0.0, 0.4 * UM, 17),
             np.linspace(0.0, 1.6 * UM, 65)]
    return Grid(Axis(edges=edges[0], boundary_lo="Periodic", boundary_hi="Periodic"),
                Axis(edges=edges[1], boundary_lo="Periodic", boundary_hi="Periodic"),
                Axis(edges=edges[2], boundary_lo="PML", boundary_hi="PML"))


def test_full_periodic_plane_wraps_and_covers_one_period():
    grid = periodic_grid()
    g = FT.geometry(grid, mon(2, 30, ((0.0, 0.4 * UM), (0.0, 0.4 * UM)), frac=0.3))
    for p in (0, 1):
        assert g["t"][p]["lo"][0] == 15 and g["t"][p]["edges"].size == 16
        ws = list(g["t"][p]["wlo"].values())
        assert all(np.array_equal(w, ws[0]) for w in ws[1:])
    np.testing.assert_allclose(float(np.abs(g["dS"]).sum()), (0.4 * UM) ** 2, rtol=1e-12)


def test_periodic_wrap_translation_invariance():
    rng = np.random.default_rng(3)
    grid = periodic_grid()
    g = FT.geometry(grid, mon(2, 30, ((0.0, 0.4 * UM), (0.0, 0.4 * UM)), frac=0.3))
    f = {c: rng.standard_normal((16, 16, 64)) for c in ("Ex", "Ey", "Hx", "Hy")}
    s0 = FT.sample((f["Ex"], f["Ey"]), (f["Hx"], f["Hy"]), g)
    for axis_t in (0, 1):
        fr = {c: np.roll(v, 1, axis=axis_t) for c, v in f.items()}
        s1 = FT.sample((fr["Ex"], fr["Ey"]), (fr["Hx"], fr["Hy"]), g)
        np.testing.assert_allclose(s1, s0, rtol=1e-10)


def test_face_elements_are_clipped_trapezoid_widths():
    e = np.array([0.0, 1.0, 2.5, 3.0, 4.0, 6.0])
    i0, i1, w = FT.axis_weights(e, 0.4, 3.2)
    # dual cells: [0,0.5] [0.5,1.75] [1.75,2.75] [2.75,3.5] [3.5,5] [5,6] clipped to [0.4,3.2]
    assert (i0, i1) == (0, 3)
    np.testing.assert_allclose(w, [0.1, 1.25, 1.0, 0.45])
    with pytest.raises(ValueError):
        FT.axis_weights(e, 7.0, 8.0)


def test_symmetry_fold_applies_mirror_parity():
    edges = [np.linspace(0.0, 1.0, 11)] * 2 + [np.linspace(0.0, 2.0, 21)]
    grid = Grid(Axis(edges=edges[0], boundary_lo="SymmetryPEC", boundary_hi="PML"),
                Axis(edges=edges[1], boundary_lo="PML", boundary_hi="PML"),
                Axis(edges=edges[2], boundary_lo="PML", boundary_hi="PML"))
    g = FT.geometry(grid, mon(2, 10, ((0.0, 0.55), (0.2, 0.8))))
    a = g["t"][0]
    assert a["lo"][0] == 0 and a["edges"][0] == 0
    # x fold, PEC symmetry (s = -1): Ex has parity -1 -> +1 x (-1) ... Hy parity -1
    assert a["wlo"]["Eu"][0] == pytest.approx(0.5 * (-1) * (-1))
    assert a["wlo"]["Hv"][0] == pytest.approx(0.5 * (-1) * (-1))


def test_refuses_samples_on_a_reflecting_edge():
    edges = [np.linspace(0.0, 1.0, 11)] * 2 + [np.linspace(0.0, 2.0, 21)]
    grid = Grid(Axis(edges=edges[0], boundary_lo="PEC", boundary_hi="PEC"),
                Axis(edges=edges[1], boundary_lo="PML", boundary_hi="PML"),
                Axis(edges=edges[2], boundary_lo="PML", boundary_hi="PML"))
    with pytest.raises(ValueError):
        FT.geometry(grid, mon(2, 10, ((0.0, 1.0), (0.2, 0.8))))
    FT.geometry(grid, mon(2, 10, ((0.2, 0.8), (0.0, 1.0))))  # absorbing y ends: dropped
