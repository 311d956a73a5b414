"""Plane flux of monitor phasors (``openem/flux.py:60-107``), used by the phasor-convergence
early-termination criterion: ``P(f) = 1/2 Re sum [E_t1 H_t2* dA_1 - E_t2 H_t1* dA_2]`` with each
term's dual face element at its own staggered position; a 2D flat axis counts as 1 um."""

from __future__ import annotations

import numpy as np

FLAT_AXIS_M = 1.0e-6


def axis_dl(ax):
    if ax.is_flat:
        one = np.array([FLAT_AXIS_M])
        return one, one
    return ax.dl, ax.dl_dual


def area_weights(grid, axis: int = 2):
    t1, t2 = [a for a in range(3) if a != axis]
    (dl1, dld1), (dl2, dld2) = axis_dl(grid.axes[t1]), axis_dl(grid.axes[t2])
    return dl1[:, None] * dld2[None, :], dld1[:, None] * dl2[None, :]


def plane_flux(data, grid, transverse=None, axis: int = 2) -> np.ndarray:
    dA_x, dA_y = area_weights(grid, axis)
    if transverse is not None:
        mask = np.zeros(dA_x.shape)
        (j0, j1), (k0, k1) = transverse
        mask[j0:j1 + 1, k0:k1 + 1] = 1.0
        dA_x = dA_x * mask
        dA_y = dA_y * mask
    ex, ey, hx, hy = data[0], data[1], data[2], data[3]
    tx = np.real(ex * np.conj(hy)) * dA_x[None]
    ty = np.real(ey * np.conj(hx)) * dA_y[None]
    return 0.5 * (tx.sum(axis=(1, 2)) - ty.sum(axis=(1, 2)))
