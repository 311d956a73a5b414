"""Algorithmic byte counts of the step, used for the HBM roofline.

Per cell-update, the step must read and write the six field components once (48 B), read a
material description, update the CPML psi auxiliaries of the cells in the boundary slabs (two
psi arrays per field family per slab axis, read and written: 16 B per slab cell per family),
update the ADE pole states of the dispersive entries (a complex float32 read and written per
pole: 16 B), and read the monitored points (six float32 per point per step).

``step_bytes_per_cell`` uses OpenEM's material description (three uint16 coefficient indices,
6 B per cell) so the figure is comparable across implementations; the per-kernel counts use
what this engine's kernels must move (one uint16 material index, 2 B per cell, read by the E
update only).
"""

from __future__ import annotations

import json
import os
import pathlib

import numpy as np

FALLBACK_HBM_GBS = 6650.0


def _slab_cells(sc) -> dict:
    nx, ny, nz = (int(v) for v in sc.shape)
    dims = (nx, ny, nz)
    out = {}
    for a in range(3):
        lo = sc.pml.get((a, "lo"))
        hi = sc.pml.get((a, "hi"))
        layers = (0 if lo is None else int(np.asarray(lo.a_E).size)) + \
                 (0 if hi is None else int(np.asarray(hi.a_E).size))
        out[a] = layers * nx * ny * nz // dims[a]
    return out


def counts(sc) -> dict:
    ncell = int(np.prod(sc.shape))
    slabs = _slab_cells(sc)
    n_pole = 0 if sc.dispersion is None else int(sc.dispersion.n_pole)
    mon_pts = 0
    for m in sc.field_monitors:
        mon_pts += int(np.prod(m.box))
    for m in sc.flux_monitors:
        t = [sc.shape[a] for a in range(3) if a != m.axis]
        mon_pts += int(t[0] * t[1])
    return {"ncell": ncell, "slab_cells": slabs, "n_pole": n_pole, "monitor_points": mon_pts}


def step_bytes_per_cell(sc) -> float:
    """Algorithmic bytes per cell-update of one full step (OpenEM's 6-byte material form)."""
    c = counts(sc)
    n = c["ncell"]
    psi = 32.0 * sum(c["slab_cells"].values())
    ade = 16.0 * c["n_pole"]
    mon = 24.0 * c["monitor_points"]
    return (48.0 + 6.0) + (psi + ade + mon) / n


def step_bytes_per_cell_complex(sc) -> float:
    """Algorithmic bytes per complex cell-update of the Bloch path: both parts of the six fields
    read and written (96 B), the 6-byte material form, both parts of the slab psi (64 B per slab
    cell and axis) and both parts of the four tangential components of every flux-plane point
    read once per step (32 B per point)."""
    c = counts(sc)
    n = c["ncell"]
    psi = 64.0 * sum(c["slab_cells"].values())
    mon = 32.0 * c["monitor_points"]
    return (96.0 + 6.0) + (psi + mon) / n


def kernel_bytes(sc, box_snapshots_in_e: bool = False) -> dict:
    """Algorithmic bytes per launch of this engine's step kernels.

    ``update_h``: E read, H read and written (36 B per cell) plus the H-side psi of the slab
    cells. ``update_e``: H read, E read and written, the material index (38 B per cell), the
    E-side psi, one float32 polarisation current per dispersive (component, cell) entry, and,
    when the E update writes the box monitors' snapshots itself, six float32 per box point.
    ``ade`` (the separate pole pass): each pole state read and written (16 B), and per entry
    E^n read and the current written (8 B). ``update_he`` (the fused step over two field banks):
    E and H each read once and written once (48 B per cell), the material index, both families'
    psi, and the polarisation currents."""
    c = counts(sc)
    n = c["ncell"]
    psi = 16.0 * sum(c["slab_cells"].values())
    n_entry = 0 if sc.dispersion is None else int(sc.dispersion.n_entry)
    snap = 24.0 * sum(int(np.prod(m.box)) for m in sc.field_monitors) if box_snapshots_in_e \
        else 0.0
    return {"update_h": 36.0 * n + psi,
            "update_e": 38.0 * n + psi + 4.0 * n_entry + snap,
            "ade": 16.0 * c["n_pole"] + 8.0 * n_entry,
            "update_he": 50.0 * n + 2.0 * psi + 4.0 * n_entry}


def kernel_bytes_complex(sc) -> dict:
    """Per launch of the complex split update, which runs the real update once on each part:
    twice the real kernels' bytes (the seam-face terms are below 1% and not counted)."""
    kb = kernel_bytes(sc)
    return {"update_h": 2.0 * kb["update_h"], "update_e": 2.0 * kb["update_e"]}


def measured_peaks(root=None) -> dict:
    """The measured HBM copy bandwidth (GB/s) of this pool's B200s, or the fallback figure."""
    root = pathlib.Path(root or pathlib.Path(__file__).resolve().parent.parent)
    p = root / "MEASURED_PEAKS.json"
    env = os.environ.get("OEM_B200_PEAKS")
    if env:
        p = pathlib.Path(env)
    try:
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}
