"""Geometry of the instantaneous (time-domain) flux of a ``FluxTimeMonitor``: the colocated
integration convention of ``openem/flux.py:146-164, 307-578``, restated.

On each primal plane of the monitor (one, or two when the plane lies a fraction ``frac`` past a
Yee boundary) the four tangential components are brought onto the primal boundary points:

* along the normal, E already sits on the plane; H is interpolated linearly by coordinate
  between the cell centres on both sides (``kh``, ``kh + 1``);
* along the transverse axis on which a component sits at cell centres (E_t1 and H_t2 along t1,
  E_t2 and H_t1 along t2), it is interpolated from the two neighbouring centres onto the edge;
* the samples are the edges whose dual cells (clipped at the monitor bounds) have non-zero width,
  the face element is the product of those trapezoid widths, with the sign of ``normal_dir``
  (and -1 for a y normal, the cyclic order);
* a sample at the very low edge of a symmetry-folded axis reads the folded cell 0 with the
  component's mirror parity; on a fully spanned periodic axis the last sample is merged into
  sample 0 and its low neighbour wraps to the last cell; samples at an absorbing grid end are
  dropped, elsewhere at the grid edge the monitor is refused.

The flux of one sample step is ``s = sum_planes w sum dS (E_t1 H_t2 - E_t2 H_t1)`` with H the
time average of its two half steps. :func:`geometry` builds the tables on the host (float64),
:func:`sample` evaluates ``s`` with numpy (the check the device kernel is tested against), and
:func:`device_tables` flattens the geometry into the index / weight arrays the device kernel
reads.
"""

from __future__ import annotations

import numpy as np

ABSORBING = ("PML", "StablePML", "Absorber")
# mirror parity of each component under reflection through a plane normal to x, y, z
MIRROR_SIGN = {"Ex": (-1, 1, 1), "Ey": (1, -1, 1), "Ez": (1, 1, -1),
               "Hx": (1, -1, -1), "Hy": (-1, 1, -1), "Hz": (-1, -1, 1)}
LABELS = ("Eu", "Hv", "Ev", "Hu")


def transverse_axes(axis: int):
    t = [a for a in range(3) if a != axis]
    return t[0], t[1]


def axis_weights(edges, lo: float, hi: float):
    """Sample run ``[i0, i1]`` of primal edges and their dual-cell widths clipped at
    ``[lo, hi]`` (the ends' cells reach only to the end edges)."""
    e = np.asarray(edges, dtype=np.float64)
    mid = 0.5 * (e[:-1] + e[1:])
    lower = np.concatenate([e[:1], mid])
    upper = np.concatenate([mid, e[-1:]])
    w = np.maximum(np.clip(upper, lo, hi) - np.clip(lower, lo, hi), 0.0)
    nz = np.flatnonzero(w > 0.0)
    if nz.size == 0:
        raise ValueError(f"the monitor range [{lo}, {hi}] intersects no integration cell")
    return int(nz[0]), int(nz[-1]), w[nz[0]:nz[-1] + 1]


def normal_planes(grid, mon):
    """The one or two primal planes along the normal with their weights, and the H colocation
    (cells ``kh``, ``kh + 1`` and weights) onto each."""
    ax = mon.axis
    e = np.asarray(grid.axes[ax].edges, dtype=np.float64)
    c = grid.axes[ax].centers
    km, fr = int(mon.plane_index), float(mon.frac)
    out = []
    for w, k in ((1.0 - fr, km), (fr, km + 1)):
        if w == 0.0:
            continue
        kh = k - 1
        if not 0 <= kh < c.size - 1:
            raise ValueError(f"flux time monitor {mon.name}: plane {k} along {'xyz'[ax]} is too "
                             "close to the grid edge for the H colocation")
        wlo = (float(c[kh + 1]) - float(e[k])) / float(c[kh + 1] - c[kh])
        out.append({"w": w, "ke": k, "kh": kh, "wh": (wlo, 1.0 - wlo)})
    return out


def tangential_axis(axt, mon, p: int, tax):
    """Samples, interpolation cells and weights along transverse axis ``tax[p]``."""
    lo, hi = mon.t_bounds[p]
    i0, i1, w = axis_weights(axt.edges, lo, hi)
    n = len(axt.edges) - 1
    fold = i0 == 0 and axt.boundary_lo in ("SymmetryPEC", "SymmetryPMC")
    wrap = i0 == 0 and i1 == n and axt.boundary_lo == "Periodic" and axt.boundary_hi == "Periodic"
    for end, bad in (("lo", i0 < 1 and not fold and not wrap), ("hi", i1 > n - 1 and not wrap)):
        if bad and getattr(axt, f"boundary_{end}") not in ABSORBING:
            raise ValueError(f"flux time monitor {mon.name}: samples [{i0}, {i1}] along "
                             f"{'xyz'[tax[p]]} reach the {end} grid edge, which is not absorbing")
    if wrap:
        w = np.concatenate([[w[0] + w[-1]], w[1:-1]])
        i1 = n - 1
    if i0 < 1 and not fold and not wrap:
        w = w[1 - i0:]
        i0 = 1
    if i1 > n - 1:
        w = w[:n - 1 - i1]
        i1 = n - 1
    e = np.asarray(axt.edges, dtype=np.float64)
    eg, cen = e[i0:i1 + 1], axt.centers
    if fold:
        below = np.concatenate([[2.0 * eg[0] - cen[0]], cen[0:i1]])
    elif wrap:
        below = np.concatenate([[cen[-1] - float(e[-1] - e[0])], cen[0:i1]])
    else:
        below = cen[i0 - 1:i1]
    wlo = (cen[i0:i1 + 1] - eg) / (cen[i0:i1 + 1] - below)
    cells_hi = np.arange(i0, i1 + 1)
    cells_lo = cells_hi - 1
    wlo_c = {lbl: wlo.copy() for lbl in LABELS}
    if wrap:
        cells_lo[0] = n - 1
    elif fold:
        cells_lo[0] = 0
        s_ax = -1.0 if axt.boundary_lo == "SymmetryPEC" else 1.0
        t1, t2 = tax
        t = tax[p]
        pairs = ((("Eu", "E" + "xyz"[t1]), ("Hv", "H" + "xyz"[t2])) if p == 0 else
                 (("Ev", "E" + "xyz"[t2]), ("Hu", "H" + "xyz"[t1])))
        for lbl, comp in pairs:
            wlo_c[lbl][0] *= MIRROR_SIGN[comp][t] * s_ax
    return {"edges": np.arange(i0, i1 + 1), "lo": cells_lo, "hi": cells_hi, "wlo": wlo_c,
            "whi": 1.0 - wlo, "trap": w}


def geometry(grid, mon) -> dict:
    ax = int(mon.axis)
    t1, t2 = transverse_axes(ax)
    g = {"axis": ax, "tax": (t1, t2), "planes": normal_planes(grid, mon)}
    g["t"] = [tangential_axis(grid.axes[t], mon, p, (t1, t2)) for p, t in enumerate((t1, t2))]
    sign = float(mon.normal_dir) * (-1.0 if ax == 1 else 1.0)
    g["dS"] = sign * np.outer(g["t"][0]["trap"], g["t"][1]["trap"])
    return g


def _take(F, ax, k, sel1, sel2, t1, t2):
    idx = [None, None, None]
    idx[ax] = k
    idx[t1] = sel1[:, None]
    idx[t2] = sel2[None, :]
    return np.asarray(F)[tuple(idx)]


def colocate(F, g: dict, label: str, plane: int):
    """One tangential component (``label`` in Eu, Ev, Hu, Hv) on the samples of one plane,
    ``(n1, n2)`` float64; ``F`` is the 3D field array of that component."""
    ax, (t1, t2) = g["axis"], g["tax"]
    pe = g["planes"][plane]
    along = 0 if label in ("Eu", "Hv") else 1
    a0, a1 = g["t"]
    if along == 0:
        lo = (a0["lo"], a1["edges"])
        hi = (a0["hi"], a1["edges"])
    else:
        lo = (a0["edges"], a1["lo"])
        hi = (a0["edges"], a1["hi"])

    def normal(sel):
        if label[0] == "E":
            return _take(F, ax, pe["ke"], sel[0], sel[1], t1, t2).astype(np.float64)
        w0, w1 = pe["wh"]
        return (w0 * _take(F, ax, pe["kh"], sel[0], sel[1], t1, t2).astype(np.float64)
                + w1 * _take(F, ax, pe["kh"] + 1, sel[0], sel[1], t1, t2))
    wl = g["t"][along]["wlo"][label]
    wh = g["t"][along]["whi"]
    shape = (-1, 1) if along == 0 else (1, -1)
    return wl.reshape(shape) * normal(lo) + wh.reshape(shape) * normal(hi)


def sample(e_t, h_t, g: dict) -> float:
    """``s = sum_planes w sum dS (E_t1 H_t2 - E_t2 H_t1)`` of 3D fields ``e_t = (E_t1, E_t2)``,
    ``h_t = (H_t1, H_t2)`` (the caller supplies the time-averaged H)."""
    s = 0.0
    for p, pe in enumerate(g["planes"]):
        eu = colocate(e_t[0], g, "Eu", p)
        ev = colocate(e_t[1], g, "Ev", p)
        hu = colocate(h_t[0], g, "Hu", p)
        hv = colocate(h_t[1], g, "Hv", p)
        s += pe["w"] * float(((eu * hv - ev * hu) * g["dS"]).sum())
    return s


def device_tables(g: dict) -> dict:
    """The flat arrays of the device kernel: per plane (w, ke, kh, wh0, wh1); per transverse
    axis the edge index, the low / high interpolation cells, the low weights of the two labels
    that interpolate along it and the high weights; the face elements."""
    a0, a1 = g["t"]
    pl = g["planes"]
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    return {
        "nplanes": len(pl),
        "w": f64([p["w"] for p in pl]), "ke": i32([p["ke"] for p in pl]),
        "kh": i32([p["kh"] for p in pl]),
        "wh": f64([v for p in pl for v in p["wh"]]),
        "n1": int(a0["edges"].size), "e1": i32(a0["edges"]), "lo1": i32(a0["lo"]),
        "hi1": i32(a0["hi"]), "wlo1": f64(np.stack([a0["wlo"]["Eu"], a0["wlo"]["Hv"]])),
        "whi1": f64(a0["whi"]),
        "n2": int(a1["edges"].size), "e2": i32(a1["edges"]), "lo2": i32(a1["lo"]),
        "hi2": i32(a1["hi"]), "wlo2": f64(np.stack([a1["wlo"]["Ev"], a1["wlo"]["Hu"]])),
        "whi2": f64(a1["whi"]),
        "dS": f64(g["dS"]),
    }
