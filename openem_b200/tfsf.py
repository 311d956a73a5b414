"""Total-field / scattered-field box at normal incidence: the incident wave comes from a 1D
auxiliary Yee line with the 3D grid's dt, spacing and permittivity profile along the injection
axis, and the six box faces get the incident-field corrections of the 3D difference equations.

Restated from ``openem/tfsf1d.py:143-412`` (the 1D line: H half step with the injection at cell
``kh``, E step with the injection at edge ``inj``, ``ex_tab[n] = E^n`` on the box edges and
``hy_tab[n] = H^{n+1/2}`` on the box cells ``alo - 1 .. ahi``, runway of ``1.05 c dt n / dl + 64``
cells at each end and a causal window, far ends checked to stay below ``1e-30`` of the injection
peak) and ``openem/sources_setup.py:120-318`` (placement checks and the 16 face corrections).

With the injection axis ``a`` and the transverse axes ``u = (a+1) % 3``, ``v = (a+2) % 3`` the
incident field is ``E = (b_u u + b_v v) E1D``, ``H = (b_u v - b_v u) H1D``; the corrections
(``N = ahi - alo + 1``; E-step terms are also multiplied by the cell's ``cb``):

    E_u  at a = alo / ahi     (+b_u, -b_u) / dl*_a          H row, column 0 / N
    E_v  at a = alo / ahi     (+b_v, -b_v) / dl*_a          H row, column 0 / N
    E_a  at u = ulo / uhi     (-b_u, +b_u) / dl*_u          H row, column 1 + (a - alo)
    E_a  at v = vlo / vhi     (-b_v, +b_v) / dl*_v          H row, column 1 + (a - alo)
    H_v  at a = alo-1 / ahi   (+b_u, -b_u) ch / dl_a        E row, column 0 / N - 1
    H_u  at a = alo-1 / ahi   (-b_v, +b_v) ch / dl_a        E row, column 0 / N - 1
    H_a  at v = vlo-1 / vhi   (-b_u, +b_u) ch / dl_v        E row, column (a - alo)
    H_a  at u = ulo-1 / uhi   (+b_v, -b_v) ch / dl_u        E row, column (a - alo)
"""

from __future__ import annotations

import numpy as np

from openem_b200.model import C_0, EPSILON_0, MU_0

SIGNS = {+1: (1.0, 1.0), -1: (-1.0, -1.0)}
RUNWAY_MARGIN = 1.05
RUNWAY_PAD = 64
UNTOUCHED_CELLS = 8
TAIL_MAX_REL = 1e-30
GAP = 4  # cells of the 1D box column beyond each box face


def cyclic_axes(a: int):
    return (a + 1) % 3, (a + 2) % 3


def runway_cells(n_steps: int, dt: float, dl: float) -> int:
    return int(np.ceil(RUNWAY_MARGIN * n_steps * C_0 * dt / dl)) + RUNWAY_PAD


def line_tables(dl1, eps1, dt: float, inj: int, direction: int, ex_inc, hy_inc, n_steps: int,
                col0: int, n_col_e: int, sigma1=None, window: bool = True):
    """Run the 1D line for ``n_steps`` and return ``(ex_tab, hy_tab)``: ``(n_steps + 1,
    n_col_e)`` E^n on edges ``col0 ..`` and ``(n_steps, n_col_e + 1)`` H^{n+1/2} on cells
    ``col0 - 1 ..``. Raises if the runway ends were reached."""
    dl1 = np.ascontiguousarray(dl1, dtype=np.float64)
    eps1 = np.ascontiguousarray(eps1, dtype=np.float64)
    n1 = int(dl1.size)
    if eps1.shape != (n1,):
        raise ValueError(f"eps1 has shape {eps1.shape}, expected ({n1},)")
    if np.size(ex_inc) < n_steps + 1 or np.size(hy_inc) < n_steps + 1:
        raise ValueError(f"the injection tables hold {np.size(ex_inc)} samples, {n_steps} steps "
                         f"need {n_steps + 1}")
    if not (UNTOUCHED_CELLS < inj < n1 - UNTOUCHED_CELLS):
        raise ValueError(f"injection plane {inj} is too close to the 1D ends (n1={n1})")
    if not (col0 > 0 and col0 + n_col_e < n1):
        raise ValueError(f"box columns [{col0}, {col0 + n_col_e}) outside the 1D line (n1={n1})")
    dld1 = np.empty_like(dl1)
    dld1[1:] = 0.5 * (dl1[1:] + dl1[:-1])
    dld1[0] = dl1[0]
    ch = dt / MU_0 / dl1
    s = (np.zeros_like(eps1) if sigma1 is None
         else np.ascontiguousarray(sigma1, np.float64) * dt / (2.0 * EPSILON_0))
    den = eps1 + s
    ca = (eps1 - s) / den
    cb = dt / EPSILON_0 / den / dld1
    sh, se = SIGNS[direction]
    kh = inj - 1 if direction > 0 else inj
    coef_h = sh * dt / MU_0 / dl1[kh]
    coef_e = se * dt / EPSILON_0 / den[inj] / dld1[inj]
    ex1 = np.zeros(n1)
    hy1 = np.zeros(n1)
    ex_tab = np.zeros((n_steps + 1, n_col_e))
    hy_tab = np.zeros((n_steps, n_col_e + 1))
    se_ = slice(col0, col0 + n_col_e)
    sh_ = slice(col0 - 1, col0 + n_col_e)
    for n in range(n_steps):
        if window:  # nothing outside n + 2 + pad cells of the injection point has moved yet
            w = n + 2 + RUNWAY_PAD
            lo, hi = max(0, inj - w), min(n1, inj + w + 1)
        else:
            lo, hi = 0, n1
        bh, ae = min(hi, n1 - 1), max(lo, 1)
        hy1[lo:bh] -= ch[lo:bh] * (ex1[lo + 1:bh + 1] - ex1[lo:bh])
        hy1[kh] += coef_h * float(ex_inc[n])
        hy_tab[n] = hy1[sh_]
        ex1[ae:hi] = ca[ae:hi] * ex1[ae:hi] - cb[ae:hi] * (hy1[ae:hi] - hy1[ae - 1:hi - 1])
        ex1[inj] += coef_e * float(hy_inc[n])
        ex_tab[n + 1] = ex1[se_]
    tol = TAIL_MAX_REL * float(np.abs(np.asarray(ex_inc)[:n_steps + 1]).max())
    m = UNTOUCHED_CELLS
    for a in (ex1, hy1):
        if max(float(np.abs(a[:m]).max()), float(np.abs(a[-m:]).max())) > tol:
            raise ValueError("the 1D runway is too short: its ends were reached")
    return ex_tab, hy_tab


def refuse_bad_placement(sc, t, n_total: int) -> None:
    """The faces and the cells beside them stay out of the CPML and the absorber slabs; the
    injection tables cover the run."""
    for a2, (lo_e, hi_e) in enumerate(zip(t.box_lo, t.box_hi)):
        n = sc.grid.axes[a2].n
        if not 1 <= lo_e < hi_e <= n - 1:
            raise ValueError(f"TFSF box {t.box_lo}..{t.box_hi} touches the grid boundary")
        c = sc.pml.get((a2, "lo"))
        if c is not None and lo_e - 2 < c.num_layers:
            raise ValueError(f"TFSF box reaches into the CPML at the low end of {'xyz'[a2]}")
        c = sc.pml.get((a2, "hi"))
        if c is not None and hi_e + 2 > n - c.num_layers:
            raise ValueError(f"TFSF box reaches into the CPML at the high end of {'xyz'[a2]}")
    for sl in sc.absorbers:
        lo_e, hi_e = t.box_lo[sl.axis], t.box_hi[sl.axis]
        nlay = int(np.size(sl.decay_int))
        if not (hi_e + 2 <= sl.g0 or lo_e - 2 >= sl.g0 + nlay):
            raise ValueError(f"TFSF box overlaps the absorber slab on {'xyz'[sl.axis]}")
    if n_total > np.size(t.ex_inc) - 1:
        raise ValueError(f"asked to run {n_total} steps, the TFSF injection table holds "
                         f"{np.size(t.ex_inc)} samples")


def face_corrections(t, grid, nk_e: int, ch: float):
    """The E-step and H-step correction faces. Each: field component (0..5), float32
    coefficient, table column ``c0 + cq q`` (float64), the face's fixed axis / index and its
    two scan axes (p, q) with start and count."""
    a = int(t.axis)
    u, v = cyclic_axes(a)
    bu, bv = float(t.pol_u), float(t.pol_v)
    lo, hi = [int(x) for x in t.box_lo], [int(x) for x in t.box_hi]
    alo, ahi, ulo, uhi, vlo, vhi = lo[a], hi[a], lo[u], hi[u], lo[v], hi[v]
    ax = grid.axes
    dl = [np.asarray(ax[q].dl, np.float64) for q in range(3)]
    dld = [np.asarray(ax[q].dl_dual, np.float64) for q in range(3)]
    start = {u: ulo, v: vlo, a: alo}
    nu_c, nu_e = uhi - ulo, uhi - ulo + 1
    nv_c, nv_e = vhi - vlo, vhi - vlo + 1
    na_c, na_e = ahi - alo, ahi - alo + 1

    def face(out, comp, fixed_ax, fixed_idx, p_ax, np_, q_ax, nq_, coef, c0, follow_a):
        if coef == 0.0:
            return
        out.append({"comp": int(comp), "coef": np.float32(coef), "c0": float(c0),
                    "cq": 1.0 if follow_a else 0.0, "fixed": (int(fixed_ax), int(fixed_idx)),
                    "p": (int(p_ax), int(start[p_ax]), int(np_)),
                    "q": (int(q_ax), int(start[q_ax]), int(nq_))})

    e, h = [], []
    face(e, u, a, alo, u, nu_c, v, nv_e, +bu / dld[a][alo], 0, False)
    face(e, u, a, ahi, u, nu_c, v, nv_e, -bu / dld[a][ahi], nk_e, False)
    face(e, v, a, alo, u, nu_e, v, nv_c, +bv / dld[a][alo], 0, False)
    face(e, v, a, ahi, u, nu_e, v, nv_c, -bv / dld[a][ahi], nk_e, False)
    face(e, a, u, ulo, v, nv_e, a, na_c, -bu / dld[u][ulo], 1, True)
    face(e, a, u, uhi, v, nv_e, a, na_c, +bu / dld[u][uhi], 1, True)
    face(e, a, v, vlo, u, nu_e, a, na_c, -bv / dld[v][vlo], 1, True)
    face(e, a, v, vhi, u, nu_e, a, na_c, +bv / dld[v][vhi], 1, True)
    face(h, 3 + v, a, alo - 1, u, nu_c, v, nv_e, +bu * ch / dl[a][alo - 1], 0, False)
    face(h, 3 + v, a, ahi, u, nu_c, v, nv_e, -bu * ch / dl[a][ahi], nk_e - 1, False)
    face(h, 3 + u, a, alo - 1, u, nu_e, v, nv_c, -bv * ch / dl[a][alo - 1], 0, False)
    face(h, 3 + u, a, ahi, u, nu_e, v, nv_c, +bv * ch / dl[a][ahi], nk_e - 1, False)
    face(h, 3 + a, v, vlo - 1, u, nu_c, a, na_e, -bu * ch / dl[v][vlo - 1], 0, True)
    face(h, 3 + a, v, vhi, u, nu_c, a, na_e, +bu * ch / dl[v][vhi], 0, True)
    face(h, 3 + a, u, ulo - 1, v, nv_c, a, na_e, +bv * ch / dl[u][ulo - 1], 0, True)
    face(h, 3 + a, u, uhi, v, nv_c, a, na_e, -bv * ch / dl[u][uhi], 0, True)
    return e, h


def box_tables(sc, n_total: int) -> dict | None:
    """Incident tables and correction faces of the scene's TFSF box (None without one)."""
    if not sc.tfsf_sources:
        return None
    if len(sc.tfsf_sources) != 1:
        raise NotImplementedError("only a single TFSF source is supported")
    t = sc.tfsf_sources[0]
    if getattr(t, "k_hat", None) is not None:
        raise NotImplementedError("oblique-incidence TFSF boxes are not supported yet")
    if getattr(t, "open_axes", ()):
        raise NotImplementedError("a TFSF box open on an axis is not supported at normal "
                                  "incidence")
    refuse_bad_placement(sc, t, n_total)
    a = int(t.axis)
    nk_e = int(t.box_hi[a]) - int(t.box_lo[a]) + 1
    scale = float(getattr(t, "amp_scale", 1.0))
    ex_tab, hy_tab = line_tables(t.dl1, t.eps1, sc.dt, int(t.inj), int(t.direction),
                                 np.asarray(t.ex_inc) * scale, np.asarray(t.hy_inc) * scale,
                                 n_total, int(t.col0), nk_e, sigma1=t.sigma1)
    e, h = face_corrections(t, sc.grid, nk_e, sc.dt / MU_0)
    return {"ex_tab": ex_tab, "hy_tab": hy_tab, "e_faces": e, "h_faces": h, "nk_e": nk_e}


FACE_DTYPE = np.dtype([("comp", np.int32), ("group", np.int32), ("coef", np.float32),
                       ("reserved", np.float32), ("c0", np.float64), ("cp", np.float64),
                       ("cq", np.float64), ("base", np.int64), ("sp", np.int64),
                       ("sq", np.int64), ("np", np.int32), ("nq", np.int32)], align=True)


def device_faces(faces, ny: int, nzp: int) -> np.ndarray:
    """The faces as the C ABI's ``oem_tfsf_face`` records, in order, grouped so that the faces
    of one group touch disjoint cells: a face starts a new group when the current group already
    holds a face of the same component on another fixed axis (the E_a / H_a faces of the u and v
    sides meet on the box edges)."""
    strides = (ny * nzp, nzp, 1)
    out = np.zeros(len(faces), dtype=FACE_DTYPE)
    group, seen = 0, {}
    for i, f in enumerate(faces):
        fa, fi = f["fixed"]
        if f["comp"] in seen and seen[f["comp"]] != fa:
            group += 1
            seen = {}
        seen.setdefault(f["comp"], fa)
        pt = [0, 0, 0]
        pt[fa] = fi
        pa, ps, pn = f["p"]
        qa, qs, qn = f["q"]
        pt[pa] = ps
        pt[qa] = qs
        out[i] = (f["comp"], group, f["coef"], 0.0, f["c0"], 0.0, f["cq"],
                  pt[0] * strides[0] + pt[1] * strides[1] + pt[2] * strides[2],
                  strides[pa], strides[qa], pn, qn)
    return out
