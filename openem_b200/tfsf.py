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
    open_axes = tuple(getattr(t, "open_axes", ()))
    for a2, (lo_e, hi_e) in enumerate(zip(t.box_lo, t.box_hi)):
        n = sc.grid.axes[a2].n
        if a2 in open_axes:
            continue  # the box spans the axis: no face there
        if not 1 <= lo_e < hi_e <= n - 1:
            raise ValueError(f"TFSF box {t.box_lo}..{t.box_hi} touches the grid boundary")
        c = sc.pml.get((a2, "lo"))
        if c is not None and lo_e - 2 < c.num_layers:
            raise ValueError(f"TFSF box reaches into the CPML at the low end of {'xyz'[a2]}")
        c = sc.pml.get((a2, "hi"))
        if c is not None and hi_e + 2 > n - c.num_layers:
            raise ValueError(f"TFSF box reaches into the CPML at the high end of {'xyz'[a2]}")
    for sl in sc.absorbers:
        if sl.axis in open_axes:
            continue
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


# ---------------------------------------------------------------------------------------------
# Oblique incidence (openem/tfsf_oblique.py, openem/tfsf1d.py:60-142)
# ---------------------------------------------------------------------------------------------
# The two terms of (curl F)_m in the cyclic basis (u, v, a) = (0, 1, 2): (r, n, s) = s dF_r/dn.
CURL_TERMS = {0: ((2, 1, +1), (1, 2, -1)),
              1: ((0, 2, +1), (2, 0, -1)),
              2: ((1, 0, +1), (0, 1, -1))}


def matched_dl(k_hat, dl_axes, dt: float, freq: float, eps_r: float = 1.0) -> float:
    """Cell size of a 1D Yee line along k_hat whose discrete phase velocity at ``freq`` equals
    the 3D grid's: solve [sin(w dt/2)/(c dt)]^2 = sum_i [sin(k k_i dl_i/2)/dl_i]^2 for k, then
    [sin(k dl1/2)/dl1]^2 = the same left side for dl1 (both by bisection on their monotone
    branch). Along an axis, a face or a body diagonal this is dl, dl/sqrt(2), dl/sqrt(3)."""
    k_hat = np.asarray(k_hat, dtype=np.float64)
    dl_axes = np.asarray(dl_axes, dtype=np.float64)
    c = C_0 / np.sqrt(float(eps_r))
    w = 2.0 * np.pi * float(freq)
    lhs = (np.sin(w * dt / 2.0) / (c * dt)) ** 2

    def rhs(k):
        return float(np.sum((np.sin(k * k_hat * dl_axes / 2.0) / dl_axes) ** 2))
    nz = np.abs(k_hat) > 1e-15
    k_hi = float(np.min(np.pi / (np.abs(k_hat[nz]) * dl_axes[nz])))
    if rhs(k_hi) < lhs:
        raise ValueError("the 3D discrete dispersion never reaches the source frequency on this "
                         "grid (dt or the frequency too large)")
    lo, hi = 0.0, k_hi
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if rhs(mid) < lhs else (lo, mid)
    k = 0.5 * (lo + hi)
    target = np.sqrt(lhs)
    if k / 2.0 < target:
        raise ValueError("no matching 1D cell size exists")
    lo, hi = 1e-12, float(np.pi / k)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if np.sin(k * mid / 2.0) / mid > target else (lo, mid)
    dl1 = 0.5 * (lo + hi)
    if c * dt > dl1:
        raise ValueError("the matched 1D cell size violates the 1D Courant limit")
    return float(dl1)


def projection_range(grid, k_hat, box_lo, box_hi):
    """[P_min, P_max] of the box grown by one cell, projected on k_hat (metres)."""
    pmin = pmax = 0.0
    for w in range(3):
        e = np.asarray(grid.axes[w].edges, dtype=np.float64)
        a = float(k_hat[w]) * float(e[max(box_lo[w] - 1, 0)])
        b = float(k_hat[w]) * float(e[min(box_hi[w] + 1, e.size - 1)])
        pmin += min(a, b)
        pmax += max(a, b)
    return pmin, pmax


def on_edge(comp: int, magnetic: bool):
    """Whether component ``comp`` sits on the primal edges (True) or cell centres along each
    axis: E_c at the centre along c, H_c on the edge along c only."""
    return tuple((w == comp) if magnetic else (w != comp) for w in range(3))


def yee_point(grid, comp: int, magnetic: bool, idx):
    edge = on_edge(comp, magnetic)
    out = np.empty(3)
    for w in range(3):
        ax = grid.axes[w]
        out[w] = (np.asarray(ax.edges, np.float64)[idx[w]] if edge[w]
                  else np.asarray(ax.centers, np.float64)[idx[w]])
    return out


def oblique_terms(t, grid, ch: float):
    """The correction terms of an oblique box: per corrected component m and curl term
    s dF_r/dn, the E-step faces (E_m on the total-field side at n = lo / hi, incident H_r from
    the cell outside) and the H-step faces (H_m on the scattered-field side at cells lo-1 / hi,
    incident E_r from the edge inside), coefficients -+s h_r / dl*_n and +-ch s e_r / dl_n; the
    terms whose coefficient vanishes are dropped (8 of the 24 at normal incidence)."""
    a = int(t.axis)
    u, v = cyclic_axes(a)
    uva = (u, v, a)
    k = np.asarray(t.k_hat, np.float64)
    e = np.asarray(t.e_hat, np.float64)
    h = np.cross(k, e)
    e_uva = [float(e[x]) for x in uva]
    h_uva = [float(h[x]) for x in uva]
    lo = [int(x) for x in t.box_lo]
    hi = [int(x) for x in t.box_hi]
    open_axes = tuple(getattr(t, "open_axes", ()))
    for m in range(3):
        for (r, n, sg) in CURL_TERMS[m]:
            nax = uva[n]
            if nax in open_axes:
                continue
            dld = np.asarray(grid.axes[nax].dl_dual, np.float64)
            dl = np.asarray(grid.axes[nax].dl, np.float64)
            for fx, cf, inc_n in ((lo[nax], -sg * h_uva[r] / dld[lo[nax]], lo[nax] - 1),
                                  (hi[nax], +sg * h_uva[r] / dld[hi[nax]], hi[nax])):
                if cf != 0.0:
                    yield {"kind": "E", "comp": uva[m], "inc": uva[r], "fixed": (nax, fx),
                           "inc_n": inc_n, "coef": cf}
            for fx, cf, inc_n in ((lo[nax] - 1, +ch * sg * e_uva[r] / dl[lo[nax] - 1], lo[nax]),
                                  (hi[nax], -ch * sg * e_uva[r] / dl[hi[nax]], hi[nax])):
                if cf != 0.0:
                    yield {"kind": "H", "comp": uva[m], "inc": uva[r], "fixed": (nax, fx),
                           "inc_n": inc_n, "coef": cf}


def oblique_faces(t, grid, ch: float):
    """E-step and H-step faces of an oblique box with real-valued table columns: a face point
    (p, q) reads the incident table at c0 + cp p + cq q, the projection of the incident
    component's Yee point on k_hat in 1D cells from ``proj0`` (H columns are shifted by half a
    cell: the H line values sit at cell centres)."""
    k = np.asarray(t.k_hat, np.float64)
    dl1 = float(t.dl1_step)
    lo = [int(x) for x in t.box_lo]
    hi = [int(x) for x in t.box_hi]
    e_faces, h_faces = [], []
    for term in oblique_terms(t, grid, ch):
        fa, fi = term["fixed"]
        pa, qa = [w for w in range(3) if w != fa]
        mag = term["kind"] == "H"
        edge = on_edge(term["comp"], mag)
        n_p = hi[pa] - lo[pa] + (1 if edge[pa] else 0)
        n_q = hi[qa] - lo[qa] + (1 if edge[qa] else 0)
        inc_idx = [0, 0, 0]
        inc_idx[fa] = term["inc_n"]
        inc_idx[pa], inc_idx[qa] = lo[pa], lo[qa]
        p0 = float(k @ yee_point(grid, term["inc"], not mag, inc_idx))
        c0 = (p0 - float(t.proj0)) / dl1 + (0.5 if term["kind"] == "E" else 0.0)
        cp = float(k[pa]) * float(grid.axes[pa].dl[lo[pa]]) / dl1
        cq = float(k[qa]) * float(grid.axes[qa].dl[lo[qa]]) / dl1
        face = {"comp": int(term["comp"]) + (3 if mag else 0), "coef": np.float32(term["coef"]),
                "c0": c0, "cp": cp, "cq": cq, "fixed": (fa, fi), "p": (pa, lo[pa], n_p),
                "q": (qa, lo[qa], n_q)}
        (h_faces if mag else e_faces).append(face)
    return e_faces, h_faces


def check_in_table(faces, row_n: int, what: str) -> None:
    """Every face point's table column lies inside the table (checked at the four corners:
    the column is linear in p and q)."""
    for f in faces:
        for p in (0, f["p"][2] - 1):
            for q in (0, f["q"][2] - 1):
                pos = f["c0"] + f.get("cp", 0.0) * p + f["cq"] * q
                if not 0.0 <= pos <= row_n - 1:
                    raise ValueError(f"{what} face column {pos:.3f} outside [0, {row_n - 1}]: "
                                     "the 1D table does not cover the box's projection")


def refuse_oblique(sc, t) -> None:
    """Oblique boxes need two cells of margin on every closed axis, a uniform grid across the
    box and a uniform, lossless, non-dispersive background on its shell."""
    open_axes = tuple(getattr(t, "open_axes", ()))
    for q in range(3):
        n = sc.grid.axes[q].n
        lo, hi = int(t.box_lo[q]), int(t.box_hi[q])
        if q not in open_axes and not 2 <= lo < hi <= n - 3:
            raise ValueError("the oblique TFSF box needs two cells of margin to the grid edge")
        dl = np.asarray(sc.grid.axes[q].dl, np.float64)[max(lo - 1, 0):min(hi + 1, n)]
        if np.ptp(dl) > 1e-12 * float(np.mean(dl)):
            raise NotImplementedError("oblique TFSF needs a uniform grid across the box")
    shell = np.zeros(sc.shape, dtype=bool)
    sl_out = tuple(slice(max(int(t.box_lo[q]) - 2, 0), int(t.box_hi[q]) + 2) for q in range(3))
    sl_in = tuple(slice(int(t.box_lo[q]) + 1, int(t.box_hi[q]) - 1)
                  if q not in open_axes else slice(None) for q in range(3))
    shell[sl_out] = True
    shell[sl_in] = False
    for eps in (sc.eps_ex, sc.eps_ey, sc.eps_ez):
        v = np.asarray(eps, np.float64)[shell]
        if v.size and np.ptp(v) > 1e-9 * max(1.0, float(np.abs(v).max())):
            raise NotImplementedError("oblique TFSF needs a uniform background on the box shell")
    for sig in (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez):
        if sig is not None and np.abs(np.asarray(sig)[shell]).max() > 0:
            raise NotImplementedError("oblique TFSF needs a lossless background on the box shell")
    if sc.dispersion is not None and sc.dispersion.n_entry:
        cells = np.zeros(int(np.prod(sc.shape)), dtype=bool)
        cells[np.asarray(sc.dispersion.cell)] = True
        if (cells.reshape(sc.shape) & shell).any():
            raise NotImplementedError("oblique TFSF needs a non-dispersive box shell")


def box_tables(sc, n_total: int) -> dict | None:
    """Incident tables and correction faces of the scene's TFSF box (None without one)."""
    if not sc.tfsf_sources:
        return None
    if len(sc.tfsf_sources) != 1:
        raise NotImplementedError("only a single TFSF source is supported")
    t = sc.tfsf_sources[0]
    oblique = getattr(t, "k_hat", None) is not None
    if getattr(t, "open_axes", ()) and not oblique:
        raise NotImplementedError("a TFSF box open on an axis is supported at oblique "
                                  "incidence only")
    refuse_bad_placement(sc, t, n_total)
    if oblique:
        refuse_oblique(sc, t)
        nk_e = int(t.n_col_e)
        scale = float(getattr(t, "amp_scale", 1.0))
        ex_tab, hy_tab = line_tables(t.dl1, t.eps1, sc.dt, int(t.inj), int(t.direction),
                                     np.asarray(t.ex_inc) * scale,
                                     np.asarray(t.hy_inc) * scale, n_total, int(t.col0), nk_e,
                                     sigma1=t.sigma1)
        e, h = oblique_faces(t, sc.grid, sc.dt / MU_0)
        check_in_table(e, nk_e + 1, "E step")
        check_in_table(h, nk_e, "H step")
        return {"ex_tab": ex_tab, "hy_tab": hy_tab, "e_faces": e, "h_faces": h, "nk_e": nk_e}
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
        out[i] = (f["comp"], group, f["coef"], 0.0, f["c0"], f.get("cp", 0.0), f["cq"],
                  pt[0] * strides[0] + pt[1] * strides[1] + pt[2] * strides[2],
                  strides[pa], strides[qa], pn, qn)
    return out
