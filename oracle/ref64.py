"""FP64 NumPy transcription of OpenEM's solver step loop -- TEST INFRASTRUCTURE ONLY.

This module is the oracle the CUDA engine is checked against, and the CPU baseline that
``bench.py`` times. Nothing in the product path imports it. It restates, in float64 and in the
launch order of ``openem/solver.py:1145-1162``, the update equations of the reference kernels:

* ``update_h`` with the CPML psi recursion ``stretch`` -- ``openem/kernels/yee.cu:60-137``;
* ``update_e`` (semi-implicit sigma, dispersion history, PEC masks) -- ``yee.cu:139-240``;
* ``dispersion_pre`` / ``dispersion_post`` -- ``openem/kernels/dispersion.cu:60-158``;
* plane-wave TF/SF injection ``inject_h`` / ``inject_e`` -- ``openem/kernels/source_dft.cu:39-73``
  with the coefficients of ``openem/sources_setup.py:93-119``;
* point dipoles ``inject_dipole(_h)`` -- ``source_dft.cu:135-206``, tables
  ``openem/sources_setup.py:419-457``;
* DFT accumulation of flux planes and field boxes -- ``source_dft.cu:208-430`` (E at
  ``(n+1) dt``, H at ``(n+1/2) dt``, H colocated ``(H[k] + H[k-1]) / 2`` on a flux plane,
  apodisation window ``openem/apodization.py:27-45``);
* field time monitors with the two-shot H average -- ``source_dft.cu:273-319``,
  ``openem/readout.py:184-197``;
* the complex Bloch path -- ``openem/kernels/bloch.cu:25-221`` and ``openem/solver.py:1263-1483``.

Coefficient tables follow ``openem/coeffs.py:21-136`` (CPML axis arrays filled with the identity
outside the layers; ``ca = (eps - s)/(eps + s + G)``, ``cb = (dt/eps0)/(eps + s + G)``) and the
index tables of ``openem/grid.py:219-304``.

The only inputs are the attributes of a ``Scene`` (OpenEM's own class or the engine's mirror).
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

EPSILON_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6
APOD_K = 0.5
# +z and -z one-face TF/SF correction signs (openem/tfsf1d.py:46)
_SIGNS = {+1: (1.0, 1.0), -1: (-1.0, -1.0)}
# one-plane TF/SF signs of a mode source per direction: (H_t1, H_t2, E_t1, E_t2)
# (openem/sources_setup.py:51-54)
_MODE_SIGNS = {+1: (-1.0, +1.0, +1.0, -1.0), -1: (+1.0, -1.0, +1.0, -1.0)}


def apod_window(t, spec):
    t = np.asarray(t, dtype=np.float64)
    w = np.ones_like(t)
    if spec is None:
        return w
    start, end, width = spec
    if start is not None:
        m = t < start
        w[m] = np.exp(-APOD_K * ((t[m] - start) / width) ** 2)
    if end is not None:
        m = t > end
        w[m] = np.exp(-APOD_K * ((t[m] - end) / width) ** 2)
    return w


def pml_axis_arrays(sc, axis: int, at: str):
    """``(a, b, 1/kappa)`` along one axis, identity ``(0, 1, 1)`` outside the layers."""
    n = sc.grid.axes[axis].n
    a, b, k = np.zeros(n), np.ones(n), np.ones(n)
    for side in ("lo", "hi"):
        c = sc.pml.get((axis, side))
        if c is None:
            continue
        m = int(np.asarray(c.a_E).size)
        sl = slice(0, m) if side == "lo" else slice(n - m, n)
        a[sl] = np.asarray(getattr(c, f"a_{at}"))
        b[sl] = np.asarray(getattr(c, f"b_{at}"))
        k[sl] = np.asarray(getattr(c, f"inv_kappa_{at}"))
    return a, b, k


def e_coeffs(sc):
    """``(ca, cb)`` per component in float64, PEC cells zeroed."""
    shape = sc.shape
    if sc.dispersion is not None and sc.dispersion.n_entry > 0:
        gg = _g_dense(sc.dispersion, shape)
    else:
        gg = (np.zeros(shape),) * 3
    ca, cb = [], []
    sig = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
    for c, eps in enumerate((sc.eps_ex, sc.eps_ey, sc.eps_ez)):
        eps = np.asarray(eps, dtype=np.float64)
        s = (np.zeros_like(eps) if sig[c] is None
             else np.asarray(sig[c], dtype=np.float64) * sc.dt / (2.0 * EPSILON_0))
        den = eps + s + gg[c]
        ca.append((eps - s) / den)
        cb.append((sc.dt / EPSILON_0) / den)
    pecs = (sc.pec_ex, sc.pec_ey, sc.pec_ez)
    for c in range(3):
        if pecs[c] is not None and np.asarray(pecs[c]).size:
            idx = np.asarray(pecs[c], dtype=np.int64)
            ca[c].ravel()[idx] = 0.0
            cb[c].ravel()[idx] = 0.0
    return ca, cb


def _g_dense(d, shape):
    out = [np.zeros(int(np.prod(shape))) for _ in range(3)]
    comp, cell, g = np.asarray(d.comp), np.asarray(d.cell), np.asarray(d.g)
    for c in range(3):
        m = comp == c
        out[c][cell[m]] = g[m]
    return tuple(o.reshape(shape) for o in out)


@dataclass
class OracleResult:
    phasors: dict = field(default_factory=dict)          # name -> (4, nf, n1, n2) complex
    field_phasors: dict = field(default_factory=dict)    # name -> (6, nf, ni, nj, nk) complex
    time_samples: dict = field(default_factory=dict)
    time_slots: dict = field(default_factory=dict)
    flux_time: dict = field(default_factory=dict)        # name -> (filled,) float64
    fields: dict = field(default_factory=dict)
    steps_run: int = 0
    seconds: float = 0.0


class Oracle:
    """Float64 state of one real-path run. ``step()`` advances one full time step."""

    def __init__(self, sc, n_total: int | None = None):
        if sc.any_bloch:
            raise ValueError("use BlochOracle for a scene with a non-zero Bloch vector")
        self.sc = sc
        self.n_total = int(n_total if n_total is not None else sc.num_time_steps)
        nx, ny, nz = self.shape = sc.shape
        self.E = [np.zeros(self.shape) for _ in range(3)]
        self.H = [np.zeros(self.shape) for _ in range(3)]
        # psi slots in the reference order: hx_y hx_z hy_z hy_x hz_x hz_y (same on E)
        self.psi_h = [np.zeros(self.shape) for _ in range(6)]
        self.psi_e = [np.zeros(self.shape) for _ in range(6)]
        tabs = [a.index_tables() for a in sc.grid.axes]
        self.nxt = [t["nxt"] for t in tabs]
        self.prv = [t["prv"] for t in tabs]
        self.mnx = [np.asarray(t["mnx"], dtype=np.float64) for t in tabs]
        self.mpv = [np.asarray(t["mpv"], dtype=np.float64) for t in tabs]
        self.pec = [t["pec"] for t in tabs]
        self.idl_p = [1.0 / a.dl for a in sc.grid.axes]
        self.idl_d = [1.0 / a.dl_dual for a in sc.grid.axes]
        self.pml_e = [pml_axis_arrays(sc, a, "E") for a in range(3)]
        self.pml_h = [pml_axis_arrays(sc, a, "H") for a in range(3)]
        self.ch = sc.dt / MU_0
        self.cw = EPSILON_0 / sc.dt
        self.ca, self.cb = e_coeffs(sc)
        self.hist = [np.zeros(self.shape) for _ in range(3)]
        self._setup_dispersion()
        self._setup_mix()
        self._setup_modulation()
        self._setup_tensor()
        self._setup_sources()
        self._setup_tfsf()
        self._setup_monitors()
        self.n = 0

    # ---- setup --------------------------------------------------------------------------
    def _setup_modulation(self):
        """Time-modulated permittivity (openem/sources_setup.py:460-518): per entry eps_s, amp,
        phase, s = sigma dt / (2 eps0) and the dispersion coupling G, all float64."""
        sc = self.sc
        self.mod = None
        mo = sc.modulation
        if mo is None or mo.n_entry == 0:
            return
        comp = np.asarray(mo.comp, np.int64)
        cell = np.asarray(mo.cell, np.int64)
        es, sd, gg = np.empty(comp.size), np.zeros(comp.size), np.zeros(comp.size)
        g = _g_dense(sc.dispersion, self.shape) if sc.any_dispersion else None
        sig = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
        for c, eps in enumerate((sc.eps_ex, sc.eps_ey, sc.eps_ez)):
            m = comp == c
            es[m] = np.asarray(eps, np.float64).ravel()[cell[m]]
            if sig[c] is not None:
                sd[m] = np.asarray(sig[c], np.float64).ravel()[cell[m]] * sc.dt / (2 * EPSILON_0)
            if g is not None:
                gg[m] = g[c].ravel()[cell[m]]
        self.mod = {"comp": comp, "cell": cell, "es": es, "sd": sd, "gg": gg,
                    "amp": np.asarray(mo.amp, np.float64),
                    "phase": np.asarray(mo.phase, np.float64), "om": 2 * np.pi * float(mo.freq)}

    def _setup_tensor(self):
        """Fully anisotropic cells (openem/kernels/tensor.cu): rows of M1 = A^-1 B and
        M2 = (dt/eps0) A^-1 per entry; the entries' update coefficients pass the curl through
        (ca = 0, cb = 1)."""
        sc = self.sc
        self.ten = None
        t = sc.tensor
        if t is None or t.n_entry == 0:
            return
        s = np.asarray(t.sigma, np.float64) * sc.dt / (2 * EPSILON_0)
        eps = np.asarray(t.eps, np.float64)
        ainv = np.linalg.inv(eps + s)
        comp = np.asarray(t.comp, np.int64)
        r = np.arange(comp.size)
        m1 = (ainv @ (eps - s))[r, comp, :]
        m2 = ((sc.dt / EPSILON_0) * ainv)[r, comp, :]
        cell = np.asarray(t.cell, np.int64)
        nx, ny, nz = self.shape
        ijk = np.stack([cell // (ny * nz), (cell // nz) % ny, cell % nz])
        for c in range(3):
            m = comp == c
            self.ca[c].ravel()[cell[m]] = 0.0
            self.cb[c].ravel()[cell[m]] = 1.0
        pec = [np.asarray(p, np.float64) for p in self.pec]
        pf = np.array([pec[(a + 1) % 3][ijk[(a + 1) % 3, e]] * pec[(a + 2) % 3][ijk[(a + 2) % 3, e]]
                       for e, a in enumerate(comp)])
        self.ten = {"comp": comp, "ijk": ijk, "m1": m1, "m2": m2, "pec": pf, "rhs": None}

    def _tensor_dot(self, m, F):
        """m_row . <F> per entry, the off-position components averaged over the 4 neighbours
        {cell, +1 along comp} x {cell, -1 along b} with the boundary masks."""
        tn = self.ten
        comp, ijk = tn["comp"], tn["ijk"]
        out = np.empty(comp.size)
        for e, a in enumerate(comp):
            c0 = ijk[:, e]
            acc = m[e, a] * F[a][tuple(c0)]
            for b in range(3):
                if b == a:
                    continue
                ca = c0.copy()
                ca[a] = self.nxt[a][c0[a]]
                cb = c0.copy()
                cb[b] = self.prv[b][c0[b]]
                cab = ca.copy()
                cab[b] = cb[b]
                wa, wb = self.mnx[a][c0[a]], self.mpv[b][c0[b]]
                avg = 0.25 * (F[b][tuple(c0)] + wa * F[b][tuple(ca)] + wb * F[b][tuple(cb)]
                              + wa * wb * F[b][tuple(cab)])
                acc += m[e, b] * avg
            out[e] = acc
        return out

    def tensor_pre(self):
        if getattr(self, "ten", None) is not None:
            self.ten["rhs"] = self._tensor_dot(self.ten["m1"], self.E)

    def tensor_post(self):
        tn = getattr(self, "ten", None)
        if tn is None:
            return
        enew = tn["rhs"] + self._tensor_dot(tn["m2"], self.E)
        for e, a in enumerate(tn["comp"]):
            self.E[a][tuple(tn["ijk"][:, e])] = enew[e] * tn["pec"][e]

    def modulate(self, n):
        """D-form coefficients of step n on the modulated entries
        (openem/kernels/modulation.cu:40-79): ca = (eps(t_n) - s) / (eps(t_n+1) + s + G),
        cb = (dt / eps0) / (eps(t_n+1) + s + G), eps(t) = eps_s + amp cos(omega t - phi)."""
        md = getattr(self, "mod", None)  # the complex path has no modulation
        if md is None:
            return
        dt = self.sc.dt
        e0 = md["es"] + md["amp"] * np.cos(md["om"] * (n * dt) - md["phase"])
        e1 = md["es"] + md["amp"] * np.cos(md["om"] * ((n + 1) * dt) - md["phase"])
        den = e1 + md["sd"] + md["gg"]
        for c in range(3):
            m = md["comp"] == c
            self.ca[c].ravel()[md["cell"][m]] = ((e0 - md["sd"]) / den)[m]
            self.cb[c].ravel()[md["cell"][m]] = ((dt / EPSILON_0) / den)[m]

    def _setup_tfsf(self):
        """TFSF box at normal incidence: the 1D auxiliary line (openem/tfsf1d.py:297-325, run
        over the whole line here) and the box geometry (openem/sources_setup.py:120-233)."""
        sc = self.sc
        self.tfsf = None
        if not getattr(sc, "tfsf_sources", None):
            return
        t = sc.tfsf_sources[0]
        oblique = getattr(t, "k_hat", None) is not None
        a = int(t.axis)
        lo, hi = [int(x) for x in t.box_lo], [int(x) for x in t.box_hi]
        nk = int(t.n_col_e) if oblique else hi[a] - lo[a] + 1
        dl1 = np.asarray(t.dl1, np.float64)
        eps1 = np.asarray(t.eps1, np.float64)
        n1 = dl1.size
        dld1 = np.concatenate([[dl1[0]], 0.5 * (dl1[1:] + dl1[:-1])])
        dt = sc.dt
        s1 = (np.zeros(n1) if t.sigma1 is None
              else np.asarray(t.sigma1, np.float64) * dt / (2 * EPSILON_0))
        ca1 = (eps1 - s1) / (eps1 + s1)
        cb1 = dt / EPSILON_0 / (eps1 + s1) / dld1
        ch1 = dt / MU_0 / dl1
        d = int(t.direction)
        inj = int(t.inj)
        kh = inj - 1 if d > 0 else inj
        sgn = _SIGNS[d]
        scale = float(getattr(t, "amp_scale", 1.0))
        ch_inj = sgn[0] * dt / MU_0 / dl1[kh]
        ce_inj = sgn[1] * dt / EPSILON_0 / (eps1[inj] + s1[inj]) / dld1[inj]
        col0 = int(t.col0)
        e1, h1 = np.zeros(n1), np.zeros(n1)
        ex_tab = np.zeros((self.n_total + 1, nk))
        hy_tab = np.zeros((self.n_total, nk + 1))
        for n in range(self.n_total):
            h1[:-1] -= ch1[:-1] * (e1[1:] - e1[:-1])
            h1[kh] += ch_inj * scale * float(t.ex_inc[n])
            hy_tab[n] = h1[col0 - 1:col0 + nk]
            e1[1:] = ca1[1:] * e1[1:] - cb1[1:] * (h1[1:] - h1[:-1])
            e1[inj] += ce_inj * scale * float(t.hy_inc[n])
            ex_tab[n + 1] = e1[col0:col0 + nk]
        self.tfsf = {"t": t, "a": a, "lo": lo, "hi": hi, "nk": nk, "ex": ex_tab, "hy": hy_tab,
                     "oblique": oblique}

    def inject_tfsf(self, side, n):
        """The box-face corrections of step n (the 16 terms of
        openem/sources_setup.py:236-272): H side with row E^n, E side (times cb) with row
        H^{n+1/2}."""
        tf = getattr(self, "tfsf", None)  # the complex path has no TFSF box
        if tf is None:
            return
        if tf["oblique"]:
            self._inject_tfsf_oblique(side, n)
            return
        t, a, lo, hi, nk = tf["t"], tf["a"], tf["lo"], tf["hi"], tf["nk"]
        u, v = (a + 1) % 3, (a + 2) % 3
        bu, bv = float(t.pol_u), float(t.pol_v)
        dl = [np.asarray(ax.dl, np.float64) for ax in self.sc.grid.axes]
        dld = [np.asarray(ax.dl_dual, np.float64) for ax in self.sc.grid.axes]

        def region(fixed_ax, fixed_idx, p_ax, p_end, q_ax, q_end):
            sl = [None, None, None]
            sl[fixed_ax] = fixed_idx
            sl[p_ax] = slice(lo[p_ax], p_end)
            sl[q_ax] = slice(lo[q_ax], q_end)
            return tuple(sl)

        def col_along_a(vals, q_ax, p_ax):
            # table values along a broadcast over the face (p_ax, q_ax order of the slice)
            shape = [1, 1]
            order = sorted([p_ax, q_ax])
            shape[order.index(a)] = -1
            return vals.reshape(shape)

        if side == "h":
            row = tf["ex"][n]
            ch = self.ch
            H = self.H
            if bu:
                H[v][region(a, lo[a] - 1, u, hi[u], v, hi[v] + 1)] += bu * ch / dl[a][lo[a] - 1] * row[0]
                H[v][region(a, hi[a], u, hi[u], v, hi[v] + 1)] -= bu * ch / dl[a][hi[a]] * row[nk - 1]
            if bv:
                H[u][region(a, lo[a] - 1, u, hi[u] + 1, v, hi[v])] -= bv * ch / dl[a][lo[a] - 1] * row[0]
                H[u][region(a, hi[a], u, hi[u] + 1, v, hi[v])] += bv * ch / dl[a][hi[a]] * row[nk - 1]
            ra = row[:nk]
            if bu:
                for idx, sg in ((lo[v] - 1, -1.0), (hi[v], 1.0)):
                    r = region(v, idx, u, hi[u], a, hi[a] + 1)
                    H[a][r] += sg * bu * ch / dl[v][idx] * col_along_a(ra, a, u)
            if bv:
                for idx, sg in ((lo[u] - 1, 1.0), (hi[u], -1.0)):
                    r = region(u, idx, v, hi[v], a, hi[a] + 1)
                    H[a][r] += sg * bv * ch / dl[u][idx] * col_along_a(ra, a, v)
        else:
            row = tf["hy"][n]
            E, cb = self.E, self.cb
            if bu:
                for idx, sg, col in ((lo[a], 1.0, 0), (hi[a], -1.0, nk)):
                    r = region(a, idx, u, hi[u], v, hi[v] + 1)
                    E[u][r] += cb[u][r] * sg * bu / dld[a][idx] * row[col]
            if bv:
                for idx, sg, col in ((lo[a], 1.0, 0), (hi[a], -1.0, nk)):
                    r = region(a, idx, u, hi[u] + 1, v, hi[v])
                    E[v][r] += cb[v][r] * sg * bv / dld[a][idx] * row[col]
            ra = row[1:nk]
            if bu:
                for idx, sg in ((lo[u], -1.0), (hi[u], 1.0)):
                    r = region(u, idx, v, hi[v] + 1, a, hi[a])
                    E[a][r] += cb[a][r] * sg * bu / dld[u][idx] * col_along_a(ra, a, v)
            if bv:
                for idx, sg in ((lo[v], -1.0), (hi[v], 1.0)):
                    r = region(v, idx, u, hi[u] + 1, a, hi[a])
                    E[a][r] += cb[a][r] * sg * bv / dld[v][idx] * col_along_a(ra, a, u)

    def _inject_tfsf_oblique(self, side, n):
        """Oblique box (openem/tfsf_oblique.py): for each term s dF_r/dn of (curl F)_m in the
        cyclic basis (u, v, a), the incident component r is evaluated at its own Yee points
        beside the face by projecting them on k_hat and interpolating the 1D line (H values at
        half cells); E_m gets -+ s h_r / dl*_n (times cb) on the total-field side of the n faces,
        H_m gets +- ch s e_r / dl_n on the scattered-field side."""
        tf = self.tfsf
        t, lo, hi = tf["t"], tf["lo"], tf["hi"]
        a = tf["a"]
        uva = ((a + 1) % 3, (a + 2) % 3, a)
        curl = {0: ((2, 1, 1.0), (1, 2, -1.0)), 1: ((0, 2, 1.0), (2, 0, -1.0)),
                2: ((1, 0, 1.0), (0, 1, -1.0))}
        k = np.asarray(t.k_hat, np.float64)
        e_vec = np.asarray(t.e_hat, np.float64)
        h_vec = np.cross(k, e_vec)
        dl1, proj0 = float(t.dl1_step), float(t.proj0)
        open_axes = tuple(getattr(t, "open_axes", ()))
        axes = self.sc.grid.axes

        def coords(comp, magnetic, w):
            edge = (w == comp) if magnetic else (w != comp)
            ax = axes[w]
            return np.asarray(ax.edges[:-1] if edge else ax.centers, np.float64)

        def span(comp, magnetic, w):
            edge = (w == comp) if magnetic else (w != comp)
            return slice(lo[w], hi[w] + (1 if edge else 0))

        def interp(row, pos):
            i0 = np.floor(pos).astype(np.int64)
            w = pos - i0
            bad_lo, bad_hi = i0 < 0, i0 >= row.size - 1
            i0 = np.clip(i0, 0, row.size - 1)
            w = np.where(bad_lo | bad_hi, 0.0, w)
            i1 = np.minimum(i0 + 1, row.size - 1)
            return row[i0] + w * (row[i1] - row[i0])

        e_side = side == "e"
        row = tf["hy"][n] if e_side else tf["ex"][n]
        for m in range(3):
            for (r, nn, sg) in curl[m]:
                nax = uva[nn]
                if nax in open_axes:
                    continue
                comp, inc = uva[m], uva[r]
                dld = np.asarray(axes[nax].dl_dual, np.float64)
                dl = np.asarray(axes[nax].dl, np.float64)
                if e_side:
                    sides = ((lo[nax], -sg * h_vec[inc] / dld[lo[nax]], lo[nax] - 1),
                             (hi[nax], sg * h_vec[inc] / dld[hi[nax]], hi[nax]))
                else:
                    sides = ((lo[nax] - 1, self.ch * sg * e_vec[inc] / dl[lo[nax] - 1], lo[nax]),
                             (hi[nax], -self.ch * sg * e_vec[inc] / dl[hi[nax]], hi[nax]))
                for fx, cf, inc_n in sides:
                    if cf == 0.0:
                        continue
                    sl = [None, None, None]
                    grids = [None, None, None]
                    for w in range(3):
                        if w == nax:
                            sl[w] = slice(fx, fx + 1)
                            grids[w] = np.array([coords(inc, e_side, w)[inc_n]])
                        else:
                            sp = span(comp, not e_side, w)
                            sl[w] = sp
                            grids[w] = coords(inc, e_side, w)[sp]
                    X, Y, Z = np.meshgrid(*grids, indexing="ij")
                    pos = (k[0] * X + k[1] * Y + k[2] * Z - proj0) / dl1 + (0.5 if e_side else 0.0)
                    val = interp(row, pos)
                    sl = tuple(sl)
                    if e_side:
                        self.E[comp][sl] += self.cb[comp][sl] * cf * val
                    else:
                        self.H[comp][sl] += cf * val

    def _setup_dispersion(self):
        d = self.sc.dispersion
        self.disp = None
        if d is None or d.n_entry == 0:
            return
        d.validate(self.shape)
        ofs = np.asarray(d.pole_ofs, dtype=np.int64)
        npole = np.diff(ofs)
        ent = np.repeat(np.arange(d.n_entry), npole)
        self.disp = {
            "comp": np.asarray(d.comp, dtype=np.int64),
            "cell": np.asarray(d.cell, dtype=np.int64),
            "ent": ent,
            "am1": np.asarray(d.am1, dtype=np.complex128),
            "b": np.asarray(d.b, dtype=np.complex128),
            "P": np.zeros(int(ofs[-1]), dtype=np.complex128),
        }

    def _setup_mix(self):
        """Slanted-interface entries (openem/device_tables.py:291-321, openem/coeffs.py:162-171):
        float64 coefficients ``k1, k2, 1 - beta, 1 / (k1 k2 + beta)``, complex pole states of
        both branches, the accumulated d_tot and the harmonic unknown d_h; the entries' update
        coefficients pass the curl through (ca = 0, cb = 1; a zeroed PEC cell stays zero)."""
        sc = self.sc
        self.mix = None
        mm = sc.dispersion_mix
        if mm is None or mm.n_entry == 0:
            return
        mm.validate(self.shape, sc.dispersion)
        k1, k2, omb, invd = mm.coefficients()
        comp = np.asarray(mm.comp, np.int64)
        cell = np.asarray(mm.cell, np.int64)
        n = comp.size
        p_ofs = np.asarray(mm.p_ofs, np.int64)
        q_ofs = np.asarray(mm.q_ofs, np.int64)
        for c in range(3):
            idx = cell[comp == c]
            self.ca[c].ravel()[idx] = 0.0
            self.cb[c].ravel()[idx] = np.where(self.cb[c].ravel()[idx] != 0.0, 1.0, 0.0)
        self.mix = {"comp": comp, "cell": cell, "k1": k1, "k2": k2, "omb": omb, "invd": invd,
                    "p_ent": np.repeat(np.arange(n), np.diff(p_ofs)),
                    "q_ent": np.repeat(np.arange(n), np.diff(q_ofs)),
                    "pa": np.asarray(mm.pa, np.complex128), "pb": np.asarray(mm.pb, np.complex128),
                    "qa": np.asarray(mm.qa, np.complex128), "qb": np.asarray(mm.qb, np.complex128),
                    "P": np.zeros(int(p_ofs[-1]), np.complex128),
                    "Q": np.zeros(int(q_ofs[-1]), np.complex128),
                    "dtot": np.zeros(n), "dh": np.zeros(n), "sp": np.zeros(n), "sq": np.zeros(n),
                    "dte": sc.dt / EPSILON_0}

    def _mix_field(self):
        m = self.mix
        out = np.empty(m["comp"].size)
        for c in range(3):
            sel = m["comp"] == c
            out[sel] = self.E[c].ravel()[m["cell"][sel]]
        return out

    def mix_pre(self):
        """Both branches advanced to the half step from E^n and d_h^n
        (openem/kernels/dispersion_mix.cu:41-85): SP = sum 2 Re(P_half), SQ = sum Re(Q_half)."""
        m = getattr(self, "mix", None)
        if m is None:
            return
        en = self._mix_field()
        n = en.size
        m["P"] += m["pa"] * m["P"] + m["pb"] * en[m["p_ent"]]
        m["Q"] += m["qa"] * m["Q"] + m["qb"] * m["dh"][m["q_ent"]]
        m["sp"] = np.zeros(n)
        np.add.at(m["sp"], m["p_ent"], 2.0 * m["P"].real)
        m["sq"] = np.zeros(n)
        np.add.at(m["sq"], m["q_ent"], m["Q"].real)

    def mix_post(self):
        """The pass-through value (stretched curl, minus J, plus the E-side sources) advances
        d_tot; the scalar equation gives d_h^{n+1}, E^{n+1} = k2 d_h + SQ, and both branches
        take their step-(n+1) terms (openem/kernels/dispersion_mix.cu:87-135)."""
        m = getattr(self, "mix", None)
        if m is None:
            return
        curl = self._mix_field()
        m["dtot"] = m["dtot"] + m["dte"] * curl
        dh = (m["dtot"] - m["k1"] * m["sq"] - m["omb"] * m["sp"]) * m["invd"]
        m["dh"] = dh
        en = m["k2"] * dh + m["sq"]
        m["P"] += m["pb"] * en[m["p_ent"]]
        m["Q"] += m["qb"] * dh[m["q_ent"]]
        for c in range(3):
            sel = m["comp"] == c
            self.E[c].ravel()[m["cell"][sel]] = en[sel]

    def _entry_field(self, F):
        d = self.disp
        out = np.empty(d["comp"].size)
        for c in range(3):
            m = d["comp"] == c
            out[m] = F[c].ravel()[d["cell"][m]]
        return out

    def _setup_sources(self):
        sc = self.sc
        az = sc.grid.axes[2]
        self.pw = []
        groups = {}
        for s in sc.sources:
            if s.axis != 2 or s.pol_axis not in (0, 1):
                raise NotImplementedError("plane waves: z propagation, Ex/Ey polarisation only")
            groups.setdefault(int(s.pol_axis), []).append(s)
        for pol, grp in sorted(groups.items()):
            s0 = grp[0]
            ks = int(s0.plane_index)
            kh = ks - 1 if s0.direction > 0 else ks
            sh, se = _SIGNS[int(s0.direction)]
            sp = -1.0 if pol == 1 else 1.0
            self.pw.append({
                "pol": pol, "ks": ks, "kh": kh,
                "coef_h": sp * sh * sc.dt / MU_0 / float(az.dl[kh]),
                "coef_e": se / float(az.dl_dual[ks]),
                "ex": sum(np.asarray(x.ex_inc, dtype=np.float64) for x in grp),
                "hy": sum(np.asarray(x.hy_inc, dtype=np.float64) for x in grp)})
        self.dip_e = self._dipole_table([d for d in sc.dipoles if not d.magnetic], half=True)
        self.dip_h = self._dipole_table([d for d in sc.dipoles if d.magnetic], half=False)
        self.modes = self._mode_tables()

    def _mode_tables(self):
        """One entry per mode source (openem/sources_setup.py:376-416): the cyclic tangential
        pair t1 = axis+1, t2 = axis+2, H plane kh and E plane ks, the four coefficients and the
        (profile, amplitude) terms, the base term followed by the broadband corrections."""
        sc = self.sc
        out = []
        for m in getattr(sc, "mode_sources", None) or []:
            a = int(m.axis)
            ax = sc.grid.axes[a]
            ks = int(m.plane_index)
            kh = ks - 1 if m.direction > 0 else ks
            s_h1, s_h2, s_e1, s_e2 = _MODE_SIGNS[int(m.direction)]
            ch = sc.dt / MU_0 * (1.0 / float(ax.dl[kh]))
            ce = 1.0 / float(ax.dl_dual[ks])
            terms_h = [(np.asarray(m.ey_inc), np.asarray(m.ez_inc), np.asarray(m.amp_e))]
            terms_e = [(np.asarray(m.hy_inc), np.asarray(m.hz_inc), np.asarray(m.amp_h))]
            for k in range(0 if m.bb_ey is None else len(m.bb_ey)):
                terms_h.append((np.asarray(m.bb_ey[k]), np.asarray(m.bb_ez[k]),
                                np.asarray(m.bb_amp_e[k])))
                terms_e.append((np.asarray(m.bb_hy[k]), np.asarray(m.bb_hz[k]),
                                np.asarray(m.bb_amp_h[k])))
            out.append({"axis": a, "t1": (a + 1) % 3, "t2": (a + 2) % 3, "ks": ks, "kh": kh,
                        "ch": (s_h1 * ch, s_h2 * ch), "ce": (s_e1 * ce, s_e2 * ce),
                        "th": terms_h, "te": terms_e})
        return out

    @staticmethod
    def _plane(F, axis, k):
        """The (n_t1, n_t2) view of plane ``k`` along ``axis`` in cyclic tangential order."""
        if axis == 0:
            return F[k, :, :]          # (y, z)
        if axis == 1:
            return F[:, k, :].T        # (z, x)
        return F[:, :, k]              # (x, y)

    def _mode_value(self, prof, amp):
        """Real path: Re(profile * amp) (openem/kernels/source_dft.cu:84-128)."""
        return (prof * amp).real

    def inject_mode_h(self, n):
        """H side: H_t1 += c_h1 * E_t2 profile * amp_e[n], H_t2 += c_h2 * E_t1 profile."""
        for md in self.modes:
            H1 = self._plane(self.H[md["t1"]], md["axis"], md["kh"])
            H2 = self._plane(self.H[md["t2"]], md["axis"], md["kh"])
            for e1, e2, amp in md["th"]:
                H1 += md["ch"][0] * self._mode_value(e2, amp[n])
                H2 += md["ch"][1] * self._mode_value(e1, amp[n])

    def inject_mode_e(self, n):
        """E side: E_t1 += cb_t1 * c_e1 * H_t2 profile * amp_h[n], E_t2 likewise with H_t1."""
        for md in self.modes:
            E1 = self._plane(self.E[md["t1"]], md["axis"], md["ks"])
            E2 = self._plane(self.E[md["t2"]], md["axis"], md["ks"])
            cb1 = self._plane(self.cb[md["t1"]], md["axis"], md["ks"])
            cb2 = self._plane(self.cb[md["t2"]], md["axis"], md["ks"])
            for h1, h2, amp in md["te"]:
                E1 += cb1 * md["ce"][0] * self._mode_value(h2, amp[n])
                E2 += cb2 * md["ce"][1] * self._mode_value(h1, amp[n])

    def _dipole_table(self, dips, half: bool):
        if not dips:
            return None
        tabs = [np.asarray(d.waveform.amp_half if half else d.waveform.amp_int,
                           dtype=np.float64) for d in dips]
        nsteps1 = min(t.size for t in tabs)
        if self.n_total > nsteps1 - 1:
            raise ValueError(f"asked to run {self.n_total} steps, dipole waveform has "
                             f"{nsteps1} samples")
        pts = []
        for s, d in enumerate(dips):
            for (i, j, k), cf in zip(np.asarray(d.indices), np.asarray(d.coef)):
                pts.append((int(d.component), int(i), int(j), int(k), float(cf), s))
        return {"pts": pts, "amp": np.stack([t[:nsteps1] for t in tabs])}

    def _setup_monitors(self):
        sc = self.sc
        nt = self.n_total
        te = (np.arange(nt, dtype=np.float64) + 1.0) * sc.dt
        th = (np.arange(nt, dtype=np.float64) + 0.5) * sc.dt
        self.t_e, self.t_h = te, th
        nx, ny, nz = self.shape
        self.fmon = []
        for m in sc.flux_monitors:
            f = np.asarray(m.freqs, dtype=np.float64)
            t1, t2 = [a for a in range(3) if a != m.axis]
            n1, n2 = self.shape[t1], self.shape[t2]
            self.fmon.append({"m": m, "f": f, "t1": t1, "t2": t2,
                              "we": apod_window(te, m.apodization),
                              "wh": apod_window(th, m.apodization),
                              "acc": np.zeros((4, f.size, n1, n2), dtype=np.complex128)})
        self.bmon = []
        for m in sc.field_monitors:
            f = np.asarray(m.freqs, dtype=np.float64)
            (i0, j0, k0), (ni, nj, nk) = m.origin, m.box
            self.bmon.append({"m": m, "f": f,
                              "sl": (slice(i0, i0 + ni), slice(j0, j0 + nj), slice(k0, k0 + nk)),
                              "we": apod_window(te, m.apodization),
                              "wh": apod_window(th, m.apodization),
                              "acc": np.zeros((6, f.size, ni, nj, nk), dtype=np.complex128)})
        self.tmon = []
        for m in sc.field_time_monitors:
            (i0, j0, k0), (ni, nj, nk) = m.origin, m.box
            self.tmon.append({"m": m, "sl": (slice(i0, i0 + ni), slice(j0, j0 + nj),
                                             slice(k0, k0 + nk)),
                              "buf": np.zeros((len(m.comps), m.num_slots, ni, nj, nk),
                                              dtype=self.E[0].dtype)})
        # flux time monitors: the colocated geometry (openem/flux.py:480-531) is a scene input
        from openem_b200 import flux_time as FT
        self.ftmon = [{"m": m, "g": FT.geometry(sc.grid, m), "buf": np.zeros(m.num_slots),
                       "ekeep": None} for m in getattr(sc, "flux_time_monitors", [])]
        # t = 0 sample, taken before the loop on zero fields (openem/solver.py:492-495)
        self._sample_time(0)
        self._sample_flux_time(0)

    def _sample_flux_time(self, m_step):
        """Instantaneous colocated flux in two shots (openem/readout.py:20-73): the second shot
        of m_step - 1 (its kept colocated E with the current H^{m-1/2}) runs before the first
        shot of m_step (E^m with H^{m-1/2}, E kept)."""
        from openem_b200 import flux_time as FT
        for ft in self.ftmon:
            m, g = ft["m"], ft["g"]
            t1, t2 = g["tax"]
            for phase, m_ref in ((1, m_step - 1), (0, m_step)):
                off = m_ref - m.step_begin
                if m_ref < 0 or off < 0 or m_ref >= m.step_end or off % m.interval:
                    continue
                slot = off // m.interval
                if slot >= m.num_slots:
                    continue
                if phase == 0:
                    ft["ekeep"] = [(FT.colocate(self.E[t1], g, "Eu", p),
                                    FT.colocate(self.E[t2], g, "Ev", p))
                                   for p in range(len(g["planes"]))]
                s = 0.0
                for p, pe in enumerate(g["planes"]):
                    eu, ev = ft["ekeep"][p]
                    hu = FT.colocate(self.H[t1], g, "Hu", p)
                    hv = FT.colocate(self.H[t2], g, "Hv", p)
                    s += pe["w"] * 0.5 * float(((eu * hv - ev * hu) * g["dS"]).sum())
                if phase == 0:
                    ft["buf"][slot] = s
                else:
                    ft["buf"][slot] += s

    # ---- one step -------------------------------------------------------------------------
    @staticmethod
    def _take(F, idx, axis):
        return np.take(F, idx, axis=axis)

    def _stretch(self, psi, d, coef, axis):
        a, b, k = coef[axis]
        sh = [1, 1, 1]
        sh[axis] = -1
        a, b, k = a.reshape(sh), b.reshape(sh), k.reshape(sh)
        psi *= b
        psi += a * d
        return k * d + psi

    def _bc(self, v, axis):
        sh = [1, 1, 1]
        sh[axis] = -1
        return np.asarray(v).reshape(sh)

    def update_h(self):
        Ex, Ey, Ez = self.E
        Hx, Hy, Hz = self.H
        nxt, mnx, idl = self.nxt, self.mnx, self.idl_p
        ph, pml = self.psi_h, self.pml_h
        fwd = lambda F, a: (self._take(F, nxt[a], a) * self._bc(mnx[a], a) - F) * self._bc(idl[a], a)
        # Hx: -(dEz/dy - dEy/dz)
        sy = self._stretch(ph[0], fwd(Ez, 1), pml, 1)
        sz = self._stretch(ph[1], fwd(Ey, 2), pml, 2)
        dHx = sy - sz
        sz2 = self._stretch(ph[2], fwd(Ex, 2), pml, 2)
        sx2 = self._stretch(ph[3], fwd(Ez, 0), pml, 0)
        dHy = sz2 - sx2
        sx3 = self._stretch(ph[4], fwd(Ey, 0), pml, 0)
        sy3 = self._stretch(ph[5], fwd(Ex, 1), pml, 1)
        dHz = sx3 - sy3
        Hx -= self.ch * dHx
        Hy -= self.ch * dHy
        Hz -= self.ch * dHz

    def inject_h(self, n):
        """H-side sources in OpenEM's order (openem/solver.py:876-918): magnetic dipoles, plane
        waves, mode sources."""
        if self.dip_h is not None:
            for c, i, j, k, cf, s in self.dip_h["pts"]:
                self.H[c][i, j, k] -= self.ch * cf * self.dip_h["amp"][s, n]
        for p in self.pw:
            Ht = self.H[1] if p["pol"] == 0 else self.H[0]
            Ht[:, :, p["kh"]] += p["coef_h"] * p["ex"][n]
        self.inject_tfsf("h", n)
        self.inject_mode_h(n)

    def disp_pre(self):
        d = self.disp
        if d is None:
            return
        en = self._entry_field(self.E)[d["ent"]]
        dP = d["am1"] * d["P"] + d["b"] * en
        d["P"] += dP
        w = np.zeros(d["comp"].size)
        np.add.at(w, d["ent"], 2.0 * dP.real)
        for c in range(3):
            m = d["comp"] == c
            self.hist[c].ravel()[d["cell"][m]] = w[m]

    def disp_post(self):
        d = self.disp
        if d is None:
            return
        en = self._entry_field(self.E)[d["ent"]]
        d["P"] += d["b"] * en

    def update_e(self):
        Ex, Ey, Ez = self.E
        Hx, Hy, Hz = self.H
        prv, mpv, idl = self.prv, self.mpv, self.idl_d
        pe, pml = self.psi_e, self.pml_e
        bwd = lambda F, a: (F - self._take(F, prv[a], a) * self._bc(mpv[a], a)) * self._bc(idl[a], a)
        px, py, pz = (self._bc(self.pec[a], a) for a in range(3))
        sy = self._stretch(pe[0], bwd(Hz, 1), pml, 1)
        sz = self._stretch(pe[1], bwd(Hy, 2), pml, 2)
        cx = sy - sz
        sz2 = self._stretch(pe[2], bwd(Hx, 2), pml, 2)
        sx2 = self._stretch(pe[3], bwd(Hz, 0), pml, 0)
        cy = sz2 - sx2
        sx3 = self._stretch(pe[4], bwd(Hy, 0), pml, 0)
        sy3 = self._stretch(pe[5], bwd(Hx, 1), pml, 1)
        cz = sx3 - sy3
        ca, cb, cw, hs = self.ca, self.cb, self.cw, self.hist
        self.E[0] = (ca[0] * Ex + cb[0] * (cx - cw * hs[0])) * py * pz
        self.E[1] = (ca[1] * Ey + cb[1] * (cy - cw * hs[1])) * pz * px
        self.E[2] = (ca[2] * Ez + cb[2] * (cz - cw * hs[2])) * px * py

    def inject_e(self, n):
        """E-side sources in OpenEM's order (openem/solver.py:955-969): plane waves, mode
        sources, electric dipoles."""
        for p in self.pw:
            c = p["pol"]
            self.E[c][:, :, p["ks"]] += self.cb[c][:, :, p["ks"]] * p["coef_e"] * p["hy"][n]
        self.inject_tfsf("e", n)
        self.inject_mode_e(n)
        if self.dip_e is not None:
            for c, i, j, k, cf, s in self.dip_e["pts"]:
                self.E[c][i, j, k] -= self.cb[c][i, j, k] * cf * self.dip_e["amp"][s, n]

    def dft(self, n):
        for mon in self.fmon:
            m, f = mon["m"], mon["f"]
            km, ax, t1, t2 = int(m.plane_index), int(m.axis), mon["t1"], mon["t2"]
            take = lambda F, k: np.take(F, k, axis=ax)
            vals = (take(self.E[t1], km), take(self.E[t2], km),
                    0.5 * (take(self.H[t1], km) + take(self.H[t1], km - 1)),
                    0.5 * (take(self.H[t2], km) + take(self.H[t2], km - 1)))
            pe = np.exp(2j * np.pi * f * self.t_e[n]) * mon["we"][n]
            ph = np.exp(2j * np.pi * f * self.t_h[n]) * mon["wh"][n]
            acc = mon["acc"]
            for c in range(4):
                acc[c] += (pe if c < 2 else ph)[:, None, None] * vals[c][None]
        for mon in self.bmon:
            f, sl = mon["f"], mon["sl"]
            pe = np.exp(2j * np.pi * f * self.t_e[n]) * mon["we"][n]
            ph = np.exp(2j * np.pi * f * self.t_h[n]) * mon["wh"][n]
            acc = mon["acc"]
            for c in range(6):
                F = self.E[c] if c < 3 else self.H[c - 3]
                acc[c] += (pe if c < 3 else ph)[:, None, None, None] * F[sl][None]

    def _sample_time(self, m_step):
        """Two-shot H average at m = m_step: E^m + H^{m-1/2}/2 now, H^{m+1/2}/2 one step later."""
        for tm in self.tmon:
            m = tm["m"]
            for add in (1, 0):
                m_ref = m_step - add
                if add and m_step == 0:
                    continue
                off = m_ref - m.step_begin
                if off < 0 or m_ref >= m.step_end or off % m.interval:
                    continue
                slot = off // m.interval
                if slot >= m.num_slots:
                    continue
                for q, c in enumerate(m.comps):
                    F = self.E[c] if c < 3 else self.H[c - 3]
                    w = (1.0 if c < 3 else 0.5) if not add else (0.0 if c < 3 else 0.5)
                    if w == 0.0:
                        continue
                    v = w * F[tm["sl"]]
                    if add:
                        tm["buf"][q, slot] += v
                    else:
                        tm["buf"][q, slot] = v

    def absorb(self, family):
        """Absorber decay (openem/kernels/absorber.cu:20-70): every slab in scene order
        multiplies the family inside its layers; E normal / H tangential components sit at the
        half cell (decay_half), the others at the whole cell (decay_int)."""
        F = self.E if family == "E" else self.H
        for sl in getattr(self.sc, "absorbers", None) or []:
            a, g0 = int(sl.axis), int(sl.g0)
            di = np.asarray(sl.decay_int, np.float64)
            dh = np.asarray(sl.decay_half, np.float64)
            sl_ = [slice(None)] * 3
            sl_[a] = slice(g0, g0 + di.size)
            sh = [1, 1, 1]
            sh[a] = -1
            for c in range(3):
                half = (c == a) if family == "E" else (c != a)
                F[c][tuple(sl_)] *= (dh if half else di).reshape(sh)

    def step(self):
        n = self.n
        self.update_h()
        self.inject_h(n)
        self.absorb("H")
        self.disp_pre()
        self.mix_pre()
        self.modulate(n)
        self.tensor_pre()
        self.update_e()
        self.inject_e(n)
        self.mix_post()
        self.tensor_post()
        self.disp_post()
        self.absorb("E")
        self._sample_time(n + 1)
        self.dft(n)
        self._sample_flux_time(n + 1)
        self.n += 1

    def load_fields(self, fields) -> None:
        """Start from the given six fields (Ex, Ey, Ez, Hx, Hy, Hz) instead of zeros. CPML psi,
        pole states and DFT accumulators still start at zero; the engine sets the same start
        with ``Plan.write_field``. Scenes with time monitors are refused (their t = 0 sample
        was taken on zero fields)."""
        if self.n:
            raise RuntimeError("load_fields must come before the first step")
        if self.tmon or getattr(self, "ftmon", []):
            raise ValueError("load_fields: scenes with time monitors are not supported")
        for F, v in zip((*self.E, *self.H), fields):
            F[...] = v

    def run(self, n_steps: int | None = None) -> OracleResult:
        n_steps = self.n_total if n_steps is None else int(n_steps)
        t0 = time.perf_counter()
        for _ in range(n_steps):
            self.step()
        return self.result(time.perf_counter() - t0)

    def result(self, seconds: float = 0.0) -> OracleResult:
        r = OracleResult(steps_run=self.n, seconds=seconds)
        for mon in self.fmon:
            r.phasors[mon["m"].name] = mon["acc"].copy()
        for mon in self.bmon:
            r.field_phasors[mon["m"].name] = mon["acc"].copy()
        for tm in self.tmon:
            m = tm["m"]
            m_last = min(self.n - 1, m.step_end - 1)
            off = m_last - m.step_begin
            filled = 0 if off < 0 else min(m.num_slots, off // m.interval + 1)
            r.time_samples[m.name] = tm["buf"][:, :filled].copy()
            r.time_slots[m.name] = filled
        for ft in getattr(self, "ftmon", []):
            m = ft["m"]
            off = min(self.n - 1, m.step_end - 1) - m.step_begin
            filled = 0 if off < 0 else min(m.num_slots, off // m.interval + 1)
            r.flux_time[m.name] = ft["buf"][:filled].copy()
        names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
        for nm, F in zip(names, (*self.E, *self.H)):
            r.fields[nm] = F.copy()
        return r


def run(sc, num_steps: int | None = None) -> OracleResult:
    """Run ``num_steps`` (default: the scene's nominal count) on the FP64 oracle."""
    if sc.any_bloch:
        return BlochOracle(sc, num_steps).run()
    return Oracle(sc, num_steps).run()


class PerturbedOracle(Oracle):
    """The FP64 oracle with float32-sized rounding noise: after every step each stored value
    (the fields, the pole states of the dispersive tables, and the accumulated d_tot and
    harmonic d_h of the mixed-form entries; real and imaginary parts apart) is multiplied by
    ``1 + u * U(-1, 1)`` with ``u = 2**-24`` (half an ulp of float32). The distance of its
    result from the clean run is the rounding floor of a float32 engine on that scene: how far
    one float32 rounding per stored value and step moves the fields. Resonant dispersive scenes
    amplify it well above 2**-24; a float32 engine cannot be held closer to the FP64 oracle
    than this floor."""

    def __init__(self, sc, n_total: int | None = None, seed: int = 0):
        super().__init__(sc, n_total)
        self._rng = np.random.default_rng(seed)

    def _noise(self, shape):
        return 1.0 + 2.0 ** -24 * self._rng.uniform(-1.0, 1.0, shape)

    def step(self):
        super().step()
        for F in (*self.E, *self.H):
            F *= self._noise(F.shape)
        states = []
        if getattr(self, "disp", None) is not None:
            states.append((self.disp, "P"))
        if getattr(self, "mix", None) is not None:
            states += [(self.mix, k) for k in ("P", "Q", "dtot", "dh")]
        for d, k in states:
            a = d[k]
            if np.iscomplexobj(a):
                d[k] = a.real * self._noise(a.shape) + 1j * a.imag * self._noise(a.shape)
            else:
                d[k] = a * self._noise(a.shape)


def fp32_floor(sc, num_steps: int | None = None, seed: int = 1, clean=None) -> dict:
    """Per-field relative L2 distance between a ``PerturbedOracle`` run and the clean run."""
    ref = clean if clean is not None else Oracle(sc, num_steps).run()
    pert = PerturbedOracle(sc, num_steps, seed).run()
    out = {}
    for nm, a in pert.fields.items():
        b = ref.fields[nm]
        out[nm] = float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
    return out


class BlochOracle(Oracle):
    """Complex-field Bloch path (``openem/kernels/bloch.cu:25-221``): fields carry re + i im,
    the periodic seam neighbour is multiplied by ``exp(+/- i 2 pi k)``; the scene subset is
    lossless and non-dispersive with plane sources excluded (``openem/solver.py:1221-1260``)."""

    def __init__(self, sc, n_total: int | None = None):
        if sc.any_dispersion or sc.any_loss or sc.any_pec or sc.sources or sc.tfsf_sources:
            raise NotImplementedError("Bloch subset: lossless, non-dispersive, no plane wave")
        if getattr(sc, "flux_time_monitors", None):
            raise NotImplementedError("oracle: flux time monitors not transcribed")
        self.sc = sc
        self.n_total = int(n_total if n_total is not None else sc.num_time_steps)
        self.shape = sc.shape
        self.E = [np.zeros(self.shape, dtype=np.complex128) for _ in range(3)]
        self.H = [np.zeros(self.shape, dtype=np.complex128) for _ in range(3)]
        self.psi_h = [np.zeros(self.shape, dtype=np.complex128) for _ in range(6)]
        self.psi_e = [np.zeros(self.shape, dtype=np.complex128) for _ in range(6)]
        tabs = [a.index_tables(k) for a, k in zip(sc.grid.axes, sc.bloch_k)]
        self.nxt = [t["nxt"] for t in tabs]
        self.prv = [t["prv"] for t in tabs]
        self.mnx = [np.asarray(t["mnx"], dtype=np.complex128) for t in tabs]
        self.mpv = [np.asarray(t["mpv"], dtype=np.complex128) for t in tabs]
        self.pec = [t["pec"] for t in tabs]
        self.idl_p = [1.0 / a.dl for a in sc.grid.axes]
        self.idl_d = [1.0 / a.dl_dual for a in sc.grid.axes]
        self.pml_e = [pml_axis_arrays(sc, a, "E") for a in range(3)]
        self.pml_h = [pml_axis_arrays(sc, a, "H") for a in range(3)]
        self.ch = sc.dt / MU_0
        self.cw = EPSILON_0 / sc.dt
        self.ca = [np.ones(self.shape) for _ in range(3)]
        self.cb = [(sc.dt / EPSILON_0) / np.asarray(e, dtype=np.float64)
                   for e in (sc.eps_ex, sc.eps_ey, sc.eps_ez)]
        self.hist = [np.zeros(self.shape) for _ in range(3)]
        self.disp = None
        self.pw = []
        self.dip_e = self._dipole_table_c([d for d in sc.dipoles if not d.magnetic], True)
        self.dip_h = self._dipole_table_c([d for d in sc.dipoles if d.magnetic], False)
        self.modes = self._mode_tables()
        self._setup_monitors()  # complex time samples (openem/kernels/bloch.cu:280-318)
        self.n = 0

    def _mode_value(self, prof, amp):
        """Complex path: the full product profile * amp (openem/kernels/bloch.cu:326-384)."""
        return prof * amp

    def _dipole_table_c(self, dips, half: bool):
        if not dips:
            return None
        tabs = [np.asarray(d.waveform.amp_half_complex if half else d.waveform.amp_int_complex,
                           dtype=np.complex128) for d in dips]
        n1 = min(t.size for t in tabs)
        pts = []
        for s, d in enumerate(dips):
            for (i, j, k), cf in zip(np.asarray(d.indices), np.asarray(d.coef)):
                pts.append((int(d.component), int(i), int(j), int(k), float(cf), s))
        return {"pts": pts, "amp": np.stack([t[:n1] for t in tabs])}


# ---- early termination on the oracle (openem/solver.py:107-203, :1165-1213) ------------------
def shutoff_sums(o: Oracle) -> tuple:
    """``(sum V |E|^2, sum V eps |E|^2, sum V |H|^2)`` of the oracle's current fields in float64.
    V is the Yee dual volume of the E component of the same index (``openem/grid.py:350-366``),
    used for H as well (``openem/solver.py:171-176``); eps the scene's relative permittivity."""
    sc = o.sc
    (xp, yp, zp) = (a.dl for a in sc.grid.axes)
    (xd, yd, zd) = (a.dl_dual for a in sc.grid.axes)
    vols = (xp[:, None, None] * yd[None, :, None] * zd[None, None, :],
            xd[:, None, None] * yp[None, :, None] * zd[None, None, :],
            xd[:, None, None] * yd[None, :, None] * zp[None, None, :])
    eps = (sc.eps_ex, sc.eps_ey, sc.eps_ez)
    e2 = [np.abs(F) ** 2 for F in o.E]
    h2 = [np.abs(F) ** 2 for F in o.H]
    m_e2 = float(sum((v * a).sum() for v, a in zip(vols, e2)))
    w_e = float(sum((v * np.asarray(ep, dtype=np.float64) * a).sum()
                    for v, ep, a in zip(vols, eps, e2)))
    w_h = float(sum((v * a).sum() for v, a in zip(vols, h2)))
    return m_e2, w_e, w_h


def run_shutoff(sc, policy, num_steps: int | None = None):
    """Run the oracle with early termination: every ``policy.interval`` steps feed the float64
    sums and (real path only) the flux of every flux monitor to ``policy.check``, and stop once
    it fires after the last source has finished and after the first time-monitor step
    (``openem/solver.py:160-203``). Returns ``(OracleResult, steps_run, triggered, trace)``,
    ``trace`` holding ``(step, m_e2, energy)`` per check."""
    from openem_b200 import flux as flux_mod
    from openem_b200 import shutoff as shutoff_mod
    o = BlochOracle(sc, num_steps) if sc.any_bloch else Oracle(sc, num_steps)
    source_end = shutoff_mod.source_end_step(sc)
    tms = list(sc.field_time_monitors) + list(getattr(sc, "flux_time_monitors", []))
    guard = max([int(m.step_begin) + 1 for m in tms] + [0])
    interval = int(policy.interval)
    trace, triggered = [], False
    while o.n < o.n_total:
        o.step()
        if o.n % interval:
            continue
        m_e2, w_e, w_h = shutoff_sums(o)
        m_u = 0.5 * (EPSILON_0 * w_e + MU_0 * w_h)
        fl = np.zeros(0)
        if o.fmon and not sc.any_bloch:
            fl = np.concatenate([flux_mod.plane_flux(mon["acc"], sc.grid, axis=int(mon["m"].axis))
                                 for mon in o.fmon])
        trace.append((o.n, m_e2, m_u))
        if policy.check(o.n, m_e2, m_u, fl) and o.n > source_end and o.n >= guard:
            triggered = True
            break
    return o.result(), o.n, triggered, trace
