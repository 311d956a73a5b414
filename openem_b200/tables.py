"""Host-side float64 table construction: everything the device plan needs, computed from a
``Scene`` with numpy before upload (OpenEM computes the same quantities in
``openem/coeffs.py``, ``openem/device_tables.py``, ``openem/sources_setup.py`` and
``openem/monitors_setup.py``). No device code runs here, so all of it is testable on a CPU.

Layout decisions (the engine's own):

* **materials** -- every cell gets one index into a table of distinct tuples
  ``(ca, cb, eps, pole set, pole count) x 3 components``; the update coefficients
  ``ca = (eps - s)/(eps + s + G)``, ``cb = (dt/eps0)/(eps + s + G)`` are evaluated in float64 and
  rounded once to float32. PEC cells and the tangential E cells on a PEC-backed wall get
  ``ca = cb = 0`` (OpenEM multiplies by a PEC mask after the update instead).
* **pole sets** -- ADE entries with identical float32 coefficient lists share one set.
* **pole storage** -- pole states are packed in padded cell order, then component, then pole;
  ``seg_ofs`` holds the number of poles before every 32-cell z segment.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

EPSILON_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6
APOD_K = 0.5
#: one-face TF/SF correction signs by propagation direction (openem/tfsf1d.py:46)
PLANE_SIGNS = {+1: (1.0, 1.0), -1: (-1.0, -1.0)}

try:  # hash-based factorisation is O(n); numpy's unique sorts
    import pandas as _pd
except Exception:  # pragma: no cover
    _pd = None


def factorize(a: np.ndarray):
    """Dense codes ``0..k-1`` for the distinct values of a 1D array (first-seen order with
    pandas, sorted order with numpy) and the number of distinct values."""
    a = np.ascontiguousarray(a).ravel()
    if _pd is not None:
        codes, uniq = _pd.factorize(a, sort=False)
        return codes.astype(np.int64, copy=False), len(uniq)
    uniq, inv = np.unique(a, return_inverse=True)
    return inv.astype(np.int64, copy=False), uniq.size


def _factorize_rows_exact(cols):
    code, n = factorize(cols[0])
    for c in cols[1:]:
        cc, m = factorize(c)
        code, n = factorize(code * m + cc)
    return code, n


def factorize_rows(cols):
    """Codes for the distinct rows of equal-length integer columns, and their count.

    One 64-bit hash per row (a multiply-xor mix of the columns, finished with the splitmix64
    avalanche) is factorised once; every row is then compared column by column with the first
    row of its code, and any collision falls back to the exact column-by-column factorisation,
    so the codes are always exact."""
    if len(cols) == 1:
        return factorize(cols[0])
    u = [np.ascontiguousarray(c).ravel().view(np.uint64) for c in cols]
    h = np.zeros(u[0].size, np.uint64)
    with np.errstate(over="ignore"):
        for c in u:
            h ^= c
            h *= np.uint64(0x9E3779B97F4A7C15)
            h ^= h >> np.uint64(29)
        h ^= h >> np.uint64(30)
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(27)
        h *= np.uint64(0x94D049BB133111EB)
        h ^= h >> np.uint64(31)
    code, n = factorize(h)
    first = np.empty(n, dtype=np.int64)
    first[code[::-1]] = np.arange(code.size - 1, -1, -1, dtype=np.int64)
    rep = first[code]
    for c in u:
        if not np.array_equal(c[rep], c):
            return _factorize_rows_exact(cols)
    return code, n


def pad_z(n: int) -> int:
    return (n + 31) // 32 * 32


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


# ---------------------------------------------------------------------------------------------
# Axes
# ---------------------------------------------------------------------------------------------

def pml_axis(sc, axis: int, at: str):
    """``(a | b | 1/kappa)`` concatenated, identity outside the layers, and the layer counts at
    the two ends (``openem/coeffs.py:21-42``)."""
    n = sc.grid.axes[axis].n
    a, b, k = np.zeros(n), np.ones(n), np.ones(n)
    lo = hi = 0
    for side in ("lo", "hi"):
        c = sc.pml.get((axis, side))
        if c is None:
            continue
        m = int(np.asarray(c.a_E).size)
        sl = slice(0, m) if side == "lo" else slice(n - m, n)
        a[sl] = np.asarray(getattr(c, f"a_{at}"), dtype=np.float64)
        b[sl] = np.asarray(getattr(c, f"b_{at}"), dtype=np.float64)
        k[sl] = np.asarray(getattr(c, f"inv_kappa_{at}"), dtype=np.float64)
        if side == "lo":
            lo = m
        else:
            hi = m
    return np.concatenate([a, b, k]), lo, hi


@dataclass
class AxisTables:
    idl_p: np.ndarray
    idl_d: np.ndarray
    nxt: np.ndarray
    prv: np.ndarray
    mnx: np.ndarray
    mpv: np.ndarray
    pec: np.ndarray
    pml_e: np.ndarray
    pml_h: np.ndarray
    lo: int
    hi: int


def axis_tables(sc, axis: int, bloch_k: float = 0.0) -> AxisTables:
    ax = sc.grid.axes[axis]
    t = ax.index_tables(bloch_k) if bloch_k else ax.index_tables()
    pe, lo_e, hi_e = pml_axis(sc, axis, "E")
    ph, _, _ = pml_axis(sc, axis, "H")
    return AxisTables(idl_p=1.0 / ax.dl, idl_d=1.0 / ax.dl_dual,
                      nxt=np.ascontiguousarray(t["nxt"], dtype=np.int32),
                      prv=np.ascontiguousarray(t["prv"], dtype=np.int32),
                      mnx=np.asarray(t["mnx"]), mpv=np.asarray(t["mpv"]),
                      pec=np.asarray(t["pec"], dtype=np.float64),
                      pml_e=pe, pml_h=ph, lo=lo_e, hi=hi_e)


# ---------------------------------------------------------------------------------------------
# Materials and pole sets
# ---------------------------------------------------------------------------------------------

@dataclass
class MaterialTables:
    table: np.ndarray        # (n_mat, 16) uint32 records
    index: np.ndarray        # (nx, ny, nz) uint16 or uint32
    n_mat: int
    set_ofs: np.ndarray      # (n_sets + 1,) int32
    coef: np.ndarray         # (n_pole_in_sets, 4) float32
    seg_ofs: np.ndarray      # (n_seg,) uint32
    n_pole_total: int
    ca: tuple                # float32 per component (for sources / checks)
    cb: tuple


def _g_dense(sc, shape):
    d = sc.dispersion
    out = [np.zeros(int(np.prod(shape))) for _ in range(3)]
    if d is not None and d.n_entry > 0:
        comp, cell, g = np.asarray(d.comp), np.asarray(d.cell, dtype=np.int64), np.asarray(d.g)
        for c in range(3):
            m = comp == c
            out[c][cell[m]] = g[m]
    return [o.reshape(shape) for o in out]


def e_coefficients(sc, tabs):
    """float32 ``(ca, cb)`` per component, PEC cells and PEC-backed wall cells zeroed."""
    shape = sc.shape
    gg = _g_dense(sc, shape)
    sig = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
    ca, cb = [], []
    for c, eps in enumerate((sc.eps_ex, sc.eps_ey, sc.eps_ez)):
        eps = np.asarray(eps, dtype=np.float64)
        # same operation order as openem/coeffs.py:132-136: den = (eps + s) + G
        s = (np.zeros_like(eps) if sig[c] is None
             else np.asarray(sig[c], dtype=np.float64) * sc.dt / (2.0 * EPSILON_0))
        den = eps + s + gg[c]
        num = eps - s
        ca.append((num / den).astype(np.float32))
        cb.append(((sc.dt / EPSILON_0) / den).astype(np.float32))
    pecs = (sc.pec_ex, sc.pec_ey, sc.pec_ez)
    for c in range(3):
        if pecs[c] is not None and np.asarray(pecs[c]).size:
            idx = np.asarray(pecs[c], dtype=np.int64)
            if idx.min() < 0 or idx.max() >= int(np.prod(shape)):
                raise ValueError(f"pec_e{'xyz'[c]} index out of range")
            ca[c].ravel()[idx] = 0.0
            cb[c].ravel()[idx] = 0.0
    # tangential E on a PEC-backed wall: component c is tangential to the walls of the two
    # other axes (openem/kernels/yee.cu:208-211)
    for a in range(3):
        zero = np.flatnonzero(tabs[a].pec == 0.0)
        if zero.size == 0:
            continue
        for c in range(3):
            if c == a:
                continue
            sl = [slice(None)] * 3
            sl[a] = zero
            ca[c][tuple(sl)] = 0.0
            cb[c][tuple(sl)] = 0.0
    # full-tensor and slanted-interface entries pass the curl through (ca = 0, cb = 1; zero stays
    # zero on a PEC-backed wall): their own passes turn it into E^{n+1}
    # (openem/kernels/tensor.cu, openem/kernels/dispersion_mix.cu, openem/coeffs.py:162-171)
    for tab in passthrough_tables(sc):
        comp = np.asarray(tab.comp)
        cell = np.asarray(tab.cell, np.int64)
        for c in range(3):
            idx = cell[comp == c]
            ca[c].ravel()[idx] = 0.0
            cb[c].ravel()[idx] = np.where(cb[c].ravel()[idx] != 0.0, 1.0, 0.0)
    return ca, cb


def passthrough_tables(sc) -> list:
    """The entry tables whose cells take the D form (tensor media, mixed dispersion)."""
    return [t for t in (sc.tensor, sc.dispersion_mix) if t is not None and t.n_entry]


def mix_tables(sc) -> dict | None:
    """Per entry of a slanted-interface table: component, cell, the pole CSR offsets of both
    branches, float32 pole coefficients as (Re(A-1), Im(A-1), Re(B), Im(B)) rows, the float32
    coefficients (k1, k2, 1 - beta, 1 / (k1 k2 + beta)) and dt / eps0
    (openem/device_tables.py:291-321); refused together with modulation or tensor media (each
    rewrites the same coefficients)."""
    mm = sc.dispersion_mix
    if mm is None or mm.n_entry == 0:
        return None
    if (sc.modulation is not None and sc.modulation.n_entry) or \
            (sc.tensor is not None and sc.tensor.n_entry):
        raise NotImplementedError("mixed dispersion together with modulation or tensor media is "
                                  "not supported")
    mm.validate(sc.shape, sc.dispersion)
    k1, k2, omb, invd = mm.coefficients()

    def rows(a, b):
        a = np.asarray(a, np.complex128)
        b = np.asarray(b, np.complex128)
        if a.size == 0:
            return np.zeros((1, 4), np.float32)
        return np.ascontiguousarray(np.stack([a.real, a.imag, b.real, b.imag], 1), np.float32)
    return {"comp": np.ascontiguousarray(mm.comp, np.int32),
            "cell": np.ascontiguousarray(mm.cell, np.int64),
            "p_ofs": np.ascontiguousarray(mm.p_ofs, np.int32),
            "q_ofs": np.ascontiguousarray(mm.q_ofs, np.int32),
            "pc": rows(mm.pa, mm.pb), "n_p": int(np.asarray(mm.pa).size),
            "qc": rows(mm.qa, mm.qb), "n_q": int(np.asarray(mm.qa).size),
            "k": np.ascontiguousarray(np.stack([k1, k2, omb, invd], 1), np.float32),
            "dte": float(sc.dt / EPSILON_0)}


def tensor_tables(sc, tabs) -> dict | None:
    """Per entry of a fully anisotropic medium: component, cell, the rows of M1 and M2 in
    float32 and the PEC-wall factor of the written value (the pec of the other two axes);
    refused together with dispersion, mixed media, modulation or PEC cells (each rewrites the
    same coefficients)."""
    ten = sc.tensor
    if ten is None or ten.n_entry == 0:
        return None
    if (sc.dispersion is not None and sc.dispersion.n_entry) or \
            (sc.dispersion_mix is not None and sc.dispersion_mix.n_entry) or \
            (sc.modulation is not None and sc.modulation.n_entry) or sc.pec_ex is not None:
        raise NotImplementedError("fully anisotropic media together with dispersion, mixed "
                                  "media, modulation or PEC cells are not supported")
    ten.validate(sc.shape, [{"nxt": t.nxt, "prv": t.prv} for t in tabs])
    m1, m2 = ten.rows(sc.dt)
    comp = np.asarray(ten.comp, np.int32)
    cell = np.asarray(ten.cell, np.int64)
    i, j, k = (np.asarray(x) for x in
               (cell // (sc.shape[1] * sc.shape[2]), (cell // sc.shape[2]) % sc.shape[1],
                cell % sc.shape[2]))
    pec = [np.asarray(t.pec, np.float64) for t in tabs]
    p = np.stack([pec[0][i], pec[1][j], pec[2][k]])
    pf = p[(comp + 1) % 3, np.arange(comp.size)] * p[(comp + 2) % 3, np.arange(comp.size)]
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    return {"comp": np.ascontiguousarray(comp), "cell": np.ascontiguousarray(cell),
            "m1": f32(m1), "m2": f32(m2), "pec": f32(pf)}


_POOL = None


def par_map(fn, n: int, parts: int = 8) -> list:
    """``[fn(lo, hi)]`` over ``parts`` consecutive slices of range(n), on worker threads
    (numpy's elementwise work releases the GIL, so large scans run in parallel)."""
    global _POOL
    if n < (1 << 20):
        return [fn(0, n)]
    if _POOL is None:
        import os
        from concurrent.futures import ThreadPoolExecutor
        _POOL = ThreadPoolExecutor(max_workers=max(8, min(16, os.cpu_count() or 8)))
    step = -(-n // parts)
    return list(_POOL.map(lambda lo: fn(lo, min(lo + step, n)), range(0, n, step)))


def _par_all(test, n: int, parts: int = 8) -> bool:
    """``all(test(lo, hi))`` over slices of range(n), on worker threads."""
    return all(bool(r) for r in par_map(test, n, parts))


def _rows_equal_first(a: np.ndarray) -> bool:
    """Every row of a 2D array equal to the first, bit for bit."""
    v = np.ascontiguousarray(a).view(np.uint64).reshape(a.shape[0], -1)
    return _par_all(lambda lo, hi: np.all(v[lo:hi] == v[0]), v.shape[0])


def entry_pole_sets(sc, bulk_shortcut: bool = True, validate: bool = True):
    """Deduplicate ADE entries by their float32 coefficient lists.

    Returns ``(comp, cell, set_id, set_ofs, coef, counts)``: per entry its component, flat cell
    and pole-set id; per set its first pole in ``coef`` ((n, 4) float32 rows
    ``Re(A-1), Im(A-1), Re(B), Im(B)``) and its pole count. ``None`` without dispersion.
    ``validate=False`` skips the table checks, for a caller that has made them."""
    d = sc.dispersion
    if d is None or d.n_entry == 0:
        return None
    if validate:
        d.validate(sc.shape)
    comp = np.asarray(d.comp)
    cell = np.asarray(d.cell)
    ofs = np.asarray(d.pole_ofs)
    am1 = np.asarray(d.am1, dtype=np.complex128)
    b = np.asarray(d.b, dtype=np.complex128)
    n = d.n_entry
    k0 = int(ofs[1] - ofs[0])
    if bulk_shortcut and 0 < k0 <= 15 and int(ofs[0]) == 0 and \
            _par_all(lambda lo, hi: np.all(np.diff(ofs[lo:hi + 1]) == k0), n):
        # every entry carries k0 poles (offsets i * k0) and, when their float64 bits agree, the
        # same coefficient list (a bulk medium): one set, found without converting every pole
        # (equal float64 values give equal float32 rows; anything else takes the general path)
        A = am1.reshape(n, k0)
        B = b.reshape(n, k0)
        if _rows_equal_first(A) and _rows_equal_first(B):
            row = np.empty((k0, 4), dtype=np.float32)
            row[:, 0], row[:, 1], row[:, 2], row[:, 3] = A[0].real, A[0].imag, B[0].real, B[0].imag
            return (comp, cell, np.zeros(n, dtype=np.int64),
                    np.asarray([0, k0], dtype=np.int32), row, np.asarray([k0], dtype=np.int32))
    ofs = ofs.astype(np.int64)
    npole = np.diff(ofs)
    if npole.max() > 15:
        raise NotImplementedError("more than 15 poles on one component")
    pc = np.empty((am1.size, 4), dtype=np.float32)
    pc[:, 0], pc[:, 1], pc[:, 2], pc[:, 3] = am1.real, am1.imag, b.real, b.imag
    set_id = np.full(d.n_entry, -1, dtype=np.int64)
    set_ofs, coefs, counts = [0], [], []
    uniform_k = np.all(npole == npole[0])
    for k in (np.array([npole[0]]) if uniform_k else np.unique(npole)):
        k = int(k)
        if k == 0:
            continue
        ent = np.arange(d.n_entry) if uniform_k else np.flatnonzero(npole == k)
        if uniform_k and np.all(ofs[:-1] == np.arange(d.n_entry) * k):
            rows = pc.reshape(d.n_entry, 4 * k)
        else:
            rows = pc[(ofs[ent][:, None] + np.arange(k)[None, :]).ravel()].reshape(ent.size, 4 * k)
        bits = rows.view(np.uint32)
        if np.all(bits == bits[0]):                       # one coefficient list for all
            code, nu, first = np.zeros(ent.size, np.int64), 1, np.zeros(1, np.int64)
        else:
            code, nu = factorize_rows([bits[:, q].astype(np.int64) for q in range(4 * k)])
            first = np.full(nu, -1, dtype=np.int64)
            order = np.arange(ent.size)
            first[code[::-1]] = order[::-1]
        base = len(counts)
        for u in range(nu):
            coefs.append(rows[first[u]].reshape(k, 4))
            counts.append(k)
            set_ofs.append(set_ofs[-1] + k)
        set_id[ent] = base + code
    coef = np.concatenate(coefs, axis=0).astype(np.float32) if coefs else np.zeros((0, 4), np.float32)
    return (comp, cell, set_id, np.asarray(set_ofs, dtype=np.int32), coef,
            np.asarray(counts, dtype=np.int32))


def pole_sets(sc):
    """Dense per-component pole-set ids (-1 = none) plus ``set_ofs``, ``coef``, ``counts``."""
    shape = sc.shape
    ep = entry_pole_sets(sc)
    if ep is None:
        return [None, None, None], np.zeros(1, np.int32), np.zeros((0, 4), np.float32), \
            np.zeros(0, np.int32)
    comp, cell, set_id, set_ofs, coef, counts = ep
    ncell = int(np.prod(shape))
    pset = []
    for c in range(3):
        arr = np.full(ncell, -1, dtype=np.int32)
        m = comp == c
        arr[cell[m]] = set_id[m].astype(np.int32)
        pset.append(arr.reshape(shape))
    return pset, set_ofs, coef, counts


def material_tables(sc, tabs) -> MaterialTables:
    shape = sc.shape
    nx, ny, nz = shape
    ca, cb = e_coefficients(sc, tabs)
    eps = [np.asarray(e, dtype=np.float32) for e in (sc.eps_ex, sc.eps_ey, sc.eps_ez)]
    pset, set_ofs, coef, counts = pole_sets(sc)
    # two 64-bit keys per component: (ca, cb) bit patterns and (eps, pole set)
    keys = []
    for c in range(3):
        k1 = (ca[c].view(np.uint32).ravel().astype(np.uint64) << np.uint64(32)) \
            | cb[c].view(np.uint32).ravel().astype(np.uint64)
        keys.append(k1.view(np.int64))
        k2 = eps[c].view(np.uint32).ravel().astype(np.uint64) << np.uint64(32)
        if pset[c] is not None:
            k2 |= (pset[c].ravel().astype(np.int64) + 1).astype(np.uint64)
        keys.append(k2.view(np.int64))
    code, n_mat = factorize_rows(keys)
    first = np.full(n_mat, -1, dtype=np.int64)
    idx = np.arange(code.size)
    first[code[::-1]] = idx[::-1]
    rec = np.zeros((n_mat, 16), dtype=np.uint32)
    npc_mat = np.zeros(n_mat, dtype=np.int64)
    for c in range(3):
        rec[:, c] = ca[c].ravel()[first].view(np.uint32)
        rec[:, 3 + c] = cb[c].ravel()[first].view(np.uint32)
        rec[:, 6 + c] = eps[c].ravel()[first].view(np.uint32)
        ps = pset[c].ravel()[first] if pset[c] is not None else np.full(n_mat, -1, np.int64)
        rec[:, 9 + c] = ps.astype(np.int32).view(np.uint32)
        npl = np.where(ps >= 0, counts[np.maximum(ps, 0)] if counts.size else 0, 0)
        rec[:, 12 + c] = npl.astype(np.int32).view(np.uint32)
        npc_mat += npl
    index = code.reshape(shape).astype(np.uint16 if n_mat <= 65535 else np.uint32)
    # poles before each 32-cell segment of the padded grid
    nzp = pad_z(nz)
    npc = np.zeros((nx, ny, nzp), dtype=np.int64)
    npc[:, :, :nz] = npc_mat[code].reshape(shape)
    seg = npc.reshape(-1, 32).sum(axis=1)
    seg_ofs = np.concatenate([[0], np.cumsum(seg)[:-1]]) if seg.size else np.zeros(0)
    total = int(seg.sum())
    if total > 0xFFFFFFFF:
        raise ValueError("more than 2^32 ADE poles")
    return MaterialTables(table=rec, index=np.ascontiguousarray(index), n_mat=n_mat,
                          set_ofs=set_ofs, coef=np.ascontiguousarray(coef),
                          seg_ofs=seg_ofs.astype(np.uint32), n_pole_total=total,
                          ca=tuple(ca), cb=tuple(cb))


# ---------------------------------------------------------------------------------------------
# Sources
# ---------------------------------------------------------------------------------------------

def plane_sources(sc):
    """Plane-wave groups (one per polarisation) with the coefficients of
    ``openem/sources_setup.py:93-119``."""
    if not sc.sources:
        return []
    az = sc.grid.axes[2]
    for s in sc.sources:
        if s.axis != 2 or s.pol_axis not in (0, 1):
            raise NotImplementedError("plane waves: propagation along z with Ex/Ey polarisation only")
        if getattr(s, "angle_theta", 0.0):
            raise NotImplementedError("oblique plane waves need the Bloch path")
    keys = {(int(s.plane_index), int(s.direction)) for s in sc.sources}
    if len(keys) != 1:
        raise NotImplementedError("plane-wave sources must share one plane and one direction")
    groups = {}
    for s in sc.sources:
        groups.setdefault(int(s.pol_axis), []).append(s)
    out = []
    for pol, grp in sorted(groups.items()):
        s0 = grp[0]
        ks = int(s0.plane_index)
        kh = ks - 1 if s0.direction > 0 else ks
        sh, se = PLANE_SIGNS[int(s0.direction)]
        sp = -1.0 if pol == 1 else 1.0
        out.append({
            "pol": pol, "kh": kh, "ks": ks,
            "coef_h": float(np.float32(sp * sh * sc.dt / MU_0 * float(1.0 / az.dl[kh]))),
            "coef_e": float(np.float32(se * float(1.0 / az.dl_dual[ks]))),
            "ex": np.ascontiguousarray(sum(np.asarray(x.ex_inc, np.float64) for x in grp)),
            "hy": np.ascontiguousarray(sum(np.asarray(x.hy_inc, np.float64) for x in grp)),
        })
    return out


def dipole_tables(sc, n_total: int, magnetic: bool, complex_amp: bool = False):
    """Flattened stencils of the electric (half-step table) or magnetic (whole-step table)
    dipoles (openem/sources_setup.py:419-470). ``complex_amp`` takes the complex analytic
    amplitude of a Bloch run: ``amp`` then holds its real and ``amp_im`` its imaginary part."""
    dips = [d for d in sc.dipoles if bool(d.magnetic) == magnetic]
    if not dips:
        return None
    if complex_amp:
        ctabs = [np.asarray(d.waveform.amp_int_complex if magnetic
                            else d.waveform.amp_half_complex, np.complex128) for d in dips]
        tabs = [np.real(t) for t in ctabs]
    else:
        tabs = [np.asarray(d.waveform.amp_int if magnetic else d.waveform.amp_half, np.float64)
                for d in dips]
    nsteps1 = min(t.size for t in tabs)
    if n_total > nsteps1 - 1:
        raise ValueError(f"asked to run {n_total} steps, but the dipole waveform only sampled "
                         f"{nsteps1} points")
    ijk, comp, coef, src = [], [], [], []
    for s, d in enumerate(dips):
        ind = np.asarray(d.indices, dtype=np.int64).reshape(-1, 3)
        cf = np.asarray(d.coef, dtype=np.float64).ravel()
        ijk.append(ind)
        comp.append(np.full(len(ind), int(d.component), np.int32))
        coef.append(cf.astype(np.float32))
        src.append(np.full(len(ind), s, np.int32))
    out = {"ijk": np.ascontiguousarray(np.concatenate(ijk).astype(np.int32)),
           "comp": np.concatenate(comp), "coef": np.concatenate(coef), "src": np.concatenate(src),
           "n_src": len(dips), "nsteps1": nsteps1,
           "amp": np.ascontiguousarray(np.stack([t[:nsteps1] for t in tabs]))}
    if complex_amp:
        out["amp_im"] = np.ascontiguousarray(np.stack([np.imag(t[:nsteps1]) for t in ctabs]))
    return out


# one-plane TF/SF signs of a mode source per direction: (H_t1, H_t2, E_t1, E_t2)
# (openem/sources_setup.py:51-54)
MODE_SIGNS = {+1: (-1.0, +1.0, +1.0, -1.0), -1: (+1.0, -1.0, +1.0, -1.0)}


def mode_tables(sc, n_total: int) -> list:
    """One injection entry per mode source (openem/sources_setup.py:376-416): planes, the
    four float32 coefficients, the (n_terms, 8, n_t1, n_t2) float32 profiles (E_t1, E_t2, H_t1,
    H_t2 as re/im planes; base term then broadband corrections) and the (n_terms, ntab, 2)
    float64 amplitude tables. Sources are injected one entry each: the injection is linear, so
    the sum over entries is the superposition OpenEM forms by merging same-face sources."""
    out = []
    for m in getattr(sc, "mode_sources", None) or []:
        a = int(m.axis)
        ax = sc.grid.axes[a]
        ks = int(m.plane_index)
        kh = ks - 1 if int(m.direction) > 0 else ks
        s_h1, s_h2, s_e1, s_e2 = MODE_SIGNS[int(m.direction)]
        ch = sc.dt / MU_0 * float(1.0 / ax.dl[kh])
        ce = float(1.0 / ax.dl_dual[ks])
        terms = [(m.ey_inc, m.ez_inc, m.hy_inc, m.hz_inc, m.amp_e, m.amp_h)]
        for k in range(0 if m.bb_ey is None else len(m.bb_ey)):
            terms.append((m.bb_ey[k], m.bb_ez[k], m.bb_hy[k], m.bb_hz[k], m.bb_amp_e[k],
                          m.bb_amp_h[k]))
        t1, t2 = (a + 1) % 3, (a + 2) % 3
        n1, n2 = int(sc.shape[t1]), int(sc.shape[t2])
        ntab = min(min(np.size(t[4]), np.size(t[5])) for t in terms)
        if n_total > ntab:
            raise ValueError(f"asked to run {n_total} steps, but the mode amplitude tables hold "
                             f"{ntab} samples")
        prof = np.empty((len(terms), 8, n1, n2), np.float32)
        amp_e = np.empty((len(terms), ntab, 2), np.float64)
        amp_h = np.empty((len(terms), ntab, 2), np.float64)
        for q, (e1, e2, h1, h2, ae, ah) in enumerate(terms):
            for r, pr in enumerate((e1, e2, h1, h2)):
                pr = np.asarray(pr, np.complex128)
                if pr.shape != (n1, n2):
                    raise ValueError(f"mode profile shape {pr.shape} != plane {(n1, n2)}")
                prof[q, 2 * r] = pr.real
                prof[q, 2 * r + 1] = pr.imag
            ae = np.asarray(ae, np.complex128)[:ntab]
            ah = np.asarray(ah, np.complex128)[:ntab]
            amp_e[q, :, 0], amp_e[q, :, 1] = ae.real, ae.imag
            amp_h[q, :, 0], amp_h[q, :, 1] = ah.real, ah.imag
        out.append({"axis": a, "kh": kh, "ks": ks, "n1": n1, "n2": n2,
                    "coef_h": (float(np.float32(s_h1 * ch)), float(np.float32(s_h2 * ch))),
                    "coef_e": (float(np.float32(s_e1 * ce)), float(np.float32(s_e2 * ce))),
                    "prof": prof, "amp_e": amp_e, "amp_h": amp_h, "ntab": int(ntab)})
    return out


# ---------------------------------------------------------------------------------------------
# Monitors
# ---------------------------------------------------------------------------------------------

def phase_table(freqs, dt: float, n_total: int, apod=None) -> np.ndarray:
    """(n_total, nf, 4) float32: cos/sin of 2 pi f t at E time (n+1) dt and H time (n+1/2) dt,
    each multiplied by its apodisation window (openem/kernels/source_dft.cu:332-362)."""
    f = np.asarray(freqs, dtype=np.float64)
    n = np.arange(n_total, dtype=np.float64)
    te, th = (n + 1.0) * dt, (n + 0.5) * dt
    we, wh = apod_window(te, apod), apod_window(th, apod)
    ae = 2.0 * np.pi * f[None, :] * te[:, None]
    ah = 2.0 * np.pi * f[None, :] * th[:, None]
    out = np.empty((n_total, f.size, 4), dtype=np.float32)
    out[..., 0] = np.cos(ae) * we[:, None]
    out[..., 1] = np.sin(ae) * we[:, None]
    out[..., 2] = np.cos(ah) * wh[:, None]
    out[..., 3] = np.sin(ah) * wh[:, None]
    return out


def batch_depth(points: int, ncomp: int, cap: int = 32, ring_bytes: float = 2e9) -> int:
    """Snapshot ring depth: up to 32 steps, halved while the ring would exceed ``ring_bytes``."""
    T = cap
    while T > 1 and T * ncomp * 4 * points > ring_bytes:
        T //= 2
    return max(T, 1)


def modulation_tables(sc, tabs, n_total: int) -> dict | None:
    """Per-entry tables of a time-modulated permittivity and the per-step (cos, sin) of the
    modulation phase at t_n and t_n+1, computed in float64 and narrowed to float32
    (``openem/sources_setup.py:460-518, 640-650``). Entries whose static ``cb`` is zero (the
    tangential E on a PEC-backed wall, which OpenEM masks after the update) are dropped: their
    coefficients stay zero."""
    mo = sc.modulation
    if mo is None or mo.n_entry == 0:
        return None
    mo.validate(sc.shape)
    if sc.any_pec or (sc.dispersion_mix is not None and sc.dispersion_mix.n_entry > 0) \
            or (sc.tensor is not None and sc.tensor.n_entry > 0):
        raise NotImplementedError(
            "a time-varying medium together with PEC/mix/tensor in one scene is not supported")
    comp = np.asarray(mo.comp, np.int64)
    cell = np.asarray(mo.cell, np.int64)
    amp = np.asarray(mo.amp, np.float64)
    phase = np.asarray(mo.phase, np.float64)
    es = np.empty(comp.size)
    sd = np.zeros(comp.size)
    gg = np.zeros(comp.size)
    sig = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
    g_maps = _g_dense(sc, sc.shape)
    for c, eps in enumerate((sc.eps_ex, sc.eps_ey, sc.eps_ez)):
        m = comp == c
        es[m] = np.asarray(eps, np.float64).ravel()[cell[m]]
        if sig[c] is not None:
            sd[m] = np.asarray(sig[c], np.float64).ravel()[cell[m]] * sc.dt / (2.0 * EPSILON_0)
        gg[m] = np.asarray(g_maps[c]).ravel()[cell[m]]
    if float(np.min(es - np.abs(amp))) <= 0.0:
        raise ValueError(f"modulated cells: min of eps_s - |amp| is "
                         f"{float(np.min(es - np.abs(amp))):.4f} <= 0, so eps(t) would go "
                         "non-positive, which is unstable")
    _, cb = e_coefficients(sc, tabs)
    keep = np.ones(comp.size, bool)
    for c in range(3):
        m = comp == c
        keep[m] = cb[c].ravel()[cell[m]] != 0.0
    om = 2.0 * np.pi * float(mo.freq)
    t = np.arange(n_total, dtype=np.float64)
    w0, w1 = om * (t * sc.dt), om * ((t + 1.0) * sc.dt)
    cs = np.ascontiguousarray(np.stack([np.cos(w0), np.sin(w0), np.cos(w1), np.sin(w1)],
                                       axis=1).astype(np.float32))
    f32 = lambda a: np.ascontiguousarray(a[keep], dtype=np.float32)
    return {"comp": np.ascontiguousarray(comp[keep], np.int32),
            "cell": np.ascontiguousarray(cell[keep], np.int64),
            "amp": f32(amp), "cph": f32(np.cos(phase)), "sph": f32(np.sin(phase)),
            "eps": f32(es), "sd": f32(sd), "gg": f32(gg), "cs": cs,
            "dte": float(sc.dt / EPSILON_0)}


def isolate_cells(table, index, cells):
    """Give each listed cell its own copy of its material record, appended after the existing
    ones: the per-step modulation kernel rewrites a modulated cell's record in place, so no other
    cell may share it. Returns the new table, index and record count."""
    cells = np.unique(np.asarray(cells, np.int64))
    flat = np.asarray(index).reshape(-1)
    n0 = int(table.shape[0])
    table = np.concatenate([table, table[flat[cells].astype(np.int64)]])
    n_mat = int(table.shape[0])
    out = flat.astype(np.uint16 if n_mat <= 65535 else np.uint32)
    out[cells] = n0 + np.arange(cells.size)
    return table, np.ascontiguousarray(out.reshape(np.asarray(index).shape)), n_mat


def absorber_tables(sc) -> list:
    """Absorber slabs in scene order: ``(axis, g0, nlay, decay_int, decay_half)``
    (openem/dispersion_setup.py:89-120)."""
    out = []
    for sl in getattr(sc, "absorbers", None) or []:
        sl.validate()
        di = np.asarray(sl.decay_int, np.float64)
        dh = np.asarray(sl.decay_half, np.float64)
        if di.size != dh.size:
            raise ValueError("absorber decay profiles differ in length")
        out.append((int(sl.axis), int(sl.g0), int(di.size), di, dh))
    return out


def dispersion_in_absorbers(sc) -> bool:
    """True when a dispersive (component, cell) entry, of the E form or of the mixed form, lies
    inside an absorber's layers."""
    if not getattr(sc, "absorbers", None):
        return False
    for d in (sc.dispersion, sc.dispersion_mix):
        if d is None or d.n_entry == 0:
            continue
        cells = np.asarray(d.cell, dtype=np.int64)
        ijk = np.unravel_index(cells, tuple(int(v) for v in sc.shape))
        for sl in sc.absorbers:
            q = ijk[int(sl.axis)]
            if np.any((q >= int(sl.g0)) & (q < int(sl.g0) + np.size(sl.decay_int))):
                return True
    return False
