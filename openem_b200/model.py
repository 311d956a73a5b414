"""Input contract of the step engine: the numpy ``Scene`` and everything it holds.

The class and field names are the ones OpenEM's own data model uses (``openem/model.py:22-927``,
``openem/grid.py:138-383``, ``openem/cpml.py:36-164``, ``openem/waveform.py:19-44``), because the
engine is a drop-in for OpenEM's step loop: a ``Scene`` built by OpenEM's scene builder, or loaded
from its ``scene.npz``, must be accepted unchanged. The solver only reads attributes, so objects of
OpenEM's own classes work too (duck typing); these classes exist so that the engine, its tests
and its benchmark run on a machine where OpenEM is not installed.

Only numpy is imported here.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# SI constants, the values OpenEM's CPML module uses (openem/cpml.py:28-31).
EPSILON_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6
ETA_0 = 376.7303136668535
C_0 = 299792458.0

#: Component order of the six field arrays (openem/model.py:265).
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

#: Boundary types whose low end is absorbing (PEC-backed) rather than wrapping.
_PERIODIC = ("Periodic", "BlochBoundary")


# ---------------------------------------------------------------------------
# Grid (openem/grid.py:138-383)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class Axis:
    """One axis of the Yee grid: primal cell edges in metres and the two boundary types."""

    edges: np.ndarray
    boundary_lo: str
    boundary_hi: str
    flat: bool | None = None

    def __post_init__(self) -> None:
        e = np.asarray(self.edges, dtype=np.float64)
        if e.ndim != 1 or e.size < 2 or not np.all(np.diff(e) > 0):
            raise ValueError("edges must be a strictly increasing 1D array of length >= 2")

    @property
    def n(self) -> int:
        return int(np.asarray(self.edges).size - 1)

    @property
    def dl(self) -> np.ndarray:
        """Primal spacing, divides the H-update differences."""
        return np.diff(np.asarray(self.edges, dtype=np.float64))

    @property
    def is_periodic(self) -> bool:
        return self.boundary_lo in _PERIODIC

    @property
    def is_flat(self) -> bool:
        return bool(self.flat) if self.flat is not None else self.n == 1

    @property
    def dl_dual(self) -> np.ndarray:
        """Dual spacing ``(dl[i] + dl[i-1]) / 2``; the cell before 0 wraps on a periodic axis
        and mirrors ``dl[0]`` otherwise (openem/grid.py:198-212)."""
        dl = self.dl
        prev = np.concatenate([[dl[-1] if self.is_periodic else dl[0]], dl[:-1]])
        return 0.5 * (dl + prev)

    @property
    def centers(self) -> np.ndarray:
        e = np.asarray(self.edges, dtype=np.float64)
        return 0.5 * (e[:-1] + e[1:])

    def index_tables(self, bloch_k: float = 0.0) -> dict:
        """Neighbour indices and multiplicative masks that encode the boundary topology
        (openem/grid.py:219-304): ``nxt/prv`` wrap on a periodic axis and clamp otherwise,
        ``mnx/mpv`` zero a neighbour that does not exist (or carry the Bloch phase at the
        seam), and ``pec`` zeroes tangential E on the PEC-backed low wall."""
        n = self.n
        i = np.arange(n)
        if self.is_periodic:
            mnx = np.ones(n)
            mpv = np.ones(n)
            if bloch_k != 0.0:
                mnx = mnx.astype(np.complex128)
                mpv = mpv.astype(np.complex128)
                mnx[n - 1] = np.exp(2j * np.pi * bloch_k)
                mpv[0] = np.exp(-2j * np.pi * bloch_k)
            return {"nxt": ((i + 1) % n).astype(np.int32), "prv": ((i - 1) % n).astype(np.int32),
                    "mnx": mnx, "mpv": mpv, "pec": np.ones(n)}
        if bloch_k != 0.0:
            raise ValueError(f"bloch_k={bloch_k:g} needs a periodic axis, this one is "
                             f"{self.boundary_lo}/{self.boundary_hi}")
        pec = np.ones(n)
        mpv = (i > 0).astype(np.float64)
        lo, hi = self.boundary_lo, self.boundary_hi
        if lo == "PMCBoundary":
            mpv[0] = -1.0
        elif lo in ("SymmetryPEC", "SymmetryPMC"):
            s = -1.0 if lo == "SymmetryPEC" else 1.0
            mpv[0] = -s
            if s < 0:
                pec[0] = 0.0
        else:
            pec[0] = 0.0
        nxt = np.minimum(i + 1, n - 1).astype(np.int32)
        mnx = (i + 1 < n).astype(np.float64)
        if hi == "PMCBoundary":
            mnx[n - 1] = 1.0
        elif hi in ("SymmetryPEC", "SymmetryPMC"):
            s = -1.0 if hi == "SymmetryPEC" else 1.0
            nxt[n - 1] = n - 2
            mnx[n - 1] = s
            if s < 0:
                pec[n - 1] = 0.0
        return {"nxt": nxt, "prv": np.maximum(i - 1, 0).astype(np.int32),
                "mnx": mnx, "mpv": mpv, "pec": pec}


@dataclass(frozen=True)
class Grid:
    x: Axis
    y: Axis
    z: Axis

    @property
    def axes(self) -> tuple[Axis, Axis, Axis]:
        return (self.x, self.y, self.z)

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.x.n, self.y.n, self.z.n)

    @property
    def num_cells(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    def yee_dual_volumes(self):
        """Dual volume of Ex/Ey/Ez at their own Yee positions (openem/grid.py:350-366)."""
        xp, yp, zp = (a.dl for a in self.axes)
        xd, yd, zd = (a.dl_dual for a in self.axes)
        o = lambda a, b, c: a[:, None, None] * b[None, :, None] * c[None, None, :]
        return o(xp, yd, zd), o(xd, yp, zd), o(xd, yd, zp)

    def yee_h_dual_volumes(self):
        xp, yp, zp = (a.dl for a in self.axes)
        xd, yd, zd = (a.dl_dual for a in self.axes)
        o = lambda a, b, c: a[:, None, None] * b[None, :, None] * c[None, None, :]
        return o(xd, yp, zp), o(xp, yd, zp), o(xp, yp, zd)


def ravel_cells(ii, jj, kk, shape):
    """Flat cell index ``(i*ny + j)*nz + k``."""
    ny, nz = int(shape[-2]), int(shape[-1])
    return (ii * ny + jj) * nz + kk


def unravel_cells(cell, shape):
    ny, nz = int(shape[-2]), int(shape[-1])
    return cell // (ny * nz), (cell // nz) % ny, cell % nz


# ---------------------------------------------------------------------------
# CPML (openem/cpml.py:36-164, Tidy3D's profile definition)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class PMLParams:
    num_layers: int
    sigma_min: float = 0.0
    sigma_max: float = 1.5
    sigma_order: int = 3
    kappa_min: float = 1.0
    kappa_max: float = 3.0
    kappa_order: int = 3
    alpha_min: float = 0.0
    alpha_max: float = 0.0
    alpha_order: int = 1


@dataclass(frozen=True)
class PMLCoeffs:
    """Per-layer recursion coefficients of one PML face, E and H positions."""

    a_E: np.ndarray
    b_E: np.ndarray
    inv_kappa_E: np.ndarray
    a_H: np.ndarray
    b_H: np.ndarray
    inv_kappa_H: np.ndarray

    @property
    def num_layers(self) -> int:
        return int(np.asarray(self.a_E).size)


def pml_depth(n: int, side: str, at: str) -> np.ndarray:
    """Normalised depth of each layer in increasing global index order. E positions sit on the
    backward-difference points, H positions half a cell further out (openem/cpml.py:55-76)."""
    if n <= 0:
        return np.zeros(0)
    i = np.arange(n, dtype=np.float64)
    if side == "lo":
        return (n - i) / n if at == "E" else (n - i - 0.5) / n
    return i / n if at == "E" else (i + 0.5) / n


def pml_build(params: PMLParams, dl: float, side: str, dt: float,
              avg_speed: float = 1.0) -> PMLCoeffs:
    """Graded sigma/kappa/alpha profile -> Roden-Gedney recursion coefficients ``(a, b, 1/k)``:
    ``b = exp(-dt/eps0 (sigma/kappa + alpha))``, ``a = (b-1) sigma / (sigma + alpha kappa) / kappa``
    (openem/cpml.py:79-164)."""
    if params.sigma_min:
        raise NotImplementedError("sigma_min != 0 has no defined grading")
    out = {}
    for at in ("E", "H"):
        s = pml_depth(params.num_layers, side, at)
        sigma = params.sigma_max * avg_speed / (ETA_0 * dl) * s ** params.sigma_order
        kappa = params.kappa_min + (params.kappa_max - params.kappa_min) * s ** params.kappa_order
        alpha = params.alpha_min + (params.alpha_max - params.alpha_min) * s ** params.alpha_order
        b = np.exp(-dt / EPSILON_0 * (sigma / kappa + alpha))
        with np.errstate(divide="ignore", invalid="ignore"):
            a = (b - 1.0) * sigma / (sigma + alpha * kappa) / kappa
        out[f"a_{at}"] = np.nan_to_num(a, nan=0.0, posinf=0.0, neginf=0.0)
        out[f"b_{at}"] = b
        out[f"inv_kappa_{at}"] = 1.0 / kappa
    return PMLCoeffs(**out)


# ---------------------------------------------------------------------------
# Waveforms (openem/waveform.py)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class Waveform:
    """Pre-sampled source amplitude at whole steps ``n dt`` and half steps ``(n+1/2) dt``."""

    amp_int: np.ndarray
    amp_half: np.ndarray
    amp_int_complex: np.ndarray
    dt: float
    amp_half_complex: np.ndarray | None = None

    @property
    def num_steps(self) -> int:
        return int(np.asarray(self.amp_int).size - 1)


@dataclass(frozen=True)
class GaussianPulse:
    """Tidy3D's ``GaussianPulse`` source time, restated from its published definition:
    complex analytic amplitude
    ``a(t) = A e^{i phase} e^{-i w0 t} e^{-(t - t0)^2 / (2 tw^2)} * (i + (t - t0) / (tw^2 w0))``
    with ``tw = 1 / (2 pi fwidth)``, ``t0 = offset tw`` and ``w0 = 2 pi freq0`` (the last factor is
    the DC-removal term; without DC removal it is ``i``). Tidy3D itself is not a dependency."""

    freq0: float
    fwidth: float
    amplitude: float = 1.0
    phase: float = 0.0
    offset: float = 5.0
    remove_dc_component: bool = True

    @property
    def twidth(self) -> float:
        return 1.0 / (2.0 * np.pi * self.fwidth)

    def amp_time(self, t) -> np.ndarray:
        t = np.asarray(t, dtype=np.float64)
        w0 = 2.0 * np.pi * self.freq0
        tw = self.twidth
        ts = t - self.offset * tw
        env = self.amplitude * np.exp(-ts * ts / (2.0 * tw * tw))
        a = np.exp(1j * self.phase) * np.exp(-1j * w0 * t) * env
        if self.remove_dc_component:
            return a * (1j + ts / (tw * tw * w0))
        return a * 1j

    def end_time(self) -> float:
        return 2.0 * self.offset * self.twidth


def sample_waveform(source_time, dt: float, num_steps: int) -> Waveform:
    """Tabulate ``source_time.amp_time`` at ``n dt`` and ``(n+1/2) dt`` for n = 0..num_steps
    (openem/waveform.py:49-66)."""
    n = np.arange(num_steps + 1, dtype=np.float64)
    a_int = np.asarray(source_time.amp_time(n * dt))
    a_half = np.asarray(source_time.amp_time((n + 0.5) * dt))
    return Waveform(amp_int=np.real(a_int).astype(np.float64),
                    amp_half=np.real(a_half).astype(np.float64),
                    amp_int_complex=a_int.astype(np.complex128), dt=dt,
                    amp_half_complex=a_half.astype(np.complex128))


# ---------------------------------------------------------------------------
# Sources (openem/model.py:22-229)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class PlaneWaveSource:
    axis: int
    plane_index: int
    direction: int
    pol_axis: int
    waveform: Waveform
    angle_theta: float
    num_freqs: int
    ex_inc: np.ndarray
    hy_inc: np.ndarray
    incident: dict | None = None
    center: float = float("nan")


@dataclass(frozen=True)
class TFSFSource:
    direction: int
    box_lo: tuple
    box_hi: tuple
    dl1: np.ndarray
    eps1: np.ndarray
    inj: int
    col0: int
    ex_inc: np.ndarray
    hy_inc: np.ndarray
    waveform: Waveform
    num_freqs: int = 1
    axis: int = 2
    pol_u: float = 1.0
    pol_v: float = 0.0
    sigma1: np.ndarray | None = None
    k_hat: tuple | None = None
    e_hat: tuple | None = None
    dl1_step: float = 0.0
    proj0: float = 0.0
    n_col_e: int = 0
    open_axes: tuple = ()
    amp_scale: float = 1.0


@dataclass(frozen=True)
class ModeSource:
    plane_index: int
    direction: int
    ey_inc: np.ndarray
    ez_inc: np.ndarray
    hy_inc: np.ndarray
    hz_inc: np.ndarray
    amp_e: np.ndarray
    amp_h: np.ndarray
    n_eff: complex
    axis: int = 0
    bb_ey: np.ndarray | None = None
    bb_ez: np.ndarray | None = None
    bb_hy: np.ndarray | None = None
    bb_hz: np.ndarray | None = None
    bb_amp_e: np.ndarray | None = None
    bb_amp_h: np.ndarray | None = None


@dataclass(frozen=True)
class PointDipole:
    """Current moment spread on Yee points: ``indices (nw, 3)``, ``coef (nw,) = weight / dV``."""

    component: int
    indices: np.ndarray
    coef: np.ndarray
    waveform: Waveform
    magnetic: bool = False


# ---------------------------------------------------------------------------
# Monitors (openem/model.py:231-419)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class FieldMonitor:
    name: str
    freqs: np.ndarray
    origin: tuple
    box: tuple
    apodization: tuple | None = None
    interval_space: tuple = (1, 1, 1)


@dataclass(frozen=True)
class FieldTimeMonitor:
    name: str
    comps: tuple
    origin: tuple
    box: tuple
    step_begin: int
    step_end: int
    interval: int
    num_slots: int

    def slot_of(self, m: int) -> int | None:
        if m < self.step_begin or m >= self.step_end:
            return None
        off = m - self.step_begin
        if off % self.interval:
            return None
        s = off // self.interval
        return s if s < self.num_slots else None


@dataclass(frozen=True)
class FluxTimeMonitor:
    name: str
    axis: int
    plane_index: int
    normal_dir: int
    step_begin: int
    step_end: int
    interval: int
    num_slots: int
    t_bounds: tuple = ((0.0, 0.0), (0.0, 0.0))
    frac: float = 0.0


@dataclass(frozen=True)
class PermittivityMonitor:
    name: str
    freqs: np.ndarray
    origin: tuple
    box: tuple


@dataclass(frozen=True)
class FluxMonitor:
    name: str
    axis: int
    plane_index: int
    normal_dir: int
    freqs: np.ndarray
    source_spectrum: np.ndarray
    transverse: tuple | None = None
    apodization: tuple | None = None
    t_bounds: tuple | None = None


@dataclass(frozen=True)
class ModeMonitorSpec:
    name: str
    plane_name: str


@dataclass(frozen=True)
class BoxFluxMonitor:
    name: str
    face_names: tuple


@dataclass(frozen=True)
class ProjectionMonitor:
    name: str
    surface_names: tuple
    normal_dirs: tuple


# ---------------------------------------------------------------------------
# Media tables (openem/model.py:421-800)
# ---------------------------------------------------------------------------

def check_csr(name: str, shape, comp, cell, ofs_list) -> np.ndarray:
    """Shape, range, monotone-offset and (comp, cell)-uniqueness checks of an entry table
    (openem/model.py:421-458). Returns the joint key ``comp * ncell + cell``."""
    comp = np.asarray(comp)
    cell = np.asarray(cell)
    n = int(comp.size)
    ncell = int(np.prod(shape))
    if comp.shape != (n,) or cell.shape != (n,):
        raise ValueError(f"{name}: comp/cell lengths differ")
    if n == 0:
        return np.zeros(0, dtype=np.int64)
    if comp.min() < 0 or comp.max() > 2:
        raise ValueError(f"{name}: comp out of range {comp.min()}..{comp.max()}")
    if cell.min() < 0 or cell.max() >= ncell:
        raise ValueError(f"{name}: cell out of range {cell.max()} >= {ncell}")
    for oname, ofs, npole in ofs_list:
        ofs = np.asarray(ofs)
        if ofs.shape != (n + 1,):
            raise ValueError(f"{name}.{oname} has shape {ofs.shape}, expected ({n + 1},)")
        if ofs[0] != 0 or ofs[-1] != npole:
            raise ValueError(f"{name}.{oname} endpoints {ofs[0]}..{ofs[-1]}, expected 0..{npole}")
        if np.any(np.diff(ofs) < 0):
            raise ValueError(f"{name}.{oname} is not monotonic")
    key = comp.astype(np.int64) * ncell + cell.astype(np.int64)
    if n < 2 or bool(np.all(key[1:] > key[:-1])):  # tables ordered by (comp, cell): unique
        return key
    seen = np.zeros(3 * ncell, dtype=bool)
    seen[key] = True
    nu = int(np.count_nonzero(seen))
    if nu != n:
        raise ValueError(f"{name}: {n - nu} duplicate (comp, cell) entries")
    return key


@dataclass(frozen=True)
class Dispersion:
    """Pole-residue ADE entries in CSR form: entry ``e`` owns poles ``pole_ofs[e]:pole_ofs[e+1]``;
    ``am1 = A - 1`` and ``b = B`` are the trapezoidal coefficients of ``dP/dt = qP + rE``;
    ``g = sum 2 Re(B)`` per entry (openem/model.py:461-526)."""

    comp: np.ndarray
    cell: np.ndarray
    pole_ofs: np.ndarray
    am1: np.ndarray
    b: np.ndarray
    g: np.ndarray

    @property
    def n_entry(self) -> int:
        return int(np.asarray(self.comp).size)

    @property
    def n_pole(self) -> int:
        return int(np.asarray(self.am1).size)

    def validate_shapes(self) -> None:
        n = self.n_entry
        for nm, arr, want in (("g", self.g, n), ("am1", self.am1, self.n_pole),
                              ("b", self.b, self.n_pole)):
            if np.asarray(arr).shape != (want,):
                raise ValueError(f"Dispersion.{nm} has shape {np.asarray(arr).shape}, "
                                 f"expected ({want},)")

    def validate(self, shape) -> None:
        self.validate_shapes()
        check_csr("Dispersion", shape, self.comp, self.cell,
                  [("pole_ofs", self.pole_ofs, self.n_pole)])

    def g_dense(self, shape):
        out = [np.zeros(int(np.prod(shape)), dtype=np.float64) for _ in range(3)]
        comp = np.asarray(self.comp)
        for c in range(3):
            m = comp == c
            out[c][np.asarray(self.cell)[m]] = np.asarray(self.g)[m]
        return tuple(o.reshape(shape) for o in out)


@dataclass(frozen=True)
class DispersionMix:
    """Slanted-interface cells (openem/model.py:529-612, openem/kernels/dispersion_mix.cu):
    eps_eff = (1 - beta) sum f_i eps_i + beta / sum (f_i / eps_i), beta the squared normal
    projection on the entry's component. The arithmetic branch carries poles of eps (``p_ofs``,
    ``pa = A - 1``, ``pb = B``, conjugate pairs counted by 2 Re), the harmonic branch poles of
    1/eps (``q_ofs``, ``qa``, ``qb``, every root listed, counted by Re) driven by its own
    unknown d_h = D_h / eps0; per step one scalar linear equation gives d_h^{n+1} and E^{n+1}.
    beta = 0 is the E form of :class:`Dispersion`, beta = 1 the pure harmonic (D) form."""

    comp: np.ndarray
    cell: np.ndarray
    p_ofs: np.ndarray
    pa: np.ndarray
    pb: np.ndarray
    q_ofs: np.ndarray
    qa: np.ndarray
    qb: np.ndarray
    beta: np.ndarray
    eps_inf: np.ndarray
    zeta_inf: np.ndarray

    @property
    def n_entry(self) -> int:
        return int(np.asarray(self.comp).size)

    def coefficients(self):
        """Per entry ``(k1, k2, 1 - beta, 1 / (k1 k2 + beta))`` in float64 with
        k1 = (1 - beta)(eps_inf + sum 2 Re(pb)) and k2 = zeta_inf + sum Re(qb): the implicit
        couplings of the two branches to step n+1."""
        n = self.n_entry
        beta = np.asarray(self.beta, np.float64)

        def seg_sum(ofs, vals):
            ofs = np.asarray(ofs, np.int64)
            out = np.zeros(n)
            cnt = np.diff(ofs)
            if vals.size:
                np.add.at(out, np.repeat(np.arange(n), cnt), vals)
            return out
        gp = seg_sum(self.p_ofs, 2.0 * np.asarray(self.pb, np.complex128).real)
        gq = seg_sum(self.q_ofs, np.asarray(self.qb, np.complex128).real)
        one_mb = 1.0 - beta
        k1 = one_mb * (np.asarray(self.eps_inf, np.float64) + gp)
        k2 = np.asarray(self.zeta_inf, np.float64) + gq
        den = k1 * k2 + beta
        if np.any(np.abs(den) < 1e-30):
            raise ValueError("mixed-cell denominator k1*k2 + beta is zero")
        return k1, k2, one_mb, 1.0 / den

    def validate(self, shape, *others) -> None:
        """Shapes, CSR offsets, (comp, cell) uniqueness, beta in [0, 1] (1e-6 slack), no entry
        shared with another dispersion table, a usable denominator."""
        n = self.n_entry
        for nm in ("beta", "eps_inf", "zeta_inf"):
            a = np.asarray(getattr(self, nm))
            if a.shape != (n,):
                raise ValueError(f"DispersionMix.{nm} has shape {a.shape}, expected ({n},)")
        for nm, ofs in (("pa", "p_ofs"), ("pb", "p_ofs"), ("qa", "q_ofs"), ("qb", "q_ofs")):
            a = np.asarray(getattr(self, nm))
            if a.ndim != 1:
                raise ValueError(f"DispersionMix.{nm} must be one-dimensional")
        if np.asarray(self.pa).size != np.asarray(self.pb).size or \
                np.asarray(self.qa).size != np.asarray(self.qb).size:
            raise ValueError("DispersionMix: pole coefficient lengths differ")
        key = check_csr("DispersionMix", shape, self.comp, self.cell,
                        [("p_ofs", self.p_ofs, int(np.asarray(self.pa).size)),
                         ("q_ofs", self.q_ofs, int(np.asarray(self.qa).size))])
        if n == 0:
            return
        beta = np.asarray(self.beta, np.float64)
        if np.any((beta < -1e-6) | (beta > 1.0 + 1e-6)):
            raise ValueError(f"beta outside [0,1]: {beta.min():.4f}..{beta.max():.4f} (the "
                             "squared normal projection; out of range means an unreliable fit)")
        ncell = int(np.prod(shape))
        for o in others:
            if o is None or o.n_entry == 0:
                continue
            ok = np.asarray(o.comp, np.int64) * ncell + np.asarray(o.cell, np.int64)
            if np.intersect1d(key, ok).size:
                raise ValueError("the same (comp, cell) appears in more than one dispersion table")
        self.coefficients()


@dataclass(frozen=True)
class TimeModulation:
    """``delta eps(t) = amp cos(2 pi freq t - phase)`` on the listed (comp, cell) entries."""

    freq: float
    comp: np.ndarray
    cell: np.ndarray
    amp: np.ndarray
    phase: np.ndarray

    @property
    def n_entry(self) -> int:
        return int(np.asarray(self.comp).size)

    def validate(self, shape) -> None:
        n = self.n_entry
        for nm, arr in (("amp", self.amp), ("phase", self.phase)):
            a = np.asarray(arr)
            if a.shape != (n,):
                raise ValueError(f"TimeModulation.{nm} has shape {a.shape}, expected ({n},)")
            if not np.all(np.isfinite(a)):
                raise ValueError(f"TimeModulation.{nm} contains non-finite values")
        if not (self.freq > 0):
            raise ValueError(f"TimeModulation.freq = {self.freq}, must be positive")
        check_csr("TimeModulation", shape, self.comp, self.cell, [])


@dataclass(frozen=True)
class TensorEps:
    """Fully anisotropic cells (openem/model.py:674-786): per (component, cell) entry the 3x3
    relative permittivity and conductivity at that component's Yee point. Entries with
    off-diagonal coupling read the other two components as 4-neighbour averages, so the table
    must be closed: every stencil point of a coupled entry is itself an entry (a ring of diagonal
    halo entries around the anisotropic region)."""

    comp: np.ndarray
    cell: np.ndarray
    eps: np.ndarray
    sigma: np.ndarray

    @property
    def n_entry(self) -> int:
        return int(np.asarray(self.comp).size)

    def rows(self, dt: float):
        """Row ``comp`` of M1 = A^-1 B and of M2 = (dt/eps0) A^-1, A = eps + s, B = eps - s,
        s = sigma dt / (2 eps0): the D-form update E^{n+1} = M1 E^n + M2 (curl H - J)."""
        s = np.asarray(self.sigma, np.float64) * (dt / (2.0 * EPSILON_0))
        eps = np.asarray(self.eps, np.float64)
        a_inv = np.linalg.inv(eps + s)
        m1 = a_inv @ (eps - s)
        m2 = (dt / EPSILON_0) * a_inv
        r = np.arange(self.n_entry)
        comp = np.asarray(self.comp)
        return m1[r, comp, :], m2[r, comp, :]

    def coupled_mask(self) -> np.ndarray:
        off = ~np.eye(3, dtype=bool)
        return ((np.abs(np.asarray(self.eps)[:, off]).max(axis=1) > 0.0)
                | (np.abs(np.asarray(self.sigma)[:, off]).max(axis=1) > 0.0))

    def validate(self, shape, tables=None) -> None:
        """Shapes, (comp, cell) uniqueness and, given the axis index tables, closure of the
        4-neighbour stencils (component b of a coupled entry of component a is read at the cell,
        one step forward along a and one step back along b)."""
        n = self.n_entry
        for name, arr in (("eps", self.eps), ("sigma", self.sigma)):
            if np.asarray(arr).shape != (n, 3, 3):
                raise ValueError(f"TensorEps.{name} has shape {np.asarray(arr).shape}, "
                                 f"expected ({n}, 3, 3)")
        key = check_csr("TensorEps", shape, self.comp, self.cell, [])
        if n == 0 or tables is None:
            return
        ncell = int(np.prod(shape))
        have = np.zeros(3 * ncell, dtype=bool)
        have[key] = True
        comp = np.asarray(self.comp)
        c = unravel_cells(np.asarray(self.cell), shape)
        eps, sig = np.asarray(self.eps), np.asarray(self.sigma)
        cpl = self.coupled_mask()
        missing = 0
        for a in range(3):
            for b in range(3):
                if a == b:
                    continue
                m = cpl & (comp == a) & ((np.abs(eps[:, a, b]) > 0) | (np.abs(sig[:, a, b]) > 0))
                if not m.any():
                    continue
                base = [np.asarray(c[w])[m] for w in range(3)]
                for fa in (False, True):
                    for fb in (False, True):
                        q = [x.copy() for x in base]
                        if fa:
                            q[a] = np.asarray(tables[a]["nxt"])[q[a]]
                        if fb:
                            q[b] = np.asarray(tables[b]["prv"])[q[b]]
                        flat = ravel_cells(q[0].astype(np.int64), q[1], q[2], shape)
                        missing += int((~have[b * ncell + flat]).sum())
        if missing:
            raise ValueError(f"TensorEps closure is broken: {missing} stencil points of coupled "
                             "entries are not entries themselves")


@dataclass(frozen=True)
class AbsorberSlab:
    """Graded absorber face: every step E and H in the layers are multiplied by the per-layer
    decay ``exp(-Gamma dt)`` (openem/model.py:770-799)."""

    axis: int
    g0: int
    decay_int: np.ndarray
    decay_half: np.ndarray

    def validate(self) -> None:
        for nm in ("decay_int", "decay_half"):
            d = np.asarray(getattr(self, nm))
            if d.ndim != 1 or not np.all((d > 0.0) & (d <= 1.0)):
                raise ValueError(f"AbsorberSlab.{nm} must be (nlay,) with factors in (0, 1]")


# ---------------------------------------------------------------------------
# Scene (openem/model.py:857-999)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class Scene:
    grid: Grid
    dt: float
    num_time_steps: int
    shutoff: float
    eps_ex: np.ndarray
    eps_ey: np.ndarray
    eps_ez: np.ndarray
    pml: dict
    sigma_ex: np.ndarray | None = None
    sigma_ey: np.ndarray | None = None
    sigma_ez: np.ndarray | None = None
    pec_ex: np.ndarray | None = None
    pec_ey: np.ndarray | None = None
    pec_ez: np.ndarray | None = None
    dispersion: Dispersion | None = None
    dispersion_mix: DispersionMix | None = None
    modulation: TimeModulation | None = None
    tensor: TensorEps | None = None
    symmetry: tuple = (0, 0, 0)
    bloch_k: tuple = (0.0, 0.0, 0.0)
    sources: list = field(default_factory=list)
    tfsf_sources: list = field(default_factory=list)
    dipoles: list = field(default_factory=list)
    mode_sources: list = field(default_factory=list)
    flux_monitors: list = field(default_factory=list)
    field_monitors: list = field(default_factory=list)
    field_time_monitors: list = field(default_factory=list)
    flux_time_monitors: list = field(default_factory=list)
    permittivity_monitors: list = field(default_factory=list)
    projection_monitors: list = field(default_factory=list)
    box_flux_monitors: list = field(default_factory=list)
    mode_monitors: list = field(default_factory=list)
    absorbers: list = field(default_factory=list)

    @property
    def shape(self):
        return self.grid.shape

    @property
    def any_dispersion(self) -> bool:
        return self.dispersion is not None and self.dispersion.n_entry > 0

    @property
    def any_dispersion_mix(self) -> bool:
        return self.dispersion_mix is not None and self.dispersion_mix.n_entry > 0

    @property
    def any_modulation(self) -> bool:
        return self.modulation is not None and self.modulation.n_entry > 0

    @property
    def any_tensor(self) -> bool:
        return self.tensor is not None and self.tensor.n_entry > 0

    @property
    def any_bloch(self) -> bool:
        return any(k != 0.0 for k in self.bloch_k)

    @property
    def any_loss(self) -> bool:
        return self.sigma_ex is not None

    @property
    def any_pec(self) -> bool:
        return self.pec_ex is not None
