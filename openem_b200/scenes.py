"""Synthetic ``Scene`` factory for the workloads the engine is measured and tested on.

Tidy3D is not available, so these builders do the part of OpenEM's scene builder
(``openem/scene/build.py:224``) that the workloads need, from first principles:

* uniform Yee grids with the 12-layer Tidy3D CPML added outside the simulation domain
  (``openem/cpml.py:149``), time step at a Courant factor of 0.99;
* staircased media: a component's cell takes the medium that contains its own Yee position;
* pole-residue media (Drude, Lorentz) reduced to trapezoidal ADE coefficients, with the DC pole
  of a Drude term moved onto the conductivity (``openem/scene/poles.py:157-188,284-296``);
* Gaussian-pulse waveforms sampled at whole and half steps, one-face plane-wave incident tables
  (``openem/scene/sources.py:19-83``), trilinear point-dipole stencils.

Every builder is deterministic for a given seed.
"""

from __future__ import annotations

import numpy as np

from openem_b200.model import (
    C_0, EPSILON_0, ETA_0, Axis, Dispersion, DispersionMix, FieldMonitor, FieldTimeMonitor, FluxMonitor,
    FluxTimeMonitor, GaussianPulse, Grid, ModeSource, PlaneWaveSource, PMLParams, PointDipole,
    Scene, TensorEps, TFSFSource, TimeModulation, pml_build, sample_waveform)

UM = 1e-6


def courant_dt(dls, courant: float = 0.99) -> float:
    """``dt = S / (c sqrt(sum 1/dl^2))`` with the smallest spacing on each axis."""
    inv = sum(1.0 / float(np.min(d)) ** 2 for d in dls)
    return courant / (C_0 * np.sqrt(inv))


def uniform_axis(n_cells: int, dl: float, lo: float, boundary: str, n_pml: int = 0) -> Axis:
    """``n_cells`` interior cells starting at ``lo`` (metres) plus ``n_pml`` layers at each end
    when the boundary is a PML."""
    extra = n_pml if boundary == "PML" else 0
    k = np.arange(-extra, n_cells + extra + 1, dtype=np.float64)
    return Axis(lo + k * dl, boundary, boundary)


def pml_dict(grid: Grid, dt: float, n_layers: int = 12) -> dict:
    """Tidy3D's default ``td.PML()`` coefficients on every PML face, graded with the end cell's
    spacing and vacuum speed."""
    params = PMLParams(num_layers=n_layers)
    out = {}
    for a, ax in enumerate(grid.axes):
        if ax.boundary_lo != "PML":
            continue
        dl = ax.dl
        out[(a, "lo")] = pml_build(params, float(dl[0]), "lo", dt)
        out[(a, "hi")] = pml_build(params, float(dl[-1]), "hi", dt)
    return out


def yee_coords(grid: Grid):
    """Per-component Yee coordinates ``(x, y, z)`` 1D arrays: Ex(ctr, edge, edge),
    Ey(edge, ctr, edge), Ez(edge, edge, ctr); H swaps edge and centre."""
    e = [np.asarray(a.edges[:-1], dtype=np.float64) for a in grid.axes]
    c = [a.centers for a in grid.axes]
    on_edge = {0: (False, True, True), 1: (True, False, True), 2: (True, True, False),
               3: (True, False, False), 4: (False, True, False), 5: (False, False, True)}
    return {k: tuple(e[a] if v[a] else c[a] for a in range(3)) for k, v in on_edge.items()}


def spectrum(source_time, dt: float, num_steps: int, freqs) -> np.ndarray:
    """Discrete source spectrum ``sum_n a(n dt) e^{i 2 pi f n dt} dt`` (stored with each flux
    monitor, used only by post-processing)."""
    t = np.arange(num_steps + 1, dtype=np.float64) * dt
    a = np.asarray(source_time.amp_time(t))
    f = np.asarray(freqs, dtype=np.float64)
    return (a[None, :] * np.exp(2j * np.pi * f[:, None] * t[None, :])).sum(axis=1) * dt


def plane_wave_tables(source_time, dt: float, num_steps: int, dl_half: float,
                      eps_r: float, direction: int = 1):
    """One-face TF/SF incident tables in a lossless medium: ``Ex_inc(n dt)`` on the source
    plane, and ``Hy_inc`` on the upstream Hy point sampled at ``(n+1/2) dt + dl_half / v``
    scaled by ``n / eta0`` (``openem/scene/sources.py:19-83``)."""
    n_r = np.sqrt(eps_r)
    v = C_0 / n_r
    n = np.arange(num_steps + 1, dtype=np.float64)
    ex_inc = np.real(np.asarray(source_time.amp_time(n * dt)))
    t_h = (n + 0.5) * dt + dl_half / v
    hy_inc = direction * np.real(np.asarray(source_time.amp_time(t_h)) * (n_r / ETA_0))
    return np.ascontiguousarray(ex_inc), np.ascontiguousarray(hy_inc)


# ---------------------------------------------------------------------------
# Pole-residue media
# ---------------------------------------------------------------------------

def drude_poles(wp: float, gamma: float):
    """Drude ``-wp^2 / (w^2 + i gamma w)`` as pole-residue pairs ``(a, c)`` in the convention
    ``chi(s) = sum c/(s-a) + c*/(s-a*)`` (s = -i w): a DC pole ``(0, wp^2/2gamma)`` and
    ``(-gamma, -wp^2/2gamma)``."""
    c = wp * wp / (2.0 * gamma)
    return [(0j, complex(c)), (complex(-gamma), complex(-c))]


def lorentz_poles(deps: float, f0: float, delta: float):
    """Lorentz ``deps f0^2 / (f0^2 - 2 i f delta - f^2)`` (Hz) as one pole-residue pair:
    ``a = -D + i wd``, ``c = -i deps w0^2 / (2 wd)`` with ``w0 = 2 pi f0``, ``D = 2 pi delta``,
    ``wd = sqrt(w0^2 - D^2)`` (underdamped)."""
    w0 = 2.0 * np.pi * f0
    d = 2.0 * np.pi * delta
    wd = np.sqrt(w0 * w0 - d * d)
    return [(complex(-d, wd), complex(0.0, -deps * w0 * w0 / (2.0 * wd)))]


def split_dc(poles, dt: float, rtol: float = 1e-9):
    """Move poles at ``a = 0`` onto a conductivity ``sigma = 2 Re(c) eps0``; return
    ``(remaining poles, sigma)`` (``openem/scene/poles.py:157-188``)."""
    keep, sigma = [], 0.0
    for a, c in poles:
        if abs(a) <= rtol / dt:
            sigma += 2.0 * c.real * EPSILON_0
        else:
            keep.append((complex(a), complex(c)))
    return keep, sigma


def trap_coeffs(poles, dt: float):
    """Trapezoidal ``(A - 1, B)`` of ``dP/dt = qP + rE``: ``A = (1 + q dt/2)/(1 - q dt/2)``,
    ``B = (r dt/2)/(1 - q dt/2)`` (``openem/scene/poles.py:284-296``)."""
    am1 = np.array([(1.0 + q * dt / 2.0) / (1.0 - q * dt / 2.0) - 1.0 for q, _ in poles],
                   dtype=np.complex128)
    b = np.array([(r * dt / 2.0) / (1.0 - q * dt / 2.0) for q, r in poles],
                 dtype=np.complex128)
    return am1, b


def build_dispersion(masks, am1, b, shape) -> Dispersion | None:
    """One entry per (component, cell) inside ``masks[c]``, every entry carrying the same
    poles; entries ordered by component then flat cell index."""
    comp, cell = [], []
    for c in range(3):
        idx = np.flatnonzero(masks[c].ravel())
        comp.append(np.full(idx.size, c, dtype=np.int32))
        cell.append(idx.astype(np.int32))
    comp = np.concatenate(comp)
    cell = np.concatenate(cell)
    n = comp.size
    if n == 0:
        return None
    p = am1.size
    g1 = float(np.sum(2.0 * b.real))
    return Dispersion(comp=comp, cell=cell,
                      pole_ofs=(np.arange(n + 1, dtype=np.int64) * p).astype(np.int32),
                      am1=np.tile(am1, n), b=np.tile(b, n), g=np.full(n, g1))


def zeta_poles(eps_inf: float, poles):
    """Pole expansion of 1/eps: ``(zeta_inf, p, r)`` with
    ``1/eps(s) = zeta_inf + sum_m r_m / (s - p_m)`` over every root (conjugates listed apart),
    for ``eps(s) = eps_inf + sum c/(s-a) + c*/(s-a*)`` (the restatement of
    ``openem/scene/poles.py:297-375``). With eps = N/D, the p_m are the zeros of N and
    ``r_m = D(p_m) / N'(p_m)``; the polynomials are built in ``u = s / scale`` (scale the largest
    |a|) so that their coefficients stay O(1). Roots within 1e-9 |u| of the imaginary axis are
    put on it; a root strictly in the right half plane is refused."""
    qs = []
    for a, c in poles:
        qs += [(complex(a), complex(c)), (np.conj(complex(a)), np.conj(complex(c)))]
    scale = max((abs(a) for a, _ in qs if abs(a) > 0), default=1.0)
    qu = [(a / scale, c / scale) for a, c in qs]
    den = np.poly([a for a, _ in qu]) if qu else np.array([1.0 + 0j])
    num = float(eps_inf) * den
    for k, (_, c) in enumerate(qu):
        rest = np.poly([a for j, (a, _) in enumerate(qu) if j != k])
        num = num + np.concatenate([np.zeros(num.size - rest.size), c * rest])
    pu = np.roots(num)
    pu = np.where(np.abs(pu.real) <= 1e-9 * np.abs(pu), 1j * pu.imag, pu)
    dnum = np.polyder(num)
    ru = np.polyval(den, pu) / np.polyval(dnum, pu)
    p, r = pu * scale, ru * scale
    if p.size and float(np.max(p.real)) > 0.0:
        raise ValueError(f"1/eps has a pole in the right half plane (max Re {np.max(p.real):.3e})")
    return 1.0 / float(eps_inf), p, r


def bulk_mix(shape, beta, pa, pb, qa, qb, eps_inf, zeta_inf, masks=None) -> DispersionMix:
    """The same two branches on every (component, cell) inside ``masks`` (all cells when None)
    with mixing weight ``beta`` (scalar or one value per entry)."""
    comp, cell = [], []
    for c in range(3):
        m = np.ones(shape, bool) if masks is None else masks[c]
        idx = np.flatnonzero(np.asarray(m).ravel())
        comp.append(np.full(idx.size, c, np.int32))
        cell.append(idx.astype(np.int64))
    comp, cell = np.concatenate(comp), np.concatenate(cell)
    n = comp.size
    pa, pb, qa, qb = (np.asarray(x, np.complex128) for x in (pa, pb, qa, qb))
    full = lambda v: np.broadcast_to(np.asarray(v, np.float64), (n,)).copy()
    return DispersionMix(comp=comp, cell=cell,
                         p_ofs=(np.arange(n + 1) * pa.size).astype(np.int64),
                         pa=np.tile(pa, n), pb=np.tile(pb, n),
                         q_ofs=(np.arange(n + 1) * qa.size).astype(np.int64),
                         qa=np.tile(qa, n), qb=np.tile(qb, n),
                         beta=full(beta), eps_inf=full(eps_inf), zeta_inf=full(zeta_inf))


def mix_pieces(eps_inf1: float, poles, eps2: float, fill: float, dt: float):
    """The two branches of a cell that holds the fraction ``fill`` of a pole-residue medium
    (eps_inf1, poles) and the rest of a constant eps2 (the layout of OpenEM's mixed-form tests):
    arithmetic eps_inf = f eps_inf1 + (1-f) eps2 with the residues times f; harmonic
    zeta_inf = f / eps_inf1 + (1-f) / eps2 with the 1/eps residues times f. Returns
    ``(eps_inf, zeta_inf, pa, pb, qa, qb)``."""
    pa, pb = trap_coeffs(poles, dt)
    z1, p1, r1 = zeta_poles(eps_inf1, poles)
    qa, qb = trap_coeffs(list(zip(p1, r1)), dt)
    return (fill * eps_inf1 + (1.0 - fill) * eps2, fill * z1 + (1.0 - fill) / eps2,
            pa, pb * fill, qa, qb * fill)


def mixed_sphere(n: int = 28, n_pml: int = 6, radius_cells: float = 5.3, num_steps: int = 300,
                 eps2: float = 2.25, eps_inf1: float = 2.0, lorentz=(1.5, 3e14, 3e13),
                 dip_freq0: float = 2.5e14, dip_fwidth: float = 1.5e14, seed: int = 5,
                 probe: bool = True) -> Scene:
    """A Lorentz sphere (eps_inf1 plus one Lorentz pair) in a constant eps2 background, with a
    point dipole beside it. Component points well inside take the E form (:class:`Dispersion`);
    points within half a cell of the surface take the mixed form with fill
    f = clip(0.5 - d / dl, 0, 1) (d the signed distance to the surface) and beta the squared
    normal projection on the component's axis, jittered by rng(seed) within [0, 1]."""
    dl = 0.02 * UM
    n_in = n - 2 * n_pml
    lo = -0.5 * n_in * dl
    axes = [uniform_axis(n_in, dl, lo, "PML", n_pml) for _ in range(3)]
    grid = Grid(*axes)
    dt = courant_dt([a.dl for a in axes])
    shape = grid.shape
    coords = yee_coords(grid)
    poles = lorentz_poles(*lorentz)
    R = radius_cells * dl
    cen = np.array([0.1, -0.05, 0.0]) * dl
    rng = np.random.default_rng(seed)
    inner, eps = [], []
    comp, cell, beta, fill = [], [], [], []
    for c in range(3):
        x, y, z = np.meshgrid(*coords[c], indexing="ij")
        rel = np.stack([x - cen[0], y - cen[1], z - cen[2]])
        r = np.sqrt((rel ** 2).sum(0))
        d = r - R
        ins = d < -0.5 * dl
        shell = np.abs(d) <= 0.5 * dl
        inner.append(ins)
        idx = np.flatnonzero(shell.ravel())
        nrm = rel[c].ravel()[idx] / np.maximum(r.ravel()[idx], 1e-30)
        b = np.clip(nrm * nrm + rng.uniform(-0.05, 0.05, idx.size), 0.0, 1.0)
        comp.append(np.full(idx.size, c, np.int32))
        cell.append(idx.astype(np.int64))
        beta.append(b)
        fill.append(np.clip(0.5 - d.ravel()[idx] / dl, 0.0, 1.0))
        e = np.full(shape, eps2)
        e[ins] = eps_inf1
        eps.append(e)
    comp, cell = np.concatenate(comp), np.concatenate(cell)
    beta, fill = np.concatenate(beta), np.concatenate(fill)
    pa, pb = trap_coeffs(poles, dt)
    z1, p1, r1 = zeta_poles(eps_inf1, poles)
    qa, qb = trap_coeffs(list(zip(p1, r1)), dt)
    ne, npp, nq = comp.size, pa.size, qa.size
    mix = DispersionMix(
        comp=comp, cell=cell,
        p_ofs=(np.arange(ne + 1) * npp).astype(np.int64),
        pa=np.tile(pa, ne), pb=(pb[None, :] * fill[:, None]).ravel(),
        q_ofs=(np.arange(ne + 1) * nq).astype(np.int64),
        qa=np.tile(qa, ne), qb=(qb[None, :] * fill[:, None]).ravel(),
        beta=beta, eps_inf=fill * eps_inf1 + (1.0 - fill) * eps2,
        zeta_inf=fill / eps_inf1 + (1.0 - fill) / eps2)
    for c in range(3):
        sel = comp == c
        eps[c].ravel()[cell[sel]] = mix.eps_inf[sel]
    disp = build_dispersion(inner, pa, pb, shape)
    pulse = GaussianPulse(freq0=dip_freq0, fwidth=dip_fwidth)
    wf = sample_waveform(pulse, dt, num_steps)
    idx, coef = dipole_stencil(grid, 0, (R + 2.5 * dl, 0.0, 0.0))
    dip = PointDipole(component=0, indices=idx, coef=coef, waveform=wf)
    fmons = []
    if probe:
        h = n // 2
        fmons.append(FieldMonitor(name="probe", freqs=np.array([dip_freq0]),
                                  origin=(h - 3, h - 3, h - 1), box=(6, 6, 2)))
    return Scene(grid=grid, dt=dt, num_time_steps=num_steps, shutoff=1e-5,
                 eps_ex=eps[0], eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 dispersion=disp, dispersion_mix=mix, dipoles=[dip], field_monitors=fmons)


# ---------------------------------------------------------------------------
# Workload 1: slab plane-wave transmission
# ---------------------------------------------------------------------------

def slab_plane_wave(nxy: int = 30, dl: float = 0.02 * UM, lz: float = 3.0 * UM,
                    eps_slab: float = 4.0, d_slab: float = 0.3 * UM,
                    src_z: float = -1.0 * UM, mon_t: float = 1.0 * UM,
                    mon_r: float = -1.2 * UM, freq0: float = 2.998e14, nfreq: int = 11,
                    run_time: float = 4e-13, n_pml: int = 12, with_slab: bool = True,
                    num_steps: int | None = None, direction: int = 1,
                    fwidth_rel: float = 0.2) -> Scene:
    """0.6 x 0.6 x 3.0 um periodic-x/y cell, 12-layer CPML on +/-z, an eps=4 slab 0.3 um thick
    at z=0, a +z Ex-polarised plane wave at z=-1.0 um (Gaussian pulse f0, fwidth=0.2 f0), flux
    planes "T" at z=+1.0 um and "R" at z=-1.2 um at 11 frequencies over f0 +/- fwidth.

    ``nxy`` may be reduced to 1: at normal incidence in a periodic cell the fields do not vary
    along x or y, so the result per unit area is unchanged."""
    nz_in = int(round(lz / dl))
    ax = uniform_axis(nxy, dl, -0.5 * nxy * dl, "Periodic")
    ay = uniform_axis(nxy, dl, -0.5 * nxy * dl, "Periodic")
    az = uniform_axis(nz_in, dl, -0.5 * lz, "PML", n_pml)
    grid = Grid(ax, ay, az)
    dt = courant_dt([ax.dl, ay.dl, az.dl]) if nxy > 1 else courant_dt([az.dl] * 3)
    n_steps = int(np.floor(run_time / dt + 1e-9)) + 1 if num_steps is None else int(num_steps)
    shape = grid.shape
    coords = yee_coords(grid)
    eps = []
    for c in range(3):
        z = coords[c][2]
        inside = np.abs(z) < 0.5 * d_slab - 1e-9 * dl
        e = np.ones(shape)
        if with_slab:
            e[:, :, inside] = eps_slab
        eps.append(e)
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth_rel * freq0)
    wf = sample_waveform(pulse, dt, n_steps)
    edges_z = np.asarray(az.edges)
    ks = int(np.argmin(np.abs(edges_z - src_z)))
    # the upstream Hy point is half a cell below the plane for +z, half a cell above for -z
    dl_half = 0.5 * float(az.dl[ks - 1] if direction > 0 else az.dl[ks])
    ex_inc, hy_inc = plane_wave_tables(pulse, dt, n_steps, dl_half, 1.0, direction)
    src = PlaneWaveSource(axis=2, plane_index=ks, direction=direction, pol_axis=0, waveform=wf,
                          angle_theta=0.0, num_freqs=1, ex_inc=ex_inc, hy_inc=hy_inc,
                          center=src_z)
    freqs = np.linspace(freq0 - fwidth_rel * freq0, freq0 + fwidth_rel * freq0, nfreq)
    spec = spectrum(pulse, dt, n_steps, freqs)
    mons = []
    for name, zc in (("T", mon_t), ("R", mon_r)):
        k = int(np.argmin(np.abs(edges_z - zc)))
        mons.append(FluxMonitor(name=name, axis=2, plane_index=k, normal_dir=1, freqs=freqs,
                                source_spectrum=spec))
    return Scene(grid=grid, dt=dt, num_time_steps=n_steps, shutoff=1e-5,
                 eps_ex=eps[0], eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 sources=[src], flux_monitors=mons)


def modulated_slab(eps_s: float = 1.0, delta: float = 0.01, fm_rel: float = 0.1,
                   phase=0.0, nxy: int = 1, dl: float = 0.025 * UM, lz: float = 4.0 * UM,
                   d_slab: float = 1.0 * UM, freq0: float = C_0 / (1.0 * UM),
                   fwidth_rel: float = 0.02, freqs=None, num_steps: int | None = None,
                   run_time: float | None = None) -> Scene:
    """A periodic-x/y cell with CPML on +-z, a +z Ex plane wave at z = -lz/2 + 0.4 um and a flux
    plane "T" at z = +lz/2 - 0.4 um, and a 1 um slab at z = 0 whose permittivity is
    ``eps_s + delta cos(2 pi fm t - phase)`` at every Yee point inside the slab, both faces
    included (so eps(t) >= eps_s - delta everywhere: below 1 the Courant step of the vacuum
    grid would be unstable). ``phase`` is a
    scalar or a function of the Yee point's (x, y, z). Monitor frequencies default to
    (f0 - fm, f0, f0 + fm)."""
    fm = fm_rel * freq0
    fwidth = fwidth_rel * freq0
    rt = run_time if run_time is not None else 10.0 / fwidth
    base = slab_plane_wave(nxy=nxy, dl=dl, lz=lz, eps_slab=eps_s, d_slab=d_slab,
                           src_z=-0.5 * lz + 0.4 * UM, mon_t=0.5 * lz - 0.4 * UM,
                           mon_r=-0.5 * lz + 0.2 * UM, freq0=freq0, nfreq=3, run_time=rt,
                           with_slab=eps_s != 1.0, num_steps=num_steps, fwidth_rel=fwidth_rel)
    f = np.asarray(freqs if freqs is not None else (freq0 - fm, freq0, freq0 + fm), np.float64)
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth)
    spec = spectrum(pulse, base.dt, base.num_time_steps, f)
    mons = [FluxMonitor(name=m.name, axis=2, plane_index=m.plane_index, normal_dir=1, freqs=f,
                        source_spectrum=spec) for m in base.flux_monitors]
    grid = base.grid
    nx, ny, nz = grid.shape
    coords = yee_coords(grid)
    comp, cell, ph = [], [], []
    eps = [np.array(e, dtype=np.float64) for e in (base.eps_ex, base.eps_ey, base.eps_ez)]
    for c in range(3):
        x, y, z = coords[c]
        kk = np.flatnonzero(np.abs(z) <= 0.5 * d_slab + 1e-6 * dl)
        eps[c][:, :, kk] = eps_s
        I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), kk, indexing="ij")
        comp.append(np.full(I.size, c))
        cell.append(((I * ny + J) * nz + K).ravel())
        if callable(phase):
            ph.append(np.asarray(phase(x[I.ravel()], y[J.ravel()], z[K.ravel()]), np.float64))
        else:
            ph.append(np.full(I.size, float(phase)))
    comp = np.concatenate(comp).astype(np.int32)
    cell = np.concatenate(cell).astype(np.int64)
    mod = TimeModulation(freq=fm, comp=comp, cell=cell, amp=np.full(comp.size, float(delta)),
                         phase=np.concatenate(ph))
    from dataclasses import replace
    return replace(base, flux_monitors=mons, modulation=mod, eps_ex=eps[0], eps_ey=eps[1],
                   eps_ez=eps[2])


def flux_time_plane(nxy: int = 16, dl: float = 0.025 * UM, plane_z: float = 0.3 * UM,
                    center=(0.013 * UM, -0.017 * UM), size=(0.27 * UM, 0.29 * UM),
                    interval: int = 1, start_step: int = 0, nfreq: int = 181,
                    run_time: float = 1.5e-13, num_steps: int | None = None,
                    full_span: bool = False) -> Scene:
    """Vacuum 0.4 x 0.4 x 1.6 um cell, periodic x/y, CPML z, a +z plane wave (GaussianPulse
    3e14 Hz, fwidth 0.6e14 Hz) at z = -0.55 um; a FluxTimeMonitor "ft" on the plane through
    ``plane_z`` (its position between two Yee boundaries sets ``frac``) with transverse bounds
    ``center +- size / 2`` (or the whole periodic cross section), a FluxMonitor "fx" at
    ``nfreq`` frequencies over f0 +- 4.5 fwidth on the boundary below it, and a FieldTimeMonitor
    "ftm" of E_x, E_y, H_x, H_y around the plane."""
    freq0, fwidth = 3.0e14, 0.6e14
    base = slab_plane_wave(nxy=nxy, dl=dl, lz=1.6 * UM, src_z=-0.55 * UM, mon_t=plane_z,
                           mon_r=-0.7 * UM, freq0=freq0, nfreq=3, run_time=run_time,
                           with_slab=False, num_steps=num_steps, fwidth_rel=fwidth / freq0)
    grid = base.grid
    ez = np.asarray(grid.axes[2].edges)
    km = int(np.searchsorted(ez, plane_z + 1e-6 * dl, side="right")) - 1
    frac = float((plane_z - ez[km]) / (ez[km + 1] - ez[km]))
    if abs(frac) < 1e-9:
        frac = 0.0
    if full_span:
        tb = tuple((float(grid.axes[a].edges[0]), float(grid.axes[a].edges[-1])) for a in (0, 1))
    else:
        tb = tuple((center[a] - 0.5 * size[a], center[a] + 0.5 * size[a]) for a in (0, 1))
    n = base.num_time_steps
    slots = (n - start_step + interval - 1) // interval
    ft = FluxTimeMonitor(name="ft", axis=2, plane_index=km, normal_dir=1, step_begin=start_step,
                         step_end=n, interval=interval, num_slots=slots, t_bounds=tb, frac=frac)
    freqs = np.linspace(freq0 - 4.5 * fwidth, freq0 + 4.5 * fwidth, nfreq)
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth)
    fx = FluxMonitor(name="fx", axis=2, plane_index=km, normal_dir=1, freqs=freqs,
                     source_spectrum=spectrum(pulse, base.dt, n, freqs))
    nx, ny, _ = grid.shape
    tm = FieldTimeMonitor(name="ftm", comps=(0, 1, 3, 4), origin=(0, 0, km - 1),
                          box=(nx, ny, 3), step_begin=start_step, step_end=n, interval=interval,
                          num_slots=slots)
    from dataclasses import replace
    return replace(base, flux_monitors=[fx], flux_time_monitors=[ft], field_time_monitors=[tm])


def tfsf_source(grid: Grid, dt: float, num_steps: int, eps_u: np.ndarray, box_lo, box_hi,
                axis: int = 2, direction: int = 1, pol=(1.0, 0.0), source_time=None,
                sigma_u: np.ndarray | None = None) -> TFSFSource:
    """A normal-incidence TFSF box source: the 1D auxiliary line copies the spacing of the box
    column (4 cells beyond each face) with a runway at both ends, its permittivity from the
    u-component profile at the box corner column, the injection point 2 cells outside the
    entry face, and incident tables with the wave impedance there
    (``openem/scene/sources.py:999-1232``). ``pol`` = (beta_u, beta_v) on the cyclic transverse
    axes u = (axis+1) % 3, v = (axis+2) % 3."""
    from openem_b200 import tfsf as TF
    a = axis
    u, v = TF.cyclic_axes(a)
    lo, hi = [int(x) for x in box_lo], [int(x) for x in box_hi]
    alo, ahi = lo[a], hi[a]
    c0, c1 = alo - TF.GAP, ahi + TF.GAP - 1
    na = grid.shape[a]
    if c0 < 0 or c1 > na - 1:
        raise ValueError(f"the TFSF box column [{c0}, {c1}] runs past the axis (n={na})")
    dl_col = np.asarray(grid.axes[a].dl, np.float64)[c0:c1 + 1]

    def column(arr):
        col = np.moveaxis(np.asarray(arr, np.float64), (u, v, a), (0, 1, 2))[lo[u], lo[v], :]
        return col[c0:c1 + 2] if c1 + 1 < col.size else np.concatenate([col[c0:], [col[-1]]])
    n_lo = TF.runway_cells(num_steps, dt, float(dl_col[0]))
    n_hi = TF.runway_cells(num_steps, dt, float(dl_col[-1]))
    dl1 = np.concatenate([np.full(n_lo, dl_col[0]), dl_col, np.full(n_hi, dl_col[-1])])
    seg = column(eps_u)
    eps1 = np.concatenate([np.full(n_lo, seg[0]), seg, np.full(n_hi - 1, seg[-1])])
    sigma1 = None
    if sigma_u is not None:
        sg = column(sigma_u)
        if np.abs(sg).max() > 0:
            sigma1 = np.concatenate([np.full(n_lo, sg[0]), sg, np.full(n_hi - 1, sg[-1])])
    col0 = n_lo + (alo - c0)
    inj = col0 - TF.GAP // 2 if direction > 0 else n_lo + (ahi - c0) + TF.GAP // 2
    kh1 = inj - 1 if direction > 0 else inj
    pulse = source_time or GaussianPulse(freq0=3e14, fwidth=1e14)
    ex_inc, hy_inc = plane_wave_tables(pulse, dt, num_steps, 0.5 * float(dl1[kh1]),
                                       float(eps1[inj]), direction)
    return TFSFSource(direction=direction, box_lo=tuple(lo), box_hi=tuple(hi), dl1=dl1,
                      eps1=eps1, inj=int(inj), col0=int(col0), ex_inc=ex_inc, hy_inc=hy_inc,
                      waveform=sample_waveform(pulse, dt, num_steps), axis=a,
                      pol_u=float(pol[0]), pol_v=float(pol[1]), sigma1=sigma1)


def tfsf_oblique_source(grid: Grid, dt: float, num_steps: int, box_lo, box_hi, k_hat, e_hat,
                        axis: int = 2, eps_bg: float = 1.0, source_time=None,
                        open_axes=()) -> TFSFSource:
    """An oblique-incidence TFSF box source (``openem/scene/sources.py:928-997``): the 1D line
    runs along +k_hat with the cell size matched to the grid's discrete dispersion at the pulse's
    centre frequency, spans the box's projection on k_hat (two cells before it, three after)
    plus a runway at both ends, and is injected two cells before the projection's start. The
    amplitude is scaled by 1/sqrt(|k_axis|) (the same power per area of the injection plane as at
    normal incidence)."""
    from openem_b200 import tfsf as TF
    k = np.asarray(k_hat, np.float64)
    k = k / np.linalg.norm(k)
    e = np.asarray(e_hat, np.float64)
    e = e - (e @ k) * k
    e = e / np.linalg.norm(e)
    pulse = source_time or GaussianPulse(freq0=3e14, fwidth=1e14)
    lo, hi = [int(x) for x in box_lo], [int(x) for x in box_hi]
    dl_axes = [float(grid.axes[q].dl[min(lo[q], grid.axes[q].n - 1)]) for q in range(3)]
    dl1v = TF.matched_dl(k, dl_axes, dt, float(pulse.freq0), eps_r=eps_bg)
    pmin, pmax = TF.projection_range(grid, k, lo, hi)
    proj0 = pmin - 2.0 * dl1v
    n_col_e = int(np.ceil((pmax - proj0) / dl1v)) + 3
    n_run = TF.runway_cells(num_steps, dt, dl1v)
    dl1 = np.full(2 * n_run + n_col_e, dl1v)
    eps1 = np.full(dl1.size, float(eps_bg))
    col0 = n_run
    inj = col0 - TF.GAP // 2
    ex_inc, hy_inc = plane_wave_tables(pulse, dt, num_steps, 0.5 * dl1v, float(eps_bg), +1)
    u, v = TF.cyclic_axes(axis)
    return TFSFSource(direction=+1, box_lo=tuple(lo), box_hi=tuple(hi), dl1=dl1, eps1=eps1,
                      inj=int(inj), col0=int(col0), ex_inc=ex_inc, hy_inc=hy_inc,
                      waveform=sample_waveform(pulse, dt, num_steps), axis=axis,
                      pol_u=float(e[u]), pol_v=float(e[v]), k_hat=tuple(float(x) for x in k),
                      e_hat=tuple(float(x) for x in e), dl1_step=float(dl1v),
                      proj0=float(proj0), n_col_e=int(n_col_e), open_axes=tuple(open_axes),
                      amp_scale=float(1.0 / np.sqrt(abs(float(k[axis])))))


def tfsf_box_scene(n: int = 40, n_pml: int = 8, dl: float = 0.02 * UM, axis: int = 2,
                   direction: int = 1, pol=(1.0, 0.0), margin: int = 5, sphere_eps: float = 0.0,
                   sphere_r: float = 0.1 * UM, substrate_eps: float = 0.0,
                   num_steps: int = 300, k_hat=None, e_hat=None, freq0: float = 3e14,
                   fwidth: float = 1e14) -> Scene:
    """An n^3 grid with CPML on every face and a TFSF box ``margin`` cells inside the CPML; a
    dielectric sphere at the centre (``sphere_eps`` > 0), a substrate filling the lower half
    along ``axis`` (``substrate_eps`` > 0, transversely uniform so it crosses the box), and a
    normal-incidence pulse along ``axis`` with polarisation ``pol`` on (u, v) -- or, with
    ``k_hat`` and ``e_hat``, an oblique one."""
    n_in = n - 2 * n_pml
    axes = [uniform_axis(n_in, dl, -0.5 * n_in * dl, "PML", n_pml) for _ in range(3)]
    grid = Grid(*axes)
    dt = courant_dt([ax.dl for ax in axes])
    coords = yee_coords(grid)
    eps = []
    for c in range(3):
        x, y, z = coords[c]
        e = np.ones(grid.shape)
        if substrate_eps > 0:
            w = (x, y, z)[axis]
            sl = [slice(None)] * 3
            sl[axis] = w < -2.0 * dl
            e[tuple(sl)] = substrate_eps
        if sphere_eps > 0:
            r2 = x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2
            e[r2 < sphere_r ** 2] = sphere_eps
        eps.append(e)
    lo = (n_pml + margin,) * 3
    hi = (n - n_pml - margin,) * 3
    u = (axis + 1) % 3
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth)
    if k_hat is not None:
        src = tfsf_oblique_source(grid, dt, num_steps, lo, hi, k_hat, e_hat, axis=axis,
                                  source_time=pulse)
    else:
        src = tfsf_source(grid, dt, num_steps, eps[u], lo, hi, axis=axis, direction=direction,
                          pol=pol, source_time=pulse)
    return Scene(grid=grid, dt=dt, num_time_steps=num_steps, shutoff=1e-5, eps_ex=eps[0],
                 eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 tfsf_sources=[src])


def tensor_region(sc: Scene, lo, hi, eps_tensor, sigma_tensor=None) -> TensorEps:
    """Entries of a fully anisotropic block over the cells [lo, hi) of every component (the
    3x3 ``eps_tensor`` / ``sigma_tensor``, or a function of the flat cell index returning them)
    plus a one-cell ring of diagonal halo entries around it carrying the scene's scalar eps and
    sigma, which closes the table under the 4-neighbour stencil (the layout of
    ``openem/scene/media.py``)."""
    shape = sc.shape
    ncell = int(np.prod(shape))
    comps, cells, eps, sig = [], [], [], []
    scal_e = (sc.eps_ex, sc.eps_ey, sc.eps_ez)
    scal_s = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
    glo = [max(lo[a] - 1, 0) for a in range(3)]
    ghi = [min(hi[a] + 1, shape[a]) for a in range(3)]
    for c in range(3):
        I, J, K = np.meshgrid(*[np.arange(glo[a], ghi[a]) for a in range(3)], indexing="ij")
        inner = ((I >= lo[0]) & (I < hi[0]) & (J >= lo[1]) & (J < hi[1]) & (K >= lo[2])
                 & (K < hi[2])).ravel()
        flat = ((I * shape[1] + J) * shape[2] + K).ravel()
        for f, core in zip(flat, inner):
            if core:
                et = eps_tensor(f) if callable(eps_tensor) else eps_tensor
                st = (sigma_tensor(f) if callable(sigma_tensor) else sigma_tensor)
                eps.append(np.asarray(et, np.float64))
                sig.append(np.zeros((3, 3)) if st is None else np.asarray(st, np.float64))
            else:
                d = np.eye(3)
                d[c, c] = float(np.asarray(scal_e[c]).ravel()[f])
                eps.append(d)
                sd = np.zeros((3, 3))
                if scal_s[c] is not None:
                    sd[c, c] = float(np.asarray(scal_s[c]).ravel()[f])
                sig.append(sd)
            comps.append(c)
            cells.append(f)
    del ncell
    return TensorEps(comp=np.asarray(comps, np.int32), cell=np.asarray(cells, np.int64),
                     eps=np.stack(eps), sigma=np.stack(sig))


def rotated_diag(e_diag, theta: float, axis: int = 2) -> np.ndarray:
    """diag(e_diag) rotated by ``theta`` about coordinate axis ``axis``."""
    c, s = np.cos(theta), np.sin(theta)
    u, v = (axis + 1) % 3, (axis + 2) % 3
    R = np.eye(3)
    R[u, u], R[u, v], R[v, u], R[v, v] = c, -s, s, c
    return R @ np.diag(np.asarray(e_diag, np.float64)) @ R.T


def slab_transmission(res_slab, res_empty, name: str = "T") -> np.ndarray:
    """``T(f) = P_slab / P_empty`` from two results' plane phasors, with the uniform-grid area
    element (the normalisation ``openem/flux.py:108-134`` uses: a reference run without the
    structure)."""
    def p(res):
        d = res.phasors[name].data
        return 0.5 * (np.real(d[0] * np.conj(d[3])).sum(axis=(1, 2))
                      - np.real(d[1] * np.conj(d[2])).sum(axis=(1, 2)))
    return p(res_slab) / p(res_empty)


def slab_analytic_T(freqs, n_slab: float = 2.0, d: float = 0.3 * UM) -> np.ndarray:
    """Single-layer thin-film transmission at normal incidence in vacuum."""
    k = 2 * np.pi * np.asarray(freqs) / C_0
    r = (1 - n_slab) / (1 + n_slab)
    ph = np.exp(2j * k * n_slab * d)
    t = (1 - r * r) * np.exp(1j * k * n_slab * d) / (1 - r * r * ph)
    return np.abs(t) ** 2


# ---------------------------------------------------------------------------
# Workload 2: dispersive bulk (Drude + Lorentz spheres, point dipole, plane DFT monitors)
# ---------------------------------------------------------------------------

def sphere_centres(n_sph: int, rmin: float, rmax: float, lo: float, hi: float, seed: int):
    """``n_sph`` non-overlapping spheres by rejection sampling: radius ~ U[rmin, rmax], centre
    ~ U over the box shrunk by the radius (the spheres stay inside the simulation domain)."""
    rng = np.random.default_rng(seed)
    out = []
    tries = 0
    while len(out) < n_sph:
        tries += 1
        if tries > 200000:
            raise RuntimeError("could not place the requested spheres")
        r = rng.uniform(rmin, rmax)
        c = rng.uniform(lo + r, hi - r, size=3)
        if all(np.linalg.norm(c - c2) >= r + r2 for c2, r2 in out):
            out.append((c, r))
    return out


def dipole_stencil(grid: Grid, comp: int, pos, magnetic: bool = False):
    """Trilinear weights of a point current moment at ``pos`` on the Yee points of ``comp``,
    divided by each point's dual volume -> ``(indices (nw, 3), coef (nw,))``."""
    coords = yee_coords(grid)[comp + (3 if magnetic else 0)]
    per_axis = []
    for a in range(3):
        co = coords[a]
        x = pos[a]
        i = int(np.argmin(np.abs(co - x)))
        if abs(co[i] - x) <= 1e-12 * max(abs(x), 1e-9):
            per_axis.append([(i, 1.0)])
            continue
        j = i + 1 if co[i] < x else i - 1
        w = (x - co[i]) / (co[j] - co[i])
        per_axis.append([(i, 1.0 - w), (j, w)])
    vols = (grid.yee_h_dual_volumes() if magnetic else grid.yee_dual_volumes())[comp]
    idx, coef = [], []
    for i, wi in per_axis[0]:
        for j, wj in per_axis[1]:
            for k, wk in per_axis[2]:
                idx.append((i, j, k))
                coef.append(wi * wj * wk / vols[i, j, k])
    return np.asarray(idx, dtype=np.int64), np.asarray(coef, dtype=np.float64)


def dispersive_spheres(n: int = 512, dl: float = 0.02 * UM, n_pml: int = 12, n_sph: int = 64,
                       rmin: float = 0.2 * UM, rmax: float = 0.6 * UM, seed: int = 0,
                       num_steps: int = 2000, nfreq: int = 8,
                       wp: float = 1.4e16, gamma: float = 1e14,
                       lorentz=(1.5, 4e14, 5e13), dip_freq0: float = 2e14,
                       dip_fwidth: float = 1e14, monitors: bool = True,
                       mon_band=(1.5e14, 2.5e14)) -> Scene:
    """``n^3`` cells in total (CPML included), CPML on all six faces, background eps=1, ``n_sph``
    non-overlapping spheres of a Drude (wp, gamma in rad/s) + Lorentz (deps, f0, delta in Hz)
    medium with eps_inf=1, a z-polarised point dipole at the centre, and three mid-plane field
    monitors (x, y and z normals) at ``nfreq`` frequencies."""
    n_in = n - 2 * n_pml
    lo = -0.5 * n_in * dl
    axes = [uniform_axis(n_in, dl, lo, "PML", n_pml) for _ in range(3)]
    grid = Grid(*axes)
    dt = courant_dt([a.dl for a in axes])
    shape = grid.shape
    coords = yee_coords(grid)
    spheres = sphere_centres(n_sph, rmin, rmax, lo, -lo, seed) if n_sph else []
    masks = []
    for c in range(3):
        x, y, z = coords[c]
        m = np.zeros(shape, dtype=bool)
        for cen, r in spheres:
            ix = np.flatnonzero(np.abs(x - cen[0]) <= r)
            iy = np.flatnonzero(np.abs(y - cen[1]) <= r)
            iz = np.flatnonzero(np.abs(z - cen[2]) <= r)
            if not (ix.size and iy.size and iz.size):
                continue
            d2 = ((x[ix, None, None] - cen[0]) ** 2 + (y[None, iy, None] - cen[1]) ** 2
                  + (z[None, None, iz] - cen[2]) ** 2)
            sub = m[ix[0]:ix[-1] + 1, iy[0]:iy[-1] + 1, iz[0]:iz[-1] + 1]
            sub |= d2 <= r * r
        masks.append(m)
    poles, sigma = split_dc(drude_poles(wp, gamma) + lorentz_poles(*lorentz), dt)
    am1, b = trap_coeffs(poles, dt)
    disp = build_dispersion(masks, am1, b, shape)
    eps = [np.ones(shape) for _ in range(3)]
    sig = [np.where(masks[c], sigma, 0.0) for c in range(3)]
    pulse = GaussianPulse(freq0=dip_freq0, fwidth=dip_fwidth)
    wf = sample_waveform(pulse, dt, num_steps)
    idx, coef = dipole_stencil(grid, 2, (0.0, 0.0, 0.0))
    dip = PointDipole(component=2, indices=idx, coef=coef, waveform=wf)
    fmons = []
    if monitors:
        freqs = np.linspace(mon_band[0], mon_band[1], nfreq)
        h = n // 2
        for a, name in enumerate(("mid_x", "mid_y", "mid_z")):
            origin = [0, 0, 0]
            box = [n, n, n]
            origin[a] = h - 1
            box[a] = 2
            fmons.append(FieldMonitor(name=name, freqs=freqs, origin=tuple(origin),
                                      box=tuple(box)))
    return Scene(grid=grid, dt=dt, num_time_steps=num_steps, shutoff=1e-5,
                 eps_ex=eps[0], eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 sigma_ex=sig[0], sigma_ey=sig[1], sigma_ez=sig[2], dispersion=disp,
                 dipoles=[dip], field_monitors=fmons)


def small_dispersive(n: int = 40, n_sph: int = 4, seed: int = 0, num_steps: int = 200,
                     n_pml: int = 8, **kw) -> Scene:
    """A scaled-down dispersive-spheres scene for oracle parity: same media and source, a
    smaller grid, fewer spheres, thinner CPML."""
    n_in = n - 2 * n_pml
    dl = 0.02 * UM
    r_hi = min(0.6 * UM, 0.22 * n_in * dl)
    r_lo = min(0.2 * UM, 0.5 * r_hi)
    return dispersive_spheres(n=n, dl=dl, n_pml=n_pml, n_sph=n_sph, rmin=r_lo,
                              rmax=r_hi, seed=seed, num_steps=num_steps, **kw)


def with_time_monitor(sc: Scene, name: str = "tmon", comps=(0, 1, 2, 3, 4, 5), origin=None,
                      box=None, step_begin: int = 0, step_end: int | None = None,
                      interval: int = 5) -> Scene:
    """Copy of ``sc`` with one field time monitor added (defaults: a small box at the grid
    centre, every ``interval`` steps)."""
    from dataclasses import replace
    nx, ny, nz = sc.shape
    if box is None:
        box = (min(4, nx), min(4, ny), min(4, nz))
    if origin is None:
        origin = tuple(max(0, s // 2 - b // 2) for s, b in zip(sc.shape, box))
    end = sc.num_time_steps if step_end is None else step_end
    slots = (end - 1 - step_begin) // interval + 1
    tm = FieldTimeMonitor(name=name, comps=tuple(comps), origin=tuple(origin), box=tuple(box),
                          step_begin=step_begin, step_end=end, interval=interval,
                          num_slots=slots)
    return replace(sc, field_time_monitors=list(sc.field_time_monitors) + [tm])


# ---------------------------------------------------------------------------------------------
# Mode-source carriers: oblique plane waves (Bloch cells) and Gaussian beams
# ---------------------------------------------------------------------------------------------

def _z_plane_coords(grid: Grid):
    """Transverse Yee coordinates of the z-normal tangential components: Ex (x ctr, y edge),
    Ey (x edge, y ctr), Hx (x edge, y ctr), Hy (x ctr, y edge)."""
    ax, ay = grid.axes[0], grid.axes[1]
    xe, ye = np.asarray(ax.edges[:-1], np.float64), np.asarray(ay.edges[:-1], np.float64)
    xc, yc = np.asarray(ax.centers, np.float64), np.asarray(ay.centers, np.float64)
    return {"Ex": (xc, ye), "Ey": (xe, yc), "Hx": (xe, yc), "Hy": (xc, ye)}


def _mode_amplitudes(source_time, dt: float, num_steps: int, delay_h: float):
    """amp_e = a(n dt), amp_h = a((n + 1/2) dt + delay_h) for n = 0..num_steps; the H delay is
    the travel time from the upstream H plane to the source plane."""
    n = np.arange(num_steps + 1, dtype=np.float64)
    amp_e = np.asarray(source_time.amp_time(n * dt), np.complex128)
    amp_h = np.asarray(source_time.amp_time((n + 0.5) * dt + delay_h), np.complex128)
    return amp_e, amp_h


def oblique_plane_wave(grid: Grid, dt: float, num_steps: int, plane_index: int, bloch_k,
                       source_time, pol: str = "s", direction: int = 1,
                       eps_r: float = 1.0) -> ModeSource:
    """z-normal mode source carrying a plane wave whose transverse wavevector is the Bloch
    vector of the cell, ``k_t = 2 pi (k_x / L_x, k_y / L_y)``: ``E = e exp(i k_t . r_t)``,
    ``H = n (k_hat x e) / eta0`` sampled at each component's Yee position, with
    ``k_z = sqrt(k^2 - |k_t|^2)`` at ``freq0`` (the angle of incidence at the carrier). ``pol``
    ``"s"``: E perpendicular to the plane of incidence (y at normal incidence); ``"p"``: in it.
    The H profile sits on the upstream H plane; its amplitude table is delayed by the half-cell
    travel time along z at the carrier angle (exact at normal incidence)."""
    ax, ay, az = grid.axes
    lx = float(ax.edges[-1] - ax.edges[0])
    ly = float(ay.edges[-1] - ay.edges[0])
    n_r = float(np.sqrt(eps_r))
    k0 = 2.0 * np.pi * source_time.freq0 * n_r / C_0
    kx = 2.0 * np.pi * float(bloch_k[0]) / lx
    ky = 2.0 * np.pi * float(bloch_k[1]) / ly
    kz2 = k0 * k0 - kx * kx - ky * ky
    if kz2 <= 0.0:
        raise ValueError("the Bloch vector is evanescent at the carrier frequency")
    kz = float(np.sqrt(kz2)) * (1 if direction > 0 else -1)
    khat = np.array([kx, ky, kz]) / k0
    zhat = np.array([0.0, 0.0, 1.0])
    s_vec = np.cross(zhat, khat)
    s_vec = np.array([0.0, 1.0, 0.0]) if np.linalg.norm(s_vec) < 1e-12 else s_vec / np.linalg.norm(s_vec)
    e = s_vec if pol == "s" else np.cross(khat, s_vec) * -1.0
    h = n_r * np.cross(khat, e) / ETA_0
    c = _z_plane_coords(grid)

    def prof(amp, name):
        x, y = c[name]
        return amp * np.exp(1j * (kx * x[:, None] + ky * y[None, :]))

    ks = int(plane_index)
    dl_half = 0.5 * float(az.dl[ks - 1] if direction > 0 else az.dl[ks])
    delay = dl_half * abs(khat[2]) * n_r / C_0
    amp_e, amp_h = _mode_amplitudes(source_time, dt, num_steps, delay)
    return ModeSource(plane_index=ks, direction=int(direction),
                      ey_inc=prof(e[0], "Ex"), ez_inc=prof(e[1], "Ey"),
                      hy_inc=prof(h[0], "Hx"), hz_inc=prof(h[1], "Hy"),
                      amp_e=amp_e, amp_h=amp_h, n_eff=complex(n_r), axis=2)


def gaussian_beam(grid: Grid, dt: float, num_steps: int, plane_index: int, waist: float,
                  source_time, pol_axis: int = 1, center=(0.0, 0.0), direction: int = 1,
                  eps_r: float = 1.0) -> ModeSource:
    """z-normal mode source of a Gaussian beam at its waist plane: E = e exp(-r^2 / w0^2)
    polarised along ``pol_axis`` (0 or 1), H = n (z_hat x E) / eta0 (paraxial), amplitude
    tables as :func:`oblique_plane_wave` at normal incidence."""
    az = grid.axes[2]
    n_r = float(np.sqrt(eps_r))
    c = _z_plane_coords(grid)
    e = np.zeros(3)
    e[pol_axis] = 1.0
    khat = np.array([0.0, 0.0, 1.0 if direction > 0 else -1.0])
    h = n_r * np.cross(khat, e) / ETA_0

    def prof(amp, name):
        x, y = c[name]
        r2 = (x[:, None] - center[0]) ** 2 + (y[None, :] - center[1]) ** 2
        return (amp * np.exp(-r2 / (waist * waist))).astype(np.complex128)

    ks = int(plane_index)
    dl_half = 0.5 * float(az.dl[ks - 1] if direction > 0 else az.dl[ks])
    amp_e, amp_h = _mode_amplitudes(source_time, dt, num_steps, dl_half * n_r / C_0)
    return ModeSource(plane_index=ks, direction=int(direction),
                      ey_inc=prof(e[0], "Ex"), ez_inc=prof(e[1], "Ey"),
                      hy_inc=prof(h[0], "Hx"), hz_inc=prof(h[1], "Hy"),
                      amp_e=amp_e, amp_h=amp_h, n_eff=complex(n_r), axis=2)


def _pixel_eps(grid: Grid, shape, npix: int, layer, lo_hi, rng):
    """Diagonal permittivity of a pixelated layer: per pixel (npix x npix in the x-y plane)
    eps_xx, eps_yy, eps_zz ~ U[lo, hi], staircased per component at its Yee position; layer =
    (z0, z1) in metres."""
    pix = rng.uniform(lo_hi[0], lo_hi[1], size=(3, npix, npix))
    ax, ay = grid.axes[0], grid.axes[1]
    x0, x1 = float(ax.edges[0]), float(ax.edges[-1])
    y0, y1 = float(ay.edges[0]), float(ay.edges[-1])
    coords = yee_coords(grid)
    eps = []
    for comp in range(3):
        x, y, z = coords[comp]
        px = np.clip(((x - x0) / (x1 - x0) * npix).astype(int), 0, npix - 1)
        py = np.clip(((y - y0) / (y1 - y0) * npix).astype(int), 0, npix - 1)
        inz = (z >= layer[0]) & (z < layer[1])
        e = np.ones(shape)
        vals = pix[comp][px[:, None], py[None, :]]
        e[:, :, inz] = vals[:, :, None]
        eps.append(e)
    return eps


def bloch_metasurface(nx: int = 256, ny: int = 256, nz: int = 1024, dl: float = 0.01 * UM,
                      n_pml: int = 12, bloch_k=(0.15, 0.0, 0.0), freq0: float = 3e14,
                      fwidth_rel: float = 0.3, npix: int = 64, layer_cells: int = 40,
                      nfreq: int = 200, num_steps: int = 20000, seed: int = 1,
                      field_monitor: bool = False) -> Scene:
    """Bloch unit cell with a pixelated diagonal-anisotropic layer: ``nx x ny x nz`` cells in
    total (CPML on +-z included), Bloch vector ``bloch_k`` (in units of 2 pi / L) on x and y,
    a ``layer_cells``-thick layer at mid-z whose ``npix x npix`` pixels draw eps_xx, eps_yy,
    eps_zz from U[2, 12] (``seed``), an s-polarised oblique plane wave (transverse wavevector =
    Bloch vector) injected upward from below the layer, and a flux monitor above it with
    ``nfreq`` frequencies over freq0 +- fwidth."""
    n_in = nz - 2 * n_pml
    axes = [Axis(np.arange(nx + 1) * dl, "BlochBoundary", "BlochBoundary"),
            Axis(np.arange(ny + 1) * dl, "Periodic", "Periodic"),
            uniform_axis(n_in, dl, -0.5 * n_in * dl, "PML", n_pml)]
    grid = Grid(*axes)
    dt = courant_dt([a.dl for a in axes])
    shape = grid.shape
    zc = 0.0
    layer = (zc - 0.5 * layer_cells * dl, zc + 0.5 * layer_cells * dl)
    eps = _pixel_eps(grid, shape, npix, layer, (2.0, 12.0), np.random.default_rng(seed))
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth_rel * freq0)
    edges_z = np.asarray(axes[2].edges)
    z_src = layer[0] - 0.25 * n_in * dl
    ks = int(np.argmin(np.abs(edges_z - z_src)))
    src = oblique_plane_wave(grid, dt, num_steps, ks, bloch_k, pulse, pol="s")
    freqs = np.linspace(freq0 * (1 - fwidth_rel), freq0 * (1 + fwidth_rel), nfreq)
    km = int(np.argmin(np.abs(edges_z - (layer[1] + 0.2 * n_in * dl))))
    mons = [FluxMonitor(name="T", axis=2, plane_index=km, normal_dir=1, freqs=freqs,
                        source_spectrum=spectrum(pulse, dt, num_steps, freqs))]
    fmons = []
    if field_monitor:
        fmons.append(FieldMonitor(name="layer_mid", freqs=freqs[:: max(1, nfreq // 4)],
                                  origin=(0, 0, nz // 2), box=(nx, ny, 1)))
    return Scene(grid=grid, dt=dt, num_time_steps=num_steps, shutoff=1e-5,
                 eps_ex=eps[0], eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 bloch_k=tuple(float(v) for v in bloch_k), mode_sources=[src],
                 flux_monitors=mons, field_monitors=fmons)


def beam_slab(nx: int = 200, ny: int = 200, nz: int = 120, dl: float = 0.025 * UM,
              n_pml: int = 12, eps_slab: float = 12.1, eps_bg: float = 2.1,
              slab_cells: int = 9, design=(80, 80), seed: int = 2, waist: float = 1.0 * UM,
              freq0: float = 1.94e14, fwidth_rel: float = 0.15, nfreq: int = 5,
              num_steps: int = 2000) -> Scene:
    """A slab (``slab_cells`` thick, eps_slab) in a background eps_bg with a ``design`` pixel
    region of the slab drawn from U[eps_bg, eps_slab] (``seed``), CPML on all faces, a
    y-polarised Gaussian beam (``waist``) injected upward below the slab and a flux monitor
    above it at ``nfreq`` frequencies over freq0 +- fwidth."""
    dims = (nx, ny, nz)
    axes = [uniform_axis(d - 2 * n_pml, dl, -0.5 * (d - 2 * n_pml) * dl, "PML", n_pml)
            for d in dims]
    grid = Grid(*axes)
    dt = courant_dt([a.dl for a in axes])
    shape = grid.shape
    rng = np.random.default_rng(seed)
    coords = yee_coords(grid)
    zlo, zhi = -0.5 * slab_cells * dl, 0.5 * slab_cells * dl
    dx, dy = design[0] * dl, design[1] * dl
    pix = rng.uniform(eps_bg, eps_slab, size=design)
    eps = []
    for comp in range(3):
        x, y, z = coords[comp]
        e = np.full(shape, eps_bg)
        inz = (z >= zlo) & (z < zhi)
        e[:, :, inz] = eps_slab
        ix = np.flatnonzero(np.abs(x) < 0.5 * dx)
        iy = np.flatnonzero(np.abs(y) < 0.5 * dy)
        px = np.clip(((x[ix] + 0.5 * dx) / dx * design[0]).astype(int), 0, design[0] - 1)
        py = np.clip(((y[iy] + 0.5 * dy) / dy * design[1]).astype(int), 0, design[1] - 1)
        sub = e[ix[0]:ix[-1] + 1, iy[0]:iy[-1] + 1, :]
        sub[:, :, inz] = pix[px[:, None], py[None, :]][:, :, None]
        eps.append(e)
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth_rel * freq0)
    edges_z = np.asarray(axes[2].edges)
    n_in = nz - 2 * n_pml
    ks = int(np.argmin(np.abs(edges_z - (zlo - 0.3 * n_in * dl))))
    src = gaussian_beam(grid, dt, num_steps, ks, waist, pulse, pol_axis=1, eps_r=eps_bg)
    freqs = np.linspace(freq0 * (1 - fwidth_rel), freq0 * (1 + fwidth_rel), nfreq)
    km = int(np.argmin(np.abs(edges_z - (zhi + 0.3 * n_in * dl))))
    mons = [FluxMonitor(name="T", axis=2, plane_index=km, normal_dir=1, freqs=freqs,
                        source_spectrum=spectrum(pulse, dt, num_steps, freqs))]
    return Scene(grid=grid, dt=dt, num_time_steps=num_steps, shutoff=1e-5,
                 eps_ex=eps[0], eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 mode_sources=[src], flux_monitors=mons)


def absorber_slabs(grid: Grid, axis: int, n_layers: int, strength: float = 0.05,
                   order: int = 3) -> list:
    """Graded absorber slabs on both ends of ``axis``: per step decay ``exp(-s d^order)`` with
    ``d`` the depth into the absorber (0 at its inner face, 1 at the wall), sampled at the
    whole-cell and half-cell positions of each layer in global index order."""
    from openem_b200.model import AbsorberSlab
    n = int(grid.shape[axis])
    lay = np.arange(n_layers, dtype=np.float64)
    lo_int = (n_layers - lay) / n_layers
    lo_half = (n_layers - lay - 0.5) / n_layers
    hi_int = lay / n_layers
    hi_half = (lay + 0.5) / n_layers
    dec = lambda d: np.exp(-strength * d ** order)
    return [AbsorberSlab(axis=axis, g0=0, decay_int=dec(lo_int), decay_half=dec(lo_half)),
            AbsorberSlab(axis=axis, g0=n - n_layers, decay_int=dec(hi_int),
                         decay_half=dec(hi_half))]


def serving_request(n: int, rng, num_steps: int, dl: float = 0.02 * UM,
                    n_pml: int = 12) -> Scene:
    """One request of a serving stream: an ``n^3`` grid (CPML on all faces included), a medium
    drawn from {non-dispersive eps ~ U[1, 12]; 1-pole Drude; 2-pole Lorentz} filling 1 to 16
    random boxes, a z dipole at a random interior point or a +z plane wave, and one flux
    monitor near the top face at 4 to 32 frequencies. ``rng`` is a numpy Generator."""
    n_pml = min(n_pml, max(4, n // 8))
    n_in = n - 2 * n_pml
    lo = -0.5 * n_in * dl
    axes = [uniform_axis(n_in, dl, lo, "PML", n_pml) for _ in range(3)]
    grid = Grid(*axes)
    dt = courant_dt([a.dl for a in axes])
    shape = grid.shape
    kind = int(rng.integers(0, 3))
    nbox = int(rng.integers(1, 17))
    coords = yee_coords(grid)
    boxes = []
    for _ in range(nbox):
        c = rng.uniform(lo * 0.8, -lo * 0.8, size=3)
        h = rng.uniform(0.05, 0.25, size=3) * (-2.0 * lo)
        boxes.append((c - h, c + h))
    masks = []
    for comp in range(3):
        x, y, z = coords[comp]
        m = np.zeros(shape, dtype=bool)
        for b0, b1 in boxes:
            ix = (x >= b0[0]) & (x <= b1[0])
            iy = (y >= b0[1]) & (y <= b1[1])
            iz = (z >= b0[2]) & (z <= b1[2])
            m |= ix[:, None, None] & iy[None, :, None] & iz[None, None, :]
        masks.append(m)
    eps = [np.ones(shape) for _ in range(3)]
    sig = None
    disp = None
    if kind == 0:
        v = float(rng.uniform(1.0, 12.0))
        for c in range(3):
            eps[c][masks[c]] = v
    else:
        if kind == 1:
            poles = drude_poles(float(rng.uniform(5e15, 1.5e16)), float(rng.uniform(5e13, 2e14)))
        else:
            poles = lorentz_poles(float(rng.uniform(0.5, 3.0)), float(rng.uniform(1e14, 4e14)),
                                  float(rng.uniform(1e13, 5e13))) + \
                lorentz_poles(float(rng.uniform(0.5, 3.0)), float(rng.uniform(1e14, 4e14)),
                              float(rng.uniform(1e13, 5e13)))
        poles, sigma = split_dc(poles, dt)
        am1, b = trap_coeffs(poles, dt)
        disp = build_dispersion(masks, am1, b, shape)
        if sigma:
            sig = [np.where(masks[c], sigma, 0.0) for c in range(3)]
    freq0, fwidth = 2e14, 1e14
    pulse = GaussianPulse(freq0=freq0, fwidth=fwidth)
    wf = sample_waveform(pulse, dt, num_steps)
    edges_z = np.asarray(axes[2].edges)
    sources, dipoles = [], []
    if rng.integers(0, 2) == 0:
        pos = rng.uniform(lo * 0.5, -lo * 0.5, size=3)
        idx, coef = dipole_stencil(grid, 2, tuple(pos))
        dipoles.append(PointDipole(component=2, indices=idx, coef=coef, waveform=wf))
    else:
        ks = n_pml + max(2, n_in // 8)
        dl_half = 0.5 * float(axes[2].dl[ks - 1])
        ex_inc, hy_inc = plane_wave_tables(pulse, dt, num_steps, dl_half, 1.0, 1)
        sources.append(PlaneWaveSource(axis=2, plane_index=ks, direction=1, pol_axis=0,
                                       waveform=wf, angle_theta=0.0, num_freqs=1,
                                       ex_inc=ex_inc, hy_inc=hy_inc,
                                       center=float(edges_z[ks])))
    nf = int(rng.integers(4, 33))
    freqs = np.linspace(freq0 - 0.5 * fwidth, freq0 + 0.5 * fwidth, nf)
    km = n - n_pml - max(2, n_in // 8)
    mons = [FluxMonitor(name="T", axis=2, plane_index=km, normal_dir=1, freqs=freqs,
                        source_spectrum=spectrum(pulse, dt, num_steps, freqs))]
    sig = sig or [None, None, None]
    return Scene(grid=grid, dt=dt, num_time_steps=num_steps, shutoff=1e-5,
                 eps_ex=eps[0], eps_ey=eps[1], eps_ez=eps[2], pml=pml_dict(grid, dt, n_pml),
                 sigma_ex=sig[0], sigma_ey=sig[1], sigma_ez=sig[2], dispersion=disp,
                 sources=sources, dipoles=dipoles, flux_monitors=mons)
