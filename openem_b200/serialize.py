"""``scene.npz`` reader and writer, key for key compatible with OpenEM's format versions 1..10
(``openem/serialize.py:44-683``), so a scene exported by OpenEM's builder runs on this engine and
a scene written here runs on OpenEM. numpy only.

The key names are a wire format and therefore identical to OpenEM's; the code is this engine's.
"""

from __future__ import annotations

import os
import pathlib

import numpy as np

from openem_b200 import model as M

FORMAT_VERSION = 10
_PML = ("a_E", "b_E", "inv_kappa_E", "a_H", "b_H", "inv_kappa_H")
_DMIX = ("comp", "cell", "p_ofs", "pa", "pb", "q_ofs", "qa", "qb", "beta", "eps_inf", "zeta_inf")
_MSRC_BB = ("bb_ey", "bb_ez", "bb_hy", "bb_hz", "bb_amp_e", "bb_amp_h")


def _opt(z, key):
    """Optional array: absent, or saved as an object (``None``), reads back as None."""
    if key not in z.files:
        return None
    try:
        a = z[key]
    except ValueError:
        return None
    if a.dtype == object or (a.shape == () and a.dtype.kind not in "fc"):
        return None
    return a


def _count(z, key) -> int:
    return int(z[key]) if key in z.files else 0


def _names(z, key):
    return z[key] if key in z.files else []


def _wave(z, prefix, dt):
    a = z[f"{prefix}_amp_int"]
    return M.Waveform(amp_int=a, amp_half=z[f"{prefix}_amp_half"],
                      amp_int_complex=a.astype(np.complex128), dt=dt)


def _apod(arr):
    return tuple(None if np.isnan(v) else float(v) for v in arr)


def _apod_pack(a):
    return np.array([np.nan if v is None else float(v) for v in a])


def load(path) -> M.Scene:
    """Read a ``scene.npz`` written by OpenEM (versions 1..10) or by :func:`save`."""
    z = np.load(path, allow_pickle=False)
    ver = int(z["format_version"])
    if not 1 <= ver <= FORMAT_VERSION:
        raise ValueError(f"scene.npz format version {ver}, accepted 1..{FORMAT_VERSION}")
    dt = float(z["dt"])
    axes = []
    for nm in "xyz":
        lo, hi = (str(v) for v in z[f"bnd_{nm}"])
        axes.append(M.Axis(z[f"edges_{nm}"], lo, hi,
                           flat=bool(z[f"flat_{nm}"]) if f"flat_{nm}" in z.files else None))
    pml = {}
    for key in z["pml_keys"]:
        a, side = str(key).split(":")
        pml[(int(a), side)] = M.PMLCoeffs(**{f: z[f"pml_{a}_{side}_{f}"] for f in _PML})

    sources = []
    for i in range(int(z["n_sources"])):
        ax, pi, dr, pol, nfr = (int(v) for v in z[f"src{i}_meta"])
        sources.append(M.PlaneWaveSource(
            axis=ax, plane_index=pi, direction=dr, pol_axis=pol, waveform=_wave(z, f"src{i}", dt),
            angle_theta=float(z[f"src{i}_angle_theta"]), num_freqs=nfr,
            ex_inc=z[f"src{i}_ex_inc"], hy_inc=z[f"src{i}_hy_inc"],
            center=float(z[f"src{i}_center"]) if f"src{i}_center" in z.files else float("nan")))

    mode_sources = []
    for i in range(_count(z, "n_mode_sources")):
        meta = [int(v) for v in z[f"msrc{i}_meta"]]
        ne = z[f"msrc{i}_n_eff"]
        mode_sources.append(M.ModeSource(
            plane_index=meta[0], direction=meta[1], n_eff=complex(ne[0], ne[1]),
            axis=meta[2] if len(meta) > 2 else 0,
            ey_inc=z[f"msrc{i}_ey_inc"], ez_inc=z[f"msrc{i}_ez_inc"],
            hy_inc=z[f"msrc{i}_hy_inc"], hz_inc=z[f"msrc{i}_hz_inc"],
            amp_e=z[f"msrc{i}_amp_e"], amp_h=z[f"msrc{i}_amp_h"],
            **{f: z[f"msrc{i}_{f}"] for f in _MSRC_BB if f"msrc{i}_{f}" in z.files}))

    tfsf = []
    for i in range(_count(z, "n_tfsf")):
        m = [int(v) for v in z[f"tfsf{i}_meta"]]
        pol = z[f"tfsf{i}_pol"] if f"tfsf{i}_pol" in z.files else np.array([1.0, 0.0])
        obl = {}
        if f"tfsf{i}_obl" in z.files:
            o = np.asarray(z[f"tfsf{i}_obl"], dtype=np.float64)
            obl = {"k_hat": tuple(float(x) for x in o[0:3]),
                   "e_hat": tuple(float(x) for x in o[3:6]),
                   "dl1_step": float(o[6]), "proj0": float(o[7]),
                   "n_col_e": int(round(float(o[8]))),
                   "amp_scale": float(o[9]) if o.size > 9 else 1.0}
        tfsf.append(M.TFSFSource(
            direction=m[0], box_lo=tuple(m[1:4]), box_hi=tuple(m[4:7]), inj=m[7], col0=m[8],
            num_freqs=m[9], axis=m[10] if len(m) > 10 else 2,
            open_axes=tuple(q for q in range(3) if len(m) > 11 and (m[11] >> q) & 1),
            pol_u=float(pol[0]), pol_v=float(pol[1]), dl1=z[f"tfsf{i}_dl1"],
            eps1=z[f"tfsf{i}_eps1"], ex_inc=z[f"tfsf{i}_ex_inc"], hy_inc=z[f"tfsf{i}_hy_inc"],
            waveform=_wave(z, f"tfsf{i}", dt),
            sigma1=z[f"tfsf{i}_sigma1"] if f"tfsf{i}_sigma1" in z.files else None, **obl))

    dipoles = []
    for i in range(_count(z, "n_dipoles")):
        ai, ah = z[f"dip{i}_amp_int"], z[f"dip{i}_amp_half"]
        aic = (ai + 1j * z[f"dip{i}_amp_int_im"] if f"dip{i}_amp_int_im" in z.files
               else ai.astype(np.complex128))
        ahc = ah + 1j * z[f"dip{i}_amp_half_im"] if f"dip{i}_amp_half_im" in z.files else None
        dipoles.append(M.PointDipole(
            component=int(z[f"dip{i}_component"]), indices=z[f"dip{i}_indices"],
            coef=z[f"dip{i}_coef"],
            waveform=M.Waveform(amp_int=ai, amp_half=ah, amp_int_complex=aic, dt=dt,
                                amp_half_complex=ahc),
            magnetic=bool(int(z[f"dip{i}_magnetic"])) if f"dip{i}_magnetic" in z.files
            else False))

    disp = None
    if "disp_comp" in z.files:
        disp = M.Dispersion(comp=z["disp_comp"], cell=z["disp_cell"], pole_ofs=z["disp_pole_ofs"],
                            am1=z["disp_am1"], b=z["disp_b"], g=z["disp_g"])
    modu = None
    if "mod_comp" in z.files:
        modu = M.TimeModulation(freq=float(z["mod_freq"]), comp=z["mod_comp"], cell=z["mod_cell"],
                                amp=z["mod_amp"], phase=z["mod_phase"])
    tensor = None
    if "tensor_comp" in z.files:
        tensor = M.TensorEps(comp=z["tensor_comp"], cell=z["tensor_cell"],
                             eps=z["tensor_eps"], sigma=z["tensor_sigma"])
    dmix = None
    if "dmix_comp" in z.files:
        dmix = M.DispersionMix(**{f: z[f"dmix_{f}"] for f in _DMIX})

    absorbers = []
    for i in range(_count(z, "n_absorbers")):
        ax, g0 = (int(v) for v in z[f"abs{i}_meta"])
        absorbers.append(M.AbsorberSlab(axis=ax, g0=g0, decay_int=z[f"abs{i}_decay_int"],
                                        decay_half=z[f"abs{i}_decay_half"]))

    flux_mons = []
    for i, name in enumerate(z["mon_names"]):
        ax, pi, nd = (int(v) for v in z[f"mon{i}_meta"])
        tk = f"mon{i}_transverse"
        flux_mons.append(M.FluxMonitor(
            name=str(name), axis=ax, plane_index=pi, normal_dir=nd, freqs=z[f"mon{i}_freqs"],
            source_spectrum=z[f"mon{i}_spectrum"],
            transverse=tuple(map(tuple, z[tk].tolist())) if tk in z.files else None,
            apodization=_apod(z[f"mon{i}_apod"]) if f"mon{i}_apod" in z.files else None,
            t_bounds=(tuple(map(tuple, z[f"mon{i}_tbounds"].tolist()))
                      if f"mon{i}_tbounds" in z.files else None)))
    field_mons = []
    for i, name in enumerate(_names(z, "fmon_names")):
        m = [int(v) for v in z[f"fmon{i}_meta"]]
        field_mons.append(M.FieldMonitor(
            name=str(name), freqs=z[f"fmon{i}_freqs"], origin=tuple(m[0:3]), box=tuple(m[3:6]),
            interval_space=tuple(m[6:9]) if len(m) > 6 else (1, 1, 1),
            apodization=_apod(z[f"fmon{i}_apod"]) if f"fmon{i}_apod" in z.files else None))
    tmons = []
    for i, name in enumerate(_names(z, "tmon_names")):
        beg, end, iv, slots = (int(v) for v in z[f"tmon{i}_meta"])
        tmons.append(M.FieldTimeMonitor(
            name=str(name), comps=tuple(int(v) for v in z[f"tmon{i}_comps"]),
            origin=tuple(int(v) for v in z[f"tmon{i}_origin"]),
            box=tuple(int(v) for v in z[f"tmon{i}_box"]), step_begin=beg, step_end=end,
            interval=iv, num_slots=slots))
    ftmons = []
    for i, name in enumerate(_names(z, "ftmon_names")):
        ax, pi, nd, beg, end, iv, slots = (int(v) for v in z[f"ftmon{i}_meta"])
        ftmons.append(M.FluxTimeMonitor(
            name=str(name), axis=ax, plane_index=pi, normal_dir=nd, step_begin=beg, step_end=end,
            interval=iv, num_slots=slots,
            t_bounds=tuple(tuple(float(v) for v in r) for r in z[f"ftmon{i}_tbounds"]),
            frac=float(z[f"ftmon{i}_frac"])))
    pmons = []
    for i, name in enumerate(_names(z, "pmon_names")):
        m = [int(v) for v in z[f"pmon{i}_meta"]]
        pmons.append(M.PermittivityMonitor(name=str(name), freqs=z[f"pmon{i}_freqs"],
                                           origin=tuple(m[0:3]), box=tuple(m[3:6])))
    projmons = [M.ProjectionMonitor(name=str(n),
                                    surface_names=tuple(str(s) for s in z[f"projmon{i}_surfaces"]),
                                    normal_dirs=tuple(str(s) for s in z[f"projmon{i}_dirs"]))
                for i, n in enumerate(_names(z, "projmon_names"))]
    bfmons = [M.BoxFluxMonitor(name=str(n), face_names=tuple(str(s) for s in z[f"bfmon{i}_faces"]))
              for i, n in enumerate(_names(z, "bfmon_names"))]
    modemons = ([M.ModeMonitorSpec(name=str(n), plane_name=str(p))
                 for n, p in zip(z["modemon_names"], z["modemon_planes"])]
                if "modemon_names" in z.files else [])

    return M.Scene(
        grid=M.Grid(*axes), dt=dt, num_time_steps=int(z["num_time_steps"]),
        shutoff=float(z["shutoff"]), eps_ex=z["eps_ex"], eps_ey=z["eps_ey"], eps_ez=z["eps_ez"],
        pml=pml, sigma_ex=_opt(z, "sigma_ex"), sigma_ey=_opt(z, "sigma_ey"),
        sigma_ez=_opt(z, "sigma_ez"),
        pec_ex=z["pec_ex"] if "pec_ex" in z.files else None,
        pec_ey=z["pec_ey"] if "pec_ey" in z.files else None,
        pec_ez=z["pec_ez"] if "pec_ez" in z.files else None,
        dispersion=disp, dispersion_mix=dmix, modulation=modu, tensor=tensor,
        symmetry=tuple(int(v) for v in z["symmetry"]) if "symmetry" in z.files else (0, 0, 0),
        bloch_k=(tuple(float(v) for v in z["bloch_k"]) if "bloch_k" in z.files
                 else (0.0, 0.0, 0.0)),
        sources=sources, tfsf_sources=tfsf, dipoles=dipoles, mode_sources=mode_sources,
        flux_monitors=flux_mons, field_monitors=field_mons, field_time_monitors=tmons,
        flux_time_monitors=ftmons, permittivity_monitors=pmons, projection_monitors=projmons,
        box_flux_monitors=bfmons, mode_monitors=modemons, absorbers=absorbers)


def save(sc, path) -> pathlib.Path:
    """Write ``sc`` as a ``scene.npz`` (format 10), atomically (temp file + rename)."""
    d = {"format_version": np.array(FORMAT_VERSION), "dt": np.array(sc.dt),
         "num_time_steps": np.array(sc.num_time_steps), "shutoff": np.array(sc.shutoff),
         "symmetry": np.array(sc.symmetry), "bloch_k": np.array(sc.bloch_k, dtype=np.float64),
         "eps_ex": sc.eps_ex, "eps_ey": sc.eps_ey, "eps_ez": sc.eps_ez}
    if sc.sigma_ex is not None:
        d.update(sigma_ex=sc.sigma_ex, sigma_ey=sc.sigma_ey, sigma_ez=sc.sigma_ez)
    if sc.pec_ex is not None:
        d.update(pec_ex=sc.pec_ex, pec_ey=sc.pec_ey, pec_ez=sc.pec_ez)
    for nm, ax in zip("xyz", sc.grid.axes):
        d[f"edges_{nm}"] = ax.edges
        if getattr(ax, "flat", None) is not None:
            d[f"flat_{nm}"] = np.array(bool(ax.flat))
        d[f"bnd_{nm}"] = np.array([ax.boundary_lo, ax.boundary_hi])
    d["pml_keys"] = np.array([f"{a}:{s}" for (a, s) in sorted(sc.pml)])
    for (a, s), c in sc.pml.items():
        for f in _PML:
            d[f"pml_{a}_{s}_{f}"] = getattr(c, f)
    d["n_sources"] = np.array(len(sc.sources))
    for i, s in enumerate(sc.sources):
        d[f"src{i}_meta"] = np.array([s.axis, s.plane_index, s.direction, s.pol_axis, s.num_freqs])
        d[f"src{i}_angle_theta"] = np.array(s.angle_theta)
        d[f"src{i}_ex_inc"] = s.ex_inc
        d[f"src{i}_hy_inc"] = s.hy_inc
        d[f"src{i}_amp_int"] = s.waveform.amp_int
        d[f"src{i}_amp_half"] = s.waveform.amp_half
        d[f"src{i}_center"] = np.array(float(getattr(s, "center", float("nan"))))
    if sc.dispersion_mix is not None and sc.dispersion_mix.n_entry > 0:
        for f in _DMIX:
            d[f"dmix_{f}"] = getattr(sc.dispersion_mix, f)
    if sc.dispersion is not None and sc.dispersion.n_entry > 0:
        dd = sc.dispersion
        d.update(disp_comp=dd.comp, disp_cell=dd.cell, disp_pole_ofs=dd.pole_ofs,
                 disp_am1=dd.am1, disp_b=dd.b, disp_g=dd.g)
    if sc.modulation is not None and sc.modulation.n_entry > 0:
        mo = sc.modulation
        d.update(mod_freq=np.array(mo.freq), mod_comp=mo.comp, mod_cell=mo.cell,
                 mod_amp=mo.amp, mod_phase=mo.phase)
    if sc.tensor is not None and sc.tensor.n_entry > 0:
        for f in ("comp", "cell", "eps", "sigma"):
            d[f"tensor_{f}"] = getattr(sc.tensor, f)
    d["n_absorbers"] = np.array(len(sc.absorbers))
    for i, sl in enumerate(sc.absorbers):
        d[f"abs{i}_meta"] = np.array([sl.axis, sl.g0])
        d[f"abs{i}_decay_int"] = sl.decay_int
        d[f"abs{i}_decay_half"] = sl.decay_half
    d["n_mode_sources"] = np.array(len(sc.mode_sources))
    for i, m in enumerate(sc.mode_sources):
        d[f"msrc{i}_meta"] = np.array([m.plane_index, m.direction, m.axis])
        d[f"msrc{i}_n_eff"] = np.array([complex(m.n_eff).real, complex(m.n_eff).imag])
        for f in ("ey_inc", "ez_inc", "hy_inc", "hz_inc", "amp_e", "amp_h"):
            d[f"msrc{i}_{f}"] = getattr(m, f)
        for f in _MSRC_BB:
            if getattr(m, f, None) is not None:
                d[f"msrc{i}_{f}"] = getattr(m, f)
    d["n_tfsf"] = np.array(len(sc.tfsf_sources))
    for i, t in enumerate(sc.tfsf_sources):
        d[f"tfsf{i}_meta"] = np.array([t.direction, *t.box_lo, *t.box_hi, t.inj, t.col0,
                                       t.num_freqs, t.axis, sum(1 << q for q in t.open_axes)])
        d[f"tfsf{i}_pol"] = np.array([t.pol_u, t.pol_v], dtype=np.float64)
        for f in ("dl1", "eps1", "ex_inc", "hy_inc"):
            d[f"tfsf{i}_{f}"] = getattr(t, f)
        if getattr(t, "sigma1", None) is not None:
            d[f"tfsf{i}_sigma1"] = t.sigma1
        if getattr(t, "k_hat", None) is not None:
            d[f"tfsf{i}_obl"] = np.array([*t.k_hat, *t.e_hat, t.dl1_step, t.proj0, t.n_col_e,
                                          t.amp_scale], dtype=np.float64)
        d[f"tfsf{i}_amp_int"] = t.waveform.amp_int
        d[f"tfsf{i}_amp_half"] = t.waveform.amp_half
    d["mon_names"] = np.array([m.name for m in sc.flux_monitors])
    for i, m in enumerate(sc.flux_monitors):
        d[f"mon{i}_meta"] = np.array([m.axis, m.plane_index, m.normal_dir])
        d[f"mon{i}_freqs"] = m.freqs
        d[f"mon{i}_spectrum"] = m.source_spectrum
        if m.transverse is not None:
            d[f"mon{i}_transverse"] = np.array(m.transverse)
        if m.apodization is not None:
            d[f"mon{i}_apod"] = _apod_pack(m.apodization)
        if getattr(m, "t_bounds", None) is not None:
            d[f"mon{i}_tbounds"] = np.array(m.t_bounds, dtype=np.float64)
    d["fmon_names"] = np.array([m.name for m in sc.field_monitors])
    for i, m in enumerate(sc.field_monitors):
        d[f"fmon{i}_meta"] = np.array([*m.origin, *m.box, *m.interval_space])
        d[f"fmon{i}_freqs"] = m.freqs
        if m.apodization is not None:
            d[f"fmon{i}_apod"] = _apod_pack(m.apodization)
    d["modemon_names"] = np.array([m.name for m in sc.mode_monitors])
    d["modemon_planes"] = np.array([m.plane_name for m in sc.mode_monitors])
    d["pmon_names"] = np.array([m.name for m in sc.permittivity_monitors])
    for i, m in enumerate(sc.permittivity_monitors):
        d[f"pmon{i}_meta"] = np.array([*m.origin, *m.box])
        d[f"pmon{i}_freqs"] = m.freqs
    d["projmon_names"] = np.array([m.name for m in sc.projection_monitors])
    for i, m in enumerate(sc.projection_monitors):
        d[f"projmon{i}_surfaces"] = np.array(m.surface_names)
        d[f"projmon{i}_dirs"] = np.array(m.normal_dirs)
    d["bfmon_names"] = np.array([m.name for m in sc.box_flux_monitors])
    for i, m in enumerate(sc.box_flux_monitors):
        d[f"bfmon{i}_faces"] = np.array(m.face_names)
    d["tmon_names"] = np.array([m.name for m in sc.field_time_monitors])
    for i, m in enumerate(sc.field_time_monitors):
        d[f"tmon{i}_meta"] = np.array([m.step_begin, m.step_end, m.interval, m.num_slots])
        d[f"tmon{i}_comps"] = np.array(m.comps)
        d[f"tmon{i}_origin"] = np.array(m.origin)
        d[f"tmon{i}_box"] = np.array(m.box)
    d["ftmon_names"] = np.array([m.name for m in sc.flux_time_monitors])
    for i, m in enumerate(sc.flux_time_monitors):
        d[f"ftmon{i}_meta"] = np.array([m.axis, m.plane_index, m.normal_dir, m.step_begin,
                                        m.step_end, m.interval, m.num_slots])
        d[f"ftmon{i}_frac"] = np.array(m.frac)
        d[f"ftmon{i}_tbounds"] = np.array(m.t_bounds, dtype=np.float64)
    d["n_dipoles"] = np.array(len(sc.dipoles))
    for i, dd in enumerate(sc.dipoles):
        d[f"dip{i}_component"] = np.array(dd.component)
        d[f"dip{i}_indices"] = dd.indices
        d[f"dip{i}_coef"] = dd.coef
        d[f"dip{i}_amp_int"] = dd.waveform.amp_int
        d[f"dip{i}_amp_half"] = dd.waveform.amp_half
        d[f"dip{i}_amp_int_im"] = np.asarray(dd.waveform.amp_int_complex).imag
        if dd.waveform.amp_half_complex is not None:
            d[f"dip{i}_amp_half_im"] = np.asarray(dd.waveform.amp_half_complex).imag
        d[f"dip{i}_magnetic"] = np.array(int(dd.magnetic))
    p = pathlib.Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_name(p.name + f".{os.getpid()}.part")
    with open(tmp, "wb") as f:
        np.savez_compressed(f, **d)
    os.replace(tmp, p)
    return p
