"""Generate the golden fixtures under ``tests/golden/`` from OpenEM's own CPU code.

Run with ``OPENEM_SRC`` set to a checkout of the OpenEM sources. Only OpenEM's numpy modules are imported -- ``openem.cpml``, ``openem.grid``,
``openem.model``, ``openem.serialize``, ``openem.tfsf1d`` (its numpy loop), ``openem.shutoff``,
``openem.apodization``, ``openem.flux`` -- none of which need cupy, tidy3d or a GPU. The engine's
own scene factory supplies the scenes, converted field by field into OpenEM's classes.

    OPENEM_SRC=<openem checkout> python tests/golden/gen_golden.py [tables tfsf1d shutoff scenes]

Outputs (all small):
    ref_tables.npz     CPML coefficients, axis index tables, dual spacings, apodisation windows,
                       plane flux of fixed phasors
    ref_tfsf1d.npz     the 1D Yee line with one-face injection (lossless slab and lossy profile)
    ref_postprocess.npz  Tidy3D-convention divisors per source type, colocation and the field
                       readout (openem.normalize, openem.colocate, openem.td_readout)
    ref_shutoff.npz    early-termination decisions on two fixed metric sequences (the decay
                       tests fire; the flux test fires while the energy decays slowly)
    ref_scene_slab.npz, ref_scene_disp.npz   scene.npz files written by OpenEM's serializer
"""

from __future__ import annotations

import dataclasses
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
SRC = os.environ.get("OPENEM_SRC")
if not SRC:
    sys.exit("set OPENEM_SRC to a checkout of the OpenEM sources")
sys.path.insert(0, str(ROOT))
sys.path.insert(0, SRC)

import openem.apodization as r_apod  # noqa: E402
import openem.colocate as r_coloc  # noqa: E402
import openem.normalize as r_norm  # noqa: E402
import openem.td_readout as r_tdr  # noqa: E402
import openem.cpml as r_cpml  # noqa: E402
import openem.flux as r_flux  # noqa: E402
import openem.grid as r_grid  # noqa: E402
import openem.model as r_model  # noqa: E402
import openem.serialize as r_ser  # noqa: E402
import openem.shutoff as r_shut  # noqa: E402
import openem.tfsf1d as r_tfsf1d  # noqa: E402
import openem.waveform as r_wave  # noqa: E402

from openem_b200 import scenes  # noqa: E402
from openem_b200.model import GaussianPulse, PMLParams  # noqa: E402

_REF_MODULES = (r_model, r_grid, r_cpml, r_wave)


def to_ref(obj):
    """Rebuild an engine model object as the OpenEM class of the same name, recursively."""
    if dataclasses.is_dataclass(obj) and not isinstance(obj, type):
        name = type(obj).__name__
        cls = next(getattr(m, name) for m in _REF_MODULES if hasattr(m, name))
        kw = {f.name: to_ref(getattr(obj, f.name)) for f in dataclasses.fields(obj)}
        return cls(**kw)
    if isinstance(obj, dict):
        return {k: to_ref(v) for k, v in obj.items()}
    if isinstance(obj, list):
        return [to_ref(v) for v in obj]
    return obj


def gen_tables(out: dict) -> None:
    dt = 3.8131497390619744e-17
    cases = [("a", PMLParams(12), 0.02e-6, 1.0),
             ("b", PMLParams(8, sigma_max=2.0, kappa_max=5.0, alpha_max=0.1, alpha_min=0.01),
              0.015e-6, 0.5)]
    for tag, p, dl, spd in cases:
        rp = r_cpml.PMLParams(**dataclasses.asdict(p))
        for side in ("lo", "hi"):
            c = r_cpml.build(rp, dl, side, dt, avg_speed=spd)
            for f in ("a_E", "b_E", "inv_kappa_E", "a_H", "b_H", "inv_kappa_H"):
                out[f"cpml_{tag}_{side}_{f}"] = getattr(c, f)
        out[f"cpml_{tag}_dl"] = np.array(dl)
        out[f"cpml_{tag}_spd"] = np.array(spd)
    out["cpml_dt"] = np.array(dt)
    rng = np.random.default_rng(7)
    edges = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, 17))]) * 1e-8
    for tag, lo, hi, k in (("per", "Periodic", "Periodic", 0.0),
                           ("pml", "PML", "PML", 0.0),
                           ("pmc", "PMCBoundary", "PMCBoundary", 0.0),
                           ("blo", "BlochBoundary", "BlochBoundary", 0.15)):
        ax = r_grid.Axis(edges, lo, hi)
        t = ax.index_tables(k)
        for key, v in t.items():
            out[f"axis_{tag}_{key}"] = v
        out[f"axis_{tag}_dl_dual"] = ax.dl_dual
    out["axis_edges"] = edges
    t = np.linspace(0, 1e-12, 501)
    for tag, spec in (("none", None), ("both", (2e-13, 7e-13, 5e-14)),
                      ("start", (3e-13, None, 1e-13))):
        out[f"apod_{tag}"] = r_apod.window(t, spec)
    out["apod_t"] = t
    sc = scenes.slab_plane_wave(nxy=4, num_steps=10)
    grid = to_ref(sc.grid)
    data = (rng.standard_normal((4, 3, 4, 4)) + 1j * rng.standard_normal((4, 3, 4, 4)))
    out["flux_data"] = data
    out["flux_val"] = r_flux.plane_flux(data, grid, axis=2)


def gen_tfsf1d(out: dict) -> None:
    dl = 0.02e-6
    n1 = 760
    dt = 0.99 * dl / (scenes.C_0 * np.sqrt(3.0))
    n_steps = 240
    pulse = GaussianPulse(freq0=3e14, fwidth=1e14)
    for tag, lossy in (("ll", False), ("ls", True)):
        dl1 = np.full(n1, dl)
        eps1 = np.ones(n1)
        eps1[410:440] = 4.0
        sigma1 = None
        if lossy:
            sigma1 = np.zeros(n1)
            sigma1[420:480] = 2e4
        inj = 380
        ex_inc, hy_inc = scenes.plane_wave_tables(pulse, dt, n_steps, 0.5 * dl, 1.0, +1)
        ex_tab, hy_tab = r_tfsf1d.tables(dl1, eps1, dt, inj, +1, ex_inc, hy_inc, n_steps,
                                         col0=400, n_col_e=40, sigma1=sigma1)
        out[f"{tag}_dl1"] = dl1
        out[f"{tag}_eps1"] = eps1
        out[f"{tag}_sigma1"] = np.zeros(n1) if sigma1 is None else sigma1
        out[f"{tag}_ex_inc"] = ex_inc
        out[f"{tag}_hy_inc"] = hy_inc
        out[f"{tag}_ex_tab"] = ex_tab
        out[f"{tag}_hy_tab"] = hy_tab
    out["dt"] = np.array(dt)
    out["inj"] = np.array(380)
    out["col0"] = np.array(400)
    out["n_col_e"] = np.array(40)
    out["n_steps"] = np.array(n_steps)


def _shutoff_sequence(steps, e2, energy, flux, prefix: str, out: dict) -> None:
    pol = r_shut.default_policy(1e-5, interval=400)
    fired, ratios, taus, rels = [], [], [], []
    for s, a, b, f in zip(steps, e2, energy, flux):
        fired.append(bool(pol.check(int(s), float(a), float(b), f)))
        ratios.append(pol.field_decay.ratio)
        taus.append(pol.energy_decay.tau)
        rels.append(pol.phasor.rel)
    out.update({prefix + "steps": steps, prefix + "e2": e2, prefix + "energy": energy,
                prefix + "flux": flux, prefix + "fired": np.array(fired),
                prefix + "ratio": np.array(ratios), prefix + "tau": np.array(taus),
                prefix + "rel": np.array(rels), prefix + "reason": np.array(pol.reason)})


def gen_shutoff(out: dict) -> None:
    rng = np.random.default_rng(11)
    steps = np.arange(1, 41) * 400
    env = np.exp(-((steps - 3000.0) / 1500.0) ** 2) + 1e-9
    e2 = env * (1.0 + 0.3 * np.cos(0.01 * steps)) * 1e-3
    energy = env * 2e-3
    flux = np.stack([1.0 - np.exp(-steps / 4000.0), 0.5 - 0.4 * np.exp(-steps / 3000.0)], 1)
    flux += 1e-6 * rng.standard_normal(flux.shape)
    _shutoff_sequence(steps, e2, energy, flux, "", out)
    # a slowly ringing resonance: the energy decays by ~1e-3 over the run (no decay test
    # fires) while the fluxes settle, so the flux test fires on its own
    steps = np.arange(1, 61) * 400
    ring = np.exp(-steps / 3500.0)
    energy = 1e-3 * (np.minimum(steps / 2000.0, 1.0) * ring + 1e-4)
    e2 = energy * (1.0 + 0.2 * np.sin(0.003 * steps))
    flux = np.stack([0.8 - 0.3 * ring, 0.1 + 0.05 * ring, -0.2 + 0.1 * ring], 1)
    flux += 1e-9 * rng.standard_normal(flux.shape)
    _shutoff_sequence(steps, e2, energy, flux, "b_", out)


def post_scenes():
    """One scene per normalising source type, built by the engine's scene factory."""
    return {
        "dip": scenes.small_dispersive(n=20, n_sph=2, num_steps=300, n_pml=6, nfreq=3),
        "pw": scenes.slab_plane_wave(nxy=3, num_steps=600),
        "mode": scenes.bloch_metasurface(nx=8, ny=8, nz=64, n_pml=8, npix=2, layer_cells=8,
                                         nfreq=5, num_steps=400, bloch_k=(0.05, 0.0, 0.0)),
        "tfsf": scenes.tfsf_box_scene(n=24, n_pml=6, num_steps=300),
    }


def gen_postprocess(out: dict) -> None:
    rng = np.random.default_rng(17)
    for tag, sc in post_scenes().items():
        rsc = to_ref(sc)
        freqs = np.linspace(1.5e14, 3.5e14, 7)
        out[f"{tag}_freqs"] = freqs
        out[f"{tag}_D"] = r_norm.norm_spectrum(rsc, freqs)
        out[f"{tag}_field"] = r_norm.field_norm(rsc, freqs)
        out[f"{tag}_flux"] = r_norm.flux_norm(rsc, freqs)
        if tag == "pw":
            m = rsc.flux_monitors[0]
            out["pw_bg"] = np.array(r_norm.background_index(rsc))
            out["pw_area"] = np.array(r_norm.monitor_area(rsc, m))
            out["pw_plane_div"] = r_norm.plane_flux_divisor(rsc, m, freqs)
            pulse = GaussianPulse(freq0=2.998e14, fwidth=0.2 * 2.998e14)
            out["pw_tscale"] = np.array(r_norm.time_scale(rsc, pulse, sc.dt, 600))
    # colocation of random data from Yee positions to primal edges (and a single-point axis)
    sc = post_scenes()["dip"]
    rsc = to_ref(sc)
    origin, box = (3, 4, 5), (6, 5, 4)
    data = rng.standard_normal((2, 6, 5, 4)) + 1j * rng.standard_normal((2, 6, 5, 4))
    out["col_data"] = data
    for comp in ("Ex", "Hy", "Ez"):
        src = r_coloc.sample_coords(rsc.grid, origin, box, comp)
        dst = [np.asarray(rsc.grid.axes[a].edges)[origin[a]:origin[a] + box[a]] for a in range(3)]
        dst[2] = dst[2][1:2]
        out[f"col_{comp}"] = r_coloc.interp_to(data, src, dst)
    out["col_snap"] = np.array([r_coloc.snap_floor(rsc.grid.axes[0].edges, c, 1e-15)
                                for c in (-1e-6, 0.0, 3.3e-8, 1e-3)])
    # the field readout of the dipole scene's mid-plane monitor with primal-edge targets
    m = rsc.field_monitors[0]
    nf = int(np.size(m.freqs))
    raw = (rng.standard_normal((6, nf) + tuple(m.box))
           + 1j * rng.standard_normal((6, nf) + tuple(m.box)))
    plans = {}
    for comp in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        for a, ax in enumerate("xyz"):
            e = np.asarray(rsc.grid.axes[a].edges)[m.origin[a]:m.origin[a] + m.box[a]] / 1e-6
            plans[f"{m.name}|{comp}:{ax}"] = e if m.box[a] > 2 else e[:1]
    fin = r_tdr.finalize(rsc, {m.name: raw}, plans)
    out["tdr_raw"] = raw
    for k, v in plans.items():
        out["plan|" + k] = v
    for k, v in fin.items():
        out["fin|" + k] = v


def main(which) -> None:
    if "tables" in which:
        d: dict = {}
        gen_tables(d)
        np.savez_compressed(HERE / "ref_tables.npz", **d)
    if "tfsf1d" in which:
        d = {}
        gen_tfsf1d(d)
        np.savez_compressed(HERE / "ref_tfsf1d.npz", **d)
    if "shutoff" in which:
        d = {}
        gen_shutoff(d)
        np.savez_compressed(HERE / "ref_shutoff.npz", **d)
    if "postprocess" in which:
        d = {}
        gen_postprocess(d)
        np.savez_compressed(HERE / "ref_postprocess.npz", **d)
    if "scenes" in which:
        slab = scenes.slab_plane_wave(nxy=2, num_steps=400)
        r_ser.save(to_ref(slab), HERE / "ref_scene_slab.npz")
        disp = scenes.with_time_monitor(scenes.small_dispersive(n=20, n_sph=2, num_steps=60,
                                                                n_pml=6, nfreq=3), interval=7)
        r_ser.save(to_ref(disp), HERE / "ref_scene_disp.npz")
    for p in sorted(HERE.glob("ref_*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main(sys.argv[1:] or ("tables", "tfsf1d", "shutoff", "postprocess", "scenes"))
