"""Host-side logic without a GPU: the scene.npz boundary, table construction, the C ABI library
(loads and exports every declared symbol), fail-closed refusal of unsupported physics."""

import dataclasses
import pathlib
import re
from dataclasses import replace

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import model as M
from openem_b200 import scenes, serialize, solver
from openem_b200 import tables as T

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"


def _eq(a, b, path="scene"):
    """Recursive equality of two model objects (arrays bit-exact)."""
    if dataclasses.is_dataclass(a):
        assert type(a).__name__ == type(b).__name__, path
        for f in dataclasses.fields(a):
            _eq(getattr(a, f.name), getattr(b, f.name), f"{path}.{f.name}")
    elif isinstance(a, dict):
        assert set(a) == set(b), path
        for k in a:
            _eq(a[k], b[k], f"{path}[{k}]")
    elif isinstance(a, (list, tuple)) and not isinstance(a, np.ndarray):
        assert len(a) == len(b), path
        for q, (x, y) in enumerate(zip(a, b)):
            _eq(x, y, f"{path}[{q}]")
    elif a is None or b is None:
        assert a is None and b is None, path
    elif isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b), err_msg=path)
    elif isinstance(a, float) and np.isnan(a):
        assert np.isnan(b), path
    else:
        assert a == b, path


@pytest.mark.parametrize("fname,build", [
    ("ref_scene_slab.npz", lambda: scenes.slab_plane_wave(nxy=2, num_steps=400)),
    ("ref_scene_disp.npz", lambda: scenes.with_time_monitor(
        scenes.small_dispersive(n=20, n_sph=2, num_steps=60, n_pml=6, nfreq=3), interval=7)),
])
def test_reads_scene_npz_written_by_openem(fname, build, tmp_path):
    """OpenEM's serializer wrote these files from the same scenes; they load field for field,
    and a round trip through this engine's writer is lossless."""
    loaded = serialize.load(GOLD / fname)
    want = build()
    for f in ("dt", "num_time_steps", "shutoff", "eps_ex", "eps_ey", "eps_ez", "sigma_ex",
              "dispersion", "pml", "dipoles", "flux_monitors", "field_monitors",
              "field_time_monitors"):
        got, ref = getattr(loaded, f), getattr(want, f)
        if f == "dipoles":  # the npz stores the complex tables as real + imaginary parts
            for a, b in zip(got, ref):
                _eq(a.indices, b.indices)
                _eq(a.coef, b.coef)
                _eq(a.waveform.amp_half, b.waveform.amp_half)
            continue
        _eq(got, ref, f)
    serialize.save(loaded, tmp_path / "again.npz")
    _eq(serialize.load(tmp_path / "again.npz"), loaded)


def test_material_tables_reconstruct_coefficients():
    sc = scenes.small_dispersive(n=24, n_sph=3, n_pml=6, num_steps=20)
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    mt = T.material_tables(sc, tabs)
    o = ref64.Oracle(sc, 5)
    idx = mt.index.astype(np.int64)
    for c in range(3):
        px, py, pz = (o._bc(o.pec[a], a) for a in range(3))
        mask = {0: py * pz, 1: pz * px, 2: px * py}[c]
        np.testing.assert_array_equal(mt.table[:, c].view(np.float32)[idx],
                                      (o.ca[c] * mask).astype(np.float32))
        np.testing.assert_array_equal(mt.table[:, 3 + c].view(np.float32)[idx],
                                      (o.cb[c] * mask).astype(np.float32))
    # poles: total count and per-segment offsets agree with the dense count
    assert mt.n_pole_total == sc.dispersion.n_pole
    npc = np.zeros((sc.shape[0], sc.shape[1], T.pad_z(sc.shape[2])), np.int64)
    npc[..., :sc.shape[2]] = sum(mt.table[:, 12 + c].view(np.int32)[idx] for c in range(3))
    seg = npc.reshape(-1, 32).sum(1)
    np.testing.assert_array_equal(mt.seg_ofs, np.concatenate([[0], np.cumsum(seg)[:-1]]))


def test_pole_sets_deduplicate_identical_coefficients():
    sc = scenes.small_dispersive(n=24, n_sph=3, n_pml=6, num_steps=20)
    comp, cell, set_id, set_ofs, coef, counts = T.entry_pole_sets(sc)
    assert set_ofs.tolist() == [0, 2] and counts.tolist() == [2]
    assert np.all(set_id == 0)
    d = sc.dispersion
    d2 = replace(d, b=d.b * np.repeat(np.linspace(0.5, 1.0, d.n_entry), 2))
    _, _, sid2, ofs2, coef2, counts2 = T.entry_pole_sets(replace(sc, dispersion=d2))
    assert counts2.size == np.unique(np.linspace(0.5, 1.0, d.n_entry).astype(np.float32)).size
    assert np.all(sid2 >= 0)


def test_plane_source_coefficients():
    sc = scenes.slab_plane_wave(nxy=1, num_steps=50)
    (ps,) = T.plane_sources(sc)
    az = sc.grid.z
    assert ps["kh"] == ps["ks"] - 1
    assert ps["coef_h"] == float(np.float32(sc.dt / T.MU_0 / az.dl[ps["kh"]]))
    assert ps["coef_e"] == float(np.float32(1.0 / az.dl_dual[ps["ks"]]))


def test_phase_table():
    f = np.array([1e14, 2e14])
    ph = T.phase_table(f, 1e-17, 5, (None, 2e-17, 1e-17))
    n = np.arange(5)
    we = T.apod_window((n + 1) * 1e-17, (None, 2e-17, 1e-17))
    np.testing.assert_allclose(ph[:, 1, 0], (np.cos(2 * np.pi * 2e14 * (n + 1) * 1e-17) * we)
                               .astype(np.float32), rtol=1e-6)
    assert ph.dtype == np.float32 and ph.shape == (5, 2, 4)


@pytest.mark.parametrize("feature", ["tfsf", "disp_in_absorber", "modulation_pec", "tensor",
                                     "mix_in_absorber", "mix_tensor", "mix_modulation"])
def test_unsupported_physics_fails_closed(feature):
    sc = scenes.slab_plane_wave(nxy=1, num_steps=10)
    sd = scenes.small_dispersive(n=20, n_sph=1, n_pml=4, num_steps=10)
    ms = replace(scenes.mixed_sphere(n=20, n_pml=4, radius_cells=3.3, num_steps=10),
                 dispersion=None)
    solver.refuse_unsupported(ms)
    bad = {
        "mix_in_absorber": replace(ms, absorbers=scenes.absorber_slabs(ms.grid, 0, 10)),
        "mix_tensor": replace(ms, tensor=M.TensorEps(np.array([0]), np.array([0]),
                                                     np.eye(3)[None], np.zeros((1, 3, 3)))),
        "mix_modulation": replace(ms, modulation=M.TimeModulation(
            1e14, np.array([0]), np.array([0]), np.array([0.1]), np.array([0.0]))),
        "tfsf": replace(sc, tfsf_sources=[replace(
            scenes.tfsf_box_scene(n=30, num_steps=10).tfsf_sources[0], open_axes=(0,))]),
        "disp_in_absorber": replace(sd, absorbers=scenes.absorber_slabs(sd.grid, 0, 10)),
        "modulation_pec": replace(sc, pec_ex=np.array([5]), modulation=M.TimeModulation(
            1e14, np.array([0]), np.array([0]), np.array([0.1]), np.array([0.0]))),
        "tensor": replace(sd, tensor=M.TensorEps(np.array([0]), np.array([0]),
                                                  np.eye(3)[None], np.zeros((1, 3, 3)))),
    }[feature]
    with pytest.raises(NotImplementedError):
        solver.refuse_unsupported(bad)


@pytest.mark.parametrize("feature", ["plane", "dispersion", "loss", "nosource"])
def test_bloch_subset_fails_closed(feature):
    """The complex path refuses what OpenEM's does (openem/solver.py:1221-1260)."""
    sd = scenes.small_dispersive(n=20, n_sph=1, n_pml=4, num_steps=10)
    plain = replace(sd, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    bad = {
        "plane": scenes.slab_plane_wave(nxy=1, num_steps=10),
        "dispersion": replace(sd, sigma_ex=None, sigma_ey=None, sigma_ez=None),
        "loss": replace(sd, dispersion=None),
        "nosource": replace(plain, dipoles=[]),
    }[feature]
    with pytest.raises(NotImplementedError):
        solver.refuse_unsupported_bloch(bad)
    solver.refuse_unsupported_bloch(plain)


@pytest.mark.parametrize("feature", ["absorber", "bloch", "mix", "tensor", "modulation"])
def test_adjoint_fails_closed(feature):
    """The discrete adjoint covers real scenes with pole-residue dispersion, without absorbers,
    slanted-interface mixed media, tensor media or time modulation; the rest is refused before
    anything reaches the device."""
    from openem_b200 import adjoint
    sd = scenes.small_dispersive(n=20, n_sph=1, n_pml=4, num_steps=10)
    plain = replace(sd, dispersion=None)
    adjoint._refuse(sd)  # pole-residue dispersion is covered
    bad = {
        "mix": replace(scenes.mixed_sphere(n=20, n_pml=4, radius_cells=3.3, num_steps=10),
                       dispersion=None),
        "tensor": replace(plain, tensor=M.TensorEps(np.array([0]), np.array([0]),
                                                    np.eye(3)[None], np.zeros((1, 3, 3)))),
        "modulation": replace(plain, modulation=M.TimeModulation(
            1e14, np.array([0]), np.array([0]), np.array([0.1]), np.array([0.0]))),
        "absorber": replace(plain, absorbers=scenes.absorber_slabs(plain.grid, 0, 3)),
        "bloch": replace(plain, bloch_k=(0.1, 0.0, 0.0)),
    }[feature]
    with pytest.raises(NotImplementedError):
        adjoint._refuse(bad)
    adjoint._refuse(plain)


def test_adjoint_coefficient_jacobian_matches_differences():
    """d(ca, cb)/d(eps, sigma) of the float64 coefficient formula against central
    differences."""
    from openem_b200 import adjoint
    sd = scenes.small_dispersive(n=12, n_sph=1, n_pml=3, num_steps=10)
    sc = replace(sd, dispersion=None)
    jac = adjoint.coefficient_jacobian(sc)
    eps0 = T.EPSILON_0
    c, cell = 1, (5, 6, 7)
    e = float(np.asarray(sc.eps_ey)[cell])
    sg = 0.0 if sc.sigma_ey is None else float(np.asarray(sc.sigma_ey)[cell])
    G = float(T._g_dense(sc, sc.shape)[c][cell])

    def coef(ev, sv):
        s = sv * sc.dt / (2 * eps0)
        den = ev + s + G
        return (ev - s) / den, (sc.dt / eps0) / den
    h = 1e-6
    ca_p, cb_p = coef(e + h, sg)
    ca_m, cb_m = coef(e - h, sg)
    np.testing.assert_allclose(jac[c][0][cell], (ca_p - ca_m) / (2 * h), rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(jac[c][1][cell], (cb_p - cb_m) / (2 * h), rtol=1e-6)
    hs = 1e-3
    ca_p, cb_p = coef(e, sg + hs)
    ca_m, cb_m = coef(e, sg - hs)
    np.testing.assert_allclose(jac[c][2][cell], (ca_p - ca_m) / (2 * hs), rtol=1e-6)
    np.testing.assert_allclose(jac[c][3][cell], (cb_p - cb_m) / (2 * hs), rtol=1e-6)


def test_modulation_tables():
    """Per-step (cos, sin) rows at t_n and t_n+1 in float64 narrowed to float32, entries on a
    PEC-backed wall dropped, eps_s - |amp| <= 0 and PEC cells refused
    (openem/sources_setup.py:460-518, 640-650)."""
    sc = scenes.modulated_slab(nxy=2, num_steps=50, phase=lambda x, y, z: 3e6 * x)
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    md = T.modulation_tables(sc, tabs, 50)
    om = 2 * np.pi * sc.modulation.freq
    n = np.arange(50.0)
    np.testing.assert_array_equal(md["cs"][:, 0], np.cos(om * n * sc.dt).astype(np.float32))
    np.testing.assert_array_equal(md["cs"][:, 3], np.sin(om * (n + 1) * sc.dt).astype(np.float32))
    assert md["comp"].size == sc.modulation.n_entry
    assert np.ptp(md["cph"]) > 0
    with pytest.raises(ValueError):
        T.modulation_tables(replace(sc, modulation=replace(
            sc.modulation, amp=np.full(sc.modulation.n_entry, 1.5))), tabs, 50)
    with pytest.raises(NotImplementedError):
        T.modulation_tables(replace(sc, pec_ex=np.array([0])), tabs, 50)
    # a PEC-backed z wall: the tangential entries on it keep ca = cb = 0
    ax = sc.grid.axes
    g2 = M.Grid(ax[0], ax[1], M.Axis(ax[2].edges, "PEC", "PEC"))
    nz = sc.shape[2]
    mo = M.TimeModulation(sc.modulation.freq, np.array([0, 2]), np.array([0, 0]),
                          np.array([0.1, 0.1]), np.zeros(2))
    sc2 = replace(sc, grid=g2, pml={}, modulation=mo)
    tabs2 = [T.axis_tables(sc2, a) for a in range(3)]
    md2 = T.modulation_tables(sc2, tabs2, 5)
    assert md2["comp"].tolist() == [2] and nz > 0


def test_isolate_cells_gives_each_cell_its_own_record():
    table = np.arange(3 * 16, dtype=np.uint32).reshape(3, 16)
    index = np.array([[0, 1, 1], [2, 1, 0]], dtype=np.uint16)
    t2, i2, n = T.isolate_cells(table, index, np.array([1, 4, 1]))
    assert n == 5 and t2.shape == (5, 16)
    flat = i2.ravel()
    assert flat[1] == 3 and flat[4] == 4
    np.testing.assert_array_equal(t2[3], table[1])
    np.testing.assert_array_equal(t2[4], table[1])
    keep = [0, 2, 3, 5]
    np.testing.assert_array_equal(flat[keep], index.ravel()[keep])


def test_dipole_table_refuses_short_waveform():
    sc = scenes.small_dispersive(n=20, n_sph=1, n_pml=4, num_steps=30)
    with pytest.raises(ValueError):
        T.dipole_tables(sc, 100, magnetic=False)


def test_library_builds_loads_and_exports_header_symbols():
    """The C ABI library builds for sm_100a and exports every function include/oem_b200.h
    declares (no device call is made)."""
    import shutil
    if shutil.which("nvcc") is None and not pathlib.Path("/usr/local/cuda/bin/nvcc").exists():
        pytest.skip("nvcc not available")
    from openem_b200 import build, lib
    build.build()
    header = (ROOT / "include" / "oem_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|const char\*)\s+(oem_\w+)\(", header, re.M))
    assert len(declared) >= 20
    so = lib.load()
    for name in declared:
        assert hasattr(so, name), name
    assert set(lib.SIGNATURES) == declared
    assert lib.load().oem_version() >= 100


def test_bulk_pole_set_shortcut_is_exact():
    """One coefficient list on every entry takes a shortcut that converts one row; its output
    equals the general deduplication's, and a single differing entry leaves the shortcut."""
    from dataclasses import replace
    from openem_b200 import tables as T
    sd = scenes.small_dispersive(n=24, n_sph=2, n_pml=4, num_steps=10)
    for sc in (sd, replace(sd, dispersion=replace(sd.dispersion, b=np.concatenate(
            [sd.dispersion.b[:-1], sd.dispersion.b[-1:] * 1.5])))):
        a = T.entry_pole_sets(sc)
        b = T.entry_pole_sets(sc, bulk_shortcut=False)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    assert T.entry_pole_sets(sd)[3].size == 2


def test_ours_npz_round_trip(tmp_path, monkeypatch):
    """The solve worker's ``ours.npz`` keys and contents (openem/nb/solve_worker.py:25-45): flux
    phasors and frequencies, field phasors, time samples, flux time series and the run summary
    round-trip; an output above the size cap leaves only the summary; a work directory asking
    for the Tidy3D-convention readout is refused."""
    from openem_b200 import results, solve_worker
    rng = np.random.default_rng(0)
    ph = rng.normal(size=(4, 3, 5, 6)) + 1j * rng.normal(size=(4, 3, 5, 6))
    res = results.Result(
        phasors={"T": results.Phasors(name="T", data=ph, freqs=np.array([1.0, 2.0, 3.0]))},
        steps_run=123, shutoff_triggered=True, stop_reason="field decay", wall_seconds=1.5,
        source_end=40, energy_trace=[(400, 1e-3)],
        field_phasors={"box": rng.normal(size=(6, 2, 3, 3, 3)) + 0j},
        time_samples={"tm": rng.normal(size=(6, 4, 2, 2, 2)).astype(np.float32)},
        flux_time={"ft": rng.normal(size=7)})
    mb = solve_worker.save_result(res, tmp_path / "ours.npz")
    assert mb > 0
    z = np.load(tmp_path / "ours.npz")
    assert set(z.files) == {"__meta", "mon:T", "monf:T", "fld:box", "tim:tm", "ftm:ft"}
    back = solve_worker.load_result(tmp_path / "ours.npz")
    np.testing.assert_array_equal(back["phasors"]["T"][0], ph)
    np.testing.assert_array_equal(back["field_phasors"]["box"], res.field_phasors["box"])
    np.testing.assert_array_equal(back["time_samples"]["tm"], res.time_samples["tm"])
    np.testing.assert_array_equal(back["flux_time"]["ft"], res.flux_time["ft"])
    assert back["meta"] == {"steps_run": 123, "triggered": True, "stop": "field decay",
                            "wall": 1.5, "source_end": 40, "energy_trace": [[400, 1e-3]]}
    monkeypatch.setenv("OPENEM_OUT_MAX_GB", "1e-9")
    assert solve_worker.save_result(res, tmp_path / "big.npz") < 0
    assert (tmp_path / "big.TOOBIG").exists() and not (tmp_path / "big.npz").exists()
    # extra entries (the Tidy3D-convention readout) travel next to the solver's own keys
    monkeypatch.setenv("OPENEM_OUT_MAX_GB", "20")
    mb = solve_worker.save_result(res, tmp_path / "extra.npz",
                                  extra={"tdf:box|Ex": np.ones((2, 1, 1, 3), complex)})
    assert mb > 0
    with np.load(tmp_path / "extra.npz") as z:
        assert "tdf:box|Ex" in z.files and "__meta" in z.files


def test_mix_tables_and_passthrough():
    """The mixed-form tables the C-ABI receives: per entry (k1, k2, 1 - beta, 1/(k1 k2 + beta))
    in float32, CSR pole rows (Re(A-1), Im(A-1), Re(B), Im(B)), and update coefficients that
    pass the curl through on the mixed cells (ca = 0, cb = 1) while the E-form interior keeps its
    own."""
    from openem_b200 import tables as T
    sc = scenes.mixed_sphere(n=20, n_pml=4, radius_cells=3.3, num_steps=10)
    mm = sc.dispersion_mix
    mx = T.mix_tables(sc)
    k1, k2, omb, invd = mm.coefficients()
    np.testing.assert_array_equal(mx["k"], np.stack([k1, k2, omb, invd], 1).astype(np.float32))
    assert mx["pc"].shape == (mx["n_p"], 4) and mx["qc"].shape == (mx["n_q"], 4)
    np.testing.assert_array_equal(mx["pc"][:, 2], np.asarray(mm.pb).real.astype(np.float32))
    np.testing.assert_array_equal(mx["q_ofs"], np.asarray(mm.q_ofs, np.int32))
    assert mx["dte"] == pytest.approx(sc.dt / 8.8541878128e-12)
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    ca, cb = T.e_coefficients(sc, tabs)
    for c in range(3):
        cells = np.asarray(mm.cell)[np.asarray(mm.comp) == c]
        assert np.all(ca[c].ravel()[cells] == 0.0) and np.all(cb[c].ravel()[cells] == 1.0)
        inner = np.asarray(sc.dispersion.cell)[np.asarray(sc.dispersion.comp) == c]
        assert np.all(cb[c].ravel()[inner] != 1.0)


def test_tensor_tables_and_passthrough():
    """The tensor tables the C-ABI receives: per entry the float32 rows of M1 = A^-1 B and
    M2 = (dt/eps0) A^-1 of its component and the PEC-wall factor of the two other axes; the
    entries' update coefficients pass the curl through (ca = 0, cb = 1)."""
    from openem_b200 import tables as T
    sd = scenes.small_dispersive(n=20, n_sph=1, n_pml=4, num_steps=10)
    sc = replace(sd, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    ten = scenes.tensor_region(sc, (8, 8, 8), (12, 12, 12),
                               scenes.rotated_diag((4.0, 2.0, 3.0), 0.5, 1),
                               np.array([[0, 80.0, 0], [-80.0, 0, 0], [0, 0, 10.0]]))
    sc = replace(sc, tensor=ten)
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    tt = T.tensor_tables(sc, tabs)
    m1, m2 = ten.rows(sc.dt)
    np.testing.assert_array_equal(tt["m1"], m1.astype(np.float32))
    np.testing.assert_array_equal(tt["m2"], m2.astype(np.float32))
    assert np.all(tt["pec"] == 1.0)  # the block sits away from every wall
    ca, cb = T.e_coefficients(sc, tabs)
    for c in range(3):
        cells = np.asarray(ten.cell)[np.asarray(ten.comp) == c]
        assert np.all(ca[c].ravel()[cells] == 0.0) and np.all(cb[c].ravel()[cells] == 1.0)


def test_nonfinite_material_coefficients_are_named(capsys):
    """A NaN in eps reaches the deduplicated material records (ca, cb, eps); the plan names it
    at set-up from that small table, before any device work."""
    from dataclasses import replace
    from openem_b200 import tables as T
    from openem_b200.solver import Plan
    sc = scenes.small_dispersive(n=20, n_sph=2, num_steps=10, n_pml=6, nfreq=2)
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    Plan._warn_nonfinite_materials(T.material_tables(sc, tabs).table)
    assert capsys.readouterr().out == ""
    eps = np.array(sc.eps_ey)
    eps[3, 4, 5] = np.inf
    bad = replace(sc, eps_ey=eps)
    Plan._warn_nonfinite_materials(T.material_tables(bad, [T.axis_tables(bad, a) for a in range(3)]).table)
    assert "non-finite" in capsys.readouterr().out


def test_device_entry_checks_match_host_checks():
    """The device table builder checks the dispersion entry table on the device before indexing
    with it; on torch CPU tensors here, every failure gives check_csr's message and a valid
    table passes."""
    import torch
    from openem_b200 import tables_gpu as TG
    shape = (4, 5, 6)
    ncell = 120
    comp = np.array([0, 0, 1, 2], np.int64)
    cell = np.array([3, 7, 7, 119], np.int64)
    ofs = np.array([0, 2, 4, 4, 6], np.int64)
    cases = [
        (comp, cell, ofs, None),
        (np.array([0, 3, 1, 2]), cell, ofs, "comp out of range"),
        (comp, np.array([3, 7, 7, 120]), ofs, "cell out of range"),
        (comp, cell, np.array([0, 2, 1, 4, 6]), "not monotonic"),
        (comp, cell, np.array([0, 2, 4, 4, 5]), "endpoints"),
        (comp[:3], cell, ofs, "lengths differ"),
        (np.array([1, 0, 1, 2]), np.array([7, 3, 7, 119]), ofs, "duplicate"),
        (np.array([1, 0, 0, 2]), np.array([7, 3, 5, 119]), ofs, None),  # unordered, unique
    ]
    for cc, kk, oo, msg in cases:
        host_err = dev_err = None
        try:
            M.check_csr("Dispersion", shape, cc, kk, [("pole_ofs", oo, 6)])
        except ValueError as e:
            host_err = str(e)
        try:
            TG._check_entries_device("Dispersion", shape, cc, kk, [("pole_ofs", oo, 6)], torch,
                                     torch.device("cpu"))
        except ValueError as e:
            dev_err = str(e)
        assert host_err == dev_err, (msg, host_err, dev_err)
        assert (msg is None) == (host_err is None) and (msg is None or msg in host_err)


def test_sparse_material_upload_is_exact():
    """A per-cell float64 array that is mostly one value crosses as (int32 index, value) pairs
    and is filled on the device (torch CPU tensors here), bit for bit, NaN and -0.0 included; a
    varied array is copied whole. The byte counts are what was sent."""
    import torch
    from openem_b200 import tables_gpu as TG
    rng = np.random.default_rng(3)
    n = 1 << 23
    a = np.zeros(n)
    a[rng.integers(0, n, 5000)] = rng.random(5000)
    a[11] = -0.0
    a[12] = np.nan
    t, nb = TG._upload_material(a, torch, torch.device("cpu"))
    assert np.array_equal(t.numpy().view(np.uint64), a.view(np.uint64))
    assert nb == 12 * int(np.count_nonzero(a.view(np.uint64) != a.view(np.uint64)[0]))
    b = rng.random(n)
    t, nb = TG._upload_material(b, torch, torch.device("cpu"))
    assert np.array_equal(t.numpy(), b) and nb == b.nbytes
    c = np.ones(n)
    c[n // 2:] = 2.0  # half the sample is off the background: copied whole without a scan
    t, nb = TG._upload_material(c, torch, torch.device("cpu"))
    assert np.array_equal(t.numpy(), c) and nb == c.nbytes
    c = np.ones(n)
    c[rng.random(n) < 0.2] = 2.0  # a fifth of the sample off (under a quarter): the scan
    t, nb = TG._upload_material(c, torch, torch.device("cpu"))  # finds > 1/8 and copies whole
    assert np.array_equal(t.numpy(), c) and nb == c.nbytes
    nanp = np.array([0x7FF8000000000123], np.uint64).view(np.float64)[0]  # a NaN with payload
    dd = np.full(n, nanp)
    dd[5] = -0.0
    t, nb = TG._upload_material(dd, torch, torch.device("cpu"))
    assert np.array_equal(t.numpy().view(np.uint64), dd.view(np.uint64)) and nb == 12
    d = np.full(n, 2.25)
    d[:1000] = 1.0  # the first cell lies in an object: the background is the common value
    t, nb = TG._upload_material(d, torch, torch.device("cpu"))
    assert np.array_equal(t.numpy(), d) and nb == 12 * 1000


def test_hashed_material_codes_equal_exact_ranking():
    """The device table builder's one-sort material codes (a 64-bit mix of each cell's six keys,
    the distinct tuples put in lexicographic order) equal the exact ranking of the key tuples;
    torch CPU tensors here."""
    import torch
    from openem_b200 import tables_gpu as TG
    g = torch.Generator().manual_seed(1)
    n = 300_000
    keys = [(torch.randint(-3, 4, (n,), generator=g) << 40) + torch.randint(0, 3, (n,), generator=g)
            for _ in range(6)]
    keys[2][::7] = torch.iinfo(torch.int64).min  # extreme key values sort first
    n1, c1 = TG._lex_codes_hashed(keys, torch, torch.device("cpu"))
    n2, c2 = TG._lex_codes_exact(keys, torch)
    assert n1 == n2 and torch.equal(c1, c2)
    tup = torch.stack(keys, 1).numpy()
    order = np.lexsort(tup.T[::-1])
    ranks = np.empty(n, np.int64)
    ranks[order] = np.arange(n)
    first = np.unique(c2.numpy(), return_index=True)[1]
    assert (np.diff(ranks[first]) > 0).all()  # codes ascend with the tuples
