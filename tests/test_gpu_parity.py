"""CUDA engine against the FP64 oracle on the same seeded scenes.

Tolerances (fp32 fields against float64 arithmetic): final fields within 1e-5 relative L2 on
the plane-wave slab; on the resonant Drude+Lorentz scene within max(2e-5, 3 x the float32
rounding floor the oracle measures for that component); DFT phasors within 1e-4 relative L2,
slab transmission within 1e-4 absolute.
"""

import numpy as np
import pytest

from oracle import ref64
from openem_b200 import scenes, solver

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def family_err(fa, fb, names):
    """Largest per-component L2 difference relative to the norm of the whole field family
    (E or H): a component that is nearly zero by symmetry does not magnify round-off."""
    den = np.sqrt(sum(float(np.linalg.norm(fb[n].ravel())) ** 2 for n in names))
    return max(float(np.linalg.norm((fa[n] - fb[n]).ravel())) for n in names) / max(den, 1e-300)


def flux(ph):
    return 0.5 * (np.real(ph[0] * np.conj(ph[3])).sum(axis=(1, 2))
                  - np.real(ph[1] * np.conj(ph[2])).sum(axis=(1, 2)))


@pytest.fixture(scope="module")
def slab_runs():
    sc = scenes.slab_plane_wave(nxy=1)
    sc0 = scenes.slab_plane_wave(nxy=1, with_slab=False)
    return {"sc": sc, "sc0": sc0, "ref": ref64.run(sc), "ref0": ref64.run(sc0),
            "gpu": solver.run(sc, use_shutoff=False, return_fields=True, verbose=False),
            "gpu0": solver.run(sc0, use_shutoff=False, verbose=False)}


def test_slab_phasors_match_oracle(slab_runs):
    r, g = slab_runs["ref"], slab_runs["gpu"]
    for name in ("T", "R"):
        assert rel_l2(g.phasors[name].data, r.phasors[name]) < 1e-4, name


def test_slab_fields_match_oracle(slab_runs):
    """Fields while the pulse crosses the slab (step 450); once it has left the 3 um cell only
    an fp32 round-off floor remains, which is no measure of the update."""
    sc = slab_runs["sc"]
    r = ref64.run(sc, 450)
    g = solver.run(sc, num_steps=450, use_shutoff=False, return_fields=True, verbose=False)
    for nm in ("Ex", "Hy"):
        assert rel_l2(g.fields[nm], r.fields[nm]) < 1e-5, nm


def test_slab_transmission_and_energy_balance(slab_runs):
    g, g0, r, r0 = (slab_runs[k] for k in ("gpu", "gpu0", "ref", "ref0"))
    T_g = flux(g.phasors["T"].data) / flux(g0.phasors["T"].data)
    R_g = -flux(g.phasors["R"].data) / flux(g0.phasors["T"].data)
    T_r = flux(r.phasors["T"]) / flux(r0.phasors["T"])
    assert np.max(np.abs(T_g - T_r)) < 1e-4
    # OpenEM prints transmission = 0.8310044973694679 at f0 for this slab (README.md:62)
    assert abs(T_g[5] - 0.8310044973694679) < 2e-5
    assert np.all(np.abs(T_g + R_g - 1.0) < 2e-4)


def test_wide_periodic_cell_equals_narrow(slab_runs):
    """At normal incidence the 30x30 periodic cell carries the 1x1 solution in every column."""
    sc = scenes.slab_plane_wave(nxy=30, num_steps=2000)
    g = solver.run(sc, use_shutoff=False, verbose=False)
    sc1 = scenes.slab_plane_wave(nxy=1, num_steps=2000)
    g1 = solver.run(sc1, use_shutoff=False, verbose=False)
    d = g.phasors["T"].data
    assert d.shape == (4, 11, 30, 30)
    np.testing.assert_allclose(d, np.broadcast_to(g1.phasors["T"].data, d.shape), rtol=1e-6,
                               atol=1e-12 * np.abs(d).max())


@pytest.fixture(scope="module")
def disp_runs():
    sc = scenes.with_time_monitor(
        scenes.small_dispersive(n=32, n_sph=4, num_steps=300, n_pml=8, nfreq=4), interval=7)
    return {"sc": sc, "ref": ref64.run(sc),
            "gpu": solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)}


def test_dispersive_fields_match_oracle(disp_runs):
    """Each component within max(2e-5, 3 x its float32 rounding floor) of the FP64 oracle.
    The floor is measured on this scene by the oracle itself, with half-ulp float32 noise
    injected into every field value each step (``ref64.fp32_floor``); on this resonant
    Drude+Lorentz scene it reaches ~1.5e-5 for Hx/Hy and ~4.7e-5 for Hz after 300 steps."""
    r, g = disp_runs["ref"], disp_runs["gpu"]
    floor = ref64.fp32_floor(disp_runs["sc"], clean=r)
    for nm in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert rel_l2(g.fields[nm], r.fields[nm]) < max(2e-5, 3.0 * floor[nm]), (nm, floor[nm])


def test_dispersive_field_monitors_match_oracle(disp_runs):
    r, g = disp_runs["ref"], disp_runs["gpu"]
    for name, data in r.field_phasors.items():
        assert g.field_phasors[name].shape == data.shape
        assert rel_l2(g.field_phasors[name], data) < 1e-4, name


def test_time_monitor_matches_oracle(disp_runs):
    r, g = disp_runs["ref"], disp_runs["gpu"]
    assert g.time_slots == r.time_slots
    for name, data in r.time_samples.items():
        assert rel_l2(g.time_samples[name], data) < 2e-5, name


def test_dispersion_changes_the_result(disp_runs):
    """The ADE is really active: dropping the poles (and the Drude conductivity) moves the
    fields by far more than the tolerance."""
    from dataclasses import replace
    sc = disp_runs["sc"]
    g = disp_runs["gpu"]
    plain = replace(sc, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    gp = solver.run(plain, use_shutoff=False, return_fields=True, verbose=False)
    assert rel_l2(gp.fields["Ez"], g.fields["Ez"]) > 1e-2


@pytest.mark.parametrize("kind", ["stream", "tma", "ws"])
@pytest.mark.parametrize("n,n_pml", [(40, 8), (42, 8), (44, 6)])
def test_pipelined_kernels_equal_basic_kernels(monkeypatch, kind, n, n_pml):
    """Each pipelined kernel pair does the arithmetic of the one-thread-per-cell kernels per
    cell; their results agree to float32 round-off. CPML depth 8 has its z-slab psi staged in
    shared memory, depth 6 read directly; 42 cells leave a partial tile of rows."""
    sc = scenes.small_dispersive(n=n, n_sph=5, num_steps=120, n_pml=n_pml, nfreq=3)
    monkeypatch.setenv("OEM_B200_KERNELS", "basic")
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    monkeypatch.setenv("OEM_B200_KERNELS", kind)
    b = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    assert family_err(b.fields, a.fields, ("Ex", "Ey", "Ez")) < 1e-6
    assert family_err(b.fields, a.fields, ("Hx", "Hy", "Hz")) < 1e-6
    for name in a.field_phasors:
        assert rel_l2(b.field_phasors[name], a.field_phasors[name]) < 1e-6, name


@pytest.mark.parametrize("n", [42, 48])
def test_box_snapshots_in_e_update_equal_snapshot_kernel(monkeypatch, n):
    """With OEM_B200_SNAP=update the E update writes the box monitors' snapshot rows itself (E
    from its registers, H from its staged tile) and the E dipoles rewrite the rows of their
    targets: the phasors equal, bit for bit, those of the separate snapshot kernel (the
    default). The centre dipole lies inside all three boxes; 42 cells leave partial tiles in y
    and z."""
    monkeypatch.setenv("OEM_B200_KERNELS", "ws")
    sc = scenes.dispersive_spheres(n=n, n_sph=3, num_steps=150, nfreq=3,
                                   rmin=0.05 * scenes.UM, rmax=0.1 * scenes.UM)
    dip = sc.dipoles[0]
    h = n // 2
    idx = np.asarray(dip.indices)
    assert ((idx >= h - 1) & (idx <= h)).all()  # the dipole's cells lie in every box
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    monkeypatch.setenv("OEM_B200_SNAP", "update")
    b = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    plan = solver.Plan(sc, 10)
    assert plan.box_snapshots_in_update() == 3
    plan.close()
    assert set(a.field_phasors) == {"mid_x", "mid_y", "mid_z"}
    for name in a.field_phasors:
        np.testing.assert_array_equal(b.field_phasors[name], a.field_phasors[name])
    for nm in a.fields:
        np.testing.assert_array_equal(b.fields[nm], a.fields[nm])
    assert float(np.abs(a.field_phasors["mid_z"]).max()) > 0.0


@pytest.mark.parametrize("n", [42, 128])
def test_pole_pass_ahead_equals_inline(monkeypatch, n):
    """Each step's pole pass run at the end of the step before it, beside the DFT snapshots
    (the default on the warp-specialised kernels), gives the same fields and phasors, bit for
    bit, as the pole pass beside the H update of its own step (OEM_B200_ADE=inline), over runs
    of 1, 2, 3 and 40 steps whose boundaries end and restart the early pole pass, and as one run
    of all 46 steps. At 42 cells the plan also replays its 32-step graphs."""
    monkeypatch.setenv("OEM_B200_KERNELS", "ws")
    r = (0.05, 0.1) if n < 64 else (0.1, 0.3)
    sc = scenes.dispersive_spheres(n=n, n_sph=4, num_steps=60, nfreq=3,
                                   rmin=r[0] * scenes.UM, rmax=r[1] * scenes.UM)
    chunks = [1, 2, 3, 40]

    def go(ahead, parts):
        if ahead:
            monkeypatch.delenv("OEM_B200_ADE", raising=False)
        else:
            monkeypatch.setenv("OEM_B200_ADE", "inline")
        plan = solver.Plan(sc, sum(parts))
        try:
            assert plan.pole_pass_ahead() == ahead
            for c in parts:
                plan.run(c)
            plan.flush()
            fields = [plan.read_field(c) for c in range(6)]
            ph = plan.field_phasors()
        finally:
            plan.close()
        return fields, ph

    f0, p0 = go(False, chunks)
    for parts in (chunks, [sum(chunks)]):
        f1, p1 = go(True, parts)
        for c in range(6):
            np.testing.assert_array_equal(f1[c], f0[c])
        assert set(p1) == set(p0) == {"mid_x", "mid_y", "mid_z"}
        for name in p0:
            np.testing.assert_array_equal(p1[name], p0[name])
    assert float(np.abs(f0[2]).max()) > 0.0


@pytest.mark.parametrize("kind", ["stream", "tma", "ws"])
def test_pipelined_kernels_periodic_slab(monkeypatch, kind):
    """Periodic x/y walls of a one-cell-wide column (every neighbour wraps) and a plane-wave
    source, against the one-thread-per-cell kernels."""
    sc = scenes.slab_plane_wave(nxy=1, num_steps=400)
    monkeypatch.setenv("OEM_B200_KERNELS", "basic")
    a = solver.run(sc, num_steps=400, use_shutoff=False, return_fields=True, verbose=False)
    monkeypatch.setenv("OEM_B200_KERNELS", kind)
    b = solver.run(sc, num_steps=400, use_shutoff=False, return_fields=True, verbose=False)
    for nm in ("Ex", "Hy"):
        assert rel_l2(b.fields[nm], a.fields[nm]) < 1e-6, nm


@pytest.mark.parametrize("chunk", [None, 64 << 10])
def test_device_tables_match_host_tables(monkeypatch, chunk):
    """Material index and pole offsets built on the GPU equal the numpy build cell for cell; with
    a small staging chunk the eps / sigma uploads go through the pinned double buffer."""
    from openem_b200 import tables as T
    from openem_b200 import tables_gpu
    if not tables_gpu.available():
        pytest.skip("torch with CUDA is not available")
    if chunk:
        monkeypatch.setattr(tables_gpu._PinnedStager, "CHUNK", chunk)
        monkeypatch.setattr(tables_gpu._PinnedStager, "_buf", None)
    sc = scenes.small_dispersive(n=48, n_sph=6, num_steps=10, n_pml=8, nfreq=2)
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    h = T.material_tables(sc, tabs)
    d = tables_gpu.material_tables_device(sc, tabs, 0)
    assert d.n_mat == h.n_mat and d.n_pole_total == h.n_pole_total
    idx_d = d.index.cpu().numpy().astype(np.int64) & 0xFFFF if d.index_bytes == 2 \
        else d.index.cpu().numpy().astype(np.int64)
    np.testing.assert_array_equal(d.table[idx_d], h.table[h.index.astype(np.int64)])
    np.testing.assert_array_equal(d.seg_ofs.cpu().numpy().view(np.uint32), h.seg_ofs)
    np.testing.assert_array_equal(d.set_ofs, h.set_ofs)
    np.testing.assert_array_equal(d.coef, h.coef)


def test_device_table_run_equals_host_table_run(monkeypatch):
    sc = scenes.small_dispersive(n=40, n_sph=5, num_steps=60, n_pml=8, nfreq=2)
    monkeypatch.setenv("OEM_B200_TABLES", "host")
    a = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    from openem_b200 import tables_gpu
    if not tables_gpu.available():
        pytest.skip("torch with CUDA is not available")
    monkeypatch.setenv("OEM_B200_TABLES", "device")
    b = solver.run(sc, use_shutoff=False, return_fields=True, verbose=False)
    for nm in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        np.testing.assert_array_equal(a.fields[nm], b.fields[nm])


@pytest.mark.parametrize("kind", ["basic", "ws"])
def test_many_box_monitors_match_oracle(monkeypatch, kind):
    """Ten box monitors of assorted shapes (one launch snapshots at most eight, so two launches
    per step; thin and ragged boxes, one touching the grid's faces) against the FP64 oracle."""
    from dataclasses import replace
    from openem_b200.model import FieldMonitor
    monkeypatch.setenv("OEM_B200_KERNELS", kind)
    sc = scenes.small_dispersive(n=36, n_sph=3, num_steps=90, n_pml=6, nfreq=2)
    freqs = np.asarray(sc.field_monitors[0].freqs)
    shapes = [((0, 0, 0), (36, 36, 36)), ((3, 5, 7), (1, 9, 2)), ((10, 2, 17), (5, 1, 3)),
              ((17, 17, 17), (2, 2, 2)), ((0, 20, 30), (36, 3, 6)), ((35, 35, 35), (1, 1, 1)),
              ((8, 8, 0), (7, 11, 36)), ((12, 0, 11), (4, 36, 1)), ((20, 21, 22), (3, 4, 5)),
              ((1, 2, 3), (33, 31, 29))]
    mons = [FieldMonitor(name=f"b{q}", freqs=freqs, origin=o, box=b)
            for q, (o, b) in enumerate(shapes)]
    sc = replace(sc, field_monitors=mons)
    ref = ref64.run(sc)
    got = solver.run(sc, use_shutoff=False, verbose=False)
    scale = float(np.abs(ref.field_phasors["b0"]).max())  # the whole-grid box
    for name, data in ref.field_phasors.items():
        g = got.field_phasors[name]
        assert g.shape == data.shape, name
        # relative L2 within 1e-4, or, for a box where the field is still weak, every value
        # within 1e-6 of the largest phasor anywhere
        assert rel_l2(g, data) < 1e-4 or float(np.abs(g - data).max()) < 1e-6 * scale, name
