"""The solve worker end to end on the GPU: a scene written as ``scene.npz``, solved from the
work directory into ``ours.npz``, equals the in-process run of the same scene."""

import numpy as np
import pytest

from openem_b200 import scenes, serialize, solve_worker, solver

pytestmark = pytest.mark.gpu


def test_solve_dir_matches_in_process_run(tmp_path):
    sc = scenes.slab_plane_wave(nxy=4, num_steps=400, nfreq=5)
    serialize.save(sc, tmp_path / "scene.npz")
    path = solve_worker.solve_dir(tmp_path, tmp_path / "out", steps=400)
    got = solve_worker.load_result(path)
    ref = solver.run(serialize.load(tmp_path / "scene.npz"), num_steps=400, use_shutoff=False,
                     verbose=False)
    assert got["meta"]["steps_run"] == 400
    for name, p in ref.phasors.items():
        np.testing.assert_array_equal(got["phasors"][name][0], p.data)
        np.testing.assert_array_equal(got["phasors"][name][1], p.freqs)


def test_solve_dir_writes_tidy3d_readout(tmp_path):
    """With ``td_coords.npz`` in the work directory, ``ours.npz`` carries the ``tdf:``/``tdc:``
    entries of the field monitors, equal to converting the in-process phasors."""
    from openem_b200 import td_convention
    sc = scenes.small_dispersive(n=24, n_sph=2, num_steps=120, n_pml=6, nfreq=3)
    serialize.save(sc, tmp_path / "scene.npz")
    m = sc.field_monitors[0]
    plans = {}
    for comp in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        for a, ax in enumerate("xyz"):
            e = np.asarray(sc.grid.axes[a].edges)[m.origin[a]:m.origin[a] + m.box[a]] / 1e-6
            plans[f"{m.name}|{comp}:{ax}"] = e if m.box[a] > 2 else e[:1]
    np.savez(tmp_path / "td_coords.npz", **plans)
    path = solve_worker.solve_dir(tmp_path, tmp_path / "out", steps=120)
    ref = solver.run(serialize.load(tmp_path / "scene.npz"), num_steps=120, use_shutoff=False,
                     verbose=False)
    want = td_convention.to_tidy3d(sc, ref.field_phasors, plans)
    with np.load(path) as z:
        for k, v in want.items():
            np.testing.assert_array_equal(z[k], v, err_msg=k)
