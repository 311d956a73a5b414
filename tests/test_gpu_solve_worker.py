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
