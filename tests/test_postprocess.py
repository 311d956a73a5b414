"""Tidy3D-convention post-processing (``openem_b200.td_convention``) against fixtures that
OpenEM's own numpy modules produced (``openem.normalize``, ``openem.colocate``,
``openem.td_readout``; ``tests/golden/gen_golden.py``): the field and flux divisors of every
source type (point dipole, plane wave, mode source, TFSF box), the plane-wave background index,
monitor area, analytic flux divisor and time scale, linear colocation from the Yee positions,
the zero-thickness snapping rule and the ``tdf:`` / ``tdc:`` field readout."""

import pathlib

import numpy as np
import pytest

from openem_b200 import scenes
from openem_b200 import td_convention as TD
from openem_b200.model import GaussianPulse

GOLD = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def gz():
    return dict(np.load(GOLD / "ref_postprocess.npz"))


def post_scenes():
    return {
        "dip": scenes.small_dispersive(n=20, n_sph=2, num_steps=300, n_pml=6, nfreq=3),
        "pw": scenes.slab_plane_wave(nxy=3, num_steps=600),
        "mode": scenes.bloch_metasurface(nx=8, ny=8, nz=64, n_pml=8, npix=2, layer_cells=8,
                                         nfreq=5, num_steps=400, bloch_k=(0.05, 0.0, 0.0)),
        "tfsf": scenes.tfsf_box_scene(n=24, n_pml=6, num_steps=300),
    }


@pytest.mark.parametrize("tag", ["dip", "pw", "mode", "tfsf"])
def test_divisors_match_openem(gz, tag):
    sc = post_scenes()[tag]
    f = gz[f"{tag}_freqs"]
    np.testing.assert_allclose(TD.injected_spectrum(sc, f), gz[f"{tag}_D"], rtol=1e-12)
    np.testing.assert_allclose(TD.field_divisor(sc, f), gz[f"{tag}_field"], rtol=1e-12)
    np.testing.assert_allclose(TD.flux_divisor(sc, f), gz[f"{tag}_flux"], rtol=1e-12)


def test_plane_wave_terms_match_openem(gz):
    sc = post_scenes()["pw"]
    m = sc.flux_monitors[0]
    f = gz["pw_freqs"]
    assert TD.background_index(sc) == pytest.approx(float(gz["pw_bg"]), rel=1e-15)
    assert TD.monitor_area(sc, m) == pytest.approx(float(gz["pw_area"]), rel=1e-15)
    np.testing.assert_allclose(TD.plane_flux_divisor(sc, m, f), gz["pw_plane_div"], rtol=1e-12)
    pulse = GaussianPulse(freq0=2.998e14, fwidth=0.2 * 2.998e14)
    assert TD.time_scale(sc, pulse, sc.dt, 600) == pytest.approx(float(gz["pw_tscale"]),
                                                                 rel=1e-12)


def test_colocation_matches_openem(gz):
    sc = post_scenes()["dip"]
    origin, box = (3, 4, 5), (6, 5, 4)
    for comp in ("Ex", "Hy", "Ez"):
        src = TD.sample_positions(sc.grid, origin, box, comp)
        dst = [np.asarray(sc.grid.axes[a].edges)[origin[a]:origin[a] + box[a]] for a in range(3)]
        dst[2] = dst[2][1:2]
        np.testing.assert_allclose(TD.interpolate(gz["col_data"], src, dst), gz[f"col_{comp}"],
                                   rtol=1e-13, atol=1e-15)
    snaps = [TD.floor_snap(sc.grid.axes[0].edges, c, 1e-15) for c in (-1e-6, 0.0, 3.3e-8, 1e-3)]
    np.testing.assert_array_equal(snaps, gz["col_snap"])


def test_colocation_refuses_extrapolation():
    sc = post_scenes()["dip"]
    src = TD.sample_positions(sc.grid, (3, 4, 5), (6, 5, 4), "Ex")
    far = [s.copy() for s in src]
    far[0] = far[0] + 3 * (far[0][1] - far[0][0])
    with pytest.raises(ValueError, match="too small"):
        TD.interpolate(np.zeros((6, 5, 4)), src, far)


def test_field_readout_matches_openem(gz):
    sc = post_scenes()["dip"]
    m = sc.field_monitors[0]
    plans = {k[5:]: v for k, v in gz.items() if k.startswith("plan|")}
    got = TD.to_tidy3d(sc, {m.name: gz["tdr_raw"]}, plans)
    want = {k[4:]: v for k, v in gz.items() if k.startswith("fin|")}
    assert set(got) == set(want)
    for k, v in want.items():
        np.testing.assert_allclose(got[k], v, rtol=1e-12, atol=1e-300, err_msg=k)
