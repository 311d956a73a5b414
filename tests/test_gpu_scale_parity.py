"""The default kernels at the sizes they are chosen for, against the FP64 oracle.

Below 1.5M cells the engine runs the one-thread-per-cell kernels; from 1.5M cells on it runs the
warp-specialised H/E kernels, the segment pole pass and, on a Bloch cell, the split complex
update. These tests run those paths with no kernel override, on grids of 128^3 and 256^3 (several
x chunks per block column, CPML on all faces, Drude+Lorentz spheres) and on the 32 x 32 x 1024
Bloch proxy of the metasurface cell with its 200-frequency flux plane.

Every cell starts from seeded random fields (``Plan.write_field``; the oracle's
``load_fields``), so that after a few steps every kernel branch -- CPML slabs on all six faces,
dispersive cells, x-chunk seams, block-row edges, the Bloch seam -- has moved data that a wrong
index or coefficient would corrupt. A point source alone would leave most of the grid at zero
for the few steps the oracle can afford at these sizes.

Tolerances: per component, the L2 difference within 1e-5 of its field family's norm (the
field tolerance the engine is held to), and every single cell's difference within 1e-4 of the
local scale, the family's RMS plus the largest magnitude within two cells (a fault in one row
or one seam cell cannot hide in the L2 norm; next to the dipole, where the injected current
makes the field much larger than the random start, float32 rounding scales with that field);
DFT phasors within 1e-4 relative L2.
"""

import numpy as np
import pytest
from scipy.ndimage import maximum_filter

from oracle import ref64
from openem_b200 import scenes, solver

pytestmark = pytest.mark.gpu

NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
FAMILIES = (NAMES[:3], NAMES[3:])


def random_start(shape, seed: int, cplx: bool = False):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(6):
        a = rng.standard_normal(shape).astype(np.float32)
        if cplx:
            a = a + 1j * rng.standard_normal(shape).astype(np.float32)
        out.append(a)
    return out


def run_engine(sc, steps: int, start, cplx: bool = False):
    """Fields and phasors of the engine after ``steps`` steps from ``start``."""
    plan = solver.Plan(sc, steps, cplx=cplx)
    try:
        for c, f in enumerate(start):
            if cplx:
                plan.write_field_complex(c, f)
            else:
                plan.write_field(c, f)
        plan.run(steps)
        plan.flush()
        plan.status()
        fields = {nm: plan.read_field(c) for c, nm in enumerate(NAMES)}
        phasors = {k: v.data for k, v in plan.flux_phasors().items()}
        phasors.update(plan.field_phasors())
        return fields, phasors
    finally:
        plan.close()


def run_oracle(sc, steps: int, start):
    o = ref64.BlochOracle(sc, steps) if sc.any_bloch else ref64.Oracle(sc, steps)
    o.load_fields(start)
    r = o.run(steps)
    ph = dict(r.phasors)
    ph.update(r.field_phasors)
    return r.fields, ph


def check_fields(fa, fb, l2_tol=1e-5, max_tol=1e-4):
    for fam in FAMILIES:
        den = np.sqrt(sum(float(np.linalg.norm(np.ravel(fb[n]))) ** 2 for n in fam))
        rms = den / np.sqrt(sum(np.size(fb[n]) for n in fam))
        for n in fam:
            b = np.asarray(fb[n])
            d = np.abs(np.asarray(fa[n]) - b)
            l2 = float(np.linalg.norm(d.ravel())) / den
            scale = maximum_filter(np.abs(b), size=5, mode="wrap") + rms
            r = d / scale
            q = np.unravel_index(int(np.argmax(r)), r.shape)
            assert l2 < l2_tol and r[q] < max_tol, (n, l2, float(r[q]), q, float(d[q]),
                                                     float(np.abs(b[q])), rms)


def check_phasors(pa, pb, tol=1e-4):
    assert set(pa) == set(pb)
    for k, b in pb.items():
        a = pa[k]
        assert a.shape == b.shape, k
        e = float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
        assert e < tol, (k, e)


def test_default_kernels_128_dispersive_match_oracle(monkeypatch):
    """128^3 (2.1M cells: the warp-specialised path), 12 Drude+Lorentz spheres, CPML 12 on all
    faces, the z dipole and three mid-plane field monitors, 40 steps."""
    monkeypatch.delenv("OEM_B200_KERNELS", raising=False)
    sc = scenes.small_dispersive(n=128, n_sph=12, n_pml=12, num_steps=40, nfreq=4)
    assert np.prod(sc.shape) >= 1.5e6
    start = random_start(sc.shape, 11)
    fa, pa = run_engine(sc, 40, start)
    fb, pb = run_oracle(sc, 40, start)
    check_fields(fa, fb)
    check_phasors(pa, pb)


def test_default_kernels_256_bulk_workload_prefix_match_oracle(monkeypatch):
    """The bulk dispersive workload's construction at 256^3 (16.8M cells: 8 spheres of radius
    0.2-0.6 um, as dense as 64 in the 512^3 cell, CPML 12, the dipole, three mid-plane monitors
    at 8 frequencies) for 8 steps. 256^3 rather than 512^3: the float64 oracle takes ~7 s per
    step here and ~1 min at 512^3."""
    monkeypatch.delenv("OEM_B200_KERNELS", raising=False)
    sc = scenes.dispersive_spheres(n=256, n_sph=8, num_steps=8)
    start = random_start(sc.shape, 12)
    fa, pa = run_engine(sc, 8, start)
    fb, pb = run_oracle(sc, 8, start)
    check_fields(fa, fb)
    check_phasors(pa, pb)


@pytest.fixture(scope="module")
def bloch_proxy():
    """The 32 x 32 x 1024 proxy of the Bloch metasurface cell (8 x 8 pixels of the diagonal
    anisotropic layer, the same transverse wavevector 0.15, the oblique plane-wave source, the
    200-frequency flux plane), 60 steps from a random complex start."""
    sc = scenes.bloch_metasurface(nx=32, ny=32, nz=1024, npix=8, num_steps=60)
    start = random_start(sc.shape, 13, cplx=True)
    return sc, start, run_oracle(sc, 60, start)


@pytest.mark.parametrize("kind", [None, "ws"])
def test_bloch_proxy_matches_oracle(monkeypatch, bloch_proxy, kind):
    """Default kernels (complex one thread per cell at 1M cells) and the split complex update
    that the full 256 x 256 x 1024 cell runs (forced here with ``OEM_B200_KERNELS=ws``)."""
    sc, start, (fb, pb) = bloch_proxy
    if kind:
        monkeypatch.setenv("OEM_B200_KERNELS", kind)
    else:
        monkeypatch.delenv("OEM_B200_KERNELS", raising=False)
    fa, pa = run_engine(sc, 60, start, cplx=True)
    assert pa["T"].shape == (4, 200, 32, 32)
    check_fields(fa, fb)
    check_phasors(pa, pb)
