"""Precision of the device DFT accumulation (float32 partials over a snapshot batch, each batch
added once to a float64 accumulator) on a small Bloch cell: the E phasors of the flux plane
against the float64 sum of the very samples the engine folded (recorded every step by a field
time monitor), with a plain float32 running sum as the comparison that shows the difference."""

import pytest

from openem_b200 import precision

pytestmark = pytest.mark.gpu


def test_dft_accumulation_matches_float64_sum():
    r = precision.study(nx=8, ny=8, nz=256, steps=3000, nfreq=16, npix=2)
    assert r["engine"] < 5e-7, r
    assert r["kahan"] < 5e-7, r
    assert r["fp32"] > 5 * r["engine"], r
