"""The allocation-free field sums against the plan's own sums, through the C ABI.

oem_field_energy_noalloc exists for callers that cannot allocate device memory where they need
these sums (fields held in another framework's memory pool, step loops that must not let
cudaMalloc synchronise the device). It keeps its scratch in a file-scope device array shared by
all calls, so it is called twice in a row here: the second call must not be disturbed by what
the first one left in that array. This file is collected last on purpose.
"""

import ctypes as C

import numpy as np
import pytest

from openem_b200 import lib as L
from openem_b200 import scenes, solver

pytestmark = pytest.mark.gpu


def test_noalloc_field_sums_match_plan_sums_twice():
    torch = pytest.importorskip("torch")
    sc = scenes.small_dispersive(n=40, n_sph=4, num_steps=80, n_pml=8, nfreq=2)
    plan = solver.Plan(sc, 80)
    try:
        plan.run(60)
        ref = plan.energy()                 # existing entry point (plan-owned scratch)
        assert np.all(ref > 0)
        lib = L.load()
        fptr = (C.c_void_p * 6)()
        nzp = C.c_int()
        L.check(lib.oem_plan_field_ptrs(plan.h, fptr, C.byref(nzp)))
        nx, ny, nz = plan.shape
        eps_t = []
        for e in (sc.eps_ex, sc.eps_ey, sc.eps_ez):
            t = torch.zeros((nx, ny, nzp.value), dtype=torch.float32, device="cuda:0")
            t[:, :, :nz] = torch.from_numpy(np.asarray(e, dtype=np.float32)).to("cuda:0")
            eps_t.append(t)
        torch.cuda.synchronize()
        eptr = (C.c_void_p * 3)(*[t.data_ptr() for t in eps_t])
        # the plan sums with spacings 1 / (1 / dl); pass the same float64 values
        sp = []
        for ax in sc.grid.axes:
            sp.append(1.0 / (1.0 / ax.dl))
            sp.append(1.0 / (1.0 / ax.dl_dual))
        spacing = np.ascontiguousarray(np.concatenate(sp), dtype=np.float64)
        outs = []
        for _ in range(2):
            out = np.zeros(3, np.float64)
            L.check(lib.oem_field_energy_noalloc(fptr, eptr, nx, ny, nz, nzp.value,
                                                 L.ptr(spacing), L.ptr(out), None),
                    "field_energy_noalloc")
            np.testing.assert_allclose(out, ref, rtol=1e-12, atol=0)
            outs.append(out)
        np.testing.assert_array_equal(outs[0], outs[1])
        # eps = NULL means relative permittivity 1: the eps-weighted sum equals the plain one
        out1 = np.zeros(3, np.float64)
        L.check(lib.oem_field_energy_noalloc(fptr, None, nx, ny, nz, nzp.value, L.ptr(spacing),
                                             L.ptr(out1), None), "field_energy_noalloc eps=NULL")
        assert out1[1] == out1[0]
        np.testing.assert_array_equal(out1[[0, 2]], outs[0][[0, 2]])
        # on a caller's own (non-default) stream the sums are the same
        side = torch.cuda.Stream(device="cuda:0")
        out2 = np.zeros(3, np.float64)
        L.check(lib.oem_field_energy_noalloc(fptr, eptr, nx, ny, nz, nzp.value, L.ptr(spacing),
                                             L.ptr(out2), C.c_void_p(side.cuda_stream)),
                "field_energy_noalloc on a side stream")
        np.testing.assert_array_equal(out2, outs[0])
        # sizes beyond the fixed scratch are refused with a clear error
        big = np.zeros(2 * (40000 + 2), np.float64)
        rc = lib.oem_field_energy_noalloc(fptr, eptr, 40000, 1, 1, 32, L.ptr(big),
                                          L.ptr(np.zeros(3)), None)
        assert rc == L.ERR_INVALID and "limit" in L.last_error()
    finally:
        plan.close()
