"""``install_into_openem()`` routes OpenEM's own callers to this engine.

Needs an OpenEM checkout on the import path (``OPENEM_SRC``; skipped otherwise). OpenEM's
solve worker and autograd hook look ``solver.run`` and ``device.Kernels`` up at call time
(``openem/nb/solve_worker.py:61``, ``openem/nb/autograd_hook.py:161,169``): after the install both
resolve to this engine without cupy, and ``Result`` / ``Phasors`` are this engine's classes."""

import os
import sys

import pytest

SRC = os.environ.get("OPENEM_SRC")
pytestmark = pytest.mark.skipif(not SRC, reason="set OPENEM_SRC to an OpenEM checkout")


def test_openem_callers_resolve_to_this_engine():
    sys.path.insert(0, SRC)
    try:
        from openem_b200 import install, solver
        assert install.install_into_openem()
        import openem.nb.solve_worker as sw
        import openem.solver
        assert openem.solver.run is solver.run
        assert sw.solver.run is solver.run        # looked up at call time by solve_dir
        k = sw.Kernels()                          # constructed before every solve
        assert isinstance(k, install.Kernels)
        from openem_b200.results import Result
        assert openem.solver.Result is Result
    finally:
        sys.path.remove(SRC)
