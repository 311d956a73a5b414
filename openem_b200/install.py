"""Route OpenEM's step loop to this engine.

OpenEM's two production callers look ``solver.run`` up as a module attribute at call time
(``openem/nb/solve_worker.py:61``, ``openem/nb/autograd_hook.py:161,169``) and construct
``device.Kernels()`` first, which needs cupy. ``install_into_openem()`` replaces
``openem.solver.run`` with :func:`openem_b200.solver.run` and provides a cupy-free
``openem.device`` module whose ``Kernels`` is an inert placeholder, so ``openem.install()`` /
``openem.run()`` run on the sm_100a engine unchanged. It is a no-op where OpenEM is not
importable.
"""

from __future__ import annotations

import sys
import types


class Kernels:
    """Stand-in for ``openem.device.Kernels``: the engine's kernels are compiled ahead of time,
    so there is nothing to JIT; the object is accepted and ignored by ``solver.run``."""

    def __init__(self, *args, **kwargs):
        self.profiler = None

    def __getitem__(self, name):
        raise KeyError(f"OpenEM kernel {name!r} is not available: the sm_100a engine runs the "
                       "step loop")


def install_into_openem() -> bool:
    """Patch the importable OpenEM package in place; returns False if it is not importable."""
    from openem_b200 import solver as ours
    dev = types.ModuleType("openem.device")
    dev.Kernels = Kernels
    dev.grid_1d = dev.grid_2d = dev.grid_3d = None
    sys.modules["openem.device"] = dev
    try:
        import openem
    except Exception:
        return False
    openem.device = dev
    try:
        import openem.solver as theirs  # imports cupy; replace it with a shell if that fails
    except Exception:
        theirs = types.ModuleType("openem.solver")
        sys.modules["openem.solver"] = theirs
        openem.solver = theirs
    theirs.run = ours.run
    from openem_b200.results import Phasors, Result
    theirs.Result = Result
    theirs.Phasors = Phasors
    return True
