"""The complex-field (Bloch) path: ``openem/solver.py:1263-1358`` (``_run_bloch``).

Fields and CPML psi are carried as real and imaginary float32 arrays on the device; the
Bloch phase ``exp(+-i 2 pi k)`` enters only through the neighbour masks at the periodic seam of
a Bloch axis. Point dipoles inject the complex analytic amplitude, mode sources (oblique plane
waves, beams) the complex product of profile and amplitude, and DFT and time monitors record
complex values. With ``k = 0`` (``force_complex``) the real and imaginary parts are two
independent real solutions, driven by the real and imaginary parts of the injection.

The supported subset is OpenEM's: lossless, non-dispersive media without PEC cells, dipole or
mode sources, DFT and time monitors, CPML and periodic / Bloch axes; anything else raises
``NotImplementedError`` before allocation (:func:`openem_b200.solver.refuse_unsupported_bloch`).
"""

from __future__ import annotations

from openem_b200 import solver


def run(sc, num_steps: int | None = None, use_shutoff: bool = True, verbose: bool = True,
        return_fields: bool = False, policy=None, device: int = 0, stream=None,
        stats: dict | None = None):
    """Run one complex-field simulation; same ``Result`` as :func:`openem_b200.solver.run`,
    with complex fields and time samples."""
    return solver.run_plan(sc, num_steps, use_shutoff, verbose, return_fields, policy, device,
                           stream, stats, cplx=True)
