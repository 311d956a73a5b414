"""Gradients of flux objectives through a time-reversed discrete adjoint of the GPU step.

The reference differentiates a simulation through tidy3d's autograd: a forward solve and an
adjoint solve (a ``CustomCurrentSource`` run for the same step count), with the gradient
assembled by tidy3d in the frequency domain (``openem/nb/autograd_hook.py:184-221``). This
engine differentiates the discrete time stepping itself instead: the forward run saves the
fields and CPML psi every ``checkpoint_every`` steps, and the adjoint runs the transpose of each
step from the last step down to the first, recomputing each segment from its checkpoint, with the
gradient accumulated in float64 on the device. The gradient is that of the float32 update
coefficients ``(ca, cb)`` of every E component and cell, mapped here to permittivity and
conductivity with ``ca = (eps - s)/(eps + s + G)``, ``cb = (dt/eps0)/(eps + s + G)``,
``s = sigma dt / (2 eps0)`` (``openem/coeffs.py:132-136``).

Objective: ``J = sum_f w_f P_f`` of one flux monitor, ``P_f`` the plane flux of
``openem/flux.py:60-107`` computed from the monitor's phasors after a fixed number of steps (no
early termination, so forward and adjoint see the same step count).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from openem_b200 import flux as flux_mod
from openem_b200 import tables as T
from openem_b200.solver import Plan

__all__ = ["FluxGradient", "flux_gradient", "default_interval", "FluxObjective",
           "flux_objective"]


def default_interval(n_steps: int) -> int:
    """Checkpoint spacing that balances checkpoint memory against the segment buffer:
    about sqrt(2 N)."""
    return max(1, int(round(math.sqrt(2.0 * max(1, n_steps)))))


@dataclass
class FluxGradient:
    value: float          # J
    flux: np.ndarray      # P_f per monitor frequency
    d_ca: np.ndarray      # dJ/dca, (3, ni, nj, nk) over the gradient box
    d_cb: np.ndarray      # dJ/dcb
    d_eps: np.ndarray     # dJ/d eps_r per component and cell
    d_sigma: np.ndarray   # dJ/d sigma (S/m) per component and cell
    steps: int
    checkpoint_every: int
    box: tuple = ()       # (i0, j0, k0, ni, nj, nk)


def _refuse(sc) -> None:
    if getattr(sc, "dispersion_mix", None) is not None and sc.dispersion_mix.n_entry > 0:
        raise NotImplementedError("the adjoint does not cover slanted-interface mixed media")
    if sc.absorbers:
        raise NotImplementedError("the adjoint does not cover absorber slabs")
    if (sc.tensor is not None and sc.tensor.n_entry) or \
            (sc.modulation is not None and sc.modulation.n_entry):
        raise NotImplementedError("the adjoint does not cover tensor media or time modulation")
    if sc.any_bloch:
        raise NotImplementedError("the adjoint covers real fields (no Bloch phase)")


def _pick(plan, monitor):
    if not plan.flux_mons:
        raise ValueError("the scene has no flux monitor")
    if monitor is None:
        return plan.flux_mons[0]
    for m, mid, shp in plan.flux_mons:
        if m.name == monitor:
            return m, mid, shp
    raise KeyError(f"no flux monitor named {monitor!r}")


def coefficient_jacobian(sc):
    """Per component: (dca/deps, dcb/deps, dca/dsigma, dcb/dsigma) in float64, zero where
    the cell is PEC (its coefficients are pinned to zero)."""
    tabs = [T.axis_tables(sc, a) for a in range(3)]
    _, cb32 = T.e_coefficients(sc, tabs)
    gg = T._g_dense(sc, sc.shape)
    sig = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
    k = sc.dt / (2.0 * T.EPSILON_0)
    out = []
    for c, eps in enumerate((sc.eps_ex, sc.eps_ey, sc.eps_ez)):
        eps = np.asarray(eps, dtype=np.float64)
        s = np.zeros_like(eps) if sig[c] is None else np.asarray(sig[c], np.float64) * k
        den = eps + s + gg[c]
        live = (np.asarray(cb32[c]) != 0.0)
        d2 = den * den
        dca_de = np.where(live, (2.0 * s + gg[c]) / d2, 0.0)
        dcb_de = np.where(live, -(sc.dt / T.EPSILON_0) / d2, 0.0)
        dca_ds = np.where(live, -(2.0 * eps + gg[c]) / d2 * k, 0.0)
        dcb_ds = np.where(live, -(sc.dt / T.EPSILON_0) / d2 * k, 0.0)
        out.append((dca_de, dcb_de, dca_ds, dcb_ds))
    return out


def flux_gradient(sc, monitor: str | None = None, weights=None, num_steps: int | None = None,
                  checkpoint_every: int | None = None, device: int = 0, stream=None,
                  box=None) -> FluxGradient:
    """Run the scene forward for a fixed step count with checkpoints, then the discrete adjoint;
    return ``J`` and its gradient with respect to the E-update coefficients, the relative
    permittivity and the conductivity of every E component and cell of ``box = (i0, j0, k0,
    ni, nj, nk)`` (default: the whole grid; a design region's box keeps the adjoint's gradient
    work to that region)."""
    _refuse(sc)
    box = tuple(int(v) for v in (box if box is not None else (0, 0, 0) + tuple(sc.shape)))
    n = int(sc.num_time_steps if num_steps is None else num_steps)
    K = int(checkpoint_every or default_interval(n))
    # the box is declared before the run: the forward pass records its E every step and the
    # reverse pass reads that instead of recomputing the segments
    plan = Plan(sc, n, device=device, stream=stream, checkpoint_every=K, gradient_box=box)
    try:
        plan.run(n)
        plan.flush()
        m, mid, shp = _pick(plan, monitor)
        data = plan.read_monitor(mid, shp)
        axis = int(m.axis)
        P = flux_mod.plane_flux(data, sc.grid, axis=axis)
        w = np.ones(P.size) if weights is None else np.asarray(weights, np.float64).ravel()
        if w.size != P.size:
            raise ValueError(f"{w.size} weights for {P.size} monitor frequencies")
        J = float(np.dot(w, P))
        dA1, dA2 = flux_mod.area_weights(sc.grid, axis)
        g_ca, g_cb = plan.adjoint_flux(mid, w, dA1, dA2, box=box)
        plan.status()
    finally:
        plan.close()
    jac = coefficient_jacobian(sc)
    sl = tuple(slice(box[a], box[a] + box[3 + a]) for a in range(3))
    d_eps = np.stack([g_ca[c] * jac[c][0][sl] + g_cb[c] * jac[c][1][sl] for c in range(3)])
    d_sig = np.stack([g_ca[c] * jac[c][2][sl] + g_cb[c] * jac[c][3][sl] for c in range(3)])
    return FluxGradient(value=J, flux=P, d_ca=g_ca, d_cb=g_cb, d_eps=d_eps, d_sigma=d_sig,
                        steps=n, checkpoint_every=K, box=box)


try:  # the torch binding is optional: the numpy API above does not need it
    import torch

    class FluxObjective(torch.autograd.Function):
        """``J(params)`` for a scene built from a parameter tensor. ``make_scene(params_np)``
        returns the Scene; ``pullback(d_eps, d_sigma, params_np)`` maps the per-cell gradient to
        the parameters' shape (for a pixel map: the sum of d_eps over each pixel's cells)."""

        @staticmethod
        def forward(ctx, params, make_scene, pullback, options):
            p = params.detach().cpu().numpy().astype(np.float64)
            g = flux_gradient(make_scene(p), **options)
            grad = np.asarray(pullback(g.d_eps, g.d_sigma, p), dtype=np.float64)
            ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype,
                                                  device=params.device))
            return torch.tensor(g.value, dtype=params.dtype, device=params.device)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad, None, None, None

    def flux_objective(params, make_scene, pullback, **options):
        return FluxObjective.apply(params, make_scene, pullback, options)

except ImportError:  # pragma: no cover
    FluxObjective = None

    def flux_objective(*a, **k):
        raise ImportError("torch is needed for flux_objective")
