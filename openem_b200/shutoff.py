"""When to stop a run early: the fields have died away, or the monitored fluxes have settled.

The step loop samples three numbers every ``interval`` steps (400, Tidy3D's cadence): the
volume-weighted ``sum V |E|^2``, the total energy ``(eps0 sum V eps |E|^2 + mu0 sum V |H|^2)/2``
and the flux of every flux monitor at every frequency. OpenEM stops on any of three tests
(criteria of ``openem/shutoff.py:19-253``, ``openem/solver.py:160-203``):

* the ``|E|^2`` sum has fallen below ``threshold`` times its largest value so far;
* the energy has fallen below ``threshold`` times its largest value so far;
* the fluxes have converged: their largest change since the previous check, relative to their
  largest magnitude, scaled by the energy's decay time over the check interval (an estimate of
  the change still to come), stays below ``tol`` on ``patience`` consecutive checks.

The decay time comes from a least-squares line through ``log(energy / running peak)`` against
the step, over the later half of the checks. Stopping is honoured only once every source has
finished (:func:`source_end_step`); the tests themselves run from the first check so that the
running peaks include the source's ramp.

Here the whole stopping state is one immutable :class:`Watch` record, advanced one check at a
time by the pure function :func:`observe`; :class:`Policy` holds the current record for the
step loop and exposes the call the loop makes (``check``) and what the result reports
(``reason``, ``summary``, the decay and energy traces).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

#: A source has finished once its envelope stays below this fraction of its peak.
SOURCE_TAIL = 1e-3

_INF = float("inf")


@dataclass(frozen=True)
class Criteria:
    """Thresholds of the three tests; ``None`` switches a test off."""

    field_threshold: float | None = 1e-5
    energy_threshold: float | None = 1e-5
    flux_tol: float | None = 1e-3
    patience: int = 3
    interval: int = 400


@dataclass(frozen=True)
class Watch:
    """Everything the tests remember between checks.

    ``field_ratio`` / ``energy_ratio`` hold, per check, the sample over the running peak at that
    check; ``flux_last`` is the previous flux vector (a tuple, so the record stays immutable);
    ``flux_remaining`` holds ``(step, estimated remaining change)`` per flux comparison."""

    steps: tuple = ()
    field_ratio: tuple = ()
    energy_ratio: tuple = ()
    energy_abs: tuple = ()
    field_peak: float = 0.0
    energy_peak: float = 0.0
    flux_last: tuple | None = None
    flux_remaining: tuple = ()
    flux_per_window: float = _INF
    streak: int = 0
    fired: tuple = ()
    reason: str = ""


def _ratio(value: float, peak: float) -> float:
    return value / peak if peak > 0 else 0.0


def decay_time(energy_ratio, steps) -> float:
    """Energy decay time in steps from the later half of the checks: ``-1 / slope`` of the
    least-squares line through ``(step, log ratio)`` of the positive ratios. ``inf`` with fewer
    than 8 checks, fewer than 4 positive ratios in that half, or a slope that is not negative."""
    n = len(energy_ratio)
    if n < 8:
        return _INF
    s = np.asarray(steps[n // 2:], dtype=np.float64)
    r = np.asarray(energy_ratio[n // 2:], dtype=np.float64)
    keep = r > 0
    if int(keep.sum()) < 4:
        return _INF
    s, y = s[keep], np.log(r[keep])
    ds = s - s.mean()
    slope = float(np.dot(ds, y - y.mean()) / np.dot(ds, ds))
    if not math.isfinite(slope) or slope >= 0:
        return _INF
    return -1.0 / slope


def observe(c: Criteria, w: Watch, step: int, e2: float, energy: float, flux) -> Watch:
    """The record after one more check at ``step`` with the ``|E|^2`` sum ``e2``, the total
    ``energy`` and the monitor fluxes ``flux`` (empty: no flux test this check)."""
    field_peak = max(w.field_peak, e2)
    energy_peak = max(w.energy_peak, energy)
    nw = replace(w, steps=w.steps + (int(step),),
                 field_ratio=w.field_ratio + (_ratio(e2, field_peak),),
                 energy_ratio=w.energy_ratio + (_ratio(energy, energy_peak),),
                 energy_abs=w.energy_abs + ((int(step), float(energy)),),
                 field_peak=field_peak, energy_peak=energy_peak, fired=())
    fired = []
    if c.field_threshold is not None and field_peak > 0 and \
            nw.field_ratio[-1] < c.field_threshold:
        fired.append(f"field_decay<{c.field_threshold:g}")
    if c.energy_threshold is not None and energy_peak > 0 and \
            nw.energy_ratio[-1] < c.energy_threshold:
        fired.append(f"energy_decay<{c.energy_threshold:g}")
    f = np.asarray(flux, dtype=np.float64).ravel()
    if c.flux_tol is not None and f.size:
        if w.flux_last is None:
            nw = replace(nw, flux_last=tuple(f))
        else:
            big = float(np.abs(f).max())
            change = float(np.abs(f - np.asarray(w.flux_last)).max()) / big if big > 0 else _INF
            tau = decay_time(nw.energy_ratio, nw.steps) if c.energy_threshold is not None \
                else _INF
            remaining = change * tau / max(c.interval, 1) if math.isfinite(tau) and tau > 0 \
                else change
            streak = w.streak + 1 if remaining < c.flux_tol else 0
            nw = replace(nw, flux_last=tuple(f), flux_per_window=change, streak=streak,
                         flux_remaining=w.flux_remaining + ((int(step), remaining),))
            if streak >= c.patience:
                fired.append(f"phasor_converged(remaining~{remaining:.2e}<{c.flux_tol:g}"
                             f" x{c.patience})")
    if fired:
        nw = replace(nw, fired=tuple(fired), reason=" + ".join(fired))
    return nw


class Policy:
    """The step loop's handle on the stopping state: ``check`` feeds one sample set and says
    whether a test fired."""

    def __init__(self, criteria: Criteria | None = None):
        self.criteria = criteria or Criteria()
        self.watch = Watch()

    @property
    def interval(self) -> int:
        return int(self.criteria.interval)

    def check(self, step: int, e2_weighted: float, energy: float, flux) -> bool:
        self.watch = observe(self.criteria, self.watch, step, e2_weighted, energy, flux)
        return bool(self.watch.fired)

    @property
    def reason(self) -> str:
        return self.watch.reason

    @property
    def field_ratio(self) -> float:
        """``|E|^2`` sum over its running peak at the latest check (NaN before the first)."""
        if self.criteria.field_threshold is None or not self.watch.field_ratio:
            return float("nan")
        return self.watch.field_ratio[-1]

    @property
    def energy_trace(self) -> list:
        """``(step, total energy)`` at every check."""
        return list(self.watch.energy_abs) if self.criteria.energy_threshold is not None else []

    @property
    def tau(self) -> float:
        return decay_time(self.watch.energy_ratio, self.watch.steps)

    def summary(self) -> str:
        w, c, out = self.watch, self.criteria, []
        if not w.steps:
            return "no check yet"
        if c.field_threshold is not None:
            q = int(np.argmin(w.field_ratio))
            out.append(f"|E|^2 sum at {w.field_ratio[-1]:.3e} of its peak (lowest "
                       f"{w.field_ratio[q]:.3e} at step {w.steps[q]})")
        if c.energy_threshold is not None:
            out.append(f"energy at {w.energy_ratio[-1]:.3e} of its peak")
        if c.flux_tol is not None and w.flux_remaining:
            out.append(f"flux change {w.flux_per_window:.3e} per check, "
                       f"{w.flux_remaining[-1][1]:.3e} still to come")
        return "; ".join(out)


def default_policy(tidy3d_shutoff: float, interval: int = 400) -> Policy:
    """All three tests: both decay thresholds at the scene's ``shutoff``, flux tolerance 1e-3
    over 3 checks (OpenEM's production default)."""
    return Policy(Criteria(field_threshold=tidy3d_shutoff, energy_threshold=tidy3d_shutoff,
                           flux_tol=1e-3, patience=3, interval=interval))


def trace_ratio(pol) -> float:
    """The ``|E|^2`` ratio of the latest check for the decay trace, from this module's
    :class:`Policy` or from an OpenEM ``shutoff.Policy`` a caller passed in."""
    if hasattr(pol, "field_ratio"):
        return float(pol.field_ratio)
    fd = getattr(pol, "field_decay", None)
    return float(fd.ratio) if fd is not None else float("nan")


def energy_trace(pol) -> list:
    """``(step, energy)`` per check, from either kind of policy."""
    if hasattr(pol, "energy_trace"):
        return list(pol.energy_trace)
    ed = getattr(pol, "energy_decay", None)
    return list(ed.abs_history) if ed is not None else []


def source_end_step(sc) -> int:
    """The last step at which some source's sampled envelope (the very table that is injected)
    is above ``SOURCE_TAIL`` of that source's peak; 0 without sources."""
    tables = [w.amp_int for w in
              [s.waveform for s in sc.sources] + [d.waveform for d in sc.dipoles]
              + [t.waveform for t in getattr(sc, "tfsf_sources", [])]]
    last = 0
    for tab in tables:
        mag = np.abs(np.asarray(tab, dtype=np.float64))
        if not mag.size or not mag.max() > 0:
            continue
        above = np.nonzero(mag > SOURCE_TAIL * mag.max())[0]
        if above.size:
            last = max(last, int(above[-1]))
    return last
