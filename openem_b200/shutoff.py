"""Early-termination policy, the same three criteria and decisions as OpenEM's
(``openem/shutoff.py:19-253``), checked every ``interval`` steps by the step loop:

* field decay -- volume-weighted instantaneous ``sum V |E|^2`` over its running maximum;
* energy decay -- ``(eps0 sum V eps |E|^2 + mu0 sum V |H|^2) / 2`` over its running maximum,
  whose second-half log slope gives the decay time ``tau``;
* phasor convergence -- the relative change of the monitor fluxes per window, extrapolated by
  ``tau / window``, below ``tol`` for ``patience`` checks in a row.

A stop is only honoured after every source has finished injecting (:func:`source_end_step`).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

#: A source counts as finished once its envelope stays below this fraction of its peak.
SOURCE_TAIL = 1e-3


@dataclass
class FieldDecay:
    threshold: float
    peak: float = 0.0
    ratio: float = float("nan")
    history: list = field(default_factory=list)

    def update(self, step: int, metric: float) -> bool:
        self.peak = max(self.peak, metric)
        self.ratio = metric / self.peak if self.peak > 0 else 0.0
        self.history.append((step, self.ratio))
        return self.peak > 0 and self.ratio < self.threshold

    @property
    def deepest(self):
        if not self.history:
            return (0, float("nan"))
        i = int(np.argmin([r for _, r in self.history]))
        return self.history[i]


@dataclass
class EnergyDecay:
    threshold: float
    peak: float = 0.0
    ratio: float = float("nan")
    history: list = field(default_factory=list)
    abs_history: list = field(default_factory=list)

    def update(self, step: int, energy: float) -> bool:
        self.abs_history.append((step, float(energy)))
        self.peak = max(self.peak, energy)
        self.ratio = energy / self.peak if self.peak > 0 else 0.0
        self.history.append((step, self.ratio))
        return self.peak > 0 and self.ratio < self.threshold

    @property
    def tau(self) -> float:
        """Decay time in steps from a linear fit of ``ln(ratio)`` over the second half of the
        checks; ``inf`` while there are too few checks or the energy is not decaying."""
        h = self.history
        if len(h) < 8:
            return float("inf")
        arr = np.asarray(h[len(h) // 2:], dtype=np.float64)
        s, r = arr[:, 0], arr[:, 1]
        good = r > 0
        if good.sum() < 4:
            return float("inf")
        slope = np.polyfit(s[good], np.log(r[good]), 1)[0]
        if slope >= 0 or not np.isfinite(slope):
            return float("inf")
        return float(-1.0 / slope)


@dataclass
class PhasorConvergence:
    tol: float = 1e-3
    patience: int = 3
    window_steps: int = 400
    _prev: np.ndarray | None = None
    streak: int = 0
    rel: float = float("inf")
    per_window: float = float("inf")
    history: list = field(default_factory=list)

    def update(self, step: int, flux, decay_tau: float | None = None) -> bool:
        cur = np.asarray(flux, dtype=np.float64)
        if self._prev is None:
            self._prev = cur
            return False
        scale = float(np.max(np.abs(cur)))
        per = float(np.max(np.abs(cur - self._prev)) / scale) if scale > 0 else float("inf")
        self._prev = cur
        self.per_window = per
        if decay_tau is not None and np.isfinite(decay_tau) and decay_tau > 0:
            self.rel = per * decay_tau / max(self.window_steps, 1)
        else:
            self.rel = per
        self.history.append((step, self.rel))
        self.streak = self.streak + 1 if self.rel < self.tol else 0
        return self.streak >= self.patience


@dataclass
class Policy:
    field_decay: FieldDecay | None = None
    energy_decay: EnergyDecay | None = None
    phasor: PhasorConvergence | None = None
    interval: int = 400
    reason: str = ""

    def check(self, step: int, e2_weighted: float, energy: float, flux) -> bool:
        fired = []
        if self.field_decay is not None and self.field_decay.update(step, e2_weighted):
            fired.append(f"field_decay<{self.field_decay.threshold:g}")
        if self.energy_decay is not None and self.energy_decay.update(step, energy):
            fired.append(f"energy_decay<{self.energy_decay.threshold:g}")
        tau = self.energy_decay.tau if self.energy_decay is not None else None
        if (self.phasor is not None and np.size(flux) > 0
                and self.phasor.update(step, flux, decay_tau=tau)):
            fired.append(f"phasor_converged(remaining~{self.phasor.rel:.2e}<{self.phasor.tol:g}"
                         f" x{self.phasor.patience})")
        if fired:
            self.reason = " + ".join(fired)
            return True
        return False

    def summary(self) -> str:
        parts = []
        if self.field_decay is not None:
            s, r = self.field_decay.deepest
            parts.append(f"field_decay now {self.field_decay.ratio:.3e}, deepest {r:.3e}@{s}")
        if self.energy_decay is not None:
            parts.append(f"energy_decay now {self.energy_decay.ratio:.3e}")
        if self.phasor is not None:
            parts.append(f"phasor per window {self.phasor.per_window:.3e}, extrapolated "
                         f"remaining {self.phasor.rel:.3e}")
        return "; ".join(parts)


def default_policy(tidy3d_shutoff: float, interval: int = 400) -> Policy:
    return Policy(field_decay=FieldDecay(threshold=tidy3d_shutoff),
                  energy_decay=EnergyDecay(threshold=tidy3d_shutoff),
                  phasor=PhasorConvergence(tol=1e-3, patience=3, window_steps=interval),
                  interval=interval)


def source_end_step(sc) -> int:
    """Last whole step at which any source's envelope is above ``SOURCE_TAIL`` of its peak."""
    end = 0
    waves = ([s.waveform for s in sc.sources] + [d.waveform for d in sc.dipoles]
             + [t.waveform for t in sc.tfsf_sources])
    for w in waves:
        a = np.abs(np.asarray(w.amp_int, dtype=np.float64))
        peak = float(a.max()) if a.size else 0.0
        if peak <= 0:
            continue
        live = np.flatnonzero(a > SOURCE_TAIL * peak)
        if live.size:
            end = max(end, int(live[-1]))
    return end
