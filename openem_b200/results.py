"""Output contract of the step engine: ``Phasors`` and ``Result``, with the field names and array
shapes of OpenEM's own result classes (``openem/results.py:18-84``), so code that consumes
OpenEM's ``Result`` (its notebook backend, the autograd hook) reads this engine's unchanged."""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Phasors:
    """Flux-plane phasors: ``data`` complex ``(4, nf, n1, n2)``, components E_t1, E_t2, H_t1,
    H_t2 with H colocated onto the E plane, transverse axes ascending."""

    name: str
    data: np.ndarray
    freqs: np.ndarray


def result_meta(res) -> dict:
    """Summary dict (``openem/results.py:32-48``)."""
    return {
        "steps_run": int(getattr(res, "steps_run", 0)),
        "triggered": bool(getattr(res, "shutoff_triggered", False)),
        "stop": getattr(res, "stop_reason", "") or "",
        "wall": float(getattr(res, "wall_seconds", 0.0)),
        "source_end": int(getattr(res, "source_end", -1)),
        "energy_trace": [[int(s), float(r)] for s, r in (getattr(res, "energy_trace", None) or [])],
    }


@dataclass
class Result:
    phasors: dict
    steps_run: int
    shutoff_triggered: bool
    decay_trace: list = field(default_factory=list)
    energy_trace: list = field(default_factory=list)
    source_end: int = -1
    wall_seconds: float = 0.0
    stop_reason: str = ""
    shutoff_summary: str = ""
    fields: dict = field(default_factory=dict)
    field_phasors: dict = field(default_factory=dict)
    time_samples: dict = field(default_factory=dict)
    time_slots: dict = field(default_factory=dict)
    flux_time: dict = field(default_factory=dict)
