"""Solve a serialized scene (``scene.npz``) on the sm_100a engine and store every monitor output
as ``ours.npz``: the wire format of OpenEM's solve worker (``openem/nb/solve_worker.py:25-45``),
so OpenEM's notebook backend reads this engine's outputs unchanged.

``ours.npz`` keys: ``mon:<name>`` flux-plane phasors (complex ``(4, nf, n1, n2)``),
``monf:<name>`` their frequencies, ``fld:<name>`` field phasors, ``tim:<name>`` time samples,
``ftm:<name>`` flux time series, and ``__meta`` (a JSON string of the run summary:
steps run, shutoff, stop reason, wall time, source end, energy trace).

In-process: :func:`solve_dir`; as a subprocess: ``python -m openem_b200.solve_worker <work>
<out> [--steps N]``. When the work directory holds ``td_coords.npz`` (target coordinates of the
field monitors in Tidy3D's convention), ``ours.npz`` also carries the ``tdf:`` / ``tdc:`` entries
of :func:`openem_b200.td_convention.to_tidy3d`, as OpenEM's worker writes them.
"""

from __future__ import annotations

import json
import os
import pathlib
import sys

import numpy as np

from openem_b200 import results, serialize, solver

OUT_MAX_GB = 20.0


def save_result(res, path, extra: dict | None = None) -> float:
    """Write ``res`` as ``ours.npz``; returns the megabytes written, or minus the megabytes that
    would have been written when they exceed ``OPENEM_OUT_MAX_GB`` (default 20; then only the
    summary goes to ``<path>.TOOBIG``)."""
    path = pathlib.Path(path)
    arrs = dict(extra or {})
    for n, p in res.phasors.items():
        arrs[f"mon:{n}"] = np.asarray(p.data)
        arrs[f"monf:{n}"] = np.asarray(p.freqs)
    for attr, tag in (("field_phasors", "fld"), ("time_samples", "tim"), ("flux_time", "ftm")):
        for n, a in (getattr(res, attr, {}) or {}).items():
            arrs[f"{tag}:{n}"] = np.asarray(a)
    meta = results.result_meta(res)
    total = sum(a.nbytes for a in arrs.values())
    if total > float(os.environ.get("OPENEM_OUT_MAX_GB", str(OUT_MAX_GB))) * 1e9:
        path.with_suffix(".TOOBIG").write_text(json.dumps(meta))
        return -total / 1e6
    np.savez(path, __meta=json.dumps(meta), **arrs)
    return total / 1e6


def load_result(path) -> dict:
    """``ours.npz`` back as ``{"meta": dict, "phasors": {name: (data, freqs)},
    "field_phasors": {...}, "time_samples": {...}, "flux_time": {...}}``."""
    with np.load(pathlib.Path(path), allow_pickle=False) as z:
        out = {"meta": json.loads(str(z["__meta"])), "phasors": {}, "field_phasors": {},
               "time_samples": {}, "flux_time": {}}
        tags = {"fld": "field_phasors", "tim": "time_samples", "ftm": "flux_time"}
        for k in z.files:
            if k.startswith("mon:"):
                n = k[4:]
                out["phasors"][n] = (z[k], z[f"monf:{n}"])
            elif k[:3] in tags and k[3:4] == ":":
                out[tags[k[:3]]][k[4:]] = z[k]
    return out


def solve_dir(work, out, steps: int | None = None) -> pathlib.Path:
    """Solve ``work/scene.npz`` (with the shutoff unless ``steps`` is given), write
    ``out/ours.npz`` and return its path."""
    work, out = pathlib.Path(work), pathlib.Path(out)
    out.mkdir(parents=True, exist_ok=True)
    sc = serialize.load(work / "scene.npz")
    res = solver.run(sc, num_steps=steps, use_shutoff=steps is None, verbose=True)
    extra = {}
    coords = work / "td_coords.npz"
    if coords.exists() and res.field_phasors:
        from openem_b200 import td_convention
        with np.load(coords) as z:
            extra = td_convention.to_tidy3d(sc, res.field_phasors, {k: z[k] for k in z.files})
    mb = save_result(res, out / "ours.npz", extra=extra)
    print(f"SOLVE|{work.name}|{res.steps_run}|{int(res.shutoff_triggered)}|"
          f"{res.stop_reason or '-'}|{int(np.prod(sc.shape))}|{res.wall_seconds:.1f}|{mb:.1f}",
          flush=True)
    return out / "ours.npz"


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("work")
    ap.add_argument("out")
    ap.add_argument("--steps", type=int, default=None)
    a = ap.parse_args(argv)
    solve_dir(a.work, a.out, steps=a.steps)
    return 0


if __name__ == "__main__":
    sys.exit(main())
