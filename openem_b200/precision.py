"""Precision of the DFT accumulation on the Bloch configuration (256 x 256 x 1024 complex cells,
a 200-frequency flux plane, 20,000 steps): ``python -m openem_b200.precision [--full]``.

The monitor phasors are sums over every step of a float32 sample times a float32 phase
(``openem/kernels/source_dft.cu:332-530``). How they are summed decides their precision over
20,000 steps. This module separates that error from everything else by recording the monitor
plane itself every step with a field time monitor and re-forming the same DFT on the host from
those very samples, with the engine's own phase table:

* ``fp64``: every product added in float64: the exact sum of the recorded terms (reference);
* ``engine``: the device path, float32 partials over a snapshot batch of up to 32 steps, each
  batch added once to a float64 accumulator;
* ``fp32``: one float32 running sum over all steps;
* ``kahan``: a float32 running sum with Kahan's compensation term.

Each is reported as max |X - fp64| / max |fp64| over points, frequencies and the two
tangential E components of the plane (a field time monitor holds E^m exactly, the DFT term of
step n is E^(n+1); its H samples are time averages of two half steps, so H is not re-formed;
the device folds every component with the same code). The default is the 32 x 32 x 1024 proxy of the configuration
(8 x 8 pixels of 4 x 4 cells, the same transverse wavevector); ``--full`` also times the 256 x 256 x 1024 cell itself.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from openem_b200 import bloch, scenes, tables


def _accumulate(samples: np.ndarray, phase: np.ndarray, batch: int) -> dict:
    """The four sums of the E samples ``samples (S, C, P)`` times the per-step E phases
    ``phase (S, nf, 4)`` (columns 0, 1)."""
    import torch
    dev = torch.device("cuda")
    S, C, P = samples.shape
    nf = phase.shape[1]
    v = torch.as_tensor(samples, device=dev)                     # complex64
    ph = torch.as_tensor(phase, device=dev)                      # float32
    pe = torch.complex(ph[..., 0], ph[..., 1])                   # (S, nf) complex64
    ref = torch.zeros((nf, C, P), dtype=torch.complex128, device=dev)
    eng = torch.zeros_like(ref)
    part = torch.zeros((nf, C, P), dtype=torch.complex64, device=dev)
    f32 = torch.zeros_like(part)
    kc = torch.zeros_like(part)
    kahan = torch.zeros_like(part)
    for s in range(S):
        term = pe[s][:, None, None] * v[s][None]                  # complex64 products
        ref += pe[s].to(torch.complex128)[:, None, None] * v[s].to(torch.complex128)[None]
        part += term
        f32 += term
        y = term - kc
        t = kahan + y
        kc = (t - kahan) - y
        kahan = t
        if (s + 1) % batch == 0 or s == S - 1:
            eng += part.to(torch.complex128)
            part.zero_()
    return {"fp64": ref.cpu().numpy(), "engine_scheme": eng.cpu().numpy(),
            "fp32": f32.to(torch.complex128).cpu().numpy(),
            "kahan": kahan.to(torch.complex128).cpu().numpy()}


def study(nx: int = 32, ny: int = 32, nz: int = 1024, steps: int = 20000, nfreq: int = 200,
          npix: int = 8) -> dict:
    """Run the proxy with the E components of its flux plane recorded every step; return the
    four errors of the E phasors."""
    # the proxy keeps the full cell's transverse wavevector: bloch_k is in units of 2 pi / Lx
    sc = scenes.bloch_metasurface(nx=nx, ny=ny, nz=nz, npix=npix, nfreq=nfreq, num_steps=steps,
                                  bloch_k=(0.15 * nx / 256, 0.0, 0.0))
    mon = sc.flux_monitors[0]
    km = int(mon.plane_index)
    sc = scenes.with_time_monitor(sc, name="plane", comps=(0, 1), origin=(0, 0, km),
                                  box=(nx, ny, 1), interval=1)
    t0 = time.perf_counter()
    res = bloch.run(sc, use_shutoff=False, verbose=False, return_fields=True)
    wall = time.perf_counter() - t0
    # slot m of the time monitor holds E^m; the DFT term of step n is E^(n+1) (the last one,
    # E^steps, is the final field)
    ts = np.asarray(res.time_samples["plane"]).astype(np.complex64)[:, :, :, :, 0]
    last = np.stack([np.asarray(res.fields[c])[:, :, km] for c in ("Ex", "Ey")])
    e = np.concatenate([ts[:, 1:], last.astype(np.complex64)[:, None]], axis=1)
    samples = np.ascontiguousarray(np.moveaxis(e, 1, 0)).reshape(steps, 2, nx * ny)
    phase = tables.phase_table(mon.freqs, sc.dt, steps, mon.apodization)
    batch = tables.batch_depth(nx * ny, 4)
    sums = _accumulate(samples, phase, batch)
    dev = np.moveaxis(np.asarray(res.phasors["T"].data)[0:2].reshape(2, nfreq, nx * ny), 0, 1)
    ref = sums["fp64"]
    scale = np.abs(ref).max()
    out = {"grid": [nx, ny, nz], "steps": steps, "nfreq": nfreq, "batch": batch,
           "run_seconds": wall}
    for name, a in (("engine", dev), ("engine_scheme_host", sums["engine_scheme"]),
                    ("fp32", sums["fp32"]), ("kahan", sums["kahan"])):
        out[name] = float(np.abs(a - ref).max() / scale)
    return out


def time_full(steps: int = 20000) -> dict:
    """Throughput of the 256 x 256 x 1024 Bloch cell with its 200-frequency flux plane."""
    import torch
    from openem_b200 import solver
    sc = scenes.bloch_metasurface(num_steps=steps)
    plan = solver.Plan(sc, steps, cplx=True)
    plan.run(20)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    plan.run(steps - 20)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    plan.status()
    plan.close()
    cells = int(np.prod(sc.shape))
    return {"grid": list(sc.shape), "steps_timed": steps - 20,
            "ms_per_step": ms / (steps - 20),
            "gcell_per_s": cells * (steps - 20) / (ms * 1e-3) / 1e9}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--full", action="store_true")
    args = ap.parse_args()
    print(json.dumps({"precision_proxy": study(steps=args.steps)}), flush=True)
    if args.full:
        print(json.dumps({"bloch_full": time_full(args.steps)}), flush=True)


if __name__ == "__main__":
    main()
