"""Run the dispersive-bulk workload at a chosen size for profiling and print per-kernel times.

    python -m openem_b200.profile_run --size 256 --steps 30 [--kernels tma|stream|basic|ws]
        [--no-pml] [--no-dispersion]

The scene is ``scenes.dispersive_spheres`` with the sphere count scaled by volume; the first 10
steps are warm-up, the rest are timed with CUDA events around each update kernel.
"""

from __future__ import annotations

import argparse
import os
from dataclasses import replace

import numpy as np


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--kernels", default=None)
    ap.add_argument("--no-pml", action="store_true")
    ap.add_argument("--no-dispersion", action="store_true")
    ap.add_argument("--no-monitors", action="store_true")
    a = ap.parse_args()
    if a.kernels:
        os.environ["OEM_B200_KERNELS"] = a.kernels
    from openem_b200 import model as M
    from openem_b200 import scenes, solver
    n = a.size
    sc = scenes.dispersive_spheres(n=n, n_sph=max(4, int(64 * (n / 512) ** 3)),
                                   num_steps=a.steps + 10, monitors=not a.no_monitors)
    if a.no_pml:
        axes = [M.Axis(ax.edges, "Periodic", "Periodic") for ax in sc.grid.axes]
        sc = replace(sc, grid=M.Grid(*axes), pml={})
    if a.no_dispersion:
        sc = replace(sc, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None)
    p = solver.Plan(sc, a.steps + 10)
    p.run(10)
    p.enable_timing(True)
    p.run(a.steps)
    p.status()
    tm = p.timing()
    cells = n ** 3
    for k, (c, ms) in tm.items():
        print(f"{k:10s} {c:5d} launches {ms / c:8.4f} ms/launch", flush=True)
    step = tm["step"][1] / tm["step"][0]
    print(f"{cells / step / 1e6:.2f} Gcell/s", flush=True)
    p.close()


if __name__ == "__main__":
    main()
