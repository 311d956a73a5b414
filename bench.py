"""Throughput benchmark of the FDTD step engine on the dispersive-bulk workload.

Workload: 512^3 cells (12-layer CPML on all faces included), dl = 0.02 um, 64 non-overlapping
Drude + Lorentz spheres (seed 0), a z-polarised point dipole at the centre, three mid-plane
field DFT monitors at 8 frequencies. A benchmark step is one FDTD time step of that grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line. ``value`` is device-timed (CUDA events on the run stream, max over
ranks) with the scene resident in HBM; ``e2e`` times the public ``solver.run`` call with host
arrays: table build and upload, the K steps, and the readout of every monitor.
``--impl reference`` times the FP64 NumPy transcription of OpenEM's step on the host cores.
Multi-GPU runs are independent replicas, one per GPU (the step has no exchange between
independent simulations).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s"
UNIT = "Gcell/s"


def workload_scene(n: int, steps: int):
    from openem_b200 import scenes
    return scenes.dispersive_spheres(n=n, num_steps=steps)


def workload_name(n: int) -> str:
    return (f"dispersive_spheres {n}^3 (CPML 12 all faces, 64 Drude+Lorentz spheres seed 0, "
            f"z-dipole, 3 mid-plane DFT monitors x 8 freqs)")


# ---------------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# distributed plumbing (replicas: barrier and max-reduction only)
# ---------------------------------------------------------------------------------------------
def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_done(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# CPU baseline: the FP64 oracle on a bounded sample of the same construction
# ---------------------------------------------------------------------------------------------
def cpu_oracle_rate(n: int, steps: int) -> tuple[float, float]:
    from openem_b200 import scenes
    from oracle import ref64
    sc = scenes.small_dispersive(n=n, n_pml=12, n_sph=max(2, int(64 * (n / 512) ** 3)),
                                 num_steps=steps + 1)
    o = ref64.Oracle(sc, steps + 1)
    o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    dt = time.perf_counter() - t0
    return n ** 3 * steps / dt / 1e9, dt


def run_reference(args):
    world, rank, _ = dist_setup(args.gpus)
    if rank != 0:
        dist_done(world)
        return
    n = args.ref_size
    from openem_b200 import scenes
    from oracle import ref64
    sc = scenes.small_dispersive(n=n, n_pml=12, n_sph=max(2, int(64 * (n / 512) ** 3)),
                                 num_steps=args.warmup + args.steps + 1)
    o = ref64.Oracle(sc, args.warmup + args.steps + 1)
    for _ in range(args.warmup):
        o.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step()
    dt = time.perf_counter() - t0
    value = n ** 3 * args.steps / dt / 1e9
    sample = (f"FP64 NumPy transcription of OpenEM's step (oracle/ref64.py), {n}^3 proxy of the "
              f"workload's construction, {args.steps} steps, 1 thread of {os.cpu_count()}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene factory)",
            "config": {"workload": workload_name(args.size) + f"; measured on a {n}^3 proxy",
                       "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    dist_done(world)


# ---------------------------------------------------------------------------------------------
# the engine
# ---------------------------------------------------------------------------------------------
def run_ours(args):
    world, rank, local = dist_setup(args.gpus)
    import torch

    from openem_b200 import roofline, solver
    torch.cuda.set_device(local)
    n = args.size
    K, W = args.steps, args.warmup
    KT = min(K, 50)  # steps of the per-kernel timing run after the timed region
    sc = workload_scene(n, W + K + KT)
    stream = torch.cuda.current_stream()
    plan = solver.Plan(sc, W + K + KT, device=local, stream=stream)
    plan.run(W)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(world)
    # the timed region: the captured step graph, as solver.run launches it
    ev0.record(stream)
    plan.run(K)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop() if clocks else None
    plan.status()
    launches = plan.launches_per_step() * K
    # per-kernel CUDA-event times (direct launches) for the roofline of the dominant kernel
    plan.enable_timing(True)
    plan.run(KT)
    plan.status()
    tm = plan.timing()
    plan.close()
    del plan
    torch.cuda.empty_cache()
    ms_max = reduce_max(ms, world)
    cells = int(np.prod(sc.shape))
    value = world * cells * K / (ms_max * 1e-3) / 1e9

    # roofline of the dominant kernel
    kb = roofline.kernel_bytes(sc)
    peaks = roofline.measured_peaks(ROOT)
    dom = max((k for k in ("update_he", "update_h", "update_e") if k in tm),
              key=lambda k: tm[k][1])
    t_launch = tm[dom][1] / tm[dom][0] * 1e-3
    achieved = kb[dom] / t_launch / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            tj = json.load(open(tfile))
            ent = tj.get(f"{dom}@{n}")
            traffic = None if ent is None else float(ent)
        except Exception:
            traffic = None
    b_cell = roofline.step_bytes_per_cell(sc)

    # end to end through the public API: tables, upload, K steps, readout
    e2e = None
    if not args.no_e2e:
        barrier(world)
        torch.cuda.synchronize()
        stats = {}
        t0 = time.perf_counter()
        solver.run(sc, num_steps=K, use_shutoff=False, verbose=False, device=local,
                   stream=stream, stats=stats)
        torch.cuda.synchronize()
        dt = reduce_max(time.perf_counter() - t0, world)
        e2e = {"value": world * cells * K / dt / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": stats["h2d_bytes"] / K,
               "d2h_bytes_per_step": stats["d2h_bytes"] / K,
               "seconds": dt}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cn, cs = args.cpu_size, args.cpu_steps
        rate, secs = cpu_oracle_rate(cn, cs)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"FP64 NumPy transcription (oracle/ref64.py) on a {cn}^3 proxy of the "
                         f"workload's construction, {cs} steps in {secs:.1f} s, 1 thread of "
                         f"{os.cpu_count()}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene factory)",
            "config": {
                "workload": workload_name(n), "grid": [n, n, n], "cells": cells,
                "parallelism": f"replicas x{world}",
                "l2": "inputs larger than L2: 3.2 GB of fields swept per step",
                "step_bytes_per_cell": b_cell,
                "step_roofline_frac": value / world * b_cell / peaks["hbm_gbs"],
                "kernels_ms_per_launch": {k: v[1] / v[0] for k, v in tm.items()},
            },
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "algorithmic_bytes_per_launch": kb[dom],
                         "peak_source": peaks["source"]},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    dist_done(world)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--ref-size", type=int, default=64)
    ap.add_argument("--cpu-size", type=int, default=96)
    ap.add_argument("--cpu-steps", type=int, default=60)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
