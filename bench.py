"""Throughput benchmark of the FDTD step engine on the dispersive-bulk workload.

Workload: 512^3 cells (12-layer CPML on all faces included), dl = 0.02 um, 64 non-overlapping
Drude + Lorentz spheres (seed 0), a z-polarised point dipole at the centre, three mid-plane
field DFT monitors at 8 frequencies. A benchmark step is one FDTD time step of that grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload bulk|bloch] [--size N] [--no-e2e] [--no-cpu] [--no-secondary]
                    [--precision]

Prints one JSON line. ``value`` is device-timed (CUDA events on the run stream, max over
ranks) with the scene resident in HBM; ``e2e`` times the public ``solver.run`` call with host
arrays: table build and upload, the K steps, and the readout of every monitor, with the three
phases' host times. ``--impl reference`` times the FP64 NumPy transcription of OpenEM's step on
the host cores. Multi-GPU runs are independent replicas, one per GPU (the step has no exchange
between independent simulations).

``--workload bloch`` measures the Bloch metasurface cell instead (256 x 256 x 1024 complex
cells, Bloch phase 0.15 on x, CPML 12 on z, a 40-cell pixelated anisotropic layer, an oblique
plane wave, one flux plane at 200 frequencies); the default run reports a short measurement of
it under ``secondary``. ``--precision`` adds the DFT accumulation study of the Bloch cell's
32 x 32 x 1024 proxy (20,000 steps, 200 frequencies) to the Bloch line. ``--size`` scales the
bulk workload (sphere count by volume) for profiling runs; per-kernel times are in
``config.kernels_ms_per_launch``.
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


def n_spheres(n: int) -> int:
    """64 spheres at 512^3, the same density at other sizes."""
    return 64 if n == 512 else max(2, int(round(64 * (n / 512) ** 3)))


def workload_scene(n: int, steps: int):
    from openem_b200 import scenes
    return scenes.dispersive_spheres(n=n, n_sph=n_spheres(n), num_steps=steps)


def workload_name(n: int) -> str:
    return (f"dispersive_spheres {n}^3 (CPML 12 all faces, {n_spheres(n)} Drude+Lorentz spheres "
            f"seed 0, z-dipole, 3 mid-plane DFT monitors x 8 freqs)")


BLOCH_NAME = ("bloch_metasurface 256x256x1024 complex (Bloch 0.15 on x, periodic y, CPML 12 on "
              "z, 40-cell 64x64-pixel diagonal anisotropic layer seed 1, oblique s plane wave, "
              "flux plane x 200 freqs)")


# ---------------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and throttle reasons sampled while the timed steps run: NVML queried every few
    milliseconds from a thread (started once the steps are queued, stopped when the device has
    finished them), so that a timed region of a few tens of milliseconds still gets samples;
    nvidia-smi at 200 ms intervals when NVML is unavailable. Reads only; changes no setting."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None
        self.nv = None
        self.handle = None
        self.samples = []
        self.smax = None
        self.stopping = False
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            # the CUDA device's PCI address as NVML's "dddddddd:bb:dd.0" string (bytes: NVML
            # reads it through a char pointer)
            pr = torch.cuda.get_device_properties(index)
            ids = (getattr(pr, "pci_domain_id", None), getattr(pr, "pci_bus_id", None),
                   getattr(pr, "pci_device_id", None))
            if all(isinstance(v, int) for v in ids):
                busid = "{:08X}:{:02X}:{:02X}.0".format(*ids).encode("ascii")
                self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(busid)
            else:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(int(index))
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self.nv = pynvml
        except Exception:
            self.nv = None

    def start(self):
        if self.nv is not None:
            self.stopping = False
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
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

    def _poll(self):
        nv = self.nv
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stopping:
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM))
                mask = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
            except Exception:
                break
            self.samples.append((sm, {k for k, b in bits.items() if mask & b}))
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.nv is not None:
            self.stopping = True
            if self.thread:
                self.thread.join(timeout=2)
            sm = [v for v, _ in self.samples]
            reasons = set().union(*[r for _, r in self.samples]) if self.samples else set()
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}
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
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


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


def reduce_max(x: float, world: int, device: str = "cuda") -> float:
    """The largest ``x`` over the ranks (the slowest replica's time sets the whole job's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
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
    sc = scenes.small_dispersive(n=n, n_pml=12, n_sph=n_spheres(n), num_steps=steps + 1)
    o = ref64.Oracle(sc, steps + 1)
    o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    dt = time.perf_counter() - t0
    return n ** 3 * steps / dt / 1e9, dt


def _ref_replica(n: int, warmup: int, steps: int, barrier, out) -> None:
    """One process of the reference arm: the oracle's step on its own copy of the proxy scene,
    timed after every replica has finished its warm-up."""
    from openem_b200 import scenes
    from oracle import ref64
    sc = scenes.small_dispersive(n=n, n_pml=12, n_sph=n_spheres(n), num_steps=warmup + steps + 1)
    o = ref64.Oracle(sc, warmup + steps + 1)
    for _ in range(warmup):
        o.step()
    barrier.wait(timeout=600)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    out.put(time.perf_counter() - t0)


def reference_procs(requested: int) -> int:
    """Processes for the reference arm: every host core this process may run on, fewer when
    the available memory would not hold a replica (about 1 GB at 128^3) on each."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    r = requested if requested > 0 else int(cores or 1)
    avail = None
    try:  # MemAvailable counts the reclaimable page cache, unlike the free pages
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    avail = int(ln.split()[1]) * 1024
    except OSError:
        pass
    if avail:
        r = min(r, max(1, int(avail // (2 << 30))))
    return max(1, r)


def run_reference(args):
    """The reference's CPU implementation of the step on all the host's cores: one process per
    core (spawned, single-threaded numpy), each stepping its own copy of the proxy scene; the
    K steps of all replicas timed together (max over replicas), throughput summed."""
    world, rank, _ = dist_setup(args.gpus)
    if rank != 0:
        dist_done(world)
        return
    import multiprocessing as mp
    n = args.ref_size
    R = reference_procs(args.ref_procs)
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"  # inherited by the spawned replicas: one thread each
    # each K-step run stays within a few minutes: at most 60 timed steps per replica (about
    # 0.8 s each at 128^3 with every core busy); the line reports the steps it timed
    K = min(args.steps, 60)
    W = min(args.warmup, 5)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(R)
    out = ctx.Queue()
    procs = [ctx.Process(target=_ref_replica, args=(n, W, K, barrier, out)) for _ in range(R)]
    for p in procs:
        p.start()
    try:
        dts = [out.get(timeout=1800) for _ in range(R)]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    dt = max(dts)
    value = R * n ** 3 * K / dt / 1e9
    sample = (f"FP64 NumPy transcription of OpenEM's step (oracle/ref64.py), {R} single-threaded "
              f"processes of {os.cpu_count()} cores, each a {n}^3 proxy of the workload's "
              f"construction, {K} timed steps after {W} warm-up steps "
              f"(max over replicas {dt:.1f} s)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": K, "warmup": W,
            "ms_per_step": dt / K * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene factory)",
            "config": {"workload": workload_name(args.size) + f"; measured on {R} replicas of a "
                                                              f"{n}^3 proxy",
                       "parallelism": f"replicas x{R} (host processes)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": R, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    dist_done(world)


# ---------------------------------------------------------------------------------------------
# the Bloch cell: throughput and the precision of its DFT accumulation
# ---------------------------------------------------------------------------------------------
def measure_bloch(steps: int, warmup: int, e2e: bool, device: int = 0, clocks=None) -> dict:
    """Device-timed steps of the 256 x 256 x 1024 Bloch cell (value in complex cell-updates
    per second), the roofline of its dominant kernel, and optionally the same steps end to end
    through ``solver.run``; ``clocks`` (a ClockSampler) samples while the timed steps run and its
    record is returned under "clocks"."""
    import torch

    from openem_b200 import roofline, scenes, solver
    KT = min(steps, 20)
    sc = scenes.bloch_metasurface(num_steps=warmup + steps + KT)
    stream = torch.cuda.current_stream()
    plan = solver.Plan(sc, warmup + steps + KT, device=device, stream=stream, cplx=True)
    plan.run(warmup)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    plan.run(steps)
    b.record(stream)
    if clocks:
        clocks.start()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    ms = a.elapsed_time(b)
    plan.status()
    launches = plan.launches_per_step() * steps
    plan.enable_timing(True)
    plan.run(KT)
    plan.status()
    tm = plan.timing()
    plan.close()
    del plan
    torch.cuda.empty_cache()
    cells = int(np.prod(sc.shape))
    value = cells * steps / (ms * 1e-3) / 1e9
    peaks = roofline.measured_peaks(ROOT)
    b_cell = roofline.step_bytes_per_cell_complex(sc)
    kb = roofline.kernel_bytes_complex(sc)
    dom = max((k for k in kb if k in tm), key=lambda k: tm[k][1])
    t_launch = tm[dom][1] / tm[dom][0] * 1e-3
    out = {"workload": BLOCH_NAME, "metric": METRIC + " (complex cells)", "value": value,
           "unit": UNIT, "steps": steps, "warmup": warmup, "ms_per_step": ms / steps,
           "dtype": "f32 (re, im)", "step_bytes_per_cell": b_cell,
           "step_roofline_frac": value * b_cell / peaks["hbm_gbs"],
           "roofline": {"bound": "hbm", "kernel": dom,
                        "achieved": kb[dom] / t_launch / 1e9, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": kb[dom] / t_launch / 1e9 / peaks["hbm_gbs"],
                        "algorithmic_bytes_per_launch": kb[dom],
                        "peak_source": peaks["source"]},
           "kernels_ms_per_launch": {k: v[1] / v[0] for k, v in tm.items()},
           "gpu_launches": launches, "clocks": clk}
    if e2e:
        torch.cuda.synchronize()
        stats = {}
        t0 = time.perf_counter()
        solver.run(sc, num_steps=steps, use_shutoff=False, verbose=False, device=device,
                   stream=stream, stats=stats)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out["e2e"] = {"value": cells * steps / dt / 1e9, "unit": UNIT,
                      "h2d_bytes_per_step": stats["h2d_bytes"] / steps,
                      "d2h_bytes_per_step": stats["d2h_bytes"] / steps, "seconds": dt,
                      "setup_s": stats["setup_s"], "step_s": stats["step_s"],
                      "readout_s": stats["readout_s"]}
    return out


def _accumulate_modes(samples: np.ndarray, phase: np.ndarray, batch: int) -> dict:
    """The DFT of the E samples ``samples (S, C, P)`` (complex64) with the per-step E phases
    ``phase (S, nf, 4)`` (columns 0, 1) summed four ways on the GPU: every product in float64;
    float32 partials over ``batch`` steps added to float64 (the engine's scheme); one float32
    running sum; a float32 running sum with Kahan's compensation."""
    import torch
    dev = torch.device("cuda")
    S, C, P = samples.shape
    nf = phase.shape[1]
    v = torch.as_tensor(samples, device=dev)
    ph = torch.as_tensor(phase, device=dev)
    pe = torch.complex(ph[..., 0], ph[..., 1])
    ref = torch.zeros((nf, C, P), dtype=torch.complex128, device=dev)
    eng = torch.zeros_like(ref)
    part = torch.zeros((nf, C, P), dtype=torch.complex64, device=dev)
    f32 = torch.zeros_like(part)
    kc = torch.zeros_like(part)
    kahan = torch.zeros_like(part)
    for s in range(S):
        term = pe[s][:, None, None] * v[s][None]
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


def dft_precision_study(nx: int = 32, ny: int = 32, nz: int = 1024, steps: int = 20000,
                        nfreq: int = 200, npix: int = 8, oracle: bool = False) -> dict:
    """Precision of the flux-plane DFT on a proxy of the Bloch cell (the same transverse
    wavevector, ``npix`` x ``npix`` pixels). The plane's E is recorded every step by a field
    time monitor; the DFT of those very samples is re-formed on the host four ways
    (:func:`_accumulate_modes`), and each, with the device phasors, is compared with the
    float64 sum of the samples (``vs_fp64_sum``: the accumulation error alone) and, with
    ``oracle``, with the FP64 oracle's phasors of the same scene (``vs_oracle``: accumulation
    plus the float32 field trajectory). Errors are max |X - ref| / max |ref| over points,
    frequencies and the two tangential E components."""
    from openem_b200 import scenes, solver, tables
    sc = scenes.bloch_metasurface(nx=nx, ny=ny, nz=nz, npix=npix, nfreq=nfreq, num_steps=steps,
                                  bloch_k=(0.15 * nx / 256, 0.0, 0.0))
    mon = sc.flux_monitors[0]
    km = int(mon.plane_index)
    sc_rec = scenes.with_time_monitor(sc, name="plane", comps=(0, 1), origin=(0, 0, km),
                                      box=(nx, ny, 1), interval=1)
    t0 = time.perf_counter()
    res = solver.run(sc_rec, use_shutoff=False, verbose=False, return_fields=True)
    wall = time.perf_counter() - t0
    # slot m of the time monitor holds E^m; the DFT term of step n is E^(n+1), the last one
    # being the final field
    ts = np.asarray(res.time_samples["plane"]).astype(np.complex64)[:, :, :, :, 0]
    last = np.stack([np.asarray(res.fields[c])[:, :, km] for c in ("Ex", "Ey")])
    e = np.concatenate([ts[:, 1:], last.astype(np.complex64)[:, None]], axis=1)
    samples = np.ascontiguousarray(np.moveaxis(e, 1, 0)).reshape(steps, 2, nx * ny)
    phase = tables.phase_table(mon.freqs, sc.dt, steps, mon.apodization)
    batch = tables.batch_depth(nx * ny, 4)
    sums = _accumulate_modes(samples, phase, batch)
    dev = np.moveaxis(np.asarray(res.phasors["T"].data)[0:2].reshape(2, nfreq, nx * ny), 0, 1)
    modes = (("engine", dev), ("engine_scheme_host", sums["engine_scheme"]),
             ("fp32", sums["fp32"]), ("kahan", sums["kahan"]))
    out = {"grid": [nx, ny, nz], "steps": steps, "nfreq": nfreq, "batch": batch,
           "run_seconds": wall}
    ref = sums["fp64"]
    out["vs_fp64_sum"] = {k: float(np.abs(a - ref).max() / np.abs(ref).max()) for k, a in modes}
    if oracle:
        from oracle import ref64
        r = ref64.run(sc)
        oref = np.moveaxis(np.asarray(r.phasors["T"])[0:2].reshape(2, nfreq, nx * ny), 0, 1)
        out["vs_oracle"] = {k: float(np.abs(a - oref).max() / np.abs(oref).max())
                            for k, a in modes + (("fp64_sum", ref),)}
    return out


# ---------------------------------------------------------------------------------------------
# the engine
# ---------------------------------------------------------------------------------------------
def run_bloch_line(args):
    world, rank, local = dist_setup(args.gpus)
    import torch
    torch.cuda.set_device(local)
    barrier(world)
    clocks = ClockSampler(local) if rank == 0 else None
    m = measure_bloch(args.steps, args.warmup, e2e=not args.no_e2e, device=local, clocks=clocks)
    clk = m.pop("clocks")
    ms_max = reduce_max(m["ms_per_step"] * args.steps, world)
    if rank == 0:
        cells = 256 * 256 * 1024
        line = {"metric": METRIC, "value": world * cells * args.steps / (ms_max * 1e-3) / 1e9,
                "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded scene factory)",
                "config": {"workload": BLOCH_NAME, "cells": cells,
                           "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2: 6.4 GB of complex fields per step",
                           "step_bytes_per_cell": m["step_bytes_per_cell"],
                           "step_roofline_frac": m["step_roofline_frac"],
                           "kernels_ms_per_launch": m["kernels_ms_per_launch"]},
                "roofline": m["roofline"], "cpu_baseline": None, "e2e": m.get("e2e"),
                "gpu_launches": m["gpu_launches"], "clocks": clk}
        if args.precision:
            line["config"]["dft_precision"] = dft_precision_study()
        print(json.dumps(line), flush=True)
    dist_done(world)


def run_serve_line(args):
    """The serving stream (``openem_b200.serve.measure_stream``): ``--requests`` requests of the
    N^3 stream, served with continuous batching against the same requests run serially; one
    replica per rank."""
    world, rank, local = dist_setup(args.gpus)
    from openem_b200 import serve
    m = serve.measure_stream(args.requests, device=local)
    value = reduce_max(-m["sims_per_s"], world)  # the slowest replica sets the whole job
    if rank == 0:
        line = {"metric": "served sims/s", "value": -value * world, "unit": "sims/s",
                "n_gpus": world, "steps": m["requests"], "warmup": 1,
                "ms_per_step": 1e3 * m["serve_seconds"] / m["requests"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded request stream)",
                "config": {"workload": "serving stream: N^3 grids, N log-uniform in [64, 384], "
                                       "1000-6000 steps, Poisson arrivals at 1.2x the serial "
                                       "capacity", **m},
                "cpu_baseline": None, "e2e": None, "gpu_launches": None, "clocks": None}
        print(json.dumps(line), flush=True)
    dist_done(world)


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
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(world)
    # the timed region: the captured step graph, as solver.run launches it; the clocks are
    # sampled from when the steps are queued until the device has finished them
    ev0.record(stream)
    plan.run(K)
    ev1.record(stream)
    if clocks:
        clocks.start()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    plan.status()
    launches = plan.launches_per_step() * K
    snap_in_e = plan.box_snapshots_in_update() > 0
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
    kb = roofline.kernel_bytes(sc, box_snapshots_in_e=snap_in_e)
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
               "seconds": dt, "setup_s": stats["setup_s"], "step_s": stats["step_s"],
               "readout_s": stats["readout_s"]}

    # a short device-timed run of the Bloch cell, reported beside the headline
    secondary = None
    if world == 1 and not args.no_secondary:
        secondary = {"bloch": measure_bloch(max(K, 50), W, e2e=False, device=local,
                                            clocks=ClockSampler(local))}

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
            "secondary": secondary,
        }
        print(json.dumps(line), flush=True)
    dist_done(world)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bulk", choices=["bulk", "bloch", "serve"])
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--ref-size", type=int, default=128)
    ap.add_argument("--ref-procs", type=int, default=0,
                    help="processes of the reference arm (0: one per host core)")
    ap.add_argument("--cpu-size", type=int, default=128)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--precision", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "bloch":
        run_bloch_line(args)
    elif args.workload == "serve":
        run_serve_line(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
