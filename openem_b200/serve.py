"""Continuous-batching simulation server on one GPU.

A request is a ``Scene`` and a step count with an arrival time. The server admits requests as
they arrive while a slot and HBM are free (admission by the plan's estimated device footprint),
builds each admitted simulation's plan (host tables, upload, graph capture) on a worker thread
while the device steps the plans already resident, gives every plan its own non-blocking CUDA
stream, and advances each in chunks of captured step graphs, so that the work of requests that
arrive while others run overlaps on the device. A finished plan is read out on its
own stream and its memory released lazily, in batches (``cudaFree`` waits for the whole device,
so freeing one plan at a time would stall every stream in flight).

Tile shapes: the warp-specialised update kernels walk a chunk of x planes per block; an
autotuner (:class:`Tuner`) times the candidate chunks once per grid-size class on a probe plan
and the server builds every plan of that class with the winner.

Each request's result is exactly what it would be alone: plans share nothing but the device.

    python -m openem_b200.serve [--requests 256 --min-n 64 --max-n 384 --min-steps 1000
                                 --max-steps 6000 --load 1.2]

(the defaults are the 256-request stream with N^3 grids, N log-uniform in [64, 384], 1000 to
6000 steps) prints one JSON line with sims/s and p50/p99 latency of the served stream against the
same requests run one at a time through :func:`openem_b200.solver.run`, and whether every served
result equals the serial one bit for bit. Scenes are built when their request is admitted.
"""

from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from openem_b200 import solver
from openem_b200.results import Result


@dataclass
class Request:
    """A simulation to serve. ``scene`` is a ``Scene``, or a callable that builds it: a stream of
    large requests then holds only the requests in flight on the host, each built on a plan
    worker when admitted. ``footprint`` (bytes) is the admission estimate; by default it is
    computed from the scene."""

    rid: int
    scene: object
    num_steps: int
    arrival: float = 0.0  # seconds after the start of serving
    footprint: int | None = None

    def build(self):
        """The request's Scene (built on each call when ``scene`` is a factory)."""
        return self.scene() if callable(self.scene) else self.scene

    def need(self) -> int:
        if self.footprint is None:
            self.footprint = footprint(self.build(), self.num_steps)
        return int(self.footprint)


@dataclass
class Done:
    rid: int
    result: Result
    arrival: float
    start: float
    finish: float

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def footprint(sc, num_steps: int) -> int:
    """Estimated device bytes of a plan of ``sc``: fields, material index, CPML psi, pole states
    and currents, monitor rings, accumulators and phase tables, plus a fixed margin."""
    nx, ny, nz = (int(v) for v in sc.shape)
    nzp = (nz + 31) // 32 * 32
    ncp = nx * ny * nzp
    b = 24 * ncp + 2 * ncp
    for a, n in enumerate((nx, ny, nz)):
        layers = sum(int(np.asarray(sc.pml[(a, s)].a_E).size) for s in ("lo", "hi")
                     if (a, s) in sc.pml)
        b += 16 * layers * (ncp // max(n, 1))
    if sc.dispersion is not None:
        npole = int(sc.dispersion.n_pole)
        b += 12 * npole + ncp // 8
    for m in sc.flux_monitors:
        t = [int(sc.shape[a]) for a in range(3) if a != m.axis]
        pts, nf = t[0] * t[1], int(np.size(m.freqs))
        b += 32 * 4 * 4 * pts + 2 * 4 * nf * pts * 8 + num_steps * nf * 16
    for m in sc.field_monitors:
        pts, nf = int(np.prod(m.box)), int(np.size(m.freqs))
        b += 32 * 6 * 4 * pts + 2 * 6 * nf * pts * 8 + num_steps * nf * 16
    return int(b + (32 << 20))


class Tuner:
    """Per grid-size class, the x-plane chunk of the update kernels that steps a probe plan
    fastest. A class is the padded grid shape; the probe is a vacuum scene of that shape with
    CPML on all faces, timed over ``steps`` steps per candidate with CUDA events."""

    def __init__(self, device: int = 0, candidates=(8, 16, 32, 64), steps: int = 30):
        import threading
        self.device = int(device)
        self.candidates = tuple(int(c) for c in candidates)
        self.steps = int(steps)
        self.cache: dict = {}
        self._lock = threading.Lock()  # plan workers tune one class at a time

    @staticmethod
    def size_class(sc) -> tuple:
        nx, ny, nz = (int(v) for v in sc.shape)
        return (nx, ny, (nz + 31) // 32 * 32)

    def xchunk(self, sc) -> int:
        key = self.size_class(sc)
        with self._lock:
            if key not in self.cache:
                self.cache[key] = self._tune(sc)
            return self.cache[key]

    def _tune(self, sc) -> int:
        from dataclasses import replace
        probe = replace(sc, dispersion=None, sigma_ex=None, sigma_ey=None, sigma_ez=None,
                        sources=[], field_monitors=[], flux_monitors=[],
                        field_time_monitors=[], num_time_steps=3 * self.steps)
        best, best_ms = 0, math.inf
        for c in self.candidates:
            if c > int(sc.shape[0]):
                continue
            p = solver.Plan(probe, 3 * self.steps, device=self.device, xchunk=c)
            try:
                p.run(self.steps)
                p.enable_timing(True)
                p.run(self.steps)
                p.status()
                tm = p.timing()
                ms = tm["update_h"][1] + tm["update_e"][1]
            finally:
                p.close()
            if ms < best_ms:
                best, best_ms = c, ms
        return best


def _plan_factory(req: Request, device: int, stream, tuner: Tuner | None):
    sc = req.build()
    xch = tuner.xchunk(sc) if tuner is not None else 0
    return solver.Plan(sc, req.num_steps, device=device, stream=stream, xchunk=xch)


class Server:
    """Admit, step and read out requests with continuous batching (see the module docstring).

    ``max_slots`` bounds the simulations in flight, ``mem_budget`` (bytes) their summed
    footprint; ``chunk`` is the number of steps issued to a plan at a time."""

    def __init__(self, device: int = 0, max_slots: int = 16, mem_budget: int | None = None,
                 chunk: int = 256, tuner: Tuner | None = None, plan_factory=None,
                 clock=time.perf_counter, stream_factory=None, event_factory=None,
                 build_workers: int = 4, keep=None):
        self.device = int(device)
        self.keep = keep  # applied to each Result as it completes (None: keep the Result)
        self.build_workers = int(build_workers)
        self.max_slots = int(max_slots)
        self.chunk = int(chunk)
        self.tuner = tuner
        self.clock = clock
        self.plan_factory = plan_factory or (lambda r, s: _plan_factory(r, self.device, s,
                                                                         self.tuner))
        if mem_budget is None:
            import torch
            free, _total = torch.cuda.mem_get_info(self.device)
            mem_budget = int(0.85 * free)
        self.mem_budget = int(mem_budget)
        if stream_factory is None:
            import torch
            stream_factory = lambda: torch.cuda.Stream(device=self.device)  # noqa: E731
            event_factory = lambda: torch.cuda.Event()  # noqa: E731
            self.device_ctx = lambda: torch.cuda.set_device(self.device)  # noqa: E731
        self.stream_factory = stream_factory
        self.event_factory = event_factory
        self.log: list = []  # (time, event, rid) for tests and reports

    def serve(self, requests) -> list:
        from concurrent.futures import ThreadPoolExecutor
        pool = ThreadPoolExecutor(max_workers=max(1, self.build_workers))
        try:
            return self._serve(requests, pool)
        finally:
            pool.shutdown(wait=True)

    def _build(self, req, stream):
        if self.device_ctx is None:
            return self.plan_factory(req, stream)
        import torch
        self.device_ctx()
        # device-side table builds run on a high-priority stream, so that their small kernels
        # are scheduled ahead of the pending blocks of the simulations in flight
        try:
            with torch.cuda.stream(torch.cuda.Stream(device=self.device, priority=-1)):
                return self.plan_factory(req, stream)
        finally:
            # the table build's temporaries stay in torch's cache otherwise, where the engine's
            # own allocations cannot reach them
            torch.cuda.empty_cache()

    device_ctx = None

    @staticmethod
    def _out_of_memory(exc) -> bool:
        return "out of memory" in str(exc) or "do not fit" in str(exc)

    @staticmethod
    def build_bytes(req) -> int:
        """Device memory a plan build needs on top of the plan while it runs (the float64 eps
        and sigma copies, keys and sort buffers of the device table build): 160 B per cell."""
        sc = req.scene if not callable(req.scene) else None
        if sc is not None:
            n = int(np.prod(sc.shape))
        else:
            n = int(req.need() // 26)  # the footprint is at least 26 B per cell
        return 160 * n

    def _serve(self, requests, pool) -> list:
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        active = []       # dicts: req, plan (or its future), stream, event, steps, start, bytes
        graveyard = []    # finished plans whose memory is released in batches
        used = 0
        hold = -1         # after a failed build: admit nothing until this many have finished
        building = 0      # transient bytes of the builds in flight
        dead_bytes = 0
        done = []
        t0 = self.clock()
        while pending or active:
            now = self.clock() - t0
            progressed = False
            # admission: arrived requests, while a slot and the memory budget allow (the plan
            # itself and, while it is being built, its build's transient buffers)
            while pending and pending[0].arrival <= now and len(active) < self.max_slots:
                if hold >= 0 and len(done) <= hold and active:
                    break
                req = pending[0]
                need = req.need()
                extra = self.build_bytes(req)
                if used + building + dead_bytes + need + extra > self.mem_budget and graveyard:
                    for p in graveyard:
                        p.close()
                    graveyard.clear()
                    dead_bytes = 0
                if used + building + need + extra > self.mem_budget and active:
                    break  # wait for a simulation to finish and free its memory
                pending.pop(0)
                stream = self.stream_factory()
                ent = {"req": req, "plan": None, "stream": stream, "event": self.event_factory(),
                       "steps": 0, "start": self.clock() - t0, "bytes": need, "extra": extra,
                       "future": pool.submit(self._build, req, stream)}
                active.append(ent)
                used += need
                building += extra
                self.log.append((ent["start"], "admit", req.rid))
                progressed = True
            # step: a built plan whose previous chunk has drained gets the next one
            for ent in list(active):
                if ent["plan"] is None:
                    if not ent["future"].done():
                        continue
                    building -= ent["extra"]
                    try:
                        ent["plan"] = ent["future"].result()  # re-raises a failed build
                    except RuntimeError as exc:
                        # the device was fuller than the estimates said: release what can be
                        # released and admit this request again once others have finished
                        if not self._out_of_memory(exc) or len(active) == 1:
                            raise
                        active.remove(ent)
                        used -= ent["bytes"]
                        for p in graveyard:
                            p.close()
                        graveyard.clear()
                        dead_bytes = 0
                        pending.insert(0, ent["req"])
                        hold = len(done)
                        self.log.append((self.clock() - t0, "retry", ent["req"].rid))
                        progressed = True
                        continue
                    self._issue(ent)
                    progressed = True
                    continue
                if not ent["event"].query():
                    continue
                req = ent["req"]
                if ent["steps"] < req.num_steps:
                    self._issue(ent)
                    progressed = True
                    continue
                res = self._readout(ent)
                if self.keep is not None:
                    res = self.keep(res)
                fin = self.clock() - t0
                done.append(Done(req.rid, res, req.arrival, ent["start"], fin))
                self.log.append((fin, "done", req.rid))
                active.remove(ent)
                used -= ent["bytes"]
                dead_bytes += ent["bytes"]
                graveyard.append(ent["plan"])
                progressed = True
            if not progressed:
                if not active and pending:
                    wait = pending[0].arrival - (self.clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
                else:
                    time.sleep(5e-5)
        for p in graveyard:
            p.close()
        return sorted(done, key=lambda d: d.rid)



    def _issue(self, ent) -> None:
        req = ent["req"]
        n = min(self.chunk, req.num_steps - ent["steps"])
        ent["plan"].run(n)
        ent["steps"] += n
        ent["event"].record(ent["stream"])

    @staticmethod
    def _readout(ent) -> Result:
        plan = ent["plan"]
        plan.flush()
        plan.status()
        tsamp, tslots = plan.time_samples(ent["steps"])
        return Result(phasors=plan.flux_phasors(), steps_run=ent["steps"],
                      shutoff_triggered=False, field_phasors=plan.field_phasors(),
                      time_samples=tsamp, time_slots=tslots)


def serial(requests, device: int = 0, keep=None) -> list:
    """The same requests one at a time through the plain engine (``solver.run``), back to back
    from t = 0, each scene built just before its run; returns Done records with the serial
    completion times. ``keep`` (a function of the Result) replaces each Result by what it
    returns, so that a long stream need not hold every result."""
    import torch
    out = []
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.rid):
        start = time.perf_counter() - t0
        res = solver.run(req.build(), num_steps=req.num_steps, use_shutoff=False, verbose=False,
                         device=device)
        torch.cuda.synchronize(device)
        out.append(Done(req.rid, keep(res) if keep else res, 0.0, start,
                        time.perf_counter() - t0))
    return out


def stream_footprint(n: int, num_steps: int, max_freqs: int = 32) -> int:
    """Admission estimate of a serving request before its scene exists: fields and index of an
    n^3 grid, CPML psi of 12-layer slabs, two poles per component in half the cells, one flux
    plane at ``max_freqs`` frequencies."""
    nzp = (n + 31) // 32 * 32
    ncp = n * n * nzp
    b = 26 * ncp + 3 * 16 * 2 * min(12, max(4, n // 8)) * n * nzp
    b += 12 * 2 * 3 * ncp // 2 + ncp // 8
    b += 32 * 4 * 4 * n * n + 2 * 4 * max_freqs * n * n * 8 + num_steps * max_freqs * 16
    return int(b + (32 << 20))


def make_stream(n_requests: int, seed: int = 3, n_range=(64, 384), step_range=(1000, 6000)):
    """The request stream: N log-uniform in ``n_range``, steps uniform in ``step_range``
    (``numpy.random.default_rng(seed)``), each scene from
    :func:`openem_b200.scenes.serving_request` with its own generator
    ``default_rng([seed, rid])``, built when the request is admitted."""
    from functools import partial

    from openem_b200 import scenes
    rng = np.random.default_rng(seed)
    reqs = []
    for q in range(n_requests):
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        steps = int(rng.integers(step_range[0], step_range[1] + 1))
        build = partial(_stream_scene, n, seed, q, steps)
        reqs.append(Request(q, build, steps, footprint=stream_footprint(n, steps)))
    return reqs


def _stream_scene(n: int, seed: int, rid: int, steps: int):
    from openem_b200 import scenes
    return scenes.serving_request(n, np.random.default_rng([seed, rid]), steps)


def digest(res) -> str:
    """A bit-exact fingerprint of a Result's flux phasors (served and serial runs compare
    these instead of holding every phasor array)."""
    import hashlib
    h = hashlib.sha1()
    for name in sorted(res.phasors):
        h.update(name.encode())
        h.update(np.ascontiguousarray(res.phasors[name].data).tobytes())
    return h.hexdigest()


def poisson_arrivals(requests, rate: float, seed: int = 3) -> None:
    """Arrival times of a Poisson process of ``rate`` requests per second, in place."""
    rng = np.random.default_rng(seed + 1)
    t = 0.0
    for r in requests:
        r.arrival = t
        t += float(rng.exponential(1.0 / rate))


def _percentiles(lat):
    lat = np.sort(np.asarray(lat))
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


def measure_stream(n_requests: int = 256, seed: int = 3, n_range=(64, 384),
                   step_range=(1000, 6000), load: float = 1.2, slots: int = 16,
                   workers: int = 4, tune: bool = False, device: int = 0) -> dict:
    """Serve a stream and run the same requests serially on the plain engine: sims/s of both,
    p50 / p99 latency, and whether every served result equals its serial one bit for bit
    (compared through :func:`digest`). ``load`` is the offered Poisson arrival rate as a multiple
    of the serial capacity measured first."""
    import torch
    torch.cuda.set_device(device)
    reqs = make_stream(n_requests, seed, n_range, step_range)
    tuner = Tuner(device) if tune else None
    # warm-up: the library and a first graph capture
    solver.run(reqs[0].build(), num_steps=10, use_shutoff=False, verbose=False, device=device)
    ser = serial(reqs, device, keep=digest)
    t_ser = ser[-1].finish
    rate = load * len(reqs) / t_ser
    poisson_arrivals(reqs, rate, seed)
    torch.cuda.empty_cache()  # the admission budget is measured from the free memory
    srv = Server(device, max_slots=slots, tuner=tuner, build_workers=workers, keep=digest)
    got = srv.serve(reqs)
    t_srv = max(d.finish for d in got) - min(r.arrival for r in reqs)
    same = all(g.result == s.result for g, s in zip(got, ser))
    p50, p99 = _percentiles([d.latency for d in got])
    s50, s99 = _percentiles([d.finish for d in ser])
    return {
        "metric": "served sims/s", "requests": len(reqs),
        "sims_per_s": len(reqs) / t_srv, "serial_sims_per_s": len(reqs) / t_ser,
        "ratio": t_ser / t_srv, "serve_seconds": t_srv, "serial_seconds": t_ser,
        "p50_latency_s": p50, "p99_latency_s": p99,
        "serial_p50_completion_s": s50, "serial_p99_completion_s": s99,
        "offered_load_x_serial": load, "arrival_rate_per_s": rate,
        "identical_to_alone": bool(same),
        "config": {"n_range": list(n_range), "step_range": list(step_range), "slots": slots,
                   "build_workers": workers, "seed": seed, "tuned": bool(tune)}}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--min-n", type=int, default=64)
    ap.add_argument("--max-n", type=int, default=384)
    ap.add_argument("--min-steps", type=int, default=1000)
    ap.add_argument("--max-steps", type=int, default=6000)
    ap.add_argument("--load", type=float, default=1.2,
                    help="offered load as a multiple of the serial capacity")
    ap.add_argument("--slots", type=int, default=16)
    ap.add_argument("--workers", type=int, default=4, help="plan-building threads")
    ap.add_argument("--tune", action="store_true", help="time the x-chunk per grid size")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(measure_stream(a.requests, a.seed, (a.min_n, a.max_n),
                                    (a.min_steps, a.max_steps), a.load, a.slots, a.workers,
                                    a.tune, a.device)), flush=True)


if __name__ == "__main__":
    main()
