"""Admission and continuous batching of the serving loop, on the host with fake plans."""

import numpy as np

from openem_b200 import scenes
from openem_b200 import serve as S


class FakeEvent:
    """Completes `lag` queries after each record (a chunk that takes a little while)."""

    def __init__(self, lag=3):
        self.lag, self.left = lag, 0

    def record(self, stream):
        self.left = self.lag

    def query(self):
        self.left -= 1
        return self.left < 0


class FakePlan:
    def __init__(self, req):
        self.req, self.steps, self.closed = req, 0, False

    def run(self, n):
        self.steps += n

    def flush(self):
        pass

    def status(self):
        pass

    def time_samples(self, steps):
        return {}, {}

    def flux_phasors(self):
        return {"T": self.req.rid}

    def field_phasors(self):
        return {}

    def close(self):
        self.closed = True


def _server(**kw):
    plans = []

    def factory(req, stream):
        plans.append(FakePlan(req))
        return plans[-1]

    srv = S.Server(plan_factory=factory, stream_factory=lambda: object(),
                   event_factory=FakeEvent, **kw)
    return srv, plans


def _reqs(n=6, steps=1000, size=48, arrival_gap=0.0):
    rng = np.random.default_rng(0)
    sc = scenes.serving_request(size, rng, 50)
    return [S.Request(q, sc, steps, q * arrival_gap) for q in range(n)]


def _max_in_flight(log):
    cur = best = 0
    for _t, ev, _rid in sorted(log, key=lambda e: (e[0], e[1] == "admit")):
        cur += 1 if ev == "admit" else -1
        best = max(best, cur)
    return best


def test_every_request_completes_with_all_steps():
    srv, plans = _server(max_slots=4, mem_budget=1 << 40, chunk=300)
    done = srv.serve(_reqs())
    assert [d.rid for d in done] == list(range(6))
    assert all(p.steps == 1000 and p.closed for p in plans)
    assert all(d.result.steps_run == 1000 for d in done)


def test_slots_bound_the_simulations_in_flight():
    srv, _ = _server(max_slots=2, mem_budget=1 << 40, chunk=250)
    srv.serve(_reqs(6))
    assert _max_in_flight(srv.log) == 2


def test_memory_budget_admits_by_footprint():
    reqs = _reqs(4)
    one = reqs[0].need()
    srv, _ = _server(max_slots=8, mem_budget=int(1.5 * one), chunk=400)
    srv.serve(reqs)
    assert _max_in_flight(srv.log) == 1
    srv2, _ = _server(max_slots=8, mem_budget=int(3.5 * one), chunk=400)
    srv2.serve(_reqs(4))
    assert _max_in_flight(srv2.log) == 3


def test_footprint_grows_with_the_grid():
    rng = np.random.default_rng(1)
    a = S.footprint(scenes.serving_request(48, rng, 100), 100)
    b = S.footprint(scenes.serving_request(96, rng, 100), 100)
    margin = 32 << 20
    assert b - margin > 4 * (a - margin) > 0


def test_make_stream_and_arrivals():
    reqs = S.make_stream(5, seed=3, n_range=(32, 48), step_range=(100, 200))
    assert all(32 <= r.build().shape[0] <= 48 and 100 <= r.num_steps <= 200 for r in reqs)
    # scenes are built on demand, the same each time, and the admission estimate bounds them
    a, b = reqs[2].build(), reqs[2].build()
    np.testing.assert_array_equal(a.eps_ex, b.eps_ex)
    assert all(r.footprint >= S.footprint(r.build(), r.num_steps) for r in reqs)
    S.poisson_arrivals(reqs, rate=10.0)
    t = [r.arrival for r in reqs]
    assert t[0] == 0.0 and all(b > a for a, b in zip(t, t[1:]))


def test_a_build_that_runs_out_of_memory_is_admitted_again():
    """A plan build that finds the device fuller than the admission estimates (the engine reports
    an out-of-memory status) is put back at the head of the queue and built again once another
    request has finished; every request still completes."""
    plans, failed = [], []

    def factory(req, stream):
        if req.rid == 2 and not failed:
            failed.append(req.rid)
            raise RuntimeError("[oem status -6] finalize: cudaMalloc of 1 bytes failed: out of "
                               "memory")
        plans.append(FakePlan(req))
        return plans[-1]

    srv = S.Server(plan_factory=factory, stream_factory=lambda: object(),
                   event_factory=FakeEvent, max_slots=4, mem_budget=1 << 40, chunk=300)
    done = srv.serve(_reqs(5))
    assert [d.rid for d in done] == list(range(5))
    ev = [(e, r) for _t, e, r in srv.log]
    assert ("retry", 2) in ev
    assert [e for e, r in ev if r == 2].count("admit") == 2
    retry_at = ev.index(("retry", 2))
    assert any(e == "done" for e, _r in ev[:ev.index(("admit", 2), retry_at)])
