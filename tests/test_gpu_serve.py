"""The serving loop on the GPU: several requests in flight, each result identical to the same
request run alone through solver.run."""

import numpy as np
import pytest

from openem_b200 import serve as S
from openem_b200 import solver

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone():
    reqs = S.make_stream(5, seed=5, n_range=(32, 56), step_range=(150, 300))
    for q, r in enumerate(reqs):
        r.arrival = 0.002 * q
    tuner = S.Tuner(candidates=(8, 16))
    srv = S.Server(max_slots=3, chunk=64, tuner=tuner)
    got = srv.serve(reqs)
    assert len(got) == 5
    ev = [e for _t, e, _r in srv.log]
    assert ev.count("admit") == 5 and ev.count("done") == 5
    for d, r in zip(got, reqs):
        alone = solver.run(r.build(), num_steps=r.num_steps, use_shutoff=False, verbose=False)
        np.testing.assert_array_equal(d.result.phasors["T"].data, alone.phasors["T"].data)


def test_pinned_stager_copies_from_several_threads():
    """Plans built on several worker threads share one pinned staging buffer: concurrent large
    copies take turns and every array arrives intact."""
    import threading
    import torch
    from openem_b200 import tables_gpu as TG
    dev = torch.device("cuda", 0)
    arrays = [np.random.default_rng(q).random((1 << 25) + 1000 * q) for q in range(4)]
    out = [None] * 4

    def run(q):
        torch.cuda.set_device(0)
        with torch.cuda.stream(torch.cuda.Stream()):
            out[q] = TG._PinnedStager.copy(arrays[q], torch, dev)
            torch.cuda.current_stream().synchronize()

    ts = [threading.Thread(target=run, args=(q,)) for q in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for a, t in zip(arrays, out):
        np.testing.assert_array_equal(t.cpu().numpy(), a)
