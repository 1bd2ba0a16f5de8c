"""Batched mode against the per-event drop-in on the same GPU: 128 uneven
events (generator configuration 3, pileup mean drawn per event from
140-250) run as two 64-event batches (CUDA-graph replay, autotuned launch
shapes) and one event at a time must give identical object counts and
identical track-candidate output lists, event by event."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu


def test_batched_equals_dropin():
    with ThreadPoolExecutor(8) as pool:
        events = list(pool.map(lambda i: gen.generate_event(3, 1000 + i), range(128)))
    es = lst.ES(device=0)
    mh = max(e.n_hits for e in events) + 1024
    batched = lst.EventSet(es, n_slots=64, max_hits=mh)
    single = lst.EventSet(es, n_slots=1, max_hits=mh)
    try:
        blob, off = lst.pack_events(events[:64])
        batched.upload_packed(0, blob, off)
        batched.autotune(0, 64)
        for b in range(2):
            part = events[64 * b:64 * (b + 1)]
            blob, off = lst.pack_events(part)
            batched.upload_packed(0, blob, off)
            batched.run_graph(0, 64)
            counts = batched.batch_counts(0, 64)
            hits, ln, seed, typ, tco, hco = batched.output(0, 64, tc_capacity=64 * 8000, hits_capacity=64 * 8000 * 14)
            for i, inp in enumerate(part):
                single.add_inputs(0, inp)
                single.run(0, 1)
                c1 = single.counts(0)
                assert c1 == counts[i], f"event {64 * b + i}"
                h1, l1, s1, t1, _, _ = single.output(0, 1)
                t0, t1_ = int(tco[i]), int(tco[i + 1])
                np.testing.assert_array_equal(l1, ln[t0:t1_])
                np.testing.assert_array_equal(s1, seed[t0:t1_])
                np.testing.assert_array_equal(t1, typ[t0:t1_])
                np.testing.assert_array_equal(h1, hits[int(hco[i]):int(hco[i + 1])])
    finally:
        single.close()
        batched.close()
        es.close()
