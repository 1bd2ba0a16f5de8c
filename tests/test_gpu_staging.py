"""Input staging on the copy stream (lst_batch_stage / lst_batch_ingest_staged):
the same object lists and outputs as lst_batch_upload, over several staged
batches that alternate between the two staging buffers, re-ingests of a
staged batch, seed-layout staging, and the error cases."""
import numpy as np
import pytest
import torch

from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


def _pinned(a):
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    t.numpy()[:] = a.view(np.uint8)
    return t.numpy()


def test_staged_batches_match_uploads(es):
    batches = [[gen.generate_event(3, 10 * b + i, 40.0) for i in range(3)] for b in range(3)]
    mh = max(e.n_hits for bt in batches for e in bt) + 1024
    ref_set = lst.EventSet(es, n_slots=3, max_hits=mh)
    s = lst.EventSet(es, n_slots=3, max_hits=mh)
    try:
        want = []
        for bt in batches:
            blob, off = lst.pack_events(bt)
            ref_set.upload_packed(0, blob, off)
            ref_set.run(0, 3)
            want.append(ref_set.output(0, 3))
        packed = [lst.pack_events(bt) for bt in batches]
        pinned = [(_pinned(b), o) for b, o in packed]
        s.stage(0, *pinned[0])
        for k in range(len(batches)):
            s.ingest_staged()
            s.run_graph(0, 3)
            if k + 1 < len(batches):
                s.stage(0, *pinned[k + 1])  # overlaps this batch's stages
            got = s.output(0, 3)
            for a, b in zip(got, want[k]):
                np.testing.assert_array_equal(a, b)
        # re-ingest the last staged batch from its buffer
        s.ingest(0, 3)
        s.run(0, 3)
        for a, b in zip(s.output(0, 3), want[-1]):
            np.testing.assert_array_equal(a, b)
    finally:
        s.close()
        ref_set.close()


def test_staged_seed_layout_matches_upload(es):
    seeds = [gen.generate_event(3, i, 40.0).seeds for i in range(2)]
    blob, off = lst.pack_seed_events(seeds)
    a = lst.EventSet(es, n_slots=2, max_hits=200000)
    b = lst.EventSet(es, n_slots=2, max_hits=200000)
    try:
        a.upload_seeds(0, blob, off)
        a.run(0, 2)
        b.stage(0, _pinned(blob), off, seed_layout=True)
        b.ingest_staged()
        b.run(0, 2)
        for x, y in zip(a.output(0, 2), b.output(0, 2)):
            np.testing.assert_array_equal(x, y)
    finally:
        a.close()
        b.close()


def test_staging_errors(es):
    s = lst.EventSet(es, n_slots=2, max_hits=100000)
    try:
        with pytest.raises(lst.LSTError):
            s.ingest_staged()  # nothing staged
        evs = [gen.generate_event(1, i) for i in range(2)]
        blob, off = lst.pack_events(evs)
        pb = _pinned(blob)
        s.stage(0, pb, off)
        with pytest.raises(lst.LSTError):
            s.stage(0, pb, off)  # the first is not ingested yet
        s.ingest_staged()
        with pytest.raises(lst.LSTError):
            s.stage(1, pb, off)  # two events from slot 1 overflow the set
    finally:
        s.close()
