"""CUDA path vs the reference CPU backend, field by field, on seeded events.

The reference side is the unmodified reference code compiled for the CPU
against the serial Alpaka shim (oracle/_ref/liblstref_cr.so, strict IEEE
build); the CUDA side is _lst_b200.so driven through its C ABI.  Every live
object of every store must match bit for bit after each stage.
"""
import numpy as np
import pytest

from oracle import compare, reflib
from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu

STAGES = ("md", "ls", "t3", "t5", "pls_clean", "pt5", "pt3", "tc")


@pytest.fixture(scope="module")
def ref():
    if not reflib.available("cr"):
        pytest.fail("reference library oracle/_ref/liblstref_cr.so is not built")
    r = reflib.RefLST("cr")
    yield r
    r.close()


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def event(es):
    ev = lst.Event(es, max_hits=400000)
    yield ev
    ev.event_set.close()


def _sizes(es, event):
    info = es.info
    return {"H": event.event_set.max_hits, "MD": info["nTotalMDs"], "LS": info["nTotalSegments"],
            "T3": info["maxTriplets"], "T5": info["maxQuintuplets"]}


def _compare_event(ref, es, event, inp, stages=STAGES):
    dtypes = lst.field_dtypes()
    names = list(dtypes)
    ref.reset()
    ref.add_inputs(inp)
    event.event_set.add_inputs(0, inp)
    problems = []
    for st in stages:
        ref.run_stage(st)
        event.event_set.run_stage(0, st)

        def get_gpu(n):
            return event.field(n)

        def get_ref(n):
            return ref.field(n, dtype=dtypes[n])

        fields = compare.stage_fields(names, [st])
        p = compare.compare_stores(get_gpu, get_ref, fields, es.info["nLowerModules"], inp.n_hits, _sizes(es, event))
        if p:
            problems.append((st, p))
    return problems


def _fmt(problems):
    return "\n".join(f"[{st}] " + "\n   ".join(p) for st, p in problems)


@pytest.mark.parametrize("index", [0, 1, 2, 3])
def test_muon_gun_events(ref, es, event, index):
    inp = gen.generate_event(1, index)
    problems = _compare_event(ref, es, event, inp)
    assert not problems, _fmt(problems)


@pytest.mark.parametrize("index", [0, 1])
def test_pu200_events(ref, es, event, index):
    inp = gen.generate_event(2, index)
    problems = _compare_event(ref, es, event, inp)
    assert not problems, _fmt(problems)
    c = event.counts()
    assert c["nTrackCandidates"] > 1000


def _ref_output(ref, dtypes):
    """LST::getOutput restated on the reference's stores (SDL/LST.cc:367-427)."""
    n = int(ref.field("tc.nTrackCandidates", dtype=np.uint32)[0])
    types = ref.field("tc.trackCandidateType", dtype=np.int16)[:n]
    seeds = ref.field("tc.pixelSeedIndex", dtype=np.int32)[:n]
    th = ref.field("tc.hitIndices", dtype=np.uint32)
    idxs = ref.field("hits.idxs", dtype=np.uint32)
    hits = []
    for i in range(n):
        t = int(types[i])
        maxn = {7: 14, 5: 10, 4: 10, 8: 4}.get(t, 0)
        out = []
        for k in range(maxn):
            g = int(th[14 * i + k])
            h = g if t == 8 else int(idxs[g])
            if t != 4 and len(out) == 3 and out[-1] == h:
                continue
            out.append(h)
        hits.append(out)
    return hits, types, seeds


@pytest.mark.parametrize("index", [0])
def test_get_output_matches_reference(ref, es, event, index):
    inp = gen.generate_event(2, 10 + index)
    ref.run_event(inp)
    event.run(inp)
    hits, ln, seed, typ = event.getOutput()
    rhits, rtypes, rseeds = _ref_output(ref, lst.field_dtypes())
    assert len(hits) == len(rhits) > 0
    assert np.array_equal(typ, rtypes)
    assert np.array_equal(seed, rseeds)
    assert np.array_equal(ln, np.array([len(h) for h in rhits], np.uint32))
    assert hits == rhits


def test_batched_uneven_events_match_reference(ref, es):
    """Four uneven events (pileup 140-250) in one batched launch per kernel."""
    inputs = [gen.generate_event(3, i) for i in range(4)]
    eset = lst.EventSet(es, n_slots=4, max_hits=max(i.n_hits for i in inputs) + 1024)
    blob, offsets = lst.pack_events(inputs)
    eset.upload_packed(0, blob, offsets)
    eset.run(0, 4)
    dtypes = lst.field_dtypes()
    names = list(dtypes)
    sizes = {"H": eset.max_hits, "MD": es.info["nTotalMDs"], "LS": es.info["nTotalSegments"],
             "T3": es.info["maxTriplets"], "T5": es.info["maxQuintuplets"]}
    counts = eset.batch_counts(0, 4)
    for slot, inp in enumerate(inputs):
        ref.run_event(inp)
        p = compare.compare_stores(lambda n: eset.field(slot, n), lambda n: ref.field(n, dtype=dtypes[n]), names,
                                   es.info["nLowerModules"], inp.n_hits, sizes)
        assert not p, f"slot {slot}: " + "; ".join(p[:8])
        assert counts[slot]["nTrackCandidates"] == int(ref.field("tc.nTrackCandidates", dtype=np.uint32)[0])
    # the batch output equals the per-slot outputs
    hits, ln, seed, typ, tco, hco = eset.output(0, 4, tc_capacity=4 * 31000, hits_capacity=4 * 31000 * 14)
    for slot in range(4):
        h1, l1, s1, t1, _, _ = eset.output(slot, 1)
        a, b = int(tco[slot]), int(tco[slot + 1])
        assert np.array_equal(ln[a:b], l1) and np.array_equal(seed[a:b], s1) and np.array_equal(typ[a:b], t1)
        assert np.array_equal(hits[int(hco[slot]):int(hco[slot + 1])], h1)
    eset.close()


def test_fallback_walks_match_reference(ref, es):
    """The fallbacks taken for overflowing events -- the warp-per-module /
    per-pLS walks instead of the candidate lists, and the pair-by-pair
    duplicate-removal and pLS cross-cleaning tests instead of the shared-memory
    staged ones -- give the reference's objects."""
    inp = gen.generate_event(2, 3)
    ev = lst.Event(es, max_hits=inp.n_hits + 1024)
    ev.event_set.set_walk(True)
    problems = _compare_event(ref, es, ev, inp)
    ev.event_set.close()
    assert not problems, _fmt(problems)


def test_cut_only_method_matches_reference(es):
    if not reflib.available("cr_cuts"):
        pytest.skip("cut-only reference variant not built")
    ref_cuts = reflib.RefLST("cr_cuts")
    inp = gen.generate_event(2, 4)
    ev = lst.Event(es, max_hits=inp.n_hits + 1024)
    ev.event_set.set_t5_method(lst.T5_CUTS)
    problems = _compare_event(ref_cuts, es, ev, inp)
    ev.event_set.close()
    ref_cuts.close()
    assert not problems, _fmt(problems)


def test_graph_replay_matches_direct_launches(es):
    inputs = [gen.generate_event(3, 10 + i) for i in range(3)]
    eset = lst.EventSet(es, n_slots=3, max_hits=max(i.n_hits for i in inputs) + 1024)
    blob, offsets = lst.pack_events(inputs)
    eset.upload_packed(0, blob, offsets)
    eset.run(0, 3)
    direct = eset.output(0, 3, tc_capacity=3 * 31000, hits_capacity=3 * 31000 * 14)
    direct_counts = eset.batch_counts(0, 3)
    for _ in range(2):  # capture, then replay
        eset.ingest(0, 3)
        eset.run_graph(0, 3)
        out = eset.output(0, 3, tc_capacity=3 * 31000, hits_capacity=3 * 31000 * 14)
        assert eset.batch_counts(0, 3) == direct_counts
        for a, b in zip(direct, out):
            assert np.array_equal(a, b)
    eset.close()
