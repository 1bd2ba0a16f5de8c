"""The CMSSW entry point on the GPU: the device seed conversion of
LST::prepareInput and the whole of LST::run through the C ABI
(lst_event_prepare_input, lst_batch_upload_seeds, lst_run) against the
reference's own SDL/LST.cc compiled for the CPU (oracle/_ref) and against the
committed known answers of tests/golden/seed_pins.json.

The conversion computes ROOT XYZVector quantities in double precision; only
log and atan2 can differ from the host libm in the last double bit, which
changes the float result only within 2^-29 of a rounding midpoint.  The
converted floats are therefore required to be bit-identical except for at
most one value in 10^5, and that one within 1 ulp; every integer output and
the complete chain downstream must match exactly."""
import json
import os
import sys

import numpy as np
import pytest

from oracle import compare, reflib
from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

PINS = json.load(open(os.path.join(HERE, "golden", "seed_pins.json")))
STAGES = ("md", "ls", "t3", "t5", "pls_clean", "pt5", "pt3", "tc")

FLOAT_PLS = (("in_ptIn_vec_", "ls.ptIn"), ("in_ptErr_vec_", "ls.ptErr"), ("in_px_vec_", "ls.px"),
             ("in_py_vec_", "ls.py"), ("in_pz_vec_", "ls.pz"), ("in_eta_vec_", "ls.eta"),
             ("in_etaErr_vec_", "ls.etaErr"), ("in_phi_vec_", "ls.phi"))
INT_PLS = (("in_charge_vec_", "ls.charge"), ("in_seedIdx_vec_", "ls.seedIdx"), ("in_superbin_vec_", "ls.superbin"),
           ("in_pixelType_vec_", "ls.pixelType"), ("in_isQuad_vec_", "ls.isQuad"))


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
def eset(es):
    s = lst.EventSet(es, n_slots=4, max_hits=400000)
    yield s
    s.close()


def _ulps(a, b):
    ai = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return np.abs(ai - bi)


def _check_floats(name, got, want):
    assert got.shape == want.shape, name
    u = _ulps(got, want)
    n_diff = int(np.count_nonzero(u))
    assert int(u.max(initial=0)) <= 1, f"{name}: {int(u.max())} ulp"
    return n_diff


def _check_conversion(eset, slot, prep):
    """GPU slot after the conversion vs the reference's prepareInput vectors."""
    c = eset.counts(slot)
    n_hits, n_pls = prep["in_trkX_"].size, prep["in_ptIn_vec_"].size
    assert (c["nHits"], c["nPixelSegments"]) == (n_hits, n_pls)
    assert (c["status"] & ~lst.STATUS_CAP_OVERFLOW) == 0
    n_diff = 0
    for k, f in (("in_trkX_", "hits.xs"), ("in_trkY_", "hits.ys"), ("in_trkZ_", "hits.zs")):
        n_diff += _check_floats(k, eset.field(slot, f, n_hits), prep[k])
    np.testing.assert_array_equal(eset.field(slot, "hits.detid", n_hits), prep["in_hitId_"])
    np.testing.assert_array_equal(eset.field(slot, "hits.idxs", n_hits), prep["in_hitIdxs_"])
    for k, f in FLOAT_PLS:
        n_diff += _check_floats(k, eset.field(slot, f, n_pls), prep[k])
    for k, f in INT_PLS:
        np.testing.assert_array_equal(eset.field(slot, f, n_pls).astype(np.int64), prep[k].astype(np.int64),
                                      err_msg=k)
    # pLS hit indices: ls.pLSHitsIdxs holds the four hit indices of each pLS
    hits4 = eset.field(slot, "ls.pLSHitsIdxs", 4 * n_pls).reshape(-1, 4) if n_pls else np.zeros((0, 4), np.uint32)
    # x, y, z, w = ntuple indices of hits 0, 2, 1, 3 (the inner and outer
    # pixel mini-doublets' anchor hits, then their outer hits)
    want4 = np.stack([prep[f"in_hitIndices_vec{i}_"] for i in (0, 2, 1, 3)], 1) if n_pls else hits4
    idxs = prep["in_hitIdxs_"]
    np.testing.assert_array_equal(hits4, idxs[want4] if n_pls else want4)
    assert n_diff <= max(1, (3 * n_hits + 8 * n_pls) // 100000)
    return n_diff


@pytest.mark.parametrize("rec", PINS["events"], ids=lambda r: f"cfg{r['config']}-ev{r['index']}")
def test_prepare_input_matches_reference(ref, eset, rec):
    seeds = gen.generate_event(rec["config"], rec["index"], rec["pileup"]).seeds
    prep = ref.prepare_input(seeds)
    eset.prepare_input(0, seeds)
    _check_conversion(eset, 0, prep)


def test_prepare_input_then_chain_matches_reference_stores(ref, es, eset):
    """Every object store after every stage, GPU (device conversion) vs the
    reference Event fed with the reference conversion."""
    seeds = gen.generate_event(3, 1, 40.0).seeds
    prep = ref.prepare_input(seeds)
    inp = reflib.prepared_event_input(prep)
    dtypes = lst.field_dtypes()
    names = list(dtypes)
    info = es.info
    sizes = {"H": eset.max_hits, "MD": info["nTotalMDs"], "LS": info["nTotalSegments"], "T3": info["maxTriplets"],
             "T5": info["maxQuintuplets"]}
    ref.reset()
    ref.add_inputs(inp)
    eset.prepare_input(0, seeds)
    problems = []
    for st in STAGES:
        ref.run_stage(st)
        eset.run_stage(0, st)
        p = compare.compare_stores(lambda n: eset.field(0, n), lambda n: ref.field(n, dtype=dtypes[n]),
                                   compare.stage_fields(names, [st]), info["nLowerModules"], inp.n_hits, sizes)
        if p:
            problems.append((st, p))
    assert not problems, problems


@pytest.mark.parametrize("rec", PINS["events"], ids=lambda r: f"cfg{r['config']}-ev{r['index']}")
def test_lst_run_matches_reference_run(ref, es, eset, rec):
    """lst_run (LST::run + hits/len/seedIdx/trackCandidateType) vs the
    reference's LST::run on the same CMSSW inputs."""
    seeds = gen.generate_event(rec["config"], rec["index"], rec["pileup"]).seeds
    want = ref.run_lst(seeds)
    algo = lst.LST(es, event_set=eset, slot=1).run_seeds(seeds)
    np.testing.assert_array_equal(algo.trackCandidateType(), want["trackCandidateType"])
    np.testing.assert_array_equal(algo.seedIdx(), want["seedIdx"])
    np.testing.assert_array_equal(algo.len(), want["len"])
    np.testing.assert_array_equal(algo.flat_hits(), want["hits"])


@pytest.mark.parametrize("rec", PINS["events"], ids=lambda r: f"cfg{r['config']}-ev{r['index']}")
def test_lst_run_matches_golden_pins(es, eset, rec):
    """The same without the reference: against the committed digests."""
    seeds = gen.generate_event(rec["config"], rec["index"], rec["pileup"]).seeds
    algo = lst.LST(es, event_set=eset, slot=2).run_seeds(seeds)
    run = {"hits": algo.flat_hits(), "len": algo.len(), "seedIdx": algo.seedIdx(),
           "trackCandidateType": algo.trackCandidateType()}
    assert algo.len().size == rec["n_tc"]
    assert {k: make_golden.array_digest(v) for k, v in sorted(run.items())} == rec["run"]
    if "output" in rec:
        assert [[int(t), int(s), h] for t, s, h in zip(algo.trackCandidateType(), algo.seedIdx(), algo.hits())] == \
            rec["output"]


def test_lst_class_reference_argument_list(ref, es, eset):
    """LST.run with the reference's argument list (see_hitIdx as nested lists)."""
    seeds = gen.generate_event(1, 1).seeds
    want = ref.run_lst(seeds)
    args = [seeds.see[k] for k in gen.SEED_FLOAT_FIELDS] + [seeds.see["see_q"], seeds.hit_lists(), seeds.ph2_detId,
                                                            seeds.ph2_x, seeds.ph2_y, seeds.ph2_z]
    algo = lst.LST(es, event_set=eset, slot=3).run(*args)
    np.testing.assert_array_equal(algo.flat_hits(), want["hits"])
    np.testing.assert_array_equal(algo.len(), want["len"])


def test_batched_seed_upload_matches_per_event_reference(ref, es):
    """Uneven events through lst_batch_upload_seeds + one batched run, with a
    re-ingest from the resident inbox, vs the reference's LST::run per event."""
    cases = [(1, 0, 0.0), (3, 2, 60.0), (1, 3, 0.0), (2, 1, 0.0), (3, 3, 20.0)]
    seeds = [gen.generate_event(c, i, p).seeds for c, i, p in cases]
    s = lst.EventSet(es, n_slots=len(seeds), max_hits=400000)
    try:
        blob, offsets = lst.pack_seed_events(seeds)
        s.upload_seeds(0, blob, offsets)
        s.run(0, len(seeds))
        first = s.output(0, len(seeds))
        s.ingest(0, len(seeds))
        s.run_graph(0, len(seeds))
        hits, ln, seed, typ, tco, hco = s.output(0, len(seeds))
        for a, b in zip(first, (hits, ln, seed, typ, tco, hco)):
            np.testing.assert_array_equal(a, b)
        for e, sd in enumerate(seeds):
            want = ref.run_lst(sd)
            t0, t1 = int(tco[e]), int(tco[e + 1])
            h0, h1 = int(hco[e]), int(hco[e + 1])
            np.testing.assert_array_equal(typ[t0:t1], want["trackCandidateType"])
            np.testing.assert_array_equal(seed[t0:t1], want["seedIdx"])
            np.testing.assert_array_equal(ln[t0:t1], want["len"])
            np.testing.assert_array_equal(hits[h0:h1], want["hits"])
    finally:
        s.close()


def _without_seeds(seeds, drop):
    keep = np.setdiff1d(np.arange(seeds.n_seeds), drop)
    lens = np.diff(seeds.hit_offsets.astype(np.int64))
    off = np.zeros(keep.size + 1, np.uint32)
    off[1:] = np.cumsum(lens[keep])
    idx = np.concatenate([seeds.hit_idx[seeds.hit_offsets[i]:seeds.hit_offsets[i + 1]] for i in keep]) \
        if keep.size else np.zeros(0, np.int32)
    return gen.SeedInput({k: v[keep] for k, v in seeds.see.items()}, off, idx, seeds.ph2_detId, seeds.ph2_x,
                         seeds.ph2_y, seeds.ph2_z)


def test_edge_cases(ref, es, eset):
    # no seeds and no hits: an empty event
    empty = gen.SeedInput({k: np.zeros(0, np.float32) for k in gen.SEED_FLOAT_FIELDS} | {"see_q": np.zeros(0, np.int32)},
                          np.zeros(1, np.uint32), np.zeros(0, np.int32), np.zeros(0, np.uint32),
                          np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32))
    algo = lst.LST(es, event_set=eset, slot=0).run_seeds(empty)
    assert algo.len().size == 0
    assert eset.counts(0)["status"] == 0

    # every seed below the pT threshold: hits only, no pLS
    seeds = gen.generate_event(3, 1, 40.0).seeds
    low = gen.SeedInput(dict(seeds.see), seeds.hit_offsets, seeds.hit_idx, seeds.ph2_detId, seeds.ph2_x, seeds.ph2_y,
                        seeds.ph2_z)
    low.see = {k: v.copy() for k, v in seeds.see.items()}
    low.see["see_stateTrajGlbPx"] *= np.float32(1e-3)
    low.see["see_stateTrajGlbPy"] *= np.float32(1e-3)
    low.see["see_ptErr"][:] = 0
    prep = ref.prepare_input(low)
    assert prep["in_ptIn_vec_"].size == 0
    eset.prepare_input(0, low)
    _check_conversion(eset, 0, prep)

    # a kept seed with only two pixel hits: dropped, slot flagged invalid,
    # the rest converted as the reference converts the event without it
    short = gen.generate_event(3, 1, 40.0).seeds
    ptl = np.hypot(short.see["see_stateTrajGlbPx"], short.see["see_stateTrajGlbPy"])
    victim = int(np.flatnonzero(ptl > 1.0)[0])
    lens = np.diff(short.hit_offsets.astype(np.int64))
    lens[victim] = 2
    off = np.zeros(short.n_seeds + 1, np.uint32)
    off[1:] = np.cumsum(lens)
    idx = np.concatenate([short.hit_idx[short.hit_offsets[i]:short.hit_offsets[i] + lens[i]]
                          for i in range(short.n_seeds)])
    bad = gen.SeedInput(short.see, off, idx, short.ph2_detId, short.ph2_x, short.ph2_y, short.ph2_z)
    eset.prepare_input(0, bad)
    c = eset.counts(0)
    assert c["status"] & lst.STATUS_INVALID_INPUT
    want = ref.prepare_input(_without_seeds(short, [victim]))
    got_seed = eset.field(0, "ls.seedIdx", c["nPixelSegments"])
    assert victim not in got_seed.tolist()
    np.testing.assert_array_equal(eset.field(0, "ls.superbin", c["nPixelSegments"]), want["in_superbin_vec_"])
    assert c["nHits"] == want["in_trkX_"].size

    # more hits than the slot holds: the event is rejected, as lst_batch_upload does
    small = lst.EventSet(es, n_slots=1, max_hits=1000)
    try:
        small.prepare_input(0, seeds)
        c = small.counts(0)
        assert c["status"] & lst.STATUS_HIT_CAPACITY
        assert (c["nHits"], c["nPixelSegments"]) == (0, 0)
    finally:
        small.close()
