"""The oracle: the reference CPU backend built from the reference sources
(oracle/_ref), checked against the committed known answers in
tests/golden/ref_pins.json, and the comparison machinery used by the parity
tests."""
import json
import os
import sys

import numpy as np
import pytest

from oracle import compare, reflib
from tracklooper_b200 import gen

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

PINS = json.load(open(os.path.join(HERE, "golden", "ref_pins.json")))


@pytest.fixture(scope="module")
def ref():
    if not reflib.available("cr"):
        pytest.fail("oracle/_ref/liblstref_cr.so is not built (run __graft_entry__.build())")
    r = reflib.RefLST("cr")
    yield r
    r.close()


@pytest.mark.parametrize("rec", PINS["events"], ids=lambda r: f"cfg{r['config']}-ev{r['index']}")
def test_generator_reproduces_pinned_inputs(rec):
    inp = gen.generate_event(rec["config"], rec["index"], rec["pileup"])
    assert (inp.n_hits, inp.n_pls) == (rec["n_hits"], rec["n_pls"])
    assert make_golden.input_digest(inp) == rec["inputs"]


@pytest.mark.parametrize("rec", PINS["events"], ids=lambda r: f"cfg{r['config']}-ev{r['index']}")
def test_reference_reproduces_pins(ref, rec):
    inp = gen.generate_event(rec["config"], rec["index"], rec["pileup"])
    counts, digests, get = make_golden.pins_for(ref, inp)
    assert counts == rec["counts"]
    assert digests == rec["digests"]
    if "output" in rec:
        assert make_golden.output_lists(get) == rec["output"]


def test_cut_only_variant_differs_only_from_t5_on(ref):
    if not reflib.available("cr_cuts"):
        pytest.skip("cut-only reference variant not built")
    cuts = reflib.RefLST("cr_cuts")
    inp = gen.generate_event(3, 0, 40.0)
    ref.run_event(inp, upto="t3")
    cuts.run_event(inp, upto="t3")
    for name in ("md.nMDs", "ls.nSegments", "t3.nTriplets"):
        assert np.array_equal(ref.field(name, dtype=np.uint32), cuts.field(name, dtype=np.uint32))
    ref.run_stage("t5")
    cuts.run_stage("t5")
    n_dnn = int(ref.field("t5.nQuintuplets", dtype=np.uint32).sum())
    n_cut = int(cuts.field("t5.nQuintuplets", dtype=np.uint32).sum())
    assert n_dnn > 0 and n_cut > 0 and n_dnn != n_cut
    cuts.close()


def test_compare_reports_bit_differences():
    L = 2
    base = {
        "ranges.miniDoubletModuleIndices": np.array([0, 4, 8], np.int32),
        "md.nMDs": np.array([2, 1, 0], np.uint32),
        "ranges.segmentModuleIndices": np.array([0, 5, 10], np.int32),
        "ls.nSegments": np.array([0, 0, 0], np.uint32),
        "ranges.tripletModuleIndices": np.array([0, 0], np.int32),
        "t3.nTriplets": np.array([0, 0], np.uint32),
        "ranges.quintupletModuleIndices": np.array([-1, -1], np.int32),
        "t5.nQuintuplets": np.array([0, 0], np.uint32),
        "pt3.nPixelTriplets": np.array([0], np.uint32),
        "pt5.nPixelQuintuplets": np.array([0], np.uint32),
        "tc.nTrackCandidates": np.array([0], np.uint32),
        "md.anchorX": np.array([1, 2, 99, 99, 3, 99, 99, 99, 99, 99, 99, 99], np.float32),
    }
    other = dict(base)
    other["md.anchorX"] = base["md.anchorX"].copy()
    other["md.anchorX"][2] = -5.0  # not a live entry: ignored
    sizes = {"H": 1, "MD": 12, "LS": 15, "T3": 7, "T5": 7}
    assert compare.compare_stores(base.get, other.get, ["md.anchorX"], L, 0, sizes) == []
    other["md.anchorX"][4] = np.nextafter(np.float32(3), np.float32(4))  # one ulp on a live entry
    p = compare.compare_stores(base.get, other.get, ["md.anchorX"], L, 0, sizes)
    assert len(p) == 1 and "1/3 differ" in p[0]
