"""The CUDA path against the committed known answers of the reference
(tests/golden/ref_pins.json), without running the reference."""
import json
import os
import sys

import numpy as np
import pytest

from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

PINS = json.load(open(os.path.join(HERE, "golden", "ref_pins.json")))


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def event(es):
    ev = lst.Event(es, max_hits=300000)
    yield ev
    ev.event_set.close()


@pytest.mark.parametrize("rec", PINS["events"], ids=lambda r: f"cfg{r['config']}-ev{r['index']}")
def test_cuda_matches_pins(es, event, rec):
    inp = gen.generate_event(rec["config"], rec["index"], rec["pileup"])
    event.run(inp)

    def get(name):
        return event.field(name)

    L = es.info["nLowerModules"]
    assert make_golden.stage_counts(get, L) == rec["counts"]
    sizes = {"H": event.event_set.max_hits, "MD": es.info["nTotalMDs"], "LS": es.info["nTotalSegments"],
             "T3": es.info["maxTriplets"], "T5": es.info["maxQuintuplets"]}
    from oracle import compare

    assert compare.store_digests(get, L, inp.n_hits, sizes) == rec["digests"]
    if "output" in rec:
        hits, ln, seed, typ = event.getOutput()
        assert [[int(t), h] for t, h in zip(typ, hits)] == rec["output"]
