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
    return lst.Event(es, max_hits=400000)


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
            break
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
