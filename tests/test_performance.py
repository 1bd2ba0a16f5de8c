"""Track-candidate efficiency / fake / duplicate definitions
(tracklooper_b200/performance.py, restating code/core/trkCore.cc:231-403 and
code/core/write_sdl_ntuple.cc:206-308) on toy inputs and on the reference
CPU backend's track candidates."""
import numpy as np
import pytest

from oracle import reflib
from tracklooper_b200 import gen, lst, performance, t5dnn


def test_match_rule_more_than_75_percent_of_distinct_hits():
    sim = np.array([0, 0, 0, 1, 1, -1, 2, 2, 2, 2])
    # 3 of 4 distinct hits from particle 0 is not more than 75%: a fake
    assert performance.match([np.array([0, 1, 2, 3])], sim)[0] == -1
    # 4 of 5 distinct hits (one hit repeated) from particle 2: matched
    assert performance.match([np.array([6, 7, 8, 9, 9, 3])], sim)[0] == 2
    # noise never matches
    assert performance.match([np.array([5, 5, 5])], sim)[0] == -1


def test_match_agrees_with_the_t5_truth_labels():
    rng = np.random.default_rng(1)
    sim = rng.integers(-1, 4, size=200)
    hits = rng.integers(0, 200, size=(500, 10))
    lab = t5dnn.truth_labels(hits, sim)
    m = performance.match(list(hits), sim)
    assert np.array_equal(lab.astype(bool), m >= 0)


def test_duplicates_and_efficiency_counts():
    sim = np.array([0, 0, 0, 0, 1, 1, 1, 1])
    particles = np.zeros((3, 7))
    particles[:, 0] = [2.0, 3.0, 0.5]  # the third is below the pt threshold
    particles[:, 3] = 1
    particles[2, 4:7] = 1.0            # another vertex: pileup
    types = np.array([4, 4, 4])
    slots = np.zeros(14 * 3, np.uint32)
    slots[0:10] = [0, 1, 2, 3, 0, 1, 2, 3, 0, 1]
    slots[14:24] = [0, 1, 2, 3, 0, 1, 2, 3, 0, 1]
    slots[28:38] = [4, 5, 6, 7, 4, 5, 6, 7, 4, 5]
    e = performance.event_performance(types, slots, np.zeros(3), np.zeros((0, 4)), sim, particles)
    assert e["tc"] == 3 and e["fake"] == 0 and e["duplicate"] == 2
    assert e["hard"]["particles"] == 2 and e["hard"]["matched"] == 2
    c = performance.combine([e, e])
    assert c["duplicate_rate"] == pytest.approx(2 / 3) and c["hard"]["efficiency"] == 1.0


@pytest.mark.skipif(not reflib.available("cr"), reason="reference library not built")
def test_single_muons_are_found_without_fakes():
    dt = lst.field_dtypes()
    ref = reflib.RefLST("cr")
    try:
        evs = []
        for i in range(6):
            inp = gen.generate_event(1, i)
            ref.run_event(inp)
            evs.append(performance.from_store(lambda f: ref.field(f, dtype=dt[f]), inp, pt_min=0.5))
        c = performance.combine(evs)
    finally:
        ref.close()
    assert c["fake"] == 0
    assert c["hard"]["efficiency"] >= 5 / 6
