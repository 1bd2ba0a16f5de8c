"""Seeded synthetic event generator: reproducible, shaped like the workloads
it stands in for (single-muon events, PU200 events, uneven pileup batches)."""
import numpy as np
import pytest

from tracklooper_b200 import gen


def test_same_seed_same_event():
    a = gen.generate_event(2, 7)
    b = gen.generate_event(2, 7)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.detId, b.detId)
    for k in a.pls:
        assert np.array_equal(a.pls[k], b.pls[k])


def test_different_seeds_differ():
    a = gen.generate_event(2, 7)
    b = gen.generate_event(2, 8)
    assert a.n_hits != b.n_hits or not np.array_equal(a.x, b.x)


def test_muon_gun_has_one_particle():
    e = gen.generate_event(1, 0)
    assert e.particles.shape[0] == 1
    assert 0.5 <= e.particles[0, 0] <= 50.0
    assert e.n_pls >= 1 and 5 <= e.n_ot_hits <= 40


def test_pu200_shape():
    e = gen.generate_event(2, 0)
    assert 80_000 <= e.n_ot_hits <= 250_000  # ~1-2e5 outer-tracker hits
    assert 3_000 <= e.n_pls <= 30_000
    # pLS hit indices point into the event's (pixel) hits
    for k in ("hitIndices0", "hitIndices1", "hitIndices2", "hitIndices3"):
        assert int(e.pls[k].max()) < e.n_hits
    assert set(np.unique(e.pls["pixelType"])) <= {0, 1, 2}
    assert set(np.unique(e.pls["isQuad"])) <= {0, 1}
    # outer-tracker hits are grouped by module (sorted by detId)
    ot = e.detId[e.detId != 1]
    assert np.all(np.diff(ot.astype(np.int64)) >= 0)


@pytest.mark.parametrize("config", [3, 5])
def test_other_configs_generate(config):
    e = gen.generate_event(config, 0)
    assert e.n_hits > 10_000 and e.n_pls > 100
