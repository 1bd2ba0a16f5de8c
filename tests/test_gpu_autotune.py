"""The launch-shape autotuner (lst_autotune / lst_autotune_load): object
lists do not depend on the launch shapes it picks, its choices stay within
each kernel's limits, and the per-geometry cache round-trips."""
import numpy as np
import pytest

from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def events():
    return [gen.generate_event(3, i, 60.0) for i in range(4)]


def _run(eset, events, graph=False):
    blob, off = lst.pack_events(events)
    eset.upload_packed(0, blob, off)
    if graph:
        eset.run_graph(0, len(events))
    else:
        eset.run(0, len(events))
    return eset.output(0, len(events))


def test_autotune_keeps_outputs_and_limits(es, events, tmp_path):
    s = lst.EventSet(es, n_slots=len(events), max_hits=max(e.n_hits for e in events) + 1024)
    try:
        before = _run(s, events)
        cache = str(tmp_path / "tune.txt")
        s.autotune(0, len(events), cache)
        shapes = s.launch_shapes()
        limits = {"kCreateMD": 8, "kMDDerived": 8, "kCreateLS": 4, "kCreateT3": 4, "kT5Eval": 4, "kPixEval<5>": 4,
                  "kPixEval<3>": 4, "kPixMid<5>": 4, "kPixMid<3>": 4}
        assert set(shapes) == set(limits)
        for k, (w, p) in shapes.items():
            assert 1 <= w <= limits[k] and 1 <= p <= 256, (k, w, p)
        for graph in (False, True):
            after = _run(s, events, graph)
            for a, b in zip(before, after):
                np.testing.assert_array_equal(a, b)
        # the cache: one line keyed by geometry hash, device, batch size, build
        lines = open(cache).read().splitlines()
        assert len(lines) == 1 and lines[0].startswith(f"g{es.geometry_hash():016x}-")
        s2 = lst.EventSet(es, n_slots=len(events), max_hits=s.max_hits)
        try:
            assert s2.autotune_load(len(events), cache)
            assert s2.launch_shapes() == shapes
            assert not s2.autotune_load(len(events) + 1, cache)
        finally:
            s2.close()
        # tuning again replaces the entry of the same key
        s.autotune(0, len(events), cache)
        assert len(open(cache).read().splitlines()) == 1
    finally:
        s.close()


def test_any_launch_shape_gives_the_same_objects(es, events):
    s = lst.EventSet(es, n_slots=len(events), max_hits=max(e.n_hits for e in events) + 1024)
    try:
        ref = _run(s, events)
        for k, (w, p) in ((0, (2, 4)), (2, (1, 32)), (3, (2, 8)), (4, (1, 4)), (5, (4, 32)), (6, (2, 8))):
            name = lst.library().lst_tune_kernel_name(k).decode()
            s.set_launch_shape(name, w, p)
        got = _run(s, events, graph=True)
        for a, b in zip(ref, got):
            np.testing.assert_array_equal(a, b)
        with pytest.raises(lst.LSTError):
            s.set_launch_shape("kCreateLS", 8, 16)  # above its 4-warp limit
        with pytest.raises(lst.LSTError):
            s.set_launch_shape("kCreateMD", 4, 0)
    finally:
        s.close()


def test_autotune_needs_resident_inputs(es, events):
    s = lst.EventSet(es, n_slots=2, max_hits=max(e.n_hits for e in events) + 1024)
    try:
        with pytest.raises(lst.LSTError):
            s.autotune(0, 2)
    finally:
        s.close()
