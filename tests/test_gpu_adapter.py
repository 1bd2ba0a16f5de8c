"""One event through the reference's C++ API on the B200 library: the
caller tests/adapter/sdl_caller.cc, written against SDL::Event<SDL::Acc> and
SDL::LST<SDL::Acc> (include/lst_sdl.hpp), against the reference CPU backend
(oracle/_ref/liblstref_cr.so) run on the same inputs: the track-candidate
store of the Event path, the mini-doublet counts per module and LST::run's
four outputs must be identical."""
import os
import subprocess

import numpy as np
import pytest

from oracle import reflib
from tests.adapter import caller_io
from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu


def test_reference_api_caller_matches_reference(tmp_path):
    if not reflib.available("cr"):
        pytest.fail("reference library oracle/_ref/liblstref_cr.so is not built")
    exe = caller_io.build(str(tmp_path))
    inp = gen.generate_event(2, 5)
    caller_io.write_input(str(tmp_path / "in.bin"), inp)
    from tracklooper_b200 import geometry

    geometry.geometry_dir()  # unpacks the geometry under <package>/data
    env = dict(os.environ, LST_BASE=os.path.dirname(os.path.abspath(lst.__file__)))
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = caller_io.read_output(str(tmp_path / "out.bin"))

    ref = reflib.RefLST("cr")
    try:
        ref.run_event(inp)
        n_tc = int(ref.field("tc.nTrackCandidates", dtype=np.uint32)[0])
        assert out["counts"][7] == n_tc > 1000
        assert np.array_equal(out["tc_type"], ref.field("tc.trackCandidateType", dtype=np.int16)[:n_tc])
        assert np.array_equal(out["tc_seed"], ref.field("tc.pixelSeedIndex", dtype=np.int32)[:n_tc])
        assert np.array_equal(out["tc_hits"], ref.field("tc.hitIndices", dtype=np.uint32)[:14 * n_tc])
        L = ref.n_lower
        assert np.array_equal(out["md_n"], ref.field("md.nMDs", dtype=np.uint32)[:L + 1])
        want = ref.run_lst(inp.seeds)
    finally:
        ref.close()
    assert np.array_equal(out["lst_hits"], want["hits"])
    assert np.array_equal(out["lst_len"], want["len"])
    assert np.array_equal(out["lst_seedIdx"], want["seedIdx"])
    assert np.array_equal(out["lst_type"], want["trackCandidateType"])
    # the counters agree with the Python mirror of the same library
    es = lst.ES(device=0)
    ev = lst.Event(es, max_hits=inp.n_hits + 1024)
    try:
        ev.run(inp)
        c = ev.counts()
        assert list(out["counts"][:8]) == [c["nHits"], c["nMiniDoublets"], c["nSegments"], c["nTriplets"],
                                           c["nQuintuplets"], c["nPixelTriplets"], c["nPixelQuintuplets"],
                                           c["nTrackCandidates"]]
    finally:
        ev.event_set.close()
        es.close()
