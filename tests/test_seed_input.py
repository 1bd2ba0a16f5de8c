"""The CMSSW entry point LST::run / LST::prepareInput on the CPU: the oracle
(the reference's SDL/LST.cc compiled in oracle/_ref with ROOT's XYZVector
restated in oracle/ref/shim/Math) against the committed known answers in
tests/golden/seed_pins.json, and the host side of the C ABI's seed packing
(lst_seed_pack runs on the host; no GPU is involved)."""
import ctypes
import json
import os
import sys

import numpy as np
import pytest

from oracle import reflib
from tracklooper_b200 import gen, lst

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

PINS = json.load(open(os.path.join(HERE, "golden", "seed_pins.json")))


@pytest.fixture(scope="module")
def ref():
    if not reflib.available("cr"):
        pytest.fail("oracle/_ref/liblstref_cr.so is not built (run __graft_entry__.build())")
    r = reflib.RefLST("cr")
    yield r
    r.close()


def _id(r):
    return f"cfg{r['config']}-ev{r['index']}"


@pytest.mark.parametrize("rec", PINS["events"], ids=_id)
def test_generator_reproduces_pinned_seeds(rec):
    seeds = gen.generate_event(rec["config"], rec["index"], rec["pileup"]).seeds
    assert (seeds.n_seeds, seeds.n_ph2) == (rec["n_seeds"], rec["n_ph2"])
    assert make_golden.seed_digest(seeds) == rec["inputs"]


@pytest.mark.parametrize("rec", [r for r in PINS["events"] if r["config"] != 5], ids=_id)
def test_reference_reproduces_seed_pins(ref, rec):
    seeds = gen.generate_event(rec["config"], rec["index"], rec["pileup"]).seeds
    got = make_golden.seed_pins_for(ref, seeds, "output" in rec)
    for key in ("n_hits", "n_pls", "prepare", "n_tc", "run"):
        assert got[key] == rec[key], key
    if "output" in rec:
        assert got["output"] == rec["output"]


def test_reference_conversion_agrees_with_generator_layout(ref):
    """Where the generator's own conversion (the standalone convention of
    code/core/trkCore.cc) and LST::prepareInput must agree -- which seeds are
    kept, their pseudo-hit indices, quadruplet flags and superbins -- they do;
    ptIn, eta, phi differ only in rounding (the generator converts from double
    precision, LST.cc from the float seed arrays)."""
    inp = gen.generate_event(2, 0)
    prep = ref.prepare_input(inp.seeds)
    assert prep["in_ptIn_vec_"].size == inp.n_pls
    for k, name in (("in_hitIndices_vec0_", "hitIndices0"), ("in_hitIndices_vec3_", "hitIndices3"),
                    ("in_isQuad_vec_", "isQuad"), ("in_superbin_vec_", "superbin")):
        np.testing.assert_array_equal(prep[k], inp.pls[name], err_msg=k)
    np.testing.assert_array_equal(prep["in_hitIdxs_"], inp.idxInNtuple)
    np.testing.assert_allclose(prep["in_ptIn_vec_"], inp.pls["ptIn"], rtol=1e-6)
    np.testing.assert_allclose(prep["in_eta_vec_"], inp.pls["eta"], rtol=1e-5, atol=1e-6)
    # pseudo-hits carry detId 1 after the outer-tracker hits
    assert np.all(prep["in_hitId_"][inp.n_ot_hits:] == 1)
    assert np.all(prep["in_hitId_"][:inp.n_ot_hits] != 1)


def _expected_blob(seeds) -> bytes:
    """The packed seed-event layout of include/lst_b200.h, built in numpy."""
    n_sh = int(seeds.hit_offsets[-1])
    parts = [np.array([seeds.n_ph2, seeds.n_seeds, n_sh, 0x4453534C], np.uint32).tobytes()]
    for a, dt in ((seeds.ph2_detId, np.uint32), (seeds.ph2_x, np.float32), (seeds.ph2_y, np.float32),
                  (seeds.ph2_z, np.float32)):
        parts.append(np.ascontiguousarray(a, dt).tobytes())
    for k in gen.SEED_FLOAT_FIELDS:
        parts.append(np.ascontiguousarray(seeds.see[k], np.float32).tobytes())
    parts.append(np.ascontiguousarray(seeds.see["see_q"], np.int32).tobytes())
    parts.append(np.ascontiguousarray(seeds.hit_offsets, np.uint32).tobytes())
    parts.append(np.ascontiguousarray(seeds.hit_idx, np.int32).tobytes())
    b = b"".join(parts)
    return b + bytes((-len(b)) % 16)


@pytest.mark.parametrize("config,index", [(1, 0), (1, 2), (3, 1)])
def test_seed_pack_layout(config, index):
    seeds = gen.generate_event(config, index, 40.0 if config == 3 else 0.0).seeds
    blob, offsets = lst.pack_seed_events([seeds])
    assert offsets.tolist() == [0]
    assert blob.size == lst.seed_packed_size(seeds.n_ph2, seeds.n_seeds, int(seeds.hit_offsets[-1]))
    assert blob.size % 16 == 0
    assert blob.tobytes() == _expected_blob(seeds)


def test_seed_pack_several_events_back_to_back():
    s = [gen.generate_event(1, i).seeds for i in range(3)]
    blob, offsets = lst.pack_seed_events(s)
    sizes = [len(_expected_blob(x)) for x in s]
    assert offsets.tolist() == [0, sizes[0], sizes[0] + sizes[1]]
    assert blob.tobytes() == b"".join(_expected_blob(x) for x in s)


def test_seed_pack_empty_event():
    empty = gen.SeedInput({k: np.zeros(0, np.float32) for k in gen.SEED_FLOAT_FIELDS} | {"see_q": np.zeros(0, np.int32)},
                          np.zeros(1, np.uint32), np.zeros(0, np.int32), np.zeros(0, np.uint32),
                          np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32))
    blob, _ = lst.pack_seed_events([empty])
    assert blob.tobytes() == _expected_blob(empty)


def _pack_one(seeds, capacity=None):
    c, keep = lst.seed_struct(seeds)
    size = lst.seed_packed_size(seeds.n_ph2, seeds.n_seeds, int(seeds.hit_offsets[-1]))
    buf = np.zeros(size if capacity is None else capacity, np.uint8)
    return lst.library().lst_seed_pack(ctypes.byref(c), buf.ctypes.data, buf.size)


def test_seed_pack_rejects_bad_inputs():
    seeds = gen.generate_event(1, 1).seeds
    assert _pack_one(seeds) == 0
    size = lst.seed_packed_size(seeds.n_ph2, seeds.n_seeds, int(seeds.hit_offsets[-1]))
    assert _pack_one(seeds, capacity=size - 16) == -1
    assert b"needs" in lst.library().lst_last_error()
    bad = gen.SeedInput(dict(seeds.see), seeds.hit_offsets.copy(), seeds.hit_idx, seeds.ph2_detId, seeds.ph2_x,
                        seeds.ph2_y, seeds.ph2_z)
    if bad.n_seeds >= 1:
        bad.hit_offsets[0] = 1
        assert _pack_one(bad) == -1
        assert b"offsets" in lst.library().lst_last_error()
    c, keep = lst.seed_struct(seeds)
    c.see_dz = None
    assert lst.library().lst_seed_pack(ctypes.byref(c), np.zeros(1 << 16, np.uint8).ctypes.data, 1 << 16) == -1
