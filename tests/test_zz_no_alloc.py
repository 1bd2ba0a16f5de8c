"""lst_batch_get_output_static (static device staging, no allocation) against
lst_batch_get_output, through the C ABI.  Kept in its own file, collected
last, so it runs both alone and after every other test."""
import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu


def _call(fn, eset, first, count, tc_cap, hit_cap):
    hits = np.full(hit_cap, 0xFFFFFFFF, np.uint32)
    ln = np.full(tc_cap, 0xFFFFFFFF, np.uint32)
    seed = np.full(tc_cap, -7, np.int32)
    typ = np.full(tc_cap, -7, np.int16)
    tco = np.zeros(count + 1, np.uint64)
    hco = np.zeros(count + 1, np.uint64)
    out = lst.Output(hits.ctypes.data, hits.size, ln.ctypes.data, seed.ctypes.data, typ.ctypes.data, ln.size,
                     tco.ctypes.data, hco.ctypes.data)
    rc = fn(eset.handle, first, count, ctypes.byref(out))
    ntc, nh = int(tco[-1]), int(hco[-1])
    return rc, (hits[:nh], ln[:ntc], seed[:ntc], typ[:ntc], tco, hco)


@pytest.fixture(scope="module")
def lib():
    lib = lst.library()
    lib.lst_batch_get_output_static.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(lst.Output)]
    lib.lst_batch_get_output_static.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


def test_static_output_matches_allocating_output(lib, es):
    inputs = [gen.generate_event(2, 40 + i) for i in range(3)]
    eset = lst.EventSet(es, n_slots=3, max_hits=max(i.n_hits for i in inputs) + 1024)
    blob, offsets = lst.pack_events(inputs)
    eset.upload_packed(0, blob, offsets)
    eset.run(0, 3)
    tc_cap, hit_cap = 3 * 31000, 3 * 31000 * 14
    for _ in range(2):  # two calls in a row of each
        rc_a, a = _call(lib.lst_batch_get_output, eset, 0, 3, tc_cap, hit_cap)
        rc_b, b = _call(lib.lst_batch_get_output_static, eset, 0, 3, tc_cap, hit_cap)
        assert rc_a == 0 and rc_b == 0, lib.lst_last_error()
        assert int(a[4][-1]) > 0
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    # a sub-range of slots
    rc_a, a = _call(lib.lst_batch_get_output, eset, 1, 2, tc_cap, hit_cap)
    rc_b, b = _call(lib.lst_batch_get_output_static, eset, 1, 2, tc_cap, hit_cap)
    assert rc_a == 0 and rc_b == 0
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    eset.close()


def test_static_output_rejects_oversize_batch(lib, es):
    n = 40  # ~150 kB of output per PU200-shaped event: well beyond the 4 MiB staging
    with ThreadPoolExecutor(max_workers=16) as pool:
        inputs = list(pool.map(lambda i: gen.generate_event(2, 60 + i), range(n)))
    eset = lst.EventSet(es, n_slots=n, max_hits=max(i.n_hits for i in inputs) + 1024)
    blob, offsets = lst.pack_events(inputs)
    eset.upload_packed(0, blob, offsets)
    eset.run(0, n)
    rc, _ = _call(lib.lst_batch_get_output_static, eset, 0, n, n * 31000, n * 31000 * 14)
    assert rc < 0
    assert b"static buffer" in lib.lst_last_error()
    # the allocating entry point still serves the whole batch, the static one a part of it
    rc_a, a = _call(lib.lst_batch_get_output, eset, 0, 4, 4 * 31000, 4 * 31000 * 14)
    rc_b, b = _call(lib.lst_batch_get_output_static, eset, 0, 4, 4 * 31000, 4 * 31000 * 14)
    assert rc_a == 0 and rc_b == 0
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    eset.close()
