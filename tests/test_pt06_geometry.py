"""The pt0.6 module and pixel maps (OT800_IT615_pt0.6), which the reference
ships in data/ but hard-codes away (SDL/LSTESData.cc:46-57 reads the pt0.8
directory; SDL/Constants.h:102-105 takes the pt cut from the compile-time
PT_CUT).  Here the event setup loads either directory and takes the pt cut
of the cuts from its name.

The reference cannot load these maps (1328 modules list more connected
modules than its 40-entry rows hold), so no reference run pins the pt0.6
results; the checks are on the maps themselves here and, on the GPU
(tests/test_gpu_pt06_geometry.py), the batched and per-event paths and the
tracer's re-evaluation of every stored object."""
import os

import numpy as np
import pytest

from tracklooper_b200 import geometry, lst

PT06 = "OT800_IT615_pt0.6"


def test_pt_cut_follows_the_geometry_name():
    for name, pt in (("OT800_IT615_pt0.8", 0.8), (PT06, 0.6)):
        es = lst.HostES(geometry.geometry_dir(name))
        assert es.info["ptCut"] == pytest.approx(pt)
        es.close()


def test_pt06_maps_differ_from_pt08():
    a = lst.HostES(geometry.geometry_dir())
    b = lst.HostES(geometry.geometry_dir(PT06))
    na = a.array("modules.nConnectedModules", np.uint16)
    nb = b.array("modules.nConnectedModules", np.uint16)
    assert na.size == nb.size and not np.array_equal(na, nb)
    a.close()
    b.close()


def test_pt06_module_map_rows_hold_every_connection():
    """The pt0.6 map lists up to 68 connected modules for 1328 modules, more
    than the reference's 40-entry rows (SDL/Constants.h:107) hold: its loader
    would write past them (SDL/ModuleMethods.h:127-134), so no reference run
    pins these maps.  Here every row holds its full list, in file order."""
    import struct

    d = geometry.geometry_dir(PT06)
    es = lst.HostES(d)
    try:
        det = es.array("modules.detIds", np.uint32)
        index = {int(x): i for i, x in enumerate(det)}
        nc = es.array("modules.nConnectedModules", np.uint16)
        mm = es.array("modules.moduleMap", np.uint16).reshape(-1, 80)
        data = open(os.path.join(d, "module_connection_tracing_merged.bin"), "rb").read()
        off, n_over = 0, 0
        while off + 8 <= len(data):
            key, n = struct.unpack_from("<II", data, off)
            conns = struct.unpack_from(f"<{n}I", data, off + 8)
            off += 8 + 4 * n
            if key not in index:
                continue
            i = index[key]
            assert nc[i] == n
            assert [int(x) for x in mm[i, :n]] == [index[c] for c in conns]
            n_over += n > 40
        assert n_over == 1328
    finally:
        es.close()
