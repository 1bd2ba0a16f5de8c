"""The event setup built on the device (lst_es_load_ex with
LST_ES_BUILD_ON_DEVICE) against the host build (csrc/es.cc), which the CPU
suite pins array by array to the reference's loader:

* every event-setup array is bit-identical, for the pt0.8 and the pt0.6
  geometry, and so are the sizes and the geometry hash;
* an event runs to the same track candidates on either setup;
* damaged geometry files give the host build's error message."""
import ctypes
import os
import shutil
import struct

import numpy as np
import pytest

from tracklooper_b200 import gen, geometry, lst

pytestmark = pytest.mark.gpu

ARRAYS = [
    "modules.detIds", "modules.moduleMap", "modules.mapdetId", "modules.mapIdx", "modules.nConnectedModules",
    "modules.drdzs", "modules.dxdys", "modules.partnerModuleIndices", "modules.layers", "modules.rings",
    "modules.modules", "modules.rods", "modules.subdets", "modules.sides", "modules.eta", "modules.r",
    "modules.isInverted", "modules.isLower", "modules.isAnchor", "modules.moduleType", "modules.moduleLayerType",
    "modules.sdlLayers", "modules.connectedPixels", "pixelmap.connectedPixelsIndex", "pixelmap.connectedPixelsSizes",
    "pixelmap.connectedPixelsIndexPos", "pixelmap.connectedPixelsSizesPos", "pixelmap.connectedPixelsIndexNeg",
    "pixelmap.connectedPixelsSizesNeg", "endcap.geoMapDetId", "endcap.geoMapPhi", "endcap.geoMapIndex",
    "caps.mdOffset", "caps.mdCap", "caps.lsOffset", "caps.lsCap", "caps.t3CapIfUsed", "caps.t5CapIfEligible",
    "hash.detHashKey", "hash.detHashVal",
]


def _raw(h, name):
    """The bytes of an event-setup array of handle h."""
    lib = lst.library()
    p, n, esz = ctypes.c_void_p(), ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.lst_es_host_array(h, name.encode(), ctypes.byref(p), ctypes.byref(n), ctypes.byref(esz)) == 0, name
    nbytes = n.value * esz.value
    return bytes((ctypes.c_char * nbytes).from_address(p.value)) if nbytes else b""


def _load(gdir, on_device):
    """(rc, message, handle) of lst_es_load_ex / lst_es_load_host."""
    lib = lst.library()
    h = ctypes.c_void_p()
    if on_device:
        rc = lib.lst_es_load_ex(str(gdir).encode(), None, 0, lst.ES_BUILD_ON_DEVICE, ctypes.byref(h))
    else:
        rc = lib.lst_es_load_host(str(gdir).encode(), ctypes.byref(h))
    return rc, lib.lst_last_error().decode(), h


@pytest.mark.parametrize("name", geometry.GEOMETRIES)
def test_device_build_matches_host_build(name):
    gdir = geometry.geometry_dir(name)
    rc_h, msg_h, hh = _load(gdir, False)
    rc_d, msg_d, hd = _load(gdir, True)
    assert rc_h == 0, msg_h
    assert rc_d == 0, msg_d
    lib = lst.library()
    try:
        for a in ARRAYS:
            assert _raw(hh, a) == _raw(hd, a), a
        ih, idv = lst.EsInfo(), lst.EsInfo()
        assert lib.lst_es_get_info(hh, ctypes.byref(ih)) == 0 and lib.lst_es_get_info(hd, ctypes.byref(idv)) == 0
        assert bytes(ih) == bytes(idv)
        assert lib.lst_es_geometry_hash(hh) == lib.lst_es_geometry_hash(hd)
    finally:
        lib.lst_es_free(hh)
        lib.lst_es_free(hd)


def test_event_on_device_built_setup():
    inp = gen.generate_event(2, 3)
    outs = []
    for on_device in (False, True):
        es = lst.ES(device=0, build_on_device=on_device)
        ev = lst.Event(es, max_hits=inp.n_hits + 1024)
        ev.run(inp)
        hits, length, seed, tc_type = ev.getOutput()
        outs.append((np.concatenate([np.asarray(h, np.int64) for h in hits]), np.asarray(length).copy(),
                     np.asarray(seed).copy(), np.asarray(tc_type).copy()))
        ev.event_set.close()
        es.close()
    assert len(outs[0][1]) > 1000
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def _copy_geometry(tmp_path):
    dst = tmp_path / "geom"
    shutil.copytree(geometry.geometry_dir(), dst)
    return dst


def _damage_pixel_map_detid(d):
    p = d / "pixelmap" / "pLS_map_layer1_subdet5.bin"
    data = bytearray(open(p, "rb").read())
    off = 0
    while True:
        key, n = struct.unpack_from("<II", data, off)
        if n > 0 and key >= 45000:
            break
        off += 8 + 4 * n
    struct.pack_into("<I", data, off + 8, 0xDEADBEEF)
    open(p, "wb").write(bytes(data))


def _too_many_connections(d):
    det = struct.unpack_from("<I", open(d / "sensor_centroids.bin", "rb").read(), 0)[0]
    with open(d / "module_connection_tracing_merged.bin", "ab") as f:
        f.write(struct.pack("<II", det, 81) + struct.pack("<81I", *([det] * 81)))


def _unknown_connection(d):
    det = struct.unpack_from("<I", open(d / "sensor_centroids.bin", "rb").read(), 0)[0]
    with open(d / "module_connection_tracing_merged.bin", "ab") as f:
        f.write(struct.pack("<III", det, 1, 0x7FFFFFF1))


def _missing_partner(d):
    data = open(d / "sensor_centroids.bin", "rb").read()
    open(d / "sensor_centroids.bin", "wb").write(data[20:])  # drops one sensor of a pair


def _duplicate_detid(d):
    data = open(d / "sensor_centroids.bin", "rb").read()
    open(d / "sensor_centroids.bin", "wb").write(data + data[:20])


def _missing_pixel_file(d):
    os.remove(d / "pixelmap" / "pLS_map_neg_layer2_subdet4.bin")


def _truncated_connection_map(d):
    full = open(d / "module_connection_tracing_merged.bin", "rb").read()
    open(d / "module_connection_tracing_merged.bin", "wb").write(full[:-2])


def _random_bytes(d):
    rng = np.random.default_rng(11)
    for name in ("sensor_centroids.bin", "module_connection_tracing_merged.bin"):
        size = os.path.getsize(d / name)
        open(d / name, "wb").write(rng.integers(0, 256, size=min(size, 1 << 16), dtype=np.uint8).tobytes())


@pytest.mark.parametrize("damage", [_damage_pixel_map_detid, _too_many_connections, _unknown_connection,
                                    _missing_partner, _duplicate_detid, _missing_pixel_file,
                                    _truncated_connection_map, _random_bytes])
def test_damaged_files_same_result_as_host_build(tmp_path, damage):
    d = _copy_geometry(tmp_path)
    damage(d)
    rc_h, msg_h, hh = _load(d, False)
    rc_d, msg_d, hd = _load(d, True)
    lib = lst.library()
    try:
        assert (rc_h == 0) == (rc_d == 0), (msg_h, msg_d)
        if rc_h:
            assert msg_d == msg_h
        else:
            for a in ARRAYS:
                assert _raw(hh, a) == _raw(hd, a), a
    finally:
        for h in (hh, hd):
            if h.value:
                lib.lst_es_free(h)
