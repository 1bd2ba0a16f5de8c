"""Host-side failure paths of the C ABI, without a GPU.

Bad geometry and weight files must come back as a negative status with a
message, never as an abort, an exception through the ABI or a runaway
allocation.  The reference throws std::runtime_error or exits on these
(SDL/ModuleConnectionMap.cc:12-48, SDL/LSTESData.cc:14-75).  Every case here
fails while the files are read, before the first CUDA call, so it runs on a
machine without a GPU."""
import ctypes
import os
import shutil
import struct

import numpy as np
import pytest

from tracklooper_b200 import geometry, lst

GEOMETRY_FILES = ("sensor_centroids.bin", "endcap_orientation.bin", "tilted_barrel_orientation.bin",
                  "module_connection_tracing_merged.bin")


def _copy_geometry(tmp_path):
    """A private copy of the geometry directory whose files a test may damage."""
    src = geometry.geometry_dir()
    dst = tmp_path / "geom"
    shutil.copytree(src, dst)
    return dst


def _load_host(path):
    lib = lst.library()
    h = ctypes.c_void_p()
    rc = lib.lst_es_load_host(str(path).encode(), ctypes.byref(h))
    msg = lib.lst_last_error().decode()
    if rc == 0:
        lib.lst_es_free(h)
    return rc, msg


def test_missing_geometry_directory(tmp_path):
    rc, msg = _load_host(tmp_path / "does-not-exist")
    assert rc < 0
    assert "sensor_centroids.bin" in msg


@pytest.mark.parametrize("name", GEOMETRY_FILES)
def test_missing_geometry_file(tmp_path, name):
    d = _copy_geometry(tmp_path)
    os.remove(d / name)
    rc, msg = _load_host(d)
    assert rc < 0
    assert name in msg


def test_empty_sensor_file(tmp_path):
    d = _copy_geometry(tmp_path)
    open(d / "sensor_centroids.bin", "wb").close()
    rc, msg = _load_host(d)
    assert rc < 0 and "sensor_centroids.bin" in msg


def test_connection_map_with_huge_count_is_not_allocated(tmp_path):
    """A record claiming 2^32-1 connections is a truncated trailing record (as
    the reference drops it at end of file): it is skipped without allocating
    16 GiB, and the records before it load."""
    d = _copy_geometry(tmp_path)
    with open(d / "module_connection_tracing_merged.bin", "ab") as f:
        f.write(struct.pack("<II", 411309061, 0xFFFFFFFF))
        f.write(struct.pack("<I", 411309062))
    rc, msg = _load_host(d)
    assert rc == 0, msg


def test_truncated_connection_map_loads_complete_records(tmp_path):
    d = _copy_geometry(tmp_path)
    full = open(d / "module_connection_tracing_merged.bin", "rb").read()
    ref = lst.HostES(str(d))
    n_ref = ref.array("modules.nConnectedModules", np.uint16).copy()
    ref.close()
    # cut in the middle of the last record: the reference's loader drops it
    open(d / "module_connection_tracing_merged.bin", "wb").write(full[:-2])
    es = lst.HostES(str(d))
    n_cut = es.array("modules.nConnectedModules", np.uint16)
    es.close()
    assert np.count_nonzero(n_cut != n_ref) <= 1


def test_connection_map_with_too_many_connections(tmp_path):
    """More connected modules than a module-map row holds (80) is an error,
    not an overrun of the row."""
    d = _copy_geometry(tmp_path)
    det = struct.unpack_from("<I", open(d / "sensor_centroids.bin", "rb").read(), 0)[0]
    with open(d / "module_connection_tracing_merged.bin", "ab") as f:
        f.write(struct.pack("<II", det, 81) + struct.pack("<81I", *([det] * 81)))
    rc, msg = _load_host(d)
    assert rc < 0 and "more than 80 connected modules" in msg


def test_corrupt_pixel_map_detid(tmp_path):
    d = _copy_geometry(tmp_path)
    p = d / "pixelmap" / "pLS_map_layer1_subdet5.bin"
    data = bytearray(open(p, "rb").read())
    off = 0
    while True:  # the first record the charge-inclusive map uses (key 45000 + superbin) that lists a module
        key, n = struct.unpack_from("<II", data, off)
        if n > 0 and key >= 45000:
            break
        off += 8 + 4 * n
    struct.pack_into("<I", data, off + 8, 0xDEADBEEF)
    open(p, "wb").write(bytes(data))
    rc, msg = _load_host(d)
    assert rc < 0 and "unknown detId" in msg


def test_random_bytes_geometry_never_aborts(tmp_path):
    """Random bytes in every geometry file: an error status or a loaded
    setup, never a crash of the process."""
    d = _copy_geometry(tmp_path)
    rng = np.random.default_rng(7)
    for name in GEOMETRY_FILES:
        size = os.path.getsize(d / name)
        open(d / name, "wb").write(rng.integers(0, 256, size=min(size, 1 << 16), dtype=np.uint8).tobytes())
    rc, msg = _load_host(d)
    assert rc < 0 or rc == 0


@pytest.mark.parametrize("nbytes", [0, 4 * 2336, 4 * 2338])
def test_wrong_size_weights_file(tmp_path, nbytes):
    """A T5 DNN weight file of the wrong size fails in lst_es_load before the
    event setup touches the device."""
    w = tmp_path / "w.bin"
    open(w, "wb").write(b"\0" * nbytes)
    lib = lst.library()
    h = ctypes.c_void_p()
    rc = lib.lst_es_load(geometry.geometry_dir().encode(), str(w).encode(), 0, ctypes.byref(h))
    assert rc < 0
    assert "wrong size" in lib.lst_last_error().decode()
    assert not h.value


def test_missing_weights_file(tmp_path):
    lib = lst.library()
    h = ctypes.c_void_p()
    rc = lib.lst_es_load(geometry.geometry_dir().encode(), str(tmp_path / "none.bin").encode(), 0,
                         ctypes.byref(h))
    assert rc < 0 and "cannot open" in lib.lst_last_error().decode()


def test_null_arguments_are_errors():
    lib = lst.library()
    h = ctypes.c_void_p()
    assert lib.lst_es_load(None, None, 0, ctypes.byref(h)) < 0
    assert lib.lst_es_load_host(None, ctypes.byref(h)) < 0
    assert lib.lst_es_get_info(None, None) < 0
    assert lib.lst_event_create(None, 1, 1, None, ctypes.byref(h)) < 0


def test_es_load_ex_flags():
    """lst_es_load_ex rejects unknown flags before touching a file or the
    device; without a usable device the device build reports an error."""
    lib = lst.library()
    h = ctypes.c_void_p()
    assert lib.lst_es_load_ex(geometry.geometry_dir().encode(), None, 0, 0x80, ctypes.byref(h)) < 0
    assert "unknown flags" in lib.lst_last_error().decode()
    assert not h.value
    assert lib.lst_es_load_ex(None, None, 0, lst.ES_BUILD_ON_DEVICE, ctypes.byref(h)) < 0
