"""Python mirror of the reference's Event API over the C ABI of _lst_b200.so.

``Event`` keeps the member names of ``SDL::Event<Acc>`` (SDL/Event.h:31-205):
addHitToEvent, addPixelSegmentToEvent, createMiniDoublets,
createSegmentsWithModuleMap, createTriplets, createQuintuplets,
pixelLineSegmentCleaning, createPixelQuintuplets, createPixelTriplets,
createTrackCandidates, resetEvent and the getNumberOf* counters, plus
``field(name)`` for any object-store array (the reference's get* getters copy
subsets of the same arrays).  ``EventSet`` exposes the batched entry points:
N event slots in one device arena, packed-input upload and stage launches over
many slots at once.

There is no fallback: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from . import geometry

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "_lst_b200.so")
DNN_WEIGHTS = os.path.join(PKG_DIR, "data", "t5dnn_reference.bin")

STAGE_MINI_DOUBLETS = 1
STAGE_SEGMENTS = 2
STAGE_TRIPLETS = 3
STAGE_QUINTUPLETS = 4
STAGE_PLS_CLEANING = 5
STAGE_PIXEL_QUINTUPLETS = 6
STAGE_PIXEL_TRIPLETS = 7
STAGE_TRACK_CANDIDATES = 8
STAGE_NAMES = {
    "md": STAGE_MINI_DOUBLETS,
    "ls": STAGE_SEGMENTS,
    "t3": STAGE_TRIPLETS,
    "t5": STAGE_QUINTUPLETS,
    "pls_clean": STAGE_PLS_CLEANING,
    "pt5": STAGE_PIXEL_QUINTUPLETS,
    "pt3": STAGE_PIXEL_TRIPLETS,
    "tc": STAGE_TRACK_CANDIDATES,
}
STAGE_ORDER = ("md", "ls", "t3", "t5", "pls_clean", "pt5", "pt3", "tc")

T5_DNN = 0
T5_CUTS = 1

STATUS_UNKNOWN_DETID = 0x1
STATUS_UNKNOWN_ENDCAP_DETID = 0x2
STATUS_HIT_CAPACITY = 0x4
STATUS_PLS_TRUNCATED = 0x8
STATUS_TC_TRUNCATED = 0x10
STATUS_CAP_OVERFLOW = 0x20
STATUS_INVALID_INPUT = 0x40

STATUS_BITS = {
    0x1: "unknown detId",
    0x2: "unknown endcap detId",
    0x4: "hit capacity",
    0x8: "pLS truncated",
    0x10: "track candidates truncated",
    0x20: "occupancy cap overflow",
    0x40: "invalid input",
}

ES_BUILD_ON_DEVICE = 1  # LST_ES_BUILD_ON_DEVICE

# Exported symbols of include/lst_b200.h.
EXPORTS = (
    "lst_last_error",
    "lst_kernel_count",
    "lst_kernel_attributes",
    "lst_es_load",
    "lst_es_load_ex",
    "lst_es_free",
    "lst_es_load_host",
    "lst_es_host_array",
    "lst_es_get_info",
    "lst_es_set_t5dnn_weights",
    "lst_event_create",
    "lst_event_destroy",
    "lst_event_memory",
    "lst_event_sync",
    "lst_event_stream",
    "lst_event_set_t5_method",
    "lst_event_set_walk",
    "lst_event_reset",
    "lst_event_add_hits",
    "lst_event_add_pixel_segments",
    "lst_event_run_stage",
    "lst_event_create_mini_doublets",
    "lst_event_create_segments",
    "lst_event_create_triplets",
    "lst_event_create_quintuplets",
    "lst_event_pixel_line_segment_cleaning",
    "lst_event_create_pixel_quintuplets",
    "lst_event_create_pixel_triplets",
    "lst_event_create_track_candidates",
    "lst_event_get_counts",
    "lst_event_get_field",
    "lst_event_field_device_ptr",
    "lst_field_count",
    "lst_field_name",
    "lst_field_info",
    "lst_packed_size",
    "lst_batch_upload",
    "lst_batch_ingest",
    "lst_batch_run",
    "lst_batch_run_graph",
    "lst_batch_get_counts",
    "lst_batch_get_output",
    "lst_event_launches",
    "lst_event_set_profiling",
    "lst_event_get_profile",
    "lst_es_set_t5dnn_threshold",
    "lst_batch_t5_probe",
    "lst_t5dnn_forward",
    "lst_t5dnn_scratch_floats",
    "lst_t5dnn_backward",
    "lst_t5dnn_last_error",
    "lst_seed_packed_size",
    "lst_seed_pack",
    "lst_batch_upload_seeds",
    "lst_event_prepare_input",
    "lst_run",
    "lst_tune_kernel_count",
    "lst_tune_kernel_name",
    "lst_event_set_launch_shape",
    "lst_event_get_launch_shape",
    "lst_es_geometry_hash",
    "lst_autotune",
    "lst_autotune_load",
    "lst_batch_stage",
    "lst_batch_ingest_staged",
)


class LSTError(RuntimeError):
    pass


class Counts(ctypes.Structure):
    """lst_counts (include/lst_b200.h)."""

    _fields_ = [
        ("nHits", ctypes.c_uint32),
        ("nPixelSegments", ctypes.c_uint32),
        ("status", ctypes.c_uint32),
        ("nMiniDoublets", ctypes.c_uint32),
        ("nSegments", ctypes.c_uint32),
        ("nTriplets", ctypes.c_uint32),
        ("nQuintuplets", ctypes.c_uint32),
        ("nPixelTriplets", ctypes.c_uint32),
        ("nPixelQuintuplets", ctypes.c_uint32),
        ("nTrackCandidates", ctypes.c_uint32),
        ("nTrackCandidatesPT5", ctypes.c_uint32),
        ("nTrackCandidatesPT3", ctypes.c_uint32),
        ("nTrackCandidatesPLS", ctypes.c_uint32),
        ("nTrackCandidatesT5", ctypes.c_uint32),
        ("nPixelTripletsFound", ctypes.c_uint32),
        ("nPixelQuintupletsFound", ctypes.c_uint32),
        ("mdBarrel", ctypes.c_uint32 * 6),
        ("mdEndcap", ctypes.c_uint32 * 5),
        ("lsBarrel", ctypes.c_uint32 * 6),
        ("lsEndcap", ctypes.c_uint32 * 5),
        ("t3Barrel", ctypes.c_uint32 * 6),
        ("t3Endcap", ctypes.c_uint32 * 5),
        ("t5Barrel", ctypes.c_uint32 * 6),
        ("t5Endcap", ctypes.c_uint32 * 5),
        ("reserved", ctypes.c_uint32 * 4),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, ctypes.Array) else int(v)
        return out


class Output(ctypes.Structure):
    """lst_output (include/lst_b200.h)."""

    _fields_ = [
        ("hits", ctypes.c_void_p),
        ("hits_capacity", ctypes.c_size_t),
        ("len", ctypes.c_void_p),
        ("seedIdx", ctypes.c_void_p),
        ("type", ctypes.c_void_p),
        ("tc_capacity", ctypes.c_size_t),
        ("event_tc_offsets", ctypes.c_void_p),
        ("event_hit_offsets", ctypes.c_void_p),
    ]


class SeedInputC(ctypes.Structure):
    """lst_seed_input (include/lst_b200.h): the CMSSW inputs of LST::run."""

    _fields_ = [("n_seeds", ctypes.c_uint32)] + [
        (name, ctypes.c_void_p)
        for name in ("see_px", "see_py", "see_pz", "see_dxy", "see_dz", "see_ptErr", "see_etaErr",
                     "see_stateTrajGlbX", "see_stateTrajGlbY", "see_stateTrajGlbZ", "see_stateTrajGlbPx",
                     "see_stateTrajGlbPy", "see_stateTrajGlbPz", "see_q", "see_hitIdx_offsets", "see_hitIdx")
    ] + [("n_ph2", ctypes.c_uint32)] + [(name, ctypes.c_void_p) for name in ("ph2_detId", "ph2_x", "ph2_y", "ph2_z")]


def seed_struct(seeds) -> tuple[SeedInputC, list]:
    """A SeedInputC over a gen.SeedInput's arrays (plus the arrays it points
    into, which must stay alive while the struct is used)."""
    from .gen import SEED_FLOAT_FIELDS

    keep = []

    def p(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    c = SeedInputC()
    c.n_seeds = seeds.n_seeds
    for name in SEED_FLOAT_FIELDS:
        setattr(c, name, p(seeds.see[name], np.float32))
    c.see_q = p(seeds.see["see_q"], np.int32)
    c.see_hitIdx_offsets = p(seeds.hit_offsets, np.uint32)
    c.see_hitIdx = p(seeds.hit_idx, np.int32)
    c.n_ph2 = seeds.n_ph2
    c.ph2_detId = p(seeds.ph2_detId, np.uint32)
    c.ph2_x = p(seeds.ph2_x, np.float32)
    c.ph2_y = p(seeds.ph2_y, np.float32)
    c.ph2_z = p(seeds.ph2_z, np.float32)
    return c, keep


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("launches", ctypes.c_uint64), ("total_ms", ctypes.c_double)]


class EsInfo(ctypes.Structure):
    _fields_ = [
        ("nModules", ctypes.c_uint32),
        ("nLowerModules", ctypes.c_uint32),
        ("pixelModule", ctypes.c_uint32),
        ("nConnectedPixels", ctypes.c_uint32),
        ("nTotalMDs", ctypes.c_uint32),
        ("nTotalSegments", ctypes.c_uint32),
        ("maxTriplets", ctypes.c_uint32),
        ("maxQuintuplets", ctypes.c_uint32),
        ("ptCut", ctypes.c_float),
    ]


_lib = None
_lib_lock = threading.Lock()


def library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads _lst_b200.so (raises if it is missing)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise LSTError(f"CUDA library not built: {path} (run __graft_entry__.build())")
        lib = ctypes.CDLL(path)
        vp, u32, i32, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_size_t
        lib.lst_last_error.restype = ctypes.c_char_p
        lib.lst_kernel_count.argtypes = []
        lib.lst_kernel_attributes.argtypes = [i32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(i32),
                                              ctypes.POINTER(i32), ctypes.POINTER(sz), ctypes.POINTER(sz)]
        lib.lst_es_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i32, ctypes.POINTER(vp)]
        lib.lst_es_load_ex.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i32, u32, ctypes.POINTER(vp)]
        lib.lst_es_free.argtypes = [vp]
        lib.lst_es_free.restype = None
        lib.lst_es_get_info.argtypes = [vp, ctypes.POINTER(EsInfo)]
        lib.lst_es_load_host.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        lib.lst_es_host_array.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(vp), ctypes.POINTER(sz), ctypes.POINTER(sz)]
        lib.lst_es_set_t5dnn_weights.argtypes = [vp, vp, sz]
        lib.lst_event_create.argtypes = [vp, i32, u32, vp, ctypes.POINTER(vp)]
        lib.lst_event_destroy.argtypes = [vp]
        lib.lst_event_destroy.restype = None
        lib.lst_event_memory.argtypes = [vp, ctypes.POINTER(sz)]
        lib.lst_event_sync.argtypes = [vp]
        lib.lst_event_stream.argtypes = [vp]
        lib.lst_event_stream.restype = vp
        lib.lst_event_set_t5_method.argtypes = [vp, i32]
        lib.lst_event_set_walk.argtypes = [vp, i32]
        lib.lst_event_reset.argtypes = [vp, i32]
        lib.lst_event_add_hits.argtypes = [vp, i32, u32] + [vp] * 5
        lib.lst_event_add_pixel_segments.argtypes = [vp, i32, u32] + [vp] * 18
        lib.lst_event_run_stage.argtypes = [vp, i32, i32]
        lib.lst_event_get_counts.argtypes = [vp, i32, ctypes.POINTER(Counts)]
        lib.lst_event_get_field.argtypes = [vp, i32, ctypes.c_char_p, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz)]
        lib.lst_event_field_device_ptr.argtypes = [
            vp, i32, ctypes.c_char_p, ctypes.POINTER(vp), ctypes.POINTER(sz), ctypes.POINTER(sz)]
        lib.lst_field_count.argtypes = []
        lib.lst_field_name.argtypes = [i32]
        lib.lst_field_name.restype = ctypes.c_char_p
        lib.lst_field_info.argtypes = [i32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(sz), ctypes.POINTER(ctypes.c_char)]
        lib.lst_packed_size.argtypes = [u32, u32]
        lib.lst_packed_size.restype = sz
        lib.lst_batch_upload.argtypes = [vp, i32, i32, vp, sz, vp]
        lib.lst_batch_ingest.argtypes = [vp, i32, i32]
        lib.lst_batch_run.argtypes = [vp, i32, i32, i32, i32]
        lib.lst_batch_run_graph.argtypes = [vp, i32, i32, i32, i32]
        lib.lst_batch_get_counts.argtypes = [vp, i32, i32, ctypes.POINTER(Counts)]
        lib.lst_batch_get_output.argtypes = [vp, i32, i32, ctypes.POINTER(Output)]
        lib.lst_event_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
        lib.lst_event_set_profiling.argtypes = [vp, i32]
        lib.lst_event_get_profile.argtypes = [vp, ctypes.POINTER(KernelTime), i32, ctypes.POINTER(i32)]
        lib.lst_es_set_t5dnn_threshold.argtypes = [vp, ctypes.c_float]
        lib.lst_batch_t5_probe.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp, vp, u32, ctypes.POINTER(u32)]
        lib.lst_t5dnn_forward.argtypes = [vp, vp, i32, vp, vp, vp, vp]
        lib.lst_t5dnn_scratch_floats.argtypes = [i32]
        lib.lst_t5dnn_scratch_floats.restype = sz
        lib.lst_t5dnn_backward.argtypes = [vp, vp, vp, vp, vp, i32, vp, vp, vp]
        lib.lst_t5dnn_last_error.restype = ctypes.c_char_p
        lib.lst_seed_packed_size.argtypes = [u32, u32, u32]
        lib.lst_seed_packed_size.restype = sz
        lib.lst_seed_pack.argtypes = [ctypes.POINTER(SeedInputC), vp, sz]
        lib.lst_batch_upload_seeds.argtypes = [vp, i32, i32, vp, sz, vp]
        lib.lst_event_prepare_input.argtypes = [vp, i32, ctypes.POINTER(SeedInputC)]
        lib.lst_run.argtypes = [vp, i32, ctypes.POINTER(SeedInputC), ctypes.POINTER(Output)]
        lib.lst_tune_kernel_count.argtypes = []
        lib.lst_tune_kernel_name.argtypes = [i32]
        lib.lst_tune_kernel_name.restype = ctypes.c_char_p
        lib.lst_event_set_launch_shape.argtypes = [vp, i32, i32, i32]
        lib.lst_event_get_launch_shape.argtypes = [vp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        lib.lst_es_geometry_hash.argtypes = [vp]
        lib.lst_es_geometry_hash.restype = ctypes.c_uint64
        lib.lst_autotune.argtypes = [vp, i32, i32, ctypes.c_char_p]
        lib.lst_autotune_load.argtypes = [vp, i32, ctypes.c_char_p]
        lib.lst_batch_stage.argtypes = [vp, i32, i32, vp, sz, vp, i32]
        lib.lst_batch_ingest_staged.argtypes = [vp]
        _lib = lib
        return lib


def _check(rc: int, what: str) -> int:
    if rc < 0:
        msg = library().lst_last_error().decode(errors="replace")
        raise LSTError(f"{what}: {msg}")
    return rc


def kernel_attributes() -> list[dict]:
    """Registers, maximum block size and memory of every kernel (needs a GPU)."""
    lib = library()
    out = []
    for i in range(lib.lst_kernel_count()):
        name, regs, mt = ctypes.c_char_p(), ctypes.c_int(), ctypes.c_int()
        local, smem = ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib.lst_kernel_attributes(i, ctypes.byref(name), ctypes.byref(regs), ctypes.byref(mt),
                                         ctypes.byref(local), ctypes.byref(smem)), "lst_kernel_attributes")
        out.append({"name": name.value.decode(), "regs": regs.value, "max_threads": mt.value,
                    "local_bytes": local.value, "smem_bytes": smem.value})
    return out


def field_names() -> list[str]:
    lib = library()
    return [lib.lst_field_name(i).decode() for i in range(lib.lst_field_count())]


_FIELD_DTYPES: dict | None = None


def field_dtypes() -> dict:
    """numpy dtype of every store field, from the library's field table."""
    global _FIELD_DTYPES
    if _FIELD_DTYPES is None:
        lib = library()
        out = {}
        for i in range(lib.lst_field_count()):
            name, esz, kind = ctypes.c_char_p(), ctypes.c_size_t(), ctypes.c_char()
            _check(lib.lst_field_info(i, ctypes.byref(name), ctypes.byref(esz), ctypes.byref(kind)), "lst_field_info")
            out[name.value.decode()] = np.dtype(f"{kind.value.decode()}{esz.value}")
        _FIELD_DTYPES = out
    return _FIELD_DTYPES


class ES:
    """Event setup on one device (SDL::LSTESDeviceData)."""

    def __init__(self, device: int = 0, weights: str | None = DNN_WEIGHTS, geometry_dir: str | None = None,
                 build_on_device: bool = False):
        """build_on_device: build the event setup with kernels on `device`
        (LST_ES_BUILD_ON_DEVICE) instead of on the host; same arrays."""
        lib = library()
        gdir = geometry_dir or geometry.geometry_dir()
        h = ctypes.c_void_p()
        _check(lib.lst_es_load_ex(gdir.encode(), weights.encode() if weights else None, device,
                                  ES_BUILD_ON_DEVICE if build_on_device else 0, ctypes.byref(h)), "lst_es_load")
        self._h = h
        self.device = device
        info = EsInfo()
        _check(lib.lst_es_get_info(h, ctypes.byref(info)), "lst_es_get_info")
        self.info = {n: (float if n == "ptCut" else int)(getattr(info, n)) for n, _ in EsInfo._fields_}

    @property
    def handle(self):
        return self._h

    def array(self, name: str, dtype) -> np.ndarray:
        """The host copy of an event-setup array (lst_es_host_array)."""
        return _es_array(self._h, name, dtype)

    def geometry_hash(self) -> int:
        return int(library().lst_es_geometry_hash(self._h))

    def set_t5dnn_threshold(self, wp: float):
        _check(library().lst_es_set_t5dnn_threshold(self._h, float(wp)), "lst_es_set_t5dnn_threshold")

    def set_t5dnn_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32).ravel()
        _check(library().lst_es_set_t5dnn_weights(self._h, w.ctypes.data, w.size), "lst_es_set_t5dnn_weights")

    def close(self):
        """Frees the event setup; event sets still using it keep it alive
        until they are closed."""
        self._closing = True
        if self._h and not getattr(self, "_users", 0):
            library().lst_es_free(self._h)
            self._h = None

    def _retain(self):
        self._users = getattr(self, "_users", 0) + 1

    def _release(self):
        self._users -= 1
        if self._users == 0 and getattr(self, "_closing", False):
            self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _es_array(h, name: str, dtype) -> np.ndarray:
    """Copy of the event-setup array `name` of handle h (lst_es_host_array)."""
    lib = library()
    p, n, esz = ctypes.c_void_p(), ctypes.c_size_t(), ctypes.c_size_t()
    _check(lib.lst_es_host_array(h, name.encode(), ctypes.byref(p), ctypes.byref(n), ctypes.byref(esz)),
           f"es array {name}")
    dt = np.dtype(dtype)
    if dt.itemsize != esz.value:
        raise LSTError(f"{name}: element size {esz.value}, asked for {dt}")
    if n.value == 0:
        return np.zeros(0, dt)
    buf = (ctypes.c_char * (n.value * esz.value)).from_address(p.value)
    return np.frombuffer(buf, dtype=dt).copy()


class HostES:
    """Event setup loaded on the host only (lst_es_load_host), for inspection."""

    def __init__(self, geometry_dir: str | None = None):
        lib = library()
        h = ctypes.c_void_p()
        gdir = geometry_dir or geometry.geometry_dir()
        _check(lib.lst_es_load_host(gdir.encode(), ctypes.byref(h)), "lst_es_load_host")
        self._h = h
        info = EsInfo()
        _check(lib.lst_es_get_info(h, ctypes.byref(info)), "lst_es_get_info")
        self.info = {n: (float if n == "ptCut" else int)(getattr(info, n)) for n, _ in EsInfo._fields_}

    def array(self, name: str, dtype) -> np.ndarray:
        return _es_array(self._h, name, dtype)

    def close(self):
        if self._h:
            library().lst_es_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EventSet:
    """N event slots on one stream (batched entry points)."""

    def __init__(self, es: ES, n_slots: int = 1, max_hits: int = 1 << 20, stream: int | None = None):
        lib = library()
        h = ctypes.c_void_p()
        _check(lib.lst_event_create(es.handle, n_slots, max_hits, stream, ctypes.byref(h)), "lst_event_create")
        self._h = h
        self.es = es
        es._retain()
        self.n_slots = n_slots
        self.max_hits = max_hits

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            library().lst_event_destroy(self._h)
            self._h = None
            self.es._release()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def memory_bytes(self) -> int:
        n = ctypes.c_size_t()
        _check(library().lst_event_memory(self._h, ctypes.byref(n)), "lst_event_memory")
        return n.value

    def stream(self) -> int:
        return library().lst_event_stream(self._h)

    def sync(self):
        _check(library().lst_event_sync(self._h), "lst_event_sync")

    def set_walk(self, on: bool):
        _check(library().lst_event_set_walk(self._h, int(bool(on))), "lst_event_set_walk")

    def set_t5_method(self, method: int):
        _check(library().lst_event_set_t5_method(self._h, method), "lst_event_set_t5_method")

    # -- per-slot inputs
    def add_hits(self, slot, x, y, z, detId, idxInNtuple) -> int:
        keep = [np.ascontiguousarray(a, dt) for a, dt in
                ((x, np.float32), (y, np.float32), (z, np.float32), (detId, np.uint32), (idxInNtuple, np.uint32))]
        rc = library().lst_event_add_hits(self._h, slot, keep[0].size, *[k.ctypes.data for k in keep])
        _check(rc, "lst_event_add_hits")
        self.sync()
        return rc

    def add_pixel_segments(self, slot, pls: dict) -> int:
        from .gen import PLS_FIELDS

        keep = [np.ascontiguousarray(pls[name], dt) for name, dt in PLS_FIELDS]
        rc = library().lst_event_add_pixel_segments(self._h, slot, keep[5].size, *[k.ctypes.data for k in keep])
        _check(rc, "lst_event_add_pixel_segments")
        self.sync()
        return rc

    def add_inputs(self, slot, inp) -> int:
        rc = self.add_hits(slot, inp.x, inp.y, inp.z, inp.detId, inp.idxInNtuple)
        if rc > 0:
            return rc
        return self.add_pixel_segments(slot, inp.pls)

    def run_stage(self, slot: int, stage) -> int:
        st = STAGE_NAMES[stage] if isinstance(stage, str) else int(stage)
        return _check(library().lst_event_run_stage(self._h, slot, st), "lst_event_run_stage")

    def reset(self, slot: int):
        _check(library().lst_event_reset(self._h, slot), "lst_event_reset")

    def counts(self, slot: int) -> dict:
        c = Counts()
        _check(library().lst_event_get_counts(self._h, slot, ctypes.byref(c)), "lst_event_get_counts")
        return c.as_dict()

    def field(self, slot: int, name: str, count: int | None = None) -> np.ndarray:
        lib = library()
        n, esz = ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib.lst_event_get_field(self._h, slot, name.encode(), None, 0, ctypes.byref(n), ctypes.byref(esz)),
               f"field {name}")
        k = n.value if count is None else min(int(count), n.value)
        dt = field_dtypes()[name]
        out = np.empty(k, dtype=dt)
        if k:
            _check(lib.lst_event_get_field(self._h, slot, name.encode(), out.ctypes.data, k, None, None),
                   f"field {name}")
        return out

    # -- batched
    def upload_packed(self, first: int, blobs: np.ndarray, offsets: np.ndarray):
        offsets = np.ascontiguousarray(offsets, np.uint64)
        _check(library().lst_batch_upload(self._h, first, offsets.size, blobs.ctypes.data, blobs.nbytes,
                                          offsets.ctypes.data), "lst_batch_upload")

    def upload_seeds(self, first: int, blobs: np.ndarray, offsets: np.ndarray):
        """lst_batch_upload_seeds: packed CMSSW seed events (pack_seed_events)."""
        offsets = np.ascontiguousarray(offsets, np.uint64)
        _check(library().lst_batch_upload_seeds(self._h, first, offsets.size, blobs.ctypes.data, blobs.nbytes,
                                                offsets.ctypes.data), "lst_batch_upload_seeds")

    def prepare_input(self, slot: int, seeds):
        """lst_event_prepare_input: LST::prepareInput + addHitToEvent + addPixelSegmentToEvent."""
        c, keep = seed_struct(seeds)
        _check(library().lst_event_prepare_input(self._h, slot, ctypes.byref(c)), "lst_event_prepare_input")

    # -- launch shapes and the autotuner
    def launch_shapes(self) -> dict:
        """{kernel: (warps per block, blocks per SM)} of the tunable kernels."""
        lib = library()
        out = {}
        for k in range(lib.lst_tune_kernel_count()):
            w, p = ctypes.c_int(), ctypes.c_int()
            _check(lib.lst_event_get_launch_shape(self._h, k, ctypes.byref(w), ctypes.byref(p)),
                   "lst_event_get_launch_shape")
            out[lib.lst_tune_kernel_name(k).decode()] = (w.value, p.value)
        return out

    def set_launch_shape(self, kernel: str, warps_per_block: int, blocks_per_sm: int):
        lib = library()
        names = [lib.lst_tune_kernel_name(k).decode() for k in range(lib.lst_tune_kernel_count())]
        _check(lib.lst_event_set_launch_shape(self._h, names.index(kernel), warps_per_block, blocks_per_sm),
               "lst_event_set_launch_shape")

    def autotune(self, first: int, count: int, cache_path: str | None = None):
        """lst_autotune on the resident inputs of slots [first, first + count)."""
        _check(library().lst_autotune(self._h, first, count, cache_path.encode() if cache_path else None),
               "lst_autotune")

    def autotune_load(self, count: int, cache_path: str) -> bool:
        return bool(_check(library().lst_autotune_load(self._h, count, cache_path.encode()), "lst_autotune_load"))

    def stage(self, first: int, blobs: np.ndarray, offsets: np.ndarray, seed_layout: bool = False):
        """lst_batch_stage: start copying packed events (pinned buffer) on the copy stream."""
        offsets = np.ascontiguousarray(offsets, np.uint64)
        self._staged_offsets = offsets  # the offsets are read when the call returns; keep them alive anyway
        _check(library().lst_batch_stage(self._h, first, offsets.size, blobs.ctypes.data, blobs.nbytes,
                                         offsets.ctypes.data, int(bool(seed_layout))), "lst_batch_stage")

    def ingest_staged(self):
        _check(library().lst_batch_ingest_staged(self._h), "lst_batch_ingest_staged")

    def ingest(self, first: int, count: int):
        _check(library().lst_batch_ingest(self._h, first, count), "lst_batch_ingest")

    def run(self, first: int, count: int, first_stage: int = STAGE_MINI_DOUBLETS,
            last_stage: int = STAGE_TRACK_CANDIDATES):
        _check(library().lst_batch_run(self._h, first, count, first_stage, last_stage), "lst_batch_run")

    def output(self, first: int, count: int, tc_capacity: int = 31000, hits_capacity: int = 31000 * 14):
        """LST::getOutput for slots [first, first + count): (hits, len, seedIdx, type, tc_offsets, hit_offsets)."""
        hits = np.empty(hits_capacity, np.uint32)
        ln = np.empty(tc_capacity, np.uint32)
        seed = np.empty(tc_capacity, np.int32)
        typ = np.empty(tc_capacity, np.int16)
        tco = np.empty(count + 1, np.uint64)
        hco = np.empty(count + 1, np.uint64)
        o = Output(hits.ctypes.data, hits.size, ln.ctypes.data, seed.ctypes.data, typ.ctypes.data, ln.size,
                   tco.ctypes.data, hco.ctypes.data)
        _check(library().lst_batch_get_output(self._h, first, count, ctypes.byref(o)), "lst_batch_get_output")
        ntc, nh = int(tco[-1]), int(hco[-1])
        return hits[:nh], ln[:ntc], seed[:ntc], typ[:ntc], tco, hco

    def launches(self) -> int:
        n = ctypes.c_uint64()
        _check(library().lst_event_launches(self._h, ctypes.byref(n)), "lst_event_launches")
        return n.value

    def set_profiling(self, on: bool):
        _check(library().lst_event_set_profiling(self._h, int(bool(on))), "lst_event_set_profiling")

    def profile(self) -> dict:
        """{kernel: (launches, total ms)} since profiling was switched on or last read."""
        arr = (KernelTime * 128)()
        n = ctypes.c_int()
        _check(library().lst_event_get_profile(self._h, arr, 128, ctypes.byref(n)), "lst_event_get_profile")
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(min(n.value, 128))}

    def run_graph(self, first: int, count: int, first_stage: int = STAGE_MINI_DOUBLETS,
                  last_stage: int = STAGE_TRACK_CANDIDATES):
        _check(library().lst_batch_run_graph(self._h, first, count, first_stage, last_stage), "lst_batch_run_graph")

    def batch_counts(self, first: int, count: int) -> list[dict]:
        arr = (Counts * count)()
        _check(library().lst_batch_get_counts(self._h, first, count, arr), "lst_batch_get_counts")
        return [c.as_dict() for c in arr]


def packed_size(n_hits: int, n_pls: int) -> int:
    return int(library().lst_packed_size(n_hits, n_pls))


def pack_event(inp, out: np.ndarray | None = None, offset: int = 0) -> np.ndarray:
    """Packs one event's inputs in the lst_batch_upload layout."""
    from .gen import PLS_FIELDS

    nh, npls = inp.n_hits, inp.n_pls
    size = packed_size(nh, npls)
    if out is None:
        out = np.zeros(size, np.uint8)
        offset = 0
    buf = out[offset:offset + size]
    hdr = np.array([nh, npls, 0, 0], np.uint32)
    parts = [hdr.view(np.uint8)]
    for a, dt in ((inp.x, np.float32), (inp.y, np.float32), (inp.z, np.float32), (inp.detId, np.uint32),
                  (inp.idxInNtuple, np.uint32)):
        parts.append(np.ascontiguousarray(a, dt).view(np.uint8))
    for name, dt in PLS_FIELDS:
        parts.append(np.ascontiguousarray(inp.pls[name], dt).view(np.uint8))
    flat = np.concatenate(parts)
    buf[:flat.size] = flat
    buf[flat.size:] = 0
    return out


def seed_packed_size(n_ph2: int, n_seeds: int, n_seed_hits: int) -> int:
    return int(library().lst_seed_packed_size(n_ph2, n_seeds, n_seed_hits))


def pack_seed_events(seed_inputs) -> tuple[np.ndarray, np.ndarray]:
    """Packs several events' CMSSW seeds (gen.SeedInput) back to back with
    lst_seed_pack; returns (blob bytes, offsets) for EventSet.upload_seeds."""
    lib = library()
    sizes = [seed_packed_size(s.n_ph2, s.n_seeds, int(s.hit_offsets[-1]) if s.n_seeds else 0) for s in seed_inputs]
    offsets = np.zeros(len(seed_inputs), np.uint64)
    if seed_inputs:
        offsets[1:] = np.cumsum(sizes[:-1])
    blob = np.zeros(int(sum(sizes)), np.uint8)
    for s, off, size in zip(seed_inputs, offsets, sizes):
        c, keep = seed_struct(s)
        _check(lib.lst_seed_pack(ctypes.byref(c), blob.ctypes.data + int(off), size), "lst_seed_pack")
    return blob, offsets


def pack_events(inputs) -> tuple[np.ndarray, np.ndarray]:
    """Packs several events back to back; returns (blob bytes, offsets)."""
    sizes = [packed_size(i.n_hits, i.n_pls) for i in inputs]
    offsets = np.zeros(len(inputs), np.uint64)
    if inputs:
        offsets[1:] = np.cumsum(sizes[:-1])
    blob = np.zeros(int(sum(sizes)), np.uint8)
    for inp, off in zip(inputs, offsets):
        pack_event(inp, blob, int(off))
    return blob, offsets


class Event:
    """One event with the member names of SDL::Event<Acc> (SDL/Event.h:31-205)."""

    def __init__(self, es: ES, max_hits: int = 1 << 20, event_set: EventSet | None = None, slot: int = 0):
        self._set = event_set or EventSet(es, 1, max_hits)
        self._slot = slot

    @property
    def event_set(self) -> EventSet:
        return self._set

    def resetEvent(self):
        self._set.reset(self._slot)

    def addHitToEvent(self, x, y, z, detId, idxInNtuple):
        return self._set.add_hits(self._slot, x, y, z, detId, idxInNtuple)

    def addPixelSegmentToEvent(self, hitIndices0, hitIndices1, hitIndices2, hitIndices3, dPhiChange, ptIn, ptErr,
                               px, py, pz, eta, etaErr, phi, charge, seedIdx, superbin, pixelType, isQuad):
        from .gen import PLS_FIELDS

        vals = (hitIndices0, hitIndices1, hitIndices2, hitIndices3, dPhiChange, ptIn, ptErr, px, py, pz, eta, etaErr,
                phi, charge, seedIdx, superbin, pixelType, isQuad)
        return self._set.add_pixel_segments(self._slot, {n: v for (n, _), v in zip(PLS_FIELDS, vals)})

    def createMiniDoublets(self):
        return self._set.run_stage(self._slot, STAGE_MINI_DOUBLETS)

    def createSegmentsWithModuleMap(self):
        return self._set.run_stage(self._slot, STAGE_SEGMENTS)

    def createTriplets(self):
        return self._set.run_stage(self._slot, STAGE_TRIPLETS)

    def createQuintuplets(self):
        return self._set.run_stage(self._slot, STAGE_QUINTUPLETS)

    def pixelLineSegmentCleaning(self):
        return self._set.run_stage(self._slot, STAGE_PLS_CLEANING)

    def createPixelQuintuplets(self):
        return self._set.run_stage(self._slot, STAGE_PIXEL_QUINTUPLETS)

    def createPixelTriplets(self):
        return self._set.run_stage(self._slot, STAGE_PIXEL_TRIPLETS)

    def createTrackCandidates(self):
        return self._set.run_stage(self._slot, STAGE_TRACK_CANDIDATES)

    def counts(self) -> dict:
        return self._set.counts(self._slot)

    def field(self, name: str, count: int | None = None) -> np.ndarray:
        return self._set.field(self._slot, name, count)

    # getNumberOf* (SDL/Event.cc:1263-1487)
    def getNumberOfMiniDoublets(self):
        return self.counts()["nMiniDoublets"]

    def getNumberOfSegments(self):
        return self.counts()["nSegments"]

    def getNumberOfTriplets(self):
        return self.counts()["nTriplets"]

    def getNumberOfQuintuplets(self):
        return self.counts()["nQuintuplets"]

    def getNumberOfPixelTriplets(self):
        return self.counts()["nPixelTriplets"]

    def getNumberOfPixelQuintuplets(self):
        return self.counts()["nPixelQuintuplets"]

    def getNumberOfTrackCandidates(self):
        return self.counts()["nTrackCandidates"]

    def getNumberOfPT5TrackCandidates(self):
        return self.counts()["nTrackCandidatesPT5"]

    def getNumberOfPT3TrackCandidates(self):
        return self.counts()["nTrackCandidatesPT3"]

    def getNumberOfPLSTrackCandidates(self):
        return self.counts()["nTrackCandidatesPLS"]

    def getNumberOfPixelTrackCandidates(self):
        c = self.counts()
        return c["nTrackCandidates"] - c["nTrackCandidatesT5"]

    def getNumberOfT5TrackCandidates(self):
        return self.counts()["nTrackCandidatesT5"]

    def getOutput(self):
        """LST::getOutput: (hits per candidate, len, seedIdx, trackCandidateType)."""
        hits, ln, seed, typ, _, _ = self._set.output(self._slot, 1)
        bounds = np.concatenate(([0], np.cumsum(ln.astype(np.int64))))
        return [hits[bounds[i]:bounds[i + 1]].tolist() for i in range(ln.size)], ln, seed, typ

    def run(self, inp, upto: str = "tc"):
        """addHitToEvent + addPixelSegmentToEvent + stages in LST::run order."""
        self._set.add_inputs(self._slot, inp)
        for st in STAGE_ORDER:
            self._set.run_stage(self._slot, st)
            if st == upto:
                break


class LST:
    """SDL::LST<Acc> (SDL/LST.h:25-111): ``run`` takes the CMSSW seed and hit
    vectors, converts them (LST::prepareInput), runs the chain and keeps the
    output that ``hits()``, ``len()``, ``seedIdx()`` and
    ``trackCandidateType()`` return."""

    def __init__(self, es: ES, max_hits: int = 1 << 20, event_set: EventSet | None = None, slot: int = 0):
        self._set = event_set or EventSet(es, 1, max_hits)
        self._slot = slot
        self._out = ([], np.zeros(0, np.uint32), np.zeros(0, np.int32), np.zeros(0, np.int16))

    @property
    def event_set(self) -> EventSet:
        return self._set

    def run(self, see_px, see_py, see_pz, see_dxy, see_dz, see_ptErr, see_etaErr, see_stateTrajGlbX,
            see_stateTrajGlbY, see_stateTrajGlbZ, see_stateTrajGlbPx, see_stateTrajGlbPy, see_stateTrajGlbPz, see_q,
            see_hitIdx, ph2_detId, ph2_x, ph2_y, ph2_z, tc_capacity: int = 31000):
        """LST::run with the reference's argument list; see_hitIdx is a list
        of per-seed index lists."""
        from .gen import SEED_FLOAT_FIELDS, SeedInput

        vals = (see_px, see_py, see_pz, see_dxy, see_dz, see_ptErr, see_etaErr, see_stateTrajGlbX, see_stateTrajGlbY,
                see_stateTrajGlbZ, see_stateTrajGlbPx, see_stateTrajGlbPy, see_stateTrajGlbPz)
        see = {k: np.asarray(v, np.float32) for k, v in zip(SEED_FLOAT_FIELDS, vals)}
        see["see_q"] = np.asarray(see_q, np.int32)
        lens = np.array([len(h) for h in see_hitIdx], np.int64)
        off = np.zeros(len(lens) + 1, np.uint32)
        off[1:] = np.cumsum(lens)
        flat = np.concatenate([np.asarray(h, np.int32) for h in see_hitIdx]) if len(lens) else np.zeros(0, np.int32)
        seeds = SeedInput(see, off, flat, np.asarray(ph2_detId, np.uint32), np.asarray(ph2_x, np.float32),
                          np.asarray(ph2_y, np.float32), np.asarray(ph2_z, np.float32))
        return self.run_seeds(seeds, tc_capacity)

    def run_seeds(self, seeds, tc_capacity: int = 31000):
        """LST::run on a gen.SeedInput (flattened see_hitIdx)."""
        c, keep = seed_struct(seeds)
        hits = np.empty(tc_capacity * 14, np.uint32)
        ln = np.empty(tc_capacity, np.uint32)
        seed = np.empty(tc_capacity, np.int32)
        typ = np.empty(tc_capacity, np.int16)
        tco = np.empty(2, np.uint64)
        hco = np.empty(2, np.uint64)
        o = Output(hits.ctypes.data, hits.size, ln.ctypes.data, seed.ctypes.data, typ.ctypes.data, ln.size,
                   tco.ctypes.data, hco.ctypes.data)
        _check(library().lst_run(self._set.handle, self._slot, ctypes.byref(c), ctypes.byref(o)), "lst_run")
        ntc, nh = int(tco[-1]), int(hco[-1])
        ln = ln[:ntc].copy()
        bounds = np.concatenate(([0], np.cumsum(ln.astype(np.int64))))
        self._flat = hits[:nh].copy()
        self._out = ([self._flat[bounds[i]:bounds[i + 1]].tolist() for i in range(ntc)], ln, seed[:ntc].copy(),
                     typ[:ntc].copy())
        return self

    def hits(self) -> list:
        return self._out[0]

    def len(self) -> np.ndarray:
        return self._out[1]

    def seedIdx(self) -> np.ndarray:
        return self._out[2]

    def trackCandidateType(self) -> np.ndarray:
        return self._out[3]

    def flat_hits(self) -> np.ndarray:
        """hits() concatenated over the candidates."""
        return getattr(self, "_flat", np.zeros(0, np.uint32))
