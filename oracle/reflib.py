"""Python handle on the LST reference CPU backend built in oracle/_ref/.

Test infrastructure only (parity checks, golden fixtures, the reference arm of
bench.py).  ``RefLST(variant)`` loads ``oracle/_ref/liblstref_<variant>.so``
(see oracle/ref/Makefile for the variants), ``run_event`` feeds one event
through ``SDL::Event`` in the order bin/sdl.cc:451-458 calls the stages, and
``field`` returns any internal array of the event as a numpy view.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

STAGES = {
    "md": 1,
    "ls": 2,
    "t3": 3,
    "t5": 4,
    "pls_clean": 5,
    "pt5": 6,
    "pt3": 7,
    "tc": 8,
}
STAGE_ORDER = ("md", "ls", "t3", "t5", "pls_clean", "pt5", "pt3", "tc")

_INT_DTYPES = {1: np.int8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def library_path(variant: str = "cr") -> str:
    return os.path.join(REF_DIR, f"liblstref_{variant}.so")


def available(variant: str = "cr") -> bool:
    return os.path.exists(library_path(variant))


class RefLST:
    """One loaded reference library plus its event setup."""

    def __init__(self, variant: str = "cr", es_base: str | None = None):
        from tracklooper_b200 import geometry

        path = library_path(variant)
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference library not built: {path}")
        lib = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        lib.lstref_es_load.restype = vp
        lib.lstref_es_load.argtypes = [ctypes.c_char_p]
        lib.lstref_es_free.argtypes = [vp]
        lib.lstref_es_counts.restype = ctypes.c_uint
        lib.lstref_es_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_uint)]
        lib.lstref_event_create.restype = vp
        lib.lstref_event_create.argtypes = [vp]
        lib.lstref_event_destroy.argtypes = [vp]
        lib.lstref_event_reset.argtypes = [vp]
        lib.lstref_event_add_hits.argtypes = [vp, ctypes.c_uint] + [vp] * 5
        lib.lstref_event_add_pixel_segments.argtypes = [vp, ctypes.c_uint] + [vp] * 18
        lib.lstref_event_run_stage.restype = ctypes.c_int
        lib.lstref_event_run_stage.argtypes = [vp, ctypes.c_int]
        lib.lstref_event_field.restype = vp
        lib.lstref_event_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
        seed_args = [ctypes.c_uint, ctypes.POINTER(vp), vp, vp, vp, ctypes.c_uint, vp, vp, vp, vp]
        lib.lstref_lst_create.restype = vp
        lib.lstref_lst_destroy.argtypes = [vp]
        lib.lstref_lst_prepare.argtypes = [vp] + seed_args
        lib.lstref_lst_run.argtypes = [vp, vp] + seed_args
        lib.lstref_lst_array.restype = vp
        lib.lstref_lst_array.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
        self.lib = lib
        geometry.geometry_dir()
        self.es = lib.lstref_es_load((es_base or geometry.ES_BASE).encode())
        if not self.es:
            raise RuntimeError("reference failed to load the event setup")
        nm, nl = ctypes.c_uint(), ctypes.c_uint()
        self.n_pixels = lib.lstref_es_counts(self.es, ctypes.byref(nm), ctypes.byref(nl))
        self.n_modules, self.n_lower = nm.value, nl.value
        self.ev = lib.lstref_event_create(self.es)

    def fork(self) -> "RefLST":
        """Another event on the same event setup (for one event per thread)."""
        other = RefLST.__new__(RefLST)
        other.lib = self.lib
        other.es = self.es
        other._owns_es = False
        other.n_pixels, other.n_modules, other.n_lower = self.n_pixels, self.n_modules, self.n_lower
        other.ev = self.lib.lstref_event_create(self.es)
        return other

    def close(self):
        if self.ev:
            self.lib.lstref_event_destroy(self.ev)
            self.ev = None
        if self.es and getattr(self, "_owns_es", True):
            self.lib.lstref_es_free(self.es)
        self.es = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ event
    def reset(self):
        self.lib.lstref_event_reset(self.ev)

    def add_inputs(self, inp):
        keep = []

        def p(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        self.lib.lstref_event_add_hits(
            self.ev,
            inp.n_hits,
            p(inp.x, np.float32),
            p(inp.y, np.float32),
            p(inp.z, np.float32),
            p(inp.detId, np.uint32),
            p(inp.idxInNtuple, np.uint32),
        )
        from tracklooper_b200.gen import PLS_FIELDS

        self.lib.lstref_event_add_pixel_segments(
            self.ev, inp.n_pls, *[p(inp.pls[name], dt) for name, dt in PLS_FIELDS]
        )

    def run_stage(self, stage: str):
        rc = self.lib.lstref_event_run_stage(self.ev, STAGES[stage])
        if rc != 0:
            raise RuntimeError(f"unknown stage {stage}")

    def run_event(self, inp, upto: str = "tc"):
        self.reset()
        self.add_inputs(inp)
        for st in STAGE_ORDER:
            self.run_stage(st)
            if st == upto:
                break

    def field(self, name: str, dtype=None, copy: bool = True) -> np.ndarray | None:
        n, sz = ctypes.c_longlong(), ctypes.c_int()
        ptr = self.lib.lstref_event_field(self.ev, name.encode(), ctypes.byref(n), ctypes.byref(sz))
        if not ptr:
            return None
        if dtype is None:
            dtype = _INT_DTYPES[sz.value]
        dtype = np.dtype(dtype)
        count = n.value * sz.value // dtype.itemsize
        buf = (ctypes.c_char * (n.value * sz.value)).from_address(ptr)
        arr = np.frombuffer(buf, dtype=dtype, count=count)
        return arr.copy() if copy else arr

    # ------------------------------------------------------------- SDL::LST
    def _seed_args(self, seeds, keep):
        from tracklooper_b200.gen import SEED_FLOAT_FIELDS

        def p(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        f13 = (ctypes.c_void_p * 13)(*[p(seeds.see[k], np.float32) for k in SEED_FLOAT_FIELDS])
        keep.append(f13)
        return [
            seeds.n_seeds,
            f13,
            p(seeds.see["see_q"], np.int32),
            p(seeds.hit_offsets, np.uint32),
            p(seeds.hit_idx, np.int32),
            seeds.n_ph2,
            p(seeds.ph2_detId, np.uint32),
            p(seeds.ph2_x, np.float32),
            p(seeds.ph2_y, np.float32),
            p(seeds.ph2_z, np.float32),
        ]

    def _lst_arrays(self, handle, names):
        out = {}
        for name in names:
            n, sz = ctypes.c_longlong(), ctypes.c_int()
            ptr = self.lib.lstref_lst_array(handle, name.encode(), ctypes.byref(n), ctypes.byref(sz))
            dt = _LST_ARRAY_DTYPES[name]
            if not ptr or n.value == 0:
                out[name] = np.zeros(0, dt)
                continue
            buf = (ctypes.c_char * (n.value * sz.value)).from_address(ptr)
            out[name] = np.frombuffer(buf, dtype=dt, count=n.value).copy()
        return out

    def prepare_input(self, seeds) -> dict:
        """LST::prepareInput (SDL/LST.cc:175-365) on CMSSW-layout seeds; returns
        its 23 ``in_*_`` vectors by member name."""
        keep = []
        h = self.lib.lstref_lst_create()
        try:
            self.lib.lstref_lst_prepare(h, *self._seed_args(seeds, keep))
            return self._lst_arrays(h, [k for k in _LST_ARRAY_DTYPES if k.startswith("in_")])
        finally:
            self.lib.lstref_lst_destroy(h)

    def run_lst(self, seeds) -> dict:
        """LST::run (SDL/LST.cc:12-161) then its output accessors: returns
        ``hits`` (all candidates' hit indices concatenated), ``len``,
        ``seedIdx`` and ``trackCandidateType``."""
        keep = []
        h = self.lib.lstref_lst_create()
        try:
            self.lib.lstref_lst_run(h, self.es, *self._seed_args(seeds, keep))
            a = self._lst_arrays(h, [k for k in _LST_ARRAY_DTYPES if k.startswith("out_")])
        finally:
            self.lib.lstref_lst_destroy(h)
        return {
            "hits": a["out_tc_hitIdxs_"],
            "len": a["out_tc_len_"],
            "seedIdx": a["out_tc_seedIdx_"],
            "trackCandidateType": a["out_tc_trackCandidateType_"],
        }


def prepared_event_input(prep: dict):
    """The outputs of LST::prepareInput (RefLST.prepare_input) as an
    EventInput, i.e. the arguments LST::run passes to addHitToEvent and
    addPixelSegmentToEvent (SDL/LST.cc:53-72)."""
    from tracklooper_b200.gen import EventInput

    names = {
        "hitIndices0": "in_hitIndices_vec0_", "hitIndices1": "in_hitIndices_vec1_",
        "hitIndices2": "in_hitIndices_vec2_", "hitIndices3": "in_hitIndices_vec3_",
        "dPhiChange": "in_deltaPhi_vec_", "ptIn": "in_ptIn_vec_", "ptErr": "in_ptErr_vec_", "px": "in_px_vec_",
        "py": "in_py_vec_", "pz": "in_pz_vec_", "eta": "in_eta_vec_", "etaErr": "in_etaErr_vec_",
        "phi": "in_phi_vec_", "charge": "in_charge_vec_", "seedIdx": "in_seedIdx_vec_",
        "superbin": "in_superbin_vec_", "pixelType": "in_pixelType_vec_", "isQuad": "in_isQuad_vec_",
    }
    pls = {k: prep[v] for k, v in names.items()}
    n = prep["in_trkX_"].size
    return EventInput(prep["in_trkX_"], prep["in_trkY_"], prep["in_trkZ_"], prep["in_hitId_"], prep["in_hitIdxs_"],
                      pls, np.full(n, -1, np.int32), np.full(pls["ptIn"].size, -1, np.int32),
                      int(np.sum(prep["in_hitId_"] != 1)), np.zeros((0, 7)))


_LST_ARRAY_DTYPES = {
    "in_trkX_": np.float32,
    "in_trkY_": np.float32,
    "in_trkZ_": np.float32,
    "in_hitId_": np.uint32,
    "in_hitIdxs_": np.uint32,
    "in_hitIndices_vec0_": np.uint32,
    "in_hitIndices_vec1_": np.uint32,
    "in_hitIndices_vec2_": np.uint32,
    "in_hitIndices_vec3_": np.uint32,
    "in_deltaPhi_vec_": np.float32,
    "in_ptIn_vec_": np.float32,
    "in_ptErr_vec_": np.float32,
    "in_px_vec_": np.float32,
    "in_py_vec_": np.float32,
    "in_pz_vec_": np.float32,
    "in_eta_vec_": np.float32,
    "in_etaErr_vec_": np.float32,
    "in_phi_vec_": np.float32,
    "in_charge_vec_": np.int32,
    "in_seedIdx_vec_": np.uint32,
    "in_superbin_vec_": np.int32,
    "in_pixelType_vec_": np.int8,
    "in_isQuad_vec_": np.int8,
    "out_tc_len_": np.uint32,
    "out_tc_seedIdx_": np.int32,
    "out_tc_trackCandidateType_": np.int16,
    "out_tc_hitIdxs_": np.uint32,
}
