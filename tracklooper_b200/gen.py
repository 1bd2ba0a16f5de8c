"""Seeded synthetic LST events (host-side inputs of SDL::Event).

``generate_event(config, index)`` returns an :class:`EventInput` holding exactly
what ``Event.addHitToEvent`` and ``Event.addPixelSegmentToEvent`` take
(SDL/Event.h:113-137), plus per-hit and per-pLS simulation truth.  The physics
model and its assumptions are documented in ``csrc/gen/lstgen.cc``.

Seeds follow ``seed = (config << 32) | event_index`` so every configuration has
its own reproducible event stream.

Configurations:
  1  single muon (pT U(0.5, 50) GeV, |eta| < 2.4)
  2  PU200-shaped: ~20 hard tracks + Poisson(200) vertices x Poisson(60) particles
  3  as 2 with the per-event pileup mean drawn U(140, 250)
  5  PU250 with 5% displaced production vertices (r ~ U(0, 10) cm)
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import threading

import numpy as np

from . import geometry

_LIB = None
_GEN = None
_lock = threading.Lock()

PLS_FIELDS = (
    ("hitIndices0", np.uint32),
    ("hitIndices1", np.uint32),
    ("hitIndices2", np.uint32),
    ("hitIndices3", np.uint32),
    ("dPhiChange", np.float32),
    ("ptIn", np.float32),
    ("ptErr", np.float32),
    ("px", np.float32),
    ("py", np.float32),
    ("pz", np.float32),
    ("eta", np.float32),
    ("etaErr", np.float32),
    ("phi", np.float32),
    ("charge", np.int32),
    ("seedIdx", np.uint32),
    ("superbin", np.int32),
    ("pixelType", np.int8),
    ("isQuad", np.int8),
)


# The float inputs of LST::run (SDL/LST.h:32-45), in argument order.
SEED_FLOAT_FIELDS = (
    "see_px",
    "see_py",
    "see_pz",
    "see_dxy",
    "see_dz",
    "see_ptErr",
    "see_etaErr",
    "see_stateTrajGlbX",
    "see_stateTrajGlbY",
    "see_stateTrajGlbZ",
    "see_stateTrajGlbPx",
    "see_stateTrajGlbPy",
    "see_stateTrajGlbPz",
)


@dataclasses.dataclass
class SeedInput:
    """One event's inputs in the CMSSW layout of LST::run (SDL/LST.h:32-52).

    ``see`` maps the 13 float seed arrays plus ``see_q`` to numpy arrays;
    ``see_hitIdx`` (a vector<vector<int>> in the reference) is stored flat,
    seed i owning ``hit_idx[hit_offsets[i]:hit_offsets[i + 1]]``.  ``ph2_*``
    are the outer-tracker hits.
    """

    see: dict
    hit_offsets: np.ndarray
    hit_idx: np.ndarray
    ph2_detId: np.ndarray
    ph2_x: np.ndarray
    ph2_y: np.ndarray
    ph2_z: np.ndarray
    seed_sim: np.ndarray | None = None

    @property
    def n_seeds(self) -> int:
        return int(self.see["see_q"].shape[0])

    @property
    def n_ph2(self) -> int:
        return int(self.ph2_x.shape[0])

    def hit_lists(self) -> list:
        """see_hitIdx as a list of per-seed lists."""
        o = self.hit_offsets
        return [self.hit_idx[o[i]:o[i + 1]].tolist() for i in range(self.n_seeds)]


@dataclasses.dataclass
class EventInput:
    """One event's inputs in the reference's Event-API layout."""

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    detId: np.ndarray
    idxInNtuple: np.ndarray
    pls: dict
    hit_sim: np.ndarray
    pls_sim: np.ndarray
    n_ot_hits: int
    particles: np.ndarray  # (n, 7): pt, eta, phi, q, vx, vy, vz
    seeds: SeedInput | None = None  # the same event before seed conversion

    @property
    def n_hits(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_pls(self) -> int:
        return int(self.pls["ptIn"].shape[0])


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(os.path.dirname(__file__), "_lstgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"generator library not built: {path} (run __graft_entry__.build())")
        lib = ctypes.CDLL(path)
        lib.lstgen_create.restype = ctypes.c_void_p
        lib.lstgen_create.argtypes = [ctypes.c_char_p]
        lib.lstgen_event.restype = ctypes.c_void_p
        lib.lstgen_event.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_double]
        lib.lstgen_event_free.argtypes = [ctypes.c_void_p]
        lib.lstgen_event_sizes.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_uint)] * 4
        lib.lstgen_event_hits.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6
        lib.lstgen_event_pls.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 19
        lib.lstgen_event_particles.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.lstgen_event_seed_sizes.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_uint)] * 2
        lib.lstgen_event_seeds.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)] + [ctypes.c_void_p] * 4
        _LIB = lib
    return _LIB


def _generator():
    global _GEN
    with _lock:
        if _GEN is None:
            g = _lib().lstgen_create(geometry.geometry_dir().encode())
            if not g:
                raise RuntimeError("failed to load the geometry for the event generator")
            _GEN = g
    return _GEN


def event_seed(config: int, index: int) -> int:
    return (int(config) << 32) | int(index)


def generate_event(config: int, index: int, pileup: float = 0.0) -> EventInput:
    """Generates event ``index`` of configuration ``config`` (1, 2, 3 or 5)."""
    lib = _lib()
    h = lib.lstgen_event(_generator(), int(config), event_seed(config, index), float(pileup))
    try:
        sizes = [ctypes.c_uint() for _ in range(4)]
        lib.lstgen_event_sizes(h, *[ctypes.byref(s) for s in sizes])
        n_hits, n_ot, n_pls, n_part = (s.value for s in sizes)
        x = np.empty(n_hits, np.float32)
        y = np.empty(n_hits, np.float32)
        z = np.empty(n_hits, np.float32)
        det = np.empty(n_hits, np.uint32)
        idx = np.empty(n_hits, np.uint32)
        sim = np.empty(n_hits, np.int32)
        lib.lstgen_event_hits(h, *[a.ctypes.data for a in (x, y, z, det, idx, sim)])
        pls = {name: np.empty(n_pls, dt) for name, dt in PLS_FIELDS}
        pls_sim = np.empty(n_pls, np.int32)
        lib.lstgen_event_pls(h, *[pls[name].ctypes.data for name, _ in PLS_FIELDS], pls_sim.ctypes.data)
        parts = np.empty((n_part, 7), np.float64)
        lib.lstgen_event_particles(h, parts.ctypes.data)
        ns, nsh = ctypes.c_uint(), ctypes.c_uint()
        lib.lstgen_event_seed_sizes(h, ctypes.byref(ns), ctypes.byref(nsh))
        see = {name: np.empty(ns.value, np.float32) for name in SEED_FLOAT_FIELDS}
        see["see_q"] = np.empty(ns.value, np.int32)
        hit_off = np.empty(ns.value + 1, np.uint32)
        hit_idx = np.empty(nsh.value, np.int32)
        seed_sim = np.empty(ns.value, np.int32)
        f13 = (ctypes.c_void_p * 13)(*[see[name].ctypes.data for name in SEED_FLOAT_FIELDS])
        lib.lstgen_event_seeds(h, f13, see["see_q"].ctypes.data, hit_off.ctypes.data, hit_idx.ctypes.data,
                               seed_sim.ctypes.data)
    finally:
        lib.lstgen_event_free(h)
    seeds = SeedInput(see, hit_off, hit_idx, det[:n_ot].copy(), x[:n_ot].copy(), y[:n_ot].copy(), z[:n_ot].copy(),
                      seed_sim)
    return EventInput(x, y, z, det, idx, pls, sim, pls_sim, n_ot, parts, seeds)
